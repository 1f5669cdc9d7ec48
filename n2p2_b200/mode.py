"""Python mirror of nnp::Mode / nnp::Prediction over the C ABI.

Method names and argument meanings follow the reference (src/libnnp/Mode.h,
Prediction.h); errors surface as the exception classes of `_lib` that stand
for the reference's std::runtime_error / std::out_of_range /
std::invalid_argument.  All evaluation runs in libn2p2b200.so on the GPU.
"""
import ctypes
import os

import numpy as np

from . import _lib
from .structure import Structure, read_structures

_P = ctypes.POINTER


def _dp(a):
    return a.ctypes.data_as(_P(ctypes.c_double))


class Mode:
    """nnp::Mode: model set-up plus evaluation of structures on one GPU."""

    def __init__(self, device=0):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._lib.n2p2_mode_create(ctypes.byref(h), int(device)))
        self._h = h
        self._batches = []

    def close(self):
        for b in self._batches:
            b.close()
        self._batches = []
        if getattr(self, "_h", None):
            self._lib.n2p2_mode_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up (Mode.cpp:56-1547) ---------------------------------------
    def initialize(self):
        _lib.check(self._lib.n2p2_mode_initialize(self._h))

    def loadSettingsFile(self, fileName="input.nn"):
        _lib.check(self._lib.n2p2_mode_load_settings_file(self._h, str(fileName).encode()))

    def setupGeneric(self, nnpDir=""):
        _lib.check(self._lib.n2p2_mode_setup_generic(self._h))

    def setupSymmetryFunctionScaling(self, fileName="scaling.data"):
        _lib.check(self._lib.n2p2_mode_setup_symmetry_function_scaling(self._h, str(fileName).encode()))

    def setupSymmetryFunctionScalingNone(self):
        _lib.check(self._lib.n2p2_mode_setup_symmetry_function_scaling_none(self._h))

    def setupNeuralNetworkWeights(self, fileNameFormat="weights.%03zu.data"):
        _lib.check(self._lib.n2p2_mode_setup_neural_network_weights(self._h, str(fileNameFormat).encode()))

    def setConnections(self, element, connections):
        c = np.ascontiguousarray(connections, dtype=np.float64)
        _lib.check(self._lib.n2p2_mode_set_connections(self._h, int(element), _dp(c), c.size))

    def setupSymmetryFunctionStatistics(self, collectStatistics=False, collectExtrapolationWarnings=False,
                                        writeExtrapolationWarnings=False, stopOnExtrapolationWarnings=False):
        _lib.check(self._lib.n2p2_mode_setup_symmetry_function_statistics(
            self._h, int(collectStatistics), int(collectExtrapolationWarnings), int(writeExtrapolationWarnings),
            int(stopOnExtrapolationWarnings)))

    def setPrecision(self, precision):
        p = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}.get(precision, precision)
        _lib.check(self._lib.n2p2_mode_set_precision(self._h, int(p)))

    def setAutotune(self, enabled=True):
        """Automatic choice of the symmetry-function kernel shapes (default on)."""
        _lib.check(self._lib.n2p2_mode_set_autotune(self._h, int(bool(enabled))))

    def setupFromDirectory(self, d, fp=None):
        """Prediction::setup sequence on a model directory."""
        self.initialize()
        self.loadSettingsFile(os.path.join(d, "input.nn"))
        self.setupGeneric()
        self.setupSymmetryFunctionScaling(os.path.join(d, "scaling.data"))
        self.setupNeuralNetworkWeights(os.path.join(d, "weights.%03zu.data"))
        return self

    # -- queries -----------------------------------------------------------
    def getMaxCutoffRadius(self):
        r = ctypes.c_double()
        _lib.check(self._lib.n2p2_mode_get_max_cutoff_radius(self._h, ctypes.byref(r)))
        return r.value

    @property
    def numElements(self):
        n = ctypes.c_int()
        _lib.check(self._lib.n2p2_mode_get_num_elements(self._h, ctypes.byref(n)))
        return n.value

    def elementSymbol(self, e):
        buf = ctypes.create_string_buffer(8)
        _lib.check(self._lib.n2p2_mode_get_element_symbol(self._h, int(e), buf, 8))
        return buf.value.decode()

    def elementIndex(self, symbol):
        e = ctypes.c_int()
        _lib.check(self._lib.n2p2_mode_get_element_index(self._h, symbol.encode(), ctypes.byref(e)))
        return e.value

    def numSymmetryFunctions(self, e):
        n = ctypes.c_int()
        _lib.check(self._lib.n2p2_mode_get_num_symmetry_functions(self._h, int(e), ctypes.byref(n)))
        return n.value

    def symmetryFunction(self, e, i):
        """(type, e1, e2, eta, rs, lambda, zeta, rc, scalingFactor) of SF i of element e."""
        t, a, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        p = np.zeros(6)
        _lib.check(self._lib.n2p2_mode_get_symmetry_function(self._h, int(e), int(i), ctypes.byref(t), ctypes.byref(a),
                                                             ctypes.byref(b), _dp(p)))
        return (t.value, a.value, b.value, *p.tolist())

    def networkTopology(self, e):
        """(neurons per layer, activation per layer) of element e's network,
        input and output layers included."""
        n = ctypes.c_int()
        _lib.check(self._lib.n2p2_mode_get_network_topology(self._h, int(e), 0, ctypes.byref(n), None, None))
        neurons = (ctypes.c_int * n.value)()
        act = (ctypes.c_int * n.value)()
        _lib.check(self._lib.n2p2_mode_get_network_topology(self._h, int(e), n.value, ctypes.byref(n), neurons, act))
        return list(neurons), list(act)

    def numDerivativeRows(self, e, en):
        n = ctypes.c_int()
        _lib.check(self._lib.n2p2_mode_get_num_derivative_rows(self._h, int(e), int(en), ctypes.byref(n)))
        return n.value

    # -- evaluation --------------------------------------------------------
    def batch(self, structures, remap=True):
        b = Batch(self)
        b.setStructures(structures, remap=remap)
        self._batches.append(b)
        return b

    def evaluateNNP(self, structures, useForces=True, storeDGdr=False):
        """Mode::evaluateNNP on each structure; fills .energy and .forces."""
        single = isinstance(structures, Structure)
        ss = [structures] if single else list(structures)
        b = self.batch(ss)
        b.setPositions(np.concatenate([s.positions for s in ss]))
        b.evaluate(forces=useForces, storeDGdr=storeDGdr)
        e = b.energies()
        f = b.forces() if useForces else None
        a0 = 0
        for k, s in enumerate(ss):
            s.energy = float(e[k])
            if f is not None:
                s.forces = f[a0:a0 + s.numAtoms].copy()
            a0 += s.numAtoms
        return b


class Batch:
    """Structures resident on the GPU (one n2p2_batch)."""

    def __init__(self, mode):
        self._mode = mode
        self._lib = mode._lib
        h = ctypes.c_void_p()
        _lib.check(self._lib.n2p2_batch_create(mode._h, ctypes.byref(h)))
        self._h = h
        self.numStructures = 0
        self.numAtoms = 0
        self.elements = None
        self.atomsPerStructure = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.n2p2_batch_destroy(self._h)
            self._h = None

    def setStructures(self, structures, remap=True):
        m = self._mode
        ss = list(structures)
        na = np.array([s.numAtoms for s in ss], dtype=np.int64)
        sym = {}
        el = np.array([sym.setdefault(x, m.elementIndex(x)) if x not in sym else sym[x]
                       for s in ss for x in s.elements], dtype=np.int32)
        boxes = np.zeros((len(ss), 3, 3))
        per = np.zeros(len(ss), dtype=np.int32)
        for k, s in enumerate(ss):
            if s.box is not None:
                boxes[k] = s.box
                per[k] = 1
        self.setArrays(na, el, boxes, per, remap)
        return self

    def setArrays(self, numAtoms, elements, boxes, periodic, remap=True):
        na = np.ascontiguousarray(numAtoms, dtype=np.int64)
        el = np.ascontiguousarray(elements, dtype=np.int32)
        bx = np.ascontiguousarray(boxes, dtype=np.float64)
        pe = np.ascontiguousarray(periodic, dtype=np.int32)
        _lib.check(self._lib.n2p2_batch_set_structures(
            self._h, na.size, na.ctypes.data_as(_P(ctypes.c_int64)), el.ctypes.data_as(_P(ctypes.c_int32)),
            _dp(bx), pe.ctypes.data_as(_P(ctypes.c_int32)), int(bool(remap))))
        self.numStructures = int(na.size)
        self.numAtoms = int(na.sum())
        self.elements = el.copy()
        self.atomsPerStructure = na.copy()
        return self

    def setPositions(self, positions):
        """Host positions [N,3] (physical units), or a device pointer (int)."""
        if isinstance(positions, int):
            _lib.check(self._lib.n2p2_batch_set_positions(self._h, ctypes.c_void_p(positions), 1))
            return
        p = np.ascontiguousarray(positions, dtype=np.float64)
        self._pos_keepalive = p
        _lib.check(self._lib.n2p2_batch_set_positions(self._h, p.ctypes.data_as(ctypes.c_void_p), 0))
        # the copy is asynchronous; keep the buffer alive until the next sync
        _lib.check(self._lib.n2p2_batch_synchronize(self._h))

    def evaluate(self, forces=True, storeDGdr=False, graph=True, symmetryFunctionsOnly=False):
        flags = (_lib.EVAL_FORCES if forces else 0) | (_lib.EVAL_STORE_DGDR if storeDGdr else 0) | \
            (0 if graph else _lib.EVAL_NO_GRAPH) | (_lib.EVAL_SF_ONLY if symmetryFunctionsOnly else 0)
        _lib.check(self._lib.n2p2_batch_evaluate(self._h, flags))

    # -- the stages of Mode::evaluateNNP as separate calls (Mode.h:298-378) --
    def calculateNeighborList(self):
        """Structure::calculateNeighborList(maxCutoffRadius, false) on every structure."""
        _lib.check(self._lib.n2p2_batch_calculate_neighbor_list(self._h))

    def calculateSymmetryFunctionGroups(self, derivatives):
        """Mode::calculateSymmetryFunctionGroups: derivatives False/True, or
        "stored" for Atom::dGdr / Atom::Neighbor::dGdr (FP64)."""
        d = _lib.DERIVATIVES_STORED if derivatives == "stored" else (1 if derivatives else 0)
        _lib.check(self._lib.n2p2_batch_calculate_symmetry_function_groups(self._h, d))

    def calculateSymmetryFunctions(self, derivatives):
        """Mode::calculateSymmetryFunctions (the same values as the groups form)."""
        d = _lib.DERIVATIVES_STORED if derivatives == "stored" else (1 if derivatives else 0)
        _lib.check(self._lib.n2p2_batch_calculate_symmetry_functions(self._h, d))

    def calculateAtomicNeuralNetworks(self, derivatives):
        _lib.check(self._lib.n2p2_batch_calculate_atomic_neural_networks(self._h, int(bool(derivatives))))

    def calculateEnergy(self):
        _lib.check(self._lib.n2p2_batch_calculate_energy(self._h))

    def calculateForces(self):
        _lib.check(self._lib.n2p2_batch_calculate_forces(self._h))

    def symmetryFunctionStatistics(self):
        """Per element: dict(count, min, max, sum, sum2) of the unscaled G of
        the last evaluation (n2p2_batch_get_symmetry_function_statistics)."""
        m = self._mode
        ne = m.numElements
        nsf = [m.numSymmetryFunctions(e) for e in range(ne)]
        counts = np.zeros(ne, dtype=np.int64)
        stats = np.zeros(4 * sum(nsf))
        _lib.check(self._lib.n2p2_batch_get_symmetry_function_statistics(
            self._h, counts.ctypes.data_as(_P(ctypes.c_int64)), _dp(stats)))
        out, at = [], 0
        for e in range(ne):
            block = stats[at:at + 4 * nsf[e]].reshape(4, nsf[e])
            at += 4 * nsf[e]
            out.append({"count": int(counts[e]), "min": block[0].copy(), "max": block[1].copy(),
                        "sum": block[2].copy(), "sum2": block[3].copy()})
        return out

    def synchronize(self):
        _lib.check(self._lib.n2p2_batch_synchronize(self._h))

    def evaluateHost(self, positions, energies, forces, useForces=True):
        flags = _lib.EVAL_FORCES if useForces else 0
        _lib.check(self._lib.n2p2_batch_evaluate_host(
            self._h, positions.ctypes.data_as(ctypes.c_void_p), energies.ctypes.data_as(ctypes.c_void_p),
            forces.ctypes.data_as(ctypes.c_void_p) if forces is not None else None, flags))

    def energies(self):
        out = np.zeros(self.numStructures)
        _lib.check(self._lib.n2p2_batch_get_energies(self._h, _dp(out)))
        return out

    def forces(self):
        out = np.zeros((self.numAtoms, 3))
        _lib.check(self._lib.n2p2_batch_get_forces(self._h, _dp(out)))
        return out

    def neighborCapacity(self):
        """(entries the neighbour buffers hold, evaluations repeated because
        new positions outgrew them)."""
        c, r = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(self._lib.n2p2_batch_get_neighbor_capacity(self._h, ctypes.byref(c), ctypes.byref(r)))
        return c.value, r.value

    def numNeighborEntries(self):
        n = ctypes.c_int64()
        _lib.check(self._lib.n2p2_batch_get_num_neighbor_entries(self._h, ctypes.byref(n)))
        return n.value

    def neighbors(self):
        M = self.numNeighborEntries()
        off = np.zeros(self.numAtoms + 1, dtype=np.int64)
        idx = np.zeros(M, dtype=np.int32)
        img = np.zeros(M, dtype=np.int32)
        d = np.zeros(M)
        dr = np.zeros((M, 3))
        _lib.check(self._lib.n2p2_batch_get_neighbors(
            self._h, off.ctypes.data_as(_P(ctypes.c_int64)), idx.ctypes.data_as(_P(ctypes.c_int32)),
            img.ctypes.data_as(_P(ctypes.c_int32)), _dp(d), _dp(dr)))
        return {"offset": off, "index": idx, "image": img, "d": d, "dr": dr}

    def _per_sf(self):
        m = self._mode
        nsf = np.array([m.numSymmetryFunctions(e) for e in range(m.numElements)])
        return int(nsf[self.elements].sum())

    def symmetryFunctions(self):
        out = np.zeros(self._per_sf())
        _lib.check(self._lib.n2p2_batch_get_symmetry_functions(self._h, _dp(out)))
        return out

    def dEdG(self):
        out = np.zeros(self._per_sf())
        _lib.check(self._lib.n2p2_batch_get_dEdG(self._h, _dp(out)))
        return out

    def atomicEnergies(self):
        out = np.zeros(self.numAtoms)
        _lib.check(self._lib.n2p2_batch_get_atomic_energies(self._h, _dp(out)))
        return out

    def dGdr(self, nbr_rows_total):
        selfd = np.zeros((self._per_sf(), 3))
        nbr = np.zeros((nbr_rows_total, 3))
        _lib.check(self._lib.n2p2_batch_get_dGdr(self._h, _dp(selfd), _dp(nbr)))
        return selfd, nbr

    def internalPositions(self):
        out = np.zeros((self.numAtoms, 3))
        _lib.check(self._lib.n2p2_batch_get_internal_positions(self._h, _dp(out)))
        return out

    def extrapolationWarnings(self):
        t = ctypes.c_int64()
        per = np.zeros(self.numAtoms, dtype=np.int32)
        _lib.check(self._lib.n2p2_batch_get_extrapolation_warnings(self._h, ctypes.byref(t),
                                                                   per.ctypes.data_as(_P(ctypes.c_int32))))
        return t.value, per

    SHAPES = ((128, 4), (160, 4), (192, 2))   # (stage capacity, warps per block) per shape index

    def autotune(self, useCache=True):
        """Times the three kernel shapes of both symmetry-function passes (the
        batch must have been evaluated once) and keeps the fastest."""
        sh = np.zeros(2, dtype=np.int32)
        ms = np.zeros(6)
        fc = ctypes.c_int32()
        _lib.check(self._lib.n2p2_batch_autotune(self._h, int(bool(useCache)), sh.ctypes.data_as(_P(ctypes.c_int32)),
                                                 _dp(ms), ctypes.byref(fc)))
        return {"values": int(sh[0]), "forces": int(sh[1]), "values_ms": ms[:3].tolist(),
                "forces_ms": ms[3:].tolist(), "from_cache": bool(fc.value)}

    def setShapes(self, values, forces):
        _lib.check(self._lib.n2p2_batch_set_shapes(self._h, int(values), int(forces)))

    def stream(self):
        s = ctypes.c_void_p()
        _lib.check(self._lib.n2p2_batch_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def profileStages(self, forces=True, storeDGdr=False):
        flags = (_lib.EVAL_FORCES if forces else 0) | (_lib.EVAL_STORE_DGDR if storeDGdr else 0)
        cap = 32
        names = ctypes.create_string_buffer(32 * cap)
        ms = np.zeros(cap)
        n = ctypes.c_int()
        _lib.check(self._lib.n2p2_batch_profile_stages(self._h, flags, cap, names, _dp(ms), ctypes.byref(n)))
        raw = names.raw
        return [(raw[32 * k:32 * k + 32].split(b"\0")[0].decode(), float(ms[k])) for k in range(n.value)]

    def countWork(self):
        c = np.zeros(10, dtype=np.int64)
        _lib.check(self._lib.n2p2_batch_count_work(self._h, c.ctypes.data_as(_P(ctypes.c_int64))))
        keys = ["entries", "radial_terms", "radial_pairs", "narrow_triplets", "narrow_terms", "wide_pairs",
                "wide_terms", "g_values", "atoms", "derivative_rows"]
        return dict(zip(keys, (int(x) for x in c)))

    def launchCount(self):
        n = ctypes.c_int()
        _lib.check(self._lib.n2p2_batch_get_launch_count(self._h, ctypes.byref(n)))
        return n.value


class Trainer:
    """Device training of a mode's networks on energies and forces (the
    distilled-student path; the reference's CPU counterpart is nnp::Training).
    Parameters are exchanged in weight-file order, element by element."""

    def __init__(self, mode, eta=1e-3, beta1=0.9, beta2=0.999, epsilon=1e-8, energyWeight=1.0, forceWeight=10.0):
        self._mode = mode
        self._lib = mode._lib
        h = ctypes.c_void_p()
        _lib.check(self._lib.n2p2_trainer_create(mode._h, ctypes.byref(h)))
        self._h = h
        _lib.check(self._lib.n2p2_trainer_set_adam(self._h, eta, beta1, beta2, epsilon))
        _lib.check(self._lib.n2p2_trainer_set_loss_weights(self._h, energyWeight, forceWeight))
        n = ctypes.c_int64()
        _lib.check(self._lib.n2p2_trainer_get_num_parameters(self._h, ctypes.byref(n)))
        self.numParameters = n.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.n2p2_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setLearningRate(self, eta):
        _lib.check(self._lib.n2p2_trainer_set_learning_rate(self._h, float(eta)))

    def parameters(self):
        out = np.zeros(self.numParameters)
        _lib.check(self._lib.n2p2_trainer_get_parameters(self._h, _dp(out)))
        return out

    def setParameters(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        if w.size != self.numParameters:
            raise ValueError("expected %d parameters" % self.numParameters)
        _lib.check(self._lib.n2p2_trainer_set_parameters(self._h, _dp(w)))

    def step(self, batch, energies, forces, update=True, gradient=False):
        """Loss (total, energy term, force term) of `batch` against physical-unit
        labels; an Adam step if `update`; the gradient too if `gradient`."""
        e = np.ascontiguousarray(energies, dtype=np.float64)
        f = np.ascontiguousarray(forces, dtype=np.float64)
        if e.size != batch.numStructures or f.size != 3 * batch.numAtoms:
            raise ValueError("labels do not match the batch")
        loss = np.zeros(3)
        g = np.zeros(self.numParameters) if gradient else None
        _lib.check(self._lib.n2p2_trainer_step(self._h, batch._h, _dp(e), _dp(f), int(bool(update)), _dp(loss),
                                               _dp(g) if g is not None else None))
        return (loss, g) if gradient else loss


class Prediction(Mode):
    """nnp::Prediction (Prediction.cpp:27-78): a Mode plus one Structure."""

    def __init__(self, directory=".", device=0):
        super().__init__(device)
        self.directory = directory
        self.fileNameSettings = os.path.join(directory, "input.nn")
        self.fileNameScaling = os.path.join(directory, "scaling.data")
        self.formatWeightsFilesShort = os.path.join(directory, "weights.%03zu.data")
        self.structure = None

    def setup(self):
        self.initialize()
        self.loadSettingsFile(self.fileNameSettings)
        self.setupGeneric()
        self.setupSymmetryFunctionScaling(self.fileNameScaling)
        self.setupNeuralNetworkWeights(self.formatWeightsFilesShort)
        self.setupSymmetryFunctionStatistics(False, False, True, False)

    def readStructureFromFile(self, fileName=None):
        fn = fileName or os.path.join(self.directory, "input.data")
        self.structure = read_structures(fn, limit=1)[0]

    def predict(self):
        self.evaluateNNP(self.structure, useForces=True)
        return self.structure
