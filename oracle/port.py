"""Python set-up + ctypes driver of the C restatement in nnp_oracle.c.

TEST INFRASTRUCTURE ONLY (the checker and the "port" CPU baseline); the
product never imports this module.

The set-up restates Mode's (reference src/libnnp/Mode.cpp:162-1547): input.nn
keywords, element map sorted by atomic number (ElementMap.cpp:36-54),
symmetry functions of types 2/3/9 in the order of SymFnc*::operator<
(SymFncExpRad.cpp:55-75, SymFncExpAngn.cpp:51-77), derivative-row tables
(Element.cpp:289-311), scaling (SymFnc.cpp:52-98, Mode.cpp:781-909), the
network topology (Mode.cpp:1227-1512) and the weights files in
NeuralNetwork::setConnections order (NeuralNetwork.cpp:147-169).
"""
import ctypes
import functools
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libnnpport.so")

Z = {s: i + 1 for i, s in enumerate(
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
    "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No".split())}
ACT = {"l": 1, "t": 2, "s": 3, "p": 4, "r": 5, "g": 6, "c": 7, "S": 8, "e": 9, "h": 10}


def available():
    return os.path.exists(LIB)


def parse_settings(text):
    kv = []
    for i, line in enumerate(text.splitlines()):
        for c in "#!":
            if c in line:
                line = line[:line.index(c)]
        w = line.split()
        if w:
            kv.append((w[0], " ".join(w[1:]), i))
    return kv


class _Model(ctypes.Structure):
    _fields_ = [("numElements", ctypes.c_int), ("maxCutoff", ctypes.c_double), ("cutoffType", ctypes.c_int),
                ("cutoffAlpha", ctypes.c_double), ("totalSF", ctypes.c_int)] + \
        [(n, ctypes.c_void_p) for n in ("sfBegin", "type", "e1", "e2", "eta", "rs", "lambda_", "zeta", "rc", "row",
                                        "numRows", "rowSF")] + \
        [("maxRows", ctypes.c_int)] + \
        [(n, ctypes.c_void_p) for n in ("scalingType", "Smin", "Gmin", "Gmax", "Gmean", "scalingFactor", "numLayers",
                                        "neurons", "activation", "wBegin", "bBegin", "weights")] + \
        [("normalizeNeurons", ctypes.c_int), ("normalize", ctypes.c_int), ("meanEnergy", ctypes.c_double),
         ("convEnergy", ctypes.c_double), ("convLength", ctypes.c_double), ("atomicEnergyOffset", ctypes.c_void_p)]


class _Result(ctypes.Structure):
    _fields_ = [("numAtoms", ctypes.c_int), ("energy", ctypes.c_double), ("energyInternal", ctypes.c_double)] + \
        [(n, ctypes.c_void_p) for n in ("forces", "positions", "nbrOffset", "nbrIndex", "nbrD", "nbrDr", "sfOffset",
                                        "G", "dEdG", "atomicEnergy")] + [("warnings", ctypes.c_int64)]


@functools.lru_cache(None)
def _lib():
    lib = ctypes.CDLL(LIB)
    lib.oracle_evaluate.restype = ctypes.c_int
    lib.oracle_evaluate.argtypes = [ctypes.POINTER(_Model), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_Result)]
    lib.oracle_free_result.argtypes = [ctypes.POINTER(_Result)]
    return lib


class PortModel:
    """Set-up of one model directory (input.nn, scaling.data, weights.%03d.data)."""

    def __init__(self, model_dir):
        kv = parse_settings(open(os.path.join(model_dir, "input.nn")).read())
        first = {}
        for k, v, i in kv:
            first.setdefault(k, v)
        self.symbols = sorted(first["elements"].split(), key=lambda s: Z[s])
        ne = len(self.symbols)
        idx = {s: i for i, s in enumerate(self.symbols)}
        self.normalize = all(k in first for k in ("mean_energy", "conv_energy", "conv_length"))
        self.meanEnergy = float(first.get("mean_energy", 0.0))
        self.convEnergy = float(first.get("conv_energy", 1.0))
        self.convLength = float(first.get("conv_length", 1.0))
        ct = first["cutoff_type"].split()
        self.cutoffType = int(ct[0])
        self.cutoffAlpha = float(ct[1]) if len(ct) > 1 else 0.0
        offs = np.zeros(ne)
        for k, v, _ in kv:
            if k == "atom_energy":
                a = v.split()
                offs[idx[a[0]]] = float(a[1])
        self.atomicEnergyOffset = offs
        # symmetry functions
        per = [[] for _ in range(ne)]
        for k, v, line in kv:
            if k != "symfunction_short":
                continue
            a = v.split()
            t = int(a[1])
            sf = {"type": t, "ec": idx[a[0]], "line": line, "rs": 0.0, "zeta": 0.0, "lambda": 0.0}
            if t == 2:
                sf.update(e1=idx[a[2]], e2=idx[a[2]], eta=float(a[3]), rs=float(a[4]), rc=float(a[5]))
            elif t in (3, 9):
                e1, e2 = sorted((idx[a[2]], idx[a[3]]))
                sf.update(e1=e1, e2=e2, eta=float(a[4]), **{"lambda": float(a[5])}, zeta=float(a[6]), rc=float(a[7]))
                if len(a) > 8:
                    sf["rs"] = float(a[8])
            else:
                raise ValueError("symmetry function type %d not restated" % t)
            if self.normalize:
                sf["eta"] /= self.convLength * self.convLength
                sf["rc"] *= self.convLength
                sf["rs"] *= self.convLength
            per[sf["ec"]].append(sf)

        def key(s):
            k = (s["ec"], s["type"], s["rc"], s["eta"], s["rs"])
            if s["type"] != 2:
                k += (s["zeta"], s["lambda"])
            return k + (s["e1"],) + ((s["e2"],) if s["type"] != 2 else ())
        for e in range(ne):
            per[e].sort(key=key)
        self.sfs = per
        self.maxCutoff = max(s["rc"] for p in per for s in p)
        # derivative rows
        rows = np.zeros((ne, ne), dtype=np.int32)
        tables = [[[] for _ in range(ne)] for _ in range(ne)]
        rowidx = []
        for ec in range(ne):
            for i, s in enumerate(per[ec]):
                r = []
                for en in range(ne):
                    rel = (en == s["e1"]) if s["type"] == 2 else (en in (s["e1"], s["e2"]))
                    if rel:
                        r.append(len(tables[ec][en]))
                        tables[ec][en].append(i)
                    else:
                        r.append(-1)
                rowidx.append(r)
            for en in range(ne):
                rows[ec, en] = len(tables[ec][en])
        self.maxRows = int(rows.max())
        rowSF = np.zeros((ne, ne, max(self.maxRows, 1)), dtype=np.int32)
        for ec in range(ne):
            for en in range(ne):
                rowSF[ec, en, :len(tables[ec][en])] = tables[ec][en]
        # scaling
        sc = "scale_symmetry_functions" in first
        ce = "center_symmetry_functions" in first
        stype = 1 if sc and not ce else 2 if ce and not sc else 3 if sc and ce else \
            4 if "scale_symmetry_functions_sigma" in first else 0
        smin = float(first.get("scale_min_short", 0.0)) if stype in (1, 3, 4) else 0.0
        smax = float(first.get("scale_max_short", 1.0)) if stype in (1, 3, 4) else 0.0
        lines = [l for l in open(os.path.join(model_dir, "scaling.data")).read().splitlines()
                 if l and not l.startswith("#")]
        flat = [s for p in per for s in p]
        n = len(flat)
        st = np.array([[float(x) for x in l.split()[2:6]] for l in lines[:n]])
        gmin, gmax, gmean, gsig = st[:, 0], st[:, 1], st[:, 2], st[:, 3]
        if stype in (1, 3):
            sfac = (smax - smin) / (gmax - gmin)
        elif stype == 4:
            sfac = (smax - smin) / gsig
        else:
            sfac = np.ones(n)
        # networks
        hid = int(first["global_hidden_layers_short"])
        nodes = [int(x) for x in first["global_nodes_short"].split()]
        acts = first["global_activation_short"].split()
        L = hid + 2
        neurons = np.zeros((ne, 8), dtype=np.int32)
        act = np.zeros((ne, 8), dtype=np.int32)
        wb = np.zeros((ne, 8), dtype=np.int32)
        bb = np.zeros((ne, 8), dtype=np.int32)
        weights = []
        for e in range(ne):
            sizes = [len(per[e])] + nodes + [1]
            neurons[e, :L] = sizes
            act[e, 0] = 1
            for l in range(1, L):
                act[e, l] = ACT[acts[l - 1]]
            c = [float(l.split()[0]) for l in open(os.path.join(model_dir, "weights.%03d.data" % Z[self.symbols[e]]))
                 if l.strip() and not l.startswith("#")]
            q = 0
            for l in range(1, L):
                nin, nout = sizes[l - 1], sizes[l]
                W = np.zeros((nout, nin))
                for j in range(nin):
                    for k in range(nout):
                        W[k, j] = c[q]
                        q += 1
                b = np.array(c[q:q + nout])
                q += nout
                wb[e, l] = len(weights)
                weights.extend(W.ravel())
                bb[e, l] = len(weights)
                weights.extend(b)
        self.numLayers = np.full(ne, L, dtype=np.int32)
        self.arrays = dict(
            sfBegin=np.cumsum([0] + [len(p) for p in per]).astype(np.int32),
            type=np.array([s["type"] for s in flat], dtype=np.int32),
            e1=np.array([s["e1"] for s in flat], dtype=np.int32),
            e2=np.array([s["e2"] for s in flat], dtype=np.int32),
            eta=np.array([s["eta"] for s in flat]), rs=np.array([s["rs"] for s in flat]),
            lambda_=np.array([s["lambda"] for s in flat]), zeta=np.array([s["zeta"] for s in flat]),
            rc=np.array([s["rc"] for s in flat]), row=np.array(rowidx, dtype=np.int32).ravel(),
            numRows=rows.ravel().copy(), rowSF=rowSF.ravel().copy(),
            scalingType=np.full(n, stype, dtype=np.int32), Smin=np.full(n, smin), Gmin=gmin.copy(),
            Gmax=gmax.copy(), Gmean=gmean.copy(), scalingFactor=np.asarray(sfac, dtype=np.float64),
            numLayers=self.numLayers, neurons=neurons.ravel().copy(), activation=act.ravel().copy(),
            wBegin=wb.ravel().copy(), bBegin=bb.ravel().copy(), weights=np.array(weights),
            atomicEnergyOffset=offs)
        m = _Model()
        m.numElements = ne
        m.maxCutoff = self.maxCutoff
        m.cutoffType = self.cutoffType
        m.cutoffAlpha = self.cutoffAlpha
        m.totalSF = n
        m.maxRows = max(self.maxRows, 1)
        for k, v in self.arrays.items():
            setattr(m, k, v.ctypes.data)
        m.normalizeNeurons = int("normalize_nodes" in first)
        m.normalize = int(self.normalize)
        m.meanEnergy = self.meanEnergy
        m.convEnergy = self.convEnergy
        m.convLength = self.convLength
        self._m = m
        self.index = idx

    def evaluate(self, structure, use_forces=True):
        """Energy/forces (physical) and internal arrays of one Structure."""
        N = structure.numAtoms
        r = np.ascontiguousarray(structure.positions, dtype=np.float64)
        el = np.array([self.index[s] for s in structure.elements], dtype=np.int32)
        box = None if structure.box is None else np.ascontiguousarray(structure.box, dtype=np.float64)
        res = _Result()
        rc = _lib().oracle_evaluate(ctypes.byref(self._m), N, r.ctypes.data, el.ctypes.data,
                                    box.ctypes.data if box is not None else None, int(use_forces), ctypes.byref(res))
        if rc != 0:
            raise RuntimeError("oracle evaluation failed")

        def arr(ptr, n, dt):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(dt)), shape=(n,)).copy() if n else \
                np.zeros(0, dtype=np.float64 if dt is ctypes.c_double else np.int64)
        off = arr(res.nbrOffset, N + 1, ctypes.c_int64)
        M = int(off[-1])
        sfo = arr(res.sfOffset, N + 1, ctypes.c_int64)
        out = {"energy": res.energy, "energy_internal": res.energyInternal,
               "forces": arr(res.forces, 3 * N, ctypes.c_double).reshape(-1, 3),
               "positions": arr(res.positions, 3 * N, ctypes.c_double).reshape(-1, 3),
               "nbr_offset": off, "nbr_index": arr(res.nbrIndex, M, ctypes.c_int64),
               "nbr_d": arr(res.nbrD, M, ctypes.c_double), "nbr_dr": arr(res.nbrDr, 3 * M, ctypes.c_double).reshape(-1, 3),
               "sf_offset": sfo, "G": arr(res.G, int(sfo[-1]), ctypes.c_double),
               "dEdG": arr(res.dEdG, int(sfo[-1]), ctypes.c_double),
               "atomic_energy": arr(res.atomicEnergy, N, ctypes.c_double), "warnings": int(res.warnings)}
        _lib().oracle_free_result(ctypes.byref(res))
        return out
