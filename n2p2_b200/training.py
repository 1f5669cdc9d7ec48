"""The update loop of the reference's training program on the GPU.

Reference: src/libnnptrain/Training.cpp -- update (:2256-3169, 2G networks,
combined update strategy, one update candidate per update), loop and its
epoch schedule (:2086-2111, :2147-2230), shuffleUpdateCandidates
(:2062-2084); the updaters KalmanFilter (KalmanFilter.cpp:126-238) and
GradientDescent (GradientDescent.cpp:81-118).

The training set's symmetry functions and dG/dr are computed once on the
device; each update evaluates the networks and the Jacobian of one
observation (a structure's energy or one force component) over that
structure's atoms and applies the updater, with no host round trip inside a
run of updates of the same property.  The weights are the mode's device
weights: after training, every batch of the mode evaluates the trained
networks.
"""
import ctypes
import os

import numpy as np

from . import _lib
from .mode import _dp

ENERGY = _lib.TRAINING_ENERGY
FORCE = _lib.TRAINING_FORCE


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


class Training:
    """Training::update for a set of structures with reference energies
    (physical units, with atomic energy offsets) and forces [N][3]."""

    def __init__(self, mode, structures, energies, forces):
        self._mode = mode
        self._lib = mode._lib
        self.structures = list(structures)
        self.batch = mode.batch(self.structures)
        self.batch.setPositions(np.concatenate([s.positions for s in self.structures]))
        h = ctypes.c_void_p()
        _lib.check(self._lib.n2p2_training_create(self.batch._h, ctypes.byref(h)))
        self._h = h
        self.energiesRef = np.ascontiguousarray(energies, dtype=np.float64)
        self.forcesRef = np.ascontiguousarray(forces, dtype=np.float64).reshape(-1, 3)
        if self.energiesRef.size != len(self.structures) or self.forcesRef.shape[0] != self.batch.numAtoms:
            raise ValueError("references do not match the structures")
        _lib.check(self._lib.n2p2_training_set_references(self._h, _dp(self.energiesRef), _dp(self.forcesRef)))
        n = ctypes.c_int64()
        _lib.check(self._lib.n2p2_training_get_num_weights(self._h, ctypes.byref(n)))
        self.numWeights = n.value
        self.atomsPerStructure = np.array([s.numAtoms for s in self.structures], dtype=np.int64)
        self.forceWeight = 1.0
        self.taskBatch = {ENERGY: 1, FORCE: 1}
        self.epoch = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.n2p2_training_destroy(self._h)
            self._h = None
        if getattr(self, "batch", None) is not None:
            self.batch.close()
            self.batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- updaters (settings keywords of nnp-train) -------------------------
    def setupUpdaterKalman(self, kalman_type=0, epsilon=1e-2, q0=0.01, qtau=2.302, qmin=1e-6, eta=0.01,
                           etatau=2.302, etamax=1.0, lambda_=0.96, nu=0.99741):
        """kalman_type 0 (standard: kalman_epsilon, _q0, _qtau, _qmin, _eta,
        _etatau, _etamax) or 1 (fading memory: kalman_lambda_short, kalman_nue_short)."""
        if kalman_type == 0:
            _lib.check(self._lib.n2p2_training_set_kalman_standard(self._h, epsilon, q0, qtau, qmin, eta, etatau,
                                                                   etamax))
        else:
            _lib.check(self._lib.n2p2_training_set_kalman_fading_memory(self._h, epsilon, q0, qtau, qmin, lambda_,
                                                                        nu))

    def setupUpdaterGradient(self, gradient_type=1, eta=1e-5, adam_eta=1e-3, beta1=0.9, beta2=0.999,
                             epsilon=1e-8):
        """gradient_type 0 (fixed step gradient_eta) or 1 (Adam)."""
        if gradient_type == 0:
            _lib.check(self._lib.n2p2_training_set_gradient_fixed(self._h, eta))
        else:
            _lib.check(self._lib.n2p2_training_set_gradient_adam(self._h, adam_eta, beta1, beta2, epsilon))

    def setForceWeight(self, w):
        self.forceWeight = float(w)
        _lib.check(self._lib.n2p2_training_set_force_weight(self._h, self.forceWeight))

    def setUpdateStrategy(self, strategy=0):
        """update_strategy 0 (combined) or 1 (one updater per element); call
        before setting up the updater."""
        _lib.check(self._lib.n2p2_training_set_update_strategy(self._h, int(strategy)))

    def setJacobianMode(self, mode=1):
        """jacobian_mode 0/1 (a task batch summed into one observation) or 2
        (every candidate its own observation; Kalman filter, combined
        strategy, at most 16)."""
        _lib.check(self._lib.n2p2_training_set_jacobian_mode(self._h, int(mode)))

    def setTaskBatchSize(self, energy=1, force=1):
        """task_batch_size_energy / task_batch_size_force: candidates summed
        into one observation per update."""
        _lib.check(self._lib.n2p2_training_set_task_batch_size(self._h, int(energy), int(force)))
        self.taskBatch = {ENERGY: int(energy), FORCE: int(force)}

    # -- updates -----------------------------------------------------------
    def update(self, prop, structure, atom=None, component=None):
        """Candidates in order (one update per task batch of them); returns
        the errors (reference - prediction, internal units) of every
        candidate, seen before its update."""
        s = np.ascontiguousarray(structure, dtype=np.int32).ravel()
        n = s.size
        errors = np.zeros(n)
        if prop == FORCE:
            a = np.ascontiguousarray(atom, dtype=np.int32).ravel()
            c = np.ascontiguousarray(component, dtype=np.int32).ravel()
            if a.size != n or c.size != n:
                raise ValueError("structure, atom and component differ in length")
            _lib.check(self._lib.n2p2_training_update(self._h, FORCE, n, _ip(s), _ip(a), _ip(c), _dp(errors)))
        else:
            _lib.check(self._lib.n2p2_training_update(self._h, ENERGY, n, _ip(s), None, None, _dp(errors)))
        return errors

    def observe(self, prop, structure, atom=0, component=0):
        """(error, Jacobian) of one observation at the current weights, no
        update; the Jacobian in weight-file order, force weight applied."""
        err = np.zeros(1)
        jac = np.zeros(self.numWeights)
        _lib.check(self._lib.n2p2_training_observe(self._h, int(prop), int(structure), int(atom), int(component),
                                                   _dp(err), _dp(jac)))
        return float(err[0]), jac

    def updateThreshold(self, prop, numUpdates, structure, atom=None, component=None, threshold=1.0, trials=3,
                        rmse=None):
        """selection_mode 2: `numUpdates` updates over the candidate list
        (see n2p2_training_update_threshold); rmse defaults to the current
        training RMSE (internal units).  Returns (candidates consumed, errors
        of the used candidates)."""
        s = np.ascontiguousarray(structure, dtype=np.int32).ravel()
        if rmse is None:
            rmse = self.trainingErrors()[0 if prop == ENERGY else 1]
        errors = np.zeros(numUpdates)
        used = ctypes.c_int32()
        if prop == FORCE:
            a = np.ascontiguousarray(atom, dtype=np.int32).ravel()
            c = np.ascontiguousarray(component, dtype=np.int32).ravel()
            _lib.check(self._lib.n2p2_training_update_threshold(self._h, FORCE, numUpdates, s.size, _ip(s), _ip(a),
                                                                _ip(c), threshold, trials, rmse, ctypes.byref(used),
                                                                _dp(errors)))
        else:
            _lib.check(self._lib.n2p2_training_update_threshold(self._h, ENERGY, numUpdates, s.size, _ip(s), None,
                                                                None, threshold, trials, rmse, ctypes.byref(used),
                                                                _dp(errors)))
        return used.value, errors

    def trainingErrors(self):
        """(RMSE energy per atom, RMSE force components), internal units."""
        out = np.zeros(2)
        _lib.check(self._lib.n2p2_training_get_errors(self._h, _dp(out)))
        return float(out[0]), float(out[1])

    def updateCandidates(self):
        """Energy candidates (structures) and force candidates (structure,
        atom, component), Training::setupUpdateCandidates for 2G."""
        e = np.arange(len(self.structures), dtype=np.int32)
        s = np.repeat(e, 3 * self.atomsPerStructure)
        a = np.concatenate([np.repeat(np.arange(n, dtype=np.int32), 3) for n in self.atomsPerStructure])
        c = np.tile(np.arange(3, dtype=np.int32), int(self.atomsPerStructure.sum()))
        return e, (s, a, c)

    def sortedCandidates(self):
        """selection_mode 1 (Training::sortUpdateCandidates,
        Training.cpp:2008-2061): candidate orders by descending error at the
        current weights -- |E_ref - E| / N per structure, |F_ref - F| per force
        component (unit factors do not change the order)."""
        b = self.batch
        b.evaluate(forces=True, storeDGdr=True, graph=False)
        E, F = b.energies(), b.forces()
        ee = np.abs((self.energiesRef - E) / self.atomsPerStructure)
        ef = np.abs(self.forcesRef - F).ravel()   # (atom, component) in candidate order
        return np.argsort(-ee, kind="stable"), np.argsort(-ef, kind="stable")

    def runEpoch(self, energyFraction=1.0, forceFraction=0.0, rng=None, selectionMode=0, threshold=1.0, trials=3):
        """One epoch of Training::loop: candidates shuffled per property, the
        energy and force updates (fraction x candidates each) in a shuffled
        schedule, each update taking the next candidate of its property
        (selectionMode 0 random order, 1 sorted by descending error) or trying
        candidates against threshold x the training RMSE at the epoch's start
        (selectionMode 2, up to `trials`).
        Returns the errors per property (internal units)."""
        rng = np.random.default_rng() if rng is None else rng
        rmse = self.trainingErrors() if selectionMode == 2 else None
        ec, (fs, fa, fc) = self.updateCandidates()
        be, bf = self.taskBatch[ENERGY], self.taskBatch[FORCE]
        ne = int(energyFraction * ec.size / be)   # updates per property
        nf = int(forceFraction * fs.size / bf)
        if selectionMode == 1:
            eo, fo = self.sortedCandidates()
        else:
            eo = rng.permutation(ec.size)
            fo = rng.permutation(fs.size)
        schedule = np.concatenate([np.full(nf, FORCE), np.full(ne, ENERGY)])
        if ne and nf:
            rng.shuffle(schedule)
        mode = {ENERGY: selectionMode, FORCE: selectionMode}
        out = self.runSchedule(schedule, {ENERGY: eo, FORCE: fo}, mode, {ENERGY: threshold, FORCE: threshold},
                               {ENERGY: trials, FORCE: trials}, rmse)
        self.epoch += 1
        return out

    def runSchedule(self, schedule, orders, selectionMode, threshold, trials, rmse=None):
        """The updates of one epoch in the order of `schedule` (ENERGY / FORCE
        per update, Training::loop's epochSchedule): each property walks its
        candidate order from where its last update stopped (wrapping), taking
        the next task batch (selection modes 0 and 1) or trying candidates
        against threshold[p] x rmse[p] (mode 2, at most trials[p]; rmse in
        internal units, the training RMSE at the epoch's start).  Per-property
        dictionaries; returns the errors of the used candidates per property."""
        ec, (fs, fa, fc) = self.updateCandidates()
        eo, fo = orders[ENERGY], orders[FORCE]
        be, bf = self.taskBatch[ENERGY], self.taskBatch[FORCE]
        schedule = np.asarray(schedule)
        errs = {ENERGY: [], FORCE: []}
        pos = {ENERGY: 0, FORCE: 0}
        k = 0
        while k < schedule.size:   # runs of one property go to the device in one call
            p = int(schedule[k])
            r = k
            while r < schedule.size and schedule[r] == p:
                r += 1
            cnt = (r - k) * (be if p == ENERGY else bf)   # candidates of this run
            if selectionMode[p] == 2:
                if p == ENERGY:
                    order = eo[(pos[p] + np.arange(ec.size)) % ec.size]
                    used, e = self.updateThreshold(ENERGY, r - k, ec[order], threshold=threshold[p], trials=trials[p],
                                                   rmse=rmse[0])
                else:
                    order = fo[(pos[p] + np.arange(fs.size)) % fs.size]
                    used, e = self.updateThreshold(FORCE, r - k, fs[order], fa[order], fc[order],
                                                   threshold=threshold[p], trials=trials[p], rmse=rmse[1])
                errs[p].append(e)
                pos[p] += used
                k = r
                continue
            if p == ENERGY:
                idx = eo[(pos[p] + np.arange(cnt)) % ec.size]
                errs[p].append(self.update(ENERGY, ec[idx]))
            else:
                idx = fo[(pos[p] + np.arange(cnt)) % fs.size]
                errs[p].append(self.update(FORCE, fs[idx], fa[idx], fc[idx]))
            pos[p] += cnt
            k = r
        return {p: (np.concatenate(v) if v else np.zeros(0)) for p, v in errs.items()}

    # -- state ---------------------------------------------------------------
    def weights(self):
        """All elements' connections, weight-file order."""
        out = np.zeros(self.numWeights)
        _lib.check(self._lib.n2p2_training_get_weights(self._h, _dp(out)))
        return out

    def setWeights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        if w.size != self.numWeights:
            raise ValueError("expected %d weights" % self.numWeights)
        _lib.check(self._lib.n2p2_training_set_weights(self._h, _dp(w)))

    def kalmanStatus(self):
        """KalmanFilter::status fields."""
        st = np.zeros(7)
        _lib.check(self._lib.n2p2_training_get_kalman_status(self._h, _dp(st)))
        keys = ("numUpdates", "Pdiag", "Poffdiag", "Kmean", "q", "eta_or_lambda", "gamma")
        return dict(zip(keys, st.tolist()))

    def errors(self):
        """RMSE of the energy per atom and of the force components over the
        set at the current weights, physical units (Training's errorTrain
        RMSEpa and RMSE)."""
        b = self.batch
        b.evaluate(forces=True, storeDGdr=True, graph=False)
        E = b.energies()
        F = b.forces()
        de = (E - self.energiesRef) / self.atomsPerStructure
        df = (F - self.forcesRef).ravel()
        return {"energy_rmse_per_atom": float(np.sqrt(np.mean(de * de))),
                "force_rmse": float(np.sqrt(np.mean(df * df)))}


# ---------------------------------------------------------------------------
# The training program (nnp-train) around the update loop
# ---------------------------------------------------------------------------

# Settings::keywordMap alternatives the training program reads under their
# primary names (Settings.cpp:138-141).
_ALIASES = {"rmse_threshold_energy": "short_energy_error_threshold",
            "rmse_threshold_force": "short_force_error_threshold",
            "energy_fraction": "short_energy_fraction",
            "force_fraction": "short_force_fraction"}


def read_settings(path):
    """Keyword -> list of value strings of an input.nn file (comments after
    '#' dropped; a keyword without values maps to [""])."""
    out = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            parts = line.split(None, 1)
            out.setdefault(parts[0], []).append(parts[1].strip() if len(parts) > 1 else "")
    return out


class ShuffleRng:
    """std::mt19937_64 with std::shuffle (n2p2_shuffle_rng_*): the generators
    Training::rngNew and rngGlobalNew (Training.h:577-579)."""

    def __init__(self, seed):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._lib.n2p2_shuffle_rng_create(ctypes.c_uint64(int(seed)), ctypes.byref(h)))
        self._h = h

    def shuffle(self, values):
        v = np.ascontiguousarray(values, dtype=np.int64)
        if v.size:
            _lib.check(self._lib.n2p2_shuffle_rng_shuffle(self._h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                                          v.size))
        return v

    def close(self):
        if getattr(self, "_h", None):
            self._lib.n2p2_shuffle_rng_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TrainingRun:
    """The reference's nnp-train program for a 2G model directory (input.nn,
    scaling.data, input.data) with the updates on the GPU: the set-up
    sequence of nnp-train.cpp (random number generators, the structure
    distribution's draws on one process, the training/test split, random
    initial weights, the update plan and updater parameters), then
    Training::loop -- per epoch the candidate shuffles, the shuffled epoch
    schedule, the updates, and the errors of both sets (the learning curve).

    References: Dataset::setupRandomNumberGenerator (Dataset.cpp:110-163),
    distributeStructures (:724-886), Training::selectSets (Training.cpp:82-228),
    randomizeNeuralNetworkWeights (:3628-3679) with
    NeuralNetwork::modifyConnections (NeuralNetwork.cpp:212-315),
    setupTraining (:737-1207), setupUpdatePlan (:3851-3959), setupSelectionMode
    (:3681-3787), loop (:2147-2254), shuffleUpdateCandidates / setEpochSchedule
    (:2062-2111), calculateError with Structure::updateError
    (Structure.cpp:1387-1415) and writeLearningCurve (:1734-1842).

    Supported: the combined update strategy, the Kalman filter (standard,
    fading memory) and gradient descent (fixed, Adam), energy and optional
    force updates, every selection mode with a constant schedule, task
    batches (threshold selection: one candidate per update), random initial
    weights with the Glorot-Bengio scaling (the reference's default) or the
    weights of `use_old_weights_short`.  One process (the reference's
    single-rank run).
    """

    def __init__(self, directory, device=0):
        from .gsl_rng import Mt19937, Taus
        from .mode import Mode
        from .structure import read_structures
        self.directory = directory
        st = read_settings(os.path.join(directory, "input.nn"))
        self.settings = st
        for kw in ("nguyen_widrow_weights_short", "precondition_weights", "normalize_data_set"):
            if kw in st:
                raise ValueError(f"keyword {kw} is not supported by this training driver")
        if int(self._get("update_strategy", "0")) != 0:
            raise ValueError("only the combined update strategy (update_strategy 0) is supported here")
        self.mode = Mode(device)
        m = self.mode
        m.initialize()
        m.loadSettingsFile(os.path.join(directory, "input.nn"))
        m.setupGeneric()
        m.setupSymmetryFunctionScaling(os.path.join(directory, "scaling.data"))
        self.normalize = all(k in st for k in ("mean_energy", "conv_energy", "conv_length"))
        self.convEnergy = float(st["conv_energy"][0]) if self.normalize else 1.0
        self.convLength = float(st["conv_length"][0]) if self.normalize else 1.0
        structures = read_structures(os.path.join(directory, "input.data"))
        # Dataset::setupRandomNumberGenerator on one process
        self.rng = Mt19937(int(self._get("random_seed")))
        self.rngGlobal = Taus(self.rng.get())
        # distributeStructures(randomize = true): one gsl_rng_uniform_int(rng, numProcs) per structure
        for _ in structures:
            self.rng.uniform_int(1)
        # selectSets
        tf = float(self._get("test_fraction"))
        test = [self.rng.uniform() < tf for _ in structures]
        self.train = [s for s, t in zip(structures, test) if not t]
        self.test = [s for s, t in zip(structures, test) if t]
        # initializeWeights
        if "use_old_weights_short" in st:
            m.setupNeuralNetworkWeights(os.path.join(directory, "weights.%03zu.data"))
        else:
            self._randomizeWeights()
        self.useForces = "use_short_forces" in st
        self.pk = [ENERGY] + ([FORCE] if self.useForces else [])
        self.training = Training(m, self.train, [s.energyRef for s in self.train],
                                 np.concatenate([s.forcesRef for s in self.train]))
        self.testBatch = m.batch(self.test) if self.test else None
        if self.testBatch is not None:
            self.testBatch.setPositions(np.concatenate([s.positions for s in self.test]))
        self._setupTraining()
        self.epoch = 0
        self.learningCurve = []

    def _get(self, key, default=None):
        for k in (key, _ALIASES.get(key)):
            if k and k in self.settings:
                return self.settings[k][0]
        if default is None:
            raise KeyError(f"keyword {key} missing from input.nn")
        return default

    def _has(self, key):
        return key in self.settings or (_ALIASES.get(key) in self.settings)

    def _randomizeWeights(self):
        """randomizeNeuralNetworkWeights: uniform connections in [weights_min,
        weights_max) from the global generator, element by element in
        connection order; then MS_GLOROTBENGIO (the weights of every tanh layer
        times sqrt(6 / (n_prev + n))) and MS_ZEROBIAS."""
        wmin = float(self._get("weights_min"))
        wmax = float(self._get("weights_max"))
        m = self.mode
        for e in range(m.numElements):
            neurons, activations = m.networkTopology(e)
            n = sum(neurons[l - 1] * neurons[l] + neurons[l] for l in range(1, len(neurons)))
            w = np.array([wmin + self.rngGlobal.uniform() * (wmax - wmin) for _ in range(n)])
            q = 0
            for l in range(1, len(neurons)):
                nw = neurons[l - 1] * neurons[l]
                if activations[l] == _ACTIVATION_TANH:
                    w[q:q + nw] *= np.sqrt(6.0 / (neurons[l - 1] + neurons[l]))
                q += nw
                w[q:q + neurons[l]] = 0.0
                q += neurons[l]
            m.setConnections(e, w)

    def _setupTraining(self):
        st, t = self.settings, self.training
        if self.useForces:
            t.setForceWeight(float(self._get("force_weight", "1.0")))
        jm = int(self._get("jacobian_mode", "1"))
        t.setJacobianMode(jm)
        # setupSelectionMode: the global keywords, then per property
        self.selectionMode = {p: 0 for p in self.pk}
        self.threshold = {p: 0.0 for p in self.pk}
        self.trials = {p: 0 for p in self.pk}
        names = {ENERGY: "energy", FORCE: "force"}
        for scope in ["all"] + self.pk:
            sfx = "" if scope == "all" else "_" + names[scope]
            props = self.pk if scope == "all" else [scope]
            if self._has("selection_mode" + sfx):
                args = self._get("selection_mode" + sfx).split()
                if len(args) != 1:
                    raise ValueError("selection mode schedules are not supported by this training driver")
                for p in props:
                    self.selectionMode[p] = int(args[0])
            if self._has("rmse_threshold" + sfx):
                for p in props:
                    self.threshold[p] = float(self._get("rmse_threshold" + sfx))
            if self._has("rmse_threshold_trials" + sfx):
                for p in props:
                    self.trials[p] = int(self._get("rmse_threshold_trials" + sfx))
        self.epochs = int(self._get("epochs"))
        # setupUpdatePlan
        e, (fs, _, _) = t.updateCandidates()
        patterns = {ENERGY: e.size, FORCE: fs.size}
        self.batchSize = {}
        self.numUpdates = {}
        for p in self.pk:
            frac = float(self._get(names[p] + "_fraction"))
            tb = int(self._get("task_batch_size_" + names[p]))
            if tb == 0:
                raise ValueError("task batches of the entire training set are not supported by this driver")
            self.batchSize[p] = tb
            self.numUpdates[p] = int(patterns[p] * frac / tb)
        t.setTaskBatchSize(self.batchSize[ENERGY], self.batchSize.get(FORCE, 1))
        total = float(sum(self.numUpdates.values()))
        ut = int(self._get("updater_type"))
        if ut == 1:
            kt = int(self._get("kalman_type", "0"))
            eps = float(self._get("kalman_epsilon"))
            q0 = float(self._get("kalman_q0"))
            qtau = float(self._get("kalman_qtau")) / total
            qmin = float(self._get("kalman_qmin"))
            if kt == 0:
                eta0 = float(self._get("kalman_eta"))
                etatau, etamax = 1.0, eta0
                if self._has("kalman_etatau") and self._has("kalman_etamax"):
                    etatau = float(self._get("kalman_etatau")) / total
                    etamax = float(self._get("kalman_etamax"))
                t.setupUpdaterKalman(0, eps, q0, qtau, qmin, eta0, etatau, etamax)
            else:
                t.setupUpdaterKalman(1, eps, q0, qtau, qmin, lambda_=float(self._get("kalman_lambda_short")),
                                     nu=float(self._get("kalman_nue_short")))
        elif ut == 0:
            gt = int(self._get("gradient_type", "0"))
            if gt == 0:
                t.setupUpdaterGradient(0, eta=float(self._get("gradient_eta")))
            else:
                t.setupUpdaterGradient(1, adam_eta=float(self._get("gradient_adam_eta")),
                                       beta1=float(self._get("gradient_adam_beta1")),
                                       beta2=float(self._get("gradient_adam_beta2")),
                                       epsilon=float(self._get("gradient_adam_epsilon")))
        else:
            raise ValueError("unknown updater type")
        # the shuffle generators, seeded from the GSL generators (Training.cpp:1041-1042)
        self.rngGlobalNew = ShuffleRng(self.rngGlobal.get())
        self.rngNew = ShuffleRng(self.rng.get())
        # update candidates in setup order (selectSets): energies by structure, forces by (structure, atom, component)
        self.orders = {ENERGY: np.arange(e.size, dtype=np.int64), FORCE: np.arange(fs.size, dtype=np.int64)}

    def errors(self):
        """calculateError: {"energy": (train, test), "force": (train, test)}
        RMSE of the energy per atom and of the force components in physical
        units (the learning curve's RMSEpa and RMSE columns)."""
        def rmse(batch, structs, stored):
            if batch is None:
                return 0.0, 0.0
            batch.evaluate(forces=True, storeDGdr=stored, graph=False)
            E, F = batch.energies(), batch.forces()
            Er = np.array([s.energyRef for s in structs])
            n = np.array([s.numAtoms for s in structs], dtype=np.float64)
            de = Er - E
            df = (np.concatenate([s.forcesRef for s in structs]) - F).ravel()
            return float(np.sqrt(np.sum(de * de / (n * n)) / len(structs))), float(np.sqrt(np.sum(df * df) / df.size))
        etr, ftr = rmse(self.training.batch, self.train, True)   # the trainer's batch keeps its stored dG/dr
        ete, fte = rmse(self.testBatch, self.test, False)
        return {"energy": (etr, ete), "force": (ftr, fte)}

    def _record(self):
        e = self.errors()
        self.learningCurve.append({"epoch": self.epoch, **e})
        return e

    def runEpoch(self):
        """One pass of Training::loop's epoch body."""
        t = self.training
        rmse = t.trainingErrors() if any(self.selectionMode[p] == 2 for p in self.pk) else None
        # the candidate vectors are shuffled (or sorted) in place: each epoch starts from the last one's order
        orders = self.orders
        for p in self.pk:
            if self.selectionMode[p] == 1:
                orders[p] = t.sortedCandidates()[0 if p == ENERGY else 1]
            else:
                orders[p] = self.rngNew.shuffle(orders[p])
        schedule = np.concatenate([np.full(self.numUpdates[p], p, dtype=np.int64) for p in reversed(self.pk)])
        if len(self.pk) > 1:
            schedule = self.rngGlobalNew.shuffle(schedule)
        t.runSchedule(schedule, orders, self.selectionMode, self.threshold, self.trials, rmse)
        self.epoch += 1
        return self._record()

    def run(self):
        """The full loop: errors of epoch 0, then `epochs` epochs; returns the
        learning curve (one dict per epoch)."""
        self.learningCurve = []
        self._record()
        for _ in range(self.epochs):
            self.runEpoch()
        return self.learningCurve

    def close(self):
        for o in ("rngNew", "rngGlobalNew", "testBatch", "training"):
            x = getattr(self, o, None)
            if x is not None:
                x.close()
                setattr(self, o, None)
        if getattr(self, "mode", None) is not None:
            self.mode.close()
            self.mode = None


_ACTIVATION_TANH = 2   # NeuralNetwork::AF_TANH
