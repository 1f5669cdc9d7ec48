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
        errs = {ENERGY: [], FORCE: []}
        pos = {ENERGY: 0, FORCE: 0}
        k = 0
        while k < schedule.size:   # runs of one property go to the device in one call
            p = schedule[k]
            r = k
            while r < schedule.size and schedule[r] == p:
                r += 1
            cnt = (r - k) * (be if p == ENERGY else bf)   # candidates of this run
            if selectionMode == 2:
                if p == ENERGY:
                    order = eo[(pos[p] + np.arange(ec.size)) % ec.size]
                    used, e = self.updateThreshold(ENERGY, r - k, ec[order], threshold=threshold, trials=trials,
                                                   rmse=rmse[0])
                else:
                    order = fo[(pos[p] + np.arange(fs.size)) % fs.size]
                    used, e = self.updateThreshold(FORCE, r - k, fs[order], fa[order], fc[order],
                                                   threshold=threshold, trials=trials, rmse=rmse[1])
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
        self.epoch += 1
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
