"""Training updates on the GPU (n2p2_b200.training) against the training
oracle (oracle/training_ref.py, itself pinned to the reference library by
finite differences in tests/test_cpu_training.py).

Observation errors and Jacobians to 1e-10 relative; updater sequences
(Kalman filter standard and fading memory, gradient descent fixed and Adam)
to 1e-9 relative in the weights after every run.  The set mixes boxes larger
than the cutoff diameter with one smaller (periodic self-images: the force
prediction leaves them out as Mode::calculateForces does, the Jacobian keeps
them as Training::collectDGdxia does)."""
import os

import numpy as np
import pytest

from n2p2_b200 import Mode, water
from n2p2_b200.training import ENERGY, FORCE, Training
from oracle import ref as oref
from tests import helpers as H

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oref.available(), reason="reference library not built")]


def _set():
    ss = [water.water_box(8, seed=4, sigma=0.1)] + water.water_batch(3, seed=21, n_min=32, n_max=48)
    E, F = [], []
    for s in ss:
        a = H.reference_snapshot(H.WATER40, s)
        E.append(a["energy"])
        F.append(a["forces"])
    return ss, np.array(E), np.concatenate(F)


@pytest.fixture(scope="module")
def data():
    ss, E, F = _set()
    from oracle import training_ref as T
    nets = T.Networks(H.WATER40)
    w0 = nets.weights + np.random.default_rng(5).normal(0.0, 0.02, nets.numWeights)   # away from the labels
    return ss, E, F, w0


def _pair(data, updater, force_weight=3.0):
    from oracle import training_ref as T
    ss, E, F, w0 = data
    m = Mode(0)
    m.setupFromDirectory(H.WATER40)
    tr = Training(m, ss, E, F)
    tr.setWeights(w0)
    tr.setForceWeight(force_weight)
    n = tr.numWeights
    kind, args = updater
    if kind == "kf":
        tr.setupUpdaterKalman(0, **args)
        up = T.KalmanFilter(n, 0, args["epsilon"], args["q0"], args["qtau"], args["qmin"], args["eta"], args["etatau"],
                            args["etamax"])
    elif kind == "kf_fading":
        tr.setupUpdaterKalman(1, epsilon=args["epsilon"], q0=args["q0"], qtau=args["qtau"], qmin=args["qmin"],
                              lambda_=args["lambda_"], nu=args["nu"])
        up = T.KalmanFilter(n, 1, args["epsilon"], args["q0"], args["qtau"], args["qmin"], lam=args["lambda_"],
                            nu=args["nu"])
    elif kind == "gd":
        tr.setupUpdaterGradient(0, eta=args["eta"])
        up = T.GradientDescent(n, 0, args["eta"])
    else:
        tr.setupUpdaterGradient(1, adam_eta=args["eta"])
        up = T.GradientDescent(n, 1, args["eta"])
    ref = T.Training(H.WATER40, ss, E, F, up, force_weight=force_weight)
    ref.nets.weights = w0.copy()
    return m, tr, ref


def test_jacobians_match_reference_analytic(data):
    """The device's observation Jacobians (kParamGrad and the force
    adjoint) against the reference's analytic derivatives
    (NeuralNetwork::calculateDEdc / calculateDFdc, NeuralNetwork.cpp:444-527,
    summed as Training::update does) at the set's current weights: 1e-10 of
    the largest entry (force Jacobians carry the force weight)."""
    m, tr, ref = _pair(data, ("gd", {"eta": 1e-3}))
    ss = data[0]
    d = str(__import__("tempfile").mkdtemp())
    try:
        import shutil
        for fn in os.listdir(H.WATER40):
            shutil.copy(os.path.join(H.WATER40, fn), d)
        from oracle import training_ref as T
        nets = T.Networks(H.WATER40)
        w = tr.weights()
        for e, sym in enumerate(nets.symbols):
            water.write_weights(os.path.join(d, "weights.%03d.data" % T.oref_z(sym)),
                                w[nets.offsets[e]:nets.offsets[e + 1]])
        p = oref.RefPrediction(d)
        try:
            for prop, s, a, c in ((ENERGY, 0, 0, 0), (ENERGY, 2, 0, 0), (FORCE, 0, 5, 2), (FORCE, 0, 0, 0),
                                  (FORCE, 2, 7, 1), (FORCE, 3, 11, 0)):
                _, J = tr.observe(prop, s, a, c)
                Jr = p.jacobian(ss[s].to_text(), 0 if prop == ENERGY else 1, a, c)
                if prop == FORCE:
                    Jr = Jr * tr.forceWeight
                assert np.abs(J - Jr).max() <= 1e-10 * np.abs(Jr).max(), (prop, s, a, c)
        finally:
            p.close()
    finally:
        __import__("shutil").rmtree(d, ignore_errors=True)
        tr.close()
        m.close()


def test_observations_match_oracle(data):
    m, tr, ref = _pair(data, ("gd", {"eta": 1e-3}))
    try:
        for prop, s, a, c in ((ENERGY, 1, 0, 0), (FORCE, 2, 7, 1), (FORCE, 0, 5, 2), (FORCE, 0, 0, 0)):
            e, J = tr.observe(prop, s, a, c)
            er, Jr = ref.observation(prop, s, a, c)
            if prop == FORCE:
                Jr = Jr * tr.forceWeight
            scale = abs(data[1][s]) if prop == ENERGY else np.abs(data[2]).max()
            assert abs(e - er) <= 1e-10 * scale, (prop, s, a, c, e, er)
            assert H.max_rel(J, Jr) <= 1e-10, (prop, s, a, c)
    finally:
        tr.close()
        m.close()


SCHEDULE = [(ENERGY, [1, 3, 0]), (FORCE, [(2, 7, 1), (0, 5, 2), (3, 11, 0)]), (ENERGY, [2, 0]),
            (FORCE, [(1, 4, 2), (0, 0, 0)])]

UPDATERS = [
    ("kf", {"epsilon": 1e-2, "q0": 0.01, "qtau": 2.302, "qmin": 1e-6, "eta": 0.01, "etatau": 2.302, "etamax": 1.0}),
    ("kf_fading", {"epsilon": 1e-2, "q0": 0.01, "qtau": 2.302, "qmin": 1e-6, "lambda_": 0.96, "nu": 0.99741}),
    ("gd", {"eta": 1e-4}),
    ("adam", {"eta": 1e-3}),
]


@pytest.mark.parametrize("updater", UPDATERS, ids=[u[0] for u in UPDATERS])
def test_update_sequence_matches_oracle(data, updater):
    m, tr, ref = _pair(data, updater)
    try:
        for prop, cands in SCHEDULE:
            if prop == ENERGY:
                errs = tr.update(ENERGY, cands)
                errs_ref = [ref.update(0, s) for s in cands]
            else:
                s, a, c = (np.array(x) for x in zip(*cands))
                errs = tr.update(FORCE, s, a, c)
                errs_ref = [ref.update(1, *x) for x in cands]
            assert np.allclose(errs, errs_ref, rtol=1e-9, atol=1e-12), (prop, errs, errs_ref)
            assert H.max_rel(tr.weights(), ref.nets.weights) <= 1e-9
        if updater[0].startswith("kf"):
            st = tr.kalmanStatus()
            assert st["numUpdates"] == 10
            assert abs(st["Pdiag"] - np.mean(np.abs(np.diag(ref.updater.P)))) <= 1e-9 * st["Pdiag"]
            assert abs(st["q"] - ref.updater.q) <= 1e-15
    finally:
        tr.close()
        m.close()


def test_epochs_reduce_errors(data):
    ss, E, F, w0 = data
    m = Mode(0)
    m.setupFromDirectory(H.WATER40)
    tr = Training(m, ss, E, F)
    try:
        tr.setWeights(w0)
        tr.setupUpdaterKalman(0)
        tr.setForceWeight(10.0)
        before = tr.errors()
        rng = np.random.default_rng(1)
        for ep in range(3):
            tr.runEpoch(energyFraction=1.0, forceFraction=0.05, rng=rng, selectionMode=2 if ep == 2 else 0)
        after = tr.errors()
        assert after["energy_rmse_per_atom"] < 0.5 * before["energy_rmse_per_atom"]
        assert after["force_rmse"] < before["force_rmse"]
        # the mode's other batches evaluate the trained weights
        b = m.batch(ss[:1])
        b.setPositions(ss[0].positions)
        b.evaluate(forces=False)
        e_trained = b.energies()[0]
        b.close()
        assert abs(e_trained - E[0]) / ss[0].numAtoms <= before["energy_rmse_per_atom"]
    finally:
        tr.close()
        m.close()


def test_task_batches_match_oracle(data):
    """task_batch_size > 1: candidates summed into one observation per update."""
    up = ("kf", UPDATERS[0][1])
    m, tr, ref = _pair(data, up)
    try:
        tr.setTaskBatchSize(energy=3, force=2)
        e = tr.update(ENERGY, [1, 3, 0, 2, 0, 1])
        e_ref = ref.update_batch(0, [(1, 0, 0), (3, 0, 0), (0, 0, 0)]) + ref.update_batch(0, [(2, 0, 0), (0, 0, 0),
                                                                                           (1, 0, 0)])
        assert np.allclose(e, e_ref, rtol=1e-9, atol=1e-12)
        cands = [(2, 7, 1), (0, 5, 2), (3, 11, 0), (1, 4, 2)]
        s, a, c = (np.array(x) for x in zip(*cands))
        f = tr.update(FORCE, s, a, c)
        f_ref = ref.update_batch(1, cands[:2]) + ref.update_batch(1, cands[2:])
        assert np.allclose(f, f_ref, rtol=1e-9, atol=1e-12)
        assert H.max_rel(tr.weights(), ref.nets.weights) <= 1e-9
        assert tr.kalmanStatus()["numUpdates"] == 4
    finally:
        tr.close()
        m.close()


@pytest.mark.parametrize("kind", ["kf", "adam"])
def test_element_strategy_matches_oracle(data, kind):
    """update_strategy 1: one updater per element with its share of the error."""
    from oracle import training_ref as T
    ss, E, F, w0 = data
    m = Mode(0)
    m.setupFromDirectory(H.WATER40)
    tr = Training(m, ss, E, F)
    try:
        tr.setWeights(w0)
        tr.setForceWeight(3.0)
        tr.setUpdateStrategy(1)
        ref = T.Training(H.WATER40, ss, E, F, None, force_weight=3.0)
        ref.nets.weights = w0.copy()
        offs = ref.nets.offsets
        sizes = [offs[e + 1] - offs[e] for e in range(len(offs) - 1)]
        if kind == "kf":
            a = UPDATERS[0][1]
            tr.setupUpdaterKalman(0, **a)
            ref.updater = [T.KalmanFilter(n, 0, a["epsilon"], a["q0"], a["qtau"], a["qmin"], a["eta"], a["etatau"],
                                          a["etamax"]) for n in sizes]
        else:
            tr.setupUpdaterGradient(1, adam_eta=1e-3)
            ref.updater = [T.GradientDescent(n, 1, 1e-3) for n in sizes]
        for prop, cands in SCHEDULE:
            if prop == ENERGY:
                errs = tr.update(ENERGY, cands)
                errs_ref = [ref.update_element(0, s) for s in cands]
            else:
                s, a_, c = (np.array(x) for x in zip(*cands))
                errs = tr.update(FORCE, s, a_, c)
                errs_ref = [ref.update_element(1, *x) for x in cands]
            assert np.allclose(errs, errs_ref, rtol=1e-9, atol=1e-12)
            assert H.max_rel(tr.weights(), ref.nets.weights) <= 1e-9
    finally:
        tr.close()
        m.close()


def test_threshold_selection_matches_oracle(data):
    """selection_mode 2: trials until an error exceeds threshold x RMSE; the
    update uses the candidate the trials stopped at."""
    m, tr, ref = _pair(data, ("kf", UPDATERS[0][1]))
    try:
        ss = data[0]
        rmse_e, rmse_f = tr.trainingErrors()
        # the oracle's training RMSE at the same weights
        de = [ref.observation(0, k)[0] / ss[k].numAtoms for k in range(len(ss))]
        assert abs(rmse_e - np.sqrt(np.mean(np.square(de)))) <= 1e-9 * rmse_e

        def oracle_threshold(prop, cands, n_updates, thr, trials, rmse):
            pos, errs = 0, []
            for _ in range(n_updates):
                for _il in range(trials):
                    k = cands[pos % len(cands)]
                    e = ref.observation(prop, *k)[0]
                    scale = ss[k[0]].numAtoms * rmse if prop == 0 else rmse
                    pos += 1
                    if abs(e) / scale > thr:
                        break
                errs.append(ref.update(prop, *k))
            return pos, errs

        ecands = [(s, 0, 0) for s in (2, 0, 3, 1, 2, 3)]
        used, errs = tr.updateThreshold(ENERGY, 3, [c[0] for c in ecands], threshold=1.0, trials=2, rmse=rmse_e)
        used_ref, errs_ref = oracle_threshold(0, ecands, 3, 1.0, 2, rmse_e)
        assert used == used_ref and np.allclose(errs, errs_ref, rtol=1e-9, atol=1e-12)
        fcands = [(2, 7, 1), (0, 5, 2), (3, 11, 0), (1, 4, 2), (0, 0, 0), (2, 3, 1)]
        s, a, c = (np.array(x) for x in zip(*fcands))
        used, errs = tr.updateThreshold(FORCE, 3, s, a, c, threshold=1.0, trials=3, rmse=rmse_f)
        used_ref, errs_ref = oracle_threshold(1, fcands, 3, 1.0, 3, rmse_f)
        assert used == used_ref and np.allclose(errs, errs_ref, rtol=1e-9, atol=1e-12)
        assert H.max_rel(tr.weights(), ref.nets.weights) <= 1e-9
    finally:
        tr.close()
        m.close()


def test_sort_selection_order(data):
    """selection_mode 1: candidates by descending error at the current weights."""
    m, tr, ref = _pair(data, ("kf", UPDATERS[0][1]))
    try:
        ss = data[0]
        eo, fo = tr.sortedCandidates()
        ee = [abs(ref.observation(0, k)[0]) / ss[k].numAtoms for k in range(len(ss))]
        assert list(eo) == list(np.argsort(-np.array(ee), kind="stable"))
        _, (fs, fa, fc) = tr.updateCandidates()
        top = [abs(ref.observation(1, fs[q], fa[q], fc[q])[0]) for q in fo[:5]]
        rest = [abs(ref.observation(1, fs[q], fa[q], fc[q])[0]) for q in fo[-5:]]
        assert all(x >= y for x, y in zip(top, top[1:])) and min(top) >= max(rest)
        tr.runEpoch(energyFraction=1.0, forceFraction=0.02, selectionMode=1)
        assert tr.kalmanStatus()["numUpdates"] > len(ss)
    finally:
        tr.close()
        m.close()


@pytest.mark.parametrize("updater", UPDATERS[:2], ids=[u[0] for u in UPDATERS[:2]])
def test_full_jacobian_matches_oracle(data, updater):
    """jacobian_mode 2: a task batch's candidates as separate observations of
    one Kalman update (m x m gain)."""
    m, tr, ref = _pair(data, updater)
    try:
        tr.setJacobianMode(2)
        tr.setTaskBatchSize(energy=3, force=2)
        e = tr.update(ENERGY, [1, 3, 0, 2, 0, 1])
        e_ref = ref.update_full(0, [(1, 0, 0), (3, 0, 0), (0, 0, 0)]) + ref.update_full(0, [(2, 0, 0), (0, 0, 0),
                                                                                         (1, 0, 0)])
        # the m x m inverse (Gauss-Jordan here, LU in numpy) rounds differently: errors are held
        # relative to the largest one of the sequence
        assert np.allclose(e, e_ref, rtol=1e-9, atol=1e-9 * np.abs(e_ref).max())
        cands = [(2, 7, 1), (0, 5, 2), (3, 11, 0), (1, 4, 2)]
        s, a, c = (np.array(x) for x in zip(*cands))
        f = tr.update(FORCE, s, a, c)
        f_ref = ref.update_full(1, cands[:2]) + ref.update_full(1, cands[2:])
        assert np.allclose(f, f_ref, rtol=1e-9, atol=1e-9 * np.abs(f_ref).max())
        assert H.max_rel(tr.weights(), ref.nets.weights) <= 1e-9
        st = tr.kalmanStatus()
        assert abs(st["Pdiag"] - np.mean(np.abs(np.diag(ref.updater.P)))) <= 1e-9 * st["Pdiag"]
    finally:
        tr.close()
        m.close()



def test_full_jacobian_alternating_ranks_and_limits(data):
    """A rank-m update followed by rank-one updates and a status read (the
    pending rank-m change of P is applied by the next rank-one pass and by
    the flush), the largest task batch (m = 16, with repeated candidates:
    H^T P H is then rank-deficient, A = H^T P H + I/eta stays positive
    definite), and the rejection of m = 17 -- all against the oracle to the
    bounds of test_full_jacobian_matches_oracle."""
    m, tr, ref = _pair(data, UPDATERS[0])
    try:
        tr.setJacobianMode(2)
        tr.setTaskBatchSize(energy=2, force=2)
        e = list(tr.update(ENERGY, [1, 3]))
        e_ref = list(ref.update_full(0, [(1, 0, 0), (3, 0, 0)]))
        # back to one observation per update: reads P with the rank-2 change pending
        tr.setJacobianMode(1)
        tr.setTaskBatchSize(energy=1, force=1)
        e += list(tr.update(ENERGY, [0]))
        e_ref += [ref.update(0, 0)]
        f = list(tr.update(FORCE, [2], [7], [1]))
        f_ref = [ref.update(1, 2, 7, 1)]
        tr.setJacobianMode(2)
        tr.setTaskBatchSize(energy=3, force=2)
        f += list(tr.update(FORCE, [0, 3], [5, 11], [2, 0]))
        f_ref += list(ref.update_full(1, [(0, 5, 2), (3, 11, 0)]))
        st = tr.kalmanStatus()   # flushes the pending rank-2 change
        assert abs(st["Pdiag"] - np.mean(np.abs(np.diag(ref.updater.P)))) <= 1e-9 * st["Pdiag"]
        tr.setJacobianMode(1)
        tr.setTaskBatchSize(energy=1, force=1)
        e += list(tr.update(ENERGY, [2]))
        e_ref += [ref.update(0, 2)]
        # the largest task batch: 16 candidates (structures repeated)
        tr.setJacobianMode(2)
        tr.setTaskBatchSize(energy=16, force=1)
        seq = [k % 4 for k in range(16)]
        e += list(tr.update(ENERGY, seq))
        e_ref += list(ref.update_full(0, [(k, 0, 0) for k in seq]))
        e, e_ref, f, f_ref = (np.array(x) for x in (e, e_ref, f, f_ref))
        assert np.allclose(e, e_ref, rtol=1e-9, atol=1e-9 * np.abs(e_ref).max())
        assert np.allclose(f, f_ref, rtol=1e-9, atol=1e-9 * np.abs(f_ref).max())
        assert H.max_rel(tr.weights(), ref.nets.weights) <= 1e-9
        # 17 candidates per update are more than the full Jacobian takes
        w = tr.weights()
        with pytest.raises(Exception, match="16"):
            tr.setTaskBatchSize(energy=17, force=1)
            tr.update(ENERGY, [k % 4 for k in range(17)])
        assert np.array_equal(tr.weights(), w)
    finally:
        tr.close()
        m.close()
