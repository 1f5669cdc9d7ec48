"""The training oracle (oracle/training_ref.py) pinned to the reference:
its energy and force Jacobians against central differences of the reference
library's own energies and forces under perturbed weight files, and its
Kalman filter against recursive least squares on a linear problem."""
import os
import shutil

import numpy as np
import pytest

from n2p2_b200 import water
from oracle import ref as oref
from tests import helpers as H

pytestmark = pytest.mark.skipif(not oref.available(), reason="reference library not built")


def _write_weights(nets, d, w):
    for e, sym in enumerate(nets.symbols):
        from oracle.training_ref import oref_z
        water.write_weights(os.path.join(d, "weights.%03d.data" % oref_z(sym)),
                            w[nets.offsets[e]:nets.offsets[e + 1]])


def test_oracle_jacobians_match_reference_finite_differences(tmp_path):
    from oracle import training_ref as T
    s = water.water_box(8, seed=4, sigma=0.1)
    nets = T.Networks(H.WATER40)
    tr = T.Training(H.WATER40, [s], [0.0], np.zeros((s.numAtoms, 3)), updater=None)
    errE, HE = tr.observation(0, 0)
    atom, comp = 5, 1
    errF, HF = tr.observation(1, 0, atom, comp)
    snap = H.reference_snapshot(H.WATER40, s)
    assert abs(-errE - snap["energy"]) <= 1e-10 * abs(snap["energy"])      # prediction = reference E
    assert abs(-errF - snap["forces"][atom, comp]) <= 1e-10 * np.abs(snap["forces"]).max()
    d = str(tmp_path)
    for fn in os.listdir(H.WATER40):
        shutil.copy(os.path.join(H.WATER40, fn), d)
    rng = np.random.default_rng(3)
    picks = np.concatenate([rng.choice(nets.numWeights, 6, replace=False), [nets.offsets[1] - 1, nets.numWeights - 1]])
    for p in picks:
        h = 1e-5 * max(1.0, abs(nets.weights[p]))
        vals = []
        for sgn in (1.0, -1.0):
            w = nets.weights.copy()
            w[p] += sgn * h
            _write_weights(nets, d, w)
            a = H.reference_snapshot(d, s)
            vals.append((a["energy"], a["forces"][atom, comp]))
        dE = (vals[0][0] - vals[1][0]) / (2 * h)
        dF = (vals[0][1] - vals[1][1]) / (2 * h)
        assert abs(HE[p] - dE) <= 1e-6 * max(1.0, np.abs(HE).max()), p
        assert abs(HF[p] - dF) <= 1e-6 * max(1.0, np.abs(HF).max()), p


@pytest.mark.parametrize("box", [(8, 4, 0.1), (32, 7, 0.05)], ids=["8mol_self_images", "32mol"])
def test_oracle_jacobians_match_reference_analytic(box):
    """The restatement's energy and force Jacobians against the reference's
    own analytic derivatives (NeuralNetwork::calculateDEdc /
    calculateDFdc, NeuralNetwork.cpp:444-527, summed over the structure's
    atoms as Training::update does): 1e-12 of the largest entry.  The
    8-molecule box is smaller than the cutoff diameter, so atoms see their
    own periodic images (the Jacobian keeps them, Training.cpp:3604-3615)."""
    from oracle import training_ref as T
    n_mol, seed, sigma = box
    s = water.water_box(n_mol, seed=seed, sigma=sigma)
    tr = T.Training(H.WATER40, [s], [0.0], np.zeros((s.numAtoms, 3)), updater=None)
    p = oref.RefPrediction(H.WATER40)
    try:
        _, HE = tr.observation(0, 0)
        JE = p.jacobian(s.to_text(), 0)
        assert np.abs(HE - JE).max() <= 1e-12 * np.abs(JE).max()
        for atom, comp in ((0, 0), (5, 1), (s.numAtoms - 1, 2)):
            _, HF = tr.observation(1, 0, atom, comp)
            JF = p.jacobian(s.to_text(), 1, atom, comp)
            assert np.abs(HF - JF).max() <= 1e-12 * np.abs(JF).max(), (atom, comp)
    finally:
        p.close()


def test_kalman_restatement_is_recursive_least_squares():
    """With q = 0 and eta fixed, one observation per update, the filter is
    recursive least squares: its state is the regularised least-squares
    solution (prior information epsilon I, unit noise 1/eta) and its P the
    inverse of the accumulated information."""
    from oracle import training_ref as T
    rng = np.random.default_rng(0)
    n = 12
    wstar = rng.normal(size=n)
    kf = T.KalmanFilter(n, 0, epsilon=1e-3, q0=0.0, qtau=0.0, qmin=0.0, eta0=1.0, etatau=0.0, etamax=1.0)
    w = np.zeros(n)
    info = np.eye(n) * 1e-3
    rhs = np.zeros(n)
    for _ in range(60):
        h = rng.normal(size=n)
        y = h @ wstar
        kf.update(w, h, y - h @ w)
        info += np.outer(h, h)
        rhs += h * y
    assert np.allclose(w, np.linalg.solve(info, rhs), rtol=0, atol=1e-10)
    assert np.allclose(w, wstar, rtol=0, atol=1e-3)
    assert np.allclose(np.tril(kf.P), np.tril(np.linalg.inv(info)), rtol=1e-8, atol=1e-12)


def test_gradient_descent_restatement():
    from oracle import training_ref as T
    w = np.array([1.0, -2.0])
    g = T.GradientDescent(2, 0, eta=0.1)
    g.update(w, np.array([1.0, 2.0]), 0.5)
    assert np.allclose(w, [1.05, -1.9])
    a = T.GradientDescent(2, 1, eta=1e-3)
    w = np.zeros(2)
    a.update(w, np.array([1.0, -1.0]), 2.0)
    # first Adam step moves every weight by ~eta along error * jacobian
    assert np.allclose(w, [1e-3, -1e-3], rtol=1e-6)
