"""Learned part: the GPU trainer's gradient against finite differences of the
CPU oracle's loss, training progress, what the trained student gains, and the
teacher fallback on extrapolation."""
import os
import time

import numpy as np
import pytest

from n2p2_b200 import student, water

from tests.helpers import GOLDEN

pytestmark = pytest.mark.gpu

TEACHER = os.path.join(GOLDEN, "models", "water56")


@pytest.fixture(scope="module")
def teacher():
    return student.load_mode(TEACHER)


@pytest.fixture(scope="module")
def student_dir(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("student"))
    student.write_student_model(d, student.training_structures(24, seed=5, n_min=32, n_max=96), seed=3)
    return d


def _file_to_port_index(pm):
    """Weight-file order -> index into the oracle's flat weight array."""
    a = pm.arrays
    ne = len(pm.symbols)
    neurons = a["neurons"].reshape(ne, 8)
    wb, bb = a["wBegin"].reshape(ne, 8), a["bBegin"].reshape(ne, 8)
    out = []
    for e in range(ne):
        L = int(pm.numLayers[e])
        for l in range(1, L):
            nin, nout = int(neurons[e, l - 1]), int(neurons[e, l])
            for j in range(nin):
                for k in range(nout):
                    out.append(int(wb[e, l]) + k * nin + j)
            for k in range(nout):
                out.append(int(bb[e, l]) + k)
    return np.array(out)


def _oracle_loss(pm, structs, E_ref, F_ref, wE=1.0, wF=10.0):
    le, lf, n_all = 0.0, 0.0, 0
    for s, st in enumerate(structs):
        r = pm.evaluate(st)
        n = st.numAtoms
        le += ((r["energy"] - E_ref[s]) / n) ** 2
        lf += float(np.sum((r["forces"] - F_ref[n_all:n_all + n]) ** 2))
        n_all += n
    return wE * le / len(structs) + wF * lf / (3 * n_all)


def test_gradient_matches_oracle_finite_differences(student_dir):
    from oracle.port import PortModel
    structs = student.training_structures(3, seed=21, n_min=32, n_max=48)
    m = student.load_mode(student_dir)
    b = m.batch(structs)
    b.setPositions(np.concatenate([s.positions for s in structs]))
    b.evaluate(forces=True, graph=False)
    rng = np.random.default_rng(2)
    E_ref = b.energies() + rng.normal(0, 0.05, len(structs))
    F_ref = b.forces() + rng.normal(0, 0.01, (b.numAtoms, 3))
    from n2p2_b200 import Trainer
    tr = Trainer(m)
    loss, grad = tr.step(b, E_ref, F_ref, update=False, gradient=True)

    pm = PortModel(student_dir)
    w = pm.arrays["weights"]            # the oracle reads this buffer in place
    idx = _file_to_port_index(pm)
    assert idx.size == tr.numParameters
    w0 = w.copy()
    l0 = _oracle_loss(pm, structs, E_ref, F_ref)
    assert abs(l0 - loss[0]) <= 1e-9 * abs(l0)
    # parameters of every layer of both elements, weights and biases
    picks = np.unique(np.concatenate([rng.choice(idx.size, 24, replace=False), [0, idx.size - 1]]))
    scale = np.max(np.abs(grad))
    for p in picks:
        h = 1e-5 * max(1.0, abs(w0[idx[p]]))
        w[idx[p]] = w0[idx[p]] + h
        lp = _oracle_loss(pm, structs, E_ref, F_ref)
        w[idx[p]] = w0[idx[p]] - h
        lm = _oracle_loss(pm, structs, E_ref, F_ref)
        w[idx[p]] = w0[idx[p]]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - grad[p]) <= 2e-6 * scale + 1e-6 * abs(fd), (p, fd, grad[p])


def test_gradient_matches_reference_analytic(student_dir):
    """The trainer's loss gradient (forward with tangents, reverse through
    both, second derivatives of the activations) against the reference's
    analytic network derivatives: with a_s = dL/dE_s and u_k = dL/dF_k of
    L = wE/S sum_s ((E_s - E_s^ref)/N_s)^2 + wF/(3N) sum_k (F_k - F_k^ref)^2,
    dL/dw = sum_s a_s dE_s/dw + sum_k u_k dF_k/dw with dE/dw and dF/dw from
    NeuralNetwork::calculateDEdc / calculateDFdc (NeuralNetwork.cpp:444-527)
    as Training::update sums them.  Bound: 1e-10 of the largest component."""
    from oracle import ref as oref
    # clusters (no periodic images): the trainer's force is calculateForces' force, which leaves an atom's
    # own periodic images out, while the training Jacobian keeps them (Training.cpp:3604-3615)
    from n2p2_b200 import Structure
    structs = [Structure(b.positions, b.elements, None)
               for b in (water.water_box(12, seed=51, sigma=0.1), water.water_box(16, seed=52, sigma=0.05))]
    m = student.load_mode(student_dir)
    b = m.batch(structs)
    b.setPositions(np.concatenate([s.positions for s in structs]))
    b.evaluate(forces=True, graph=False)
    E, F = b.energies(), b.forces()
    rng = np.random.default_rng(4)
    E_ref = E + rng.normal(0, 0.05, len(structs))
    F_ref = F + rng.normal(0, 0.01, F.shape)
    from n2p2_b200 import Trainer
    wE, wF = 1.0, 10.0
    tr = Trainer(m, energyWeight=wE, forceWeight=wF)
    _, grad = tr.step(b, E_ref, F_ref, update=False, gradient=True)
    p = oref.RefPrediction(student_dir)
    try:
        S, N = len(structs), b.numAtoms
        g_ref, a0 = np.zeros_like(grad), 0
        for k, s in enumerate(structs):
            n = s.numAtoms
            a = wE / S * 2.0 * (E[k] - E_ref[k]) / (n * n)
            u = wF / (3.0 * N) * 2.0 * (F[a0:a0 + n] - F_ref[a0:a0 + n])
            g_ref += p.loss_gradient(s.to_text(), a, u)
            a0 += n
    finally:
        p.close()
    assert np.abs(grad - g_ref).max() <= 1e-10 * np.abs(g_ref).max()


def test_parameters_round_trip(student_dir):
    from n2p2_b200 import Trainer
    m = student.load_mode(student_dir)
    tr = Trainer(m)
    w = tr.parameters()
    assert w.size == 2 * (14 * 16 + 16 + 16 * 16 + 16 + 16 + 1)
    w2 = w * 1.01
    tr.setParameters(w2)
    assert np.array_equal(tr.parameters(), w2)


def test_training_gain_and_speed(teacher, student_dir):
    train = student.training_structures(192, seed=31, n_min=32, n_max=128)
    held = student.training_structures(32, seed=32, n_min=32, n_max=128)
    E, F = student.label(teacher, train)
    Eh, Fh = student.label(teacher, held)
    m = student.load_mode(student_dir)
    apa = [s.numAtoms for s in held]

    def held_error():
        Es, Fs = student.label(m, held)
        return student.errors(Es, Fs, Eh, Fh, apa)

    before = held_error()
    tr = student.StudentTraining(m, train, E, F, batch_size=16, eta=2e-3, seed=1)
    l_first = tr.epoch()
    for _ in range(7):
        tr.epoch()
    assert tr.history[-1] < 0.5 * l_first
    after = held_error()
    # the trained network is much closer to the teacher than the untrained one
    assert after["energy_meV_per_atom_rms"] < 0.3 * before["energy_meV_per_atom_rms"]
    assert after["force_meV_per_A_rms"] < 0.5 * before["force_meV_per_A_rms"]

    # and it is cheaper than the teacher on the same structures
    big = water.water_batch(64, seed=41, n_min=128, n_max=512)
    pos = np.concatenate([s.positions for s in big])

    def timed(mode):
        b = mode.batch(big)
        b.setPositions(pos)
        for _ in range(2):   # sizes the lists, tunes the kernel shapes and records the graph
            b.evaluate(forces=True)
        b.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            b.evaluate(forces=True)
        b.synchronize()
        return (time.perf_counter() - t0) / 3
    assert timed(m) < 0.7 * timed(teacher)


def test_fallback_on_extrapolation(teacher, student_dir):
    held = student.training_structures(6, seed=51, n_min=32, n_max=64)
    # compress one box by 15 %: its symmetry functions leave the scaling range
    s = held[2]
    s.positions = s.positions * 0.85
    s.box = s.box * 0.85
    m = student.load_mode(student_dir, extrapolation=True)
    ev = student.StudentEvaluator(m, teacher, held, monitor=2, seed=0)
    E, F, flagged = ev.evaluate()
    assert flagged[2]
    Et, Ft = student.label(teacher, [held[2]])
    assert E[2] == Et[0]
    a0 = sum(x.numAtoms for x in held[:2])
    assert np.array_equal(F[a0:a0 + held[2].numAtoms], Ft)
    assert 0 < ev.fallback_rate() <= 1
    assert len(ev.monitor_log) == 1 and ev.monitor_log[0]["energy_meV_per_atom_rms"] >= 0


def test_force_contributions_sum_to_forces(teacher):
    """The per-atom force contributions the descriptor selection spans
    (dE_i/dG_is dG_is/dr_k over each atom and its neighbours) add up to the
    teacher's forces."""
    structs = student.training_structures(2, seed=9, n_min=32, n_max=48)
    b = teacher.batch(structs)
    b.setPositions(np.concatenate([s.positions for s in structs]))
    b.evaluate(forces=True, storeDGdr=True, graph=False)
    nb = b.neighbors()
    off = nb["offset"]
    F = np.zeros((b.numAtoms, 3))
    for i, g in enumerate(student._contribution_vectors(teacher, b, b.dEdG())):
        F[i] += g[0]
        np.add.at(F, nb["index"][off[i]:off[i + 1]], g[1:])
    ref = b.forces()
    assert np.abs(-F - ref).max() <= 1e-10 * np.abs(ref).max()
    b.close()


def test_force_span_selection(teacher, tmp_path):
    """Descriptor selection from the candidate grid: the per-element budget
    of radial and angular functions, a residual that falls with each choice,
    and a chosen set that spans the teacher's force contributions better than
    the fixed default set does."""
    sample = student.training_structures(3, seed=12, n_min=32, n_max=48)
    lines, rep = student.select_by_force_span(teacher, sample, str(tmp_path / "cand"))
    for sym in ("H", "O"):
        mine = [l.split() for l in lines if l.split()[1] == sym]
        assert sum(p[2] == "2" for p in mine) == 8 and sum(p[2] == "3" for p in mine) == 6
        tr = rep[sym]["residual_after_each_choice"]
        assert len(tr) == 14 and all(a >= b - 1e-12 for a, b in zip(tr, tr[1:]))
        assert rep[sym]["residual_all_candidates"] <= tr[-1] < 1.0
    # the fixed set's residual on the same sample, through a candidate model of its own functions
    fixed = str(tmp_path / "fixed")
    student.write_student_model(fixed, sample, sf_lines=student.student_sf_lines())
    fm = student.load_mode(fixed)
    stats = student.force_span_statistics(teacher, fm, sample)
    for e, sym in enumerate(("H", "O")):
        M, B, c = stats[e]
        fixed_res = student.span_residual(M, B, c, range(M.shape[1])) / float(c.sum())
        assert rep[sym]["residual_after_each_choice"][-1] < fixed_res
    fm.close()
