"""Host-side pieces of the student recipe without a GPU: the force-span
descriptor selection (Gram-statistics residual and greedy choice), the
per-neighbour derivative tables it reads dG/dr through, and the candidate
descriptor grid."""
import os

import numpy as np
import pytest

from n2p2_b200 import student, water
from n2p2_b200.mode import Mode
from oracle import port
from tests import helpers as H


def _synthetic(rng, atoms=40, dim=30, cols=10, gen=(1, 4, 7)):
    V = rng.normal(size=(atoms, dim, cols))
    a = rng.normal(size=(atoms, len(gen)))
    f = np.einsum("adk,ak->ad", V[:, :, list(gen)], a)
    M = np.einsum("adi,adj->aij", V, V)
    B = np.einsum("adi,ad->ai", V, f)
    c = np.einsum("ad,ad->a", f, f)
    return V, f, M, B, c


def test_span_residual_equals_least_squares():
    rng = np.random.default_rng(3)
    V, f, M, B, c = _synthetic(rng)
    S = [0, 2, 5]
    direct = sum(np.sum((f[i] - V[i][:, S] @ np.linalg.lstsq(V[i][:, S], f[i], rcond=None)[0]) ** 2)
                 for i in range(len(f)))
    assert abs(student.span_residual(M, B, c, S, ridge=0.0) - direct) <= 1e-9 * c.sum()
    assert student.span_residual(M, B, c, []) == pytest.approx(c.sum())


def test_greedy_selection_finds_generating_columns_within_type_budget():
    rng = np.random.default_rng(4)
    _, _, M, B, c = _synthetic(rng, gen=(1, 4, 7))
    types = [2, 2, 2, 2, 3, 3, 3, 3, 3, 3]
    chosen, trace = student.greedy_span_selection(M, B, c, types, {2: 1, 3: 2})
    assert sorted(chosen) == [1, 4, 7]
    assert trace[-1] < 1e-8 and all(a >= b for a, b in zip(trace, trace[1:]))
    chosen, _ = student.greedy_span_selection(M, B, c, types, {2: 2, 3: 1})
    assert sum(types[j] == 2 for j in chosen) == 2 and sum(types[j] == 3 for j in chosen) == 1


@pytest.mark.skipif(not port.available(), reason="C restatement not built")
@pytest.mark.parametrize("model", [H.WATER56, os.path.join(H.GOLDEN, "examples", "Cu2S_PBE")])
def test_derivative_tables_match_restatement(model):
    """Row order of the per-neighbour dG/dr (ascending function index per
    neighbour element) equals the oracle's table."""
    m = Mode(0)
    m.setupFromDirectory(model)
    pm = port.PortModel(model)
    tab = student._derivative_tables(m)
    rowSF = pm.arrays["rowSF"].reshape(m.numElements, m.numElements, -1)
    for e in range(m.numElements):
        for en in range(m.numElements):
            assert len(tab[e][en]) == m.numDerivativeRows(e, en)
            assert tab[e][en] == list(rowSF[e, en, :len(tab[e][en])])
    m.close()


def test_candidate_grid_is_a_valid_descriptor(tmp_path):
    t = Mode(0)
    t.setupFromDirectory(H.WATER56)
    lines = student.candidate_sf_lines(t, rc_angular=8.0)
    assert len(lines) == len(set(lines))
    d = str(tmp_path)
    with open(os.path.join(d, "input.nn"), "w") as f:
        f.write(water.input_nn_text(lines, nodes=(4, 4), scaling=False))
    m = Mode(0)
    m.initialize()
    m.loadSettingsFile(os.path.join(d, "input.nn"))
    m.setupGeneric()
    for e in range(2):
        sfs = [m.symmetryFunction(e, i) for i in range(m.numSymmetryFunctions(e))]
        assert sum(f[0] == 2 for f in sfs) == 16 + 4          # teacher's radial + 2 widths x 2 neighbours
        assert sum(f[0] == 3 for f in sfs) == 3 * 4 * 4 * 2   # pairs x eta x zeta x lambda
        assert all(f[7] == 8.0 for f in sfs if f[0] == 3)
    m.close()
    t.close()


def test_gaussian_plan_and_specialised_admissibility():
    """The selection's copy of the engine's Gaussian plan, and the group rules
    of the model-specialised kernels it keeps the chosen set within."""
    assert student.gaussian_bases([0.001, 0.01, 0.03, 0.06, 0.15, 0.3, 0.6, 1.5]) == [0.001, 0.03, 0.6, 1.5]
    assert student.gaussian_bases([0.03, 0.01]) == [0.01]
    assert student.gaussian_bases([0.001, 0.03]) == [0.001, 0.03]        # ratio 30 > 16
    # (type, e1, e2, eta, rs, lambda, zeta, rc, scaling)
    ang = lambda eta, lam, zeta, e1=0, e2=1, rc=12.0: (3, e1, e2, eta, 0.0, lam, zeta, rc, 1.0)
    rad = lambda eta, e1=0: (2, e1, e1, eta, 0.0, 0.0, 0.0, 12.0, 1.0)
    sfs = [ang(0.01, 1, 1), ang(0.03, -1, 4), ang(0.001, 1, 1), ang(0.003, 1, 2), ang(0.001, 1, 1, e1=1),
           rad(0.001), rad(0.03), rad(0.6), rad(1.5), rad(1.0), rad(3.0)]
    ok = student.specialised_kernel_admissible(sfs)
    assert ok([0], 1)              # widths 0.01, 0.03 share a base
    assert not ok([0, 1], 2)       # a third width
    assert not ok([0], 3)          # 0.01 and 0.003: two bases
    assert ok([0, 1], 4)           # another element pair is another group
    assert ok([5, 6, 7], 8)        # four radial bases
    assert not ok([5, 6, 7, 8], 9)  # a fifth
    assert ok([5, 6, 7, 8], 10)    # 3.0 = 2 x 1.5: shares the last base
