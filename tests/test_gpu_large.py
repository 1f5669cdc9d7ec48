"""The large single-system configuration: a 36,864-molecule water box
(110,592 atoms, 1.0 g/cm^3, 0.15 bohr displacements) with the 56-function
model (G2 + narrow G3 + wide G9, 56-64-64-1 softplus).

The reference library cannot evaluate 110k atoms within a test, so the full
size is checked through properties that hold exactly in exact arithmetic --
zero net force, translation invariance, and additivity under periodic
replication of a smaller box -- while a 512-molecule box of the same recipe
is compared with the reference directly."""
import numpy as np
import pytest

from n2p2_b200 import Structure, water
from tests import helpers as H
from tests.test_gpu_parity import TOL_E, _compare_structure

pytestmark = pytest.mark.gpu

LARGE_MOLECULES = 36864


@pytest.fixture(scope="module")
def large():
    return water.water_box(LARGE_MOLECULES, seed=2024, sigma=0.15)


@pytest.fixture(scope="module")
def mode56():
    return H.gpu_mode(H.WATER56)


def _replicate(s, n=2):
    L = np.diag(s.box)
    pos, el = [], []
    for a in range(n):
        for b in range(n):
            for c in range(n):
                pos.append(s.positions + np.array([a, b, c]) * L)
                el += s.elements
    return Structure(np.concatenate(pos), el, box=s.box * n)


def test_water56_box512_matches_reference(mode56):
    s = water.water_box(512, seed=3, sigma=0.15)
    b = H.gpu_batch(mode56, [s])
    snap = H.reference_snapshot(H.WATER56, s)
    _compare_structure(b, 0, s.numAtoms, snap, 0, b.energies(), b.forces())
    assert H.max_rel(b.atomicEnergies(), snap["atomic_energy"]) <= TOL_E


def test_large_fp64_invariances(mode56, large):
    assert large.numAtoms == 3 * LARGE_MOLECULES
    b = H.gpu_batch(mode56, [large])
    E0, F0 = b.energies()[0], b.forces()
    # Newton's third law: the pair contributions cancel
    assert np.abs(F0.sum(axis=0)).max() <= 1e-10 * np.abs(F0).sum()
    # rigid translation (atoms are re-folded into the cell)
    shifted = Structure(large.positions + np.array([0.37, -1.13, 2.29]), large.elements, box=large.box)
    b2 = H.gpu_batch(mode56, [shifted])
    assert abs(b2.energies()[0] - E0) <= 1e-11 * abs(E0)
    assert H.max_rel(b2.forces(), F0) <= 1e-9


def test_large_periodic_replication(mode56):
    cell = water.water_box(LARGE_MOLECULES // 8, seed=77, sigma=0.15)
    big = _replicate(cell, 2)
    assert big.numAtoms == 3 * LARGE_MOLECULES
    bc = H.gpu_batch(mode56, [cell])
    bb = H.gpu_batch(mode56, [big])
    assert abs(bb.energies()[0] - 8 * bc.energies()[0]) <= 1e-11 * abs(bb.energies()[0])
    Fc = bc.forces()
    assert H.max_rel(bb.forces(), np.tile(Fc, (8, 1))) <= 1e-9


def test_large_mixed_within_budget(large):
    m64 = H.gpu_mode(H.WATER56)
    b64 = H.gpu_batch(m64, [large])
    mm = H.gpu_mode(H.WATER56, precision="mixed")
    bm = H.gpu_batch(mm, [large])
    de = abs(bm.energies()[0] - b64.energies()[0]) / large.numAtoms * H.HA_TO_MEV
    df = np.abs(bm.forces() - b64.forces()).max() * H.HA_PER_BOHR_TO_MEV_PER_A
    assert de <= 1.0
    assert df <= 30.0
