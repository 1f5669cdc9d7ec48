"""LAMMPS interface on the GPU against the reference's own InterfaceLammps
(oracle/_ref/libnnplammps.so), both driven as pair_style hdnnp drives them on
one rank: local atoms wrapped into a periodic water box, ghost images around
it, full neighbour lists with a skin, Angstrom / eV units.

Tolerances: energies within 1e-10 relative, atomic energies and the forces on
every local and ghost atom within 1e-10 of the largest force component (the
plain-FP64 target); the mixed form within the 1 meV/atom and 30 meV/A
budget; the ghost forces folded back to their owners reproduce the periodic
batch path."""
import numpy as np
import pytest

from n2p2_b200 import Structure, water
from n2p2_b200.lammps import InterfaceLammps
from oracle import lammps_ref
from tests import helpers as H

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not lammps_ref.available(), reason="reference LAMMPS interface not built")]

A_TO_BOHR = 1.0 / H.BOHR_TO_A
EV_TO_HA = 1.0 / H.HA_TO_EV
PAIR_CUT_A = 6.5                      # pair_style cutoff (>= 12 bohr = 6.35 A)
LIST_CUT_A = PAIR_CUT_A + 1.0         # plus the neighbour skin
TYPES = {"H": 1, "O": 2}


def _domain(s, type_of=TYPES):
    return H.lammps_domain(s, LIST_CUT_A * A_TO_BOHR, type_of, length=H.BOHR_TO_A)


def _ours(model, dom, emap="1:H,2:O", ntypes=2, precision="fp64", lmp=None):
    if lmp is None:
        lmp = InterfaceLammps().initialize(model, emap, False, False, 0, -1, A_TO_BOHR, EV_TO_HA, PAIR_CUT_A,
                                           ntypes, 0)
        lmp.setPrecision(precision)
    n = dom["nlocal"]
    lmp.setLocalAtoms(n, dom["type"][:n])
    lmp.transferNeighborList(dom["ilist"], dom["numneigh"], dom["firstneigh"], dom["x"], dom["type"], PAIR_CUT_A)
    lmp.process()
    F = np.zeros((len(dom["x"]), 3))
    lmp.getForces(F)
    return lmp, lmp.getEnergy(), F


def _reference(model, dom, emap="1:H,2:O", ntypes=2, mapped=(1, 2)):
    ref = lammps_ref.RefInterfaceLammps(model, emap, A_TO_BOHR, EV_TO_HA, PAIR_CUT_A, ntypes)
    e = H.pair_style_entries(dom, PAIR_CUT_A)
    local = dom["type"][:dom["nlocal"]]
    out = ref.evaluate(local, e["offset"], e["j"], e["type"], e["dr"], e["d2"], len(dom["x"]),
                       num_centres=int(np.isin(local, mapped).sum()))
    ref.close()
    return out


@pytest.mark.parametrize("model,nmol", [(H.WATER40, 64), (H.WATER56, 96)], ids=["water40", "water56"])
def test_matches_reference_interface(model, nmol):
    s = water.water_box(nmol, seed=3, sigma=0.1)
    dom = _domain(s)
    E_ref, Ea_ref, F_ref = _reference(model, dom)
    lmp, E, F = _ours(model, dom)
    assert abs(E - E_ref) <= 1e-10 * abs(E_ref)
    Ea = np.array([lmp.getAtomicEnergy(i) for i in range(dom["nlocal"])])
    assert np.abs(Ea - Ea_ref).max() <= 1e-10 * np.abs(Ea_ref).max()
    scale = np.abs(F_ref).max()
    assert np.abs(F - F_ref).max() <= 1e-10 * scale
    assert np.abs(F[dom["nlocal"]:]).max() > 1e-3 * scale      # ghosts do receive forces
    # the same lists through addNeighbor one entry at a time: bitwise the same
    e = H.pair_style_entries(dom, PAIR_CUT_A)
    lmp.setLocalAtoms(dom["nlocal"], dom["type"][:dom["nlocal"]])
    for i in range(dom["nlocal"]):
        for q in range(e["offset"][i], e["offset"][i + 1]):
            lmp.addNeighbor(i, e["j"][q], e["j"][q] + 1, e["type"][q], *e["dr"][q], e["d2"][q])
    lmp.process()
    F2 = np.zeros_like(F)
    lmp.getForces(F2)
    assert lmp.getEnergy() == E and np.array_equal(F2, F)
    lmp.close()


def test_folded_forces_match_the_periodic_batch():
    s = water.water_box(64, seed=4, sigma=0.1)
    dom = _domain(s)
    lmp, E, F = _ours(H.WATER40, dom)
    folded = np.zeros((dom["nlocal"], 3))
    np.add.at(folded, dom["owner"], F)
    m = H.gpu_mode(H.WATER40)
    b = H.gpu_batch(m, [s])
    E_b = b.energies()[0] * H.HA_TO_EV
    F_b = b.forces() * H.HA_TO_EV / H.BOHR_TO_A
    assert abs(E - E_b) <= 1e-10 * abs(E_b)
    assert np.abs(folded - F_b).max() <= 1e-10 * np.abs(F_b).max()
    lmp.close()


def test_type_map_with_ignored_type():
    """Types swapped by the map and a third LAMMPS type the model does not
    know (its atoms are neither centres nor neighbours), as in the reference."""
    s = water.water_box(64, seed=5, sigma=0.1)
    dom = _domain(s, {"H": 2, "O": 1})
    extra = np.arange(0, dom["nlocal"], 17)          # relabel some local atoms (and their images) as type 3
    relabel = np.isin(dom["owner"], extra)
    dom["type"] = np.where(relabel, 3, dom["type"]).astype(np.int32)
    E_ref, Ea_ref, F_ref = _reference(H.WATER40, dom, emap="2:H,1:O", ntypes=3)
    lmp, E, F = _ours(H.WATER40, dom, emap="2:H,1:O", ntypes=3)
    assert abs(E - E_ref) <= 1e-10 * abs(E_ref)
    assert np.abs(F - F_ref).max() <= 1e-10 * np.abs(F_ref).max()
    Ea = np.array([lmp.getAtomicEnergy(i) for i in range(Ea_ref.size)])
    assert np.abs(Ea - Ea_ref).max() <= 1e-10 * np.abs(Ea_ref).max()
    assert np.all(F[relabel] == 0.0)
    lmp.close()


def test_md_steps_reuse_the_interface():
    """Several steps with moving atoms on one interface (new lists every
    step), each against the reference; repeating a step is bitwise stable."""
    s = water.water_box(64, seed=6, sigma=0.1)
    rng = np.random.default_rng(0)
    lmp = None
    for step in range(3):
        pos = s.positions + rng.normal(scale=0.02, size=s.positions.shape)
        st = Structure(pos, s.elements, box=s.box)
        dom = _domain(st)
        E_ref, _, F_ref = _reference(H.WATER40, dom)
        lmp, E, F = _ours(H.WATER40, dom, lmp=lmp)
        assert abs(E - E_ref) <= 1e-10 * abs(E_ref)
        assert np.abs(F - F_ref).max() <= 1e-10 * np.abs(F_ref).max()
    _, E2, F2 = _ours(H.WATER40, dom, lmp=lmp)
    assert E2 == E and np.array_equal(F2, F)
    lmp.close()


def test_mixed_precision_within_budget():
    s = water.water_box(64, seed=7, sigma=0.1)
    dom = _domain(s)
    lmp64, E64, F64 = _ours(H.WATER40, dom)
    lmpm, Em, Fm = _ours(H.WATER40, dom, precision="mixed")
    assert abs(Em - E64) / dom["nlocal"] * 1e3 <= 1.0          # meV/atom
    assert np.abs(Fm - F64).max() * 1e3 <= 30.0                 # meV/A
    lmp64.close()
    lmpm.close()


def test_extrapolation_warnings_counted_like_the_reference():
    """A compressed box leaves the scaling range: the warning count of the
    last step equals the reference's."""
    s = water.water_box(64, seed=8, sigma=0.05)
    s = Structure(s.positions * 0.93, s.elements, box=s.box * 0.93)
    dom = _domain(s)
    ref = lammps_ref.RefInterfaceLammps(H.WATER40, "1:H,2:O", A_TO_BOHR, EV_TO_HA, PAIR_CUT_A, 2, showew=True)
    e = H.pair_style_entries(dom, PAIR_CUT_A)
    ref.evaluate(dom["type"][:dom["nlocal"]], e["offset"], e["j"], e["type"], e["dr"], e["d2"], len(dom["x"]))
    n_ref = ref.num_extrapolation_warnings()
    ref.close()
    lmp = InterfaceLammps().initialize(H.WATER40, "1:H,2:O", True, False, 0, -1, A_TO_BOHR, EV_TO_HA, PAIR_CUT_A,
                                       2, 0)
    _ours(H.WATER40, dom, lmp=lmp)
    assert n_ref > 0 and lmp.getNumExtrapolationWarnings() == n_ref
    lmp.clearExtrapolationWarnings()
    assert lmp.getNumExtrapolationWarnings() == 0
    lmp.close()
