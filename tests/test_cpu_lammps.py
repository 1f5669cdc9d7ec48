"""LAMMPS interface set-up without a GPU: for the same arguments,
n2p2_lammps_initialize succeeds or fails exactly where the reference's own
InterfaceLammps::initialize (InterfaceLammps.cpp:51-255, oracle/_ref/
libnnplammps.so) does, with the same message, and reports the largest cutoff
in LAMMPS units."""
import pytest

from n2p2_b200.lammps import InterfaceLammps
from oracle import lammps_ref
from tests import helpers as H

pytestmark = pytest.mark.skipif(not lammps_ref.available(), reason="reference LAMMPS interface not built")

A_TO_BOHR = 1.0 / H.BOHR_TO_A
EV_TO_HA = 1.0 / H.HA_TO_EV

CASES = [
    # emap, cflength, lammps cutoff, LAMMPS types, same message expected
    ("1:H,2:O", 1.0, 12.0, 2, True),
    ("2:H, 1:O", A_TO_BOHR, 6.5, 2, True),            # blanks removed, types swapped, Angstrom
    ("1:H,2:O", 1.0, 11.9, 2, True),                  # cutoff below the symmetry functions'
    ("", 1.0, 12.0, 2, True),                         # default map
    ("", 1.0, 12.0, 3, True),                         # default map needs one type per element
    ("1:H,2:O,3:H", 1.0, 12.0, 3, True),              # more pairs than elements
    ("1=H", 1.0, 12.0, 2, True),                      # not type:element
    ("3:H", 1.0, 12.0, 2, True),                      # type beyond the LAMMPS types
    ("1:H", 1.0, 12.0, 3, True),                      # types 2, 3 ignored
    ("1:C", 1.0, 12.0, 2, False),                     # unknown element: both refuse
]


@pytest.mark.parametrize("emap,cfl,cut,ntypes,same", CASES)
def test_initialize_agrees_with_reference(emap, cfl, cut, ntypes, same):
    ref_err = None
    try:
        ref = lammps_ref.RefInterfaceLammps(H.WATER40, emap, cfl, EV_TO_HA, cut, ntypes)
        ref.close()
    except RuntimeError as e:
        ref_err = str(e)
    lmp = InterfaceLammps()
    err = None
    try:
        lmp.initialize(H.WATER40, emap, False, False, 0, -1, cfl, EV_TO_HA, cut, ntypes, 0)
    except Exception as e:
        err = str(e)
    assert (err is None) == (ref_err is None), (err, ref_err)
    if err is None:
        assert lmp.getMaxCutoffRadius() == pytest.approx(12.0 / cfl, rel=1e-15)
    elif same:
        assert err.strip().splitlines()[0] in ref_err, (err, ref_err)
    lmp.close()


def test_initialize_twice_is_refused():
    lmp = InterfaceLammps().initialize(H.WATER40, "1:H,2:O", False, False, 0, -1, 1.0, 1.0, 12.0, 2, 0)
    with pytest.raises(Exception, match="already initialized"):
        lmp.initialize(H.WATER40, "1:H,2:O", False, False, 0, -1, 1.0, 1.0, 12.0, 2, 0)
    lmp.close()


def test_local_atoms_and_neighbours_checked_on_the_host():
    lmp = InterfaceLammps().initialize(H.WATER40, "1:H", False, False, 0, -1, 1.0, 1.0, 12.0, 3, 0)
    lmp.setLocalAtoms(3, [1, 2, 3])
    with pytest.raises(Exception, match="type out of range"):
        lmp.setLocalAtoms(2, [1, 4])
    lmp.setLocalAtoms(3, [1, 2, 3])
    lmp.addNeighbor(0, 5, 6, 1, 1.0, 0.0, 0.0, 1.0)     # mapped pair
    lmp.addNeighbor(1, 5, 6, 1, 1.0, 0.0, 0.0, 1.0)     # centre of an ignored type: dropped
    lmp.addNeighbor(0, 6, 7, 2, 1.0, 0.0, 0.0, 1.0)     # neighbour of an ignored type: dropped
    with pytest.raises(Exception, match="local atom index out of range"):
        lmp.addNeighbor(3, 5, 6, 1, 1.0, 0.0, 0.0, 1.0)
    lmp.close()
