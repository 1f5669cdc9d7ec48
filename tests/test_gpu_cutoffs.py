"""Angular groups with a smaller cutoff than the neighbour list's: the stage
is sorted by distance and the groups enumerate only the neighbours inside
their cutoff.  FP64 energies and forces against the CPU oracle, mixed form
within its budget."""
import numpy as np
import pytest

from n2p2_b200 import student
from tests import helpers as H

pytestmark = pytest.mark.gpu


def test_smaller_angular_cutoff_matches_oracle(tmp_path):
    from oracle.port import PortModel
    d = str(tmp_path / "model")
    lines = student.student_sf_lines(rc=12.0, rc_angular=7.0)
    structs = student.training_structures(6, seed=61, n_min=32, n_max=96)
    student.write_student_model(d, structs, seed=4, sf_lines=lines)
    m = student.load_mode(d)
    b = H.gpu_batch(m, structs)
    E, F = b.energies(), b.forces()
    pm = PortModel(d)
    a0 = 0
    for k, s in enumerate(structs[:3]):
        r = pm.evaluate(s)
        assert abs(E[k] - r["energy"]) <= 1e-10 * abs(r["energy"])
        assert H.max_rel(F[a0:a0 + s.numAtoms], r["forces"]) <= 1e-10
        a0 += s.numAtoms
    mm = student.load_mode(d, precision="mixed")
    bm = H.gpu_batch(mm, structs)
    apa = np.array([s.numAtoms for s in structs])
    assert (np.abs(bm.energies() - E) / apa * H.HA_TO_MEV).max() <= 1.0
    assert (np.abs(bm.forces() - F) * H.HA_PER_BOHR_TO_MEV_PER_A).max() <= 30.0
