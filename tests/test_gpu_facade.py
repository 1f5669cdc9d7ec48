"""The C++ facade (include/n2p2_b200_mode.hpp) driven like nnp-predict:
evaluateNNP and the separate stages on the reference's Cu2S_PBE prediction
example (G2/G3/G9, poly2, softplus, sigma scaling, normalised units) give the
energy and forces of the reference's regression test within 1e-10
(relative; forces relative to the largest component), G within 1e-12 and
dE/dG within 1e-10 of the reference library, and the neighbour counts of its
lists; both routes give the same bits."""
import json
import os
import subprocess

import numpy as np
import pytest

from n2p2_b200 import read_structures
from tests import helpers as H
from tests.test_cpu_facade import build_facade_driver

pytestmark = pytest.mark.gpu


def test_facade_predict_matches_reference(tmp_path):
    exe = build_facade_driver(tmp_path)
    d = os.path.join(H.GOLDEN, "examples", "Cu2S_PBE")
    r = subprocess.run([exe, "predict", d], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    gold = json.load(open(os.path.join(d, "golden.json")))
    F = np.array(out["forces"]).reshape(-1, 3)
    assert abs(out["energy"] - gold["energy"]) <= 1e-10 * abs(gold["energy"])
    assert H.max_rel(F, np.array(gold["forces"])) <= 1e-10
    # the stages one by one: the same bits
    assert np.array(out["energy_stages"]).view(np.int64) == np.array(out["energy"]).view(np.int64)
    assert np.array_equal(np.array(out["forces_stages"]).view(np.int64), np.array(out["forces"]).view(np.int64))
    assert out["energy_again"] == out["energy"]
    s = read_structures(os.path.join(d, "input.data"))[0]
    snap = H.reference_snapshot(d, s)
    assert H.max_rel(H.unscaled(d, s, np.array(out["G"])), H.unscaled(d, s, snap["G"])) <= 1e-12
    assert H.max_rel(np.array(out["dEdG"]), snap["dEdG"]) <= 1e-10
    assert np.array_equal(np.array(out["num_neighbors"], dtype=np.int64), np.diff(snap["nbr_offset"]))
    # an atom moved after an evaluation: recomputed, as a fresh reference prediction of the moved structure
    s.positions[0, 0] += 0.01
    moved = H.reference_snapshot(d, s)
    assert moved["energy"] != snap["energy"]
    assert abs(out["energy_moved"] - moved["energy"]) <= 1e-10 * abs(moved["energy"])
