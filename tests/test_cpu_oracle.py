"""The CPU oracles, pinned before they are trusted.

* oracle/_ref/libnnpref.so (the reference library built from its own
  sources) reproduces the reference's regression goldens
  (test/cpp/ExamplePrediction.h) to the reference test's 1000 eps.
* oracle/nnp_oracle.c (the C restatement) reproduces the cutoff-function
  known answers of test/cpp/test_CutoffFunction.cpp to 100 eps and matches
  the reference library bit for bit on neighbour lists, remapped positions, G
  and energies, forces to 1e-13 relative.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from n2p2_b200 import read_structures, water
from oracle import port, ref
from tests import helpers as H

EPS = np.finfo(np.float64).eps
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference library not built (oracle/Makefile)")
needs_port = pytest.mark.skipif(not port.available(), reason="C restatement not built (oracle/Makefile)")


@needs_ref
@pytest.mark.parametrize("name", ["H2O_RPBE-D3", "Cu2S_PBE"])
def test_reference_build_reproduces_goldens(name):
    d = os.path.join(H.GOLDEN, "examples", name)
    gold = json.load(open(os.path.join(d, "golden.json")))
    s = read_structures(os.path.join(d, "input.data"))[0]
    a = H.reference_snapshot(d, s)
    assert abs(a["energy"] - gold["energy"]) <= 1000 * EPS
    assert np.abs(a["forces"] - np.array(gold["forces"])).max() <= 1000 * EPS


@needs_port
def test_port_cutoff_functions_known_answers():
    g = json.load(open(os.path.join(H.GOLDEN, "cutoff_functions.json")))
    lib = ctypes.CDLL(port.LIB)
    lib.oracle_cutoff.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    for t, f_ref, df_ref in zip(g["types"], g["f"], g["df"]):
        f, df = ctypes.c_double(), ctypes.c_double()
        lib.oracle_cutoff(t, g["alpha"], g["rc"], g["r"], ctypes.byref(f), ctypes.byref(df))
        assert abs(f.value - f_ref) <= 100 * EPS, t
        assert abs(df.value - df_ref) <= 100 * EPS, t
        lib.oracle_cutoff(t, g["alpha"], g["rc"], g["rc"], ctypes.byref(f), ctypes.byref(df))
        assert f.value == 0.0 and df.value == 0.0


def _structures():
    out = []
    for name in ["H2O_RPBE-D3", "Cu2S_PBE"]:
        d = os.path.join(H.GOLDEN, "examples", name)
        out.append((d, read_structures(os.path.join(d, "input.data"))[0]))
    out.append((H.WATER40, water.water_box(64, seed=0)))
    out.append((H.WATER40, water.water_batch(1, seed=3, n_min=90, n_max=90)[0]))
    return out


@needs_ref
@needs_port
@pytest.mark.parametrize("case", range(4))
def test_port_matches_reference_library(case):
    d, s = _structures()[case]
    a = H.reference_snapshot(d, s)
    o = port.PortModel(d).evaluate(s)
    assert np.array_equal(o["nbr_offset"], a["nbr_offset"])
    assert np.array_equal(o["nbr_index"], a["nbr_index"])
    assert np.array_equal(o["nbr_d"].view(np.int64), a["nbr_d"].view(np.int64))
    assert np.array_equal(o["nbr_dr"].view(np.int64), a["nbr_dr"].view(np.int64))
    assert np.array_equal(o["positions"].view(np.int64), a["positions"].view(np.int64))
    assert np.array_equal(o["G"].view(np.int64), a["G"].view(np.int64))
    assert o["energy"] == a["energy"]
    assert H.max_rel(o["forces"], a["forces"]) <= 1e-13


def test_reference_nnp_train_reproduces_its_regression_values(tmp_path):
    """The reference's nnp-train built here from its own sources
    (oracle/_ref/nnp-train: one process, stand-ins for MPI, GSL's generators
    and Eigen's Kalman-filter operations) reproduces the learning curve its
    regression test asserts for H2O_RPBE-D3 (test/cpp/Example_nnp_train.h,
    1e-8 absolute): the oracle of the training driver is pinned."""
    import json
    import shutil
    import subprocess
    exe = os.path.join(H.ROOT, "oracle", "_ref", "nnp-train")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/nnp-train not built (needs the reference sources)")
    d = os.path.join(H.GOLDEN, "training", "H2O_RPBE-D3")
    for fn in ("input.nn", "scaling.data", "input.data"):
        shutil.copy(os.path.join(d, fn), tmp_path)
    subprocess.run([exe], cwd=tmp_path, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    g = json.load(open(os.path.join(d, "golden.json")))
    rows = {}
    for line in open(tmp_path / "learning-curve.out"):
        c = line.split()
        if c and not c[0].startswith("#"):
            rows[int(c[0])] = [float(c[1]), float(c[2]), float(c[9]), float(c[10])]
    last = rows[g["last_epoch"]]
    want = [g["rmse_energy_train"], g["rmse_energy_test"], g["rmse_forces_train"], g["rmse_forces_test"]]
    for a, b in zip(last, want):
        assert abs(a - b) <= g["accuracy"], (last, want)
