"""The header-only C++ facade of nnp::Mode / nnp::Structure
(include/n2p2_b200_mode.hpp) compiles as C++11 against the C ABI and maps
the library's status codes to the reference's exception types; no GPU (the
set-up half of the API runs on the host)."""
import os
import shutil
import subprocess

import pytest

from tests import helpers as H

ROOT = H.ROOT


def build_facade_driver(out_dir):
    """g++ the facade test driver (tests/cpp/facade_predict.cpp) against the
    in-tree library; returns the executable's path."""
    from n2p2_b200 import _lib
    lib = _lib.load()  # noqa: F841  (the library must exist)
    exe = os.path.join(str(out_dir), "facade_predict")
    libdir = os.path.join(ROOT, "n2p2_b200")
    subprocess.run(["g++", "-std=c++11", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_predict.cpp"), "-o", exe, "-L", libdir, "-ln2p2b200",
                    "-Wl,-rpath," + libdir], check=True)
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_facade_compiles_and_maps_errors(tmp_path):
    exe = build_facade_driver(tmp_path)
    d = os.path.join(H.GOLDEN, "examples", "Cu2S_PBE")
    r = subprocess.run([exe, "errors", d], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    import json
    out = json.loads(r.stdout)
    assert out["numAtoms"] == 144 and out["failures"] == 0
