"""The C-ABI library builds for sm_100a, loads without a GPU and exports every
entry point that include/n2p2_b200.h declares (no compute calls)."""
import ctypes
import os
import re

from n2p2_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "n2p2_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(n2p2_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n
    # the Python declarations cover the same set
    assert set(names) == set(_lib.SIGNATURES)


def test_version_and_error_strings_without_gpu():
    lib = _lib.load()
    assert b"sm_100a" in lib.n2p2_version()
    assert isinstance(lib.n2p2_last_error(), bytes)


def test_null_handles_are_rejected():
    lib = _lib.load()
    assert lib.n2p2_mode_setup_generic(None) == _lib.ERR_NULL
    assert lib.n2p2_batch_evaluate(None, 1) == _lib.ERR_NULL
    assert b"null" in lib.n2p2_last_error()
