"""ctypes wrapper of oracle/_ref/libnnpref*.so (the reference n2p2 library built
from its own sources plus ref_harness.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline legs.  The product never imports this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def lib_path(fast=False):
    return os.path.join(_HERE, "_ref", "libnnpref_fast.so" if fast else "libnnpref.so")


def available(fast=False):
    return os.path.exists(lib_path(fast))


def _lib(fast=False):
    key = bool(fast)
    if key in _LIBS:
        return _LIBS[key]
    lib = ctypes.CDLL(lib_path(fast))
    vp, i64, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
    lib.nnpref_create.restype = vp
    lib.nnpref_create.argtypes = [ctypes.c_char_p, ctypes.c_int]
    lib.nnpref_destroy.argtypes = [vp]
    lib.nnpref_last_error.restype = ctypes.c_char_p
    for n in ("num_elements",):
        getattr(lib, "nnpref_" + n).restype = i64
        getattr(lib, "nnpref_" + n).argtypes = [vp]
    lib.nnpref_num_sf.restype = i64
    lib.nnpref_num_sf.argtypes = [vp, i64]
    lib.nnpref_num_rows.restype = i64
    lib.nnpref_num_rows.argtypes = [vp, i64, i64]
    lib.nnpref_max_cutoff.restype = dbl
    lib.nnpref_max_cutoff.argtypes = [vp]
    lib.nnpref_predict.restype = ctypes.c_int
    lib.nnpref_predict.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    lib.nnpref_energy.restype = dbl
    lib.nnpref_energy.argtypes = [vp]
    lib.nnpref_energy_internal.restype = dbl
    lib.nnpref_energy_internal.argtypes = [vp]
    for n in ("forces", "forces_internal", "positions", "box", "nbr_d", "nbr_dr", "G", "dEdG",
              "dGdr_self", "dGdr_nbr", "atomic_energy"):
        f = getattr(lib, "nnpref_" + n)
        f.restype = i64
        f.argtypes = [vp, ctypes.POINTER(dbl), i64]
    for n in ("nbr_offset", "nbr_index", "sf_offset", "row_offset"):
        f = getattr(lib, "nnpref_" + n)
        f.restype = i64
        f.argtypes = [vp, ctypes.POINTER(i64), i64]
    lib.nnpref_jacobian.restype = i64
    lib.nnpref_jacobian.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, i64, ctypes.c_int, ctypes.POINTER(dbl), i64]
    lib.nnpref_loss_gradient.restype = i64
    lib.nnpref_loss_gradient.argtypes = [vp, ctypes.c_char_p, dbl, ctypes.POINTER(dbl), ctypes.POINTER(dbl), i64]
    lib.nnpref_time_sf_batch.restype = dbl
    lib.nnpref_time_sf_batch.argtypes = [ctypes.c_char_p, i64, ctypes.POINTER(ctypes.c_char_p), i64]
    lib.nnpref_time_batch.restype = dbl
    lib.nnpref_time_batch.argtypes = [ctypes.c_char_p, i64, ctypes.POINTER(ctypes.c_char_p), i64,
                                      ctypes.POINTER(dbl)]
    _LIBS[key] = lib
    return lib


class RefPrediction:
    """The reference's Prediction sequence on one model directory."""

    def __init__(self, model_dir, fast=False, write_warnings=False):
        self._lib = _lib(fast)
        self._h = self._lib.nnpref_create(model_dir.encode(), int(write_warnings))
        if not self._h:
            raise RuntimeError("reference setup failed: " + self._lib.nnpref_last_error().decode())

    def close(self):
        if self._h:
            self._lib.nnpref_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def num_elements(self):
        return self._lib.nnpref_num_elements(self._h)

    def num_sf(self, e):
        return self._lib.nnpref_num_sf(self._h, e)

    def num_rows(self, ec, en):
        return self._lib.nnpref_num_rows(self._h, ec, en)

    @property
    def max_cutoff(self):
        return self._lib.nnpref_max_cutoff(self._h)

    def predict(self, text, use_forces=True):
        rc = self._lib.nnpref_predict(self._h, text.encode(), int(use_forces))
        if rc != 0:
            raise RuntimeError("reference predict failed: " + self._lib.nnpref_last_error().decode())
        return self

    def _get(self, name, dtype):
        f = getattr(self._lib, "nnpref_" + name)
        n = f(self._h, None, 0)
        out = np.zeros(n, dtype=dtype)
        if n:
            ct = ctypes.c_double if dtype == np.float64 else ctypes.c_int64
            f(self._h, out.ctypes.data_as(ctypes.POINTER(ct)), n)
        return out

    def jacobian(self, text, prop, atom=0, comp=0):
        """Jacobian of a training observation (0: energy, 1: force component)
        from the reference's NeuralNetwork::calculateDEdc / calculateDFdc, all
        elements' weights in file order (internal units)."""
        n = self._lib.nnpref_jacobian(self._h, text.encode(), int(prop), int(atom), int(comp), None, 0)
        if n < 0:
            raise RuntimeError("reference jacobian failed: " + self._lib.nnpref_last_error().decode())
        out = np.zeros(n)
        self._lib.nnpref_jacobian(self._h, text.encode(), int(prop), int(atom), int(comp),
                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
        return out

    def loss_gradient(self, text, a_energy, u_forces):
        """sum aE dE/dw + sum_k u_k dF_k/dw through one structure (the
        reference's calculateDEdc / calculateDFdc), internal units."""
        u = np.ascontiguousarray(u_forces, dtype=np.float64).ravel()
        n = self._lib.nnpref_loss_gradient(self._h, text.encode(), float(a_energy),
                                           u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None, 0)
        if n < 0:
            raise RuntimeError("reference gradient failed: " + self._lib.nnpref_last_error().decode())
        out = np.zeros(n)
        self._lib.nnpref_loss_gradient(self._h, text.encode(), float(a_energy),
                                       u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
        return out

    @property
    def energy(self):
        return self._lib.nnpref_energy(self._h)

    @property
    def energy_internal(self):
        return self._lib.nnpref_energy_internal(self._h)

    def arrays(self):
        d = {}
        for n in ("forces", "forces_internal", "positions", "box", "nbr_d", "nbr_dr", "G", "dEdG",
                  "dGdr_self", "dGdr_nbr", "atomic_energy"):
            d[n] = self._get(n, np.float64)
        for n in ("nbr_offset", "nbr_index", "sf_offset", "row_offset"):
            d[n] = self._get(n, np.int64)
        d["forces"] = d["forces"].reshape(-1, 3)
        d["forces_internal"] = d["forces_internal"].reshape(-1, 3)
        d["positions"] = d["positions"].reshape(-1, 3)
        d["box"] = d["box"].reshape(3, 3)
        d["nbr_dr"] = d["nbr_dr"].reshape(-1, 3)
        d["dGdr_self"] = d["dGdr_self"].reshape(-1, 3)
        d["dGdr_nbr"] = d["dGdr_nbr"].reshape(-1, 3)
        d["energy"] = self.energy
        d["energy_internal"] = self.energy_internal
        return d


def time_batch(model_dir, texts, threads, fast=True):
    """Wall seconds of evaluateNNP over `texts` on `threads` host threads."""
    lib = _lib(fast)
    arr = (ctypes.c_char_p * len(texts))(*[t.encode() for t in texts])
    energies = np.zeros(len(texts))
    sec = lib.nnpref_time_batch(model_dir.encode(), len(texts), arr, threads,
                                energies.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if sec < 0:
        raise RuntimeError("reference timing failed: " + lib.nnpref_last_error().decode())
    return sec, energies


def time_sf_batch(model_dir, texts, threads, fast=True):
    """Wall seconds of the per-structure work of nnp-scaling (neighbour list +
    calculateSymmetryFunctionGroups without derivatives) over `texts` on
    `threads` host threads."""
    lib = _lib(fast)
    arr = (ctypes.c_char_p * len(texts))(*[t.encode() for t in texts])
    sec = lib.nnpref_time_sf_batch(model_dir.encode(), len(texts), arr, threads)
    if sec < 0:
        raise RuntimeError("reference timing failed: " + lib.nnpref_last_error().decode())
    return sec

