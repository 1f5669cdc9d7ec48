"""ctypes wrapper of oracle/_ref/libnnplammps.so: the reference's own
nnp::InterfaceLammps (src/libnnpif/LAMMPS/InterfaceLammps.cpp) built from its
sources with libnnp, driven the way pair_style hdnnp drives it.

TEST INFRASTRUCTURE ONLY: imported by tests/.  The product never imports
this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def lib_path(fast=False):
    """The parity build, or with `fast` the timed-baseline build (-O3, FMA)."""
    return os.path.join(_HERE, "_ref", "libnnplammps_fast.so" if fast else "libnnplammps.so")


def available(fast=False):
    return os.path.exists(lib_path(fast))


def _lib(fast=False):
    if fast not in _LIBS:
        lib = ctypes.CDLL(lib_path(fast))
        vp, i64, dbl, ip = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        lib.nnplmp_last_error.restype = ctypes.c_char_p
        lib.nnplmp_create.restype = vp
        lib.nnplmp_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ip, dbl, dbl, dbl, ip]
        lib.nnplmp_destroy.argtypes = [vp]
        lib.nnplmp_set_local_atoms.argtypes = [vp, ip, vp]
        lib.nnplmp_add_neighbors.argtypes = [vp, ip, vp, vp, vp, vp, vp]
        lib.nnplmp_process.argtypes = [vp]
        lib.nnplmp_energy.restype = dbl
        lib.nnplmp_energy.argtypes = [vp]
        lib.nnplmp_atomic_energy.restype = dbl
        lib.nnplmp_atomic_energy.argtypes = [vp, ip]
        lib.nnplmp_get_forces.argtypes = [vp, vp, i64]
        lib.nnplmp_num_ew.restype = i64
        lib.nnplmp_num_ew.argtypes = [vp]
        _LIBS[fast] = lib
    return _LIBS[fast]


class RefInterfaceLammps:
    """One reference InterfaceLammps (initialize with the given units/map)."""

    def __init__(self, model_dir, emap, cflength, cfenergy, lammps_cutoff, ntypes, showew=False, fast=False):
        self._fast = fast
        lib = _lib(fast)
        d = model_dir if model_dir.endswith("/") else model_dir + "/"
        self._h = lib.nnplmp_create(d.encode(), emap.encode(), int(showew), cflength, cfenergy, lammps_cutoff,
                                    ntypes)
        if not self._h:
            raise RuntimeError(lib.nnplmp_last_error().decode())

    def close(self):
        if self._h:
            _lib(self._fast).nnplmp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise RuntimeError(_lib(self._fast).nnplmp_last_error().decode())

    def evaluate(self, local_types, offset, j, jtype, dr, d2, nall, num_centres=None):
        """setLocalAtoms + addNeighbor for every entry + process; returns
        (energy, atomic energies of the first num_centres mapped local atoms
        (default: all local atoms), forces [nall][3] added to zeros)."""
        lib = _lib(self._fast)
        t = np.ascontiguousarray(local_types, dtype=np.int32)
        off = np.ascontiguousarray(offset, dtype=np.int64)
        jj = np.ascontiguousarray(j, dtype=np.int32)
        jt = np.ascontiguousarray(jtype, dtype=np.int32)
        r = np.ascontiguousarray(dr, dtype=np.float64)
        q = np.ascontiguousarray(d2, dtype=np.float64)
        self._check(lib.nnplmp_set_local_atoms(self._h, t.size, t.ctypes.data))
        self._check(lib.nnplmp_add_neighbors(self._h, t.size, off.ctypes.data, jj.ctypes.data, jt.ctypes.data,
                                             r.ctypes.data, q.ctypes.data))
        self._check(lib.nnplmp_process(self._h))
        E = lib.nnplmp_energy(self._h)
        n = t.size if num_centres is None else int(num_centres)
        Ea = np.array([lib.nnplmp_atomic_energy(self._h, i) for i in range(n)])
        F = np.zeros((nall, 3))
        self._check(lib.nnplmp_get_forces(self._h, F.ctypes.data, nall))
        return E, Ea, F

    def num_extrapolation_warnings(self):
        return int(_lib(self._fast).nnplmp_num_ew(self._h))
