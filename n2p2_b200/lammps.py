"""Python mirror of nnp::InterfaceLammps (reference
src/libnnpif/LAMMPS/InterfaceLammps.h) over the C ABI (n2p2_lammps_*): the
object a LAMMPS pair style drives every MD step.

    lmp = InterfaceLammps()
    lmp.initialize("hdnnp/", "1:H,2:O", False, False, 0, -1, cflength, cfenergy, cutoff, 2, 0)
    lmp.setLocalAtoms(nlocal, atom_type)                 # LAMMPS types, 1-based
    lmp.transferNeighborList(ilist, numneigh, firstneigh, x, atom_type, cutoff)
    lmp.process()
    E = lmp.getEnergy()
    lmp.getForces(f)                                     # adds into f[nall][3]

Positions, energies and forces are in LAMMPS units (cflength / cfenergy
convert, as in the reference); ghost atoms receive forces that LAMMPS folds
back to their owners.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check

_P = ctypes.POINTER


def _pointers(base, offsets):
    """A C array of pointers base + offsets[k] (bytes), built without a Python loop."""
    addr = (np.uint64(base) + np.asarray(offsets, dtype=np.uint64)) if len(offsets) else np.zeros(1, np.uint64)
    return (ctypes.c_void_p * len(addr)).from_buffer_copy(np.ascontiguousarray(addr, dtype=np.uint64).tobytes())


def _rows(a):
    """LAMMPS-style row pointers (double**) into a C-contiguous [n][3] array."""
    return _pointers(a.ctypes.data, np.arange(len(a), dtype=np.uint64) * np.uint64(a.strides[0]))


class InterfaceLammps:
    def __init__(self, device=0):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        check(self._lib.n2p2_lammps_create(ctypes.byref(h), int(device)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.n2p2_lammps_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up --------------------------------------------------------------
    def initialize(self, directory, emap, showew, resetew, showewsum, maxew, cflength, cfenergy, lammpsCutoff,
                   lammpsNtypes, myRank=0):
        check(self._lib.n2p2_lammps_initialize(self._h, str(directory).encode(), (emap or "").encode(), int(showew),
                                               int(resetew), int(showewsum), int(maxew), float(cflength),
                                               float(cfenergy), float(lammpsCutoff), int(lammpsNtypes),
                                               int(myRank)))
        return self

    def setPrecision(self, precision):
        p = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}.get(precision, precision)
        check(self._lib.n2p2_lammps_set_precision(self._h, int(p)))

    def getMaxCutoffRadius(self):
        r = ctypes.c_double()
        check(self._lib.n2p2_lammps_get_max_cutoff_radius(self._h, ctypes.byref(r)))
        return r.value

    # -- per step ------------------------------------------------------------
    def setLocalAtoms(self, numAtomsLocal, atomType):
        t = np.ascontiguousarray(atomType, dtype=np.int32)
        check(self._lib.n2p2_lammps_set_local_atoms(self._h, int(numAtomsLocal), t.ctypes.data))

    def addNeighbor(self, i, j, tag, type, dx, dy, dz, d2):
        check(self._lib.n2p2_lammps_add_neighbor(self._h, int(i), int(j), int(tag), int(type), float(dx), float(dy),
                                                 float(dz), float(d2)))

    def transferNeighborList(self, ilist, numneigh, firstneigh, x, atomType, maxCutoffRadius):
        """PairHDNNP::transferNeighborList with LAMMPS's arrays: ilist[inum],
        numneigh[nlocal], firstneigh (one index array per local atom, or a flat
        array with numneigh giving the split), x[nall][3], atomType[nall]."""
        il = np.ascontiguousarray(ilist, dtype=np.int32)
        nn = np.ascontiguousarray(numneigh, dtype=np.int32)
        if isinstance(firstneigh, np.ndarray) and firstneigh.ndim == 1:
            flat = np.ascontiguousarray(firstneigh, dtype=np.int32)
        else:
            flat = np.ascontiguousarray(np.concatenate([np.asarray(a, dtype=np.int32) for a in firstneigh])
                                        if len(firstneigh) else np.zeros(0, dtype=np.int32))
        starts = np.concatenate([[0], np.cumsum(nn, dtype=np.int64)[:-1]]) if nn.size else np.zeros(0, np.int64)
        fn = _pointers(flat.ctypes.data, starts.astype(np.uint64) * np.uint64(4))
        xa = np.ascontiguousarray(x, dtype=np.float64)
        xr = _rows(xa)
        ty = np.ascontiguousarray(atomType, dtype=np.int32)
        check(self._lib.n2p2_lammps_transfer_neighbor_list(self._h, int(il.size), il.ctypes.data, nn.ctypes.data,
                                                           ctypes.cast(fn, ctypes.c_void_p),
                                                           ctypes.cast(xr, ctypes.c_void_p), ty.ctypes.data,
                                                           float(maxCutoffRadius)))

    def process(self):
        check(self._lib.n2p2_lammps_process(self._h))

    def getEnergy(self):
        e = ctypes.c_double()
        check(self._lib.n2p2_lammps_get_energy(self._h, ctypes.byref(e)))
        return e.value

    def getAtomicEnergy(self, index):
        e = ctypes.c_double()
        check(self._lib.n2p2_lammps_get_atomic_energy(self._h, int(index), ctypes.byref(e)))
        return e.value

    def getForces(self, f):
        """Adds the forces on local and ghost atoms into f ([nall][3] float64,
        C-contiguous, modified in place)."""
        if not (isinstance(f, np.ndarray) and f.dtype == np.float64 and f.flags.c_contiguous and f.ndim == 2
                and f.shape[1] == 3):
            raise TypeError("f must be a C-contiguous float64 array of shape [nall, 3]")
        rows = _rows(f)
        check(self._lib.n2p2_lammps_get_forces(self._h, ctypes.cast(rows, ctypes.c_void_p)))

    def getNumExtrapolationWarnings(self):
        c = ctypes.c_int64()
        check(self._lib.n2p2_lammps_get_num_extrapolation_warnings(self._h, ctypes.byref(c)))
        return c.value

    def clearExtrapolationWarnings(self):
        check(self._lib.n2p2_lammps_clear_extrapolation_warnings(self._h))
