"""Structures in the n2p2 `input.data` format (host-side I/O).

Reading follows Structure::readFromLines (reference src/libnnp/Structure.cpp:142-271):
keywords begin / comment / lattice / atom / energy / charge / end, numbers
converted with correct rounding (strtod in the library), so positions are
bit-identical to what the reference reads.  Remapping into the cell and unit
normalisation happen on the GPU (see Batch).
"""
import numpy as np


class Structure:
    """One configuration: positions [N,3], element symbols, optional box."""

    def __init__(self, positions, elements, box=None, comment="", energy_ref=0.0, charge_ref=0.0,
                 forces_ref=None, charges_ref=None):
        self.positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        self.elements = list(elements)
        self.box = None if box is None else np.ascontiguousarray(box, dtype=np.float64).reshape(3, 3)
        self.comment = comment
        self.energyRef = float(energy_ref)
        self.chargeRef = float(charge_ref)
        n = len(self.elements)
        self.forcesRef = np.zeros((n, 3)) if forces_ref is None else np.asarray(forces_ref, dtype=np.float64)
        self.chargesRef = np.zeros(n) if charges_ref is None else np.asarray(charges_ref, dtype=np.float64)
        # filled by a prediction
        self.energy = 0.0
        self.forces = None
        if self.positions.shape[0] != n:
            raise ValueError("positions and elements differ in length")

    @property
    def numAtoms(self):
        return len(self.elements)

    @property
    def isPeriodic(self):
        return self.box is not None

    def to_text(self):
        """input.data block with %24.16E numbers (exact round trip)."""
        out = ["begin"]
        if self.comment:
            out.append("comment " + self.comment)
        if self.box is not None:
            for k in range(3):
                out.append("lattice %24.16E %24.16E %24.16E" % tuple(self.box[k]))
        fr = self.forcesRef
        for a in range(self.numAtoms):
            x, y, z = self.positions[a]
            out.append("atom %24.16E %24.16E %24.16E %2s %24.16E %24.16E %24.16E %24.16E %24.16E" %
                       (x, y, z, self.elements[a], self.chargesRef[a], 0.0, fr[a, 0], fr[a, 1], fr[a, 2]))
        out.append("energy %24.16E" % self.energyRef)
        out.append("charge %24.16E" % self.chargeRef)
        out.append("end")
        return "\n".join(out) + "\n"


def read_structures(path_or_text, is_text=False, limit=None):
    """All structures of an input.data file (or text): Structure::readFromLines
    on every begin..end block, read by the library in one pass
    (n2p2_structures_*; numbers bit-identical to the reference's)."""
    import ctypes
    import os

    from . import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    lim = -1 if limit is None else int(limit)
    if is_text:
        data = path_or_text.encode()
        _lib.check(lib.n2p2_structures_read_text(data, len(data), lim, ctypes.byref(h)))
    else:
        _lib.check(lib.n2p2_structures_read_file(os.fsencode(path_or_text), lim, ctypes.byref(h)))
    try:
        S, N = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(lib.n2p2_structures_get_count(h, ctypes.byref(S), ctypes.byref(N)))
        S, N = S.value, N.value
        na = np.zeros(S, dtype=np.int64)
        boxes = np.zeros((S, 3, 3))
        per = np.zeros(S, dtype=np.int32)
        E = np.zeros(S)
        Q = np.zeros(S)
        _lib.check(lib.n2p2_structures_get_structure_arrays(h, na.ctypes.data, boxes.ctypes.data, per.ctypes.data,
                                                            E.ctypes.data, Q.ctypes.data))
        pos = np.zeros((N, 3))
        sym = np.zeros(N, dtype="S4")
        q = np.zeros(N)
        f = np.zeros((N, 3))
        _lib.check(lib.n2p2_structures_get_atom_arrays(h, pos.ctypes.data, sym.ctypes.data, q.ctypes.data,
                                                       f.ctypes.data))
        symbols = sym.astype(str)
        buf = ctypes.create_string_buffer(1 << 16)
        out, a0 = [], 0
        for k in range(S):
            a1 = a0 + int(na[k])
            _lib.check(lib.n2p2_structures_get_comment(h, k, buf, len(buf)))
            out.append(Structure(pos[a0:a1], symbols[a0:a1].tolist(), boxes[k] if per[k] else None,
                                 buf.value.decode(), E[k], Q[k], f[a0:a1], q[a0:a1]))
            a0 = a1
        return out
    finally:
        lib.n2p2_structures_destroy(h)


def write_structures(path, structures):
    with open(path, "w") as f:
        for s in structures:
            f.write(s.to_text())
