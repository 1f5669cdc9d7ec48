"""Structures in the n2p2 `input.data` format (host-side I/O).

Parsing follows Structure::readFromLines (reference src/libnnp/Structure.cpp:142-271):
keywords begin / comment / lattice / atom / energy / charge / end, numbers
converted with correct rounding (Python float == C atof on glibc), so
positions are bit-identical to what the reference reads.  Remapping into the
cell and unit normalisation happen on the GPU (see Batch).
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


def parse_lines(lines):
    """Structure::readFromLines on one begin..end block."""
    box_rows, pos, el, q, fref = [], [], [], [], []
    comment, energy, charge = "", 0.0, 0.0
    first = lines[0].split()
    if not first or first[0] != "begin":
        raise RuntimeError('ERROR: Unexpected line content, expected "begin" keyword.\n')
    for line in lines:
        w = line.split()
        if not w:
            continue
        k = w[0]
        if k == "begin":
            for word in w[1:]:
                if word not in ("set=train", "set=test"):
                    raise RuntimeError('ERROR: Unknown keyword in structure specification, check "begin" arguments.\n')
        elif k == "comment":
            p = line.find("comment")
            comment = line[:p] + line[p + len("comment") + 1:]
        elif k == "lattice":
            if len(box_rows) > 2:
                raise RuntimeError("ERROR: Too many box vectors.\n")
            box_rows.append([float(w[1]), float(w[2]), float(w[3])])
        elif k == "atom":
            pos.append([float(w[1]), float(w[2]), float(w[3])])
            el.append(w[4])
            q.append(float(w[5]))
            fref.append([float(w[7]), float(w[8]), float(w[9])])
        elif k == "energy":
            energy = float(w[1])
        elif k == "charge":
            charge = float(w[1])
        elif k == "end":
            if len(box_rows) not in (0, 3):
                raise RuntimeError("ERROR: Strange number of box vectors.\n")
            break
        else:
            raise RuntimeError('ERROR: Unexpected file content, unknown keyword "%s".\n' % k)
    box = np.array(box_rows) if len(box_rows) == 3 else None
    return Structure(np.array(pos), el, box, comment, energy, charge, np.array(fref).reshape(-1, 3), np.array(q))


def read_structures(path_or_text, is_text=False, limit=None):
    """All structures of an input.data file (or text)."""
    text = path_or_text if is_text else open(path_or_text).read()
    out, block = [], []
    for line in text.splitlines():
        if not line.strip():
            continue
        block.append(line)
        if line.split()[0] == "end":
            out.append(parse_lines(block))
            block = []
            if limit is not None and len(out) >= limit:
                break
    return out


def write_structures(path, structures):
    with open(path, "w") as f:
        for s in structures:
            f.write(s.to_text())
