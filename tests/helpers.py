"""Shared helpers of the test suite: reference snapshots and GPU runs."""
import os

import numpy as np

from oracle import ref as oref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
WATER40 = os.path.join(GOLDEN, "models", "water40")
WATER56 = os.path.join(GOLDEN, "models", "water56")

# 1 Ha = 27211.386 meV, 1 bohr = 0.529177 A
HA_TO_MEV = 27211.386
HA_PER_BOHR_TO_MEV_PER_A = 27211.386 / 0.529177


def reference_snapshot(model_dir, structure, use_forces=True):
    """Reference Prediction of one structure: dict of internal arrays."""
    p = oref.RefPrediction(model_dir)
    try:
        p.predict(structure.to_text(), use_forces=use_forces)
        return p.arrays()
    finally:
        p.close()


def reference_energies_forces(model_dir, structures, threads=None):
    """Energies and forces (physical units) of the reference library's
    Prediction on every structure, structures spread over host threads (one
    reference Mode per thread; the library calls release the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    import threading
    threads = threads or max(1, min(16, len(os.sched_getaffinity(0))))
    local = threading.local()

    def one(s):
        if not hasattr(local, "p"):
            local.p = oref.RefPrediction(model_dir)
        local.p.predict(s.to_text())
        return local.p.energy, local.p._get("forces", np.float64).reshape(-1, 3)

    with ThreadPoolExecutor(threads) as ex:
        out = list(ex.map(one, structures))
    return np.array([e for e, _ in out]), [f for _, f in out]


def gpu_mode(model_dir, precision="fp64"):
    from n2p2_b200 import Mode
    m = Mode(0)
    m.setupFromDirectory(model_dir)
    m.setPrecision(precision)
    return m


def gpu_batch(mode, structures, forces=True, store=False):
    b = mode.batch(structures)
    b.setPositions(np.concatenate([s.positions for s in structures]))
    b.evaluate(forces=forces, storeDGdr=store)
    b.synchronize()
    return b


def split_neighbors(nb, atom_begin, atom_end):
    """Neighbour entries of atoms [atom_begin, atom_end) with local indices."""
    off = nb["offset"]
    e0, e1 = off[atom_begin], off[atom_end]
    return {"offset": off[atom_begin:atom_end + 1] - e0, "index": nb["index"][e0:e1] - atom_begin,
            "d": nb["d"][e0:e1], "dr": nb["dr"][e0:e1]}


def max_rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def scaling_table(model_dir):
    """Per-SF (Smin, scalingFactor, Gmean/Gmin offset) to unscale G, in the
    order of the scaling file (elements by atomic number, SFs sorted)."""
    from oracle.port import PortModel
    pm = PortModel(model_dir)
    a = pm.arrays
    return pm, a


def unscaled(model_dir, structure, G):
    """Raw G (SymFnc::unscale, SymFnc.cpp:197-223) of a concatenated G array."""
    pm, a = scaling_table(model_dir)
    out = np.empty_like(G)
    k = 0
    for sym in structure.elements:
        e = pm.index[sym]
        b0, b1 = a["sfBegin"][e], a["sfBegin"][e + 1]
        for s in range(b0, b1):
            t = a["scalingType"][s]
            v = G[k]
            if t == 0:
                u = v
            elif t == 1:
                u = (v - a["Smin"][s]) / a["scalingFactor"][s] + a["Gmin"][s]
            elif t == 2:
                u = v + a["Gmean"][s]
            else:
                u = (v - a["Smin"][s]) / a["scalingFactor"][s] + a["Gmean"][s]
            out[k] = u
            k += 1
    return out


ATOMIC_NUMBERS = {"H": 1, "He": 2, "Li": 3, "C": 6, "N": 7, "O": 8, "F": 9, "S": 16, "Cu": 29}


def unscaled_from_files(model_dir, structure, G):
    """Raw G of a concatenated scaled G array, from the model's own
    input.nn scaling keywords (Mode::setupSymmetryFunctionScaling,
    Mode.cpp:794-830) and scaling.data rows (elements by atomic number, SFs
    in sorted order), undone as SymFnc::unscale (SymFnc.cpp:197-223)."""
    keys, elements = {}, []
    for line in open(os.path.join(model_dir, "input.nn")):
        w = line.split("#")[0].split()
        if w:
            keys[w[0]] = w[1:]
            if w[0] == "elements":
                elements = w[1:]
    smin = float(keys["scale_min_short"][0]) if "scale_min_short" in keys else 0.0
    smax = float(keys["scale_max_short"][0]) if "scale_max_short" in keys else 1.0
    sc, ce, sg = ("scale_symmetry_functions" in keys, "center_symmetry_functions" in keys,
                  "scale_symmetry_functions_sigma" in keys)
    rows = np.loadtxt(os.path.join(model_dir, "scaling.data"), ndmin=2)
    order = sorted(elements, key=lambda e: ATOMIC_NUMBERS[e])
    table = {sym: rows[rows[:, 0] == k + 1] for k, sym in enumerate(order)}
    out = np.empty_like(G)
    k = 0
    for sym in structure.elements:
        t = table[sym]
        v = G[k:k + len(t)]
        gmin, gmax, gmean, gsig = t[:, 2], t[:, 3], t[:, 4], t[:, 5]
        if sc and ce:
            u = (v - smin) / ((smax - smin) / (gmax - gmin)) + gmean
        elif sc:
            u = (v - smin) / ((smax - smin) / (gmax - gmin)) + gmin
        elif ce:
            u = v + gmean
        elif sg:
            u = (v - smin) / ((smax - smin) / gsig) + gmean
        else:
            u = v
        out[k:k + len(t)] = u
        k += len(t)
    assert k == G.size
    return out


def reference_noise(model_dir, structure, dedg=False):
    """Relative energy and force spread (and with dedg=True the dE/dG spread)
    between the reference built with FMA contraction (-O3, x86-64-v3) and
    without (-O2, -ffp-contract=off): the floating-point noise floor of the
    reference on this input."""
    if not oref.available(fast=True):
        return (0.0, 0.0, 0.0) if dedg else (0.0, 0.0)
    a = reference_snapshot(model_dir, structure)
    p = oref.RefPrediction(model_dir, fast=True)
    try:
        p.predict(structure.to_text())
        b = p.arrays()
    finally:
        p.close()
    spread = (abs(a["energy"] - b["energy"]) / abs(a["energy"]), max_rel(b["forces"], a["forces"]))
    return spread + (max_rel(b["dEdG"], a["dEdG"]),) if dedg else spread


BOHR_TO_A = 0.529177210903
HA_TO_EV = 27.211386245988


def lammps_domain(s, list_cut, type_of, length=1.0):
    """One LAMMPS rank holding a whole orthorhombic periodic box: local atoms
    wrapped into the cell, ghost images of them within `list_cut` (bohr)
    outside it, and full neighbour lists of the local atoms (every local or
    ghost atom j != i within list_cut, ascending j).  Coordinates are returned
    in bohr x `length`.  Returns dict(x [nall,3], type [nall] (LAMMPS types
    from type_of[element symbol]), owner [nall], nlocal, numneigh [nlocal],
    firstneigh (flat, int32), ilist)."""
    import itertools
    box = np.asarray(s.box, dtype=np.float64)
    assert np.allclose(box, np.diag(np.diag(box))), "orthorhombic boxes only"
    L = np.diag(box)
    assert np.all(L > list_cut), "one image layer must cover the list cutoff"
    n = s.numAtoms
    frac = s.positions / L
    frac -= np.floor(frac)
    local = frac * L
    xs, owners = [local], [np.arange(n)]
    for sh in itertools.product((-1, 0, 1), repeat=3):
        if sh == (0, 0, 0):
            continue
        f = frac + np.array(sh, dtype=np.float64)
        keep = np.all((f >= -list_cut / L) & (f < 1.0 + list_cut / L), axis=1)
        xs.append(f[keep] * L)
        owners.append(np.nonzero(keep)[0])
    x = np.concatenate(xs)
    owner = np.concatenate(owners)
    types = np.array([type_of[e] for e in s.elements], dtype=np.int32)[owner]
    numneigh, firstneigh = [], []
    for i in range(n):
        d = x - x[i]
        d2 = np.einsum("ij,ij->i", d, d)
        js = np.nonzero(d2 <= list_cut * list_cut)[0]
        js = js[js != i]
        numneigh.append(js.size)
        firstneigh.append(js.astype(np.int32))
    return {"x": x * length, "type": types, "owner": owner, "nlocal": n,
            "numneigh": np.array(numneigh, dtype=np.int32), "firstneigh": np.concatenate(firstneigh),
            "ilist": np.arange(n, dtype=np.int32)}


def pair_style_entries(dom, pair_cut):
    """The entries PairHDNNP::transferNeighborList hands to addNeighbor:
    per local atom, neighbours with d2 <= pair_cut^2 (d2 summed in the pair
    style's order), as CSR (offset, j, type, dr [E,3], d2)."""
    x, off, js, dr, d2s = dom["x"], [0], [], [], []
    start = 0
    for i in range(dom["nlocal"]):
        nb = dom["firstneigh"][start:start + dom["numneigh"][i]]
        start += dom["numneigh"][i]
        for j in nb:
            dx, dy, dz = x[i, 0] - x[j, 0], x[i, 1] - x[j, 1], x[i, 2] - x[j, 2]
            d2 = dx * dx + dy * dy + dz * dz
            if d2 <= pair_cut * pair_cut:
                js.append(j)
                dr.append((dx, dy, dz))
                d2s.append(d2)
        off.append(len(js))
    js = np.array(js, dtype=np.int32)
    return {"offset": np.array(off, dtype=np.int64), "j": js, "type": dom["type"][js],
            "dr": np.array(dr, dtype=np.float64).reshape(-1, 3), "d2": np.array(d2s, dtype=np.float64)}


def python_read_structures(text):
    """An independent restatement of Structure::readFromLines (reference
    Structure.cpp:142-271) in Python, the checker of the library's reader:
    list of dicts (positions, elements, box, comment, energy, charge,
    forces, charges)."""
    out, block = [], []
    for line in text.splitlines():
        if not line.strip():
            continue
        block.append(line)
        if line.split()[0] != "end":
            continue
        box, pos, el, q, f = [], [], [], [], []
        comment, energy, charge = "", 0.0, 0.0
        if block[0].split()[0] != "begin":
            raise RuntimeError('ERROR: Unexpected line content, expected "begin" keyword.\n')
        for ln in block:
            w = ln.split()
            k = w[0]
            if k == "comment":
                p = ln.find("comment")
                comment = ln[:p] + ln[p + 8:]
            elif k == "lattice":
                box.append([float(w[1]), float(w[2]), float(w[3])])
            elif k == "atom":
                pos.append([float(w[1]), float(w[2]), float(w[3])])
                el.append(w[4])
                q.append(float(w[5]))
                f.append([float(w[7]), float(w[8]), float(w[9])])
            elif k == "energy":
                energy = float(w[1])
            elif k == "charge":
                charge = float(w[1])
        out.append({"positions": np.array(pos).reshape(-1, 3), "elements": el,
                    "box": np.array(box) if len(box) == 3 else None, "comment": comment, "energy": energy,
                    "charge": charge, "forces": np.array(f).reshape(-1, 3), "charges": np.array(q)})
        block = []
    return out
