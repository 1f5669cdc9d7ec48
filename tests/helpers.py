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
