"""nnp-scaling on the GPU: symmetry-function statistics of a structure file
under a model's settings, written as scaling.data.

Reference: src/application/nnp-scaling.cpp:30-171 (settings, scaling none,
statistics collection, Mode::calculateSymmetryFunctionGroups per structure),
libnnptrain/Dataset.cpp:974-1100 (collectSymmetryFunctionStatistics,
writeSymmetryFunctionScaling) and SymFncStatistics::addValue
(libnnp/SymFncStatistics.cpp:80-89).  The structures are evaluated in batches
(symmetry functions only, no weights needed); per batch the device reduces
min, max, sum and sum of squares of the unscaled G per element and function,
and the batches are merged in file order.

    python -m n2p2_b200.scaling [directory] [--output scaling.data]
"""
import argparse
import math
import os

import numpy as np

from .structure import read_structures


def collect_statistics(mode, structures, chunk=2048):
    """Dataset::collectSymmetryFunctionStatistics over `structures`: per
    element dict(count, min, max, sum, sum2) (arrays over its functions)."""
    acc, b = None, None
    for c0 in range(0, len(structures), chunk):
        sub = structures[c0:c0 + chunk]
        if b is None:
            b = mode.batch(sub)
        else:
            b.setStructures(sub)
        b.setPositions(np.concatenate([s.positions for s in sub]))
        b.evaluate(forces=False, graph=False, symmetryFunctionsOnly=True)
        st = b.symmetryFunctionStatistics()
        if acc is None:
            acc = st
            continue
        for a, s in zip(acc, st):
            a["count"] += s["count"]
            a["min"] = np.minimum(a["min"], s["min"])
            a["max"] = np.maximum(a["max"], s["max"])
            a["sum"] = a["sum"] + s["sum"]
            a["sum2"] = a["sum2"] + s["sum2"]
    if b is not None:
        b.close()
    return acc


def scaling_rows(stats):
    """(element index, function index, min, max, mean, sigma) rows of
    Dataset::writeSymmetryFunctionScaling (Dataset.cpp:1066-1082): mean =
    sum / n, sigma = sqrt((sum2 - sum^2 / n) / (n - 1))."""
    rows = []
    for e, st in enumerate(stats):
        n = st["count"]
        for i in range(len(st["min"])):
            s, s2 = float(st["sum"][i]), float(st["sum2"][i])
            mean = s / n if n else math.nan
            sigma = math.sqrt((s2 - s * s / n) / (n - 1)) if n > 1 else math.nan
            rows.append((e + 1, i + 1, float(st["min"][i]), float(st["max"][i]), mean, sigma))
    return rows


def write_scaling(path, stats):
    """scaling.data in the reference's column layout (%10d %10d %24.16E x 4)."""
    with open(path, "w") as f:
        f.write("#" * 80 + "\n# Symmetry function scaling data.\n" + "#" * 80 + "\n")
        f.write("# Col  Name      Description\n")
        for k, (name, what) in enumerate((("e_index", "Element index."), ("sf_index", "Symmetry function index."),
                                          ("sf_min", "Symmetry function minimum."),
                                          ("sf_max", "Symmetry function maximum."),
                                          ("sf_mean", "Symmetry function mean."),
                                          ("sf_sigma", "Symmetry function sigma."))):
            f.write("# %-4d %-9s %s\n" % (k + 1, name, what))
        f.write("#" * 80 + "\n")
        for r in scaling_rows(stats):
            f.write("%10d %10d %24.16E %24.16E %24.16E %24.16E\n" % r)


def nnp_scaling(directory=".", output=None, device=0, chunk=2048, structures=None):
    """The nnp-scaling sequence on `directory` (input.nn, input.data, or the
    given structures); writes `output` (default directory/scaling.data) and
    returns the statistics."""
    from .mode import Mode
    m = Mode(device)
    try:
        m.initialize()
        m.loadSettingsFile(os.path.join(directory, "input.nn"))
        m.setupGeneric()
        m.setupSymmetryFunctionScalingNone()
        if structures is None:
            structures = read_structures(os.path.join(directory, "input.data"))
        stats = collect_statistics(m, structures, chunk)
        write_scaling(output or os.path.join(directory, "scaling.data"), stats)
        return stats
    finally:
        m.close()


def main():
    ap = argparse.ArgumentParser(description="nnp-scaling on the GPU (scaling.data only)")
    ap.add_argument("directory", nargs="?", default=".")
    ap.add_argument("--output", default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    nnp_scaling(a.directory, a.output, a.device)


if __name__ == "__main__":
    main()
