"""nnp-scaling on the GPU (n2p2_b200.scaling) against the reference's
sequence: the unscaled G of every atom from the reference library, added up
per element and function in file order (SymFncStatistics::addValue,
SymFncStatistics.cpp:80-89).  Counts exact; min / max within 1e-12 and
sums within 1e-11 of the largest |G| (the tolerance of G itself); the
written scaling.data loads into a model again."""
import os

import numpy as np
import pytest

from n2p2_b200 import Structure, read_structures, scaling, water
from tests import helpers as H

pytestmark = pytest.mark.gpu

EXAMPLES = [os.path.join(H.GOLDEN, "examples", n) for n in ("H2O_RPBE-D3", "Cu2S_PBE")]


def _structures(model):
    if model in EXAMPLES:
        s0 = read_structures(os.path.join(model, "input.data"))[0]
        rng = np.random.default_rng(1)
        out = [s0]
        for k in range(4):
            out.append(Structure(s0.positions + rng.normal(scale=0.02, size=s0.positions.shape), s0.elements,
                                 box=s0.box))
        return out
    return water.water_batch(5, seed=12, n_min=32, n_max=96, sigma_range=(0.05, 0.2))


def _reference_statistics(model, structs):
    pm, _ = H.scaling_table(model)
    ne = len(pm.symbols)
    acc = None
    for s in structs:
        snap = H.reference_snapshot(model, s, use_forces=False)
        G = H.unscaled(model, s, snap["G"])
        off = snap["sf_offset"]
        if acc is None:
            acc = [None] * ne
        for a, sym in enumerate(s.elements):
            e = pm.index[sym]
            g = G[off[a]:off[a + 1]]
            if acc[e] is None:
                acc[e] = {"count": 0, "min": np.full(g.size, np.inf), "max": np.full(g.size, -np.inf),
                          "sum": np.zeros(g.size), "sum2": np.zeros(g.size)}
            r = acc[e]
            r["count"] += 1
            r["sum"] += g
            r["sum2"] += g * g
            r["min"] = np.minimum(r["min"], g)
            r["max"] = np.maximum(r["max"], g)
    return acc


@pytest.mark.parametrize("model", EXAMPLES + [H.WATER56], ids=["H2O_RPBE-D3", "Cu2S_PBE", "water56"])
def test_statistics_match_reference_sequence(model, tmp_path):
    structs = _structures(model)
    ref = _reference_statistics(model, structs)
    out = str(tmp_path / "scaling.data")
    stats = scaling.nnp_scaling(model, output=out, structures=structs, chunk=2)   # merges three batches
    for e, (st, r) in enumerate(zip(stats, ref)):
        assert st["count"] == r["count"]
        scale = max(np.abs(r["min"]).max(), np.abs(r["max"]).max())
        assert np.abs(st["min"] - r["min"]).max() <= 1e-12 * scale
        assert np.abs(st["max"] - r["max"]).max() <= 1e-12 * scale
        assert np.abs(st["sum"] - r["sum"]).max() <= 1e-11 * scale * r["count"]
        assert np.abs(st["sum2"] - r["sum2"]).max() <= 1e-11 * scale * scale * r["count"]
    # the file: the reference's columns, readable as a model's scaling
    rows = [l.split() for l in open(out) if l.strip() and not l.startswith("#")]
    expect = scaling.scaling_rows(stats)
    assert len(rows) == len(expect)
    for got, want in zip(rows, expect):
        assert int(got[0]) == want[0] and int(got[1]) == want[1]
        assert np.allclose([float(x) for x in got[2:]], want[2:], rtol=1e-15, atol=0.0, equal_nan=True)
    from n2p2_b200 import Mode
    m = Mode(0)
    m.initialize()
    m.loadSettingsFile(os.path.join(model, "input.nn"))
    m.setupGeneric()
    m.setupSymmetryFunctionScaling(out)
    m.close()


def test_symmetry_functions_only_needs_no_weights():
    """An evaluation of symmetry functions alone runs without weights; a full
    evaluation of the same model still refuses."""
    from n2p2_b200 import Mode
    m = Mode(0)
    m.initialize()
    m.loadSettingsFile(os.path.join(H.WATER40, "input.nn"))
    m.setupGeneric()
    m.setupSymmetryFunctionScalingNone()
    s = water.water_box(32, seed=3)
    b = m.batch([s])
    b.setPositions(s.positions)
    b.evaluate(forces=False, graph=False, symmetryFunctionsOnly=True)
    assert np.isfinite(b.symmetryFunctions()).all()
    with pytest.raises(Exception, match="weights"):
        b.evaluate(forces=True)
    m.close()
