"""Autotuned kernel shapes: every shape gives bitwise the same energies and
forces (atoms of every tier included), the tuner picks the fastest measured
shape and the cache file round-trips."""
import json

import numpy as np
import pytest

from n2p2_b200 import Structure, water
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _compressed(s, f):
    return Structure(s.positions * f, s.elements, box=s.box * f)


@pytest.fixture(scope="module")
def boxes():
    b = water.water_batch(10, seed=5, n_min=32, n_max=256)
    # ~1.4x and ~4x water density: atoms beyond the 128/160/192 and 384-entry tiers
    b.append(_compressed(water.water_box(64, seed=8, sigma=0.05), 0.89))
    b.append(_compressed(water.water_box(48, seed=9, sigma=0.05), 0.63))
    return b


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_shapes_are_equivalent_and_tuned(boxes, precision, tmp_path, monkeypatch):
    monkeypatch.setenv("N2P2_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    m = H.gpu_mode(H.WATER40, precision=precision)
    b = m.batch(boxes)
    b.setPositions(np.concatenate([s.positions for s in boxes]))
    b.evaluate(forces=True, graph=False)
    nb = b.neighbors()
    counts = np.diff(nb["offset"])
    assert counts.max() > 384 and ((counts > 128) & (counts <= 384)).any()
    ref = None
    for v in range(3):
        b.setShapes(v, 2 - v)
        b.evaluate(forces=True)
        out = (b.energies(), b.forces())
        if ref is None:
            ref = out
        else:
            assert np.array_equal(out[0].view(np.int64), ref[0].view(np.int64))
            assert np.array_equal(out[1].view(np.int64), ref[1].view(np.int64))
    r = b.autotune(useCache=True)
    assert not r["from_cache"]
    assert all(t > 0 for t in r["values_ms"] + r["forces_ms"])
    assert r["values"] == int(np.argmin(r["values_ms"])) and r["forces"] == int(np.argmin(r["forces_ms"]))
    cache = json.load(open(tmp_path / "tune.json"))
    assert len(cache) == 1
    entry = next(iter(cache.values()))
    assert entry["values"] == r["values"] and entry["forces"] == r["forces"]
    r2 = b.autotune(useCache=True)
    assert r2["from_cache"] and (r2["values"], r2["forces"]) == (r["values"], r["forces"])
    b.evaluate(forces=True)
    assert np.array_equal(b.energies().view(np.int64), ref[0].view(np.int64))
    assert np.array_equal(b.forces().view(np.int64), ref[1].view(np.int64))
