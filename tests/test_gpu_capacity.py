"""Neighbour-capacity overflow on replayed evaluations.

The first evaluation of a batch sizes its neighbour buffers; later ones
replay the recorded work with those buffers.  New positions that make the
lists longer (a compressed frame, an MD step, a denser training batch) must
never return energies or forces with atoms missing: the library grows the
buffers and evaluates again before any result is read.  The reference's
list is a std::vector and never truncates (Structure.cpp:287-398), so the
bar is the plain-FP64 parity bound against the reference library: energies
within 1e-10 relative, forces within 1e-10 of the largest component.
"""
import numpy as np
import pytest

from n2p2_b200 import Structure
from n2p2_b200 import water
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL_E = 1e-10
TOL_F = 1e-10


def _slab(s, factor):
    """The box's molecules (O, H, H) pulled rigidly into a layer of
    `factor` times the box height around its middle plane (same box, vacuum
    above and below): a slab frame.  Pairs inside the layer see more of
    their periodic images within the cutoff, so the lists grow well beyond
    those of the uniform box the buffers were sized for (e.g. 1.9x for 192
    molecules at factor 0.3)."""
    box = np.asarray(s.box)
    pos = s.positions.reshape(-1, 3, 3)
    frac = pos[:, 0] @ np.linalg.inv(box)
    frac -= np.floor(frac)
    target = frac.copy()
    target[:, 2] = 0.5 + factor * (frac[:, 2] - 0.5)
    shift = (target - frac) @ box + (frac - pos[:, 0] @ np.linalg.inv(box)) @ box
    return Structure((pos + shift[:, None, :]).reshape(-1, 3), s.elements, box)


def _check_against_reference(structures, E, F):
    a0 = 0
    for k, s in enumerate(structures):
        snap = H.reference_snapshot(H.WATER40, s)
        assert abs(E[k] - snap["energy"]) <= TOL_E * abs(snap["energy"]), k
        # the reference's own FMA/no-FMA spread bounds what 1e-10 can mean on a frame far outside the
        # scaling range (as in the other water parity tests)
        tol_f = max(TOL_F, 2.0 * H.reference_noise(H.WATER40, s)[1])
        assert H.max_rel(F[a0:a0 + s.numAtoms], snap["forces"]) <= tol_f, k
        a0 += s.numAtoms


def test_denser_positions_after_graph_replay():
    boxes = [water.water_box(192, seed=21), water.water_box(200, seed=22)]
    m = H.gpu_mode(H.WATER40)
    b = m.batch(boxes)
    b.setPositions(np.concatenate([s.positions for s in boxes]))
    b.evaluate(forces=True)          # sizes the buffers
    b.evaluate(forces=True)          # recorded and replayed from here on
    b.synchronize()
    cap0, rec0 = b.neighborCapacity()
    assert rec0 == 0
    entries0 = b.numNeighborEntries()
    assert entries0 <= cap0

    dense = [_slab(s, 0.3) for s in boxes]
    b.setPositions(np.concatenate([s.positions for s in dense]))
    b.evaluate(forces=True)          # replay with the old buffers: the lists do not fit
    E, F = b.energies(), b.forces()
    cap1, rec1 = b.neighborCapacity()
    entries1 = b.numNeighborEntries()
    assert entries1 > cap0, "the compressed frame must outgrow the first buffers"
    assert rec1 == 1 and cap1 >= entries1
    _check_against_reference(dense, E, F)

    # the next replay (recorded again with the grown buffers) gives the same bits
    b.evaluate(forces=True)
    E2, F2 = b.energies(), b.forces()
    assert np.array_equal(E.view(np.int64), E2.view(np.int64))
    assert np.array_equal(F.view(np.int64), F2.view(np.int64))
    assert b.neighborCapacity()[1] == 1


def test_denser_positions_through_host_evaluation():
    """The same through the end-to-end call (host positions in, host energies
    and forces out, one call per frame)."""
    boxes = [water.water_box(192, seed=23)]
    m = H.gpu_mode(H.WATER40)
    b = m.batch(boxes)
    n = b.numAtoms
    E = np.zeros(len(boxes))
    F = np.zeros((n, 3))
    pos = np.ascontiguousarray(np.concatenate([s.positions for s in boxes]))
    b.evaluateHost(pos, E, F)
    b.evaluateHost(pos, E, F)
    cap0, _ = b.neighborCapacity()
    dense = [_slab(s, 0.3) for s in boxes]
    pos = np.ascontiguousarray(np.concatenate([s.positions for s in dense]))
    b.evaluateHost(pos, E, F)
    cap1, rec1 = b.neighborCapacity()
    assert rec1 == 1 and cap1 > cap0
    _check_against_reference(dense, E, F)


def _same_lists(a, b):
    assert np.array_equal(a["offset"], b["offset"])
    assert np.array_equal(a["index"], b["index"])
    assert np.array_equal(a["image"], b["image"])
    assert np.array_equal(a["d"].view(np.int64), b["d"].view(np.int64))
    assert np.array_equal(a["dr"].view(np.int64), b["dr"].view(np.int64))


def test_one_pass_search_and_stride_overflow():
    """After the first evaluation (count pass, scan, fill pass) a batch
    searches once into a fixed stride per atom (its largest count plus 1/8
    and 16).  The one-pass lists equal the two-pass lists bit for bit, on the
    same positions and on new ones.  New positions that make one atom's list
    outgrow the stride (forty molecules of one box moved onto a shell of
    2 bohr around its first oxygen) make the replayed evaluation run the
    fill pass on the device as well: no repeated evaluation, the same
    capacity, and lists and energies equal those of a fresh batch of the same
    frames -- in that evaluation and in the next, recorded with a wider
    stride."""
    boxes = [water.water_box(n, seed=60 + k) for k, n in enumerate([64, 96, 128, 160] * 3)]
    m = H.gpu_mode(H.WATER40)
    b = m.batch(boxes)
    b.setPositions(np.concatenate([s.positions for s in boxes]))
    b.evaluate(forces=True)          # two passes; sizes the buffers and the stride
    ref = b.neighbors()
    E0 = b.energies()
    b.evaluate(forces=True)          # one pass from here on
    _same_lists(b.neighbors(), ref)
    assert np.array_equal(b.energies().view(np.int64), E0.view(np.int64))
    cap0, rec0 = b.neighborCapacity()
    counts0 = np.diff(ref["offset"])

    rng = np.random.default_rng(3)
    moved = []
    for s in boxes:
        p = s.positions + rng.normal(scale=0.05, size=s.positions.shape)
        moved.append(Structure(p, s.elements, s.box))
    b.setPositions(np.concatenate([s.positions for s in moved]))
    b.evaluate(forces=True)
    fresh = H.gpu_batch(m, moved)
    _same_lists(b.neighbors(), fresh.neighbors())
    assert b.neighborCapacity() == (cap0, rec0)

    last = boxes[-1]
    p = last.positions.reshape(-1, 3, 3).copy()
    centre = p[0, 0]
    dirs = rng.normal(size=(40, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    for k in range(40):
        p[k + 1] += centre + 2.0 * dirs[k] - p[k + 1, 0]
    dense = boxes[:-1] + [Structure(p.reshape(-1, 3), last.elements, last.box)]
    fresh = H.gpu_batch(m, dense)
    nb = fresh.neighbors()
    stride = ((counts0.max() + counts0.max() // 8 + 16 + 7) // 8) * 8
    assert np.diff(nb["offset"]).max() > stride, "one atom must outgrow the search stride"
    assert len(nb["d"]) <= cap0, "the total must still fit the buffers"
    b.setPositions(np.concatenate([s.positions for s in dense]))
    for _ in range(2):               # the replay with the old stride, then one recorded with a wider one
        b.evaluate(forces=True)
        _same_lists(b.neighbors(), nb)
        assert np.allclose(b.energies(), fresh.energies(), rtol=1e-12, atol=0.0)
        assert b.neighborCapacity() == (cap0, rec0)
