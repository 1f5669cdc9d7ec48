"""The allocation-free neighbour-list entry point against the batched one.

n2p2_neighbor_list_noalloc serves callers that cannot allocate device memory
where they need a neighbour list (memory owned by the caller's pool
allocator, loops that must not pay cudaMalloc's synchronisation): the caller
passes device buffers and the library's fixed scratch array does the rest.
Its entries must equal those of n2p2_batch_get_neighbors for the same
structure -- index, image code, distance and distance vector bit for bit
(tolerance 0, as for every neighbour-list comparison in this suite) -- on two
calls in a row, since the calls share the scratch array, for a periodic box
and for a cluster without one.  Inputs beyond the documented limits fail with
N2P2_ERR_RUNTIME (the kernels write nothing out of bounds on the way), and a
valid call right after a rejected one is still exact.  This file is
collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from n2p2_b200 import _lib
from n2p2_b200 import water
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _noalloc(torch, pos_internal, box_internal, cutoff, capacity):
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n = pos_internal.shape[0]
    pos = torch.from_numpy(np.ascontiguousarray(pos_internal)).to(dev)
    off = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    idx = torch.zeros(capacity, dtype=torch.int32, device=dev)
    img = torch.zeros(capacity, dtype=torch.int32, device=dev)
    d = torch.zeros(capacity, dtype=torch.float64, device=dev)
    dr = torch.zeros(capacity * 3, dtype=torch.float64, device=dev)
    box = None if box_internal is None else np.ascontiguousarray(box_internal, dtype=np.float64)
    total = ctypes.c_int64()
    stream = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(lib.n2p2_neighbor_list_noalloc(
        ctypes.c_void_p(pos.data_ptr()), n, None if box is None else box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        cutoff, capacity,
        ctypes.c_void_p(off.data_ptr()), ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(img.data_ptr()),
        ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(dr.data_ptr()), ctypes.byref(total), ctypes.c_void_p(stream)))
    m = total.value
    return {"offset": off.cpu().numpy(), "index": idx[:m].cpu().numpy(), "image": img[:m].cpu().numpy(),
            "d": d[:m].cpu().numpy(), "dr": dr[:3 * m].cpu().numpy().reshape(-1, 3)}


def test_noalloc_neighbor_list_matches_batched_path_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    m = H.gpu_mode(H.WATER40)
    cutoff = m.getMaxCutoffRadius()
    for seed, n_mol in ((0, 64), (5, 96)):   # two calls in a row with different inputs
        s = water.water_box(n_mol, seed=seed)
        b = H.gpu_batch(m, [s])
        ref = b.neighbors()
        got = _noalloc(torch, b.internalPositions(), s.box, cutoff, capacity=len(ref["d"]) + 64)
        assert np.array_equal(got["offset"], ref["offset"])
        assert np.array_equal(got["index"], ref["index"])
        assert np.array_equal(got["image"], ref["image"])
        assert np.array_equal(got["d"].view(np.int64), ref["d"].view(np.int64))
        assert np.array_equal(got["dr"].view(np.int64), ref["dr"].view(np.int64))


def _assert_same(got, ref):
    assert np.array_equal(got["offset"], ref["offset"])
    assert np.array_equal(got["index"], ref["index"])
    assert np.array_equal(got["image"], ref["image"])
    assert np.array_equal(got["d"].view(np.int64), ref["d"].view(np.int64))
    assert np.array_equal(got["dr"].view(np.int64), ref["dr"].view(np.int64))


def test_noalloc_cluster_and_rejections():
    """A cluster (no box: one cell, no images) bit-identical to the batched
    path; then each documented rejection, each followed by a valid call."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from n2p2_b200 import Structure
    m = H.gpu_mode(H.WATER40)
    cutoff = m.getMaxCutoffRadius()
    box_s = water.water_box(48, seed=3)
    cluster = Structure(box_s.positions, box_s.elements, None)
    b = H.gpu_batch(m, [cluster])
    ref = b.neighbors()
    pos = b.internalPositions()
    _assert_same(_noalloc(torch, pos, None, cutoff, capacity=len(ref["d"]) + 64), ref)

    # more atoms than the scratch holds: rejected on the host before any launch
    big = np.zeros((8193, 3))
    with pytest.raises(_lib.N2P2Error, match="8192"):
        _noalloc(torch, big, None, cutoff, capacity=16)
    # output capacity one entry short: the call reports the count it needed
    with pytest.raises(_lib.N2P2Error, match="capacity too small"):
        _noalloc(torch, pos, None, cutoff, capacity=len(ref["d"]) - 1)
    _assert_same(_noalloc(torch, pos, None, cutoff, capacity=len(ref["d"])), ref)
    # a dense cluster: 300 atoms in a ball of radius 3, every pair within the
    # cutoff, 299 neighbours per atom > 256
    rng = np.random.default_rng(0)
    v = rng.normal(size=(300, 3))
    dense = 3.0 * v / np.linalg.norm(v, axis=1)[:, None] * rng.random((300, 1)) ** (1.0 / 3.0)
    with pytest.raises(_lib.N2P2Error, match="256"):
        _noalloc(torch, dense, None, cutoff, capacity=300 * 300)
    # and the shared scratch still gives exact lists afterwards
    _assert_same(_noalloc(torch, pos, None, cutoff, capacity=len(ref["d"]) + 64), ref)


def test_noalloc_recorded_in_cuda_graph():
    """The call recorded into a CUDA graph (torch.cuda.graph) and replayed:
    no host copy or wait at capture (numEntries -1), then after each replay
    the status call reports the count and passes the device-side checks, and
    the entries equal the batched path's bit for bit -- for the captured
    positions and, after new positions are copied into the captured buffer,
    for the new structure (same box, same atom count)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    lib = _lib.load()
    m = H.gpu_mode(H.WATER40)
    cutoff = m.getMaxCutoffRadius()
    s1, s2 = water.water_box(64, seed=0), water.water_box(64, seed=9)
    assert np.array_equal(s1.box, s2.box)
    refs, poss = [], []
    for s in (s1, s2):
        b = H.gpu_batch(m, [s])
        refs.append(b.neighbors())
        poss.append(b.internalPositions())
    n = s1.numAtoms
    capacity = max(len(r["d"]) for r in refs) + 64
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(np.ascontiguousarray(poss[0])).to(dev)
    off = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    idx = torch.zeros(capacity, dtype=torch.int32, device=dev)
    img = torch.zeros(capacity, dtype=torch.int32, device=dev)
    d = torch.zeros(capacity, dtype=torch.float64, device=dev)
    dr = torch.zeros(capacity * 3, dtype=torch.float64, device=dev)
    box = np.ascontiguousarray(s1.box, dtype=np.float64)
    ptr = ctypes.c_void_p

    def call(stream, total):
        _lib.check(lib.n2p2_neighbor_list_noalloc(
            ptr(pos.data_ptr()), n, box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cutoff, capacity,
            ptr(off.data_ptr()), ptr(idx.data_ptr()), ptr(img.data_ptr()), ptr(d.data_ptr()), ptr(dr.data_ptr()),
            ctypes.byref(total), ptr(stream)))

    def entries(total):
        k = total.value
        return {"offset": off.cpu().numpy(), "index": idx[:k].cpu().numpy(), "image": img[:k].cpu().numpy(),
                "d": d[:k].cpu().numpy(), "dr": dr[:3 * k].cpu().numpy().reshape(-1, 3)}

    total = ctypes.c_int64()
    call(torch.cuda.current_stream(dev).cuda_stream, total)   # direct call first (scratch address lookup)
    _assert_same(entries(total), refs[0])
    g = torch.cuda.CUDAGraph()
    captured = ctypes.c_int64(0)
    with torch.cuda.graph(g):
        call(torch.cuda.current_stream(dev).cuda_stream, captured)
    assert captured.value == -1
    for k in (0, 1):
        pos.copy_(torch.from_numpy(np.ascontiguousarray(poss[k])).to(dev))
        off.zero_()
        g.replay()
        total = ctypes.c_int64()
        _lib.check(lib.n2p2_neighbor_list_noalloc_status(n, ptr(off.data_ptr()), capacity, ctypes.byref(total),
                                                         ptr(torch.cuda.current_stream(dev).cuda_stream)))
        assert total.value == len(refs[k]["d"])
        _assert_same(entries(total), refs[k])
    del g
