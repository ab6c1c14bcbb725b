"""The cell sort that allocates nothing (ladds_gpu_cell_sort_noalloc) against
the cell order of the contexts' own scans (ladds_gpu_cell_order), on calls in a
row that share the entry point's fixed scratch array: rows longer than a CTA's
shared-memory sort, rows of every warp-sort width, a LEO population on the
default grid, and the size and key errors in between.

Collected last, and self-contained so that it also runs alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return torch, capi


def _population(r):
    n = len(r)
    return dict(x=r[:, 0], y=r[:, 1], z=r[:, 2], vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                radius=np.full(n, 1.0), aom=np.full(n, 1e-8), bc_inv=np.full(n, 1e-3),
                id=np.arange(n, dtype=np.uint64), activity=np.zeros(n, np.int8))


def long_rows_case(rng):
    """25 rows of ~8000 objects (beyond the 4096-object shared-memory sort)."""
    box = ([5000.0, -2.5, -2.5], [9000.0, 2.5, 2.5])
    r = rng.uniform(box[0], box[1], size=(200_000, 3))
    return _population(r), dict(cutoff=1.0, boxMin=box[0], boxMax=box[1])


def mixed_rows_case(rng):
    """Uniform background (rows of ~5) plus rows of chosen lengths, one per
    (iy, iz): every branch of the row sort (rank, 2/4/8-slot warp bitonic,
    shared-memory CTA, global-memory CTA)."""
    box = ([6950.0, -50.0, -50.0], [7050.0, 50.0, 50.0])
    parts = [rng.uniform(box[0], box[1], size=(50_000, 3))]
    for k, length in enumerate([3, 31, 32, 33, 64, 65, 128, 129, 256, 257, 1000, 4096, 4097, 6000]):
        iy, iz = 7 + 3 * k, 60 - 2 * k
        p = np.empty((length, 3))
        p[:, 0] = rng.uniform(box[0][0], box[1][0], length)
        p[:, 1] = box[0][1] + iy + rng.uniform(0.1, 0.9, length)
        p[:, 2] = box[0][2] + iz + rng.uniform(0.1, 0.9, length)
        parts.append(p)
    r = np.concatenate(parts)
    r = r[rng.permutation(len(r))]
    return _population(r), dict(cutoff=1.0, boxMin=box[0], boxMax=box[1])


def leo_case(capi):
    """Population 0 on the default grid (80 km cells, 250 x 250 rows)."""
    return capi.generate_population(0, 4242, 100_000), dict()


def context_order(capi, pop, kw):
    """Keys in slot order, the context's sorted keys and slots, and the grid."""
    with capi.Context(capi.default_config(**kw)) as ctx:
        ctx.upload(pop)
        ctx.conjunctions(10.0)
        keys, slots = ctx.cell_order()
        dims, _, _ = ctx.grid()
    by_slot = np.empty_like(keys)
    by_slot[slots] = keys
    return by_slot, keys, slots, dims


def noalloc_sort(torch, capi, keys_by_slot, dims, n=None):
    """One call through the C ABI; device buffers come from torch (the caller)."""
    L = capi.lib()
    n = len(keys_by_slot) if n is None else n
    rows = dims[1] * dims[2]
    dkeys = torch.from_numpy(keys_by_slot.view(np.int32)).cuda()
    sorted_keys = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    order = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    row_start = torch.full((rows + 1,), -1, dtype=torch.int32, device="cuda")
    msg = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.ladds_gpu_cell_sort_noalloc(0, C.c_void_p(stream), C.c_void_p(dkeys.data_ptr()), n,
                                       C.byref((C.c_int32 * 3)(*dims)), C.c_void_p(sorted_keys.data_ptr()),
                                       C.c_void_p(order.data_ptr()), C.c_void_p(row_start.data_ptr()), msg, 256)
    torch.cuda.synchronize()
    return (rc, msg.value.decode(), sorted_keys.cpu().numpy().view(np.uint32)[:n],
            order.cpu().numpy().view(np.uint32)[:n], row_start.cpu().numpy().view(np.uint32))


def test_noalloc_sort_matches_context_order(env):
    torch, capi = env
    rng = np.random.default_rng(20260)
    cases = [long_rows_case(rng), mixed_rows_case(rng), leo_case(capi)]
    expected = [context_order(capi, pop, kw) for pop, kw in cases]
    for by_slot, _, _, dims in expected:
        assert dims[1] * dims[2] <= capi.NOALLOC_SORT_MAX_ROWS and len(by_slot) <= capi.NOALLOC_SORT_MAX_OBJECTS

    # the calls in a row, each over the scratch left by the one before
    got = []
    for k, (by_slot, _, _, dims) in enumerate(expected):
        got.append(noalloc_sort(torch, capi, by_slot, dims))
        if k == 1:  # a rejected key between two sorts
            bad = by_slot.copy()
            bad[len(bad) // 2] = np.uint32(dims[0] * dims[1] * dims[2])
            rc, msg, *_ = noalloc_sort(torch, capi, bad, dims)
            assert rc == capi.ERR_INVALID_ARG and "beyond the grid" in msg

    longest = []
    for (by_slot, keys, slots, dims), (rc, msg, skeys, order, row_start) in zip(expected, got):
        assert rc == capi.OK, msg
        assert np.array_equal(skeys, keys)
        assert np.array_equal(order, slots)
        rows = (keys // np.uint32(dims[0])).astype(np.int64)
        ref_start = np.searchsorted(rows, np.arange(dims[1] * dims[2] + 1), side="left")
        assert np.array_equal(row_start.astype(np.int64), ref_start)
        longest.append(int(np.max(np.diff(ref_start))))
    assert longest[0] > 4096 and longest[1] >= 6000  # the global-memory row sort ran


def test_noalloc_sort_twice_same_input(env):
    """Two identical calls in a row give identical output (scratch cleared)."""
    torch, capi = env
    rng = np.random.default_rng(7)
    pop, kw = mixed_rows_case(rng)
    by_slot, keys, slots, dims = context_order(capi, pop, kw)
    first = noalloc_sort(torch, capi, by_slot, dims)
    second = noalloc_sort(torch, capi, by_slot, dims)
    for rc, msg, skeys, order, _ in (first, second):
        assert rc == capi.OK, msg
        assert np.array_equal(skeys, keys) and np.array_equal(order, slots)
    assert np.array_equal(first[4], second[4])


def test_noalloc_sort_rejects_sizes_beyond_its_maximum(env):
    torch, capi = env
    small = np.zeros(4, np.uint32)
    rc, msg, *_ = noalloc_sort(torch, capi, small, (10, 300, 300), n=4)
    assert rc == capi.ERR_TOO_LARGE and "too large" in msg
    big = np.zeros(capi.NOALLOC_SORT_MAX_OBJECTS + 1, np.uint32)
    rc, msg, *_ = noalloc_sort(torch, capi, big, (4, 4, 4))
    assert rc == capi.ERR_TOO_LARGE and "too large" in msg
    # a valid call after the rejections
    keys = np.random.default_rng(3).integers(0, 64, size=1000).astype(np.uint32)
    rc, msg, skeys, order, row_start = noalloc_sort(torch, capi, keys, (4, 4, 4))
    assert rc == capi.OK, msg
    ref = np.lexsort((np.arange(1000), keys))
    assert np.array_equal(order, ref.astype(np.uint32)) and np.array_equal(skeys, keys[ref])
    assert np.array_equal(row_start.astype(np.int64), np.searchsorted(keys[ref] // 4, np.arange(17)))


def test_noalloc_sort_empty_input_and_no_row_table(env):
    """n = 0 fills the row table with zeros; a NULL row table is allowed."""
    torch, capi = env
    rc, msg, skeys, order, row_start = noalloc_sort(torch, capi, np.zeros(0, np.uint32), (4, 4, 4))
    assert rc == capi.OK, msg
    assert len(skeys) == 0 and len(order) == 0 and np.all(row_start == 0)
    keys = np.random.default_rng(11).integers(0, 64, size=500).astype(np.uint32)
    L = capi.lib()
    dkeys = torch.from_numpy(keys.view(np.int32)).cuda()
    out_keys = torch.empty(500, dtype=torch.int32, device="cuda")
    out_order = torch.empty(500, dtype=torch.int32, device="cuda")
    msg = C.create_string_buffer(256)
    rc = L.ladds_gpu_cell_sort_noalloc(0, C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                       C.c_void_p(dkeys.data_ptr()), 500, C.byref((C.c_int32 * 3)(4, 4, 4)),
                                       C.c_void_p(out_keys.data_ptr()), C.c_void_p(out_order.data_ptr()), None, msg,
                                       256)
    assert rc == capi.OK, msg.value
    ref = np.lexsort((np.arange(500), keys))
    assert np.array_equal(out_order.cpu().numpy().view(np.uint32), ref.astype(np.uint32))


def test_noalloc_sort_refuses_a_capturing_stream(env):
    """The call synchronises its stream, so a capturing stream is refused
    before anything is enqueued (the capture stays valid)."""
    torch, capi = env
    L = capi.lib()
    keys = torch.zeros(16, dtype=torch.int32, device="cuda")
    out_keys = torch.empty(16, dtype=torch.int32, device="cuda")
    out_order = torch.empty(16, dtype=torch.int32, device="cuda")
    msg = C.create_string_buffer(256)
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        rc = L.ladds_gpu_cell_sort_noalloc(0, C.c_void_p(side.cuda_stream), C.c_void_p(keys.data_ptr()), 16,
                                           C.byref((C.c_int32 * 3)(4, 4, 4)), C.c_void_p(out_keys.data_ptr()),
                                           C.c_void_p(out_order.data_ptr()), None, msg, 256)
        out_keys.add_(1)  # the capture still records work after the refusal
    assert rc == capi.ERR_INVALID_ARG and "capturing" in msg.value.decode()
    g.replay()
    torch.cuda.synchronize()
    del g
