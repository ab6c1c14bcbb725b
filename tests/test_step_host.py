"""ladds_gpu_step_host: one iteration with the positions and velocities in host
memory, moved in chunks that are propagated while the next chunk crosses PCIe
(pinned, pageable and mixed host arrays).  It must equal set_state + step(1) +
get_state bit for bit: the state, the records, the cell order and the device
copy of the population afterwards."""
import numpy as np
import pytest

from helpers import describe_diff, records_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def pinned_state(arrays):
    import torch

    out = []
    for a in arrays:
        p = torch.empty(len(a), dtype=torch.float64, pin_memory=True).numpy()
        p[:] = a
        out.append(p)
    return out


def run_pair(capi, pop, iters, precision, k=1, pair_cap=1 << 16, in_place=True, pinned=True, pre=0):
    kw = dict(componentMask=capi.PROP_ALL, precision=precision, conjunctionThreshold=10.0,
              timestepsPerCollisionDetection=k, pairCapacity=pair_cap)
    with capi.Context(capi.default_config(**kw)) as a, capi.Context(capi.default_config(**kw)) as b:
        a.upload(pop)
        b.upload(pop)
        if pre:  # graph-replayed iterations first: step_host must keep the buffer roles they were made with
            assert records_equal(a.step(pre).records, b.step(pre).records)
            pop = dict(zip(("x", "y", "z", "vx", "vy", "vz"), a.get_state()))
        # pinned: asynchronous copies that overlap; pageable: staged by the library
        stage = pinned_state if pinned else (lambda arrays: [np.array(a, dtype=np.float64) for a in arrays])
        host = stage([pop[f] for f in ("x", "y", "z", "vx", "vy", "vz")])
        total = 0
        for it in range(iters):
            a.set_state(*host)
            ra = a.step(1)
            sa = a.get_state()
            if in_place:
                rb = b.step_host(host)
            else:
                out = stage([np.zeros(len(h)) for h in host])
                rb = b.step_host(host, out)
                host = out
            for x, y in zip(sa, host):
                assert np.array_equal(x, y), f"state differs at iteration {it}"
            assert records_equal(ra.records, rb.records), describe_diff(ra.records, rb.records)
            assert int(rb.stats.records) == len(rb.records) and int(rb.stats.iterations) == 1
            total += len(rb.records)
        assert a.iteration() == b.iteration() == iters + pre
        da, db = a.download(), b.download()
        for f in da:
            assert np.array_equal(da[f], db[f]), f
        if iters % k == 0 or k == 1:
            ka, sa_ = a.cell_order()
            kb, sb = b.cell_order()
            assert np.array_equal(ka, kb) and np.array_equal(sa_, sb)
        # the device copy left by step_host serves device-resident calls
        assert records_equal(a.step(2).records, b.step(2).records)
    return total


@pytest.mark.parametrize("pinned", [True, False])
def test_step_host_matches_three_calls_split(capi, pinned):
    pop = capi.generate_population(0, 2024, 400_000)  # three chunks
    assert run_pair(capi, pop, 3, capi.PRECISION_SPLIT, pinned=pinned) > 0


def test_step_host_pageable_out_of_place(capi):
    pop = capi.generate_population(0, 2030, 300_000)
    run_pair(capi, pop, 2, capi.PRECISION_FP64, in_place=False, pinned=False)


def test_step_host_matches_three_calls_fp64_out_of_place(capi):
    pop = capi.generate_population(0, 2025, 150_000)  # one chunk
    run_pair(capi, pop, 2, capi.PRECISION_FP64, in_place=False)


def test_step_host_iterations_without_scan(capi):
    pop = capi.generate_population(0, 2026, 300_000)
    run_pair(capi, pop, 4, capi.PRECISION_SPLIT, k=3)


@pytest.mark.parametrize("pre", [1, 2, 5])
def test_step_host_after_graph_replayed_steps(capi, pre):
    pop = capi.generate_population(0, 2031, 300_000)
    run_pair(capi, pop, 3, capi.PRECISION_SPLIT, pre=pre)


def test_step_host_device_buffer_growth(capi):
    """A record buffer of 8 entries overflows: the scan runs again after growth."""
    pop = capi.generate_population(0, 2027, 300_000)
    assert run_pair(capi, pop, 2, capi.PRECISION_SPLIT, pair_cap=8) > 8


def test_step_host_pending_records(capi):
    """A caller buffer that is too small: the iteration is taken and its records
    wait for ladds_gpu_pending_records."""
    import ctypes as C

    pop = capi.generate_population(0, 2028, 200_000)
    kw = dict(componentMask=capi.PROP_ALL, conjunctionThreshold=10.0)
    with capi.Context(capi.default_config(**kw)) as a, capi.Context(capi.default_config(**kw)) as b:
        a.upload(pop)
        b.upload(pop)
        ref = a.step(1).records
        assert len(ref) > 1
        host = pinned_state([pop[f] for f in ("x", "y", "z", "vx", "vy", "vz")])
        ptrs = (C.c_void_p * 6)(*[h.ctypes.data for h in host])
        one = np.zeros(1, dtype=capi.PAIR_DTYPE)
        n = C.c_size_t()
        rc = b._L.ladds_gpu_step_host(b.handle, len(host[0]), ptrs, ptrs, one.ctypes.data_as(C.c_void_p), 1,
                                      C.byref(n), None)
        assert rc == capi.ERR_CAPACITY and n.value == len(ref)
        assert b.iteration() == 1
        got = np.zeros(n.value, dtype=capi.PAIR_DTYPE)
        rc = b._L.ladds_gpu_pending_records(b.handle, got.ctypes.data_as(C.c_void_p), len(got), C.byref(n))
        assert rc == 0 and records_equal(got, ref)
        rc = b._L.ladds_gpu_pending_records(b.handle, got.ctypes.data_as(C.c_void_p), len(got), C.byref(n))
        assert rc == 0 and n.value == 0  # released once read
        for x, y in zip(a.get_state(), host):
            assert np.array_equal(x, y)


def test_step_host_rejects_bad_arguments(capi):
    pop = capi.generate_population(0, 2029, 1000)
    with capi.Context(capi.default_config()) as ctx:
        ctx.upload(pop)
        with pytest.raises(ValueError):
            ctx.step_host([pop["x"]] * 5)
        with pytest.raises(ValueError):
            ctx.step_host([pop["x"][:10]] * 6)
        assert ctx.iteration() == 0


def test_step_host_mixed_pinned_and_pageable(capi):
    """Each array on its own: pageable ones go through the pinned staging."""
    pop = capi.generate_population(0, 2032, 300_000)
    kw = dict(componentMask=capi.PROP_ALL, conjunctionThreshold=10.0)
    names = ("x", "y", "z", "vx", "vy", "vz")
    with capi.Context(capi.default_config(**kw)) as a, capi.Context(capi.default_config(**kw)) as b:
        a.upload(pop)
        b.upload(pop)
        pinned = pinned_state([pop[f] for f in names])
        host_in = pinned[:3] + [np.array(pop[f]) for f in names[3:]]
        for it in range(2):
            a.set_state(*host_in)
            ra = a.step(1)
            out = [np.zeros(len(pop["x"])) for _ in range(3)] + pinned_state([np.zeros(len(pop["x"]))] * 3)
            rb = b.step_host(host_in, out)
            for x, y in zip(a.get_state(), out):
                assert np.array_equal(x, y), f"state differs at iteration {it}"
            assert records_equal(ra.records, rb.records), describe_diff(ra.records, rb.records)
            host_in = out


def test_step_host_pinned_in_pageable_out(capi):
    """Pinned inputs with mostly pageable outputs (staged back through the
    context's pinned buffer): same result."""
    pop = capi.generate_population(0, 2033, 300_000)
    kw = dict(componentMask=capi.PROP_ALL, precision=capi.PRECISION_SPLIT, conjunctionThreshold=10.0)
    with capi.Context(capi.default_config(**kw)) as a, capi.Context(capi.default_config(**kw)) as b:
        a.upload(pop)
        b.upload(pop)
        host = pinned_state([pop[f] for f in ("x", "y", "z", "vx", "vy", "vz")])
        for it in range(2):
            a.set_state(*host)
            ra = a.step(1)
            sa = a.get_state()
            out = [np.zeros(len(h)) for h in host]
            out[3] = pinned_state([out[3]])[0]  # one output array page-locked, the others pageable
            rb = b.step_host(host, out)
            for x, y in zip(sa, out):
                assert np.array_equal(x, y), f"state differs at iteration {it}"
            assert records_equal(ra.records, rb.records), describe_diff(ra.records, rb.records)
            host = pinned_state(out)
