"""Slab decomposition over ranks (ladds_b200.slabs): the union of the ranks'
records equals the single-context records, iteration by iteration, while
objects migrate between slabs.  Multi-rank runs are gloo process groups of 2
and 3 ranks on 127.0.0.1 (spawned processes); on the CPU the engine is the
oracle (tests/helpers.OracleEngine), on the GPU every rank holds its own
context on the one device (the ranks exchange host lists; no kernel of one
rank waits on another)."""
import os
import socket

import numpy as np
import pytest

from helpers import OracleEngine, records_without_slots

BOX = ([6500.0, -500.0, -500.0], [7500.0, 500.0, 500.0])
CUTOFF, CELL, DT, ITERS = 20.0, 20.0, 1.0, 4
SCAN_KW = dict(factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0, conjunction_threshold=2.0)


def population(seed=3, n=3000, span=250.0):
    rng = np.random.default_rng(seed)
    r = np.array([7000.0, 0.0, 0.0]) + rng.uniform(-span / 2, span / 2, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    v = d * rng.uniform(0.0, 8.0, size=(n, 1))  # up to 8 km per 1 s step: objects cross slab borders
    radius = np.exp(rng.uniform(np.log(0.01), np.log(5.0), n))
    mass = 2700 * 4 / 3 * np.pi * radius ** 3
    parent = np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF))
    parent[100:140] = np.uint64(9)
    return dict(x=r[:, 0], y=r[:, 1], z=r[:, 2], vx=v[:, 0], vy=v[:, 1], vz=v[:, 2], radius=radius,
                aom=np.pi * radius ** 2 * 1e-6 / mass, bc_inv=2.2 * np.pi * radius ** 2 / mass,
                id=np.arange(n, dtype=np.uint64) * 3 + 1, parent=parent,
                activity=rng.choice([0, 0, 1, 2], size=n).astype(np.int8))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_split_layers():
    from ladds_b200.slabs import split_layers

    hist = np.zeros(50)
    hist[19:32] = 100
    b = split_layers(hist, 3, 1)
    assert b[0] == 0 and b[-1] == 50 and all(b1 > b0 for b0, b1 in zip(b[:-1], b[1:]))
    counts = [hist[b0:b1].sum() for b0, b1 in zip(b[:-1], b[1:])]
    assert max(counts) - min(counts) <= 100  # one layer of imbalance at most
    assert split_layers(np.zeros(8), 4, 2) == [0, 2, 4, 6, 8]  # empty histogram: minimal slabs
    b = split_layers(np.r_[np.zeros(10), 1000.0], 3, 2)  # everything in the top layer
    assert all(b1 - b0 >= 2 for b0, b1 in zip(b[:-1], b[1:]))
    with pytest.raises(ValueError):
        split_layers(np.ones(5), 3, 2)


def oracle_engine(oracle, pop):
    return OracleEngine(oracle, pop, BOX[0], BOX[1], CUTOFF, CELL, oracle.KEP | oracle.J2, DT, **SCAN_KW)


def gpu_engine(pop):
    from ladds_b200 import capi

    ctx = capi.Context(capi.default_config(deltaT=DT, componentMask=capi.KEP | capi.J2, cutoff=CUTOFF,
                                           cellSize=CELL, boxMin=BOX[0], boxMax=BOX[1],
                                           collisionDistanceFactor=SCAN_KW["factor"],
                                           minDetectionRadius=SCAN_KW["min_detection_radius"],
                                           evasionCutoff=SCAN_KW["evasion_cutoff"],
                                           conjunctionThreshold=SCAN_KW["conjunction_threshold"]))
    ctx.upload(pop)
    return ctx


def _rank_main(rank, world, port, kind, out_dir):
    import datetime
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (here, root, os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist

    from ladds_b200.slabs import SlabDecomposition

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        pop = population()
        if kind == "oracle":
            import oracle_py

            engine = oracle_engine(oracle_py, pop)
        else:
            engine = gpu_engine(pop)
        slabs = SlabDecomposition(engine)
        bounds = slabs.distribute()
        sizes = slabs.all_gather(engine.size())
        per_iter = [slabs.gather_records(slabs.iterate(DT)) for _ in range(ITERS)]
        moved = slabs.all_gather(slabs.migrated)
        if rank == 0:
            np.savez(os.path.join(out_dir, "ranks.npz"), bounds=np.array(bounds), sizes=np.array(sizes),
                     moved=np.array(moved), **{f"it{k}": r for k, r in enumerate(per_iter)})
        if kind == "gpu":
            engine.close()
    finally:
        dist.destroy_process_group()


def run_ranks(world, kind, tmp_path):
    import torch.multiprocessing as mp

    mp.spawn(_rank_main, args=(world, free_port(), kind, str(tmp_path)), nprocs=world, join=True)
    return np.load(os.path.join(tmp_path, "ranks.npz"))


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_match_single_rank_oracle(oracle, tmp_path, world):
    got = run_ranks(world, "oracle", tmp_path)
    pop = population()
    assert got["sizes"].sum() == len(pop["x"]) and np.all(got["sizes"] > 0)
    single = oracle_engine(oracle, pop)
    for k in range(ITERS):
        single.integrate(1)
        ref = single.conjunctions(DT)
        assert len(ref) > 50
        assert records_without_slots(got[f"it{k}"]) == records_without_slots(ref), f"iteration {k}"
    assert got["moved"].sum() > 0  # objects changed slabs during the run


def halo_split(oracle, pop):
    """The population reordered with its upper half of cell layers last, and
    the first slot of that half (the halo)."""
    e = oracle_engine(oracle, pop)
    iz = e.layers()
    upper = np.nonzero(iz >= np.median(iz))[0]
    order = np.r_[np.setdiff1d(np.arange(len(iz)), upper), upper]
    return {k: v[order] for k, v in pop.items()}, len(iz) - len(upper), pop["id"][upper]


def test_halo_objects_are_targets_only(oracle):
    """The upper layers declared halo: no pair of two halo objects is listed,
    every pair with one own object is."""
    pop = population(seed=8)
    full = oracle_engine(oracle, pop).conjunctions(DT)
    reordered, start, halo_ids = halo_split(oracle, pop)
    e = oracle_engine(oracle, reordered)
    e.set_halo(start)
    part = e.conjunctions(DT)
    halo_ids = set(halo_ids.tolist())
    want = full[[not (int(r["idA"]) in halo_ids and int(r["idB"]) in halo_ids) for r in full]]
    assert 0 < len(want) < len(full)
    assert records_without_slots(want) == records_without_slots(part)


@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


@pytest.mark.gpu
def test_gpu_slab_primitives(capi):
    pop = population(seed=5, n=4000)
    with gpu_engine(pop) as ctx:
        dims, reach, cell = ctx.grid()
        hist = ctx.layer_histogram()
        iz = np.clip(np.floor((pop["z"] - BOX[0][2]) * (1.0 / cell)), 0, dims[2] - 1).astype(int)
        assert np.array_equal(hist, np.bincount(iz, minlength=dims[2]))
        sel = ctx.select_layers(24, 26)
        assert len(sel) > 100 and np.array_equal(sel, np.nonzero((iz >= 24) & (iz < 26))[0])
        ctx.mark_deleted(sel[:5])
        assert len(ctx.select_layers(24, 26)) == len(sel) - 5  # deleted objects are not selected
        ids_before = ctx.get_objects(np.arange(ctx.size()))["id"]
        ctx.remove_slots(sel)
        assert ctx.size() == len(pop["x"]) - len(sel)
        left = ctx.get_objects(np.arange(ctx.size()))["id"]
        assert np.array_equal(left, np.delete(ids_before, sel))  # survivors keep their relative order


@pytest.mark.gpu
def test_gpu_halo_scan_matches_oracle(capi, oracle):
    """The GPU scan with a halo equals the oracle engine's (halo-halo pairs dropped)."""
    reordered, start, _ = halo_split(oracle, population(seed=8))
    e = oracle_engine(oracle, reordered)
    e.set_halo(start)
    ref = e.conjunctions(DT)
    with gpu_engine(reordered) as ctx:
        ctx.set_halo(start)
        got = ctx.conjunctions(DT)
        ctx.set_halo(None)
        assert len(ctx.conjunctions(DT)) > len(got)
    assert len(ref) > 10
    assert records_without_slots(got) == records_without_slots(ref)


@pytest.mark.gpu
def test_gpu_slabs_match_single_context(capi, tmp_path):
    got = run_ranks(2, "gpu", tmp_path)
    single = gpu_engine(population())
    try:
        for k in range(ITERS):
            single.integrate(1)
            ref = single.conjunctions(DT)
            assert len(ref) > 50
            assert records_without_slots(got[f"it{k}"]) == records_without_slots(ref), f"iteration {k}"
    finally:
        single.close()
    assert got["moved"].sum() > 0


@pytest.mark.gpu
def test_gpu_device_exchange_primitives(capi):
    """pack_layers / append_records / truncate on device buffers: the packed
    records are get_objects of the selected slots in cell order, appending them
    to another context reproduces them, removal and truncation keep the rest in
    order, and host memory is refused as a buffer."""
    import torch

    pop = population(seed=6, n=4000)
    rec_bytes = capi.STATE_RECORD_DTYPE.itemsize
    with gpu_engine(pop) as a, gpu_engine(population(seed=7, n=500)) as b:
        a.conjunctions(DT)  # cell order
        keys, slots = a.cell_order()
        sel = a.select_layers(24, 27)
        buf = torch.empty(len(sel) * rec_bytes, dtype=torch.uint8, device="cuda")
        with pytest.raises(capi.LaddsError) as e:
            a.pack_layers(24, 27, False, buf, len(sel) - 1)
        assert e.value.code == capi.ERR_CAPACITY
        got = a.pack_layers(24, 27, False, buf, len(sel))
        assert got == len(sel) > 100
        rec = np.frombuffer(buf.cpu().numpy().tobytes(), dtype=capi.STATE_RECORD_DTYPE)
        in_order = slots[np.isin(slots, sel)]  # the selected slots in cell order
        assert rec.tobytes() == a.get_objects(in_order).tobytes()
        n0 = b.size()
        b.append_records(buf, got)
        assert b.size() == n0 + got
        assert b.get_objects(np.arange(n0, n0 + got)).tobytes() == rec.tobytes()
        b.truncate(n0)
        assert b.size() == n0
        with pytest.raises(capi.LaddsError):  # host memory is not a device buffer
            b.append_records(torch.zeros(rec_bytes, dtype=torch.uint8), 1)
        ids_before = a.get_objects(np.arange(a.size()))["id"]
        assert a.pack_layers(24, 27, True, None, 0) == len(sel)  # removed without being packed
        assert a.size() == len(pop["x"]) - len(sel)
        assert np.array_equal(a.get_objects(np.arange(a.size()))["id"], np.delete(ids_before, sel))
