"""GPU parity tests: the sm_100a path through the C ABI against the CPU oracle.

Bar: conjunction records and cell-sort order bit-exact; positions within
1e-6 km after 100 FP64 steps (Kepler + J2 and the full set); split precision
within 1e-6 km of the FP64 oracle after 100 steps as well.
"""
import json
import math
import os

import numpy as np
import pytest

from helpers import describe_diff, from_lists, records_equal, to_oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def ctx_for(capi, **kw):
    return capi.Context(capi.default_config(**kw))


# ---------------------------------------------------------------- known answers
def _collisions(recs, capi):
    return recs[(recs["flags"] & capi.PAIR_COLLISION) != 0]


def test_three_particles_gpu(capi, oracle):
    pop = from_lists([[i / 1000.0, 0, 0] for i in range(3)], [[0, float(i), 0] for i in range(3)], [0, 1, 2],
                     [0, 0, 0], [1.0] * 3, [0.6] * 3)
    with ctx_for(capi, cutoff=1.0, minDetectionRadius=0.01, evasionCutoff=0.1) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(10.0)
    col = _collisions(recs, capi)
    got = sorted((int(r["idA"]), int(r["idB"]), float(r["dl2"]), tuple(r["point"])) for r in col)
    assert got == [(0, 1, 1e-6, (0.0005, 0.0, 0.0)), (1, 2, 1e-6, (0.0015, 0.0, 0.0))]
    p = oracle.scan_params(cutoff=1.0, dt=10.0, min_detection_radius=0.01, evasion_cutoff=0.1)
    assert records_equal(recs, oracle.scan_bruteforce(to_oracle(oracle, pop), p))


def test_mix_activity_states_gpu(capi, oracle):
    rs = [[0, 0, 0], [0, 0, 0.1], [0.1, 0, 0], [0.1, 0, 0.1], [0, 0.1, 0], [0, 0.1, 0.1], [0.1, 0.1, 0],
          [0.1, 0.1, 0.1]]
    ids = [0, 0, 1, 1, 2, 3, 4, 5]
    acts = [0, 0, 0, 0, 1, 1, 2, 2]
    radii = [0.001, 0.001, 1, 1, 1, 1, 1, 1]
    pop = from_lists(rs, [[0, 0, 0]] * 8, ids, acts, [1.0] * 8, radii)
    with ctx_for(capi, cutoff=1.0, minDetectionRadius=0.01, evasionCutoff=0.1) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(10.0)
    col = _collisions(recs, capi)
    assert len(col) == 14
    assert np.all(np.isnan(col["dl2"]))  # the reference's 0/0 path
    p = oracle.scan_params(cutoff=1.0, dt=10.0, min_detection_radius=0.01, evasion_cutoff=0.1)
    assert records_equal(recs, oracle.scan_bruteforce(to_oracle(oracle, pop), p))


@pytest.mark.parametrize("factor,expected", [(1.0, 0), (2.0, 1)])
def test_collision_distance_factor_gpu(capi, factor, expected):
    pop = from_lists([[0, 0, 0], [3e-3, 0, 0]], [[1, 0, 0], [-1, 0, 0]], [1, 2], [0, 0], [1.0, 1.0], [1.0, 1.0])
    with ctx_for(capi, cutoff=80.0, collisionDistanceFactor=factor, minDetectionRadius=0.1) as ctx:
        ctx.upload(pop)
        assert len(_collisions(ctx.conjunctions(1.0), capi)) == expected


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLDEN, "interpolation_cases.json")))["cases"])
def test_linear_interpolation_gpu(capi, case):
    pop = from_lists([case["x1"], case["x2"]], [case["v1"], case["v2"]], [0, 1], [0, 0], [1.0, 1.0], [1000.0] * 2)
    with ctx_for(capi, cutoff=80.0, collisionDistanceFactor=10.0, minDetectionRadius=0.1) as ctx:
        ctx.upload(pop)
        col = _collisions(ctx.conjunctions(case["dt"]), capi)
    assert len(col) == 1
    assert float(col[0]["dl2"]) == case["expected_dl2"]
    assert tuple(float(v) for v in col[0]["point"]) == tuple(case["expected_point"])


# ------------------------------------------------------- dense random populations
def dense_population(seed, n=6000, span=250.0):
    """Objects in a box around (7000, 0, 0) km: many cutoff candidates and
    records in every list; includes duplicated states (NaN path), shared
    parents, duplicated ids, every activity state and deleted objects."""
    rng = np.random.default_rng(seed)
    r = np.array([7000.0, 0.0, 0.0]) + rng.uniform(-span / 2, span / 2, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    v = d * rng.uniform(0.0, 8.0, size=(n, 1))
    r[n - 10:] = r[:10]  # identical states
    v[n - 10:] = v[:10]
    radius = np.exp(rng.uniform(np.log(0.01), np.log(5.0), n))
    mass = 2700 * 4 / 3 * np.pi * radius ** 3
    ids = np.arange(n, dtype=np.uint64)
    ids[100:110] = ids[0:10]  # duplicate ids
    parent = np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF))
    parent[200:260] = np.uint64(777)
    act = rng.choice([0, 0, 0, 1, 2], size=n).astype(np.int8)
    return dict(x=r[:, 0], y=r[:, 1], z=r[:, 2], vx=v[:, 0], vy=v[:, 1], vz=v[:, 2], radius=radius,
                aom=np.pi * radius ** 2 * 1e-6 / mass, bc_inv=2.2 * np.pi * radius ** 2 / mass, id=ids,
                parent=parent, activity=act)


DENSE_BOX = ([6500.0, -500.0, -500.0], [7500.0, 500.0, 500.0])
DENSE_KW = dict(cutoff=20.0, collisionDistanceFactor=2000.0, minDetectionRadius=0.05, evasionCutoff=3.0,
                conjunctionThreshold=2.0, boxMin=DENSE_BOX[0], boxMax=DENSE_BOX[1])


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("screen", [0, 1])
@pytest.mark.parametrize("cell", [0.0, 7.0, 10.0, 33.0, 60.0])
def test_scan_bitexact_vs_oracle(capi, oracle, cell, screen, walk):
    pop = dense_population(11)
    dt = 10.0
    with ctx_for(capi, cellSize=cell, scanScreen=screen, walkForm=walk, **DENSE_KW) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(dt)
        keys, slots = ctx.cell_order()
        dims, reach, cs = ctx.grid()
    p = oracle.scan_params(cutoff=20.0, dt=dt, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    grid = oracle.make_grid(DENSE_BOX[0], DENSE_BOX[1], cell, 20.0)
    assert tuple(grid.n) == dims and grid.reach == reach and grid.cellSize == cs
    opop = to_oracle(oracle, pop)
    ref = oracle.scan_cells(opop, p, grid)
    brute = oracle.scan_bruteforce(opop, p)
    assert records_equal(ref, brute), describe_diff(ref, brute)
    assert len(recs) > 100
    for flag in (capi.PAIR_COLLISION, capi.PAIR_EVASION, capi.PAIR_CONJUNCTION):
        assert np.any(recs["flags"] & flag)
    assert records_equal(recs, ref), describe_diff(recs, ref)
    okeys = oracle.cell_keys(opop, grid)
    operm = oracle.stable_sort(okeys)
    assert np.array_equal(slots, operm)
    assert np.array_equal(keys, okeys[operm])


@pytest.mark.parametrize("screen", [0, 1])
@pytest.mark.parametrize("cell", [0.0, 10.0])
def test_scan_dense_cells_bitexact(capi, oracle, cell, screen):
    """Cells of hundreds of objects (the dense bin, scanned by cell tiles) next
    to sparse cells (the per-object walk): records bit-exact vs the oracle."""
    rng = np.random.default_rng(5)
    parts = [dense_population(21, n=4000)]
    for n_c, span, centre in ((3000, 30.0, (7010.0, 5.0, -3.0)), (600, 8.0, (6950.0, -40.0, 25.0)),
                              (400, 2.0, (7100.0, 60.0, 60.0))):
        c = dense_population(int(rng.integers(1 << 30)), n=n_c, span=span)
        for k, off in zip("xyz", np.array(centre) - np.array([7000.0, 0.0, 0.0])):
            c[k] = c[k] + off
        parts.append(c)
    pop = {k: np.concatenate([p_[k] for p_ in parts]) for k in parts[0]}
    pop["id"] = np.arange(len(pop["x"]), dtype=np.uint64)
    with ctx_for(capi, cellSize=cell, scanScreen=screen, **DENSE_KW) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(10.0)
    p = oracle.scan_params(cutoff=20.0, dt=10.0, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    grid = oracle.make_grid(DENSE_BOX[0], DENSE_BOX[1], cell, 20.0)
    ref = oracle.scan_cells(to_oracle(oracle, pop), p, grid)
    assert len(ref) > 1000
    assert records_equal(recs, ref), describe_diff(recs, ref)


@pytest.mark.parametrize("n,span", [(5000, 6.0), (3000, 40.0), (300, 60.0)])
def test_cell_order_rows_of_every_length(capi, oracle, n, span):
    """Rows of > 4096, 33-256 and <= 32 objects take different sort paths
    (blocked bitonic: stages inside 4096-element blocks in shared memory, the
    wider ones in global memory; shared-memory / multi-slot warp bitonic; one
    register per lane); the order must equal the stable sort by key."""
    pop = dense_population(21, n=n, span=span)
    with ctx_for(capi, **DENSE_KW) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(10.0)
        keys, slots = ctx.cell_order()
    opop = to_oracle(oracle, pop)
    grid = oracle.make_grid(DENSE_BOX[0], DENSE_BOX[1], 0.0, 20.0)
    okeys = oracle.cell_keys(opop, grid)
    operm = oracle.stable_sort(okeys)
    assert np.array_equal(slots, operm) and np.array_equal(keys, okeys[operm])
    p = oracle.scan_params(cutoff=20.0, dt=10.0, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    ref = oracle.scan_cells(opop, p, grid)
    assert records_equal(recs, ref), describe_diff(recs, ref)


def test_functor_pairs_vs_oracle(capi, oracle):
    """ladds_gpu_functor_pairs (the AoSFunctor call shape) against the oracle's
    CollisionFunctor::AoSFunctor restatement, pair by pair."""
    rng = np.random.default_rng(31)
    n = 4000
    pop = dense_population(32, n=2 * n, span=30.0)
    objs = np.zeros(2 * n, dtype=capi.OBJECT_DTYPE)
    objs["r"] = np.stack([pop["x"], pop["y"], pop["z"]], 1)
    objs["v"] = np.stack([pop["vx"], pop["vy"], pop["vz"]], 1)
    objs["radius"] = pop["radius"]
    objs["id"] = pop["id"]
    objs["parentId"] = pop["parent"]
    objs["activity"] = pop["activity"]
    objs["slot"] = np.arange(2 * n)
    first, second = objs[:n], objs[n:]
    params = capi.ScanParams(20.0, 10.0, 2000.0, 0.05, 3.0, 2.0, 1e-9)
    with ctx_for(capi, **DENSE_KW) as ctx:
        recs = ctx.functor_pairs(params, first, second)
    p = oracle.scan_params(cutoff=20.0, dt=10.0, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    expected = []
    for k in range(n):
        a, b = first[k], second[k]
        if (int(b["id"]), int(b["slot"])) < (int(a["id"]), int(a["slot"])):
            a, b = b, a
        f, dl2, point = oracle.functor_pair(p, a["r"], a["v"], float(a["radius"]), int(a["activity"]),
                                            int(a["parentId"]), b["r"], b["v"], float(b["radius"]),
                                            int(b["activity"]), int(b["parentId"]))
        if f:
            expected.append((int(a["id"]), int(b["id"]), int(a["slot"]), int(b["slot"]), dl2, tuple(point), f))
    got = [(int(r["idA"]), int(r["idB"]), int(r["slotA"]), int(r["slotB"]), float(r["dl2"]),
            tuple(float(v) for v in r["point"]), int(r["flags"])) for r in recs]
    key = lambda t: (t[0], t[1], t[2], t[3])
    assert len(expected) > 50
    assert len(got) == len(expected)
    for g, e in zip(sorted(got, key=key), sorted(expected, key=key)):
        assert g[:4] == e[:4] and g[6] == e[6]
        assert (math.isnan(g[4]) and math.isnan(e[4])) or g[4] == e[4]
        assert all((math.isnan(x) and math.isnan(y)) or x == y for x, y in zip(g[5], e[5]))


@pytest.mark.parametrize("cutoff,conj", [(20.0, 2.0), (12.0, 0.5)])
def test_scan_with_explicit_params(capi, oracle, cutoff, conj):
    pop = dense_population(33, n=5000)
    params = capi.ScanParams(cutoff, 7.0, 1500.0, 0.05, 2.0, conj, 1e-9)
    with ctx_for(capi, **DENSE_KW) as ctx:
        ctx.upload(pop)
        recs = ctx.scan(params)
    p = oracle.scan_params(cutoff=cutoff, dt=7.0, factor=1500.0, min_detection_radius=0.05, evasion_cutoff=2.0,
                           conjunction_threshold=conj)
    ref = oracle.scan_bruteforce(to_oracle(oracle, pop), p)
    assert records_equal(recs, ref), describe_diff(recs, ref)


def test_scan_with_deleted_objects(capi, oracle):
    pop = dense_population(12, n=3000)
    dead = np.arange(0, 3000, 7, dtype=np.uint32)
    with ctx_for(capi, **DENSE_KW) as ctx:
        ctx.upload(pop)
        ctx.mark_deleted(dead)
        recs = ctx.conjunctions(10.0)
    opop = to_oracle(oracle, pop)
    opop.dummy[dead] = 1
    p = oracle.scan_params(cutoff=20.0, dt=10.0, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    ref = oracle.scan_bruteforce(opop, p)
    assert records_equal(recs, ref), describe_diff(recs, ref)
    assert not np.isin(recs["slotA"], dead).any() and not np.isin(recs["slotB"], dead).any()


def test_pair_buffer_overflow_retries(capi, oracle):
    pop = dense_population(13, n=4000)
    with ctx_for(capi, pairCapacity=1, **DENSE_KW) as small, ctx_for(capi, **DENSE_KW) as big:
        small.upload(pop)
        big.upload(pop)
        a = small.step(3, cap=1 << 20)  # device buffer of one record: overflow, grow, re-run
        b = big.step(3)
        c = small.step(2, cap=1)  # caller buffer too small: rolled back, re-called with the needed size
        d = big.step(2)
    assert a.stats.retries >= 1
    assert records_equal(a.records, b.records)
    assert records_equal(c.records, d.records)


# --------------------------------------------------------------- propagation
def _state(pop):
    return np.stack([pop["x"], pop["y"], pop["z"]], 1), np.stack([pop["vx"], pop["vy"], pop["vz"]], 1)


def test_two_body_fixture_gpu(capi):
    d = json.load(open(os.path.join(GOLDEN, "two_body_10s.json")))
    r0, v0, r1, v1 = (np.asarray(d[k]) for k in ("r0", "v0", "r1", "v1"))
    pop = dict(x=r0[:, 0], y=r0[:, 1], z=r0[:, 2], vx=v0[:, 0], vy=v0[:, 1], vz=v0[:, 2], radius=np.ones(10),
               aom=np.zeros(10), bc_inv=np.zeros(10), id=np.arange(10))
    for dt, steps in ((10.0, 1), (1.0, 10)):
        with ctx_for(capi, deltaT=dt, componentMask=capi.KEP) as ctx:
            ctx.upload(pop)
            ctx.integrate(steps)
            r, v = _state(ctx.download())
        assert np.max(np.abs(r - r1)) < 2e-6 and np.max(np.abs(v - v1)) < 2e-9


@pytest.mark.parametrize("mask_name,precision", [("KEPJ2", 0), ("FULL", 0), ("FULL", 1), ("KEPJ2", 1)])
def test_propagation_vs_oracle_100_steps(capi, oracle, mask_name, precision):
    mask = capi.KEP | capi.J2 if mask_name == "KEPJ2" else capi.PROP_ALL
    pop = capi.generate_population(0, 1000, 10000)
    pop["activity"][::50] = capi.EVASIVE_PRESERVING
    with ctx_for(capi, componentMask=mask, precision=precision) as ctx:
        ctx.upload(pop)
        ctx.integrate(100)
        got = ctx.download()
    opop = to_oracle(oracle, pop)
    oracle.propagate(opop, mask, 10.0, 100)
    rg, vg = _state(got)
    ro = np.stack([opop.x, opop.y, opop.z], 1)
    vo = np.stack([opop.vx, opop.vy, opop.vz], 1)
    assert np.max(np.abs(rg - ro)) < 1e-6, np.max(np.abs(rg - ro))
    assert np.max(np.abs(vg - vo)) < 1e-9
    assert np.array_equal(got["id"], pop["id"])


@pytest.mark.parametrize("k", [1, 3])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [1, 255, 256, 257, 4096, 70_001])
def test_staged_propagation_equals_register_kernel(capi, n, precision, k):
    """The propagation before a scan (persistent grid, 256-object tiles brought
    into shared memory by bulk copies, the partial last tile read directly)
    gives the state of the multi-step register kernel bit for bit, with the
    scan every step and every third step."""
    pop = capi.generate_population(0, 77, n)
    pop["activity"][::50] = capi.EVASIVE_PRESERVING
    states = []
    for use_step in (False, True):
        with ctx_for(capi, componentMask=capi.PROP_ALL, precision=precision, useGraphs=0,
                     timestepsPerCollisionDetection=k) as ctx:
            ctx.upload(pop)
            for _ in range(2):
                if use_step:
                    ctx.step(k)
                else:
                    ctx.integrate(k)
            states.append(ctx.download())
    for key in ("x", "y", "z", "vx", "vy", "vz", "id"):
        assert np.array_equal(states[0][key], states[1][key]), key


@pytest.mark.parametrize("screen", [0, 1])
def test_graph_replay_equals_eager(capi, screen):
    pop = dense_population(14, n=5000)
    outs = []
    for graphs in (0, 1):
        with ctx_for(capi, useGraphs=graphs, deltaT=1.0, componentMask=capi.KEP | capi.J2, scanScreen=screen,
                     **DENSE_KW) as ctx:
            ctx.upload(pop)
            r1 = ctx.step(7)
            r2 = ctx.step(7)  # second call replays the cached graph
            outs.append((r1.records, r2.records, ctx.download(), ctx.cell_order()))
    a, b = outs
    assert records_equal(a[0], b[0]) and records_equal(a[1], b[1])
    for k in ("x", "vz", "id"):
        assert np.array_equal(a[2][k], b[2][k])
    assert np.array_equal(a[3][0], b[3][0]) and np.array_equal(a[3][1], b[3][1])


def test_step_records_match_oracle_scan_of_gpu_state(capi, oracle):
    """Each iteration's records equal the oracle's scan of the state the GPU
    produced for that iteration (bit-exact)."""
    pop = dense_population(15, n=4000)
    p = oracle.scan_params(cutoff=20.0, dt=1.0, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    with ctx_for(capi, deltaT=1.0, componentMask=capi.KEP | capi.J2, **DENSE_KW) as ctx:
        ctx.upload(pop)
        for it in range(3):
            res = ctx.step(1)
            state = ctx.download()
            ref = oracle.scan_bruteforce(to_oracle(oracle, state), p, step=it)
            assert records_equal(res.records, ref), describe_diff(res.records, ref)


def test_timesteps_per_collision_detection(capi):
    """SimulationTest.cpp:144-193: two bodies approaching at 20 km/s, k = 2;
    conjunction counts 0 / 0 / 1 after 1 / 2 / 3 iterations."""
    rmin = 6378.137 + 150.0
    pop = from_lists([[rmin + 100.0, 20.0, 0.0], [rmin + 100.0, -20.0, 0.0]], [[0, -10.0, 0], [0, 10.0, 0]], [0, 1],
                     [0, 0], [1.0, 1.0], [1.0, 1.0])
    for iterations, expected in ((1, 0), (2, 0), (3, 1)):
        with ctx_for(capi, deltaT=1.0, componentMask=capi.KEP, timestepsPerCollisionDetection=2) as ctx:
            ctx.upload(pop)
            res = ctx.step(iterations)
            assert int(res.stats.collisions) == expected, iterations


def test_nonfinite_state_is_reported_and_rolled_back(capi):
    pop = capi.generate_population(0, 5, 1000)
    pop["x"][3] = pop["y"][3] = pop["z"][3] = 0.0  # at the geocentre: 1/r -> inf
    with ctx_for(capi) as ctx:
        ctx.upload(pop)
        with pytest.raises(capi.LaddsError) as e:
            ctx.step(2)
        assert e.value.code == capi.ERR_NONFINITE
        back = ctx.download()
        assert np.array_equal(back["x"], pop["x"]) and ctx.iteration() == 0


def fragment_clouds(seed):
    """A dense population plus two breakup clouds 10 km apart: 3000 fragments
    of parent 4242 within 0.5 km of one point (one cell, many dense-bin
    chunks), 1000 of parent 5151 around a second point, and 20 objects with a
    parent id beyond 32 bits inside the first cloud (left to the functor's own
    parent test)."""
    rng = np.random.default_rng(seed)
    base = dense_population(seed, n=3000)
    parts = [base]
    for centre, count, parent in (((7050.0, 30.0, -20.0), 3000, 4242), ((7060.0, 30.0, -20.0), 1000, 5151),
                                  ((7050.0, 30.0, -20.0), 20, 1 << 40)):
        r = np.array(centre) + rng.uniform(-0.5, 0.5, size=(count, 3))
        v = np.array([0.0, 7.5, 0.0]) + rng.normal(scale=0.05, size=(count, 3))
        radius = np.exp(rng.uniform(np.log(0.01), np.log(0.2), count))
        mass = 2700 * 4 / 3 * np.pi * radius ** 3
        parts.append(dict(x=r[:, 0], y=r[:, 1], z=r[:, 2], vx=v[:, 0], vy=v[:, 1], vz=v[:, 2], radius=radius,
                          aom=np.pi * radius ** 2 * 1e-6 / mass, bc_inv=2.2 * np.pi * radius ** 2 / mass,
                          id=np.zeros(count, np.uint64), parent=np.full(count, np.uint64(parent)),
                          activity=np.zeros(count, np.int8)))
    pop = {k: np.concatenate([p_[k] for p_ in parts]) for k in base}
    pop["id"] = np.arange(len(pop["x"]), dtype=np.uint64) + 10
    return pop


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("screen", [0, 1])
@pytest.mark.parametrize("cell", [0.0, 7.0])
def test_breakup_clouds_bitexact_vs_oracle(capi, oracle, cell, screen, walk):
    """Fragments of one breakup start at one point: their pairs are skipped
    before they become candidates (whole blocks of one group in the dense-bin
    tiles, single pairs in the walk), the crowded cell is shared out in
    chunks, and the records still equal the oracle's, which skips them in the
    functor (CollisionFunctor.cpp:64-67)."""
    pop = fragment_clouds(31)
    dt = 10.0
    with ctx_for(capi, cellSize=cell, scanScreen=screen, walkForm=walk, **DENSE_KW) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(dt)
    p = oracle.scan_params(cutoff=20.0, dt=dt, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    opop = to_oracle(oracle, pop)
    ref = oracle.scan_cells(opop, p, oracle.make_grid(DENSE_BOX[0], DENSE_BOX[1], cell, 20.0))
    assert records_equal(ref, oracle.scan_bruteforce(opop, p, cap=len(ref) + 1024))
    big = set(range(10 + 3000 + 4000, 10 + 3000 + 4020))  # the 32-bit-overflow parents: records with the cloud
    assert sum(1 for r in ref if int(r["idA"]) in big or int(r["idB"]) in big) > 1000
    assert records_equal(recs, ref), describe_diff(recs, ref)


def test_escaping_particles_leave_the_container(capi):
    """Simulation.cpp:314, :381-387: after an integration, particles outside
    the box and particles whose state became non-finite leave the container.
    The integration keeps the non-finite state (LADDS_ERR_NONFINITE);
    ladds_gpu_remove_escaping drops both kinds, the rest steps on."""
    pop = capi.generate_population(0, 12, 2000)
    pop["x"][3] = pop["y"][3] = pop["z"][3] = 0.0  # at the geocentre: 1/r -> inf
    pop["x"][7], pop["y"][7], pop["z"][7] = 9999.0, 0.0, 0.0  # leaves the +-10000 km box within a step
    pop["vx"][7], pop["vy"][7], pop["vz"][7] = 5.0, 0.0, 0.0
    with ctx_for(capi) as ctx:
        ctx.upload(pop)
        assert ctx.remove_escaping().size == 0  # nothing leaves before the step
        assert ctx.integrate(1, allow_nonfinite=True) is False
        assert ctx.iteration() == 1
        gone = ctx.remove_escaping()
        assert sorted(gone.tolist()) == [3, 7] and ctx.size() == 1998
        back = ctx.download()
        assert np.all(np.isfinite(back["x"])) and not np.isin([3, 7], back["id"]).any()
        ctx.step(2)  # the rest integrates and scans normally
        assert ctx.remove_escaping().size == 0


def test_burnup_removal_and_append(capi):
    pop = capi.generate_population(0, 6, 5000)
    low = capi.generate_population(0, 99, 100)
    scale = (6378.137 + 100.0) / np.linalg.norm(np.stack([low["x"], low["y"], low["z"]], 1), axis=1)
    for k in ("x", "y", "z"):
        low[k] = low[k] * scale
    low["id"] = np.arange(10000, 10100, dtype=np.uint64)
    with ctx_for(capi) as ctx:
        ctx.upload(pop)
        ctx.conjunctions(10.0)  # reorder the device arrays first
        ctx.append(low)
        assert ctx.size() == 5100
        removed = ctx.remove_below(150.0)
        assert sorted(removed.tolist()) == list(range(10000, 10100))
        back = ctx.download()
    assert np.array_equal(back["id"], pop["id"]) and np.array_equal(back["x"], pop["x"])


@pytest.mark.parametrize("reserve", [0, 7000])
def test_reserve_then_append_steps_like_without(capi, reserve):
    """ladds_gpu_reserve changes no result: with room reserved before the
    append (no reallocation) the state and records after the append and two
    steps equal those of a context that grew on the append."""
    pop = capi.generate_population(0, 21, 5000)
    extra = capi.generate_population(0, 22, 600)
    extra["id"] = np.arange(20000, 20600, dtype=np.uint64)
    outs = []
    for res in (0, reserve):
        with ctx_for(capi, useGraphs=1) as ctx:
            ctx.upload(pop)
            if res:
                ctx.reserve(res)
                ctx.reserve(10)  # never shrinks
            r0 = ctx.step(3)
            ctx.append(extra)
            r1 = ctx.step(3)
            outs.append((r0.records, r1.records, ctx.download()))
    a, b = outs
    assert records_equal(a[0], b[0]) and records_equal(a[1], b[1])
    for k in ("x", "y", "z", "vx", "vy", "vz", "id"):
        assert np.array_equal(a[2][k], b[2][k]), k


def test_clear_parents(capi):
    pop = capi.generate_population(0, 8, 1000)
    pop["parent"][:] = 5
    with ctx_for(capi) as ctx:
        ctx.upload(pop)
        ctx.clear_parents()
        assert np.all(ctx.download()["parent"] == capi.SIZE_MAX)


@pytest.mark.parametrize("near_rel", [1e-9, 1e-6])
def test_threshold_neighbourhood_records_bitexact(capi, oracle, near_rel):
    """Pairs whose closest approach sits within 1e-6 relative of the collision,
    evasion or conjunction threshold, and pairs at the cutoff itself: the
    evaluation's binary32 screen must keep every pair that yields a record
    (near-band flags included); records bit-exact vs the oracle."""
    rng = np.random.default_rng(17)
    n_pairs = 900
    dt = 10.0
    radii = np.exp(rng.uniform(np.log(0.05), np.log(3.0), size=(n_pairs, 2)))
    acts = rng.choice([0, 0, 1, 2], size=(n_pairs, 2)).astype(np.int8)
    factor = 2000.0
    sep = (radii[:, 0] + radii[:, 1]) * factor / 1000.0
    kind = np.arange(n_pairs) % 4
    thr = np.where(kind == 0, sep, np.where(kind == 1, 3.0, np.where(kind == 2, 2.0, 20.0)))
    target = thr * (1.0 + rng.uniform(-2e-6, 2e-6, n_pairs))
    rs, vs = [], []
    for p in range(n_pairs):
        ra = np.array([6600.0 + 45.0 * (p % 20), -450.0 + 45.0 * ((p // 20) % 20), -450.0 + 45.0 * (p // 400)])
        va = rng.normal(size=3)
        va *= 7.5 / np.linalg.norm(va)
        dv = rng.normal(size=3)
        dv *= rng.uniform(0.5, 12.0) / np.linalg.norm(dv)
        if kind[p] == 3:  # at the cutoff: separation now, no relative motion along it
            m = rng.normal(size=3)
            m *= target[p] / np.linalg.norm(m)
            rb = ra - m
        else:  # closest approach inside the step, perpendicular to dv
            m = np.cross(dv, rng.normal(size=3))
            m *= target[p] / np.linalg.norm(m)
            rb = ra - m - dv * (dt * rng.uniform(0.2, 0.8))
        rs += [ra, rb]
        vs += [va, va - dv]
    ids = list(range(2 * n_pairs))
    pop = from_lists(rs, vs, ids, acts.reshape(-1).tolist(), [1.0] * (2 * n_pairs), radii.reshape(-1).tolist())
    kw = dict(DENSE_KW)
    with ctx_for(capi, nearThresholdRel=near_rel, **kw) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(dt)
    p = oracle.scan_params(cutoff=20.0, dt=dt, factor=factor, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0, near_rel=near_rel)
    grid = oracle.make_grid(DENSE_BOX[0], DENSE_BOX[1], 0.0, 20.0)
    ref = oracle.scan_cells(to_oracle(oracle, pop), p, grid)
    assert records_equal(recs, ref), describe_diff(recs, ref)
    assert len(ref) > 150  # about half of the pairs sit just inside a threshold
    if near_rel >= 1e-6:
        near = capi.PAIR_NEAR_COLLISION | capi.PAIR_NEAR_EVASION | capi.PAIR_NEAR_CONJUNCTION | capi.PAIR_NEAR_GATE
        assert np.sum((ref["flags"] & near) != 0) > 50


# ---------------------------------------------------------------- host-owned state
def test_host_owned_state_round_trip(capi, oracle):
    """set_state / get_state exchange positions and velocities in slot (upload)
    order while the device keeps the population in cell order: get_state equals
    download, a set_state'd state comes back unchanged, and the records of a
    scan after set_state are the oracle's for that state."""
    pop = dense_population(21, n=4000)
    rng = np.random.default_rng(5)
    with ctx_for(capi, deltaT=1.0, componentMask=capi.KEP | capi.J2, **DENSE_KW) as ctx:
        ctx.upload(pop)
        ctx.step(3)  # the device order is now the cell order, not the upload order
        _, slots = ctx.cell_order()
        assert not np.array_equal(slots, np.arange(len(slots)))
        got = ctx.get_state()
        down = ctx.download()
        for a, k in zip(got, ("x", "y", "z", "vx", "vy", "vz")):
            assert np.array_equal(a, down[k])
        new = [a + rng.normal(scale=0.5 if i < 3 else 1e-3, size=a.shape) for i, a in enumerate(got)]
        ctx.set_state(*new)
        for a, b in zip(ctx.get_state(), new):
            assert np.array_equal(a, b)
        recs = ctx.conjunctions(1.0)
        state = ctx.download()
    for k, a in zip(("x", "y", "z", "vx", "vy", "vz"), new):
        assert np.array_equal(state[k], a)
    p = oracle.scan_params(cutoff=20.0, dt=1.0, factor=2000.0, min_detection_radius=0.05, evasion_cutoff=3.0,
                           conjunction_threshold=2.0)
    ref = oracle.scan_bruteforce(to_oracle(oracle, state), p, step=2)  # records carry the last iteration
    assert len(ref) > 20
    assert records_equal(recs, ref), describe_diff(recs, ref)
