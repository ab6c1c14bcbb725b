"""Parity at the benchmark's own sizes and at the edges of the input space.

* the 1e6-object population of the throughput benchmark (full force set,
  dt 10 s, 80 km cutoff, 0.1 km thresholds): the records of a graph-replayed
  step and the cell-sort order are the oracle's, bit for bit, on the state the
  GPU produced;
* the constellation population (four Walker shells + debris) and the 8e6
  scale population in its autotuned form: the same;
* empty and single-object populations, and objects outside the cell-grid box
  (clamped into its boundary cells) next to each other.
"""
import numpy as np
import pytest

from helpers import describe_diff, from_lists, records_equal, to_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def oracle_params(oracle, cfg, dt):
    return oracle.scan_params(cutoff=cfg.cutoff, dt=dt, factor=cfg.collisionDistanceFactor,
                              min_detection_radius=cfg.minDetectionRadius, evasion_cutoff=cfg.evasionCutoff,
                              conjunction_threshold=cfg.conjunctionThreshold, near_rel=cfg.nearThresholdRel)


def check_step_against_oracle(capi, oracle, pop, steps, **kw):
    cfg = capi.default_config(componentMask=capi.PROP_ALL, precision=capi.PRECISION_SPLIT, **kw)
    with capi.Context(cfg) as ctx:
        ctx.upload(pop)
        res = ctx.step(steps)  # a multi-step call: captured graphs, scan every step
        last = res.records[res.records["step"] == steps - 1]
        state = ctx.download()
        keys, slots = ctx.cell_order()
        dims, reach, cell = ctx.grid()
    grid = oracle.make_grid(list(cfg.boxMin), list(cfg.boxMax), cfg.cellSize, cfg.cutoff)
    assert tuple(grid.n) == dims and grid.reach == reach and grid.cellSize == cell
    opop = to_oracle(oracle, state)
    ref = oracle.scan_cells(opop, oracle_params(oracle, cfg, cfg.deltaT), grid, step=steps - 1)
    assert len(ref) > 0
    assert records_equal(last, ref), describe_diff(last, ref)
    okeys = oracle.cell_keys(opop, grid)
    operm = oracle.stable_sort(okeys)
    assert np.array_equal(slots, operm)
    assert np.array_equal(keys, okeys[operm])
    return len(res.records)


def test_benchmark_population_1e6(capi, oracle):
    pop = capi.generate_population(0, 1001, 1_000_000)
    assert check_step_against_oracle(capi, oracle, pop, 3) >= 1


def test_constellation_population(capi, oracle):
    pop = capi.generate_population(2, 1002, 4224 + 300_000)
    check_step_against_oracle(capi, oracle, pop, 2)


def test_scale_population_8e6(capi, oracle):
    """The scale form (7.5M small debris in two Gaussian shells + 500k) in the
    form the autotuner picks for it: 40 km cells, full buffers screened in place."""
    pop = capi.generate_population(4, 1004, 8_000_000)
    assert check_step_against_oracle(capi, oracle, pop, 2, cellSize=40.00004, scanScreen=capi.SCREEN_BUFFER) > 100


def test_empty_and_single_object(capi):
    with capi.Context(capi.default_config()) as ctx:
        ctx.upload(capi.empty_population(0))
        assert len(ctx.step(5).records) == 0
        ctx.integrate(3)
        assert len(ctx.conjunctions(10.0)) == 0 and ctx.size() == 0
        one = from_lists([[7000.0, 0, 0]], [[0, 7.5, 0]], [1], [0], [1.0], [1.0])
        ctx.append(one)
        assert len(ctx.step(2).records) == 0 and ctx.size() == 1
        assert ctx.iteration() == 10


def test_objects_outside_the_box(capi, oracle):
    """Objects beyond the grid box are clamped into its boundary cells; pairs
    among them and with objects inside are found as by the oracle."""
    rng = np.random.default_rng(4)
    n = 3000
    r = np.array([7000.0, 0.0, 0.0]) + rng.uniform(-60, 60, size=(n, 3))
    r[: n // 3, 0] += 1030.0          # x beyond boxMax (8000) by up to ~90 km
    r[n // 3: n // 2, 2] -= 1070.0    # z below boxMin (-1000)
    v = rng.normal(size=(n, 3))
    v *= rng.uniform(0.0, 5.0, size=(n, 1)) / np.linalg.norm(v, axis=1, keepdims=True)
    pop = from_lists(r, v, np.arange(n), np.zeros(n, np.int8), np.full(n, 10.0), np.full(n, 1.0))
    kw = dict(cutoff=20.0, collisionDistanceFactor=2000.0, evasionCutoff=3.0, conjunctionThreshold=2.0,
              boxMin=[6000.0, -1000.0, -1000.0], boxMax=[8000.0, 1000.0, 1000.0])
    cfg = capi.default_config(**kw)
    with capi.Context(cfg) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(10.0)
    opop = to_oracle(oracle, pop)
    p = oracle_params(oracle, cfg, 10.0)
    ref = oracle.scan_cells(opop, p, oracle.make_grid(kw["boxMin"], kw["boxMax"], 0.0, 20.0))
    brute = oracle.scan_bruteforce(opop, p)
    assert records_equal(ref, brute), describe_diff(ref, brute)
    assert len(ref) > 20
    assert records_equal(recs, ref), describe_diff(recs, ref)


@pytest.mark.parametrize("box,cell", [(5.0e5, 0.0), (2.0e5, 2.0)])
def test_coarsened_grid(capi, oracle, box, cell):
    """A box too large for 32-bit cell keys at the requested edge (or for 65535
    cells per axis): the grid is coarsened by 1.25x until it fits, identically
    in the library and the oracle; cell order and records still match the
    oracle and its brute force."""
    rng = np.random.default_rng(11)
    n = 4000
    r = np.array([7000.0, 0.0, 0.0]) + rng.uniform(-150, 150, size=(n, 3))
    v = rng.normal(size=(n, 3))
    v *= rng.uniform(0.0, 5.0, size=(n, 1)) / np.linalg.norm(v, axis=1, keepdims=True)
    pop = from_lists(r, v, np.arange(n), np.zeros(n, np.int8), np.full(n, 10.0), np.full(n, 1.0))
    kw = dict(cutoff=10.0, cellSize=cell, collisionDistanceFactor=2000.0, evasionCutoff=3.0,
              conjunctionThreshold=2.0, boxMin=[-box] * 3, boxMax=[box] * 3)
    cfg = capi.default_config(**kw)
    with capi.Context(cfg) as ctx:
        ctx.upload(pop)
        recs = ctx.conjunctions(10.0)
        keys, slots = ctx.cell_order()
        dims, reach, cell_used = ctx.grid()
    grid = oracle.make_grid(kw["boxMin"], kw["boxMax"], cell, kw["cutoff"])
    assert tuple(grid.n) == dims and grid.reach == reach and grid.cellSize == cell_used
    assert cell_used > 10.0 and max(dims) <= 65535 and int(np.prod(dims, dtype=np.uint64)) <= 1 << 32
    opop = to_oracle(oracle, pop)
    p = oracle_params(oracle, cfg, 10.0)
    ref = oracle.scan_cells(opop, p, grid)
    assert len(ref) > 0
    assert records_equal(recs, ref), describe_diff(recs, ref)
    assert records_equal(ref, oracle.scan_bruteforce(opop, p))
    okeys = oracle.cell_keys(opop, grid)
    operm = oracle.stable_sort(okeys)
    assert np.array_equal(slots, operm) and np.array_equal(keys, okeys[operm])
