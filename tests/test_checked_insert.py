"""Checked insertion of constellation satellites (Simulation::checkedInsert,
Simulation.cpp:475-507) against the reference's own cases
(tests/testladds/SimulationTest.cpp:200-256 and :18-96) and the oracle."""
import numpy as np
import pytest

from helpers import from_lists

P = np.array([6871.0, 0.0, 0.0])  # SimulationTest.h:76
CUTOFF = 0.04                     # SimulationTest.h:77
CORNER = np.array([CUTOFF, CUTOFF, CUTOFF])
# SimulationTest.cpp:236-256: (position of the tested satellite, position is safe)
REFERENCE_CASES = [(P, False), (P + [2 * CUTOFF, 0, 0], True), (P + [CUTOFF, 0, 0], False),
                   (P + 0.6 * CORNER, True), (P + 0.4 * CORNER, False)]


@pytest.mark.parametrize("pos,safe", REFERENCE_CASES)
def test_oracle_reference_cases(oracle, pos, safe):
    delayed = oracle.checked_insert(([P[0]], [P[1]], [P[2]]), ([pos[0]], [pos[1]], [pos[2]]), CUTOFF)
    assert bool(delayed[0]) == (not safe)


@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def one(pos, ident):
    return from_lists([pos], [[0.0, 0.0, 0.0]], [ident], [0], [1.0], [1.0])


@pytest.mark.gpu
@pytest.mark.parametrize("pos,safe", REFERENCE_CASES)
def test_reference_cases_gpu(capi, pos, safe):
    with capi.Context(capi.default_config()) as ctx:
        ctx.upload(one(P, 0))
        delayed = ctx.checked_insert(one(pos, 1), CUTOFF)
        assert bool(delayed[0]) == (not safe)
        assert ctx.size() == (2 if safe else 1)


@pytest.mark.gpu
def test_delayed_insertion_sequence(capi):
    """SimulationTest.cpp:18-96: two satellites one Kepler second apart on the
    same orbit, and copies of both to insert; delayed counts per iteration
    2, 1, 1, 0, 0, 0 while the population advances one step of 1 s each time."""
    p1 = ([6871.0, 0.0, 0.0], [0.0, 4.8958309146899, 5.83462408131549])
    p2 = ([6870.99577848984, 4.89582991243564, 5.83462288687537],
          [-0.00844301944979238, 4.89582790671436, 5.83462049654983])
    initial = from_lists([p1[0], p2[0]], [p1[1], p2[1]], [1, 2], [0, 0], [1.0, 1.0], [1.0, 1.0])
    new = from_lists([p1[0], p2[0]], [p1[1], p2[1]], [1, 4], [0, 0], [1.0, 1.0], [1.0, 1.0])
    cfg = capi.default_config(deltaT=1.0, componentMask=capi.KEP)
    with capi.Context(cfg) as ctx:
        ctx.upload(initial)
        pending = new
        counts = []
        for _ in range(6):
            delayed = ctx.checked_insert(pending, 0.04)
            keep = delayed.astype(bool)
            pending = {k: (v[keep] if isinstance(v, np.ndarray) else v) for k, v in pending.items()}
            counts.append(int(keep.sum()))
            assert ctx.size() == 4 - counts[-1]
            ctx.integrate(1)
    assert counts == [2, 1, 1, 0, 0, 0]


@pytest.mark.gpu
def test_random_batches_match_oracle(capi, oracle):
    rng = np.random.default_rng(23)
    n_old, n_new, c = 20000, 3000, 0.5
    old = np.array([7000.0, 0.0, 0.0]) + rng.uniform(-20, 20, size=(n_old, 3))
    base = old[rng.integers(0, n_old, n_new)]
    new = base + rng.normal(scale=0.4, size=(n_new, 3))  # about half within the cutoff of an existing one
    new[n_new // 2:] = new[: n_new - n_new // 2] + rng.normal(scale=0.3, size=(n_new - n_new // 2, 3))
    new[10:20] = old[:10]  # exactly on existing particles
    new[-1] = new[-2]      # two identical new satellites
    acts = np.zeros(n_old, np.int8)
    pop = from_lists(old, np.zeros_like(old), list(range(n_old)), acts, [1.0] * n_old, [1.0] * n_old)
    batch = from_lists(new, np.zeros_like(new), list(range(n_old, n_old + n_new)), np.zeros(n_new, np.int8),
                       [1.0] * n_new, [1.0] * n_new)
    with capi.Context(capi.default_config()) as ctx:
        ctx.upload(pop)
        ctx.mark_deleted(np.arange(0, n_old, 7, dtype=np.uint32))  # deleted objects do not block
        delayed = ctx.checked_insert(batch, c)
        size = ctx.size()
    dummy = np.zeros(n_old, np.uint8)
    dummy[::7] = 1
    ref = oracle.checked_insert(tuple(old.T), tuple(new.T), c, dummy=dummy)
    assert np.array_equal(delayed, ref)
    assert 0.2 < ref.mean() < 0.9
    assert size == n_old + int(n_new - ref.sum())
