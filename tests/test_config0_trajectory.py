"""End-to-end parity on the plain FP64 CPU-runnable workload: GPU and oracle
run independently from the same upload and are compared at every step.

Workload: 10,000 objects of population 0 (a = R + U[400, 1500] km, e U[0, 0.02],
i U[0, 180] deg, radius logU[0.01, 5] m), central body + J2, FP64, dt 10 s,
100 iterations, the conjunction scan after every integration (the loop of
Simulation.cpp:297, :389-397), 80 km cutoff.

The GPU runs its own trajectory (one ladds_gpu_step call per iteration), the
oracle its own (oracle_propagate + oracle_scan_cells, C restatement of the
Yoshida step and of CollisionFunctor::AoSFunctor).  The two trajectories agree
to about 1e-12 km, not bit for bit (the GPU's force evaluation uses fused
multiply-adds), so every iteration is compared as follows:

* cell-sort order: keys and object order identical (a cell boundary within
  1e-12 km of an object would be the only excuse, and none occurs);
* record set: the same (step, idA, idB) keys with the same list bits
  (collision / evasion / conjunction); a pair may differ only if either run
  flags it in the 1e-9-relative near band of the threshold it crosses or of
  the cutoff gate (CollisionFunctor.cpp:75, :85, :90, :112; such pairs are
  listed separately);
* record values: dl^2 and the point within 1e-8 km of the oracle's (the
  trajectories' own difference), final positions within 1e-6 km.

Two threshold settings: the workload's 0.1 km (few or no records at this
density), and a conjunction threshold of 80 km, under which every pair that
passes the cutoff gate is a record -- the whole gated pair set of every
iteration is then compared.
"""
import numpy as np
import pytest

from helpers import to_oracle

pytestmark = pytest.mark.gpu

N_OBJECTS, STEPS, DT = 10_000, 100, 10.0
LIST_BITS = 1 | 2 | 4  # collision, evasion, conjunction
NEAR_BITS = 8 | 16 | 32 | 64  # their near bands and the cutoff gate's


@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def by_key(recs):
    return {(int(r["step"]), int(r["idA"]), int(r["idB"])): r for r in recs}


def compare_iteration(got, ref, step):
    """Record sets of one iteration: equal outside the near bands, values
    within the trajectories' difference.  Returns the number of near-band
    pairs that differ in membership or list bits."""
    g, o = by_key(got), by_key(ref)
    excused = 0
    for k in set(g) | set(o):
        a, b = g.get(k), o.get(k)
        near = any(r is not None and int(r["flags"]) & NEAR_BITS for r in (a, b))
        if a is None or b is None:
            assert near, f"iteration {step}: pair {k} only in {'oracle' if a is None else 'GPU'} and not near"
            excused += 1
            continue
        if (int(a["flags"]) & LIST_BITS) != (int(b["flags"]) & LIST_BITS):
            assert near, f"iteration {step}: pair {k} flags {int(a['flags'])} vs {int(b['flags'])}"
            excused += 1
        assert int(a["slotA"]) == int(b["slotA"]) and int(a["slotB"]) == int(b["slotB"])
        dlg, dlo = np.sqrt(float(a["dl2"])), np.sqrt(float(b["dl2"]))
        assert abs(dlg - dlo) <= 1e-8, (step, k, dlg, dlo)
        assert np.max(np.abs(a["point"] - b["point"])) <= 1e-8, (step, k)
    return excused


@pytest.mark.parametrize("threshold_km", [0.1, 80.0])
def test_config0_independent_trajectories(capi, oracle, threshold_km):
    mask = capi.KEP | capi.J2
    pop = capi.generate_population(0, 1000, N_OBJECTS)
    cfg = capi.default_config(componentMask=mask, precision=capi.PRECISION_FP64, deltaT=DT,
                              conjunctionThreshold=threshold_km)
    gpu = []
    with capi.Context(cfg) as ctx:
        ctx.upload(pop)
        for _ in range(STEPS):
            res = ctx.step(1)
            keys, slots = ctx.cell_order()
            gpu.append((res.records.copy(), keys, slots))
        final = ctx.download()

    grid = oracle.make_grid(list(cfg.boxMin), list(cfg.boxMax), cfg.cellSize, cfg.cutoff)
    params = oracle.scan_params(cutoff=cfg.cutoff, dt=DT, factor=cfg.collisionDistanceFactor,
                                min_detection_radius=cfg.minDetectionRadius, evasion_cutoff=cfg.evasionCutoff,
                                conjunction_threshold=threshold_km, near_rel=cfg.nearThresholdRel)
    opop = to_oracle(oracle, pop)
    total_records = excused = 0
    for s in range(STEPS):
        oracle.propagate(opop, mask, DT, 1, t0=DT * s)
        ref = oracle.scan_cells(opop, params, grid, step=s)
        okeys = oracle.cell_keys(opop, grid)
        operm = oracle.stable_sort(okeys)
        recs, keys, slots = gpu[s]
        assert np.array_equal(slots, operm), f"cell order differs at iteration {s}"
        assert np.array_equal(keys, okeys[operm]), f"cell keys differ at iteration {s}"
        excused += compare_iteration(recs, ref, s)
        total_records += len(ref)
    rg = np.stack([final["x"], final["y"], final["z"]], 1)
    ro = np.stack([opop.x, opop.y, opop.z], 1)
    assert np.max(np.abs(rg - ro)) < 1e-6
    if threshold_km == 80.0:
        # the gated pair set: about 140 pairs per iteration at this density
        assert total_records > 50 * STEPS, total_records
    assert excused <= max(1, total_records // 10000)
