"""Adjoint of the propagation for conjunction pairs.

Checks: the oracle's tangent-linear (forward-mode) loss derivative against
central finite differences (CPU); the GPU forward loss against the oracle; the
GPU adjoint gradient against the tangent-linear reference and against central
finite differences (h = 1e-6 relative, with its Richardson extrapolation);
checkpoint-interval invariance; a directional finite-difference check of all
pairs at the benchmark size (4096 pairs, 1080 steps) through the GPU forward.

Tolerances: gradient vs tangent-linear 1e-7 relative (norm over the 12 state
components; the two sides propagate with different rounding); vs Richardson-
extrapolated central differences 1e-6; the plain h = 1e-6 central difference
carries a truncation error of up to ~1e-4 relative on these pairs (it converges
to the tangent-linear value as h shrinks), so it is held to 1e-4.
"""
import numpy as np
import pytest

STEPS = 1080
DT = 10.0


def pairs16(capi_pairs):
    """ADJ_PAIR_DTYPE records -> (P, 16) rows of the oracle."""
    p = capi_pairs
    return np.concatenate([p["rA"], p["vA"], p["rB"], p["vB"], p["bcInvA"][:, None], p["bcInvB"][:, None],
                           p["aomA"][:, None], p["aomB"][:, None]], axis=1)


def to_records(rows, capi):
    out = np.zeros(len(rows), dtype=capi.ADJ_PAIR_DTYPE)
    out["rA"], out["vA"], out["rB"], out["vB"] = rows[:, 0:3], rows[:, 3:6], rows[:, 6:9], rows[:, 9:12]
    out["bcInvA"], out["bcInvB"], out["aomA"], out["aomB"] = rows[:, 12], rows[:, 13], rows[:, 14], rows[:, 15]
    return out


def tangent_gradient(oracle, rows, steps, mask):
    n = len(rows)
    g = np.zeros((n, 14))
    for k in range(14):
        d = np.zeros((n, 14))
        d[:, k] = 1.0
        g[:, k] = oracle.pair_losses(rows, steps, dt=DT, mask=mask, dirs=d)[2]
    return g


def central_fd(oracle, rows, steps, mask, rel, comps=range(12), with_stable=False):
    """Central differences with step rel * |x_k|; with_stable also returns, per
    pair, whether every perturbed evaluation kept the unperturbed argmin step
    (the min over steps is smooth only while its argmin stays put)."""
    out = np.zeros((len(rows), len(comps)))
    arg0 = oracle.pair_losses(rows, steps, dt=DT, mask=mask)[1]
    stable = np.ones(len(rows), dtype=bool)
    for i, k in enumerate(comps):
        h = rel * np.abs(rows[:, k])
        up, dn = rows.copy(), rows.copy()
        up[:, k] += h
        dn[:, k] -= h
        mu, au, _ = oracle.pair_losses(up, steps, dt=DT, mask=mask)
        md, ad, _ = oracle.pair_losses(dn, steps, dt=DT, mask=mask)
        out[:, i] = (mu - md) / (2 * h)
        stable &= (au == arg0) & (ad == arg0)
    return (out, stable) if with_stable else out


def rel_norm(a, b):
    return np.linalg.norm(a - b, axis=-1) / np.linalg.norm(b, axis=-1)


# ------------------------------------------------------------------ CPU only
def oracle_pairs(oracle, n, steps, seed):
    """A from population-0-like elements, B = A + offset at steps / 2, back-propagated (oracle)."""
    from ladds_b200 import capi

    pop = capi.generate_population(0, seed, 2 * n)
    rng = np.random.default_rng(seed)
    rows = np.zeros((n, 16))
    keys = ("x", "y", "z", "vx", "vy", "vz", "radius", "aom", "bc_inv")
    for p in range(n):
        a, b = 2 * p, 2 * p + 1
        A = oracle.Population(*[pop[k][a:a + 1].copy() for k in keys])
        half = steps // 2
        oracle.propagate(A, oracle.FULL, DT, half)
        dr = rng.normal(size=3)
        dr *= rng.uniform(0.05, 2.0) / np.linalg.norm(dr)
        dv = rng.normal(size=3)
        dv *= rng.uniform(0.01, 0.5) / np.linalg.norm(dv)
        B = oracle.Population(A.x + dr[0], A.y + dr[1], A.z + dr[2], A.vx + dv[0], A.vy + dv[1], A.vz + dv[2],
                              pop["radius"][b:b + 1], pop["aom"][b:b + 1], pop["bc_inv"][b:b + 1])
        oracle.propagate(B, oracle.FULL, -DT, half, t0=DT * half)
        rows[p, 0:6] = [pop[k][a] for k in keys[:6]]
        rows[p, 6:12] = [B.x[0], B.y[0], B.z[0], B.vx[0], B.vy[0], B.vz[0]]
        rows[p, 12:16] = [pop["bc_inv"][a], pop["bc_inv"][b], pop["aom"][a], pop["aom"][b]]
    return rows


def test_oracle_tangent_linear_matches_finite_differences(oracle):
    rows = oracle_pairs(oracle, 3, 300, seed=5)
    miss, tca, _ = oracle.pair_losses(rows, 300, dt=DT)
    assert np.all(tca > 100) and np.all(miss < 5.0)  # close approaches near the middle
    g = tangent_gradient(oracle, rows, 300, oracle.FULL)[:, :12]
    fd1 = central_fd(oracle, rows, 300, oracle.FULL, 1e-6)
    fd2 = central_fd(oracle, rows, 300, oracle.FULL, 5e-7)
    rich = (4.0 * fd2 - fd1) / 3.0
    assert np.all(rel_norm(g, rich) < 1e-6), rel_norm(g, rich)
    assert np.all(rel_norm(g, fd1) < 1e-4), rel_norm(g, fd1)


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


@pytest.fixture(scope="module")
def gpu_pairs(capi):
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        pairs, tca = ctx.adjoint_make_pairs(2024, 64, STEPS)
    return pairs, tca


@pytest.mark.gpu
def test_made_pairs_meet_near_the_planned_step(capi, gpu_pairs):
    pairs, tca = gpu_pairs
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        loss, miss, step, ms = ctx.adjoint_forward(pairs, STEPS)
    # the minimum is at the planned step unless the two orbits pass closer at another crossing
    assert np.mean(np.abs(step - tca) <= 1) > 0.7
    assert np.all(np.sqrt(miss) < 2.05)
    assert loss == pytest.approx(float(np.sum(miss)), rel=1e-12)


@pytest.mark.gpu
def test_adjoint_forward_matches_oracle(capi, oracle, gpu_pairs):
    pairs, _ = gpu_pairs
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        _, miss, step, _ = ctx.adjoint_forward(pairs, STEPS)
    omiss, ostep, _ = oracle.pair_losses(pairs16(pairs), STEPS, dt=DT)
    assert np.array_equal(step, ostep)
    assert np.max(np.abs(miss - omiss) / omiss) < 1e-6


@pytest.mark.gpu
def test_adjoint_gradient_matches_tangent_linear(capi, oracle, gpu_pairs):
    pairs, _ = gpu_pairs
    pairs = pairs[:32]
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        ctx.adjoint_forward(pairs, STEPS, 64)
        dx, dbc, _ = ctx.adjoint_backward()
    g = tangent_gradient(oracle, pairs16(pairs), STEPS, oracle.FULL)
    assert np.all(rel_norm(dx, g[:, :12]) < 1e-7), rel_norm(dx, g[:, :12])
    # the drag sensitivities are tiny at these altitudes; compare them on their own scale
    scale = np.maximum(np.abs(g[:, 12:]), 1e-30)
    assert np.all(np.abs(dbc - g[:, 12:]) / scale < 1e-5), np.abs(dbc - g[:, 12:]) / scale


@pytest.mark.gpu
def test_adjoint_gradient_matches_central_differences(capi, oracle, gpu_pairs):
    """Pairs whose finite-difference stencil keeps the argmin step: the loss is
    smooth there and the differences converge to the gradient.  (Where two
    adjacent steps give nearly the same minimum the stencil switches between
    them and the difference quotient carries an O(h) kink error instead.)"""
    pairs, _ = gpu_pairs
    pairs = pairs[:8]
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        ctx.adjoint_forward(pairs, STEPS, 64)
        dx, _, _ = ctx.adjoint_backward()
    rows = pairs16(pairs)
    fd1, st1 = central_fd(oracle, rows, STEPS, oracle.FULL, 1e-6, with_stable=True)
    fd2, st2 = central_fd(oracle, rows, STEPS, oracle.FULL, 5e-7, with_stable=True)
    smooth = st1 & st2
    assert np.sum(smooth) >= 4, smooth
    rich = (4.0 * fd2 - fd1) / 3.0
    assert np.all(rel_norm(dx, rich)[smooth] < 1e-6), rel_norm(dx, rich)
    assert np.all(rel_norm(dx, fd1)[smooth] < 1e-4), rel_norm(dx, fd1)


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_the_gradient(capi, gpu_pairs):
    pairs, _ = gpu_pairs
    pairs = pairs[:16]
    grads = []
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        for ck in (1, 7, 64, STEPS):
            ctx.adjoint_forward(pairs, STEPS, ck)
            dx, dbc, _ = ctx.adjoint_backward()
            grads.append((dx.copy(), dbc.copy()))
    for dx, dbc in grads[1:]:
        assert np.array_equal(dx, grads[0][0]) and np.array_equal(dbc, grads[0][1])


@pytest.mark.gpu
def test_adjoint_directional_fd_at_benchmark_size(capi):
    """All 4096 pairs, 1080 steps: g . d against finite differences of the GPU
    forward loss along a random direction d of the 12 state components (each
    pair its own direction), h = 1e-6 |x| with h/2 and h/4 for Richardson
    extrapolation; the perturbed pairs run as extra pairs of one forward batch.
    The loss is a minimum over steps and over the clamped closest-approach time,
    so stencils can straddle a kink; bench.fd_classify takes, per pair, the
    side(s) whose points keep the argmin step (central if both agree)."""
    import bench

    n = 4096
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        pairs, _ = ctx.adjoint_make_pairs(77, n, STEPS)
        ctx.adjoint_forward(pairs, STEPS, 64)
        dx, _, _ = ctx.adjoint_backward()
        rows = pairs16(pairs)
        rng = np.random.default_rng(3)
        d = rng.normal(size=(n, 12)) * np.abs(rows[:, :12])  # relative scale per component
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        eps = 1e-6 * np.linalg.norm(rows[:, :12], axis=1)
        batch = []
        for f in bench.FD_STENCIL:
            r = rows.copy()
            r[:, :12] += f * eps[:, None] * d
            batch.append(r)
        _, miss, step, _ = ctx.adjoint_forward(to_records(np.concatenate(batch), capi), STEPS, 64)
        _, miss0, step0, _ = ctx.adjoint_forward(pairs, STEPS, 64)
    k = len(bench.FD_STENCIL)
    rel, counts = bench.fd_classify(np.sum(dx * d, axis=1), miss0, miss.reshape(k, n), step0,
                                    step.reshape(k, n), eps)
    resolved = np.isfinite(rel)
    # a stencil side that keeps the argmin step and is smooth exists for most pairs
    assert np.mean(resolved) > 0.8, counts
    assert np.median(rel[resolved]) < 1e-7, np.median(rel[resolved])
    # where both sides agree (no kink within the stencil) the gradient meets 1e-6
    assert counts["central"] > n // 2, counts
    assert counts["central_meeting_tol"] >= 0.99 * counts["central"], counts


@pytest.mark.gpu
def test_adjoint_edge_cases(capi):
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL)) as ctx:
        with pytest.raises(capi.LaddsError):  # no forward sweep yet
            ctx.adjoint_backward()
        pairs, _ = ctx.adjoint_make_pairs(9, 3, 200)
        pairs["rB"][1] = pairs["rA"][1]  # identical objects: the reference's 0/0 path, NaN at every step
        pairs["vB"][1] = pairs["vA"][1]
        pairs["bcInvB"][1] = pairs["bcInvA"][1]
        pairs["aomB"][1] = pairs["aomA"][1]
        loss, miss, step, _ = ctx.adjoint_forward(pairs, 200, 64)
        dx, dbc, _ = ctx.adjoint_backward()
    assert step[1] == 0 and not np.isfinite(miss[1])
    assert np.all(dx[1] == 0) and np.all(dbc[1] == 0)
    assert np.isfinite(loss) and loss == pytest.approx(miss[0] + miss[2], rel=1e-12)
    assert np.all(np.isfinite(dx)) and np.any(dx[0] != 0)
