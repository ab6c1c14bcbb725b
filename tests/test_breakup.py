"""Collision breakups on the host (restated NASA standard breakup model) and
their device append, after BreakupWrapperTest.cpp:14-49: the crashed objects
are gone, the fragments have new ids and carry the parent id.  The published
model's laws are checked statistically (parity with the external
esa/NASA-breakup-model-cpp is unpinned: its source is not in the tree)."""
import math

import numpy as np
import pytest

from helpers import from_lists


@pytest.fixture(scope="module")
def capi():
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def obj(capi, r, v, radius, mass, ident):
    o = np.zeros(1, dtype=capi.STATE_RECORD_DTYPE)
    o["r"], o["v"], o["radius"], o["id"] = r, v, radius, ident
    o["aom"] = math.pi * radius ** 2 * 1e-6 / mass
    o["bcInv"] = 2.2 * math.pi * radius ** 2 / mass
    return o


def cfg(capi, min_lc=0.05, conserve=0):
    return capi.BreakupConfig(min_lc, conserve, 2.2)


def test_catastrophic_fragment_count_and_attributes(capi):
    a = obj(capi, [7000.0, 0, 0], [0, 7.5, 0], 0.5, 300.0, 11)
    b = obj(capi, [7000.0, 0, 0], [0, 0, 7.5], 0.3, 100.0, 12)
    frags, nid = capi.breakup_collision(cfg(capi), 5, a, b, [7000.0, 1.0, 2.0], 11, 1000)
    # catastrophic (0.5 * 100 kg * (10.6 km/s)^2 / 300 kg >> 40 J/g): M = 400 kg
    expected = math.floor(0.1 * 400.0 ** 0.75 * (0.05 ** -1.71 - 1.0 ** -1.71))
    n = len(frags["x"])
    assert n == expected and nid == 1000 + n
    assert np.array_equal(frags["id"], np.arange(1000, 1000 + n, dtype=np.uint64))
    assert np.all(frags["parent"] == 11) and np.all(frags["activity"] == 0)
    assert np.all(frags["x"] == 7000.0) and np.all(frags["y"] == 1.0) and np.all(frags["z"] == 2.0)
    lc = 2 * frags["radius"]
    assert lc.min() >= 0.05 and lc.max() <= 1.0
    # Lc power law: P(Lc > 0.1) = (0.1^-1.71 - 1) / (0.05^-1.71 - 1)
    p = (0.1 ** -1.71 - 1) / (0.05 ** -1.71 - 1)
    assert abs(np.mean(lc > 0.1) - p) < 4 * math.sqrt(p * (1 - p) / n)
    # area over mass from aom [km^2/kg] -> chi; delta-v around 0.9 chi + 2.9 (log10 m/s), sigma 0.4
    chi = np.log10(frags["aom"] * 1e6)
    v = np.stack([frags["vx"], frags["vy"], frags["vz"]], 1)
    dv = np.minimum(np.linalg.norm(v - a["v"][0], axis=1), np.linalg.norm(v - b["v"][0], axis=1)) * 1e3
    resid = np.log10(dv) - (0.9 * chi + 2.9)
    assert abs(np.mean(resid)) < 0.05 and abs(np.std(resid) - 0.4) < 0.05
    assert np.allclose(frags["bc_inv"], 2.2 * frags["aom"] * 1e6)


def test_non_catastrophic_and_mass_conservation(capi):
    a = obj(capi, [7000.0, 0, 0], [0, 7.5, 0], 2.0, 2000.0, 1)
    b = obj(capi, [7000.0, 0, 0], [0, 7.5, 0.05], 0.1, 0.01, 2)  # 0.5 * 0.01 * 50^2 / 2000 = 6e-3 J/g
    frags, _ = capi.breakup_collision(cfg(capi, 0.01), 9, a, b, [7000.0, 0, 0], 1, 50)
    expected = math.floor(0.1 * (0.01 * 0.05 ** 2) ** 0.75 * (0.01 ** -1.71 - 4.0 ** -1.71))  # M = mp v^2
    assert len(frags["x"]) == expected
    big = obj(capi, [7000.0, 0, 0], [0, 7.5, 0], 1.0, 50.0, 3)
    frags2, _ = capi.breakup_collision(cfg(capi, 0.01, conserve=1), 2, big, big, [7000.0, 0, 0], 3, 0)
    frags2b, _ = capi.breakup_collision(cfg(capi, 0.01, conserve=0), 2, big, big, [7000.0, 0, 0], 3, 0)
    mass = math.pi * frags2["radius"] ** 2 * 1e-6 / frags2["aom"]
    assert mass.sum() <= 100.0 and len(frags2["x"]) <= len(frags2b["x"])
    again, _ = capi.breakup_collision(cfg(capi, 0.01, conserve=1), 2, big, big, [7000.0, 0, 0], 3, 0)
    assert all(np.array_equal(frags2[k], again[k]) for k in frags2)  # deterministic in the seed


@pytest.mark.gpu
def test_breakup_wrapper_on_the_device(capi):
    """BreakupWrapperTest.cpp:14-49: two particles 1000 km above the Earth whose
    paths cross at [R + 1000, 0, 0]; one iteration with a breakup leaves more
    than two particles, all with ids above the crashed ones."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    R = 6378.137
    pop = from_lists([[R + 1000.0, -1.0, 0.0], [R + 1000.0, 0.0, -1.0]], [[0.0, 2.0, 0.0], [0.0, 0.0, 2.0]], [0, 1],
                     [0, 0], [1.0, 1.0], [1.0, 1.0])
    with capi.Context(capi.default_config(deltaT=1.0, componentMask=capi.KEP, cutoff=80.0,
                                          minDetectionRadius=0.05)) as ctx:
        ctx.upload(pop)
        res = ctx.step(1)
        col = res.records[(res.records["flags"] & capi.PAIR_COLLISION) != 0]
        assert len(col) == 1
        nb, nf, nid = ctx.breakup(res.records, capi.BreakupConfig(0.05, 1, 2.2), 7, 2)
        assert nb == 1 and nf > 2 and nid == 2 + nf
        objs = ctx.get_objects(np.arange(ctx.size(), dtype=np.uint32))
        live = objs[objs["deleted"] == 0]
        assert len(live) == nf and np.all(live["id"] > 1) and np.all(live["parentId"] == 0)
        # the fragments propagate and are scanned with the rest (spawn protection: no records among them)
        after = ctx.step(2)
        assert len(after.records) == 0
