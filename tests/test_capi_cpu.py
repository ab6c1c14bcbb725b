"""CPU-only checks of the C-ABI library: it loads without a GPU, exports every
symbol that include/ladds_gpu.h declares, refuses to create a context without a
device, and its host-side population generator matches a numpy restatement."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def capi():
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def header_functions():
    src = open(os.path.join(ROOT, "include", "ladds_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ladds_\w+)\s*\(", src)))


def test_exports_every_declared_symbol(capi):
    L = capi.lib()
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(capi.EXPORTED)
    assert L.ladds_gpu_abi_version() == 4


def test_config_layout_matches_header(capi):
    cfg = capi.default_config()
    assert cfg.deltaT == 10.0 and cfg.cutoff == 80.0 and cfg.timestepsPerCollisionDetection == 1
    assert cfg.minDetectionRadius == 0.05 and cfg.evasionCutoff == 0.1
    assert list(cfg.boxMin) == [-10000.0] * 3 and list(cfg.boxMax) == [10000.0] * 3


def test_create_without_gpu_is_an_error_not_a_crash(capi):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(capi.LaddsError) as e:
        capi.Context()
    assert e.value.code == capi.ERR_NO_DEVICE


# ---------------- numpy restatement of the population generator ----------------
M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix(x):
    x = x + np.uint64(0x9E3779B97F4A7C15)
    z = x
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x, z ^ (z >> np.uint64(31))


def _rotl(x, k):
    return (x << np.uint64(k)) | (x >> np.uint64(64 - k))


class NpRng:
    def __init__(self, seed, k):
        with np.errstate(over="ignore"):
            x = np.uint64(seed) ^ (k.astype(np.uint64) * np.uint64(0xD1B54A32D192ED03))
            self.s = []
            for _ in range(4):
                x, z = _splitmix(x)
                self.s.append(z)

    def next(self):
        s = self.s
        with np.errstate(over="ignore"):
            result = _rotl(s[1] * np.uint64(5), 7) * np.uint64(9)
            t = s[1] << np.uint64(17)
            s[2] = s[2] ^ s[0]
            s[3] = s[3] ^ s[1]
            s[1] = s[1] ^ s[2]
            s[0] = s[0] ^ s[3]
            s[2] = s[2] ^ t
            s[3] = _rotl(s[3], 45)
        return result

    def uniform(self):
        return (self.next() >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def np_elements_to_state(a, e, inc, raan, argp, M, mu=398600.4418):
    E = M.copy()
    for _ in range(50):
        dE = (E - e * np.sin(E) - M) / (1.0 - e * np.cos(E))
        E = E - dE
    cE, sE = np.cos(E), np.sin(E)
    b = np.sqrt(1 - e * e)
    xp, yp = a * (cE - e), a * b * sE
    n = np.sqrt(mu / a ** 3)
    Ed = n / (1 - e * cE)
    vxp, vyp = -a * sE * Ed, a * b * cE * Ed
    cO, sO, cw, sw, ci, si = np.cos(raan), np.sin(raan), np.cos(argp), np.sin(argp), np.cos(inc), np.sin(inc)
    P = np.stack([cO * cw - sO * sw * ci, sO * cw + cO * sw * ci, sw * si], 1)
    Q = np.stack([-cO * sw - sO * cw * ci, -sO * sw + cO * cw * ci, cw * si], 1)
    return xp[:, None] * P + yp[:, None] * Q, vxp[:, None] * P + vyp[:, None] * Q


def np_population0(seed, n):
    g = NpRng(seed, np.arange(n, dtype=np.uint64))
    h = 400 + 1100 * g.uniform()
    e = 0.02 * g.uniform()
    inc = math.pi * g.uniform()
    raan = 2 * math.pi * g.uniform()
    argp = 2 * math.pi * g.uniform()
    M = 2 * math.pi * g.uniform()
    radius = np.exp(np.log(0.01) + (np.log(5.0) - np.log(0.01)) * g.uniform())
    r, v = np_elements_to_state(6378.137 + h, e, inc, raan, argp, M)
    mass = 2700 * 4 / 3 * math.pi * radius ** 3
    return r, v, radius, mass


def test_population0_matches_numpy_restatement(capi):
    n = 2000
    pop = capi.generate_population(0, 1000, n)
    r, v, radius, mass = np_population0(1000, n)
    np.testing.assert_allclose(pop["radius"], radius, rtol=1e-14)
    np.testing.assert_allclose(np.stack([pop["x"], pop["y"], pop["z"]], 1), r, rtol=0, atol=1e-8)
    np.testing.assert_allclose(np.stack([pop["vx"], pop["vy"], pop["vz"]], 1), v, rtol=0, atol=1e-11)
    np.testing.assert_allclose(pop["aom"], math.pi * radius ** 2 * 1e-6 / mass, rtol=1e-14)
    np.testing.assert_allclose(pop["bc_inv"], 2.2 * math.pi * radius ** 2 / mass, rtol=1e-14)
    assert np.array_equal(pop["id"], np.arange(n, dtype=np.uint64))
    assert np.all(pop["parent"] == capi.SIZE_MAX) and np.all(pop["activity"] == 0)
    # distribution sanity: altitude of the semi-major axis in [400, 1500], radii in [0.01, 5]
    rn = np.linalg.norm(r, axis=1)
    assert rn.min() > 6378.137 + 400 * 0.97 - 200 and rn.max() < 6378.137 + 1500 + 200
    assert radius.min() >= 0.01 and radius.max() <= 5.0


def test_population_slices_are_independent(capi):
    a = capi.generate_population(0, 7, 1000)
    b = capi.generate_population(0, 7, 500)
    assert np.array_equal(a["x"][:500], b["x"])


def test_population2_shells(capi):
    pop = capi.generate_population(2, 1002, 6000)
    sats = 4224
    assert np.all(pop["activity"][:sats] == capi.EVASIVE) and np.all(pop["activity"][sats:] == capi.PASSIVE)
    alt = np.linalg.norm(np.stack([pop["x"], pop["y"], pop["z"]], 1), axis=1) - 6378.137
    shells = [(0, 1584, 550), (1584, 2304, 570), (2304, 3024, 1200), (3024, 4224, 1325)]
    for a, b, h in shells:
        np.testing.assert_allclose(alt[a:b], h, atol=1e-6)


def test_population4_mixture(capi):
    pop = capi.generate_population(4, 1004, 40000)
    n_small = 40000 - 40000 // 16
    alt = np.linalg.norm(np.stack([pop["x"], pop["y"], pop["z"]], 1), axis=1) - 6378.137
    assert pop["radius"][:n_small].max() <= 0.1 and pop["radius"][:n_small].min() >= 0.01
    a_small = alt[:n_small]
    # elements are drawn in [300, 2000] km for a; e <= 0.02 moves |r| by at most ~170 km
    assert a_small.min() > 300 - 180 and a_small.max() < 2000 + 180
    frac_low = np.mean(a_small < 1100)
    assert 0.45 < frac_low < 0.55


def test_elements_to_state_energy(capi):
    a, e = 7000.0, 0.01
    r, v = capi.elements_to_state(a, e, 0.3, 0.2, 0.1, 1.0)
    energy = 0.5 * v @ v - 398600.4418 / np.linalg.norm(r)
    assert abs(energy - (-398600.4418 / (2 * a))) < 1e-9
