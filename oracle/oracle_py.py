"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/ and ``__graft_entry__.smoke()`` to
check the GPU results, and by ``bench.py``'s CPU-baseline leg.  The product library never
imports this module.  See ``ladds_oracle.h`` for what each function restates
and for its parity status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

KEP, J2, C22, S22, SOL, LUN, SRP, DRAG, J3 = (1 << k for k in range(9))
FULL = KEP | J2 | C22 | S22 | SOL | LUN | SRP | DRAG | J3
PASSIVE, EVASIVE, EVASIVE_PRESERVING = 0, 1, 2
FLAG_COLLISION, FLAG_EVASION, FLAG_CONJUNCTION = 1, 2, 4
FLAG_NEAR_COLLISION, FLAG_NEAR_EVASION, FLAG_NEAR_CONJUNCTION, FLAG_NEAR_GATE = 8, 16, 32, 64
SIZE_MAX = np.uint64(0xFFFFFFFFFFFFFFFF)
JD_EPOCH_2022 = 2459580.5

PAIR_DTYPE = np.dtype(
    [
        ("idA", "<u8"),
        ("idB", "<u8"),
        ("slotA", "<u4"),
        ("slotB", "<u4"),
        ("dl2", "<f8"),
        ("point", "<f8", (3,)),
        ("step", "<u4"),
        ("flags", "<u4"),
    ]
)
assert PAIR_DTYPE.itemsize == 64


class ScanParams(C.Structure):
    _fields_ = [
        ("cutoff", C.c_double),
        ("dt", C.c_double),
        ("collisionDistanceFactor", C.c_double),
        ("minDetectionRadius", C.c_double),
        ("evasionCutoff", C.c_double),
        ("conjunctionThreshold", C.c_double),
        ("nearRel", C.c_double),
    ]


class Grid(C.Structure):
    _fields_ = [
        ("boxMin", C.c_double * 3),
        ("cellSize", C.c_double),
        ("invCell", C.c_double),
        ("n", C.c_int32 * 3),
        ("reach", C.c_int32),
    ]


class Ephem(C.Structure):
    _fields_ = [("sun", C.c_double * 3), ("moon", C.c_double * 3), ("cosT", C.c_double), ("sinT", C.c_double)]


def build() -> None:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.oracle_interpolate.argtypes = [dp, dp, dp, dp, C.c_double, dp, dp]
        L.oracle_functor_pair.restype = C.c_uint32
        L.oracle_functor_pair.argtypes = [
            C.POINTER(ScanParams), dp, dp, C.c_double, C.c_int, C.c_uint64,
            dp, dp, C.c_double, C.c_int, C.c_uint64, dp, dp,
        ]
        L.oracle_scan_bruteforce.restype = C.c_size_t
        L.oracle_scan_bruteforce.argtypes = [C.c_size_t] + [C.c_void_p] * 11 + [
            C.POINTER(ScanParams), C.c_uint32, C.c_void_p, C.c_size_t]
        L.oracle_make_grid.argtypes = [dp, dp, C.c_double, C.c_double, C.POINTER(Grid)]
        L.oracle_cell_keys.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Grid), C.c_void_p]
        L.oracle_stable_sort.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p]
        L.oracle_scan_cells.restype = C.c_size_t
        L.oracle_scan_cells.argtypes = [C.c_size_t] + [C.c_void_p] * 11 + [
            C.POINTER(ScanParams), C.POINTER(Grid), C.c_uint32, C.c_void_p, C.c_size_t, C.c_int]
        L.oracle_sort_pairs.argtypes = [C.c_size_t, C.c_void_p]
        L.oracle_gmst0.restype = C.c_double
        L.oracle_gmst0.argtypes = [C.c_double]
        L.oracle_ephemeris.argtypes = [C.c_double, C.c_double, C.c_double, C.POINTER(Ephem)]
        L.oracle_accel.argtypes = [C.c_uint32, C.c_int, dp, dp, C.c_double, C.c_double, C.POINTER(Ephem), dp]
        L.oracle_propagate.argtypes = [C.c_size_t] + [C.c_void_p] * 10 + [
            C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]
        L.oracle_pair_losses.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_double,
                                         C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_checked_insert.restype = C.c_size_t
        L.oracle_checked_insert.argtypes = [C.c_size_t] + [C.c_void_p] * 4 + [C.c_size_t] + [C.c_void_p] * 3 + [
            C.c_double, C.c_void_p]
        L.oracle_density.restype = C.c_double
        L.oracle_density.argtypes = [C.c_double]
        _lib = L
    return _lib


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def scan_params(cutoff=80.0, dt=10.0, factor=1.0, min_detection_radius=0.05, evasion_cutoff=0.1,
                conjunction_threshold=0.1, near_rel=1e-9) -> ScanParams:
    return ScanParams(cutoff, dt, factor, min_detection_radius, evasion_cutoff, conjunction_threshold, near_rel)


def interpolate(ri, vi, rj, vj, dt):
    dr = np.zeros(3)
    p2 = np.zeros(3)
    lib().oracle_interpolate(_dp(ri), _dp(vi), _dp(rj), _dp(vj), dt, _dp(dr), _dp(p2))
    return dr, p2


def functor_pair(params, ri, vi, rad_i, act_i, parent_i, rj, vj, rad_j, act_j, parent_j):
    dl2 = np.zeros(1)
    point = np.zeros(3)
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (ri, vi, rj, vj)]
    f = lib().oracle_functor_pair(C.byref(params), _dp(a[0]), _dp(a[1]), rad_i, act_i, int(parent_i),
                                  _dp(a[2]), _dp(a[3]), rad_j, act_j, int(parent_j), _dp(dl2), _dp(point))
    return int(f), float(dl2[0]), point


class Population:
    """Plain SoA numpy population (host side of the oracle)."""

    def __init__(self, x, y, z, vx, vy, vz, radius, aom, bc_inv, ids=None, parent=None, activity=None, dummy=None):
        n = len(x)
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        self.x, self.y, self.z = f(x), f(y), f(z)
        self.vx, self.vy, self.vz = f(vx), f(vy), f(vz)
        self.radius, self.aom, self.bc_inv = f(radius), f(aom), f(bc_inv)
        self.id = np.ascontiguousarray(np.arange(n, dtype=np.uint64) if ids is None else ids, dtype=np.uint64)
        self.parent = np.ascontiguousarray(np.full(n, SIZE_MAX, dtype=np.uint64) if parent is None else parent,
                                           dtype=np.uint64)
        self.activity = np.ascontiguousarray(np.zeros(n, np.int8) if activity is None else activity, dtype=np.int8)
        self.dummy = np.ascontiguousarray(np.zeros(n, np.uint8) if dummy is None else dummy, dtype=np.uint8)

    @property
    def n(self):
        return len(self.x)

    def copy(self):
        return Population(self.x.copy(), self.y.copy(), self.z.copy(), self.vx.copy(), self.vy.copy(),
                          self.vz.copy(), self.radius.copy(), self.aom.copy(), self.bc_inv.copy(), self.id.copy(),
                          self.parent.copy(), self.activity.copy(), self.dummy.copy())

    def _scan_args(self):
        return [_ptr(a) for a in (self.x, self.y, self.z, self.vx, self.vy, self.vz, self.radius, self.id,
                                  self.parent, self.activity, self.dummy)]


def scan_bruteforce(pop: Population, params: ScanParams, step=0, cap=None):
    cap = cap if cap is not None else max(1024, pop.n * 4)
    out = np.zeros(cap, dtype=PAIR_DTYPE)
    n = lib().oracle_scan_bruteforce(pop.n, *pop._scan_args(), C.byref(params), step, _ptr(out), cap)
    assert n <= cap, "oracle pair buffer too small"
    out = out[:n].copy()
    lib().oracle_sort_pairs(n, _ptr(out))
    return out


def make_grid(box_min, box_max, cell_size, cutoff) -> Grid:
    g = Grid()
    lib().oracle_make_grid(_dp(np.asarray(box_min, float)), _dp(np.asarray(box_max, float)), cell_size, cutoff,
                           C.byref(g))
    return g


def cell_keys(pop: Population, grid: Grid):
    keys = np.zeros(pop.n, dtype=np.uint32)
    lib().oracle_cell_keys(pop.n, _ptr(pop.x), _ptr(pop.y), _ptr(pop.z), C.byref(grid), _ptr(keys))
    return keys


def stable_sort(keys):
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    perm = np.zeros(len(keys), dtype=np.uint32)
    lib().oracle_stable_sort(len(keys), _ptr(keys), _ptr(perm))
    return perm


def scan_cells(pop: Population, params: ScanParams, grid: Grid, step=0, cap=None, nthreads=0):
    cap = cap if cap is not None else max(1024, pop.n * 4)
    out = np.zeros(cap, dtype=PAIR_DTYPE)
    n = lib().oracle_scan_cells(pop.n, *pop._scan_args(), C.byref(params), C.byref(grid), step, _ptr(out), cap,
                                nthreads)
    if n > cap:
        return scan_cells(pop, params, grid, step, cap=n, nthreads=nthreads)
    return out[:n].copy()


def gmst0(jd_epoch=JD_EPOCH_2022):
    return lib().oracle_gmst0(jd_epoch)


def ephemeris(tau, jd_epoch=JD_EPOCH_2022):
    e = Ephem()
    lib().oracle_ephemeris(jd_epoch, gmst0(jd_epoch), tau, C.byref(e))
    return e


def accel(mask, activity, r, v, aom, bc_inv, eph: Ephem):
    a = np.zeros(3)
    lib().oracle_accel(mask, activity, _dp(r), _dp(v), aom, bc_inv, C.byref(eph), _dp(a))
    return a


def density(h):
    return lib().oracle_density(h)


def propagate(pop: Population, mask, dt, steps, t0=0.0, jd_epoch=JD_EPOCH_2022, nthreads=0):
    """Propagate ``pop`` in place by ``steps`` Yoshida-4 steps."""
    lib().oracle_propagate(pop.n, _ptr(pop.x), _ptr(pop.y), _ptr(pop.z), _ptr(pop.vx), _ptr(pop.vy), _ptr(pop.vz),
                           _ptr(pop.aom), _ptr(pop.bc_inv), _ptr(pop.activity), _ptr(pop.dummy), mask, jd_epoch,
                           t0, dt, steps, nthreads)


def pair_losses(pairs, steps, dt=10.0, mask=FULL, dirs=None, t0=0.0, jd_epoch=JD_EPOCH_2022, nthreads=0):
    """Per-pair min over steps of the squared interpolated miss distance, its
    step, and (with dirs, 14 per pair) its tangent-linear derivative along dirs.
    pairs: (P, 16) float64 = rA, vA, rB, vB, bcInvA, bcInvB, aomA, aomB."""
    pairs = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1, 16)
    n = len(pairs)
    miss = np.zeros(n)
    tca = np.zeros(n, dtype=np.int32)
    dmiss = np.zeros(n) if dirs is not None else None
    d = None if dirs is None else np.ascontiguousarray(dirs, dtype=np.float64).reshape(n, 14)
    lib().oracle_pair_losses(n, _ptr(pairs), _ptr(d), mask, jd_epoch, t0, dt, steps, _ptr(miss), _ptr(tca),
                             _ptr(dmiss), nthreads)
    return miss, tca, dmiss


def checked_insert(existing_xyz, new_xyz, cutoff, dummy=None):
    """Simulation::checkedInsert restated: delayed flags of the new satellites."""
    ex = [np.ascontiguousarray(a, dtype=np.float64) for a in existing_xyz]
    nw = [np.ascontiguousarray(a, dtype=np.float64) for a in new_xyz]
    delayed = np.zeros(len(nw[0]), dtype=np.uint8)
    d = None if dummy is None else np.ascontiguousarray(dummy, dtype=np.uint8)
    lib().oracle_checked_insert(len(ex[0]), _ptr(ex[0]), _ptr(ex[1]), _ptr(ex[2]), _ptr(d), len(nw[0]),
                                _ptr(nw[0]), _ptr(nw[1]), _ptr(nw[2]), cutoff, _ptr(delayed))
    return delayed
