"""Synthetic populations and population files, host only.

ctypes binding of ``libladds_population.so``: the population generator, the
binary SoA population file and the element conversion of
``ladds_b200/csrc/population.cpp`` compiled with g++ alone (no CUDA), so that
a process that only needs populations -- the benchmark's CPU reference arm --
loads no GPU code.  ``ladds_b200.capi`` re-exports these functions.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libladds_population.so")

OK, ERR_INVALID_ARG, ERR_CAPACITY = 0, 1, 3

POP_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "radius", "aom", "bc_inv", "id", "parent", "activity")
_POP_DTYPES = dict(x=np.float64, y=np.float64, z=np.float64, vx=np.float64, vy=np.float64, vz=np.float64,
                   radius=np.float64, aom=np.float64, bc_inv=np.float64, id=np.uint64, parent=np.uint64,
                   activity=np.int8)
SIZE_MAX = np.uint64(0xFFFFFFFFFFFFFFFF)

EXPORTED = ["ladds_population_generate", "ladds_population_write", "ladds_population_read",
            "ladds_elements_to_state"]


class LaddsError(RuntimeError):
    """A non-zero status of a library call (the codes of include/ladds_gpu.h)."""

    def __init__(self, code, msg):
        super().__init__(f"ladds_gpu error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Loads the in-tree host library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ladds_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, sz, i = C.c_void_p, C.c_size_t, C.c_int
    L.ladds_population_generate.argtypes = [i, C.c_uint64, sz] + [vp] * 12
    L.ladds_population_write.argtypes = [C.c_char_p, sz] + [vp] * 12
    L.ladds_population_read.argtypes = [C.c_char_p, sz, C.POINTER(sz)] + [vp] * 12
    L.ladds_elements_to_state.argtypes = [C.c_double] * 6 + [vp, vp]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def empty_population(n: int) -> dict:
    return {k: np.zeros(n, dtype=t) for k, t in _POP_DTYPES.items()}


def as_population(d: dict) -> dict:
    """The twelve upload arrays, contiguous and typed; parent defaults to
    SIZE_MAX (no parent), activity to passive, id to the index."""
    out = {}
    n = len(d["x"])
    for k, t in _POP_DTYPES.items():
        if k in d and d[k] is not None:
            out[k] = np.ascontiguousarray(d[k], dtype=t)
        elif k == "parent":
            out[k] = np.full(n, SIZE_MAX, dtype=np.uint64)
        elif k == "activity":
            out[k] = np.zeros(n, dtype=np.int8)
        elif k == "id":
            out[k] = np.arange(n, dtype=np.uint64)
        else:
            raise KeyError(k)
    return out


def generate_population(which: int, seed: int, n: int) -> dict:
    """Seeded population `which` (0, 2 or 4) of n objects (ladds_population_generate)."""
    pop = empty_population(n)
    rc = lib().ladds_population_generate(which, seed, n, *[_p(pop[k]) for k in POP_FIELDS])
    if rc:
        raise LaddsError(rc, "population generation failed")
    return pop


def save_population(path: str, pop: dict):
    """Writes a population as a binary SoA population file (ladds_population_write)."""
    pop = as_population(pop)
    rc = lib().ladds_population_write(os.fsencode(path), len(pop["x"]), *[_p(pop[k]) for k in POP_FIELDS])
    if rc:
        raise LaddsError(rc, f"cannot write population file {path}")


def load_population(path: str) -> dict:
    """Reads a binary SoA population file (ladds_population_read)."""
    n = C.c_size_t()
    rc = lib().ladds_population_read(os.fsencode(path), 0, C.byref(n), *([None] * 12))
    if rc not in (OK, ERR_CAPACITY):
        raise LaddsError(rc, f"not a population file: {path}")
    pop = empty_population(n.value)
    rc = lib().ladds_population_read(os.fsencode(path), n.value, C.byref(n), *[_p(pop[k]) for k in POP_FIELDS])
    if rc:
        raise LaddsError(rc, f"not a population file: {path}")
    return pop


def elements_to_state(a, e, inc, raan, argp, M):
    """Keplerian elements (km, rad) -> position (km) and velocity (km/s)."""
    r = np.zeros(3)
    v = np.zeros(3)
    rc = lib().ladds_elements_to_state(a, e, inc, raan, argp, M, _p(r), _p(v))
    if rc:
        raise LaddsError(rc, "elements_to_state failed")
    return r, v
