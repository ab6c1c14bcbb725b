"""ctypes binding of ``libladds_gpu.so`` (the C ABI in ``include/ladds_gpu.h``).

This is the Python face of the library used by the tests and the benchmark;
the C++ host mirror of the reference interface lives in ``ladds_b200/host``.
The shared library is built in-tree by ``ladds_b200.build``; if it is missing
the import fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libladds_gpu.so")

(OK, ERR_INVALID_ARG, ERR_CUDA, ERR_CAPACITY, ERR_NONFINITE, ERR_NO_DEVICE, ERR_DEVICE_CHECK, ERR_ALLOC, ERR_STATE,
 ERR_TOO_LARGE) = range(10)
NOALLOC_SORT_MAX_OBJECTS, NOALLOC_SORT_MAX_ROWS = 262144, 65536
KEP, J2, C22, S22, SOL, LUN, SRP, DRAG, J3 = (1 << k for k in range(9))
PROP_ALL = 0x1FF
PASSIVE, EVASIVE, EVASIVE_PRESERVING = 0, 1, 2
PRECISION_FP64, PRECISION_SPLIT = 0, 1
SCREEN_LISTS, SCREEN_BUFFER = 0, 1
WALK_AUTO, WALK_GROUPED, WALK_ROWS = 0, 1, 2
PAIR_COLLISION, PAIR_EVASION, PAIR_CONJUNCTION = 1, 2, 4
PAIR_NEAR_COLLISION, PAIR_NEAR_EVASION, PAIR_NEAR_CONJUNCTION, PAIR_NEAR_GATE = 8, 16, 32, 64
SIZE_MAX = np.uint64(0xFFFFFFFFFFFFFFFF)

PAIR_DTYPE = np.dtype([("idA", "<u8"), ("idB", "<u8"), ("slotA", "<u4"), ("slotB", "<u4"), ("dl2", "<f8"),
                       ("point", "<f8", (3,)), ("step", "<u4"), ("flags", "<u4")])
assert PAIR_DTYPE.itemsize == 64


from .population import LaddsError  # noqa: E402  (one error type for both libraries)


class GpuConfig(C.Structure):
    _fields_ = [
        ("deltaT", C.c_double),
        ("componentMask", C.c_uint32),
        ("epochJD", C.c_double),
        ("startTime", C.c_double),
        ("cutoff", C.c_double),
        ("collisionDistanceFactor", C.c_double),
        ("minDetectionRadius", C.c_double),
        ("evasionCutoff", C.c_double),
        ("conjunctionThreshold", C.c_double),
        ("nearThresholdRel", C.c_double),
        ("precision", C.c_int32),
        ("timestepsPerCollisionDetection", C.c_int32),
        ("cellSize", C.c_double),
        ("boxMin", C.c_double * 3),
        ("boxMax", C.c_double * 3),
        ("device", C.c_int32),
        ("propagateBlock", C.c_int32),
        ("scanBlock", C.c_int32),
        ("useGraphs", C.c_int32),
        ("pairCapacity", C.c_uint64),
        ("scanScreen", C.c_int32),
        ("walkForm", C.c_int32),
    ]


class StepStats(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("scans", C.c_uint64), ("records", C.c_uint64),
                ("collisions", C.c_uint64), ("evasions", C.c_uint64), ("conjunctions", C.c_uint64),
                ("retries", C.c_uint64), ("deviceMs", C.c_double)]


class PhaseTimes(C.Structure):
    PHASES = ("propagate", "bucket", "rowsort", "permute", "candidates", "evaluate")
    _fields_ = ([(p + "Ms", C.c_double) for p in PHASES] + [("totalMs", C.c_double)]
                + [(p + "Launches", C.c_uint64) for p in PHASES])


EXPORTED = [
    "ladds_gpu_abi_version", "ladds_gpu_config_default", "ladds_gpu_create", "ladds_gpu_destroy",
    "ladds_gpu_last_error", "ladds_gpu_upload", "ladds_gpu_append", "ladds_gpu_download", "ladds_gpu_set_state",
    "ladds_gpu_get_state", "ladds_gpu_size", "ladds_gpu_iteration", "ladds_gpu_set_iteration",
    "ladds_gpu_integrate", "ladds_gpu_conjunctions", "ladds_gpu_step", "ladds_gpu_remove_below",
    "ladds_gpu_mark_deleted", "ladds_gpu_remove_escaping", "ladds_gpu_clear_parents", "ladds_gpu_cell_order",
    "ladds_gpu_grid",
    "ladds_gpu_phase_times", "ladds_gpu_set_profiling", "ladds_population_generate", "ladds_elements_to_state",
    "ladds_gpu_functor_pairs", "ladds_gpu_scan", "ladds_gpu_cell_sort_noalloc", "ladds_gpu_adjoint_forward",
    "ladds_gpu_adjoint_backward", "ladds_gpu_adjoint_make_pairs", "ladds_gpu_autotune", "ladds_records_pack",
    "ladds_records_write_csv", "ladds_gpu_checked_insert", "ladds_gpu_get_objects", "ladds_breakup_collision",
    "ladds_gpu_breakup", "ladds_gpu_select_layers", "ladds_gpu_layer_histogram", "ladds_gpu_remove_slots",
    "ladds_gpu_set_halo", "ladds_gpu_pack_layers", "ladds_gpu_append_records", "ladds_gpu_truncate",
    "ladds_gpu_step_host", "ladds_gpu_pending_records", "ladds_population_write",
    "ladds_population_read", "ladds_gpu_reserve",
]

STATE_RECORD_DTYPE = np.dtype([("r", "<f8", (3,)), ("v", "<f8", (3,)), ("radius", "<f8"), ("aom", "<f8"),
                               ("bcInv", "<f8"), ("id", "<u8"), ("parentId", "<u8"), ("activity", "<i4"),
                               ("deleted", "<u4")])
assert STATE_RECORD_DTYPE.itemsize == 96


class BreakupConfig(C.Structure):
    _fields_ = [("minLc", C.c_double), ("enforceMassConservation", C.c_int32), ("coefficientOfDrag", C.c_double)]

COLLISION_INFO_DTYPE = np.dtype([("idA", "<u4"), ("idB", "<u4"), ("distanceSquared", "<f4")])
assert COLLISION_INFO_DTYPE.itemsize == 12

ADJ_PAIR_DTYPE = np.dtype([("rA", "<f8", (3,)), ("vA", "<f8", (3,)), ("rB", "<f8", (3,)), ("vB", "<f8", (3,)),
                           ("bcInvA", "<f8"), ("bcInvB", "<f8"), ("aomA", "<f8"), ("aomB", "<f8")])
assert ADJ_PAIR_DTYPE.itemsize == 128

OBJECT_DTYPE = np.dtype([("r", "<f8", (3,)), ("v", "<f8", (3,)), ("radius", "<f8"), ("id", "<u8"),
                         ("parentId", "<u8"), ("activity", "<i4"), ("slot", "<u4")])
assert OBJECT_DTYPE.itemsize == 80


class TuneTrial(C.Structure):
    _fields_ = [("cellSize", C.c_double), ("reach", C.c_int32), ("propagateBlock", C.c_int32),
                ("scanBlock", C.c_int32), ("chunkSteps", C.c_int32), ("scanScreen", C.c_int32),
                ("walkForm", C.c_int32), ("msPerStep", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ScanParams(C.Structure):
    _fields_ = [("cutoff", C.c_double), ("dt", C.c_double), ("collisionDistanceFactor", C.c_double),
                ("minDetectionRadius", C.c_double), ("evasionCutoff", C.c_double),
                ("conjunctionThreshold", C.c_double), ("nearThresholdRel", C.c_double)]

_lib = None


def lib():
    """Loads the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ladds_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, sz, i = C.c_void_p, C.c_size_t, C.c_int
    L.ladds_gpu_abi_version.restype = i
    L.ladds_gpu_config_default.argtypes = [C.POINTER(GpuConfig)]
    L.ladds_gpu_create.argtypes = [C.POINTER(GpuConfig), C.POINTER(vp)]
    L.ladds_gpu_destroy.argtypes = [vp]
    L.ladds_gpu_last_error.restype = C.c_char_p
    L.ladds_gpu_last_error.argtypes = [vp]
    L.ladds_gpu_upload.argtypes = [vp, sz] + [vp] * 12
    L.ladds_gpu_append.argtypes = [vp, sz] + [vp] * 12
    L.ladds_gpu_reserve.argtypes = [vp, sz]
    L.ladds_gpu_download.argtypes = [vp, sz, C.POINTER(sz)] + [vp] * 12
    L.ladds_gpu_set_state.argtypes = [vp, sz] + [vp] * 6
    L.ladds_gpu_get_state.argtypes = [vp, sz] + [vp] * 6
    L.ladds_gpu_size.argtypes = [vp, C.POINTER(sz)]
    L.ladds_gpu_iteration.argtypes = [vp, C.POINTER(C.c_int64)]
    L.ladds_gpu_set_iteration.argtypes = [vp, C.c_int64]
    L.ladds_gpu_integrate.argtypes = [vp, i]
    L.ladds_gpu_conjunctions.argtypes = [vp, C.c_double, vp, sz, C.POINTER(sz), C.POINTER(sz), C.POINTER(sz),
                                         C.POINTER(sz)]
    L.ladds_gpu_step.argtypes = [vp, i, vp, sz, C.POINTER(sz), C.POINTER(StepStats)]
    L.ladds_population_write.argtypes = [C.c_char_p, sz] + [vp] * 12
    L.ladds_population_read.argtypes = [C.c_char_p, sz, C.POINTER(sz)] + [vp] * 12
    L.ladds_gpu_step_host.argtypes = [vp, sz, C.POINTER(vp), C.POINTER(vp), vp, sz, C.POINTER(sz),
                                      C.POINTER(StepStats)]
    L.ladds_gpu_pending_records.argtypes = [vp, vp, sz, C.POINTER(sz)]
    L.ladds_gpu_remove_below.argtypes = [vp, C.c_double, C.POINTER(sz), vp, sz]
    L.ladds_gpu_remove_escaping.argtypes = [vp, C.POINTER(sz), vp, sz]
    L.ladds_gpu_mark_deleted.argtypes = [vp, vp, sz]
    L.ladds_gpu_clear_parents.argtypes = [vp]
    L.ladds_gpu_cell_order.argtypes = [vp, sz, C.POINTER(sz), vp, vp]
    L.ladds_gpu_grid.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    L.ladds_gpu_phase_times.argtypes = [vp, C.POINTER(PhaseTimes)]
    L.ladds_gpu_set_profiling.argtypes = [vp, i]
    L.ladds_population_generate.argtypes = [i, C.c_uint64, sz] + [vp] * 12
    L.ladds_elements_to_state.argtypes = [C.c_double] * 6 + [vp, vp]
    L.ladds_gpu_functor_pairs.argtypes = [vp, C.POINTER(ScanParams), sz, vp, vp, vp, sz, C.POINTER(sz)]
    L.ladds_gpu_scan.argtypes = [vp, C.POINTER(ScanParams), vp, sz, C.POINTER(sz)]
    L.ladds_gpu_adjoint_forward.argtypes = [vp, vp, sz, i, i, vp, vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.ladds_gpu_adjoint_backward.argtypes = [vp, vp, vp, C.POINTER(C.c_double)]
    L.ladds_gpu_adjoint_make_pairs.argtypes = [vp, C.c_uint64, sz, i, vp, vp]
    L.ladds_gpu_get_objects.argtypes = [vp, vp, sz, vp]
    L.ladds_breakup_collision.argtypes = [C.POINTER(BreakupConfig), C.c_uint64, vp, vp, vp, C.c_uint64,
                                          C.POINTER(C.c_uint64), sz, C.POINTER(sz)] + [vp] * 12
    L.ladds_gpu_breakup.argtypes = [vp, vp, sz, C.POINTER(BreakupConfig), C.c_uint64, C.POINTER(C.c_uint64),
                                    C.POINTER(sz), C.POINTER(sz)]
    L.ladds_gpu_checked_insert.argtypes = [vp, sz] + [vp] * 12 + [C.c_double, vp, C.POINTER(sz)]
    L.ladds_records_pack.argtypes = [vp, sz, C.c_uint32, vp, sz, C.POINTER(sz)]
    L.ladds_records_write_csv.argtypes = [C.c_char_p, i, vp, sz, C.c_uint32]
    L.ladds_gpu_autotune.argtypes = [vp, i, C.POINTER(TuneTrial), sz, C.POINTER(sz), C.POINTER(TuneTrial)]
    L.ladds_gpu_select_layers.argtypes = [vp, C.c_int32, C.c_int32, vp, sz, C.POINTER(sz)]
    L.ladds_gpu_layer_histogram.argtypes = [vp, vp, sz]
    L.ladds_gpu_remove_slots.argtypes = [vp, vp, sz]
    L.ladds_gpu_set_halo.argtypes = [vp, sz]
    L.ladds_gpu_pack_layers.argtypes = [vp, C.c_int32, C.c_int32, i, vp, sz, C.POINTER(sz)]
    L.ladds_gpu_append_records.argtypes = [vp, vp, sz]
    L.ladds_gpu_truncate.argtypes = [vp, sz]
    L.ladds_gpu_cell_sort_noalloc.argtypes = [i, vp, vp, sz, C.POINTER(C.c_int32 * 3), vp, vp, vp, C.c_char_p, sz]
    _lib = L
    return L


def default_config(**overrides) -> GpuConfig:
    cfg = GpuConfig()
    lib().ladds_gpu_config_default(C.byref(cfg))
    for k, v in overrides.items():
        if k in ("boxMin", "boxMax"):
            getattr(cfg, k)[:] = list(v)
        else:
            setattr(cfg, k, v)
    return cfg


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


from .population import POP_FIELDS, as_population, empty_population  # noqa: E402,F401
from . import population as _population  # noqa: E402


def generate_population(which: int, seed: int, n: int) -> dict:
    """Seeded population `which` of n objects (host library, no GPU code)."""
    return _population.generate_population(which, seed, n)


def save_population(path: str, pop: dict):
    """Writes a population as a binary SoA population file (ladds_population_write)."""
    _population.save_population(path, pop)


def load_population(path: str) -> dict:
    """Reads a binary SoA population file (ladds_population_read)."""
    return _population.load_population(path)


def elements_to_state(a, e, inc, raan, argp, M):
    return _population.elements_to_state(a, e, inc, raan, argp, M)


@dataclass
class StepResult:
    records: np.ndarray
    stats: StepStats


class Context:
    """One device context (``ladds_gpu_ctx``)."""

    def __init__(self, config: GpuConfig | None = None, **overrides):
        self._L = lib()
        cfg = config if config is not None else default_config()
        for k, v in overrides.items():
            if k in ("boxMin", "boxMax"):
                getattr(cfg, k)[:] = list(v)
            else:
                setattr(cfg, k, v)
        self.config = cfg
        h = C.c_void_p()
        rc = self._L.ladds_gpu_create(C.byref(cfg), C.byref(h))
        if rc:
            raise LaddsError(rc, "ladds_gpu_create failed")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.ladds_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc:
            msg = self._L.ladds_gpu_last_error(self._h)
            raise LaddsError(rc, msg.decode() if msg else "")

    @property
    def handle(self):
        return self._h

    def upload(self, pop: dict):
        pop = as_population(pop)
        self._keep = pop
        self._check(self._L.ladds_gpu_upload(self._h, len(pop["x"]), *[_p(pop[k]) for k in POP_FIELDS]))

    def append(self, pop: dict):
        pop = as_population(pop)
        self._check(self._L.ladds_gpu_append(self._h, len(pop["x"]), *[_p(pop[k]) for k in POP_FIELDS]))

    def reserve(self, capacity: int):
        """Device capacity for at least `capacity` objects (appends up to it reallocate nothing)."""
        self._check(self._L.ladds_gpu_reserve(self._h, int(capacity)))

    def size(self) -> int:
        n = C.c_size_t()
        self._check(self._L.ladds_gpu_size(self._h, C.byref(n)))
        return n.value

    def iteration(self) -> int:
        it = C.c_int64()
        self._check(self._L.ladds_gpu_iteration(self._h, C.byref(it)))
        return it.value

    def set_iteration(self, it: int):
        self._check(self._L.ladds_gpu_set_iteration(self._h, it))

    def download(self) -> dict:
        n = self.size()
        pop = empty_population(n)
        got = C.c_size_t()
        self._check(self._L.ladds_gpu_download(self._h, n, C.byref(got), *[_p(pop[k]) for k in POP_FIELDS]))
        return pop

    def set_state(self, x, y, z, vx, vy, vz):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, vx, vy, vz)]
        self._check(self._L.ladds_gpu_set_state(self._h, len(arrs[0]), *[_p(a) for a in arrs]))

    def get_state(self):
        n = self.size()
        arrs = [np.zeros(n) for _ in range(6)]
        self._check(self._L.ladds_gpu_get_state(self._h, n, *[_p(a) for a in arrs]))
        return arrs

    def integrate(self, steps: int, allow_nonfinite: bool = False) -> bool:
        """Yoshida steps; with allow_nonfinite a state that became non-finite is
        kept (returns False) for remove_escaping, as the reference loop does."""
        rc = self._L.ladds_gpu_integrate(self._h, steps)
        if allow_nonfinite and rc == ERR_NONFINITE:
            return False
        self._check(rc)
        return True

    def conjunctions(self, dt_scan: float, cap: int | None = None):
        cap = 4096 if cap is None else cap
        while True:
            out = np.zeros(max(cap, 1), dtype=PAIR_DTYPE)
            n, nc, ne, nj = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_size_t()
            rc = self._L.ladds_gpu_conjunctions(self._h, dt_scan, _p(out), cap, C.byref(n), C.byref(nc),
                                                C.byref(ne), C.byref(nj))
            if rc == ERR_CAPACITY:
                cap = n.value
                continue
            self._check(rc)
            return out[: n.value].copy()

    def step(self, iterations: int, cap: int | None = None, out: np.ndarray | None = None) -> StepResult:
        if out is not None:
            cap = len(out)
        cap = 4096 if cap is None else cap
        while True:
            buf = out if (out is not None and len(out) >= cap) else np.zeros(max(cap, 1), dtype=PAIR_DTYPE)
            n = C.c_size_t()
            st = StepStats()
            rc = self._L.ladds_gpu_step(self._h, iterations, _p(buf), cap, C.byref(n), C.byref(st))
            if rc == ERR_CAPACITY and n.value > cap:
                cap = n.value
                out = None
                continue
            self._check(rc)
            return StepResult(buf[: n.value].copy(), st)

    def step_host(self, state_in, state_out=None, out: np.ndarray | None = None) -> StepResult:
        """One iteration with the positions and velocities in host memory
        (ladds_gpu_step_host): state_in = (x, y, z, vx, vy, vz) float64 arrays in
        slot order; state_out receives the new state (default: state_in, in place).
        Pinned arrays (torch pin_memory) let the copies overlap."""
        n = self.size()
        ins = list(state_in)
        outs = ins if state_out is None else list(state_out)
        if len(ins) != 6 or len(outs) != 6:
            raise ValueError("six state arrays: x, y, z, vx, vy, vz")
        for a in ins + outs:
            if a.shape != (n,) or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("state arrays must be contiguous float64 of the population size")
        if any(not a.flags.writeable for a in outs):
            raise ValueError("state_out arrays must be writeable")
        buf = out if out is not None else np.zeros(4096, dtype=PAIR_DTYPE)
        got = C.c_size_t()
        st = StepStats()
        rc = self._L.ladds_gpu_step_host(self._h, n, (C.c_void_p * 6)(*[a.ctypes.data for a in ins]),
                                         (C.c_void_p * 6)(*[a.ctypes.data for a in outs]), _p(buf), len(buf),
                                         C.byref(got), C.byref(st))
        if rc == ERR_CAPACITY and got.value > len(buf):  # the iteration was taken; its records wait
            buf = np.zeros(got.value, dtype=PAIR_DTYPE)
            rc = self._L.ladds_gpu_pending_records(self._h, _p(buf), len(buf), C.byref(got))
        self._check(rc)
        return StepResult(buf[: got.value].copy(), st)

    def cell_order(self):
        n = self.size()
        keys = np.zeros(n, dtype=np.uint32)
        slots = np.zeros(n, dtype=np.uint32)
        got = C.c_size_t()
        self._check(self._L.ladds_gpu_cell_order(self._h, n, C.byref(got), _p(keys), _p(slots)))
        return keys, slots

    def grid(self):
        dims = (C.c_int32 * 3)()
        reach = C.c_int32()
        cell = C.c_double()
        self._check(self._L.ladds_gpu_grid(self._h, dims, C.byref(reach), C.byref(cell)))
        return tuple(dims), reach.value, cell.value

    def remove_below(self, min_altitude: float):
        n = self.size()
        # one id buffer reused across calls (a fresh population-sized buffer per call costs more than the call)
        if getattr(self, "_removed_ids", None) is None or len(self._removed_ids) < max(n, 1):
            self._removed_ids = np.empty(max(n, 1), dtype=np.uint64)
        ids = self._removed_ids
        removed = C.c_size_t()
        self._check(self._L.ladds_gpu_remove_below(self._h, min_altitude, C.byref(removed), _p(ids), n))
        return ids[: removed.value].copy()

    def remove_escaping(self):
        """Ids of the objects removed for leaving the container (non-finite
        state or outside the box; ladds_gpu_remove_escaping)."""
        n = self.size()
        if getattr(self, "_removed_ids", None) is None or len(self._removed_ids) < max(n, 1):
            self._removed_ids = np.empty(max(n, 1), dtype=np.uint64)
        ids = self._removed_ids
        removed = C.c_size_t()
        self._check(self._L.ladds_gpu_remove_escaping(self._h, C.byref(removed), _p(ids), n))
        return ids[: removed.value].copy()

    def mark_deleted(self, slots):
        slots = np.ascontiguousarray(slots, dtype=np.uint32)
        self._check(self._L.ladds_gpu_mark_deleted(self._h, _p(slots), len(slots)))

    def clear_parents(self):
        self._check(self._L.ladds_gpu_clear_parents(self._h))

    # ---- slab decomposition primitives (ladds_b200.slabs)
    def select_layers(self, iz_lo: int, iz_hi: int) -> np.ndarray:
        """Slots (ascending) of the live objects in the cell layers [iz_lo, iz_hi)."""
        cap = max(self.size(), 1)
        out = np.zeros(cap, dtype=np.uint32)
        n = C.c_size_t()
        self._check(self._L.ladds_gpu_select_layers(self._h, iz_lo, iz_hi, _p(out), cap, C.byref(n)))
        return out[: n.value].copy()

    def layer_histogram(self) -> np.ndarray:
        nz = self.grid()[0][2]
        out = np.zeros(nz, dtype=np.uint64)
        self._check(self._L.ladds_gpu_layer_histogram(self._h, _p(out), nz))
        return out

    def remove_slots(self, slots):
        slots = np.ascontiguousarray(slots, dtype=np.uint32)
        self._check(self._L.ladds_gpu_remove_slots(self._h, _p(slots), len(slots)))

    def set_halo(self, halo_start: int | None):
        """Objects with slot >= halo_start are pair-scan targets only (None: no halo)."""
        self._check(self._L.ladds_gpu_set_halo(self._h, (1 << 64) - 1 if halo_start is None else halo_start))

    # device-resident exchange: buffers are device memory of this context's
    # device, given as a pointer (int) or an object with data_ptr() (a torch tensor)
    @staticmethod
    def _dptr(buf):
        return C.c_void_p(buf if isinstance(buf, int) else buf.data_ptr())

    def pack_layers(self, iz_lo: int, iz_hi: int, remove: bool, out, cap: int) -> int:
        """State records of the live objects of cell layers [iz_lo, iz_hi) into
        device memory `out` (cap records); returns their number."""
        n = C.c_size_t()
        self._check(self._L.ladds_gpu_pack_layers(self._h, iz_lo, iz_hi, int(bool(remove)),
                                                  self._dptr(out) if out is not None else None, cap,
                                                  C.byref(n)))
        return n.value

    def torch_device(self) -> str:
        """The torch device of this context's GPU (for exchange buffers)."""
        return f"cuda:{self.config.device}"

    def append_records(self, records, m: int):
        """Appends m objects from state records in device memory."""
        if m:
            self._check(self._L.ladds_gpu_append_records(self._h, self._dptr(records), m))

    def truncate(self, n: int):
        """Deletes the objects with slot >= n."""
        self._check(self._L.ladds_gpu_truncate(self._h, n))

    def scan(self, params: ScanParams, cap: int = 4096):
        """Conjunction scan of the current state with explicit functor scalars."""
        while True:
            out = np.zeros(max(cap, 1), dtype=PAIR_DTYPE)
            n = C.c_size_t()
            rc = self._L.ladds_gpu_scan(self._h, C.byref(params), _p(out), cap, C.byref(n))
            if rc == ERR_CAPACITY and n.value > cap:
                cap = n.value
                continue
            self._check(rc)
            return out[: n.value].copy()

    def functor_pairs(self, params: ScanParams, first: np.ndarray, second: np.ndarray):
        """CollisionFunctor::AoSFunctor over explicit pairs (OBJECT_DTYPE arrays)."""
        first = np.ascontiguousarray(first, dtype=OBJECT_DTYPE)
        second = np.ascontiguousarray(second, dtype=OBJECT_DTYPE)
        cap = max(16, len(first))
        while True:
            out = np.zeros(cap, dtype=PAIR_DTYPE)
            n = C.c_size_t()
            rc = self._L.ladds_gpu_functor_pairs(self._h, C.byref(params), len(first), _p(first), _p(second),
                                                 _p(out), cap, C.byref(n))
            if rc == ERR_CAPACITY:
                cap = n.value
                continue
            self._check(rc)
            return out[: n.value].copy()

    def get_objects(self, slots) -> np.ndarray:
        """State records (STATE_RECORD_DTYPE) of the objects with the given slots."""
        slots = np.ascontiguousarray(slots, dtype=np.uint32)
        out = np.zeros(max(len(slots), 1), dtype=STATE_RECORD_DTYPE)
        self._check(self._L.ladds_gpu_get_objects(self._h, _p(slots), len(slots), _p(out)))
        return out[: len(slots)]

    def breakup(self, records: np.ndarray, cfg: "BreakupConfig", seed: int, next_id: int):
        """BreakupWrapper::simulateBreakup for the collision records; returns
        (breakups, fragments, next free id)."""
        records = np.ascontiguousarray(records, dtype=PAIR_DTYPE)
        nid = C.c_uint64(next_id)
        nb, nf = C.c_size_t(), C.c_size_t()
        self._check(self._L.ladds_gpu_breakup(self._h, _p(records), len(records), C.byref(cfg), seed,
                                              C.byref(nid), C.byref(nb), C.byref(nf)))
        return nb.value, nf.value, nid.value

    def checked_insert(self, pop: dict, constellation_cutoff: float) -> np.ndarray:
        """Simulation::checkedInsert: appends the satellites of `pop` that have no
        particle within the cutoff; returns the delayed flags (1 = not inserted)."""
        pop = as_population(pop)
        n = len(pop["x"])
        delayed = np.zeros(max(n, 1), dtype=np.uint8)
        got = C.c_size_t()
        self._check(self._L.ladds_gpu_checked_insert(self._h, n, *[_p(pop[k]) for k in POP_FIELDS],
                                                     constellation_cutoff, _p(delayed), C.byref(got)))
        return delayed[:n].copy()

    def autotune(self, steps_per_trial: int = 16):
        """Times cell edges, block shapes and chunk lengths; applies the fastest.
        Returns (best, [trials]) as dicts."""
        trials = (TuneTrial * 64)()
        n = C.c_size_t()
        best = TuneTrial()
        self._check(self._L.ladds_gpu_autotune(self._h, steps_per_trial, trials, 64, C.byref(n), C.byref(best)))
        return best.as_dict(), [trials[i].as_dict() for i in range(min(n.value, 64))]

    # ---- adjoint of the propagation for conjunction pairs
    def adjoint_make_pairs(self, seed: int, n_pairs: int, steps: int):
        """Synthetic pairs of the differentiation benchmark; returns (pairs, tca)."""
        pairs = np.zeros(n_pairs, dtype=ADJ_PAIR_DTYPE)
        tca = np.zeros(n_pairs, dtype=np.int32)
        self._check(self._L.ladds_gpu_adjoint_make_pairs(self._h, seed, n_pairs, steps, _p(pairs), _p(tca)))
        return pairs, tca

    def adjoint_forward(self, pairs: np.ndarray, steps: int, checkpoint_every: int = 64):
        """Loss sum_p min_s dl2; returns (loss, missSq, tcaStep, device ms)."""
        pairs = np.ascontiguousarray(pairs, dtype=ADJ_PAIR_DTYPE)
        n = len(pairs)
        miss = np.zeros(n, dtype=np.float64)
        tca = np.zeros(n, dtype=np.int32)
        loss, ms = C.c_double(), C.c_double()
        self._check(self._L.ladds_gpu_adjoint_forward(self._h, _p(pairs), n, steps, checkpoint_every, _p(miss),
                                                      _p(tca), C.byref(loss), C.byref(ms)))
        self._adj_n = n
        return loss.value, miss, tca, ms.value

    def adjoint_backward(self):
        """Gradients of the last forward sweep: (dL/d(rA, vA, rB, vB) [P, 12], dL/d(bcA, bcB) [P, 2], ms)."""
        n = getattr(self, "_adj_n", 0)
        dx = np.zeros((max(n, 1), 12), dtype=np.float64)
        dbc = np.zeros((max(n, 1), 2), dtype=np.float64)
        ms = C.c_double()
        self._check(self._L.ladds_gpu_adjoint_backward(self._h, _p(dx), _p(dbc), C.byref(ms)))
        return dx[:n], dbc[:n], ms.value

    def set_profiling(self, on: bool):
        self._check(self._L.ladds_gpu_set_profiling(self._h, 1 if on else 0))

    def phase_times(self) -> PhaseTimes:
        t = PhaseTimes()
        self._check(self._L.ladds_gpu_phase_times(self._h, C.byref(t)))
        return t


def pack_records(records: np.ndarray, flag_mask: int) -> np.ndarray:
    """Records with (flags & flag_mask) in the HDF5 CollisionInfo layout (idA, idB as u32, dl2 as f32)."""
    records = np.ascontiguousarray(records, dtype=PAIR_DTYPE)
    out = np.zeros(max(len(records), 1), dtype=COLLISION_INFO_DTYPE)
    n = C.c_size_t()
    rc = lib().ladds_records_pack(_p(records), len(records), flag_mask, _p(out), len(out), C.byref(n))
    if rc:
        raise LaddsError(rc, "ladds_records_pack failed")
    return out[: n.value].copy()


def write_records_csv(path: str, records: np.ndarray, flag_mask: int, append: bool = False) -> None:
    """CSV "Iteration,P1,P2,SquaredDistance" of the records with (flags & flag_mask)."""
    records = np.ascontiguousarray(records, dtype=PAIR_DTYPE)
    rc = lib().ladds_records_write_csv(path.encode(), 1 if append else 0, _p(records), len(records), flag_mask)
    if rc:
        raise LaddsError(rc, f"ladds_records_write_csv({path}) failed")


def breakup_collision(cfg: BreakupConfig, seed: int, a: np.ndarray, b: np.ndarray, point, parent_id: int,
                      next_id: int, cap: int = 1 << 16):
    """Fragments of one collision (host NASA-breakup restatement): (population dict, next free id)."""
    a = np.ascontiguousarray(a, dtype=STATE_RECORD_DTYPE)
    b = np.ascontiguousarray(b, dtype=STATE_RECORD_DTYPE)
    pt = np.ascontiguousarray(point, dtype=np.float64)
    while True:
        pop = empty_population(cap)
        nid = C.c_uint64(next_id)
        got = C.c_size_t()
        rc = lib().ladds_breakup_collision(C.byref(cfg), seed, _p(a), _p(b), _p(pt), parent_id, C.byref(nid), cap,
                                           C.byref(got), *[_p(pop[k]) for k in POP_FIELDS])
        if rc == ERR_CAPACITY:
            cap = got.value
            continue
        if rc:
            raise LaddsError(rc, "ladds_breakup_collision failed")
        return {k: v[: got.value].copy() for k, v in pop.items()}, nid.value
