"""Shared helpers of the test suite (conversions between the product's
population dicts and the oracle's Population, record comparison)."""
import math

import numpy as np


def to_oracle(oracle, pop):
    return oracle.Population(pop["x"], pop["y"], pop["z"], pop["vx"], pop["vy"], pop["vz"], pop["radius"],
                             pop["aom"], pop["bc_inv"], pop["id"], pop["parent"], pop["activity"])


def from_lists(rs, vs, ids, acts, masses, radii, parents=None, cd=2.2):
    """Builds a population like the reference tests' Particle(...) calls with
    calculateBcInv(0., 1., 1., 2.2)."""
    rs = np.asarray(rs, float)
    vs = np.asarray(vs, float)
    n = len(rs)
    aom = np.array([math.pi * radii[k] ** 2 * 1e-6 / masses[k] for k in range(n)])
    bc = np.full(n, cd * math.pi / 1.0)
    return dict(x=rs[:, 0], y=rs[:, 1], z=rs[:, 2], vx=vs[:, 0], vy=vs[:, 1], vz=vs[:, 2],
                radius=np.asarray(radii, float), aom=aom, bc_inv=bc, id=np.asarray(ids, np.uint64),
                parent=None if parents is None else np.asarray(parents, np.uint64),
                activity=np.asarray(acts, np.int8))


def records_equal(a, b):
    """Bit-exact equality of two record arrays (NaN == NaN by bit pattern)."""
    if len(a) != len(b):
        return False
    return a.tobytes() == b.tobytes()


def describe_diff(a, b, limit=5):
    sa = {(int(r["step"]), int(r["idA"]), int(r["idB"]), int(r["slotA"]), int(r["slotB"])): r for r in a}
    sb = {(int(r["step"]), int(r["idA"]), int(r["idB"]), int(r["slotA"]), int(r["slotB"])): r for r in b}
    only_a = sorted(set(sa) - set(sb))[:limit]
    only_b = sorted(set(sb) - set(sa))[:limit]
    diff = [k for k in sorted(set(sa) & set(sb)) if sa[k].tobytes() != sb[k].tobytes()][:limit]
    return f"len {len(a)} vs {len(b)}; only first {only_a}; only second {only_b}; differing {diff}"


class OracleEngine:
    """The engine interface of ladds_b200.slabs (the capi.Context methods it
    calls) on the CPU oracle, for multi-rank tests of the decomposition logic
    without a GPU: integration by the oracle's Yoshida steps, the pair scan by
    the oracle's cell scan, halo objects as targets only (halo-halo pairs
    dropped)."""

    def __init__(self, oracle, pop, box_min, box_max, cutoff, cell, mask, dt, **scan_kw):
        from ladds_b200 import capi

        self.o, self.capi = oracle, capi
        self.pop = to_oracle(oracle, pop)
        self.cutoff, self.mask, self.dt = cutoff, mask, dt
        self.grid_ = oracle.make_grid(box_min, box_max, cell, cutoff)
        self.scan_kw = scan_kw
        self.halo = None
        self.it = 0

    def grid(self):
        g = self.grid_
        return (g.n[0], g.n[1], g.n[2]), g.reach, g.cellSize

    def size(self):
        return self.pop.n

    def layers(self):
        keys = self.o.cell_keys(self.pop, self.grid_).astype(np.int64)
        return keys // (int(self.grid_.n[0]) * int(self.grid_.n[1]))

    def layer_histogram(self):
        iz = self.layers()[self.pop.dummy == 0]
        return np.bincount(iz, minlength=int(self.grid_.n[2])).astype(np.uint64)

    def select_layers(self, lo, hi):
        iz = self.layers()
        return np.nonzero((iz >= lo) & (iz < hi) & (self.pop.dummy == 0))[0].astype(np.uint32)

    def get_objects(self, slots):
        p, s = self.pop, np.asarray(slots, dtype=np.int64)
        out = np.zeros(len(s), dtype=self.capi.STATE_RECORD_DTYPE)
        out["r"] = np.stack([p.x[s], p.y[s], p.z[s]], 1)
        out["v"] = np.stack([p.vx[s], p.vy[s], p.vz[s]], 1)
        for f, a in (("radius", p.radius), ("aom", p.aom), ("bcInv", p.bc_inv), ("id", p.id),
                     ("parentId", p.parent), ("activity", p.activity), ("deleted", p.dummy)):
            out[f] = a[s]
        return out

    def _fields(self, p=None):
        p = self.pop if p is None else p
        return [p.x, p.y, p.z, p.vx, p.vy, p.vz, p.radius, p.aom, p.bc_inv, p.id, p.parent, p.activity, p.dummy]

    def remove_slots(self, slots):
        keep = np.ones(self.pop.n, bool)
        keep[np.asarray(slots, dtype=np.int64)] = False
        self.pop = self.o.Population(*[a[keep] for a in self._fields()])

    def append(self, pop):
        add = self._fields(to_oracle(self.o, pop))
        self.pop = self.o.Population(*[np.concatenate([a, b]) for a, b in zip(self._fields(), add)])

    def set_halo(self, start):
        self.halo = start

    # device-resident exchange of ladds_b200.slabs, on host memory: buffers are
    # CPU torch tensors (uint8) holding state records
    def torch_device(self):
        return "cpu"

    def pack_layers(self, lo, hi, remove, out, cap):
        sel = self.select_layers(lo, hi)
        if len(sel) and (out is not None or not remove):
            if len(sel) > cap:
                raise self.capi.LaddsError(self.capi.ERR_CAPACITY, "pack_layers: more particles than the output")
            rec = self.get_objects(sel)
            out[: rec.nbytes].numpy()[:] = np.frombuffer(rec.tobytes(), dtype=np.uint8)
        if remove and len(sel):
            self.remove_slots(sel)
        return len(sel)

    def append_records(self, buf, m):
        if m:
            from ladds_b200.slabs import records_to_population

            rec = np.frombuffer(buf[: m * self.capi.STATE_RECORD_DTYPE.itemsize].numpy().tobytes(),
                                dtype=self.capi.STATE_RECORD_DTYPE)
            self.append(records_to_population(rec))

    def truncate(self, n0):
        if n0 < self.pop.n:
            self.remove_slots(np.arange(n0, self.pop.n))

    def integrate(self, steps):
        self.o.propagate(self.pop, self.mask, self.dt, steps, t0=self.dt * self.it)
        self.it += steps

    def conjunctions(self, dt_scan):
        params = self.o.scan_params(cutoff=self.cutoff, dt=dt_scan, **self.scan_kw)
        recs = self.o.scan_cells(self.pop, params, self.grid_, step=max(self.it - 1, 0))  # as the C ABI
        if self.halo is not None:
            recs = recs[(recs["slotA"] < self.halo) | (recs["slotB"] < self.halo)]
        return recs


def records_without_slots(recs):
    """Records as comparable bytes without the rank-local slot fields, in (step, idA, idB) order."""
    r = recs[np.lexsort((recs["idB"], recs["idA"], recs["step"]))].copy()
    r["slotA"] = 0
    r["slotB"] = 0
    return r.tobytes()
