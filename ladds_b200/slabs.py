"""Slab decomposition of the hot path over ranks (one process per GPU).

This is the role of LADDS' MPI mode -- the domain decomposition
(distributedMemParallelization/AltitudeBasedDecomposition.cpp:131-179,
RegularGridDecomposition.cpp), the particle communication
(ParticleCommunicator.cpp) and the migrant conjunction checks
(ParticleMigrationHandler.cpp:11-56, called at Simulation.cpp:313-376) --
restated for the cell grid of the pair scan:

* rank r owns the objects whose cell layer iz (the z index of the cell key)
  lies in [bounds[r], bounds[r+1]); the bounds split the layers by object
  count (a layer histogram summed over the ranks), every slab at least
  `reach` layers thick;
* every iteration the ranks integrate their objects, hand emigrants (objects
  now in another rank's layers) to their new owners, and, on scan
  iterations, ship their lowest `reach` layers to the rank below as its halo:
  each rank scans its own objects against each other and against the halo
  (halo objects are scan targets only, never sources), then drops the halo.

A pair within the cutoff lies in layers at most `reach` apart, and the
half-shell walk finds it from its lower object, so exactly one rank scans it:
the union of the ranks' records is the single-context record set, bit for bit
(records carry global ids; slots are rank-local).  The reference's MPI mode
instead scans each rank's container alone and checks migrants in a swept box,
which misses pairs across rank borders that involve no migrant.

Exchanges are host-side object lists (96-byte state records) through
``torch.distributed`` collectives -- all-gathers of the emigrants and of the
halos, so every rank takes the same collective steps in the same order.  The
engine is a ``capi.Context`` (one per rank, on its own GPU); anything with
the same methods works.
"""
from __future__ import annotations

import numpy as np

from . import capi


def _dist():
    import torch.distributed as dist

    return dist if dist.is_available() and dist.is_initialized() else None


def split_layers(hist: np.ndarray, world: int, reach: int) -> list[int]:
    """Layer bounds [b_0 = 0, ..., b_world = nz] splitting the objects of the
    layer histogram into `world` slabs of about equal count, each slab at
    least `reach` layers thick (so that a rank's halo comes from the next
    rank alone)."""
    nz = len(hist)
    thick = max(1, reach)
    if nz < world * thick:
        raise ValueError(f"{nz} cell layers cannot hold {world} slabs of {thick} layers")
    cum = np.concatenate([[0], np.cumsum(np.asarray(hist, dtype=np.float64))])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        b = int(np.searchsorted(cum, total * r / world, side="left"))
        b = max(b, bounds[-1] + thick)        # this slab at least `thick` layers
        b = min(b, nz - (world - r) * thick)  # room for the remaining slabs
        bounds.append(b)
    bounds.append(nz)
    return bounds


def records_to_population(rec: np.ndarray) -> dict:
    """Population dict (capi.POP_FIELDS) of state records (capi.STATE_RECORD_DTYPE)."""
    return dict(x=rec["r"][:, 0].copy(), y=rec["r"][:, 1].copy(), z=rec["r"][:, 2].copy(),
                vx=rec["v"][:, 0].copy(), vy=rec["v"][:, 1].copy(), vz=rec["v"][:, 2].copy(),
                radius=rec["radius"].copy(), aom=rec["aom"].copy(), bc_inv=rec["bcInv"].copy(),
                id=rec["id"].copy(), parent=rec["parentId"].copy(), activity=rec["activity"].astype(np.int8))


def sort_records(recs: np.ndarray) -> np.ndarray:
    """Records in (step, idA, idB) order -- the order of a single context's records."""
    if not len(recs):
        return recs
    return recs[np.lexsort((recs["idB"], recs["idA"], recs["step"]))]


class SlabDecomposition:
    """One rank's share of a slab-decomposed population.

    ``engine`` holds this rank's objects (``distribute`` cuts a population that
    every rank uploaded whole down to the rank's slab).  ``group`` is the
    torch.distributed process group (None: the default group; a single
    process when torch.distributed is not initialised)."""

    def __init__(self, engine, group=None):
        self.e = engine
        self.group = group
        d = _dist()
        self.world = d.get_world_size(group) if d else 1
        self.rank = d.get_rank(group) if d else 0
        dims, reach, _ = engine.grid()
        self.nz, self.reach = int(dims[2]), int(reach)
        self.bounds: list[int] | None = None
        self.migrated = 0  # emigrants handed over by this rank so far

    def all_gather(self, obj) -> list:
        """obj of every rank, in rank order (a single process: [obj])."""
        d = _dist()
        if not d or self.world == 1:
            return [obj]
        out = [None] * self.world
        d.all_gather_object(out, obj, group=self.group)
        return out

    # ------------------------------------------------------------------ setup
    def distribute(self, bounds: list[int] | None = None) -> list[int]:
        """Fixes the slab bounds (from the summed layer histograms unless
        given) and removes every object outside this rank's slab."""
        if bounds is None:
            hists = self.all_gather(np.asarray(self.e.layer_histogram(), dtype=np.uint64))
            bounds = split_layers(np.sum(hists, axis=0), self.world, self.reach)
        if len(bounds) != self.world + 1 or bounds[0] != 0 or bounds[-1] != self.nz:
            raise ValueError("slab bounds must run from 0 to the number of cell layers, one slab per rank")
        if any(b1 - b0 < max(1, self.reach) for b0, b1 in zip(bounds[:-1], bounds[1:])):
            raise ValueError("every slab must be at least `reach` cell layers thick")
        self.bounds = list(bounds)
        lo, hi = self.bounds[self.rank], self.bounds[self.rank + 1]
        out = np.concatenate([self.e.select_layers(0, lo), self.e.select_layers(hi, self.nz)])
        if len(out):
            self.e.remove_slots(out)
        return self.bounds

    # ------------------------------------------------------------- iteration
    def migrate(self) -> int:
        """Hands the objects that left this rank's layers to their owners and
        appends the arrivals; returns the number of arrivals."""
        leaving, slots = {}, []
        for d in range(self.world):
            if d == self.rank:
                continue
            s = self.e.select_layers(self.bounds[d], self.bounds[d + 1])
            if len(s):
                leaving[d] = self.e.get_objects(s)
                slots.append(s)
        if slots:
            self.e.remove_slots(np.concatenate(slots))
            self.migrated += sum(len(s) for s in slots)
        arrivals = [g[self.rank] for g in self.all_gather(leaving) if self.rank in g]
        if arrivals:
            self.e.append(records_to_population(np.concatenate(arrivals)))
        return int(sum(len(a) for a in arrivals))

    def scan(self, dt_scan: float) -> np.ndarray:
        """Pair scan of this rank's objects with each other and with the halo
        (the next rank's lowest `reach` layers); records of this rank."""
        lo = self.bounds[self.rank]
        mine = self.e.select_layers(lo, lo + self.reach)
        halos = self.all_gather(self.e.get_objects(mine) if len(mine) else None)
        halo = halos[self.rank + 1] if self.rank + 1 < self.world else None
        n0 = self.e.size()
        if halo is not None and len(halo):
            self.e.append(records_to_population(halo))
            self.e.set_halo(n0)
        try:
            recs = self.e.conjunctions(dt_scan)
        finally:
            self.e.set_halo(None)
            n1 = self.e.size()
            if n1 > n0:
                self.e.remove_slots(np.arange(n0, n1, dtype=np.uint32))
        return recs

    def iterate(self, dt_scan: float | None) -> np.ndarray:
        """One iteration of the reference loop on this rank: integrate, hand
        over emigrants, then (dt_scan not None) the pair scan with the halo."""
        self.e.integrate(1)
        self.migrate()
        if dt_scan is None:
            return np.zeros(0, dtype=capi.PAIR_DTYPE)
        return self.scan(dt_scan)

    def gather_records(self, recs: np.ndarray) -> np.ndarray:
        """All ranks' records, in single-context order, on every rank."""
        return sort_records(np.concatenate(self.all_gather(np.asarray(recs))))
