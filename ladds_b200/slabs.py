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

Exchanges stay on the device: the library packs the emigrants and the halo
as 96-byte state records into device buffers (ladds_gpu_pack_layers), one
``all_to_all_single`` of ``torch.distributed`` moves them between the ranks
(NCCL: device to device over NVLink; counts first, then the records), and the
receivers append them from device memory (ladds_gpu_append_records).  Every
rank takes the same collective steps in the same order; no particle crosses
the host.  Under a gloo group (CPU tests, or several ranks sharing one GPU)
the buffers are staged through host memory for the collective only.  The
engine is a ``capi.Context`` (one per rank, on its own GPU); anything with
the same methods works.
"""
from __future__ import annotations

import numpy as np

from . import capi

REC = capi.STATE_RECORD_DTYPE.itemsize  # bytes of one state record


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
        """obj of every rank, in rank order (a single process: [obj]); small
        host values only (bounds, counts, test results)."""
        d = _dist()
        if not d or self.world == 1:
            return [obj]
        out = [None] * self.world
        d.all_gather_object(out, obj, group=self.group)
        return out

    def _device(self):
        return self.e.torch_device() if hasattr(self.e, "torch_device") else "cpu"

    def exchange(self, send, counts: list[int]):
        """All-to-all of state records: counts[d] records of `send` (a uint8
        device tensor, destinations in rank order) go to rank d.  Returns the
        received records (a uint8 tensor on the engine's device, sources in rank
        order) and their number.  Counts travel first (one int64 per rank)."""
        import torch

        d = _dist()
        dev = self._device()
        if not d or self.world == 1:
            return torch.empty(0, dtype=torch.uint8, device=dev), 0
        stage = d.get_backend(self.group) == "gloo" and torch.device(dev).type == "cuda"
        cdev = "cpu" if stage else dev
        sc = torch.tensor(counts, dtype=torch.int64, device=cdev)
        rc = torch.empty_like(sc)
        d.all_to_all_single(rc, sc, group=self.group)
        recv_counts = [int(v) for v in rc.tolist()]
        payload = send.to(cdev) if stage else send
        recv = torch.empty(sum(recv_counts) * REC, dtype=torch.uint8, device=cdev)
        d.all_to_all_single(recv, payload, output_split_sizes=[c * REC for c in recv_counts],
                            input_split_sizes=[c * REC for c in counts], group=self.group)
        return (recv.to(dev) if stage else recv), sum(recv_counts)

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
        self.e.pack_layers(0, lo, True, None, 0)  # removed, not packed
        self.e.pack_layers(hi, self.nz, True, None, 0)
        return self.bounds

    # ------------------------------------------------------------- iteration
    def _pack(self, ranges, remove: bool):
        """State records of the live objects of the layer ranges (one per rank,
        None: nothing for that rank) packed back to back into one device
        buffer; returns it and the per-rank counts."""
        import torch

        hist = np.asarray(self.e.layer_histogram(), dtype=np.int64)
        counts = [0 if r is None else int(hist[r[0]:r[1]].sum()) for r in ranges]
        buf = torch.empty(max(sum(counts), 1) * REC, dtype=torch.uint8, device=self._device())
        off = 0
        for r, c in zip(ranges, counts):
            if c:
                got = self.e.pack_layers(r[0], r[1], remove, buf[off * REC:], c)
                if got != c:
                    raise RuntimeError(f"layer histogram and packing disagree ({got} vs {c})")
                off += c
        return buf[: off * REC], counts

    def migrate(self) -> int:
        """Hands the objects that left this rank's layers to their owners and
        appends the arrivals; returns the number of arrivals."""
        ranges = [None if d == self.rank else (self.bounds[d], self.bounds[d + 1]) for d in range(self.world)]
        send, counts = self._pack(ranges, remove=True)
        self.migrated += sum(counts)
        recv, m = self.exchange(send, counts)
        self.e.append_records(recv, m)
        return m

    def scan(self, dt_scan: float) -> np.ndarray:
        """Pair scan of this rank's objects with each other and with the halo
        (the next rank's lowest `reach` layers); records of this rank."""
        lo = self.bounds[self.rank]
        ranges = [None] * self.world
        if self.rank > 0:  # this rank's lowest layers are the halo of the rank below
            ranges[self.rank - 1] = (lo, lo + self.reach)
        send, counts = self._pack(ranges, remove=False)
        halo, m = self.exchange(send, counts)
        n0 = self.e.size()
        if m:
            self.e.append_records(halo, m)
            self.e.set_halo(n0)
        try:
            recs = self.e.conjunctions(dt_scan)
        finally:
            self.e.set_halo(None)
            self.e.truncate(n0)
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
