"""Benchmark of the LADDS propagate + conjunction hot path on B200.

Workload (the configuration the headline metric is quoted on): 1,000,000
objects from the seeded population 0 (a = R + U[400,1500] km, e U[0,0.02],
i U[0,180] deg, radius logU[0.01,5] m), full perturbation set (KEP, J2, J3,
C22, S22, Sun, Moon, SRP, drag), dt = 10 s, conjunction scan every step with
the 80 km cell-list cutoff and the 0.1 km conjunction threshold.

One step = one iteration of the reference loop (Simulation.cpp:287-415):
Yoshida-4 step of every object, then the conjunction scan.  ``value`` is the
split-precision object-steps/s with the population resident in HBM; the FP64
figure and their ratio are reported beside it, and further legs measure:
split vs FP64 per population (position drift and the conjunction sets compared
pair by pair), the constellation and 8e6 scale populations (autotuned), the
adjoint of 4096 conjunction pairs with its finite-difference check, and the 8e6
population's breakups over one day.  The line ends with ``targets``, a
summary of those figures against the targets (mixed / FP64, drift, conjunction
sets, adjoint / forward, finite-difference agreement, breakup counts).  ``e2e`` runs the same steps through the C ABI in the host-owned
mode of the drop-in (ladds_gpu_step_host): per step the positions/velocities
go host->device from pinned memory, the step runs, positions/velocities and
the conjunction records come back; ``e2e.device_resident`` is the drop-in's own data flow, the
population kept on the device and each iteration's records read back.
``--impl reference`` times the CPU restatement of the reference path (the
oracle; the reference itself cannot be built here).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_OBJECTS = 1_000_000
SEED = 1001
METRIC = "object-steps/s, mixed vs FP64 on B200 at <=1 m/day drift; adjoint/forward time"
WORKLOAD = "population 0, 1e6 objects, full perturbations, dt 10 s, scan every step (80 km cutoff, 0.1 km threshold)"
STEPS_PER_DAY = 8640


# ----------------------------------------------------------------- helpers
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        import datetime

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ----------------------------------------------------------- algorithmic work
def algorithmic_units(n):
    """Per-step algorithmic bytes of each phase: the bytes the phase must move per object
    at the least, from the data each kernel reads and writes (listed per entry)."""
    return {
        # read r, v, aom, bcInv, tag (68 B), write r, v (48 B), write the cell key (4 B)
        "propagate": {"bytes": n * 120},
        # count (key 4), scatter (key + tag 8 in, record + source 12 out)
        "bucket": {"bytes": n * (4 + 8 + 12)},
        # row sort: record + source in (12), sorted key + slot out (8)
        "rowsort": {"bytes": n * (12 + 8)},
        # gather r, v, aom, bcInv, tag (68 B) + perm 4 into cell order, radius by slot (8 B); write 68 B SoA
        # + 32 B binary32 position / velocity copies (radius, id, parent stay in slot order)
        "permute": {"bytes": n * (68 + 4 + 8 + 68 + 32)},
        # own key, tag, posf (24 B) + the closest-approach screen of the pre-filtered pairs: binary32
        # position + velocity of both objects (64 B, ~1.5 pairs per object)
        "candidates": {"bytes": n * (24 + 96)},
        # FP64 records of the few screened pairs (a few per thousand objects): no per-object traffic
        "evaluate": {"bytes": 0},
    }


def profiled_traffic(n):
    """DRAM bytes per launch of each phase's main kernel from the committed ncu
    summary (1e6 objects), scaled to n objects, and the same capture's issue
    and DRAM utilisation (fractions) of that kernel."""
    out, util = {}, {}
    try:
        for line in open(os.path.join(ROOT, "profiles", "dram_traffic_population0_1e6.txt")):
            if line.strip() and not line.startswith("#"):
                f = line.split()
                out[f[0]] = int(f[2]) * n / 1e6
                if len(f) >= 5:
                    util[f[0]] = {"issue_active": float(f[3]) / 100.0, "dram_throughput": float(f[4]) / 100.0}
    except (OSError, ValueError):
        pass
    return out, util


def propagation_flops(mask_full=True):
    # counted FP operations per force evaluation of the restated model (transcendentals as 1):
    # radius terms 8, Kepler 8, J2 18, J3 25, C22/S22 42, Sun 24, Moon 24, SRP 28, drag 28 + band
    # search = 208; Kepler + J2 alone 33; + 42 for the drift / kick updates of a step
    f_eval = 208 if mask_full else 33
    return 3 * f_eval + 42


def measure_peaks():
    try:
        import ctypes as C

        from ladds_b200 import build

        lib = C.CDLL(build.build_peaks())
        f64, f32 = C.c_double(), C.c_double()
        lib.ladds_measure_fma_tflops.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        if lib.ladds_measure_fma_tflops(0, C.byref(f64), C.byref(f32)) == 0:
            return f64.value, f32.value
    except Exception:
        pass
    return None, None


def measured_peaks_file():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(p))
    except Exception:
        return {}


# ------------------------------------------------------------- CPU baseline
def bench_population(args, seed):
    """The benchmark's population: the binary SoA population file given with
    --population, else the seeded population 0 of --n-objects objects."""
    from ladds_b200 import population  # host-only library: no GPU code in the process

    if args.population:
        return population.load_population(args.population)
    return population.generate_population(0, seed, args.n_objects)


def workload_name(args, n):
    if args.population:
        return (f"population file {os.path.basename(args.population)} ({n} objects), " + WORKLOAD.split(", ", 2)[2])
    return WORKLOAD


def bench_config(args, n):
    """The workload both arms print, key for key: what is computed, not how."""
    return {"workload": workload_name(args, n), "n_objects": n, "dt_s": 10.0, "scan_every_steps": 1,
            "cutoff_km": 80.0, "conjunction_threshold_km": 0.1,
            "forces": "KEP J2 J3 C22 S22 SOL LUN SRP DRAG"}


def cpu_baseline(pop, budget_s=20.0, steps_cap=None):
    """Times the oracle (C + OpenMP restatement of the reference path) on the host
    cores: full Yoshida step of the full force set + linked-cell scan."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O

    opop = O.Population(pop["x"], pop["y"], pop["z"], pop["vx"], pop["vy"], pop["vz"], pop["radius"], pop["aom"],
                        pop["bc_inv"], pop["id"], pop["parent"], pop["activity"])
    grid = O.make_grid([-10000.0] * 3, [10000.0] * 3, 0.0, 80.0)
    params = O.scan_params(cutoff=80.0, dt=10.0)
    cores = os.cpu_count() or 1
    # one full step first, to size the sample
    t0 = time.perf_counter()
    O.propagate(opop, O.FULL, 10.0, 1, t0=0.0)
    O.scan_cells(opop, params, grid, step=0)
    t_full = time.perf_counter() - t0
    return O, opop, grid, params, t_full, cores


def wedge_population(pop, frac):
    """Objects with longitude in [0, 2 pi frac): a same-density sample."""
    lon = np.arctan2(pop["y"], pop["x"]) % (2 * math.pi)
    keep = lon < 2 * math.pi * frac
    return {k: (v[keep] if isinstance(v, np.ndarray) else v) for k, v in pop.items()}


def run_reference(args, world, rank):
    """--impl reference: the CPU restatement on all host cores, bounded sample per step."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O

    pop = bench_population(args, SEED)
    grid = O.make_grid([-10000.0] * 3, [10000.0] * 3, 0.0, 80.0)
    params = O.scan_params(cutoff=80.0, dt=10.0)

    def to_o(p):
        return O.Population(p["x"], p["y"], p["z"], p["vx"], p["vy"], p["vz"], p["radius"], p["aom"], p["bc_inv"],
                            p["id"], p["parent"], p["activity"])

    # size the per-step sample so that warm-up + timed steps fit the budget
    probe = to_o(wedge_population(pop, 0.05))
    t0 = time.perf_counter()
    O.propagate(probe, O.FULL, 10.0, 1)
    O.scan_cells(probe, params, grid)
    t_probe = max(time.perf_counter() - t0, 1e-4)
    per_obj = t_probe / max(probe.n, 1)
    budget = args.reference_budget
    m_target = budget / max(args.steps + args.warmup, 1) / per_obj
    frac = min(1.0, max(m_target / max(len(pop["x"]), 1), 1e-4))
    sample = to_o(wedge_population(pop, frac))
    for w in range(args.warmup):
        O.propagate(sample, O.FULL, 10.0, 1, t0=10.0 * w)
        O.scan_cells(sample, params, grid, step=w)
    t0 = time.perf_counter()
    for s in range(args.steps):
        O.propagate(sample, O.FULL, 10.0, 1, t0=10.0 * (args.warmup + s))
        O.scan_cells(sample, params, grid, step=args.warmup + s)
    el = time.perf_counter() - t0
    value = sample.n * args.steps / el
    cores = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "object-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "population file" if args.population else "synthetic (seeded population 0)",
        "config": bench_config(args, len(pop["x"])),
        "parallelism": "1 process, OpenMP",
        "l2": "n/a (CPU)",
        "cpu_baseline": {"value": value, "unit": "object-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{sample.n} objects (longitude wedge of {frac:.4f} of the population, same "
                                   f"density) x {args.steps} steps per timed step"},
        "e2e": {"value": value, "unit": "object-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------ other workloads
def workload_leg(capi, device, which, n, steps, tune):
    """Throughput of population `which` (2: four constellation shells + debris,
    4: small-debris mixture) with the full force set in split precision, scan
    every step; optionally autotuned first (cell edge, block shapes, chunk)."""
    pop = capi.generate_population(which, SEED + which, n)
    out = {"population": which, "n_objects": n, "steps": steps}
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL, precision=capi.PRECISION_SPLIT,
                                          device=device, pairCapacity=1 << 18)) as ctx:
        ctx.upload(pop)
        ctx.step(4)
        if tune:
            best, trials = ctx.autotune(16)
            out["autotuned"] = best
            out["trials"] = len(trials)
        ctx.step(8)
        res = ctx.step(steps)
        ms = res.stats.deviceMs
        out.update({"value": n * steps / (ms * 1e-3), "unit": "object-steps/s", "ms_per_step": ms / steps,
                    "records": int(res.stats.records), "collisions": int(res.stats.collisions)})
    return out


# ------------------------------------------------------------ drift legs
def closest_approach(ri, vi, rj, vj, dt):
    """Distance at the endpoint and least distance of the straight segments
    back-extrapolated over [-dt, 0] (the geometry of
    DistanceApproximation.cpp:13-58, in numpy binary64; for classifying
    differing records, not for parity)."""
    dr, dv = ri - rj, vi - vj
    o = dr - dv * dt
    dv2 = np.sum(dv * dv, axis=-1)
    with np.errstate(invalid="ignore", divide="ignore"):
        t = np.clip(-np.sum(o * dv, axis=-1) / dv2, 0.0, dt)
    t = np.where(np.isfinite(t), t, 0.0)
    m = o + dv * t[..., None]
    return np.sqrt(np.sum(dr * dr, axis=-1)), np.sqrt(np.sum(m * m, axis=-1))


def objects_at_steps(capi, cfg, pop, wanted):
    """{(step, slot): (r, v)}: the states of the wanted (step, slot) pairs, by
    re-running the population from its start and stopping after each wanted
    step (a record of step s is scanned on the state after s + 1 iterations)."""
    out = {}
    by_step = {}
    for s_, sl in wanted:
        by_step.setdefault(s_, set()).add(sl)
    with capi.Context(cfg) as ctx:
        ctx.upload(pop)
        done = 0
        for s_ in sorted(by_step):
            if s_ + 1 > done:
                ctx.step(s_ + 1 - done)
                done = s_ + 1
            slots = np.array(sorted(by_step[s_]), dtype=np.uint32)
            objs = ctx.get_objects(slots)
            for sl, o in zip(slots, objs):
                out[(s_, int(sl))] = (np.array(o["r"]), np.array(o["v"]), float(o["radius"]), int(o["activity"]))
    return out


LIST_BITS = 1 | 2 | 4  # collision, evasion, conjunction
NEAR_BITS = 8 | 16 | 32 | 64  # near bands of those thresholds and of the cutoff gate


def classify_differences(capi, cfgs, pop, recs, dt):
    """The conjunction sets (records with a collision, evasion or conjunction
    bit) of the two precisions, pair by pair.  Records that carry only a
    near-band flag (listed separately, not part of the set) are counted apart.
    A pair whose list bits differ is near-flagged when either run flags it in
    the near band of a threshold or of the cutoff gate; otherwise its
    split-vs-FP64 difference at that step (states re-run to that step in both
    precisions) is set against its margin to the threshold it crosses: the
    difference is explained when the threshold (or the cutoff) lies within the
    pair's drift bound |dr_A| + |dr_B| + dt (|dv_A| + |dv_B|) of its distance."""
    key = lambda r: (int(r["step"]), int(r["idA"]), int(r["idB"]))
    ta = {key(r): r for r in recs["split"]}
    tb = {key(r): r for r in recs["fp64"]}
    flags = lambda t, k: int(t[k]["flags"]) if k in t else 0
    in_set = {name: sum(1 for r in t.values() if int(r["flags"]) & LIST_BITS) for name, t in (("split", ta),
                                                                                            ("fp64", tb))}
    near_only = sum(1 for k in set(ta) ^ set(tb) if not (flags(ta, k) | flags(tb, k)) & LIST_BITS)
    diff, near = [], 0
    for k in sorted(set(ta) | set(tb)):
        fa, fb = flags(ta, k), flags(tb, k)
        if (fa & LIST_BITS) == (fb & LIST_BITS):
            continue
        if (fa | fb) & NEAR_BITS:
            near += 1
            continue
        diff.append((k, ta.get(k, tb.get(k)), "split" if fa & LIST_BITS else "fp64"))
    out = {"set_split": in_set["split"], "set_fp64": in_set["fp64"], "set_differences": near + len(diff),
           "near_flagged": near, "not_near_flagged": len(diff), "near_band_only_records_differing": near_only}
    if not diff:
        out["explained_by_drift"] = 0
        return out
    wanted = set()
    for _, r, _ in diff:
        wanted.add((int(r["step"]), int(r["slotA"])))
        wanted.add((int(r["step"]), int(r["slotB"])))
    st = {name: objects_at_steps(capi, cfgs[name], pop, wanted) for name in ("split", "fp64")}
    cfg = cfgs["fp64"]
    rows = []
    for k, r, where in diff:
        s_, a, b = int(r["step"]), int(r["slotA"]), int(r["slotB"])
        (ra, va, rad_a, _), (rb, vb, rad_b, _) = st["split"][(s_, a)], st["split"][(s_, b)]
        (ra2, va2, _, _), (rb2, vb2, _, _) = st["fp64"][(s_, a)], st["fp64"][(s_, b)]
        bound = (np.linalg.norm(ra - ra2) + np.linalg.norm(rb - rb2)
                 + dt * (np.linalg.norm(va - va2) + np.linalg.norm(vb - vb2)))
        d1, dl1 = closest_approach(ra, va, rb, vb, dt)
        d2, dl2 = closest_approach(ra2, va2, rb2, vb2, dt)
        thr = [cfg.conjunctionThreshold, cfg.evasionCutoff,
               (rad_a + rad_b) * cfg.collisionDistanceFactor / 1000.0]
        m, t = min([(abs(dl1 - t_), t_) for t_ in thr] + [(abs(d1 - cfg.cutoff), cfg.cutoff)])
        rows.append({"step": s_, "in": where, "margin_km": float(m), "threshold_km": t, "bound_km": float(bound),
                     "dl_split_km": float(dl1), "dl_fp64_km": float(dl2)})
    explained = [x for x in rows if x["margin_km"] <= x["bound_km"] * (1 + 1e-6) + 1e-12]
    out.update({"explained_by_drift": len(explained),
                "max_margin_m": max(x["margin_km"] for x in rows) * 1e3,
                "max_margin_rel": max(x["margin_km"] / x["threshold_km"] for x in rows),
                "max_pair_drift_bound_m": max(x["bound_km"] for x in rows) * 1e3, "examples": rows[:3]})
    return out


def drift_leg(capi, device, pop, steps, cfg_kw=None):
    """Split vs FP64 from the same start over `steps` iterations (scan every
    iteration): RMS / max position difference at the end, record counts, and
    the records that only one precision lists, classified."""
    cfg_kw = dict(cfg_kw or {})
    cfgs = {name: capi.default_config(componentMask=capi.PROP_ALL, precision=prec, device=device,
                                      pairCapacity=1 << 18, **cfg_kw)
            for name, prec in (("split", capi.PRECISION_SPLIT), ("fp64", capi.PRECISION_FP64))}
    finals, recs, ms = {}, {}, {}
    for name in ("split", "fp64"):
        with capi.Context(cfgs[name]) as ctx:
            ctx.upload(pop)
            r = ctx.step(steps)
            d = ctx.download()
            finals[name] = (np.stack([d["x"], d["y"], d["z"]], 1), np.stack([d["vx"], d["vy"], d["vz"]], 1))
            recs[name] = r.records
            ms[name] = r.stats.deviceMs
    dr = finals["split"][0] - finals["fp64"][0]
    dv = finals["split"][1] - finals["fp64"][1]
    dt = cfgs["fp64"].deltaT
    out = {"n_objects": len(pop["x"]), "steps": steps, "hours": steps * dt / 3600.0,
           "rms_m": float(np.sqrt(np.mean(np.sum(dr * dr, 1)))) * 1e3,
           "max_m": float(np.max(np.linalg.norm(dr, axis=1)) * 1e3),
           "max_dv_mm_s": float(np.max(np.linalg.norm(dv, axis=1)) * 1e6),
           "records_split": len(recs["split"]), "records_fp64": len(recs["fp64"]),
           "ms_per_step_split": ms["split"] / steps, "ms_per_step_fp64": ms["fp64"] / steps}
    out["differences"] = classify_differences(capi, cfgs, pop, recs, dt)
    return out


def breakup_leg(capi, device, pop, iterations, cfg_kw, min_altitude=150.0):
    """Config 4 form over `iterations` iterations of the reference loop
    (Simulation.cpp:287-415): integrate; burn-ups below min_altitude removed
    (:302); particles leaving the container (outside the box, or a non-finite
    state) removed (:314, :381-387); the conjunction scan; every collision
    handed to the NASA breakup model on the host (BreakupWrapper.cpp:13-45),
    its fragment count recorded.  The population is the same all day (the
    fragments are counted, not appended): a breakup of these solid spheres
    (2700 kg/m^3, up to 5 m: 1.4e6 kg) yields up to ~7e5 fragments at one point,
    whose same-parent pairs the cell scan would visit quadratically.  After the
    day, the first breakup is applied for real -- fragments appended on the
    device (ladds_gpu_breakup) -- and propagated one step.  Also the expected
    collision count of the conjunction records, sum of ((r_A + r_B) / 0.1 km)^2
    over them (the fraction of a uniform-in-area miss distribution inside the
    collision radius)."""
    cfg = capi.default_config(componentMask=capi.PROP_ALL, precision=capi.PRECISION_SPLIT, device=device,
                              pairCapacity=1 << 18, **cfg_kw)
    bcfg = capi.BreakupConfig(0.05, 1, 2.2)
    n = len(pop["x"])
    next_id = int(np.max(pop["id"])) + 1 if n else 0
    tot = dict(collisions=0, breakups=0, fragments=0, conjunctions=0, burnups=0, escaped=0, nonfinite_steps=0)
    expected = 0.0
    first = None
    t0 = time.perf_counter()
    with capi.Context(cfg) as ctx:
        ctx.upload(pop)
        ctx.reserve(n + n // 8)  # room for fragments: appends reallocate nothing
        for it in range(iterations):
            if not ctx.integrate(1, allow_nonfinite=True):
                tot["nonfinite_steps"] += 1
            tot["burnups"] += len(ctx.remove_below(min_altitude))
            tot["escaped"] += len(ctx.remove_escaping())
            rec = ctx.conjunctions(cfg.deltaT)
            col = rec[(rec["flags"] & capi.PAIR_COLLISION) != 0]
            conj = rec[(rec["flags"] & capi.PAIR_CONJUNCTION) != 0]
            tot["conjunctions"] += len(conj)
            if len(conj):
                objs = ctx.get_objects(np.concatenate([conj["slotA"], conj["slotB"]]))
                ra, rb = objs["radius"][: len(conj)], objs["radius"][len(conj):]
                expected += float(np.sum(((ra + rb) * cfg.collisionDistanceFactor * 1e-3 / 0.1) ** 2))
            for q, r in enumerate(col):
                tot["collisions"] += 1
                a, b = ctx.get_objects([r["slotA"], r["slotB"]])
                frags, _ = capi.breakup_collision(bcfg, 1000 + it + q, a, b, r["point"], int(r["idA"]), next_id)
                if len(frags["x"]):
                    tot["breakups"] += 1
                    tot["fragments"] += len(frags["x"])
                    if first is None:
                        first = (it, col[q:q + 1].copy())
        wall = time.perf_counter() - t0
        applied = None
        if first is not None:  # the first breakup appended on the device, then one propagation step
            n0 = ctx.size()
            t1 = time.perf_counter()
            nb, nf, next_id = ctx.breakup(first[1], bcfg, 1000 + first[0], next_id)
            t_append = time.perf_counter() - t1
            ok = ctx.integrate(1, allow_nonfinite=True)
            gone = len(ctx.remove_escaping())
            applied = {"iteration": first[0], "breakups": nb, "fragments_appended": nf, "objects_before": n0,
                       "objects_after": ctx.size(), "append_ms": t_append * 1e3,
                       "propagated_one_step": True, "nonfinite_after_step": not ok, "escaped_after_step": gone}
    out = {"iterations": iterations, "hours": iterations * cfg.deltaT / 3600.0, **tot,
           "expected_collisions_from_conjunctions": expected, "first_breakup_applied": applied,
           "ms_per_iteration_wall": wall * 1e3 / iterations}
    out["applied_run"] = applied_breakup_run(capi, cfg, bcfg, pop, iterations, min_altitude)
    return out


def applied_breakup_run(capi, cfg, bcfg, pop, iterations, min_altitude, wall_budget_s=45.0):
    """The same loop with every breakup applied: fragments appended on the
    device (ladds_gpu_breakup), burn-ups and escaping fragments removed, until
    the day ends, the wall budget is spent or a call fails.  Fragments of one
    breakup start at one point; their same-parent pairs are skipped by the
    functor (spawn protection) but still visited by the cell scan, so a large
    breakup slows the following iterations until the cloud disperses."""
    n = len(pop["x"])
    next_id = int(np.max(pop["id"])) + 1 if n else 0
    tot = dict(iterations=0, breakups=0, fragments=0, burnups=0, escaped=0)
    parts = ("integrate", "burnups", "escaping", "scan", "breakups")
    times = []  # per iteration: wall seconds of each part
    err = None
    t0 = time.perf_counter()
    with capi.Context(cfg) as ctx:
        ctx.upload(pop)
        ctx.reserve(n + n // 8)  # room for fragments: appends reallocate nothing
        try:
            for it in range(iterations):
                t = [time.perf_counter()]
                ctx.integrate(1, allow_nonfinite=True)
                t.append(time.perf_counter())
                tot["burnups"] += len(ctx.remove_below(min_altitude))
                t.append(time.perf_counter())
                tot["escaped"] += len(ctx.remove_escaping())
                t.append(time.perf_counter())
                rec = ctx.conjunctions(cfg.deltaT)
                t.append(time.perf_counter())
                if np.any(rec["flags"] & capi.PAIR_COLLISION):
                    nb, nf, next_id = ctx.breakup(rec, bcfg, 1000 + it, next_id)
                    tot["breakups"] += nb
                    tot["fragments"] += nf
                t.append(time.perf_counter())
                tot["iterations"] = it + 1
                times.append(np.diff(t))
                if time.perf_counter() - t0 > wall_budget_s:
                    break
            if times:  # where the last iterations' time goes, on the device
                ctx.set_profiling(True)
                ctx.conjunctions(cfg.deltaT)
                pt = ctx.phase_times()
                device_scan = {p: round(getattr(pt, p + "Ms"), 3) for p in capi.PhaseTimes.PHASES}
                ctx.set_profiling(False)
        except Exception as ex:  # noqa: BLE001
            err = str(ex)[:160]
        size = ctx.size()
    last = np.mean(times[-100:], axis=0) * 1e3 if times else np.zeros(len(parts))
    return {**tot, "objects_after": size, "stopped_by": "error" if err else
            ("wall budget" if tot["iterations"] < iterations else "end of run"), "error": err,
            "ms_per_iteration_last_100": float(np.sum(last)),
            "ms_last_100_by_part": {p: round(float(v), 3) for p, v in zip(parts, last)},
            "device_ms_of_one_scan_at_the_end": device_scan if times and not err else None,
            "wall_budget_s": wall_budget_s}


# ---------------------------------------------------------- adjoint leg
FD_STENCIL = (1.0, -1.0, 0.5, -0.5, 0.25, -0.25)  # multiples of h of the perturbed evaluations


def fd_classify(gd, f0, fm, step0, stepm, eps, tol=1e-6, consistency=1e-3, with_classes=False):
    """Finite-difference check of directional derivatives gd (one per pair)
    from the losses f0 at x and fm[k] at x + FD_STENCIL[k] h d, with the argmin
    steps step0 / stepm[k] of each evaluation.

    The loss is a minimum over steps (and, inside a step, over the clamped
    closest-approach time), so it has kinks where two branches tie; the
    gradient is the derivative of the branch active at x.  Per pair and per
    side: a side whose three points keep the argmin step gives a one-sided
    Richardson extrapolation of D(t) = (f(t) - f0) / t over t = h, h/2, h/4,
    (8 D(h/4) - 6 D(h/2) + D(h)) / 3 (error O(h^3)), provided its two
    second-order estimates 2 D(h/2) - D(h) and 2 D(h/4) - D(h/2) agree to
    `consistency` (a kink inside the step -- the clamp of the closest-approach
    time -- between the side's points breaks that); the central quotients
    C(t) = (f(t) - f(-t)) / 2t give (64 C(h/4) - 20 C(h/2) + C(h)) / 45 (error
    O(h^6)).  Both sides usable and agreeing to tol: the central value.  Both
    usable but disagreeing: a kink within h/4 of x, on an unknown side
    ("ambiguous", the closer side's error is reported).  One side usable: that
    side.  Neither: unresolved at this h.  Returns the per-pair relative
    errors and the counts of each class (and, with_classes, the per-pair
    class masks)."""
    keep = stepm == step0[None, :]
    d = lambda k, t: (fm[k] - f0) / (t * eps)  # one-sided quotient at t h (t may be negative)
    # a side is usable when its three points keep the argmin step and its two
    # second-order estimates agree (a clamp kink inside the step breaks them)
    r1p, r2p = 2.0 * d(2, 0.5) - d(0, 1.0), 2.0 * d(4, 0.25) - d(2, 0.5)
    r1m, r2m = 2.0 * d(3, -0.5) - d(1, -1.0), 2.0 * d(5, -0.25) - d(3, -0.5)
    fwd, bwd = (4.0 * r2p - r1p) / 3.0, (4.0 * r2m - r1m) / 3.0
    smooth_p = np.abs(r1p - r2p) <= consistency * np.maximum(np.abs(r2p), 1e-300)
    smooth_m = np.abs(r1m - r2m) <= consistency * np.maximum(np.abs(r2m), 1e-300)
    keep_p = keep[0] & keep[2] & keep[4] & smooth_p
    keep_m = keep[1] & keep[3] & keep[5] & smooth_m
    c = lambda kp, km, t: (fm[kp] - fm[km]) / (2.0 * t * eps)
    cen = (64.0 * c(4, 5, 0.25) - 20.0 * c(2, 3, 0.5) + c(0, 1, 1.0)) / 45.0
    scale = np.maximum(np.abs(cen), 1e-300)
    both = keep_p & keep_m
    agree = both & (np.abs(fwd - bwd) <= tol * scale)
    rel = np.full(len(gd), np.inf)
    err = lambda ref: np.abs(gd - ref) / np.maximum(np.abs(ref), 1e-300)
    rel[agree] = err(cen)[agree]
    kink = both & ~agree
    rel[kink] = np.minimum(err(fwd), err(bwd))[kink]
    only_p, only_m = keep_p & ~keep_m, keep_m & ~keep_p
    rel[only_p] = err(fwd)[only_p]
    rel[only_m] = err(bwd)[only_m]
    unresolved = ~keep_p & ~keep_m
    counts = {"central": int(agree.sum()), "ambiguous": int(kink.sum()), "forward_only": int(only_p.sum()),
              "backward_only": int(only_m.sum()), "unresolved": int(unresolved.sum()),
              "central_meeting_tol": int(np.sum(rel[agree] <= tol))}
    if with_classes:
        return rel, counts, {"central": agree, "one_sided": only_p | only_m, "ambiguous": kink}
    return rel, counts


FD_LADDER = (1e-6, 1e-7, 1e-8)  # relative step sizes of the finite-difference ladder


def fd_ladder(levels, tol=1e-6):
    """Per pair, the finite-difference value at the largest h of the ladder
    where it is resolved, in the order central (both sides smooth and
    agreeing), one-sided, ambiguous (a kink within h/4): a kink of the
    minimum-over-steps loss that lies inside the stencil at h usually lies
    outside it at h/10 or h/100, and the binary64 round-off of the quotients
    stays near 1e-16 |x| / (h |d|) <= 1e-8 of the derivative at h = 1e-8 |x|.
    levels: [(h_rel, rel, classes)] from fd_classify(..., with_classes=True)."""
    n = len(levels[0][1])
    best, level = np.full(n, np.inf), np.full(n, -1)
    for cls_name in ("central", "one_sided", "ambiguous"):
        for li, (_, rel, cls) in enumerate(levels):
            m = (level < 0) & cls[cls_name]
            best[m], level[m] = rel[m], li
    fin = best[np.isfinite(best)]
    return {"h": [h for h, _, _ in levels],
            "resolved_at": [int(np.sum(level == li)) for li in range(len(levels))],
            "unresolved": int(np.sum(level < 0)),
            "meets_1e-6": int(np.sum(best <= tol)), "meets_1e-6_frac": float(np.mean(best <= tol)),
            "rel_err_median": float(np.median(fin)) if len(fin) else None,
            "rel_err_p99": float(np.quantile(fin, 0.99)) if len(fin) else None}


def adjoint_leg(capi, device, n_pairs=4096, steps=1080, ck=64, reps=3):
    """Differentiation workload: 4096 pairs, 1080 FP64 steps of the full force
    set, checkpoints every 64 steps.  Device times of the forward sweep (loss +
    checkpoints) and of the backward sweep (segment recompute + reverse sweep),
    and a directional finite-difference check of every pair's gradient at
    h = 1e-6 |x| (fd_classify), and per pair at the largest h of 1e-6, 1e-7,
    1e-8 |x| where it is resolved (fd_ladder)."""
    with capi.Context(capi.default_config(componentMask=capi.PROP_ALL, device=device)) as ctx:
        pairs, _ = ctx.adjoint_make_pairs(77, n_pairs, steps)
        ctx.adjoint_forward(pairs, steps, ck)
        ctx.adjoint_backward()
        fwd, bwd = [], []
        for _ in range(reps):
            fwd.append(ctx.adjoint_forward(pairs, steps, ck)[3])
            dx, _, ms = ctx.adjoint_backward()
            bwd.append(ms)
        rows = np.concatenate([pairs["rA"], pairs["vA"], pairs["rB"], pairs["vB"]], axis=1)
        rng = np.random.default_rng(3)
        d = rng.normal(size=rows.shape) * np.abs(rows)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        _, miss0, step0, _ = ctx.adjoint_forward(pairs, steps, ck)
        gd = np.sum(dx * d, axis=1)
        k = len(FD_STENCIL)
        levels = []
        for h_rel in FD_LADDER:
            eps = h_rel * np.linalg.norm(rows, axis=1)
            batch = []
            for f in FD_STENCIL:
                q = pairs.copy()
                r = rows + f * eps[:, None] * d
                q["rA"], q["vA"], q["rB"], q["vB"] = r[:, 0:3], r[:, 3:6], r[:, 6:9], r[:, 9:12]
                batch.append(q)
            _, miss, stepP, _ = ctx.adjoint_forward(np.concatenate(batch), steps, ck)
            lv = fd_classify(gd, miss0, miss.reshape(k, n_pairs), step0, stepP.reshape(k, n_pairs), eps,
                             with_classes=True)
            if not levels:
                rel, counts, _ = lv
            levels.append((h_rel, lv[0], lv[2]))
    ladder = fd_ladder(levels)
    fin = rel[np.isfinite(rel)]
    f_ms, b_ms = float(np.median(fwd)), float(np.median(bwd))
    fd = {"direction": "random per pair, 12 state components, relative scaling", "h": "1e-6 |x|, h/2, h/4",
          "pairs": n_pairs, **counts,
          "meets_1e-6": int(np.sum(rel <= 1e-6)), "meets_1e-6_frac": float(np.mean(rel <= 1e-6)),
          "rel_err_median": float(np.median(fin)) if len(fin) else None,
          "rel_err_p99": float(np.quantile(fin, 0.99)) if len(fin) else None,
          "ladder": ladder}
    return {"pairs": n_pairs, "steps": steps, "checkpoint_every": ck, "forward_ms": f_ms, "backward_ms": b_ms,
            "backward_over_forward": b_ms / f_ms, "forward_plus_backward_over_forward": (f_ms + b_ms) / f_ms,
            "fd_check": fd,
            "fd_summary": {"meets_1e-6_frac": fd["meets_1e-6_frac"], "unresolved": counts["unresolved"],
                           "median": fd["rel_err_median"],
                           "ladder_meets_1e-6_frac": ladder["meets_1e-6_frac"],
                           "ladder_unresolved": ladder["unresolved"]}}


# ------------------------------------------------------------------ GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=STEPS_PER_DAY)
    ap.add_argument("--warmup", type=int, default=16)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-objects", type=int, default=N_OBJECTS)
    ap.add_argument("--population", default=None,
                    help="binary SoA population file (ladds_population_write) instead of the seeded population 0")
    ap.add_argument("--e2e-steps", type=int, default=40)
    ap.add_argument("--no-drift", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-workloads", action="store_true")
    ap.add_argument("--drift-steps-8m", type=int, default=STEPS_PER_DAY // 3,
                    help="iterations of the split-vs-FP64 comparison on the 8e6 population (0: skip)")
    ap.add_argument("--breakup-steps", type=int, default=STEPS_PER_DAY,
                    help="iterations of the 8e6 breakup run (host breakups, device append; 0: skip)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--reference-budget", type=float, default=150.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        # rank 0 alone times the CPU path; no process group (there is no collective)
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_init(args)

    from ladds_b200 import build, capi

    build.build_gpu()
    pop = bench_population(args, SEED + rank)  # replicas: one population per rank (or the file's)
    n = len(pop["x"])

    def make_ctx(precision, graphs=1):
        return capi.Context(capi.default_config(componentMask=capi.PROP_ALL, precision=precision, device=local,
                                                useGraphs=graphs, pairCapacity=1 << 16))

    results = {}
    for name, prec in (("split", capi.PRECISION_SPLIT), ("fp64", capi.PRECISION_FP64)):
        ctx = make_ctx(prec)
        ctx.upload(pop)
        ctx.step(args.warmup)
        # the timed call captures its CUDA graphs (one per 128-step chunk) before
        # its first timing event, so device time covers the replay only
        dist_barrier(world)
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            res = ctx.step(args.steps)
            wall = time.perf_counter() - t0
        dev_ms = dist_max(res.stats.deviceMs, world)
        results[name] = dict(ms=dev_ms, wall=wall, records=int(res.stats.records), clocks=clk.summary(),
                             conj=int(res.stats.conjunctions), coll=int(res.stats.collisions))
        # per-phase device times (eager, CUDA events on the library stream), same workload
        ctx.set_profiling(True)
        ctx.step(min(args.steps, 64))
        pt = ctx.phase_times()
        results[name]["phases"] = {p: getattr(pt, p + "Ms") for p in capi.PhaseTimes.PHASES}
        results[name]["phases"]["steps"] = min(args.steps, 64)
        results[name]["phases"]["launches"] = {p: getattr(pt, p + "Launches") for p in capi.PhaseTimes.PHASES}
        ctx.set_profiling(False)
        ctx.close()

    # the characterisation legs run once, in the one-GPU run: with replicas on
    # several GPUs they would hold every GPU while rank 0 alone works
    legs = world == 1
    workloads = {}
    if not args.no_workloads and legs:
        for name, which, n_obj, steps, tune in (("constellation_shells", 2, 2_004_224, 128, True),
                                                ("scale_8M", 4, 8_000_000, 32, True)):
            try:
                workloads[name] = workload_leg(capi, local, which, n_obj, steps, tune)
            except Exception as ex:  # noqa: BLE001
                workloads[name] = {"error": str(ex)[:200]}

    adjoint = None
    if not args.no_adjoint and legs:
        try:
            adjoint = adjoint_leg(capi, local)
        except Exception as ex:  # noqa: BLE001
            adjoint = {"error": str(ex)[:200]}
            print(f"adjoint leg failed: {ex}", file=sys.stderr)

    # split vs FP64 from the same start, per population: the benchmark's own
    # population over one day, the constellation population over one day, the
    # 8e6 scale population (in its autotuned cell form) over --drift-steps-8m
    drift = {}
    scale_kw = {}
    tuned = workloads.get("scale_8M", {}).get("autotuned")
    if tuned:
        scale_kw = {k: tuned[k] for k in ("cellSize", "scanScreen", "walkForm", "propagateBlock", "scanBlock")}
    if not args.no_drift and legs:
        for name, mk_pop, steps, kw in (
                ("population0_1e6", lambda: pop, STEPS_PER_DAY, {}),
                ("constellation_shells_2e6", lambda: capi.generate_population(2, SEED + 2, 2_004_224),
                 STEPS_PER_DAY, {}),
                ("scale_8e6", lambda: capi.generate_population(4, SEED + 4, 8_000_000), args.drift_steps_8m,
                 scale_kw)):
            if steps <= 0:
                continue
            try:
                drift[name] = drift_leg(capi, local, mk_pop(), steps, kw)
            except Exception as ex:  # noqa: BLE001
                drift[name] = {"error": str(ex)[:200]}
                print(f"drift leg {name} failed: {ex}", file=sys.stderr)

    breakups = None
    if not args.no_workloads and legs and args.breakup_steps > 0:
        try:
            breakups = breakup_leg(capi, local, capi.generate_population(4, SEED + 4, 8_000_000),
                                   args.breakup_steps, scale_kw)
        except Exception as ex:  # noqa: BLE001
            breakups = {"error": str(ex)[:200]}
            print(f"breakup leg failed: {ex}", file=sys.stderr)

    # end to end through the C ABI, host-owned container: H2D state, step, D2H state + records
    e2e = None
    try:
        import torch

        ctx = make_ctx(capi.PRECISION_SPLIT, graphs=0)
        ctx.upload(pop)
        ctx.step(2)
        pinned = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(6)]
        st = ctx.get_state()
        for a, b in zip(pinned, st):
            a[:] = b
        out = np.zeros(1 << 16, dtype=capi.PAIR_DTYPE)
        ctx.step_host(pinned, out=out)  # warm-up
        dist_barrier(world)
        t0 = time.perf_counter()
        rec_bytes = 0
        for _ in range(args.e2e_steps):
            r = ctx.step_host(pinned, out=out)
            rec_bytes += len(r.records) * 64 + 8
        el = dist_max(time.perf_counter() - t0, world)
        e2e = {"value": world * n * args.e2e_steps / el, "unit": "object-steps/s",
               "h2d_bytes_per_step": 48 * n, "d2h_bytes_per_step": int(48 * n + rec_bytes / args.e2e_steps),
               "steps": args.e2e_steps,
               "mode": "host-owned state, pinned: ladds_gpu_step_host per iteration (chunked copies in and out "
                       "overlapped with the propagation and the scan)"}
        # the same iterations as three calls: set_state / step(1) / get_state
        dist_barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            ctx.set_state(*pinned)
            ctx.step(1, out=out)
            ctx._check(ctx._L.ladds_gpu_get_state(ctx.handle, n, *[a.ctypes.data_as(capi.C.c_void_p)
                                                                    for a in pinned]))
        el = dist_max(time.perf_counter() - t0, world)
        e2e["three_calls"] = {"value": world * n * args.e2e_steps / el, "unit": "object-steps/s",
                              "mode": "set_state / step(1) / get_state per iteration, pinned"}
        # the same with pageable arrays (a std::vector's storage: ladds::Integrator without residency)
        pageable = [np.array(a) for a in pinned]
        dist_barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            ctx.set_state(*pageable)
            ctx.step(1, out=out)
            ctx._check(ctx._L.ladds_gpu_get_state(ctx.handle, n, *[a.ctypes.data_as(capi.C.c_void_p)
                                                                    for a in pageable]))
        el = dist_max(time.perf_counter() - t0, world)
        e2e["three_calls_pageable"] = {"value": world * n * args.e2e_steps / el, "unit": "object-steps/s",
                                       "mode": "set_state / step(1) / get_state per iteration, pageable "
                                               "(staged through the context's pinned buffer)"}
        # the drop-in's own data flow (ladds::HotPathLoop): the population stays on the device and
        # each iteration's records come back to the host (pinned) from one ladds_gpu_step(1) call
        outp = torch.empty((1 << 16) * capi.PAIR_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True).numpy()
        outp = outp.view(capi.PAIR_DTYPE)
        dist_barrier(world)
        t0 = time.perf_counter()
        rec_bytes = 0
        for _ in range(args.e2e_steps):
            r = ctx.step(1, out=outp)
            rec_bytes += len(r.records) * 64 + 8
        el = dist_max(time.perf_counter() - t0, world)
        e2e["device_resident"] = {"value": world * n * args.e2e_steps / el, "unit": "object-steps/s",
                                  "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(rec_bytes / args.e2e_steps),
                                  "mode": "device-resident population, records to pinned host memory "
                                          "(ladds_gpu_step(1) per iteration)"}
        ctx.close()
    except Exception as ex:  # noqa: BLE001
        e2e = {"value": None, "unit": "object-steps/s", "error": str(ex)[:200]}

    if rank != 0:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    split, fp64 = results["split"], results["fp64"]
    value = world * n * args.steps / (split["ms"] * 1e-3)
    fp64_value = world * n * args.steps / (fp64["ms"] * 1e-3)

    # roofline of the dominant kernel (from the per-phase device times)
    units = algorithmic_units(n)
    ph = split["phases"]
    per = {k: ph[k] / ph["steps"] for k in capi.PhaseTimes.PHASES}
    dominant = max(per, key=per.get)
    peaks = measured_peaks_file()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    f64_peak, f32_peak = measure_peaks()
    kernels = {}
    for k, ms in per.items():
        gbs = units[k]["bytes"] / (ms * 1e-3) / 1e9 if ms > 0 else None
        kernels[k] = {"ms_per_step": ms, "algorithmic_bytes": units[k]["bytes"], "achieved_gbs": gbs,
                      "hbm_frac": gbs / hbm_peak if gbs else None}
    fp64_ph = fp64["phases"]
    prop64_ms = fp64_ph["propagate"] / fp64_ph["steps"]
    prop_flops = propagation_flops() * n
    kernels["propagate_fp64_mode"] = {"ms_per_step": prop64_ms, "algorithmic_flops": prop_flops,
                                      "achieved_tflops": prop_flops / (prop64_ms * 1e-3) / 1e12,
                                      "fp64_fma_peak_tflops_measured": f64_peak}
    if f64_peak:
        kernels["propagate_fp64_mode"]["fp64_frac"] = kernels["propagate_fp64_mode"]["achieved_tflops"] / f64_peak
    dk = kernels[dominant]
    traffic_all, util = profiled_traffic(n)
    traffic = traffic_all.get(dominant)
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": dk["achieved_gbs"], "peak": hbm_peak,
                "unit": "GB/s", "frac": dk["hbm_frac"], "traffic": traffic,
                "traffic_source": "profiles/dram_traffic_population0_1e6.txt (one ncu capture, scaled by n/1e6)"
                if traffic else None,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else "fallback"}
    if dominant in util:  # what the same ncu capture shows bounds the kernel instead of HBM
        u = util[dominant]
        roofline["ncu_issue_active"] = u["issue_active"]
        roofline["ncu_dram_throughput"] = u["dram_throughput"]
        roofline["limiter"] = ("instruction issue" if u["issue_active"] > 0.6 and u["dram_throughput"] < 0.3
                               else "hbm" if u["dram_throughput"] > 0.5 else "latency")

    cpu = None
    if not args.no_cpu and world == 1:
        try:
            O, opop, grid, params, t_full, cores = cpu_baseline(bench_population(args, SEED))
            steps = max(1, int(args.cpu_budget / max(t_full, 1e-3)))
            t0 = time.perf_counter()
            for s in range(steps):
                O.propagate(opop, O.FULL, 10.0, 1, t0=10.0 * (s + 1))
                O.scan_cells(opop, params, grid, step=s + 1)
            el = time.perf_counter() - t0
            cpu = {"value": n * steps / el, "unit": "object-steps/s", "cores": cores, "kind": "port",
                   "sample": f"{steps} full steps of the 1e6-object workload (oracle, OpenMP {cores} threads)"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "error": str(ex)[:200]}

    # kernels per step from the profiled run, + one ephemeris kernel per 128-step chunk
    launches_per_step = sum(split["phases"]["launches"].values()) / split["phases"]["steps"]
    # the precision split changes the propagation only: the step-level ratio
    # cannot exceed the FP64 step over its non-propagation part
    fp64_per = {k: fp64_ph[k] / fp64_ph["steps"] for k in capi.PhaseTimes.PHASES}
    shared_ms = max(sum(fp64_per.values()) - fp64_per["propagate"], 1e-9)
    targets = {
        "mixed_over_fp64": value / fp64_value,
        "fp64_value": fp64_value,
        "propagate_fp64_over_split": fp64_per["propagate"] / max(per["propagate"], 1e-12),
        "mixed_over_fp64_bound_propagation_free": sum(fp64_per.values()) / shared_ms,
        "drift": {k: ({"steps": v["steps"], "rms_m": round(v["rms_m"], 5), "max_m": round(v["max_m"], 4),
                       "set": [v["differences"]["set_split"], v["differences"]["set_fp64"]],
                       "set_differences": v["differences"]["set_differences"],
                       "near_flagged": v["differences"]["near_flagged"],
                       "explained_by_drift": v["differences"]["explained_by_drift"]} if "error" not in v else v)
                  for k, v in drift.items()},
        "adjoint_over_forward": (adjoint or {}).get("backward_over_forward"),
        "adjoint_fd": (adjoint or {}).get("fd_summary"),
        "breakups_8e6": ({**{k: breakups[k] for k in ("iterations", "collisions", "breakups", "fragments",
                                                       "expected_collisions_from_conjunctions")},
                          "applied": {k: breakups["applied_run"][k] for k in ("iterations", "breakups", "fragments",
                                                                              "stopped_by")}}
                         if breakups and "error" not in breakups else breakups),
        "value_over_cpu_baseline": value / cpu["value"] if cpu and cpu.get("value") else None,
        "legs": "this run" if legs else "reported by the one-GPU run (replicas: timed steps and e2e only)",
    }
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "object-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": split["ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+f32 (split)",
        "data": "population file" if args.population else "synthetic (seeded population 0)",
        "config": bench_config(args, n),
        "precision": "split (FP64 central, J2, accumulation; FP32 J3, C22/S22, Sun, Moon, SRP, drag)",
        "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
        "l2": "inputs larger than L2: per-step working set ~450 MB (state 2 x 92 MB + keys + packed)",
        "kernels": kernels,
        "workloads": workloads,
        "adjoint": adjoint,
        "drift": drift,
        "breakups": breakups,
        "records": {"split": split["records"], "fp64": fp64["records"]},
        "wall_s": {"split": split["wall"], "fp64": fp64["wall"]},
        "e2e": e2e,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": split["clocks"],
        "gpu_launches": int(round(launches_per_step * args.steps)) + (args.steps + 127) // 128,
        "fp64": {"value": fp64_value, "ms_per_step": fp64["ms"] / args.steps},
        "targets": targets,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
