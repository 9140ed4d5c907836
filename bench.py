"""Throughput of the trace -> deposit -> merge -> update hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload lognormal128]
                    [--ticks T] [--impl ours|reference]

A step is one batch of T ticks of the workload: all rays of those ticks are
traced, sorted and deposited, and every particle they hit is updated once
per tick, as run_epoch() does (loop.c:128-147). The metric is ray-particle
hits per second (hits = stat.total_deposit_count, the summed hit-list
lengths), over the whole pipeline -- a stricter clock than the reference's
own hits/s, which counts only trace + deposit time.

Workloads (seeded synthetic fields; no dataset is involved; the default is
lognormal128, the 2M-particle case the hits/s target is stated at):
  iliev64       64^3 uniform particles in a 6.6 kpc box, one corner source of
                5e48 photons/s at 13.6 eV, 1024 rays/tick, isothermal 1e4 K
  iliev32       32^3, 32 rays/tick (the reference's CPU-sized case)
  lognormal128  128^3 particles on a log-normal field (sigma 1), 16 sources,
                8192 rays/tick, 8-bin 1e5 K blackbody, non-isothermal
  lognormal256  256^3 particles on a log-normal field (sigma 1.5), 256
                sources of 1e46-1e49 photons/s, 65536 rays/tick, one tick
                per step, non-isothermal; without the recombination and
                helium legs

--gpus N under torchrun runs N independent replicas, one per GPU (the path
is single-GPU; no data crosses GPUs), barrier + max over ranks for time.
The host-core baseline (cpu_baseline) is timed in one-GPU runs only.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DEFAULT_TICKS = {"iliev32": 400, "iliev64": 100, "lognormal128": 8, "lognormal256": 1}
REF_TICKS = {"iliev32": 40, "iliev64": 4, "lognormal128": 1, "lognormal256": 1}   # per step of --impl reference
SIDE_LEGS = ("iliev32", "iliev64", "lognormal128")
# Algorithmic bytes. Per hit (the whole path): pos 12 + sml 4 + lambdaH 8 +
# mass 4 + FP64 absorbed photons 8. Per kernel group, per unit it processes:
# trace fill reads pos+sml (16) and writes (ipar 4, d 8, b 8) per hit; the
# sort reads the slab (ipar, d, b: 20), writes the sorted lists (20) and
# gathers the smoothing length (16) for the kernel value; the slot
# order reads ipar twice (8), writes the hit into its run and reads and
# writes it once more in the run sort (12), plus the per-(tick, particle)
# counters and their scan (12 B per key, ~4 B per hit here): 24 B; deposit
# reads (ipar 4, kern 8) and the hit particle's lambdaH 8 and mass 4 and
# writes an FP64 deposit per hit (32 B), plus an FP64 heat when not
# isothermal (DEPOSIT_HEAT_BYTES); the update reads ~60 B and writes ~40 B
# of particle state per active (tick, particle) pair.
BYTES_PER_HIT = 36
GROUP_BYTES = {"trace_count": (16, "hit"), "trace_fill": (36, "hit"), "sort": (56, "hit"),
               "slots": (24, "hit"), "deposit": (32, "hit"), "update": (100, "active particle")}
DEPOSIT_HEAT_BYTES = 8


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampled every 100 ms on a reader thread; start() returns once
    the first sample has arrived so the samples cover the timed region."""

    def __init__(self, device: int):
        self.proc = None
        self.device = device
        self.lines = []
        self.t_start = None

    def start(self):
        import threading
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                self.lines.append((time.time(), line))
        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5:
            time.sleep(0.01)
        self.t_start = time.time()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t_end = time.time()
        time.sleep(0.15)
        self.proc.terminate()
        self.thread.join(timeout=5)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        window = [l for t, l in self.lines if self.t_start - 0.1 <= t <= t_end + 0.1] or [l for _, l in self.lines]
        for line in window:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make(workload: str):
    from psphray_b200 import fields
    return fields.make_workload(workload)


_REF = None


def cpu_baseline_reference(w, seconds: float = 15.0, threads: int | None = None, ticks=None):
    """The reference's own CPU code (oracle/_ref) on a bounded sample of the
    same workload: hits/s over its trace + deposit time, as its stat counters
    define it, with all host threads. Falls back to the C restatement."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    threads = threads or os.cpu_count()
    try:
        from refpy import LIB_PATH, Reference
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(LIB_PATH)
        from psphray_b200.api import RATES_HUI
        # The reference's non-isothermal solver raises SIGTRAP (solve.c:137-139)
        # wherever one step of cooling exceeds the internal energy, which the
        # dense cells of the log-normal field reach; its hits/s clock covers
        # trace + deposit only, which do not depend on the solver, so the
        # sample runs its isothermal solver.
        global _REF
        if _REF is None:       # the reference keeps its state in globals: one instance per process
            _REF = Reference(RATES_HUI, w.field.units, isothermal=True, threads=threads)
        ref = _REF
        ref.load(w.field)
        ref.build_tree(8)
        ref.reset_stats()
        t0 = time.time()
        n = 0
        while (time.time() - t0 < seconds and (ticks is None or n < ticks)) or n == 0:
            n += 1
            ref.tick(w.schedule.rays_for_tick(n), n, w.tick_time)
        st = ref.stats()
        hits_s = st["hits"] / (st["raytrace_time"] + st["deposit_time"])
        full = (st["raytrace_time"] + st["deposit_time"] + st["merge_time"] + st["update_time"])
        return {"value": hits_s, "unit": "hits/s", "cores": threads, "kind": "reference",
                "sample": f"{n} ticks x {w.schedule.nray} rays of {w.name}"
                          f"{'' if w.isothermal else ' (isothermal solver; see bench.py)'}, trace+deposit clock "
                          f"({st['hits']:.0f} hits); whole tick incl. LSODA update: "
                          f"{st['hits'] / full:.4g} hits/s, {full / n * 1e3:.3g} ms/tick"}
    except FileNotFoundError:
        from oracle import Oracle
        from psphray_b200 import api
        phys = api.Physics(w.field.units, isothermal=w.isothermal)
        orc = Oracle(w.field, phys, isothermal=w.isothermal)
        orc.build_tree(8)
        t0 = time.time()
        n = hits = 0
        while time.time() - t0 < seconds or n == 0:
            n += 1
            hits += orc.tick(w.schedule.rays_for_tick(n), n, w.tick_time)["hits"]
        dt = time.time() - t0
        return {"value": hits / dt, "unit": "hits/s", "cores": 1, "kind": "port",
                "sample": f"{n} ticks x {w.schedule.nray} rays of {w.name}, whole tick, 1 thread"}


def reduce_over_ranks(t_local: float, hits: float, dist, device):
    """Max of the ranks' times and sum of their hits (all ranks get both)."""
    import torch
    if dist is None:
        return t_local, hits
    t = torch.tensor([t_local], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    h = torch.tensor([hits], device=device, dtype=torch.float64)
    dist.all_reduce(h)
    return float(t.item()), float(h.item())


def dist_setup(gpus: int):
    if gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, 0, None
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ["RANK"]); world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    import torch
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return rank, world, local, dist


def run_reference(args):
    """--impl reference: the reference's own CPU code (oracle/_ref) on the
    same workload, all host threads, each step a bounded sample of ticks;
    hits/s on the reference's own clock (trace + deposit, stat.h:49-55)."""
    rank, world, local, dist = dist_setup(args.gpus)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refpy import LIB_PATH, Reference
    w = make(args.workload)
    if not os.path.exists(LIB_PATH):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpsphray_ref.so not built "
                          "(it is compiled from the reference sources by oracle/Makefile)"}), flush=True)
        return
    from psphray_b200.api import RATES_HUI
    threads = os.cpu_count()
    # isothermal solver: the reference's non-isothermal one traps on the
    # log-normal field (solve.c:137-139); the clock below excludes the solver
    ref = Reference(RATES_HUI, w.field.units, isothermal=True, threads=threads)
    ref.load(w.field)
    ref.build_tree(8)
    per = args.ref_ticks or REF_TICKS[args.workload]
    tick = 0
    hits = clock = 0.0
    for k in range(args.warmup + args.steps):
        ref.reset_stats()
        for _ in range(per):
            tick += 1
            ref.tick(w.schedule.rays_for_tick(tick), tick, w.tick_time)
        st = ref.stats()
        if k >= args.warmup:
            hits += st["hits"]
            clock += st["raytrace_time"] + st["deposit_time"]
    v = hits / clock
    base = {"value": v, "unit": "hits/s", "cores": threads, "kind": "reference",
            "sample": f"{args.steps} steps x {per} ticks x {w.schedule.nray} rays of {args.workload}, "
                      f"trace+deposit clock, {hits:.0f} hits"}
    line = {"impl": "reference", "metric": "ray-particle hits/s", "value": v, "unit": "hits/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": clock / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "ticks_per_step": per},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "hits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def surrogate_leg(ctx, w, R, T, ts, surr_path, dev, stream, nsurr=4, tol=1e-3):
    """The chemistry surrogate against the integrator: the same nsurr steps
    of T ticks from one state, plain and with the network (trained weights
    shipped in psphray_b200/data); GPU s per simulated Myr, the accepted
    fraction and the x_HII difference between the two."""
    import torch
    from psphray_b200.surrogate import Surrogate
    net = Surrogate.load(surr_path)
    for src in w.schedule.sources:          # one tick's photons at the first tick, as in a run
        src.lastemit = ts - 1
    s_rays = [torch.from_numpy(w.schedule.rays_for_ticks(ts + i * T, T).view(np.uint8)).to(f"cuda:{dev}")
              for i in range(nsurr)]
    st0 = ctx.state()
    keep = {k: st0[k] for k in ("lambdaH", "ie", "lasthit")}
    res = {}
    for mode in ("plain", "surrogate"):
        ctx.set_state(**keep)
        if mode == "surrogate":
            net.install(ctx, tol=tol)
        ms, acc, act = 0.0, 0.0, 0.0
        for i in range(nsurr):
            e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = ctx.run_ticks_device(s_rays[i].data_ptr(), R, T, ts + i * T, w.tick_time)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            acc += st["surrogate_accepted"]
            act += st["active"]
        res[mode] = (ms, acc / max(act, 1.0), 1.0 - ctx.lambdaH())
        if mode == "surrogate":
            Surrogate.uninstall(ctx)
    myr = nsurr * T * w.tick_time / w.field.units.MYR
    xp, xs = res["plain"][2], res["surrogate"][2]
    rel = np.abs(xs - xp) / np.maximum(xp, 1e-6)
    return {"tol": tol, "steps": nsurr, "ticks_per_step": T, "weights": os.path.basename(surr_path),
            "gpu_s_per_sim_myr_plain": res["plain"][0] / 1e3 / myr,
            "gpu_s_per_sim_myr_surrogate": res["surrogate"][0] / 1e3 / myr,
            "accepted_fraction": res["surrogate"][1],
            "x_HII_rel_diff": {"p50": float(np.median(rel)), "p99": float(np.percentile(rel, 99)),
                               "max": float(rel.max())}}


def timed_steps(ctx, rays_dev, R, T, t_first, tick_time, stream, nsteps):
    """nsteps batches of T ticks timed with CUDA events: (ms, hits, syncs)."""
    import torch
    ms = hits = syncs = 0.0
    for s in range(nsteps):
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = ctx.run_ticks_device(rays_dev[s].data_ptr(), R, T, t_first + s * T, tick_time)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        hits += st["hits"]
        syncs += st["host_syncs"]
    return ms, hits, syncs


def default_physics_leg(w, dev, stream, dev_rays, R, T, nrs):
    """The reference's default physics together (config.c:25,28,31: helium,
    secondary ionisation, recombination rays, not isothermal) on the same
    particles (hydrogen mass fraction 0.76) and rays: hits/s."""
    from psphray_b200 import api
    from psphray_b200.units import Units
    hu = Units(hmf=0.76)
    hf = dataclasses.replace(w.field, units=hu)
    c = api.Context(dev)
    c.set_stream(stream.cuda_stream)
    c.set_physics(api.Physics(hu, isothermal=w.isothermal, h_only=False, secondary_ionization=True,
                              on_the_spot=False))
    c.load(hf)
    c.build_tree(8)
    c.set_recombination(nrec=100)
    for s in range(2):      # (sizing the buffers, then capturing the tick graph)
        c.run_ticks_device(dev_rays[s].data_ptr(), R, T, 1 + s * T, w.tick_time)
    ms, hits, syncs = timed_steps(c, dev_rays[2:], R, T, 1 + 2 * T, w.tick_time, stream, nrs)
    c.close()
    return {"value": hits / (ms / 1e3), "unit": "hits/s", "ms_per_tick": ms / (nrs * T), "hmf": 0.76,
            "secondary_ionization": True, "on_the_spot": False, "nrec_per_species": 100, "steps": nrs,
            "ticks_per_step": T, "host_syncs_per_step": syncs / nrs}


def full_pipeline_leg(dev, stream, cpu: bool):
    """The full pipeline's field (256^3 = 16.8M particles, sigma 1.5, 256
    sources, 65536 rays per tick, not isothermal), one tick per step: hits/s
    and GPU s per simulated Myr, plain and with the surrogate, and the
    reference's own CPU code on a bounded sample of the same ticks."""
    import torch
    from psphray_b200 import api
    w = make("lognormal256")
    R, T = w.schedule.nray, 1
    c = api.Context(dev)
    c.set_stream(stream.cuda_stream)
    c.set_physics(api.Physics(w.field.units, isothermal=w.isothermal))
    c.load(w.field)
    c.build_tree(8)
    nst = 4
    rays = [torch.from_numpy(w.schedule.rays_for_ticks(1 + s, 1).view(np.uint8)).to(f"cuda:{dev}")
            for s in range(nst + 2)]
    for s in range(2):
        c.run_ticks_device(rays[s].data_ptr(), R, T, 1 + s, w.tick_time)
    ms, hits, syncs = timed_steps(c, rays[2:], R, T, 3, w.tick_time, stream, nst)
    value = hits / (ms / 1e3)
    myr = nst * T * w.tick_time / w.field.units.MYR
    out = {"workload": "lognormal256", "particles": w.field.n, "rays_per_tick": R, "value": value,
           "unit": "hits/s", "ms_per_tick": ms / nst, "gpu_s_per_sim_myr": ms / 1e3 / myr,
           "host_syncs_per_step": syncs / nst}
    surr_path = os.path.join(ROOT, "psphray_b200", "data", "surrogate_lognormal128.npz")
    if os.path.exists(surr_path):
        out["surrogate"] = surrogate_leg(c, w, R, T, 3 + nst, surr_path, dev, stream, nsurr=3)
    c.close()
    del rays
    torch.cuda.empty_cache()
    if cpu:
        base = cpu_baseline_reference(make("lognormal256"), seconds=10.0, ticks=1)
        out["cpu_baseline"] = base
        out["vs_cpu"] = value / base["value"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="lognormal128")
    ap.add_argument("--ticks", type=int, default=0, help="ticks per step (default per workload)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-ticks", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default launch shapes")
    ap.add_argument("--no-full-pipeline", action="store_true", help="skip the 16.8M-particle leg")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    dev = local
    torch.cuda.set_device(dev)
    from psphray_b200 import api
    from psphray_b200.fields import RAY_DTYPE

    w = make(args.workload)
    T = args.ticks or DEFAULT_TICKS[args.workload]
    R = w.schedule.nray
    nsteps = args.warmup + args.steps
    phys = api.Physics(w.field.units, isothermal=w.isothermal)
    ctx = api.Context(dev)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_physics(phys)
    ctx.load(w.field)
    ctx.build_tree(8)
    tinfo = ctx.tree_info()

    # rays of every step, resident in HBM before timing (inputs of `value`)
    host_rays = [w.schedule.rays_for_ticks(1 + s * T, T) for s in range(nsteps)]
    dev_rays = [torch.from_numpy(r.view(np.uint8)).to(f"cuda:{dev}") for r in host_rays]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")   # > 126 MB L2
    torch.cuda.synchronize(dev)

    # launch shapes chosen by the library's autotuner on the first step's
    # rays (every trial restores the particle state), before the warm-up
    tune, tune_ms = (ctx.autotune(dev_rays[0].data_ptr(), R, T, 1, w.tick_time, reps=2)
                     if not args.no_autotune else (ctx.tune(), None))
    for s in range(args.warmup):
        ctx.run_ticks_device(dev_rays[s].data_ptr(), R, T, 1 + s * T, w.tick_time)
    torch.cuda.synchronize(dev)

    clocks = Clocks(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    torch.cuda.nvtx.range_push("timed_steps")      # lets a profiler capture exactly these launches
    total_ms, hits, launches, sat, active, syncs = 0.0, 0.0, 0.0, 0.0, 0.0, 0.0
    per_step = []
    kms = {k: 0.0 for k in api.KERNELS}
    kn = {k: 0.0 for k in api.KERNELS}
    for s in range(args.warmup, nsteps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = ctx.run_ticks_device(dev_rays[s].data_ptr(), R, T, 1 + s * T, w.tick_time)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        hits += st["hits"]
        sat += st["saturated"]
        active += st["active"]
        per_step.append(round(e0.elapsed_time(e1), 3))
        launches += st["launches"]
        syncs += st["host_syncs"]
    torch.cuda.synchronize(dev)
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    t_max, hits_all = reduce_over_ranks(total_ms / 1e3, hits, dist, torch.device("cuda", dev))
    value = hits_all / t_max
    sim_myr = args.steps * T * w.tick_time / w.field.units.MYR

    # e2e: the public host-buffer call, pinned host rays, result read back;
    # one untimed step first (it sizes the library's host-call buffers)
    pinned = [torch.from_numpy(r.view(np.uint8)).pin_memory() for r in host_rays[args.warmup - 1:]]
    e2e_hits = 0.0
    lam_pinned = torch.empty(w.field.n, dtype=torch.float64).pin_memory()   # the result read back each step
    lam = lam_pinned.numpy()
    ctx.run_ticks(np.frombuffer(pinned[0].numpy(), dtype=RAY_DTYPE), R, T, 1 + nsteps * T, w.tick_time)
    ctx.lambdaH(out=lam)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i, pr in enumerate(pinned[1:]):
        rays = np.frombuffer(pr.numpy(), dtype=RAY_DTYPE)
        st = ctx.run_ticks(rays, R, T, 1 + (nsteps + 1 + i) * T, w.tick_time)
        ctx.lambdaH(out=lam)
        e2e_hits += st["hits"]
    torch.cuda.synchronize(dev)
    e2e_t, e2e_hits = reduce_over_ranks(time.perf_counter() - t0, e2e_hits, dist, torch.device("cuda", dev))

    # the same through psg_run_ticks_emit: rays emitted on the device from the
    # workload's sources (no rays cross the bus), state read back every step
    sch = w.schedule
    t1 = 1 + 2 * nsteps * T
    srcs = [dataclasses.replace(src, lastemit=t1 - 1) for src in sch.sources]   # one tick's photons at t1
    ctx.set_sources(srcs, [(sch.energies, sch.eweights)], seed=sch.seed)
    ctx.run_ticks_emit(R, T, t1, w.tick_time)
    em_hits = 0.0
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in range(args.steps):
        st = ctx.run_ticks_emit(R, T, t1 + (i + 1) * T, w.tick_time)
        ctx.lambdaH(out=lam)
        em_hits += st["hits"]
    torch.cuda.synchronize(dev)
    em_t, em_hits = reduce_over_ranks(time.perf_counter() - t0, em_hits, dist, torch.device("cuda", dev))

    # chemistry surrogate (not isothermal): the same steps from one state,
    # on the integrator and with the network (trained weights shipped in
    # psphray_b200/data), GPU s per simulated Myr and the x_HII difference
    surrogate = None
    surr_path = os.path.join(ROOT, "psphray_b200", "data", "surrogate_lognormal128.npz")
    if not w.isothermal and os.path.exists(surr_path):
        ts = t1 + (args.steps + 2) * T
        surrogate = surrogate_leg(ctx, w, R, T, ts, surr_path, dev, stream)
    # the side legs (recombination rays, helium) load further contexts of the
    # same field; the 16.8 M-particle field is measured without them
    recombination = helium = None
    if args.workload in SIDE_LEGS:
        # recombination rays (onTheSpot = false): the same rays on a context
        # with case-A recombination, nrec = 100 recombination rays per tick
        # emitted on the device; the ticks then run one at a time
        rctx = api.Context(dev)
        rctx.set_stream(stream.cuda_stream)
        rctx.set_physics(api.Physics(w.field.units, isothermal=w.isothermal, on_the_spot=False))
        rctx.load(w.field)
        rctx.build_tree(8)
        rctx.set_recombination(nrec=100)
        # two untimed calls: the first runs its ticks one by one and sizes
        # the buffers, the second captures the tick graph that later calls
        # replay
        nrs = min(3, nsteps - 2)
        for s in range(2):
            rctx.run_ticks_device(dev_rays[s].data_ptr(), R, T, 1 + s * T, w.tick_time)
        r_ms, r_hits, r_rays, r_syncs = 0.0, 0.0, 0.0, 0.0
        torch.cuda.nvtx.range_push("recombination_steps")
        for s in range(2, 2 + nrs):
            e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = rctx.run_ticks_device(dev_rays[s].data_ptr(), R, T, 1 + s * T, w.tick_time)
            e1.record(stream)
            e1.synchronize()
            r_ms += e0.elapsed_time(e1)
            r_hits += st["hits"]
            r_rays += st["rec_rays"]
            r_syncs += st["host_syncs"]
        torch.cuda.nvtx.range_pop()
        rctx.close()
        recombination = {"value": r_hits / (r_ms / 1e3), "unit": "hits/s", "ms_per_tick": r_ms / (nrs * T),
                         "rec_rays_per_tick": r_rays / (nrs * T), "steps": nrs, "ticks_per_step": T,
                         "host_syncs_per_step": r_syncs / nrs}

        # helium and secondary ionisation (HOnly = false, hydrogen mass fraction
        # 0.76): the same particles and rays, three-species deposit with the
        # secondary-ionisation table and the helium update, on the spot
        from psphray_b200.units import Units
        hu = Units(hmf=0.76)
        hf = dataclasses.replace(w.field, units=hu)
        hctx = api.Context(dev)
        hctx.set_stream(stream.cuda_stream)
        hctx.set_physics(api.Physics(hu, isothermal=w.isothermal, h_only=False, secondary_ionization=True))
        hctx.load(hf)
        hctx.build_tree(8)
        hctx.run_ticks_device(dev_rays[0].data_ptr(), R, T, 1, w.tick_time)
        h_ms, h_hits = 0.0, 0.0
        torch.cuda.nvtx.range_push("helium_steps")
        for s in range(1, 1 + nrs):
            e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = hctx.run_ticks_device(dev_rays[s].data_ptr(), R, T, 1 + s * T, w.tick_time)
            e1.record(stream)
            e1.synchronize()
            h_ms += e0.elapsed_time(e1)
            h_hits += st["hits"]
        torch.cuda.nvtx.range_pop()
        hctx.close()
        helium = {"value": h_hits / (h_ms / 1e3), "unit": "hits/s", "ms_per_tick": h_ms / (nrs * T),
                  "hmf": 0.76, "secondary_ionization": True, "steps": nrs, "ticks_per_step": T}

    # the reference's default physics together, and the full pipeline's
    # field (one-GPU runs on the default workload: they add a few minutes)
    default_physics = full_pipeline = None
    if args.workload in SIDE_LEGS:
        default_physics = default_physics_leg(w, dev, stream, dev_rays, R, T, min(3, nsteps - 2))
    if args.workload == "lognormal128" and world == 1 and not args.no_full_pipeline:
        full_pipeline = full_pipeline_leg(dev, stream, cpu=rank == 0 and not args.no_cpu_baseline)

    # the per-kernel-group breakdown: the same steps again (later ticks) with
    # the library's per-launch events on -- kept out of the timed steps,
    # whose launches they would slow
    ctx.set_timing(True)
    tp = t1 + (args.steps + 8) * T
    for i, s in enumerate(range(args.warmup, nsteps)):
        flush.zero_()
        st = ctx.run_ticks_device(dev_rays[s].data_ptr(), R, T, tp + i * T, w.tick_time)
        for k in api.KERNELS:
            kms[k] += st["kernel_ms"][k]
            kn[k] += st["kernel_launches"][k]
    torch.cuda.synchronize(dev)
    ctx.set_timing(False)

    # roofline of the dominant kernel group
    peak, peak_kind = peaks()
    dom = max(api.KERNELS, key=lambda k: kms[k])
    unit_bytes, unit_name = GROUP_BYTES[dom]
    if dom == "deposit" and not w.isothermal:
        unit_bytes += DEPOSIT_HEAT_BYTES
    units = active if unit_name == "active particle" else hits
    achieved = units * unit_bytes / (kms[dom] / 1e3) / 1e9 if kms[dom] > 0 else None
    path_gbs = value / world * BYTES_PER_HIT / 1e9    # per GPU, over the whole step
    # groups launched once per tick (deposit, update) vs once per step
    per_tick = dom in ("deposit", "update")
    alg_per_launch = units * unit_bytes / (args.steps * (T if per_tick else 1))
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"{dom}_{args.workload}_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            traffic = json.load(f).get("bytes_per_launch")

    line = {"metric": "ray-particle hits/s", "value": value, "unit": "hits/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "particles": w.field.n, "rays_per_tick": R,
                       "ticks_per_step": T, "hits_per_step": hits / args.steps,
                       "tree_cells": tinfo["ncells"], "l2": "256 MiB buffer zeroed between steps",
                       "parallelism": f"replicas{world}"},
            "gpu_s_per_sim_myr": t_max / sim_myr,
            "gpu_launches": launches,
            "host_syncs_per_step": syncs / args.steps,
            "tune": dict(tune, batch_ms=tune_ms),
            "saturated_deposits_per_step": sat / args.steps,
            "step_ms": per_step,
            "kernel_ms_per_step": {k: kms[k] / args.steps for k in api.KERNELS},
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "peak_source": peak_kind,
                         "bytes_per_unit": unit_bytes, "unit_counted": unit_name,
                         "launch": "one tick" if per_tick else "one step",
                         "algorithmic_bytes_per_launch": alg_per_launch,
                         "units_per_step": units / args.steps,
                         "path_achieved_gbs": path_gbs,
                         "path_frac": path_gbs / peak},
            "clocks": clk,
            "surrogate": surrogate,
            "recombination": recombination,
            "helium": helium,
            "default_physics": default_physics,
            "full_pipeline": full_pipeline,
            "e2e_device_emission": {"value": em_hits / em_t, "unit": "hits/s", "h2d_bytes_per_step": 0,
                                    "d2h_bytes_per_step": int(lam.nbytes)},
            "e2e": {"value": e2e_hits / e2e_t, "unit": "hits/s",
                    "h2d_bytes_per_step": int(host_rays[0].nbytes),
                    "d2h_bytes_per_step": int(lam.nbytes)}}
    # the host-core baseline: rank 0 of a one-GPU run only (with more ranks,
    # their host threads would share the cores it is timed on)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_reference(make(args.workload), seconds=args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
