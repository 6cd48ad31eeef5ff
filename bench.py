#!/usr/bin/env python
"""Benchmark of the velocity-and-timestep path on B200.

Workload (one "step"): the reference's time-loop body (src/run.f90:41-93)
with its default options -- ghost gather, octree build, Biot-Savart velocity
(LIA + Barnes-Hut walk with 26 periodic images; FP32 pair terms with FP64
recentring and compensated sums), Adams-Bashforth update, pinsert, the
reconnection candidate search on the tree built before the move, precon
(original), premove, ghost gather and periodic wrap -- on the large isotropic
tangle: 3000 rings, R ~ U(0.004, 0.015) cm, delta 3e-4 cm (N = 802,906
points), periodic box 0.1 cm, theta 0.5, dt 1e-7 s.  This is the largest
configuration of the path that runs on one GPU.  Inputs are seeded synthetic
rings (no dataset).

Metric: direct-equivalent Biot-Savart pair interactions per second,
N * N_active * 27 per step / step time (the unit the O(N^2) direct form would
have to evaluate), whole job over all ranks.  Every rank runs an independent
replica (the path does not shard; "replicas only").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--suite large|tangle|batch|gradient|ring|direct] [--quick]

Under torchrun each rank drives cuda:LOCAL_RANK; the timed region is bracketed
by a barrier and a synchronize, and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "BS direct-equivalent pair-interactions/s (mixed BH velocity+step)"
UNIT = "pairs/s"
FLOP_LEAF = 38.0   # algorithmic FP32 FLOP of one straight-segment pair term
FLOP_FAR = 50.0    # algorithmic FP32 FLOP of one monopole+dipole cell term
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--suite", default="large",
                    choices=["large", "tangle", "batch", "gradient", "ring", "direct"],
                    help="large: the headline line; the others print only that workload's "
                         "entry")
    ap.add_argument("--batch-config", default=None,
                    help="--suite batch: warps_per_block,blocks_per_sm,order instead of the tuner")
    ap.add_argument("--quick", action="store_true",
                    help="headline timing only (no comparators, e2e or CPU baseline)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi clock/throttle sampler.  It is started before the warm-up
    (its start-up must not land in the timed region) and only the samples
    stamped inside the timed window are kept."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self, t0: float, t1: float) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait(timeout=5)
        self.f.flush()
        import datetime as _dt

        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            r = [x.strip() for x in line.split(",")]
            try:
                ts = _dt.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except (ValueError, IndexError):
                continue
            rows.append((ts, r))
        inside = [r for ts, r in rows if t0 - 0.25 <= ts <= t1 + 0.25]
        if not inside:  # window shorter than the sampling period: nearest samples
            inside = [r for ts, r in sorted(rows, key=lambda z: abs(z[0] - (t0 + t1) / 2))[:2]]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in inside:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def job_time_ms(ms_local: float, ws: int, device="cuda") -> float:
    """The job's time for the timed region: the maximum over ranks of each
    rank's device-timed milliseconds (every rank calls this, in the same order)."""
    if ws <= 1:
        return ms_local
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(units_per_step: float, ms_per_step: float, ws: int) -> float:
    """Whole-job throughput: every rank runs an independent replica of the
    step, so the job processes ws times the units of one replica."""
    return ws * units_per_step / (ms_per_step * 1e-3)


def workload(seed: int):
    from qvort_b200 import workloads as W

    return W.large_tangle(seed)


def workload_config(w, ws: int = 1) -> dict:
    """The `config` object of the JSON line, identical in both arms."""
    return {
        "workload": (f"large tangle: 3000 rings R~U(0.004,0.015) cm, delta 3e-4 cm, "
                     f"N={w.n}, periodic L=0.1 cm (26 images), Barnes-Hut theta 0.5, AB ladder, "
                     f"dt 1e-7 s, default loop (pinsert, pclose_tree, precon, premove "
                     f"every step)"),
        "n_points": w.n,
        "l2": "inputs (tree packs ~0.2 GB) larger than L2, and L2 flushed between timed steps",
        "parallelism": f"replicas x{ws} (the path does not shard)",
    }


# ----------------------------------------------------------------------- CPU
def cpu_step_rate(w, seconds_budget: float = 12.0, nthreads: int | None = None):
    """Oracle (the C restatement, OpenMP over targets) on the host cores: one
    step of the same loop on a bounded sample -- ghost gathers, tree build, AB
    update, candidate search and the sequential line operations (pinsert,
    precon, premove) on every point; the velocity on an evenly strided subset
    of targets sized to `seconds_budget`, scaled to all targets.  Returns
    (step seconds, sample text, threads used)."""
    from oracle import oracle as O

    nthreads = nthreads or os.cpu_count() or 1
    p = O.params(**w.params)
    x, inf, beh = w.x.copy(), w.infront, w.behind
    t0 = time.perf_counter()
    g = O.ghosts(p, x, inf, beh)
    t_g = time.perf_counter() - t0
    t0 = time.perf_counter()
    tree = O.Tree(p, x, g[0], inf)
    t_b = time.perf_counter() - t0
    # probe the per-target cost on a small stride, then size the sample
    probe = np.arange(0, w.n, max(1, w.n // 256), dtype=np.int32)
    t0 = time.perf_counter()
    O.velocity(p, x, inf, beh, g, tree, targets=probe, nthreads=nthreads)
    per = (time.perf_counter() - t0) / len(probe)
    m = int(min(w.n, max(len(probe), seconds_budget / max(per, 1e-9))))
    tg = np.linspace(0, w.n - 1, m).astype(np.int32)
    t0 = time.perf_counter()
    u, *_ = O.velocity(p, x, inf, beh, g, tree, targets=tg, nthreads=nthreads)
    t_v = (time.perf_counter() - t0) * w.n / m
    uf = np.zeros_like(x)
    uf[tg] = u
    h = [np.zeros_like(x) for _ in range(3)]
    t0 = time.perf_counter()
    xn, *_ = O.pmotion_ab(p.dt, x, uf, *h, inf)
    t_ab = time.perf_counter() - t0
    st = O.line_state(w.n, 2 * w.n, x=xn, u=uf, infront=inf, behind=beh, gi=g[0], gb=g[1],
                      gii=g[2], gbb=g[3])
    t0 = time.perf_counter()
    n2, _ = O.pinsert(p, w.n, st)
    t_l = time.perf_counter() - t0
    t0 = time.perf_counter()
    cl, cd = O.pclose_tree(tree, st["x"][:n2], st["infront"][:n2], st["behind"][:n2],
                           np.zeros(n2, np.int32), nthreads)
    t_c = time.perf_counter() - t0
    st["closest"][:n2], st["closestd"][:n2] = cl, cd
    t0 = time.perf_counter()
    O.precon(p, n2, st)
    O.premove(p, n2, st)
    t_l += time.perf_counter() - t0
    tree.close()
    t_step = t_g * 2 + t_b + t_v + t_ab + t_c + t_l
    sample = (f"1 step of the same loop: ghosts, tree build, AB, pinsert, candidate search, "
              f"precon, premove on all {w.n} points; velocity on {m} evenly strided "
              f"targets, scaled by {w.n}/{m}")
    return t_step, sample, nthreads


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    w = workload(args.seed)
    pairs = float(w.n) * w.n * 27
    for _ in range(args.warmup):
        cpu_step_rate(w, seconds_budget=0.5)
    ts = []
    t_wall = time.perf_counter()
    sample, cores = "", 0
    for _ in range(args.steps):
        t, sample, cores = cpu_step_rate(w, seconds_budget=1.5)
        ts.append(t)
    wall = time.perf_counter() - t_wall
    t = float(np.mean(ts))
    v = pairs / t
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random rings)",
        "config": workload_config(w, args.gpus),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample,
                         "note": "no Fortran compiler on this image: the reference's own "
                                 "Fortran/OpenMP path cannot be built; this is the C "
                                 "restatement of it (oracle/qv_oracle.c)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------- GPU
def time_steps(ctx, stream, torch, itime: int, steps: int, flush=None):
    """CUDA-event time of `steps` calls of qv_step on `stream` (the context's
    stream), L2 flushed before each outside the events; returns (ms per step,
    next itime)."""
    evs = []
    for k in range(steps):
        with torch.cuda.stream(stream):
            if flush is not None:
                flush.fill_(k & 0xFF)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            itime += 1
            ctx.step(itime)
            e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs) / steps, itime


def our_arm(args):
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from qvort_b200 import lib as L

    w = workload(args.seed)
    n = w.n
    pairs_step = float(n) * n * 27
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    # reconnections on (line_ops 2): pinsert, candidate search, precon, premove
    ctx = L.Context(L.default_params(**w.params, precision="mixed", line_ops=2), stream=sp)
    ctx.set_points(w.x, w.infront, w.behind)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    clocks = Clocks(local)
    clocks.start()
    itime = 0
    for _ in range(max(3, args.warmup)):
        itime += 1
        ctx.step(itime)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    launches0 = ctx.counters()["launches"]
    torch.cuda.synchronize()
    t_wall0 = time.time()
    ms_local, itime = time_steps(ctx, stream, torch, itime, args.steps, flush)
    clk = clocks.stop(t_wall0, time.time())
    launches = ctx.counters()["launches"] - launches0
    ms_step = job_time_ms(ms_local, ws)
    if ws > 1:
        torch.distributed.barrier()
    value = job_value(pairs_step, ms_step, ws)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair terms, f64 recentring/LIA/AB/tree/search",
        "data": "synthetic (seeded random rings)",
        "config": workload_config(w, ws),
        "n_points_end": ctx.n,
        "steps_per_s": 1e3 / ms_step * ws,
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    if not args.quick and rank == 0:
        line.update(extras(ctx, w, stream, L, torch, itime, flush))
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def _rel(a, b):
    return (float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())),
            float((np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)).max()))


def walk_roofline(ctx, L, stream, nprof: int = 3, traffic_file: str = "walk_large_traffic.json"):
    """Phase times over nprof profiled steps and the roofline of the dominant
    kernel, the mixed Barnes-Hut walk: algorithmic FLOPs counted on the device
    (38 per leaf pair, 50 per far cell) over the CUDA-event time of its launch
    (the walk_kernel phase; the non-local phase adds the fix-ups and the
    reduction of the per-image partial sums)."""
    itime = 10_000
    ctx.profile(True)
    ctx.step(itime)          # the first profiled step creates the events; not counted
    ctx.phase_times(reset=True)
    for _ in range(nprof):
        itime += 1
        ctx.step(itime)
    ph = ctx.phase_times(reset=True)
    ctx.profile(False)
    cnt = ctx.counters()
    walk_ms = ph["walk_kernel"] / nprof
    flops = cnt["leaf_evals"] * FLOP_LEAF + cnt["far_evals"] * FLOP_FAR
    peak = L.probe_fp32(stream.cuda_stream)
    achieved = flops / (walk_ms * 1e-3) / 1e12
    traffic, traffic_src = None, None
    prof = ROOT / "profiles" / traffic_file
    if prof.exists():
        d = json.loads(prof.read_text())
        traffic, traffic_src = d.get("bytes_per_launch"), d.get("source")
    roof = {
        "kernel": "k_walk32 (Barnes-Hut walk, mixed)", "bound": "fp32",
        "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
        "traffic": traffic,
        "traffic_source": traffic_src or "no capture committed",
        "peak_source": "measured FP32 FMA throughput on this GPU (qv_probe_fp32); "
                       "MEASURED_PEAKS.json has no FP32-pipe figure",
        "flop_model": f"{FLOP_LEAF:.0f} FLOP/leaf pair + {FLOP_FAR:.0f} FLOP/far cell "
                      "(algorithmic; theta tests, recentring and Kahan excluded)",
        "leaf_evals": cnt["leaf_evals"], "far_evals": cnt["far_evals"], "walk_ms": walk_ms,
        "walk_phase_ms": ph["nonlocal"] / nprof,
        "timing": "CUDA events around the walk kernel's launch on the context's stream",
    }
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    if traffic and peaks_file.exists():
        hbm = json.loads(peaks_file.read_text()).get("hbm_gbs")
        if hbm:
            gbs = traffic / (walk_ms * 1e-3) / 1e9
            roof["hbm"] = {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                           "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)"}
    return {k: v / nprof for k, v in ph.items()}, roof


def precision_pair(L, torch, w, stream, flush, steps: int = 3, warmup: int = 2):
    """The same workload in FP64 (the reference's arithmetic, same Barnes-Hut
    algorithm): CUDA-event step time, and the mixed velocity's error against the
    FP64 velocity on every target of the initial state."""
    sp = stream.cuda_stream
    vel = {}
    out = {}
    for prec in ("mixed", "fp64"):
        c = L.Context(L.default_params(**dict(w.params, precision=prec, line_ops=2)), stream=sp)
        c.set_points(w.x, w.infront, w.behind)
        vel[prec] = c.velocity(False)[0]
        if prec == "fp64":
            it = 0
            for _ in range(warmup):
                it += 1
                c.step(it)
            torch.cuda.synchronize()
            ms, _ = time_steps(c, stream, torch, it, steps, flush)
            out["fp64_bh"] = {"ms_per_step": ms, "pairs_per_s": float(w.n) * w.n * 27 / (ms * 1e-3),
                              "steps": steps, "timing": "CUDA events, L2 flushed between steps"}
        c.close()
    rms, mx = _rel(vel["mixed"], vel["fp64"])
    out["error"] = {"mixed_vs_fp64_bh_rms_rel": rms, "mixed_vs_fp64_bh_max_rel": mx,
                    "targets": w.n, "state": "initial"}
    return out


def e2e_rate(L, torch, w, stream, steps: int = 10):
    """The same step end to end through the C ABI with pinned host buffers
    (the Fortran shim's per-step pattern: gather f(:) in, step, scatter f(:)
    out in one qv_step_exchange call); wall clock around the calls."""
    n = w.n
    pairs_step = float(n) * n * 27
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
    cap = n + n // 4  # room for insertions (the host grows f(:) when pcount grows)
    hx = pin((cap, 3), torch.float64); hx[:n] = w.x
    hinf = pin((cap,), torch.int32); hinf[:n] = w.infront
    hbeh = pin((cap,), torch.int32); hbeh[:n] = w.behind
    hist = [pin((cap, 3), torch.float64) for _ in range(3)]
    for h in hist:
        h[:] = 0
    hcl = pin((cap,), torch.int32); hcl[:] = 0
    hu = pin((cap, 3), torch.float64)
    hcd = pin((cap,), torch.float64)
    c = L.Context(L.default_params(**w.params, precision="mixed", line_ops=2),
                  stream=stream.cuda_stream)
    cur = [n]
    moved = [0, 0]
    inp = dict(x=hx, infront=hinf, behind=hbeh, u1=hist[0], u2=hist[1], u3=hist[2], closest=hcl)
    outp = dict(x=hx, u=hu, u1=hist[0], u2=hist[1], u3=hist[2], infront=hinf, behind=hbeh,
                closest=hcl, closestd=hcd)

    def e2e_step(it):
        n_in = cur[0]
        m = cur[0] = c.step_exchange(it, n_in, cap, inp, outp)
        moved[0] += n_in * (24 + 8 + 72 + 4)      # x, links, history, closest in
        moved[1] += m * (24 + 24 + 72 + 4 + 8 + 8)  # x, u, history, closest(d), links out

    for it in range(3):
        e2e_step(it + 1)
    torch.cuda.synchronize()
    moved[0] = moved[1] = 0
    t0 = time.perf_counter()
    for it in range(steps):
        e2e_step(it + 4)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / steps
    c.close()
    return {"value": pairs_step / (ms * 1e-3), "unit": UNIT,
            "h2d_bytes_per_step": moved[0] // steps, "d2h_bytes_per_step": moved[1] // steps,
            "ms_per_step": ms,
            "path": "qv_step_exchange (line_ops 2): pinned host in x, links, AB history, "
                    "closest; out x, u, history, links, closest, closestd; wall clock"}


def extras(ctx, w, stream, L, torch, itime, flush):
    out = {}
    n = w.n
    pairs_step = float(n) * n * 27
    # ---- phase breakdown and the dominant kernel (the tree walk)
    ph, roof = walk_roofline(ctx, L, stream)
    out["phases_ms_per_step"] = ph
    out["roofline"] = roof
    out["evals_per_step"] = roof["leaf_evals"] + roof["far_evals"] + 2 * n
    # ---- mixed against FP64 on the same algorithm: time and error
    pp = precision_pair(L, torch, w, stream, flush)
    out["fp64_bh"] = pp["fp64_bh"]
    out["error"] = pp["error"]
    # ---- end to end through the C ABI with pinned host buffers
    out["e2e"] = e2e_rate(L, torch, w, stream)
    # ---- the random-ring tangle (N = 24.7k): mixed and FP64 Barnes-Hut steps,
    # the FP64 direct form (the >= 5x comparison), errors
    out["tangle"] = tangle_rate(L, torch, stream, flush)
    # ---- gradients/s on the differentiation workload
    out["gradient"] = gradient_rate(L, torch)
    # ---- batched ensemble: 512 independent open systems in one graph per step
    out["batch"] = batch_rate(L, torch)
    # ---- CPU baseline (oracle port on this host's cores), bounded sample
    t, sample, cores = cpu_step_rate(w)
    out["cpu_baseline"] = {"value": pairs_step / t, "unit": UNIT, "cores": cores, "kind": "port",
                           "sample": sample, "ms_per_step": t * 1e3}
    return out


def tangle_rate(L, torch, stream, flush, steps: int = 10, warmup: int = 3) -> dict:
    """The random-ring tangle: 100 rings, R ~ U(0.008, 0.02) cm, delta 5e-4 cm
    (N = 24,707), periodic L = 0.1, theta 0.4, the default loop.  Mixed and FP64
    Barnes-Hut steps and the FP64 direct form's step, CUDA events; errors of
    the mixed velocity against FP64 Barnes-Hut and of FP64 Barnes-Hut against
    the FP64 direct sum at the initial state."""
    from qvort_b200 import workloads as W

    w = W.tangle(0)
    n = w.n
    pairs_step = float(n) * n * 27
    sp = stream.cuda_stream
    out = {"workload": f"tangle: 100 rings R~U(0.008,0.02) cm, delta 5e-4 cm, N={n}, periodic "
                       f"L=0.1, theta 0.4, default loop", "n_points": n}
    vel = {}
    for key, prm, k in (("mixed", dict(precision="mixed"), steps),
                        ("fp64_bh", dict(precision="fp64"), steps),
                        ("fp64_direct", dict(precision="fp64", velocity="BS", tree_theta=0.0), 2)):
        pr = dict(w.params, line_ops=2)
        pr.update(prm)
        c = L.Context(L.default_params(**pr), stream=sp)
        c.set_points(w.x, w.infront, w.behind)
        vel[key] = c.velocity(False)[0]
        it = 0
        for _ in range(warmup if k > 2 else 1):
            it += 1
            c.step(it)
        torch.cuda.synchronize()
        ms, _ = time_steps(c, stream, torch, it, k, flush)
        out[key] = {"ms_per_step": ms, "pairs_per_s": pairs_step / (ms * 1e-3)}
        c.close()
    out["mixed_speedup_vs_fp64_bh"] = out["fp64_bh"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["mixed_speedup_vs_fp64_direct"] = (out["fp64_direct"]["ms_per_step"] /
                                           out["mixed"]["ms_per_step"])
    rms, mx = _rel(vel["mixed"], vel["fp64_bh"])
    rms_a, mx_a = _rel(vel["fp64_bh"], vel["fp64_direct"])
    out["error"] = {"mixed_vs_fp64_bh_rms_rel": rms, "mixed_vs_fp64_bh_max_rel": mx,
                    "bh_vs_fp64_direct_rms_rel": rms_a, "bh_vs_fp64_direct_max_rel": mx_a}
    return out


def gradient_rate(L, torch, steps: int = 256, reps: int = 2) -> dict:
    from qvort_b200 import adjoint as A
    from qvort_b200 import workloads as W

    w = W.trefoil_rings(smooth=True)
    prm = dict(w.params, velocity="Tree", tree_theta=0.4, precision="mixed", dt=1e-8)
    s = A.FilamentSystem(L.default_params(**prm), w.infront, w.behind)
    A.gradient(w.x, s, 16, 16)          # warm-up: buffers, tree capacity
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        A.gradient(w.x, s, steps, 16)
    torch.cuda.synchronize()
    sec = (time.perf_counter() - t0) / reps
    s.close()
    return {"value": 1.0 / sec, "unit": "gradients/s", "s_per_gradient": sec,
            "workload": f"16 trefoil rings, N={w.n}, smooth seeded 1e-5 cm displacement, "
                        f"periodic L=0.1, K={steps} AB steps at dt 1e-8 s (below the "
                        f"timestep_check bound {W.dt_max(w):.2e} s at the actual spacing), "
                        "checkpoint every 16, Tree theta 0.4 mixed forward, FP64 adjoint "
                        "(velocity, energy and AB step, all CUDA); loss = E(x_K) + "
                        "sum |x_K - x_0|^2; wall clock"}


def ring_rate(L, torch, steps: int = 1000) -> dict:
    """The single ring: N = 200, R = 0.01 cm, radial noise 1e-5, open, direct
    Biot-Savart + LIA in FP64, dt 1e-7, 1000 AB steps through qv_step, against
    the oracle's own steps on one host core; and the ring's translational
    speed against the formula the reference prints (src/initial_loop.f90:17-19)."""
    from oracle import oracle as O
    from qvort_b200 import workloads as W

    w = W.ring()
    c = L.Context(L.default_params(**dict(w.params, precision="fp64")))
    c.set_points(w.x, w.infront, w.behind)
    c.step(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(2, 102):
        c.step(it)
    step_s = (time.perf_counter() - t0) / 100
    t0 = time.perf_counter()
    c.steps(102, steps)            # one CUDA graph of a step, replayed; one wait
    gpu_s = (time.perf_counter() - t0) / steps
    x, u = c.get_points()
    c.close()
    R = 0.01
    v_ref = w.params["quant_circ"] / (4 * np.pi * R) * (np.log(8 * R / w.params["corea"]) - 0.5)
    st = O.State(O.params(**w.params), w.x, w.infront, w.behind)
    st.step()
    t0 = time.perf_counter()
    k = 50
    for _ in range(k):
        st.step()
    cpu_s = (time.perf_counter() - t0) / k
    n = w.n
    return {"workload": "ring N=200, R=0.01 cm, open, BS direct + LIA, FP64, dt 1e-7",
            "gpu_ms_per_step": gpu_s * 1e3, "gpu_steps_per_s": 1. / gpu_s,
            "gpu_ms_per_qv_step_call": step_s * 1e3,
            "gpu_pairs_per_s": n * n / gpu_s, "cpu_ms_per_step": cpu_s * 1e3,
            "cpu_steps_per_s": 1. / cpu_s, "cpu_cores": 1, "cpu_kind": "port",
            "ring_speed_cm_s": float(abs(np.mean(u[:, 2]))), "formula_speed_cm_s": float(v_ref),
            "timing": "wall clock around qv_steps (1000 steps, graph replay, one wait); "
                      "qv_step called per step (one wait each) for comparison"}


def direct_rate(L, torch, steps: int = 3, warmup: int = 1) -> dict:
    """The direct Biot-Savart sum (velocity BS, every segment against every
    target in all 27 images) on the tangle's initial state, FP64 and mixed:
    CUDA-event time of one velocity evaluation (LIA, compaction, source pack,
    direct kernel, reduction) and the mixed form's error against the FP64 one."""
    from qvort_b200 import workloads as W

    w = W.tangle(0)
    out, vel = {}, {}
    for prec in ("fp64", "mixed"):
        c = L.Context(L.default_params(**dict(w.params, precision=prec, velocity="BS",
                                              tree_theta=0.0)))
        c.set_points(w.x, w.infront, w.behind)
        for _ in range(max(1, warmup)):
            vel[prec] = c.velocity(False)[0]
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            c.velocity(False)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        n = w.n  # every slot of the initial tangle is active
        out[prec] = {"ms_per_velocity": ms, "pairs_per_s": float(n) * n * 27 / (ms * 1e-3)}
        c.close()
    rms, mx = _rel(vel["mixed"], vel["fp64"])
    out["error"] = {"mixed_vs_fp64_direct_rms_rel": rms, "mixed_vs_fp64_direct_max_rel": mx}
    out["workload"] = (f"tangle N={w.n}, periodic L=0.1 (27 images), direct sum (theta 0); "
                       "CUDA events around qv_velocity calls")
    return out


def batch_rate(L, torch, steps: int = 20, config=None) -> dict:
    """512 independent open systems (rings and leap-frogging pairs, N log-uniform
    in [100, 8000], dt from {5e-8, 1e-7, 2e-7}, direct below 2000 points,
    Barnes-Hut theta 0.4 above) advanced by qv_batch_step, against the same
    systems stepped one after another through single-system contexts."""
    from qvort_b200 import workloads as W

    ws = W.batch_systems()
    n_all = sum(w.n for w in ws)
    pairs = float(sum(w.n * w.n for w in ws))
    p = L.default_params(**dict(ws[0].params, boundary="open", velocity="Tree", tree_theta=0.4,
                                precision="mixed"))
    b = L.Batch(p, [(w.x, w.infront, w.behind) for w in ws], [w.params["velocity"] for w in ws],
                [w.params["dt"] for w in ws])
    if config:  # a given launch shape (warps per block, blocks per SM, order) instead of the tuner
        b.set_config(*config)
        tuned = {"warps_per_block": config[0], "blocks_per_sm": config[1], "order": config[2],
                 "given": True}
    else:
        tuned = b.tune(3)
    u_batch = b.velocity()
    b.step(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.step(steps)
    ms = (time.perf_counter() - t0) * 1e3 / steps
    st = b.stats()
    b.close()
    # the same systems one at a time (the per-system launch sequence of qv_step's
    # velocity + update), and the bitwise comparison of their velocities
    ctxs, equal = [], True
    for w, u in zip(ws, np.split(u_batch, np.cumsum([w.n for w in ws])[:-1])):
        c = L.Context(L.default_params(**dict(w.params, precision="mixed")))
        c.set_points(w.x, w.infront, w.behind)
        equal = equal and bool(np.array_equal(c.velocity(False)[0], u))
        ctxs.append((c, w.params["velocity"] == "Tree"))

    # the comparator: the same systems one after another, each through its own
    # context at its fastest -- a direct system replays a CUDA graph of its step
    # (qv_steps: one host wait for all K steps), a Barnes-Hut system runs qv_step
    # per step (its tree build reads the node count back)
    K = 20

    def seq_steps(it0):
        for c, tree in ctxs:
            if tree:
                for k in range(K):
                    c.step(it0 + k)
            else:
                c.steps(it0, K)

    seq_steps(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    seq_steps(1 + K)
    torch.cuda.synchronize()
    seq_ms = (time.perf_counter() - t0) * 1e3 / K
    for c, _ in ctxs:
        c.close()
    return {"ms_per_step": ms, "system_steps_per_s": len(ws) * 1e3 / ms,
            "pairs_per_s": pairs / (ms * 1e-3), "sequential_ms_per_step": seq_ms,
            "speedup_vs_sequential": seq_ms / ms, "velocities_bitwise_equal_to_sequential": equal,
            "graph": st["graph"], "tuned": tuned, "leaf_evals": st["leaf_evals"],
            "far_evals": st["far_evals"],
            "sequential": "each system through its own context, one after another: direct "
                          "systems replay a CUDA graph of their step (qv_steps, one wait per "
                          f"{K} steps), Barnes-Hut systems call qv_step per step; wall clock",
            "workload": f"512 open systems, N={n_all} points ({sum(w.params['velocity'] == 'Tree' for w in ws)} "
                        "Barnes-Hut theta 0.4, the rest direct), per-system dt; pairs = sum N_s^2 "
                        "(direct-equivalent); wall clock over the graph replays"}


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.suite != "large":
        import torch

        from qvort_b200 import lib as L

        if args.suite == "batch":
            cfg = [int(v) for v in args.batch_config.split(",")] if args.batch_config else None
            r = batch_rate(L, torch, args.steps, cfg)
        elif args.suite == "tangle":
            s = torch.cuda.Stream()
            r = tangle_rate(L, torch, s, torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8,
                                                   device="cuda"), args.steps, args.warmup)
        elif args.suite == "ring":
            r = ring_rate(L, torch)
        elif args.suite == "direct":
            r = direct_rate(L, torch, args.steps, args.warmup)
        else:
            r = gradient_rate(L, torch)
        print(json.dumps({"suite": args.suite, **r}), flush=True)
        return 0
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
