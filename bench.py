#!/usr/bin/env python
"""Benchmark of the PPPM-TDBEM time step on B200: Gcell-steps/s and achieved HBM GB/s.

Workload (default, --workload moving): a moving perturbed icosphere (5120 triangles, radius
0.08 m, translating 0.05 sin(2 pi 3 t) m and rotating 2 rad/s) beside a static 1280-triangle
plate at res 64, band-limited noise accelerations, motion frames at 1 kHz (69 PPPM steps per
frame).  One benchmark step = one motion frame: update_mesh (lists + cache refresh) plus the
69 time steps of that frame.  `value` is device-resident (inputs uploaded before timing);
`e2e` drives the same frames through the public API from pinned host buffers and reads the
listener samples back every frame.  --workload static runs the 1280-triangle sphere at
res 32 without motion (benchmark step = 100 time steps).  --workload large runs two moving
20480-triangle icospheres at res 128 (2.1 M cells, ~6.2 M face pairs; one benchmark step = one
1 kHz motion frame of 82 time steps).  --workload batch: 64 independent scenes in one batched
run (scenes/s); --workload adjoint: the transposed step against the forward step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank advances its own copy of the scene (replicas, weak
scaling); value = cells x steps over all ranks / max rank time.  The reference arm runs the
reference CUDA solver compiled from source (oracle/_ref) on rank 0, or the CPU oracle when
that build is absent.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "pppm-tdbem_b200", "python"))

from pppm_b200 import scenes  # noqa: E402

L2_FLUSH_BYTES = 256 << 20
CPU_SAMPLE_STEPS = 10


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=60, help="timed benchmark steps (motion frames)")
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="moving", choices=["moving", "static", "batch", "adjoint", "large"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fp64-check", action="store_true")
    p.add_argument("--summarize-launches", metavar="CSV",
                   help="print per-kernel launches / total time / share from an ncu "
                        "gpu__time_duration.sum CSV log of this benchmark, and exit")
    return p.parse_args()


# ---------------------------------------------------------------- distributed ---------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    import torch

    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(ws, x):
    import torch

    if ws == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- clocks --------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- workloads -----------
class Workload:
    """Frames of the benchmark: per frame the vertex positions and the step range."""

    def __init__(self, kind, nframes):
        self.kind = kind
        self.moving = kind in ("moving", "large")
        if self.moving:
            sc = scenes.MovingScene() if kind == "moving" else scenes.LargeScene()
            self.scene = sc
            self.ranges = scenes.frame_ranges(sc, nframes)
            self.verts = [sc.frame_verts(f) for f in range(nframes + 1)]
            self.name = ("moving icosphere (5120 tris) + static plate (1280 tris), res 64, 1 kHz motion frames"
                         if kind == "moving" else
                         "two moving icospheres (2 x 20480 tris), res 128, 1 kHz motion frames")
        else:
            sc = scenes.StaticSphere()
            self.scene = sc
            per = 100
            self.ranges = [(f * per, (f + 1) * per) for f in range(nframes + 1)]
            self.verts = [sc.verts for _ in range(nframes + 1)]
            self.name = "static icosphere (1280 tris), res 32"
        self.total_steps = self.ranges[-1][1]
        self.res = sc.res
        self.tris = sc.tris
        self.listener = sc.listener
        self.acc = sc.acc(0, self.total_steps)


def algorithmic_bytes(counts, res, nt):
    """Compulsory bytes per launch of each per-step kernel (FP32 scheme)."""
    m = res - 2
    n3, p3, pf = counts[0], counts[1], counts[4]
    abc = 6 * m * m
    stencil = 12 * m ** 3 + 16 * abc + 4 * n3 + 16 * nt  # p^t, p^{t-1}, p^{t+1}; ghosts; corrections; acc -> 4 ring copies
    # face pairs (weights 64, scale 8, neighbour index 4); per triangle: corners, interpolation
    # weights, far-field values, start, denominator, 4 Dirichlet copies, its own history windows;
    # the near-field terms: 54 grid-cache records (64 + scale 8) read, 54 terms written
    face = pf * (64 + 8 + 4) + nt * (8 * 4 + 8 * 4 + 8 * 4 + 8 + 8 + 16 + 2 * 64) + nt * 54 * (64 + 8 + 4)
    # per pair: triangle index 4, record offset 1, two terms 8; per cell: index, start, p read/write, next
    near = p3 * (4 + 1 + 8) + n3 * (4 + 8 + 4 + 4 + 4)
    return {"stencil": stencil, "face": face, "near": near}


def conv_bytes(counts, nt, pairs):
    """Compulsory bytes of one launch of the face-pair convolution: per pair its weights (64),
    scale (8) and neighbour index (4); per triangle its list start, its own two history windows
    (2 x 64) and its output sum(s); the two-step pass also reads the next acceleration row."""
    pf = counts[4]
    return pf * (64 + 8 + 4) + nt * (4 + 2 * 64 + (8 + 4 if pairs else 4))


def fix_bytes(counts, nt):
    """Compulsory bytes of the completion of a two-step pass: per pair its tap-1 factor and
    neighbour index; per triangle its list start, the neighbour value it gathers, the partial sum
    read and the sum written."""
    return counts[4] * (4 + 4) + nt * (4 + 4 + 4 + 4)


def load_traffic(workload):
    """ncu DRAM bytes (read + write) per launch by kernel for one workload, from
    profiles/traffic.txt (lines: workload kernel bytes)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            f = line.split()
            if len(f) >= 3 and not line.startswith("#") and f[0] == workload:
                try:
                    out[f[1]] = float(f[2])
                except ValueError:
                    pass
    return out


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return float(json.load(open(path))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


# ---------------------------------------------------------------- our arm -------------
def run_ours(args, ws, rank, local):
    import torch

    from pppm_b200 import Solver

    W, K = args.warmup, args.steps
    wl = Workload(args.workload, W + K)
    sc = wl.scene
    dev = torch.device("cuda", local)
    # one non-default stream for the solver, the L2 flush and every timing event (with the
    # default stream the solver would create its own, which those events would not see)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    acc_dev = torch.from_numpy(wl.acc).to(dev)
    verts_dev = [torch.from_numpy(v).to(dev) for v in wl.verts]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    s = Solver(wl.res, sc.h, sc.dt, sc.min_pos, device=local, stream=stream.cuda_stream)
    s.set_mesh(wl.verts[0], wl.tris)
    s.add_listener(*wl.listener)
    # face-stage autotuner on the first frame's mesh (setup, untimed): picks one or two steps per
    # pass over the face pairs and the block size of the face kernels
    tune = s.autotune(reps=20)

    def frame(f, timed_events=None):
        a, b = wl.ranges[f]
        if f > 0 and wl.moving:
            s.update_mesh(verts_dev[f])
        s.step(acc_dev[a:b])

    for f in range(0, W + 1):  # frame 0 = the set_mesh frame, then W warm-up frames
        frame(f)
    torch.cuda.synchronize()
    launches0 = s.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    total_ms = 0.0
    step_ms = 0.0
    steps = 0
    for f in range(W + 1, W + K + 1):
        flush.zero_()
        e0, em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a, b = wl.ranges[f]
        e0.record(stream)
        if wl.moving:
            s.update_mesh(verts_dev[f])
        em.record(stream)
        s.step(acc_dev[a:b])
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        step_ms += em.elapsed_time(e1)
        steps += b - a
    barrier(ws)
    clk = clocks.stop()
    launches = s.launch_count() - launches0
    t_max = max_over_ranks(ws, total_ms)
    cells = float(wl.res) ** 3
    value = cells * steps * ws / (t_max * 1e-3) / 1e9

    # per-kernel durations (measurement mode: events around each kernel, synchronised)
    s.enable_timing(True)
    a, b = wl.ranges[W + K]
    s.step(acc_dev[a:b])
    us_st, us_face, us_near, nt_timed = s.kernel_times()
    s.enable_timing(False)
    counts = [int(x) for x in s.dump("counts")]
    alg = {k: int(v) for k, v in algorithmic_bytes(counts, wl.res, len(wl.tris)).items()}
    times = {"stencil": us_st, "face": us_face, "near": us_near}
    # the dominant kernel of the recorded steps: the tuned face-pair convolution (its launch time
    # from the autotuner's events on the solver's stream, last frame's mesh: re-tuned here)
    tune = s.autotune(reps=20)
    pairs, threads = tune["best"]
    nt = len(wl.tris)
    top = "conv2" if pairs else "conv"
    top_us = tune["launch_us"][tune["best"]][0]
    top_bytes = conv_bytes(counts, nt, pairs)
    peak, peak_kind = measured_peak()
    achieved = float(top_bytes / (top_us * 1e-6) / 1e9)
    traffic = load_traffic(args.workload).get(top)
    # split of a timed frame: update_mesh, then the frame's time steps (one recorded graph)
    us_update = (total_ms - step_ms) * 1e3 / K
    us_per_step = step_ms * 1e3 / steps

    # end-to-end through the public API from pinned host buffers
    e2e = None
    if not args.no_e2e:
        s2 = Solver(wl.res, sc.h, sc.dt, sc.min_pos, device=local, stream=stream.cuda_stream)
        s2.set_option("conv_pairs", pairs)
        s2.set_option("face_threads", threads)
        s2.set_option("terms_pairs", tune["terms_pairs"])
        s2.set_mesh(wl.verts[0], wl.tris)
        s2.add_listener(*wl.listener)
        acc_pin = torch.from_numpy(wl.acc).pin_memory()
        verts_pin = [torch.from_numpy(v).pin_memory() for v in wl.verts]
        out_pin = torch.empty((200,), dtype=torch.float32).pin_memory()
        h2d = d2h = 0
        for f in range(0, W + 1):
            a, b = wl.ranges[f]
            if f > 0 and wl.moving:
                s2.update_mesh(verts_pin[f])
            s2.step(acc_pin[a:b])
        barrier(ws)
        t0 = time.perf_counter()
        steps2 = 0
        for f in range(W + 1, W + K + 1):
            a, b = wl.ranges[f]
            if wl.moving:
                s2.update_mesh(verts_pin[f])
                h2d += verts_pin[f].numel() * 4
            s2.step(acc_pin[a:b])
            h2d += (b - a) * len(wl.tris) * 4
            done = s2.listeners(first=a, count=b - a)
            d2h += done.nbytes
            steps2 += b - a
        torch.cuda.synchronize()
        te = max_over_ranks(ws, time.perf_counter() - t0)
        e2e = {"value": cells * steps2 * ws / te / 1e9, "unit": "Gcell-steps/s",
               "h2d_bytes_per_step": h2d // K, "d2h_bytes_per_step": d2h // K}
        s2.close()
        del out_pin

    # error of the timed FP32 run against the FP64 scheme of the same library on the GPU, over the
    # same frames (set-up and warm-up frames included; outside the timed region)
    fp64_err = None
    if not args.no_fp64_check:
        n = wl.ranges[W + K][1]
        got = s.listeners(0, n)[:, 0].astype(np.float64)
        s64 = Solver(wl.res, sc.h, sc.dt, sc.min_pos, device=local, stream=stream.cuda_stream, precision="fp64")
        s64.set_mesh(wl.verts[0], wl.tris)
        s64.add_listener(*wl.listener)
        for f in range(0, W + K + 1):
            a, b = wl.ranges[f]
            if f > 0 and wl.moving:
                s64.update_mesh(verts_dev[f])
            s64.step(acc_dev[a:b])
        ref = s64.listeners(0, n)[:, 0].astype(np.float64)
        s64.close()
        den = float(np.linalg.norm(ref))
        fp64_err = {"rel_l2": float(np.linalg.norm(got - ref) / den) if den > 0 else None, "time_steps": int(n),
                    "reference": "the same frames in the FP64 scheme (PPPM_PRECISION_FP64) on the GPU"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl)

    s.close()
    line = {
        "metric": "Gcell-steps/s, %s (time step + motion-frame refresh)" % wl.name,
        "value": round(value, 4), "unit": "Gcell-steps/s", "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": round(t_max / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded meshes, trajectories and accelerations)",
        "config": {"workload": wl.name, "res": wl.res, "triangles": int(len(wl.tris)),
                   "time_steps_per_bench_step": round(steps / K, 2), "time_steps_timed": steps,
                   "bench_step": "one motion frame: update_mesh + its time steps" if wl.moving
                   else "100 time steps", "l2": "flushed (256 MiB write) between timed iterations",
                   "parallelism": "replicas x%d" % ws, "precision": "fp32 grids, fp16+scale weights",
                   "n3_cells": int(counts[0]), "pairs_3x3x3": int(counts[1]), "face_pairs": int(counts[4])},
        "roofline": {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes": int(top_bytes), "kernel_launch_us": round(top_us, 3),
                     "autotune": {"best": {"two_steps_per_pass": bool(pairs), "threads": threads,
                                           "terms_two_steps_per_pass": bool(tune["terms_pairs"])},
                                  "decided_by": "64 recorded steps per option set (phase 2)",
                                  "finish_us_per_two_steps": {k: round(v, 2) for k, v in tune["finish_us"].items()},
                                  "step_us_by_config": {"%s/%d/%s" % (("single", "pairs")[p], t,
                                                                      "terms2" if m else "terms1"): round(u, 2)
                                                        for (p, t, m), u in (tune["step_us"] or {}).items()},
                                  "us_per_two_steps": {"%s/%d" % (("single", "pairs")[p], t): round(u, 2)
                                                       for (p, t), u in tune["us"].items()}},
                     "fix_us": round(tune["launch_us"][tune["best"]][1], 3) if pairs else None,
                     "fix_bytes": int(fix_bytes(counts, nt)) if pairs else None,
                     "kernel_us_measurement_mode": {k: round(v, 3) for k, v in times.items()},
                     "update_mesh_us": round(us_update, 1), "time_step_us": round(us_per_step, 2),
                     "gb_per_s_all_kernels": round(sum(alg.values()) / (sum(times.values()) * 1e-6) / 1e9, 1)},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
        "error_vs_fp64": fp64_err,
    }
    return line


# ---------------------------------------------------------------- batched scenes ------
BATCH_SCENES = 64
BATCH_SEED = 11
BATCH_NAME = ("64 scenes from seed 11: res in {24,32,48,64}, perturbed icosphere subdivision 2-4 "
              "(320-5120 tris), 1000-4000 steps each")


def batch_listener(res):
    return (res - 4, res // 2, res // 2)


def batch_acc(spec, device):
    """(steps, nt) float32 accelerations of one batch scene: a sine at the scene's frequency on
    every triangle (device tensor, or pinned host tensor for device == "pinned")."""
    import torch

    t = torch.arange(spec["steps"], dtype=torch.float64) * float(spec["dt"])
    a = torch.sin(2 * math.pi * spec["freq"] * t).to(torch.float32)
    a = a[:, None].expand(spec["steps"], len(spec["tris"])).contiguous()
    return a.pin_memory() if device == "pinned" else a.to(device)


def run_batch(args, ws, rank, local):
    """Scenes/s of the 64-scene batch: one benchmark step = every scene run through all of its
    time steps, batched (pppm_batch_run) and, for comparison, scene by scene (pppm_step)."""
    import torch

    from pppm_b200 import Batch, Solver

    W, K = args.warmup, args.steps
    all_specs = scenes.batch_scenes(BATCH_SCENES, BATCH_SEED)
    # N ranks: a static partition of the scenes by estimated cost, no exchange while stepping,
    # one gather of the listener series at the end (strong scaling: the 64-scene job is fixed)
    mine = scenes.shard_by_cost(all_specs, ws)[rank]
    specs = [all_specs[i] for i in mine]
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    solvers = []
    for sp in specs:
        s = Solver(sp["res"], sp["h"], sp["dt"], sp["min_pos"], device=local, stream=stream.cuda_stream)
        s.set_mesh(sp["verts"], sp["tris"])
        s.add_listener(*batch_listener(sp["res"]))
        solvers.append(s)
    accs = [batch_acc(sp, dev) for sp in specs]
    t_start = [s.t for s in solvers]
    batch = Batch(solvers)

    def rewind():
        for s, t0 in zip(solvers, t_start):
            s.reset_fields()
            s.rewind_listeners()
            s.t = t0

    def timed(run, reps, clocks=None):
        for _ in range(W):
            rewind()
            run()
        torch.cuda.synchronize()
        launches0 = sum(s.launch_count() for s in solvers)
        if clocks:
            clocks.start()
        barrier(ws)
        ms = 0.0
        for _ in range(reps):
            rewind()
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        barrier(ws)
        clk = clocks.stop() if clocks else None
        return max_over_ranks(ws, ms), sum(s.launch_count() for s in solvers) - launches0, clk

    def run_batched():
        batch.run(accs)

    def run_sequential():
        for s, a in zip(solvers, accs):
            s.step(a)

    clocks = ClockSampler(local)
    ms_b, launches, clk = timed(run_batched, K, clocks)
    ms_s, launches_s, _ = timed(run_sequential, max(1, min(K, 2)))
    reps_s = max(1, min(K, 2))
    series_b = [s.listeners() for s in solvers]
    rewind()
    run_sequential()
    same = all(np.array_equal(a, s.listeners()) for a, s in zip(series_b, solvers))
    value = BATCH_SCENES * K / (ms_b * 1e-3)
    seq = BATCH_SCENES * reps_s / (ms_s * 1e-3)
    cell_steps = sum(float(sp["res"]) ** 3 * sp["steps"] for sp in all_specs)
    # compulsory bytes of the whole job (per-step kernel bytes of each scene x its steps)
    job_bytes = 0.0
    for sp, s in zip(specs, solvers):
        counts = [int(x) for x in s.dump("counts")]
        job_bytes += sum(algorithmic_bytes(counts, sp["res"], len(sp["tris"])).values()) * sp["steps"]
    gather_ms, gathered = 0.0, len(specs)
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([job_bytes], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        job_bytes = float(t.item())
        # the job's result: every scene's listener series on every rank
        barrier(ws)
        t0 = time.perf_counter()
        parts = [None] * ws
        dist.all_gather_object(parts, [(i, s.listeners()) for i, s in zip(mine, solvers)])
        gather_ms = max_over_ranks(ws, (time.perf_counter() - t0) * 1e3)
        gathered = len({i for part in parts for i, _ in part})
        same = bool(int(max_over_ranks(ws, 0.0 if same else 1.0)) == 0)

    e2e = None
    if not args.no_e2e:
        pinned = [batch_acc(sp, "pinned") for sp in specs]
        h2d = sum(a.numel() * 4 for a in pinned)
        d2h = 0
        for _ in range(W):
            rewind()
            batch.run(pinned)
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(K):
            rewind()
            batch.run(pinned)
            d2h = 0
            for s in solvers:
                d2h += s.listeners().nbytes
        torch.cuda.synchronize()
        te = max_over_ranks(ws, time.perf_counter() - t0)
        e2e = {"value": round(BATCH_SCENES * K / te, 3), "unit": "scenes/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h)}
        del pinned

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_batch_baseline(specs)
    batch.close()
    for s in solvers:
        s.close()
    return {
        "metric": "scenes/s, %s" % BATCH_NAME, "value": round(value, 3), "unit": "scenes/s", "n_gpus": ws,
        "steps": K, "warmup": W, "ms_per_step": round(ms_b / K, 3), "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded meshes and accelerations)",
        "config": {"workload": BATCH_NAME, "scenes": BATCH_SCENES, "time_steps_per_bench_step":
                   int(sum(sp["steps"] for sp in all_specs)), "gcell_steps_per_bench_step": round(cell_steps / 1e9, 3),
                   "bench_step": "every scene through all of its time steps (one pppm_batch_run call)",
                   "l2": "flushed (256 MiB write) between timed iterations",
                   "parallelism": "scenes sharded by estimated cost over %d ranks, no exchange while stepping" % ws
                   if ws > 1 else "one GPU", "scenes_on_rank0": len(specs), "series_gathered": gathered,
                   "gather_ms": round(gather_ms, 3)},
        "sequential": {"value": round(seq, 3), "unit": "scenes/s", "reps": reps_s, "ms_per_rep": round(ms_s / reps_s, 3),
                       "gpu_launches_per_rep": int(launches_s // reps_s), "listeners_bit_identical": bool(same)},
        "batched_over_sequential": round(value / seq, 3),
        "roofline": {"bound": "hbm", "kernel": "all step kernels of the job", "traffic": None,
                     "algorithmic_bytes_per_bench_step": int(job_bytes),
                     "achieved": round(job_bytes * K / (ms_b * 1e-3) / 1e9, 1),
                     "achieved_sequential": round(job_bytes * reps_s / (ms_s * 1e-3) / 1e9, 1),
                     "peak": measured_peak()[0], "unit": "GB/s", "peak_kind": measured_peak()[1],
                     "frac": round(job_bytes * K / (ms_b * 1e-3) / 1e9 / measured_peak()[0], 4)},
        "gcell_steps_per_s": round(cell_steps * K / (ms_b * 1e-3) / 1e9, 3),
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
    }


# ---------------------------------------------------------------- adjoint -------------
ADJ_NAME = ("moving-scene geometry held static at res 48 (5120-tri perturbed sphere + 1280-tri plate), "
            "4000 steps, loss ||s - s_target||^2, gradient w.r.t. every acceleration (FP32)")


def run_adjoint(args, ws, rank, local):
    """Cost of the gradient against the forward run: one benchmark step = the 4000-step forward
    run (pppm_step, device-resident accelerations) and the adjoint sweep over the same steps
    (pppm_adjoint from dL/dsignal on the device)."""
    import torch

    from pppm_b200 import Solver

    W, K = args.warmup, args.steps
    sc = scenes.MovingScene(res=48)
    nsteps = 4000
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    s = Solver(sc.res, sc.h, sc.dt, sc.min_pos, device=local, stream=stream.cuda_stream)
    s.set_mesh(sc.frame_verts(0), sc.tris)
    s.add_listener(*sc.listener)
    acc = torch.from_numpy(sc.acc(0, nsteps)).to(dev)
    target = torch.zeros((nsteps, 1), dtype=torch.float32, device=dev)
    sig = torch.empty((nsteps, 1), dtype=torch.float32, device=dev)
    t0 = s.t

    def forward():
        s.reset_fields()
        s.rewind_listeners()
        s.t = t0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record(stream)
        s.step(acc)
        e1.record(stream)
        s.series(0, nsteps, out=sig)
        return e0, e1

    def backward():
        g = 2 * (sig - target)
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        grad = s.adjoint(g, fresh=True)
        e1.record(stream)
        return e0, e1, grad

    for _ in range(W):
        forward()
        backward()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    launches0 = s.launch_count()
    f_ms = b_ms = 0.0
    for _ in range(K):
        f0, f1 = forward()
        b0, b1, grad = backward()
        b1.synchronize()
        f_ms += f0.elapsed_time(f1)
        b_ms += b0.elapsed_time(b1)
    barrier(ws)
    clk = clocks.stop()
    launches = s.launch_count() - launches0
    f_ms, b_ms = max_over_ranks(ws, f_ms), max_over_ranks(ws, b_ms)
    finite = bool(torch.isfinite(grad).all().item())
    s.close()
    ratio = b_ms / f_ms
    cells = float(sc.res) ** 3
    return {
        "metric": "adjoint / forward cost, %s" % ADJ_NAME, "value": round(ratio, 4), "unit": "x forward",
        "n_gpus": ws, "steps": K, "warmup": W, "ms_per_step": round((f_ms + b_ms) / K, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded mesh and accelerations)",
        "config": {"workload": ADJ_NAME, "res": sc.res, "triangles": int(len(sc.tris)), "time_steps": nsteps,
                   "bench_step": "forward run + adjoint sweep", "l2": "flushed (256 MiB write) before each timed run",
                   "parallelism": "replicas x%d" % ws},
        "forward_us_per_step": round(f_ms * 1e3 / (K * nsteps), 3),
        "adjoint_us_per_step": round(b_ms * 1e3 / (K * nsteps), 3),
        "forward_gcell_steps_per_s": round(cells * nsteps * K * ws / (f_ms * 1e-3) / 1e9, 3),
        "adjoint_gcell_steps_per_s": round(cells * nsteps * K * ws / (b_ms * 1e-3) / 1e9, 3),
        "gradient_finite": finite, "cpu_baseline": None, "e2e": None, "gpu_launches": int(launches), "clocks": clk,
    }


def cpu_batch_baseline(specs, sample=4, steps=20):
    """The CPU restatement on the first `sample` batch scenes, `steps` time steps each (set_mesh
    untimed), extrapolated to every step of those scenes: scenes/s on the host cores."""
    from oracle.oracle import Oracle, oracle_threads

    est = 0.0
    for sp in specs[:sample]:
        o = Oracle(sp["res"], sp["h"], sp["dt"], sp["min_pos"])
        o.set_mesh(sp["verts"], sp["tris"])
        acc = np.ones((steps, len(sp["tris"])), np.float32)
        t0 = time.perf_counter()
        o.step(acc, listeners=[batch_listener(sp["res"])])
        est += (time.perf_counter() - t0) / steps * sp["steps"]
        o.close()
    return {"value": round(sample / est, 5), "unit": "scenes/s", "cores": oracle_threads(), "kind": "port",
            "sample": "first %d scenes, %d time steps each, extrapolated to their full step counts (C restatement "
                      "with OpenMP)" % (sample, steps)}


def cpu_baseline(wl):
    """The CPU restatement (oracle/) on the host cores: one benchmark step of the same
    workload (set_mesh untimed)."""
    from oracle.oracle import Oracle, oracle_threads

    sc = wl.scene
    o = Oracle(wl.res, sc.h, sc.dt, sc.min_pos)
    o.set_mesh(wl.verts[0], wl.tris)
    f = 1
    a, b = wl.ranges[f]
    # the large scene's frame takes about a minute on the host: time update_mesh and the first
    # CPU_SAMPLE_STEPS of its steps, and extrapolate the steps to the whole frame
    n = b - a if wl.kind != "large" else min(b - a, CPU_SAMPLE_STEPS)
    t0 = time.perf_counter()
    if wl.moving:
        o.update_mesh(wl.verts[f])
    t1 = time.perf_counter()
    o.step(wl.acc[a:a + n], listeners=[wl.listener])
    t2 = time.perf_counter()
    o.close()
    dt = (t1 - t0) + (t2 - t1) * (b - a) / n
    sample = "one benchmark step (%d time steps%s) of the same workload, C restatement with OpenMP" % (
        b - a, " + update_mesh" if wl.moving else "")
    if n < b - a:
        sample += "; update_mesh and the first %d time steps timed, the steps extrapolated to %d" % (n, b - a)
    return {"value": round(float(wl.res) ** 3 * (b - a) / dt / 1e9, 5), "unit": "Gcell-steps/s",
            "cores": oracle_threads(), "kind": "port", "sample": sample}


# ---------------------------------------------------------------- reference arm -------
def run_reference(args, ws, rank, local):
    if rank != 0:
        return None
    W, K = args.warmup, args.steps
    if args.workload == "batch":
        return run_reference_batch(args)
    if args.workload == "adjoint":
        return {"impl": "reference", "metric": "adjoint / forward cost, %s" % ADJ_NAME,
                "unavailable": "the reference has no adjoint"}
    wl = Workload(args.workload, W + K)
    sc = wl.scene
    from oracle import oracle as O

    ndebug = None
    if O.reference_available():
        import torch

        acc_dev = torch.from_numpy(wl.acc).cuda()
        nt = len(wl.tris)
        ptr0 = acc_dev.data_ptr()

        def timed_run(nd):
            """W warm-up and K timed frames of the reference build (nd: the -DNDEBUG build)."""
            r = O.Reference(wl.res, sc.h, sc.dt, sc.min_pos, ndebug=nd)
            r.set_mesh(wl.verts[0], wl.tris)
            if wl.moving:
                for v in wl.verts[1:]:
                    r.check_mesh(v)  # validate the whole trajectory against the reference capacities
                r.set_checks(False)

            def frame(f):
                a, b = wl.ranges[f]
                if f > 0 and wl.moving:
                    r.update_mesh(wl.verts[f])
                r.run_device(ptr0 + a * nt * 4, b - a, wl.listener)

            for f in range(0, W + 1):
                frame(f)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            steps = 0
            for f in range(W + 1, W + K + 1):
                frame(f)
                steps += wl.ranges[f][1] - wl.ranges[f][0]
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            r.close()
            return float(wl.res) ** 3 * steps / dt / 1e9

        value = timed_run(False)
        if O.reference_available(ndebug=True):
            ndebug = {"value": round(timed_run(True), 5), "unit": "Gcell-steps/s",
                      "build": "the same reference sources built with -DNDEBUG (no device sync after every launch)"}
        kind, cores, sample = "reference", 0, ("reference CUDA solver built from source (oracle/_ref, upstream flags: "
                                                "device sync after every launch), %d frames" % K)
    else:
        from oracle.oracle import Oracle, oracle_threads

        o = Oracle(wl.res, sc.h, sc.dt, sc.min_pos)
        o.set_mesh(wl.verts[0], wl.tris)
        t0 = time.perf_counter()
        steps = 0
        for f in range(1, min(W + K, 3) + 1):
            a, b = wl.ranges[f]
            if wl.moving:
                o.update_mesh(wl.verts[f])
            o.step(wl.acc[a:b], listeners=[wl.listener])
            steps += b - a
        dt = time.perf_counter() - t0
        value = float(wl.res) ** 3 * steps / dt / 1e9
        kind, cores, sample = "port", oracle_threads(), "CPU restatement, %d frames" % min(W + K, 3)
    return {"impl": "reference", "metric": "Gcell-steps/s, %s (time step + motion-frame refresh)" % wl.name,
            "value": round(value, 5), "unit": "Gcell-steps/s", "n_gpus": 1, "steps": K, "warmup": W,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded meshes, trajectories and accelerations)",
            "config": {"workload": wl.name, "res": wl.res, "triangles": int(len(wl.tris))},
            "cpu_baseline": {"value": round(value, 5), "unit": "Gcell-steps/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 5), "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_ndebug": ndebug}


def run_reference_batch(args):
    """The reference solver (oracle/_ref) run scene by scene over the 64-scene batch: one timed
    pass (each scene's set_mesh untimed), after one warm-up scene."""
    from oracle import oracle as O

    line = {"impl": "reference", "metric": "scenes/s, %s" % BATCH_NAME, "unit": "scenes/s"}
    if not O.reference_available():
        line["unavailable"] = "reference solver not built (oracle/_ref)"
        return line
    import torch

    specs = scenes.batch_scenes(BATCH_SCENES, BATCH_SEED)

    def one(sp):
        r = O.Reference(sp["res"], sp["h"], sp["dt"], sp["min_pos"])
        try:
            r.set_mesh(sp["verts"], sp["tris"])
            acc = batch_acc(sp, torch.device("cuda"))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r.run_device(acc.data_ptr(), sp["steps"], batch_listener(sp["res"]))
            torch.cuda.synchronize()
            return time.perf_counter() - t0
        finally:
            r.close()

    try:
        one(specs[0])
        total = sum(one(sp) for sp in specs)
    except RuntimeError as e:
        line["unavailable"] = "reference solver rejected a batch scene: %s" % e
        return line
    value = BATCH_SCENES / total
    line.update({"value": round(value, 4), "n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": True,
                 "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                 "data": "synthetic (seeded meshes and accelerations)",
                 "config": {"workload": BATCH_NAME, "scenes": BATCH_SCENES},
                 "cpu_baseline": {"value": round(value, 4), "unit": "scenes/s", "cores": 0, "kind": "reference",
                                  "sample": "reference CUDA solver built from source, the 64 scenes one after another "
                                            "(set_mesh untimed)"},
                 "e2e": {"value": round(value, 4), "unit": "scenes/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    return line


def summarize_launches(path):
    """Per-kernel launch count, total and mean device time and share of an ncu launch list."""
    import collections
    import csv

    with open(path) as f:
        lines = [l for l in f if not l.startswith("==")]
    agg = collections.defaultdict(lambda: [0, 0.0])
    scale = {"ns": 1e-3, "nsecond": 1e-3, "us": 1.0, "usecond": 1.0, "ms": 1e3, "msecond": 1e3}
    for row in csv.DictReader(lines):
        if row.get("Metric Name") != "gpu__time_duration.sum":
            continue
        name = row["Kernel Name"].split("(")[0].replace("pb::<unnamed>::", "").replace("void ", "")
        agg[name][0] += 1
        agg[name][1] += float(row["Metric Value"].replace(",", "")) * scale.get(row["Metric Unit"], 1.0)
    total = sum(v[1] for v in agg.values())
    print("| kernel | launches | total us | mean us | share |")
    print("|---|---|---|---|---|")
    for name, (n, t) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
        print("| %s | %d | %.1f | %.2f | %.1f%% |" % (name, n, t, t / n, 100 * t / total))


def main():
    args = parse()
    if args.summarize_launches:
        summarize_launches(args.summarize_launches)
        return
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        line = run_reference(args, ws, rank, local)
    elif args.workload == "batch":
        line = run_batch(args, ws, rank, local)
    elif args.workload == "adjoint":
        line = run_adjoint(args, ws, rank, local)
    else:
        line = run_ours(args, ws, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
