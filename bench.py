#!/usr/bin/env python
"""Benchmark of the PPPM-TDBEM time step on B200: Gcell-steps/s and achieved HBM GB/s.

Workload (default, --workload moving): a moving perturbed icosphere (5120 triangles, radius
0.08 m, translating 0.05 sin(2 pi 3 t) m and rotating 2 rad/s) beside a static 1280-triangle
plate at res 64, band-limited noise accelerations, motion frames at 1 kHz: 8820 time steps in
128 frames.  One benchmark step = that whole run on a fresh handle (set_mesh of frame 0 is the
untimed set-up; then frame 0's steps and 127 x (update_mesh + the frame's steps)).  `value` is
device-resident (inputs uploaded before timing); `e2e` drives the same runs through the public
API from pinned host buffers and reads the listener samples back every frame.  --workload static
runs the 1280-triangle sphere at res 32 without motion (benchmark step = its whole 2000-step
run).  --workload large runs two moving 20480-triangle icospheres at res 128 (2.1 M cells, ~6.2 M
face pairs; one benchmark step = one 1 kHz motion frame of 82 time steps).  --workload batch: 64
independent scenes in one batched run (scenes/s); --workload adjoint: the transposed step
against the forward step (static geometry, res 48); --workload adjoint-moving: the gradient of the
large scene's moving run through motion checkpoints every 200 steps, against the run;
--workload large-batch: the large scene batched x4 with four seeds.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: with --gpus N > 1 and no torchrun environment the script starts N ranks itself
(torch.distributed.run on 127.0.0.1).  Every rank advances its own copy of the scene (replicas,
weak scaling); value = cells x steps over all ranks / max rank time; the batch workload shards
its scenes over the ranks.  The reference arm runs the reference CUDA solver compiled from
source (oracle/_ref) on rank 0, or the CPU oracle when that build is absent.
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
    p.add_argument("--steps", type=int, default=10, help="timed benchmark steps (whole runs; frames for large)")
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="moving",
                   choices=["moving", "static", "batch", "adjoint", "adjoint-moving", "large", "large-batch"])
    p.add_argument("--adjoint-steps", type=int, default=20000,
                   help="time steps of the adjoint-moving run (the large scene's 20000 by default)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fp64-check", action="store_true")
    p.add_argument("--profile-frame", type=int, metavar="F",
                   help="profiling driver: run the workload's frames 0..F-1, then frame F (update_mesh + its "
                        "steps) inside the NVTX range 'profile_frame', and exit (for ncu --nvtx-include); the "
                        "launch options are --options, not the autotuner's (a profiler distorts its timings)")
    p.add_argument("--options", default="1,128,0", metavar="PAIRS,THREADS,TERMS",
                   help="launch options of --profile-frame: conv_pairs, face_threads, terms_pairs")
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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
    """The scene of a single-scene benchmark and its motion frames.

    moving  the whole 8820-step run of the moving sphere + plate (128 motion frames at 1 kHz);
            one benchmark step = that whole run on a fresh handle: frame 0 after set_mesh, then
            127 x (update_mesh + the frame's steps)
    static  the whole 2000-step run of the pulsating sphere; one benchmark step = that run
    large   two moving 20480-triangle spheres at res 128; one benchmark step = one motion frame
            (update_mesh + its ~82 steps) of a continuing run (the whole 20000-step run takes
            seconds per repetition)
    """

    def __init__(self, kind, nframes=None):
        self.kind = kind
        self.moving = kind in ("moving", "large")
        self.whole_run = kind in ("moving", "static")
        if kind == "moving":
            sc = scenes.MovingScene()
            self.name = "moving icosphere (5120 tris) + static plate (1280 tris), res 64, 1 kHz motion frames"
        elif kind == "large":
            sc = scenes.LargeScene()
            self.name = "two moving icospheres (2 x 20480 tris), res 128, 1 kHz motion frames"
        else:
            sc = scenes.StaticSphere()
            self.name = "static icosphere (1280 tris), res 32"
        self.scene = sc
        if kind == "moving":
            n = sc.frame_of_step(sc.steps - 1) + 1
            self.ranges = scenes.frame_ranges(sc, n - 1)
            self.ranges[-1] = (self.ranges[-1][0], sc.steps)
        elif kind == "large":
            self.ranges = scenes.frame_ranges(sc, nframes)
        else:
            self.ranges = [(0, sc.steps)]
        self.verts = [sc.frame_verts(f) for f in range(len(self.ranges))] if self.moving else [sc.verts]
        self.total_steps = self.ranges[-1][1]
        self.res = sc.res
        self.tris = sc.tris
        self.listener = sc.listener
        self.acc = sc.acc(0, self.total_steps)


def algorithmic_bytes(counts, res, nt):
    """Compulsory bytes per launch of each step kernel kind (FP32 scheme), by the arrays each
    reads and writes once: counts = pppm_dump(COUNTS) of the current mesh."""
    m = res - 2
    n3, p3, pf = counts[0], counts[1], counts[4]
    # p^t and p^{t-1} read, p^{t+1} written per cell; the ghost layer of p^t written; the
    # correction read at corrected cells; the corrected-cell bit mask
    stencil = 12 * m ** 3 + 4 * 6 * m * m + 4 * n3 + m ** 3 // 8
    # per pair: weights 64 (16 taps x half2), scale 8, neighbour 4; per triangle: list start 8,
    # its two history windows 2 x 64 (read once whatever the number of pairs naming it), sum out
    conv = pf * 76 + nt * (8 + 128 + 4 + 4)
    conv2 = pf * 76 + nt * (8 + 128 + 4 + 4 + 8)  # + next acceleration row, second sum
    fix = pf * 8 + nt * 20  # per pair tap-1 factor and neighbour; per triangle start, D, sums
    # per triangle: 8 corners (interp weight, cell index, far value), conv sum, denominator,
    # 4 Dirichlet copies + last D, own N and D windows, 54 grid-cache records (64 + 8), 54 terms
    # written, next Neumann value (4 copies) from the acceleration row
    corners = 8 * (4 + 4 + 4)
    finish = nt * (corners + 4 + 8 + 20 + 128 + 54 * 72 + 54 * 4 + 20)
    finish1 = finish + nt * (54 * 4 + 4)  # + partial terms of the next step
    finish2 = nt * (corners + 4 + 8 + 20 + 3 * 54 * 4 + 20)  # terms from partials and factors
    near = p3 * (4 + 1 + 8) + n3 * (4 + 4 + 4 + 4 + 4 + 4)
    nwrite = nt * 20
    face = pf * 76 + nt * (8 + 4) + finish
    # the split stencil: the corrected cells (list index, p^t, p^{t-1}, the correction, p^{t+1}) and
    # the rest of the grid (as the whole stencil without the corrected cells)
    stencil_corr = n3 * (4 + 12 + 4)
    stencil_bulk = 12 * (m ** 3 - n3) + 4 * 6 * m * m + m ** 3 // 8
    return {"stencil": stencil, "conv": conv, "conv2": conv2, "fix": fix, "finish": finish, "finish1": finish1,
            "finish2": finish2, "near": near, "nwrite": nwrite, "face": face, "stencil_corr": stencil_corr,
            "stencil_bulk": stencil_bulk}


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


def config_of(wl):
    """The workload's config dict, printed alike by both arms."""
    sc = wl.scene
    return {"workload": wl.name, "res": wl.res, "triangles": int(len(wl.tris)),
            "time_steps_per_bench_step": wl.total_steps if wl.whole_run else "one motion frame (~%d)" %
            round(wl.total_steps / len(wl.ranges)),
            "motion_frames_per_bench_step": len(wl.ranges) if wl.whole_run else 1,
            "bench_step": ("the whole %d-step run on a fresh handle (set_mesh untimed, then every frame's "
                           "update_mesh and steps)" % sc.steps) if wl.whole_run and wl.moving else
                          ("the whole %d-step run on a fresh handle (set_mesh untimed)" % sc.steps)
                          if wl.whole_run else "one motion frame of a continuing run: update_mesh + its steps",
            "l2": "flushed (256 MiB write) before each timed benchmark step",
            "precision": "fp32 grids, fp16+scale weights (the reference's scheme)"}


# ---------------------------------------------------------------- our arm -------------
def run_ours(args, ws, rank, local):
    import torch

    from pppm_b200 import Solver

    W, K = args.warmup, args.steps
    wl = Workload(args.workload, None if args.workload != "large" else W + K + 1)
    sc = wl.scene
    dev = torch.device("cuda", local)
    # one non-default stream for the solver, the L2 flush and every timing event (with the
    # default stream the solver would create its own, which those events would not see)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    acc_dev = torch.from_numpy(wl.acc).to(dev)
    verts_dev = [torch.from_numpy(v).to(dev) for v in wl.verts]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    nt = len(wl.tris)
    cells = float(wl.res) ** 3

    def new_solver(opts=None, precision="fp32", on_stream=True, weights="ref32"):
        s = Solver(wl.res, sc.h, sc.dt, sc.min_pos, device=local, stream=stream.cuda_stream if on_stream else None,
                   precision=precision, weights=weights)
        for k, v in (opts or {}).items():
            s.set_option(k, v)
        s.set_mesh(wl.verts[0], wl.tris)
        s.add_listener(*wl.listener)
        return s

    # face-stage autotuner on the first frame's mesh (set-up, untimed): one or two steps per pass
    # over the face pairs and over the grid-cache records, block size of the face kernels
    s0 = new_solver()
    if args.profile_frame is not None:
        p_, t_, m_ = (int(x) for x in args.options.split(","))
        tune, opts = None, {"conv_pairs": p_, "face_threads": t_, "terms_pairs": m_}
    else:
        tune = s0.autotune(reps=20)
        opts = {"conv_pairs": tune["best"][0], "face_threads": tune["best"][1], "terms_pairs": tune["terms_pairs"]}

    if args.profile_frame is not None:
        # the frames before the profiled one run as usual; the profiled frame is bracketed by an
        # NVTX range so that a profiler can take exactly its launches
        s = new_solver(opts)
        f_prof = min(args.profile_frame, len(wl.ranges) - 1)
        for f in range(f_prof):
            a, b = wl.ranges[f]
            if f > 0 and wl.moving:
                s.update_mesh(verts_dev[f])
            s.step(acc_dev[a:b])
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("profile_frame")
        a, b = wl.ranges[f_prof]
        if f_prof > 0 and wl.moving:
            s.update_mesh(verts_dev[f_prof])
        s.step(acc_dev[a:b])
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        s.close()
        s0.close()
        return None

    def frames(s, fr, events=None):
        for f in fr:
            a, b = wl.ranges[f]
            if f > 0 and wl.moving:
                if events is not None:
                    events[f][0].record(stream)
                s.update_mesh(verts_dev[f])
                if events is not None:
                    events[f][1].record(stream)
            s.step(acc_dev[a:b])

    clocks = ClockSampler(local)
    total_ms = upd_ms = 0.0
    steps = 0
    launches = 0
    series_last = None
    if wl.whole_run:
        all_frames = range(len(wl.ranges))
        for _ in range(W):
            s = new_solver(opts)
            frames(s, all_frames)
            s.close()
        torch.cuda.synchronize()
        clocks.start()
        barrier(ws)
        for r in range(K):
            s = new_solver(opts)  # set_mesh of frame 0: the one-off set-up, untimed
            launches0 = s.launch_count()
            ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in wl.ranges]
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            frames(s, all_frames, ev)
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            upd_ms += sum(ev[f][0].elapsed_time(ev[f][1]) for f in range(1, len(wl.ranges))) if wl.moving else 0.0
            steps += wl.total_steps
            launches += s.launch_count() - launches0
            if r == K - 1:
                series_last = s.listeners()[:, 0]
            s.close()
        barrier(ws)
    else:
        s = s0
        frames(s, range(0, W + 1))  # frame 0 = the set_mesh frame, then W warm-up frames
        torch.cuda.synchronize()
        launches0 = s.launch_count()
        clocks.start()
        barrier(ws)
        for f in range(W + 1, W + K + 1):
            flush.zero_()
            e0, em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a, b = wl.ranges[f]
            e0.record(stream)
            s.update_mesh(verts_dev[f])
            em.record(stream)
            s.step(acc_dev[a:b])
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            upd_ms += e0.elapsed_time(em)
            steps += b - a
        barrier(ws)
        launches = s.launch_count() - launches0
    clk = clocks.stop()
    t_max = max_over_ranks(ws, total_ms)
    value = cells * steps * ws / (t_max * 1e-3) / 1e9
    n_upd = K * (len(wl.ranges) - 1) if wl.whole_run else K
    us_update = upd_ms * 1e3 / max(n_upd, 1)
    us_per_step = (total_ms - upd_ms) * 1e3 / steps

    # per-kernel table over the frames of one benchmark step: launches of each kind and their
    # algorithmic bytes from a measurement-mode run (its per-kind launch counts, each frame's mesh
    # counts), durations from pppm_time_kernels (each kind's launches back to back in one recorded
    # graph, no event between them) at eight frames spread over the run
    sp = new_solver(opts) if wl.whole_run else s0
    sp.enable_timing(True)
    kind_bytes = {}
    prof_frames = list(range(len(wl.ranges))) if wl.whole_run else [W + K + 1]
    sampled = set(prof_frames[:: max(1, len(prof_frames) // 8)])
    dur = {}
    prev = {}
    for f in prof_frames:
        a, b = wl.ranges[f]
        if f > 0 and wl.moving:
            sp.update_mesh(verts_dev[f])
        counts = [int(x) for x in sp.dump("counts")]
        if f in sampled:
            for k, us in sp.time_kernels(20).items():
                dur.setdefault(k, []).append(us)
        sp.step(acc_dev[a:b])
        prof = sp.kernel_profile()
        alg = algorithmic_bytes(counts, wl.res, nt)
        for k, (us, n) in prof.items():
            dn = n - prev.get(k, 0)
            kind_bytes[k] = kind_bytes.get(k, 0.0) + dn * alg.get(k, 0)
            prev[k] = n
    prof = sp.kernel_profile()
    sp.enable_timing(False)
    counts_last = [int(x) for x in sp.dump("counts")]
    if wl.whole_run:
        sp.close()
    peak, peak_kind = measured_peak()
    prof.pop("empty", None)
    prof.pop("nwrite", None)  # a 20-byte-per-triangle copy at the start of each call
    per = {k: statistics.mean(dur[k]) for k in prof if k in dur}
    total_us = sum(per[k] * prof[k][1] for k in per)
    kernels = {}
    for k in sorted(per, key=lambda k: -per[k] * prof[k][1]):
        n = prof[k][1]
        b = kind_bytes.get(k, 0.0) / n
        kernels[k] = {"launches": n, "us_per_launch": round(per[k], 3), "share": round(per[k] * n / total_us, 4),
                      "algorithmic_bytes_per_launch": int(b), "gb_per_s": round(b / (per[k] * 1e-6) / 1e9, 1),
                      "frac": round(b / (per[k] * 1e-6) / 1e9 / peak, 4)}
    top = next(iter(kernels))
    traffic = load_traffic(args.workload).get(top)
    prof = {k: (per[k], prof[k][1]) for k in per}
    main_path = [k for k in ("stencil", "stencil_corr", "finish", "finish1", "finish2", "near") if k in kernels]
    path_bytes = sum(kind_bytes.get(k, 0.0) for k in main_path)
    path_us = sum(prof[k][0] * prof[k][1] for k in main_path)

    # end-to-end through the public API from pinned host buffers: vertices and accelerations
    # copied in and the listener samples read back every frame
    e2e = None
    if not args.no_e2e:
        acc_pin = torch.from_numpy(wl.acc).pin_memory()
        verts_pin = [torch.from_numpy(v).pin_memory() for v in wl.verts]

        def run_e2e(s, fr):
            h2d = d2h = n = 0
            for f in fr:
                a, b = wl.ranges[f]
                if f > 0 and wl.moving:
                    s.update_mesh(verts_pin[f])
                    h2d += verts_pin[f].numel() * 4
                s.step(acc_pin[a:b])
                h2d += (b - a) * nt * 4
                d2h += s.listeners(first=a, count=b - a).nbytes
                n += b - a
            return h2d, d2h, n

        te, h2d, d2h, steps2 = 0.0, 0, 0, 0
        if wl.whole_run:
            for r in range(W + K):
                s2 = new_solver(opts)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                x = run_e2e(s2, range(len(wl.ranges)))
                torch.cuda.synchronize()
                if r >= W:
                    te += time.perf_counter() - t0
                    h2d, d2h, steps2 = h2d + x[0], d2h + x[1], steps2 + x[2]
                s2.close()
        else:
            s2 = new_solver(opts)
            run_e2e(s2, range(0, W + 1))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            h2d, d2h, steps2 = run_e2e(s2, range(W + 1, W + K + 1))
            torch.cuda.synchronize()
            te = time.perf_counter() - t0
            s2.close()
        te = max_over_ranks(ws, te)
        e2e = {"value": round(cells * steps2 * ws / te / 1e9, 4), "unit": "Gcell-steps/s",
               "h2d_bytes_per_step": h2d // K, "d2h_bytes_per_step": d2h // K}

    # error of the timed FP32 run against the FP64 scheme of the same library on the GPU, over the
    # same steps (outside the timed region)
    fp64_err = None
    if not args.no_fp64_check:
        if wl.whole_run:
            got = series_last.astype(np.float64)
            fr = range(len(wl.ranges))
        else:
            got = s0.listeners(0, wl.ranges[W + K + 1][1])[:, 0].astype(np.float64)
            fr = range(0, W + K + 2)
        s64 = new_solver(precision="fp64")
        frames(s64, fr)
        ref = s64.listeners(0, len(got))[:, 0].astype(np.float64)
        s64.close()
        den = float(np.linalg.norm(ref))
        fp64_err = {"rel_l2": float(np.linalg.norm(got - ref) / den) if den > 0 else None, "time_steps": int(len(got)),
                    "reference": "the same steps in the FP64 scheme (PPPM_PRECISION_FP64) on the GPU"}
        if wl.moving and wl.whole_run:
            # PPPM_WEIGHTS_FP64 (singular face integrals in FP64): its refresh cost beside the default
            # weights over the first 17 frames, and its listener error against the FP64 scheme
            nfr = min(17, len(wl.ranges))
            cost = {}
            for wname in ("ref32", "fp64"):
                sw = new_solver(opts, weights=wname)
                upd = []
                for f in range(nfr):
                    a, b = wl.ranges[f]
                    if f:
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        sw.update_mesh(verts_dev[f])
                        e1.record(stream)
                        e1.synchronize()
                        upd.append(e0.elapsed_time(e1) * 1e3)
                    sw.step(acc_dev[a:b])
                n = wl.ranges[nfr - 1][1]
                sv = sw.listeners(0, n)[:, 0].astype(np.float64)
                sw.close()
                d0 = float(np.linalg.norm(ref[:n]))
                cost[wname] = {"update_mesh_us": round(statistics.median(upd), 1),
                               "rel_l2_vs_fp64": float(np.linalg.norm(sv - ref[:n]) / d0) if d0 > 0 else None}
            fp64_err["weights_fp64"] = {"frames": nfr, "time_steps": int(wl.ranges[nfr - 1][1]), **{
                "update_mesh_us_" + k: v["update_mesh_us"] for k, v in cost.items()}, **{
                "rel_l2_vs_fp64_" + k: v["rel_l2_vs_fp64"] for k, v in cost.items()}}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl)

    s0.close()
    cfg = config_of(wl)
    cfg.update({"parallelism": "replicas x%d" % ws, "n3_cells": int(counts_last[0]),
                "pairs_3x3x3": int(counts_last[1]), "face_pairs": int(counts_last[4])})
    line = {
        "metric": "Gcell-steps/s, %s (time step + motion-frame refresh)" % wl.name,
        "value": round(value, 4), "unit": "Gcell-steps/s", "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": round(t_max / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded meshes, trajectories and accelerations)", "config": cfg,
        "roofline": {"bound": "hbm", "kernel": top, "achieved": kernels[top]["gb_per_s"], "peak": peak,
                     "unit": "GB/s", "frac": kernels[top]["frac"], "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes": kernels[top]["algorithmic_bytes_per_launch"],
                     "kernel_launch_us": kernels[top]["us_per_launch"],
                     "how": "kernel with the largest share of time (launches x duration) over one benchmark "
                            "step's frames; achieved = its algorithmic bytes per launch / its duration per launch "
                            "(pppm_time_kernels: 20 back-to-back launches in one recorded graph, events around "
                            "the graph, at %d frames spread over the run)" % len(sampled),
                     "kernels": kernels,
                     "main_path": {"kernels": main_path, "achieved": round(path_bytes / (path_us * 1e-6) / 1e9, 1),
                                   "frac": round(path_bytes / (path_us * 1e-6) / 1e9 / peak, 4)},
                     "autotune": {"best": {"two_steps_per_pass": bool(opts["conv_pairs"]),
                                           "threads": opts["face_threads"],
                                           "terms_two_steps_per_pass": bool(opts["terms_pairs"])},
                                  "step_us_by_config": {"%s/%d/%s" % (("single", "pairs")[p], t,
                                                                      "terms2" if m else "terms1"): round(u, 2)
                                                        for (p, t, m), u in (tune["step_us"] or {}).items()}},
                     "update_mesh_us": round(us_update, 1), "time_step_us": round(us_per_step, 2)},
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
        alg = algorithmic_bytes(counts, sp["res"], len(sp["tris"]))
        job_bytes += (alg["stencil"] + alg["face"] + alg["near"]) * sp["steps"]
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


# ---------------------------------------------------------------- large scene batched --
LARGE_BATCH = 4
LARGE_BATCH_NAME = ("4 large moving scenes (res 128, two 20480-tri perturbed icospheres each, seeds 23, 123, 223, "
                    "323), 1 kHz motion frames, batched")


def run_large_batch(args, ws, rank, local):
    """The large moving scene batched x4 with different seeds: one benchmark step = one motion
    frame of all four scenes (each scene's update_mesh, then one pppm_batch_run over the frame's
    steps), against the same frames stepped scene by scene (update_mesh + pppm_step per scene)."""
    import torch

    from pppm_b200 import Batch, Solver

    W, K = args.warmup, args.steps
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    nfr = 2 * (W + K) + 2
    scs = [scenes.LargeScene(seed=23 + 100 * i) for i in range(LARGE_BATCH)]
    ranges = [scenes.frame_ranges(sc, nfr) for sc in scs]
    accs = [torch.from_numpy(sc.acc(0, r[-1][1])).to(dev) for sc, r in zip(scs, ranges)]
    verts = [[torch.from_numpy(sc.frame_verts(f)).to(dev) for f in range(nfr + 1)] for sc in scs]

    def make():
        out = []
        for sc in scs:
            s = Solver(sc.res, sc.h, sc.dt, sc.min_pos, device=local, stream=stream.cuda_stream)
            s.set_mesh(sc.frame_verts(0), sc.tris)
            s.add_listener(*sc.listener)
            out.append(s)
        return out

    def frame_batched(ss, b, f):
        rows = []
        for i, s in enumerate(ss):
            if f:
                s.update_mesh(verts[i][f])
            a, e = ranges[i][f]
            rows.append(accs[i][a:e])
        b.run(rows)

    def frame_sequential(ss, f):
        for i, s in enumerate(ss):
            if f:
                s.update_mesh(verts[i][f])
            a, e = ranges[i][f]
            s.step(accs[i][a:e])

    def timed(run, frames_timed, clocks=None):
        ms, steps = 0.0, 0
        if clocks:
            clocks.start()
        barrier(ws)
        for f in frames_timed:
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run(f)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            steps += sum(r[f][1] - r[f][0] for r in ranges)
        barrier(ws)
        return max_over_ranks(ws, ms), steps, (clocks.stop() if clocks else None)

    bat = make()
    b = Batch(bat)
    for f in range(0, W + 1):
        frame_batched(bat, b, f)
    launches0 = sum(s.launch_count() for s in bat)
    ms_b, steps_b, clk = timed(lambda f: frame_batched(bat, b, f), range(W + 1, W + K + 1), ClockSampler(local))
    launches = sum(s.launch_count() for s in bat) - launches0
    series_b = [s.listeners() for s in bat]
    b.close()
    for s in bat:
        s.close()
    seq = make()
    for f in range(0, W + 1):
        frame_sequential(seq, f)
    ms_s, steps_s, _ = timed(lambda f: frame_sequential(seq, f), range(W + 1, W + K + 1))
    same = all(np.array_equal(a, s.listeners()) for a, s in zip(series_b, seq))
    for s in seq:
        s.close()
    cells = float(scs[0].res) ** 3
    value = cells * steps_b * ws / (ms_b * 1e-3) / 1e9
    seq_value = cells * steps_s * ws / (ms_s * 1e-3) / 1e9
    return {
        "metric": "Gcell-steps/s, %s" % LARGE_BATCH_NAME, "value": round(value, 4), "unit": "Gcell-steps/s",
        "n_gpus": ws, "steps": K, "warmup": W, "ms_per_step": round(ms_b / K, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded meshes, trajectories "
        "and accelerations)",
        "config": {"workload": LARGE_BATCH_NAME, "scenes": LARGE_BATCH, "res": scs[0].res,
                   "triangles_per_scene": int(len(scs[0].tris)),
                   "bench_step": "one motion frame of all scenes: update_mesh per scene + one pppm_batch_run",
                   "l2": "flushed (256 MiB write) before each timed frame", "parallelism": "replicas x%d" % ws},
        "sequential": {"value": round(seq_value, 4), "unit": "Gcell-steps/s",
                       "how": "the same frames, update_mesh + pppm_step scene by scene"},
        "batched_over_sequential": round(value / seq_value, 3), "listeners_bit_identical": bool(same),
        "cpu_baseline": None, "e2e": None, "gpu_launches": int(launches), "clocks": clk,
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


ADJM_NAME = ("two moving icospheres (2 x 20480 tris), res 128, loss ||s - s_target||^2, gradient w.r.t. "
             "every acceleration, motion checkpoints every 200 steps (FP32)")


def run_adjoint_moving(args, ws, rank, local):
    """Cost of the gradient of a moving run against the run itself: one benchmark step = the
    forward run of the large scene (update_mesh per 1 kHz motion frame, a motion checkpoint every
    200 steps, device-resident accelerations) and the backward (each frame's tables rebuilt from
    its segment's checkpoint, the adjoint sweep), both through autograd.moving_listener_signal;
    beside it the same run without checkpoints."""
    import torch

    from pppm_b200 import Solver
    from pppm_b200.autograd import moving_listener_signal

    W, K = args.warmup, args.steps
    sc = scenes.LargeScene()
    nsteps = min(args.adjoint_steps, sc.steps)
    nframes = sc.frame_of_step(nsteps - 1) + 1
    ranges = scenes.frame_ranges(sc, nframes - 1)
    ranges[-1] = (ranges[-1][0], nsteps)
    frames = [(a, sc.frame_verts(f)) for f, (a, b) in enumerate(ranges)]
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    s = Solver(sc.res, sc.h, sc.dt, sc.min_pos, device=local, stream=stream.cuda_stream)
    s.set_mesh(frames[0][1], sc.tris)
    s.add_listener(*sc.listener)
    acc = torch.from_numpy(sc.acc(0, nsteps)).to(dev).requires_grad_(True)
    target = torch.zeros((nsteps, 1), dtype=torch.float32, device=dev)
    t0 = s.t
    peak = {"checkpoints": 0, "bytes": 0}

    def restart():
        s.reset_fields()
        s.rewind_listeners()
        s.t = t0

    def plain():
        restart()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for f, (a, b) in enumerate(ranges):
            if f:
                s.update_mesh(frames[f][1])
            s.step(acc.detach()[a:b])
        e1.record(stream)
        s.update_mesh(frames[0][1])
        return e0, e1

    def forward_backward():
        restart()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(stream)
        sig = moving_listener_signal(s, acc, frames, checkpoint_steps=200)
        e[1].record(stream)
        n, b = s.checkpoint_info()
        peak["checkpoints"], peak["bytes"] = max(peak["checkpoints"], n), max(peak["bytes"], b)
        loss = ((sig - target) ** 2).sum()
        e[2].record(stream)
        (grad,) = torch.autograd.grad(loss, acc)
        e[3].record(stream)
        return e, grad

    for _ in range(W):
        plain()
        forward_backward()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    launches0 = s.launch_count()
    p_ms = f_ms = b_ms = 0.0
    for _ in range(K):
        p0, p1 = plain()
        e, grad = forward_backward()
        e[3].synchronize()
        p_ms += p0.elapsed_time(p1)
        f_ms += e[0].elapsed_time(e[1])
        b_ms += e[2].elapsed_time(e[3])
    barrier(ws)
    clk = clocks.stop()
    launches = s.launch_count() - launches0
    p_ms, f_ms, b_ms = max_over_ranks(ws, p_ms), max_over_ranks(ws, f_ms), max_over_ranks(ws, b_ms)
    finite = bool(torch.isfinite(grad).all().item())

    # where the backward's time goes: the reverse sweep on one frame's tables, one rebuild of
    # the transposed tables after a mesh update, one update_mesh
    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    g1 = torch.ones((200, 1), dtype=torch.float32, device=dev)
    s.adjoint(g1[:1], fresh=True)  # tables of the current frame
    sweep_ms = timed(lambda: s.adjoint(g1, fresh=True))
    upd_ms = timed(lambda: s.update_mesh(frames[1][1]))
    one_ms = timed(lambda: s.adjoint(g1[:1], fresh=True))  # rebuilds the tables, then one step
    s.close()
    cells = float(sc.res) ** 3
    return {
        "metric": "adjoint / forward cost, %s" % ADJM_NAME, "value": round(b_ms / f_ms, 4), "unit": "x forward",
        "n_gpus": ws, "steps": K, "warmup": W, "ms_per_step": round((p_ms + f_ms + b_ms) / K, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded meshes, trajectories and accelerations)",
        "config": {"workload": ADJM_NAME, "res": sc.res, "triangles": int(len(sc.tris)), "time_steps": nsteps,
                   "motion_frames": nframes, "checkpoint_steps": 200,
                   "bench_step": "plain run + forward run with checkpoints + backward",
                   "l2": "inputs (a %d MB acceleration history) larger than L2" % (nsteps * len(sc.tris) * 4 >> 20),
                   "parallelism": "replicas x%d" % ws},
        "plain_run_ms": round(p_ms / K, 2), "forward_ms": round(f_ms / K, 2), "backward_ms": round(b_ms / K, 2),
        "checkpoint_overhead": round(f_ms / p_ms - 1, 4), "backward_vs_plain_run": round(b_ms / p_ms, 4),
        "checkpoints": peak["checkpoints"], "checkpoint_bytes": int(peak["bytes"]),
        "adjoint_us_per_step_fixed_tables": round(sweep_ms * 1e3 / 200, 2),
        "forward_us_per_step_plain": round(p_ms * 1e3 / (K * nsteps), 2),
        "table_rebuild_ms": round(one_ms - sweep_ms / 200, 3), "update_mesh_ms": round(upd_ms, 3),
        "plain_gcell_steps_per_s": round(cells * nsteps * K * ws / (p_ms * 1e-3) / 1e9, 3),
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


def cpu_baseline(wl, budget_s=10.0):
    """The CPU restatement (oracle/) on the host cores over a bounded sample of the same workload
    (set_mesh untimed): motion frames from frame 1 on (update_mesh + the frame's steps) until about
    budget_s seconds have passed; the static run in chunks of 100 steps likewise; the large scene's
    first frame with its steps sampled (a whole frame takes about a minute on the host)."""
    from oracle.oracle import Oracle, oracle_threads

    sc = wl.scene
    o = Oracle(wl.res, sc.h, sc.dt, sc.min_pos)
    o.set_mesh(wl.verts[0], wl.tris)
    elapsed, steps, nframes = 0.0, 0, 0
    if wl.kind == "large":
        a, b = wl.ranges[1]
        n = min(b - a, CPU_SAMPLE_STEPS)
        t0 = time.perf_counter()
        o.update_mesh(wl.verts[1])
        t1 = time.perf_counter()
        o.step(wl.acc[a:a + n], listeners=[wl.listener])
        t2 = time.perf_counter()
        elapsed, steps = (t1 - t0) + (t2 - t1) * (b - a) / n, b - a
        sample = ("frame 1 of the same workload: update_mesh and the first %d of its %d time steps timed, the "
                  "steps extrapolated to the frame; C restatement with OpenMP" % (n, b - a))
    elif wl.moving:
        for f in range(1, len(wl.ranges)):
            a, b = wl.ranges[f]
            t0 = time.perf_counter()
            o.update_mesh(wl.verts[f])
            o.step(wl.acc[a:b], listeners=[wl.listener])
            elapsed += time.perf_counter() - t0
            steps += b - a
            nframes += 1
            if elapsed >= budget_s:
                break
        sample = ("motion frames 1-%d of the same run (update_mesh + %d time steps), C restatement with "
                  "OpenMP" % (nframes, steps))
    else:
        while steps < wl.total_steps and elapsed < budget_s:
            n = min(100, wl.total_steps - steps)
            t0 = time.perf_counter()
            o.step(wl.acc[steps:steps + n], listeners=[wl.listener])
            elapsed += time.perf_counter() - t0
            steps += n
        sample = "the first %d time steps of the same run, C restatement with OpenMP" % steps
    o.close()
    return {"value": round(float(wl.res) ** 3 * steps / elapsed / 1e9, 5), "unit": "Gcell-steps/s",
            "cores": oracle_threads(), "kind": "port", "sample": sample}


# ---------------------------------------------------------------- reference arm -------
def own_library_mapped():
    """Paths of this repository's native library mapped into this process (must be none in the
    reference arm)."""
    try:
        return sorted({line.split()[-1] for line in open("/proc/self/maps") if "libpppm_b200" in line})
    except OSError:
        return []


def run_reference(args, ws, rank, local):
    if rank != 0:
        return None
    W, K = args.warmup, args.steps
    if args.workload == "batch":
        return run_reference_batch(args)
    if args.workload == "adjoint":
        return {"impl": "reference", "metric": "adjoint / forward cost, %s" % ADJ_NAME,
                "unavailable": "the reference has no adjoint"}
    if args.workload == "adjoint-moving":
        return {"impl": "reference", "metric": "adjoint / forward cost, %s" % ADJM_NAME,
                "unavailable": "the reference has no adjoint"}
    if args.workload == "large-batch":
        return run_reference_large_batch(args)
    wl = Workload(args.workload, None if args.workload != "large" else W + K + 1)
    sc = wl.scene
    from oracle import oracle as O

    ndebug = None
    if O.reference_available():
        import torch

        acc_dev = torch.from_numpy(wl.acc).cuda()
        nt = len(wl.tris)
        ptr0 = acc_dev.data_ptr()

        def new_ref(nd):
            r = O.Reference(wl.res, sc.h, sc.dt, sc.min_pos, ndebug=nd)
            r.set_mesh(wl.verts[0], wl.tris)
            return r

        def frame(r, f):
            a, b = wl.ranges[f]
            if f > 0 and wl.moving:
                r.update_mesh(wl.verts[f])
            r.run_device(ptr0 + a * nt * 4, b - a, wl.listener)
            return b - a

        def timed_run(nd, W=W, K=K):
            """W warm-up and K timed benchmark steps of the reference build (nd: the -DNDEBUG
            build); whole-run workloads on a fresh solver per benchmark step (set_mesh untimed)."""
            if wl.moving:
                r = new_ref(nd)
                for v in wl.verts[1:]:
                    r.check_mesh(v)  # validate the whole trajectory against the reference capacities
                r.close()
            dt, steps = 0.0, 0
            if wl.whole_run:
                for i in range(W + K):
                    r = new_ref(nd)
                    r.set_checks(False)
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    n = sum(frame(r, f) for f in range(len(wl.ranges)))
                    torch.cuda.synchronize()
                    if i >= W:
                        dt += time.perf_counter() - t0
                        steps += n
                    r.close()
            else:
                r = new_ref(nd)
                r.set_checks(False)
                for f in range(0, W + 1):
                    frame(r, f)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                steps = sum(frame(r, f) for f in range(W + 1, W + K + 1))
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                r.close()
            return float(wl.res) ** 3 * steps / dt / 1e9

        value = timed_run(False)
        if O.reference_available(ndebug=True):
            nd_k = min(K, 5)
            ndebug = {"value": round(timed_run(True, 1, nd_k), 5), "unit": "Gcell-steps/s", "steps": nd_k,
                      "build": "the same reference sources built with -DNDEBUG (no device sync after every launch)"}
        kind, cores, sample = "reference", 1, ("reference CUDA solver built from source (oracle/_ref, upstream "
                                               "flags: device sync after every launch) driven by one host thread, "
                                               "%d benchmark steps" % K)
    else:
        from oracle.oracle import Oracle, oracle_threads

        o = Oracle(wl.res, sc.h, sc.dt, sc.min_pos)
        o.set_mesh(wl.verts[0], wl.tris)
        t0 = time.perf_counter()
        steps = 0
        for f in range(1, min(len(wl.ranges) - 1, 3) + 1):
            a, b = wl.ranges[f]
            if wl.moving:
                o.update_mesh(wl.verts[f])
            o.step(wl.acc[a:b], listeners=[wl.listener])
            steps += b - a
        dt = time.perf_counter() - t0
        value = float(wl.res) ** 3 * steps / dt / 1e9
        kind, cores, sample = "port", oracle_threads(), "CPU restatement, motion frames 1-3"
    mapped = own_library_mapped()
    if mapped:
        raise RuntimeError("reference arm has this repository's library mapped: %s" % mapped)
    cfg = config_of(wl)
    cfg["parallelism"] = "one GPU (rank 0)"
    return {"impl": "reference", "metric": "Gcell-steps/s, %s (time step + motion-frame refresh)" % wl.name,
            "value": round(value, 5), "unit": "Gcell-steps/s", "n_gpus": ws, "steps": K, "warmup": W,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded meshes, trajectories and accelerations)", "config": cfg,
            "cpu_baseline": {"value": round(value, 5), "unit": "Gcell-steps/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 5), "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_ndebug": ndebug, "native_libraries_of_this_repo_mapped": mapped}


def run_reference_large_batch(args):
    """The reference solver on the four large scenes, scene by scene within each motion frame
    (update_mesh + the frame's steps), over the same timed frames as the batched arm."""
    from oracle import oracle as O

    line = {"impl": "reference", "metric": "Gcell-steps/s, %s" % LARGE_BATCH_NAME, "unit": "Gcell-steps/s"}
    if not O.reference_available():
        line["unavailable"] = "reference solver not built (oracle/_ref)"
        return line
    import torch

    W, K = args.warmup, args.steps
    nfr = W + K + 1
    scs = [scenes.LargeScene(seed=23 + 100 * i) for i in range(LARGE_BATCH)]
    ranges = [scenes.frame_ranges(sc, nfr) for sc in scs]
    accs = [torch.from_numpy(sc.acc(0, r[-1][1])).cuda() for sc, r in zip(scs, ranges)]
    refs = []
    for sc in scs:
        r = O.Reference(sc.res, sc.h, sc.dt, sc.min_pos)
        r.set_mesh(sc.frame_verts(0), sc.tris)
        refs.append(r)
    try:
        dt, steps = 0.0, 0
        for f in range(0, W + K + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            n = 0
            for i, (sc, r) in enumerate(zip(scs, refs)):
                if f:
                    r.update_mesh(sc.frame_verts(f))
                a, e = ranges[i][f]
                r.run_device(accs[i].data_ptr() + a * len(sc.tris) * 4, e - a, sc.listener)
                n += e - a
            torch.cuda.synchronize()
            if f > W:
                dt += time.perf_counter() - t0
                steps += n
    finally:
        for r in refs:
            r.close()
    value = float(scs[0].res) ** 3 * steps / dt / 1e9
    mapped = own_library_mapped()
    if mapped:
        raise RuntimeError("reference arm has this repository's library mapped: %s" % mapped)
    line.update({"value": round(value, 5), "n_gpus": 1, "steps": K, "warmup": W, "higher_is_better": True,
                 "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                 "data": "synthetic (seeded meshes, trajectories and accelerations)",
                 "config": {"workload": LARGE_BATCH_NAME, "scenes": LARGE_BATCH, "res": scs[0].res,
                            "triangles_per_scene": int(len(scs[0].tris)),
                            "bench_step": "one motion frame of all scenes, scene by scene"},
                 "cpu_baseline": {"value": round(value, 5), "unit": "Gcell-steps/s", "cores": 1, "kind": "reference",
                                  "sample": "reference CUDA solver built from source, the four scenes one after "
                                            "another within each frame, %d frames" % K},
                 "e2e": {"value": round(value, 5), "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    return line


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
    mapped = own_library_mapped()
    if mapped:
        raise RuntimeError("reference arm has this repository's library mapped: %s" % mapped)
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


def relaunch_under_torchrun(n):
    """bench.py --gpus N outside torchrun: start N ranks of this same command on this node and
    return their exit status (rank 0 prints the line)."""
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.summarize_launches:
        summarize_launches(args.summarize_launches)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_under_torchrun(args.gpus))
    ws, rank, local = dist_setup()
    if ws != args.gpus and rank == 0:
        print("warning: --gpus %d but %d ranks" % (args.gpus, ws), file=sys.stderr)
    if args.impl == "reference":
        line = run_reference(args, ws, rank, local)
    elif args.workload == "batch":
        line = run_batch(args, ws, rank, local)
    elif args.workload == "adjoint":
        line = run_adjoint(args, ws, rank, local)
    elif args.workload == "adjoint-moving":
        line = run_adjoint_moving(args, ws, rank, local)
    elif args.workload == "large-batch":
        line = run_large_batch(args, ws, rank, local)
    else:
        line = run_ours(args, ws, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    elif args.profile_frame is not None and rank == 0:
        print("profiled frame %d" % args.profile_frame, flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
