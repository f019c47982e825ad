#!/usr/bin/env python
"""Benchmark of the full-field DIC solve on B200: grid points per second.

Workload (one "step" = one full-field solve of one deformed frame against a
cached reference, i.e. frames 2+ of a fixed-reference batch): 4096 x 4096
uint8 Gaussian-blob speckle (0.02 blobs/px^2, sigma U[1.5, 3], amplitude
U[180, 220], background 30), deformed by u = 0.005 x + 2 sin(2 pi y / 256),
v = -0.003 y + 1.5 sin(2 pi x / 384) with N(0, 2^2) noise; step 4, subset 31,
strain window 31, 4x4 bicubic, whole image as ROI (1,048,576 grid nodes).

  value     grid points written per second, inputs resident in HBM
            (semper_b200_run_device), device time = CUDA events on the
            engine's stream, max over ranks;
  e2e       the same metric through the public C ABI (semper_run) with the
            frame in pinned host memory: host->device frame copy and
            device->host read of the packed points inside the timed region;
  roofline  the IC-GN solve kernel (Path A launch): algorithmic FP32 FLOPs
            (117 per subset pixel per iteration for the 4x4 kernel) over its
            CUDA-event duration, against the FP32 CUDA-core peak;
  cpu_baseline
            the CPU restatement of the reference path (OpenMP, all host
            threads) on a bounded ROI sample of the same frame pair.

With --impl reference, rank 0 times that CPU implementation alone on the same
metric and configuration (a bounded ROI sample per step) and prints its line.
Multi-GPU (torchrun): every rank solves its own independent frame pair (its
own speckle seed), no data-path collective; value = all ranks' points / the
slowest rank's time ("weak" scaling).
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "semper-dic-engine_b200"))

FLOP_PER_PIXEL_ITER = {False: 117, True: 181}  # 4x4 bicubic / 6x6 Keys, per subset pixel per IC-GN iteration
METRIC = "DIC grid points/sec on 1 B200 at <=0.01 px vs FP64; learned vs lattice seeding"
WORKLOADS = {
    "cfg1": ("cfg1: 4096x4096 uint8 speckle, u=0.005x+2sin(2pi y/256), v=-0.003y+1.5sin(2pi x/384), "
             "noise sigma 2, step 4, subset 31, strain window 31, 4x4 bicubic, fixed reference (frames 2+)"),
    "cfg4-plain": ("target settings: 4096x4096 uint8 speckle under the cfg1 field, noise sigma 2, step 8, "
                   "subset 41, strain window 41, 4x4 bicubic, fixed reference (frames 2+)"),
    "cfg4-large": ("large deformation, lattice seeding from the device global-motion estimate: 4096x4096 uint8 "
                   "speckle under a rotation ~U[0,180) deg about the centre, a translation up to 60 px and a "
                   "smooth random field of 5 px amplitude (Gaussian covariance, length 300 px), noise sigma 2; "
                   "step 8, subset 41, strain window 41, 4x4 bicubic; rect the centred 2744x2744 square that "
                   "stays inside the deformed frame at any rotation; fixed reference (frames 2+)"),
    "cfg4-learned": ("large deformation, learned seeding: the cfg4-large pair (4096x4096, rotation ~U[0,180) deg, "
                     "translation up to 60 px, 5 px random field, noise sigma 2; step 8, subset 41, strain window "
                     "41, 4x4 bicubic, the centred 2744x2744 rect) seeded by the proposal network with its shipped "
                     "weights (global model and per-anchor guesses, judged by the lattice's keep rule); fixed "
                     "reference (frames 2+)"),
}
WORKLOAD = WORKLOADS["cfg1"]


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def _peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# DRAM bytes per subset pixel-iteration of the IC-GN fast pass (the Path A
# launch), from one `ncu --set full` capture per solve setting (summaries in
# profiles/icgn_solve_cfg1.md and profiles/icgn_solve_cfg4.md): the cfg1 pair
# at 2048x2048, step 4, subset 31 read and wrote 145.3 MB over 969,920,963
# pixel-iterations; the target-settings pair at 2048x2048, step 8, subset 41
# 95.5 MB over 408,104,775. Traffic grows with the pixel-iterations, so a
# launch's traffic is this figure times the launch's own pixel-iterations.
NCU_BYTES_PER_PIXEL_ITER = {31: 145.3e6 / 969920963, 41: 95.5e6 / 408104775}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.out = out
        return False

    def summary(self):
        if self.proc is None or not getattr(self, "out", ""):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in csv.reader(io.StringIO(self.out)):
            if len(row) < 9:
                continue
            try:
                sm.append(float(row[1]))
                smax.append(float(row[2]))
            except ValueError:
                continue
            for n, v in zip(names, row[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(ref, dfm, prm, fp64=False, model=None):
    """The CPU restatement (built with the reference's compiler flags) on the
    central 1024 x 1024 ROI of the frame pair at the same settings, reference cache warm (the solve timed is the second on
    the reference), given the global model the device used (None: none).
    Returns (points, seconds, attempted)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle

    n = ref.shape[0]
    side = min(1024, n)
    x0 = (n - side) // 2
    p = [x0, x0, side, side, prm.step, prm.subset_size, prm.strain_window, prm.use_6x6_interpolator]
    o = oracle.Oracle(fp64, kind="contract" if fp64 else "reference_flags")
    o.set_reference(ref)
    o.run(dfm, p, model_h=model)  # frame 1: fills the grid scan + Hessian pool cache
    t0 = time.perf_counter()
    rc, pts, met = o.run(dfm, p, model_h=model)
    dt = time.perf_counter() - t0
    return rc, dt, int(met[0]), pts, p


def accuracy_sample(eng, ref, dfm, prm, warp, p, gm):
    """The device's field on the CPU sample's ROI against the same solve in
    FP64 (the CPU restatement in double, given the same global model) and
    against the synthetic warp's true displacement; after the timed region."""
    import semper_b200 as sb

    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle

    roi = sb.params((p[0], p[1], p[2], p[3]), p[4], p[5], p[6], six=bool(p[7]))
    model = gm["H"] if gm["locked"] else None
    eng.set_global_model(model)  # both solves seeded from the same model
    rc, pts, _ = eng.run(dfm, roi)
    eng.set_global_model(None)
    o = oracle.Oracle(True)
    o.set_reference(ref)
    orc, opts, _ = o.run(dfm, p, model_h=model)
    if rc <= 0 or orc <= 0:
        return {"note": f"no points to compare (device {rc}, FP64 {orc})"}
    key = {(float(x), float(y)): i for i, (x, y) in enumerate(opts[:, :2])}
    both = [(i, key[(float(x), float(y))]) for i, (x, y) in enumerate(pts[:, :2]) if (float(x), float(y)) in key]
    a = np.array([pts[i] for i, _ in both])
    b = np.array([opts[j] for _, j in both])
    d = np.abs(a[:, 2:4] - b[:, 2:4])
    u, v = sb.displacement(warp, pts[:, 0], pts[:, 1])
    t = np.hypot(pts[:, 2] - u, pts[:, 3] - v)
    return {"roi": [p[0], p[1], p[2], p[3]], "points_device": int(rc), "points_fp64": int(orc),
            "points_compared": len(both),
            "vs_fp64_max_px": float(d.max()), "vs_fp64_rms_px": float(np.sqrt(np.mean(d ** 2))),
            "vs_fp64_strain_max": float(np.abs(a[:, 4:7] - b[:, 4:7]).max()),
            "vs_true_field_rms_px": float(np.sqrt(np.mean(t ** 2))), "vs_true_field_max_px": float(t.max())}


def compare_seedings(ref, dfm, prm, warp):
    """The same pair seeded three ways, one run each after a warm-up run, out
    of the timed region: the proposal network, the device global-motion
    estimate, and the anchor lattice alone (the reference's AUTO_SEARCH
    without a model). Points, seeding time and error against the true field."""
    import semper_b200 as sb

    res = {}
    for mode in ("learned", "global_motion", "lattice_only"):
        eng = sb.Engine()
        eng.set_reference(ref)
        if mode == "learned":
            eng.set_proposal(sb.Proposal.trained(), True)
        if mode != "global_motion":
            eng.set_global_motion(False)
        eng.run(dfm, prm)
        rc, pts, _ = eng.run(dfm, prm)
        t, _ = eng.last_timings()
        r = {"points": int(rc), "seed_ms": round(t["seed"], 3), "total_ms": round(t["total"], 3)}
        if rc > 0:
            u, v = sb.displacement(warp, pts[:, 0], pts[:, 1])
            r["vs_true_field_rms_px"] = float(np.sqrt(np.mean((pts[:, 2] - u) ** 2 + (pts[:, 3] - v) ** 2)))
        res[mode] = r
        eng.close()
    return res


REF_SAMPLE_SIDE = 1024


def run_reference(args, rank):
    """The reference arm: the CPU restatement built with the reference's own
    compiler flags, on every host thread, on the central 1024x1024 ROI of the
    headline pair (about 62 k points a step; the full 4096x4096 frame takes
    about 25 s a step on the CPU). Its inputs come from the checker's own build
    of the speckle generator: this arm loads no library of the package."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle

    import semper_b200 as sb

    sb.use_synth_library(oracle.synth_path())
    ref, dfm, prm, _ = sb.config_pair(1)
    side = REF_SAMPLE_SIDE
    x0 = (ref.shape[0] - side) // 2
    p = [x0, x0, side, side, prm.step, prm.subset_size, prm.strain_window, 0]
    o = oracle.Oracle(False, kind="reference_flags")
    o.set_reference(ref)
    for _ in range(max(args.warmup, 1)):
        o.run(dfm, p)
    pts_total, t_total = 0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rc, _, _ = o.run(dfm, p)
        t_total += time.perf_counter() - t0
        pts_total += rc
    v = pts_total / t_total
    cores = len(os.sched_getaffinity(0))
    sample = (f"central {side}x{side} ROI ({p[2] // p[4]}^2 grid) of the cfg1 4096x4096 pair, reference cache "
              f"warm, no global model; CPU restatement built with the reference's flags (-O3 -ffast-math "
              f"-fno-finite-math-only -ffp-contract=off), OpenMP on {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": sample, "same_config": False,
                   "differs_by": "a 1024x1024 ROI of the same pair and settings instead of the whole frame"},
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def aggregate(points, ms_per_step, steps, dist=None, device="cpu"):
    """Whole-job throughput of independent replicas: every rank's points over
    the slowest rank's time (max over ranks), summed over ranks. Returns
    (points/s, slowest ms per step)."""
    import torch

    ms_t = torch.tensor([ms_per_step], device=device, dtype=torch.float64)
    pts_t = torch.tensor([points], device=device, dtype=torch.float64)
    if dist:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
        dist.all_reduce(pts_t, op=dist.ReduceOp.SUM)
    ms_max = float(ms_t.item())
    return float(pts_t.item()) / steps / (ms_max / 1000.0), ms_max


def measure_frames(args, wl, rank, world, local_rank, dist):
    """Times one workload's frames on this rank: device-resident runs (value),
    then the public C ABI from pinned host memory (e2e). Returns the pieces of
    the JSON line; the CPU-baseline and accuracy legs run on rank 0 at N=1."""
    import torch

    import semper_b200 as sb

    if wl in ("cfg4-large", "cfg4-learned"):
        ref, dfm, prm, warp, _sim = sb.large_motion_pair(args.size, pair=rank)
    else:
        ref, dfm, prm, warp = sb.config_pair(4 if wl == "cfg4-plain" else 1, size=args.size, pair=rank)
    H, W = ref.shape
    grid_nodes = (prm.rect_w // prm.step) * (prm.rect_h // prm.step)
    capacity = grid_nodes * 8

    eng = sb.Engine()
    assert eng.set_reference(ref) == 0
    net = None
    if wl == "cfg4-learned":
        net = sb.Proposal.trained()
        assert eng.set_proposal(net, True) == 0
    d_def = torch.from_numpy(dfm).cuda()
    d_out = torch.empty(capacity, dtype=torch.float32, device="cuda")

    # frame 1 on the reference: grid scan + Hessian pool built (reported apart)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc, met = eng.run_device(d_def, prm, d_out, capacity)
    first_ms = 1000 * (time.perf_counter() - t0)
    assert rc > 0, rc
    first_t, _ = eng.last_timings()

    for _ in range(args.warmup):
        rc, met = eng.run_device(d_def, prm, d_out, capacity)

    stream = torch.cuda.ExternalStream(eng.stream_handle())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    phases, counts = [], []
    pts = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            rc, met = eng.run_device(d_def, prm, d_out, capacity)
            t, c = eng.last_timings()
            phases.append(t)
            counts.append(c)
            pts += rc
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    value, ms_max = aggregate(pts, ms, args.steps, dist, "cuda")

    # e2e: public C ABI, frame in pinned host memory, points read back
    h_frame = torch.from_numpy(dfm).pin_memory()
    frame_np = h_frame.numpy()
    h_out = torch.empty(capacity, dtype=torch.float32).pin_memory().numpy()
    e2e_ms = []
    rc_e2e = 0
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        # the points stay in the caller's pinned buffer, where semper_run
        # wrote them (no copy by the Python binding inside the timed call)
        rc_e2e, _, _ = eng.run(frame_np, prm, capacity=capacity, out=h_out, copy=False)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_ms.append(1000 * dt)
    e2e_t = torch.tensor([statistics.mean(e2e_ms)], device="cuda", dtype=torch.float64)
    if dist:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = rc_e2e * world / (float(e2e_t.item()) / 1000.0)

    # roofline of the IC-GN solve kernel (Path A launch)
    six = bool(prm.use_6x6_interpolator)
    a_ms = statistics.mean(p["path_a"] for p in phases)
    a_pix = statistics.mean(c["path_a_pixel_iters"] for c in counts)
    flops = FLOP_PER_PIXEL_ITER[six] * a_pix
    achieved = flops / (a_ms / 1000.0) / 1e12
    peaks, peak_src = _peaks()
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    fp32_peak = sms * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    bpp = NCU_BYTES_PER_PIXEL_ITER.get(prm.subset_size) if not six else None
    traffic = None if bpp is None else bpp * a_pix
    gm = eng.last_global_motion()
    learned = None
    if net is not None:
        L = eng.last_learned()
        learned = {"kept": L["kept"], "network_ms": round(L["ms"], 3), "patch_pairs": L["pairs"],
                   "grid_inliers": L["inliers"], "anchors_judging": L["anchors"],
                   "model_vs_anchors_px": {"mean": round(L["err_mean_px"], 3), "max": round(L["err_max_px"], 3)}}
        if L["kept"]:
            gm = {"locked": True, "theta": float(np.arctan2(L["H"][1, 0], L["H"][0, 0])), "scale": 1.0,
                  "t": (float(L["H"][0, 2]), float(L["H"][1, 2])), "H": L["H"]}

    out = {
        "value": value, "ms_per_step": ms_max,
        "config": {"workload": WORKLOADS[wl] if args.size == 4096 else f"{WORKLOADS[wl]} [resized to {W}x{H}]",
                   "image": [W, H], "grid_nodes": grid_nodes,
                   "attempted": int(met[0]), "points_per_step": rc,
                   "parallelism": f"replicas x{world} (independent frame pairs)",
                   "l2": f"inputs larger than L2: reference planes {12 * W * H / 1e6:.0f} MB + Hessian pool "
                         f"{177 * grid_nodes / 1e6:.0f} MB + deformed planes {12 * W * H / 1e6:.0f} MB per step"},
        "frames_per_s": 1000.0 / ms_max * world,
        "attempted_points_per_s": int(met[0]) * world / (ms_max / 1000.0),
        "first_frame_ms": round(first_ms, 2),
        "first_frame_pool_ms": round(first_t["pool"], 3),
        "phases_ms": {k: round(statistics.mean(p[k] for p in phases), 3) for k in phases[0]},
        "mean_icgn_iters_per_point": float(met[8]),
        "fast_pass_shape": {0: "reference from the planes", 1: "reference staged", -1: "undecided"}[
            eng.fast_pass_shape(prm.subset_size, six)],
        "global_model": {"locked": gm["locked"], "rotation_deg": float(np.degrees(gm["theta"])),
                         "scale": gm["scale"], "translation_px": [float(gm["t"][0]), float(gm["t"][1])]},
        "e2e": {"value": e2e_value, "unit": "points/s",
                "h2d_bytes_per_step": int(W * H), "d2h_bytes_per_step": int(rc_e2e * 32)},
        "roofline": {"kernel": "icgn solve (Path A launch)", "bound": "fp32", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": traffic,
                     "traffic_source": None if traffic is None else
                     f"ncu DRAM bytes per pixel-iteration of a 2048x2048 capture at subset {prm.subset_size} "
                     f"x {int(a_pix)} pixel-iterations",
                     "peak_source": f"{sms} SMs x 128 FP32 lanes x 2 x {peaks.get('sm_max_mhz', 1965.0)} MHz "
                                    f"({peak_src} sm_max_mhz)",
                     "algorithmic": f"{FLOP_PER_PIXEL_ITER[six]} FLOP per subset pixel per iteration x "
                                    f"{int(a_pix)} pixel-iterations per launch"},
        "clocks": clk.summary(),
        "gpu_launches": int(sum(c["launches"] for c in counts)),
    }
    if learned is not None:
        out["learned_seeding"] = learned
        out.pop("global_model")
        if rank == 0:
            out["seeding_compared"] = compare_seedings(ref, dfm, prm, warp)
    if rank == 0 and world == 1 and not args.no_cpu:
        crc, cdt, catt, cpts, cp = cpu_sample(ref, dfm, prm, model=gm["H"] if gm["locked"] else None)
        out["cpu_baseline"] = {"value": crc / cdt, "unit": "points/s", "cores": len(os.sched_getaffinity(0)),
                               "kind": "port",
                               "sample": f"central {cp[2]}x{cp[3]} ROI ({cp[2] // cp[4]}^2 grid, {catt} attempted) "
                                         f"of the same pair, reference cache warm, {cdt:.2f} s"}
        out["accuracy"] = accuracy_sample(eng, ref, dfm, prm, warp, cp, gm)
    eng.close()
    return out


def run_b200(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    m = measure_frames(args, args.workload, rank, world, local_rank, dist)
    # The default line also measures the target settings (4096^2, step 8,
    # subset 41 under the same field), where the task states its speed-up and
    # roofline targets; every rank takes the same steps.
    tgt = None
    if args.workload == "cfg1" and not args.no_target:
        tgt = measure_frames(args, "cfg4-plain", rank, world, local_rank, dist)
    if rank == 0:
        line = {"metric": METRIC, "value": m["value"], "unit": "points/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
        line.update({k: v for k, v in m.items() if k not in ("value", "ms_per_step")})
        if tgt is not None:
            t = {"value": tgt["value"], "unit": "points/s", "ms_per_step": tgt["ms_per_step"]}
            t.update({k: v for k, v in tgt.items() if k not in ("value", "ms_per_step")})
            line["target_settings"] = t
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_cfg3(args, rank, world=1, local_rank=0):
    """cfg3 (batched incremental DIC): args.sequences 2048x2048 sequences, each
    with its own seed, under a monotone uniaxial stretch (25 % over 128
    frames) plus a rigid rotation (30 deg over 128 frames), noise sigma 1.5,
    subset 21, step 6, window 21, advanced together through
    semper_b200_inc_batch_process (one session per sequence, their solves
    interleaved on the device; host frames in, host points out). A step is
    one frame of every sequence; warm-up frames are solved but not timed.
    Frames 1..W+K of the 128-frame sequences are run (the first W+K of the
    workload's frames)."""
    import math

    import torch

    import semper_b200 as sb

    dist = _init_dist(world, local_rank)
    n = args.size if args.size != 4096 else 2048
    S_all = max(1, args.sequences)
    # N > 1: the sequences are split over the ranks (equal cost each), every
    # rank advancing its own on its GPU; no data crosses ranks
    seq_ids = sb.shard([1] * S_all, rank, world)
    S = len(seq_ids)
    total = args.warmup + args.steps
    t_gen = time.perf_counter()
    refs = [sb.speckle(n, n, 3000 + 17 * q) for q in seq_ids]

    def frame(q, t):
        th, s = math.radians(30.0) * t / 128.0, 0.25 * t / 128.0
        a = (math.cos(th) * (1 + s) - 1, -math.sin(th), math.sin(th) * (1 + s), math.cos(th) - 1)
        return sb.speckle(n, n, 3000 + 17 * q, sb.warp_block(cx=n / 2, cy=n / 2, a=a), 1.5, 4000 + 1000 * q + t)

    frames = [[frame(q, t) for q in seq_ids] for t in range(1, total + 1)]
    gen_s = time.perf_counter() - t_gen
    m = n // 8
    prm = sb.params((m, m, n - 2 * m, n - 2 * m), 6, 21, 21)
    cap = ((n - 2 * m) // 6) ** 2 * 8
    b = sb.IncrementalBatch(max(S, 1))
    for q in range(S):
        assert b.init(q, refs[q], prm, args.interval) == 0
    acc = {"i": 0, "all_pts": 0}

    def step():
        fr = frames[acc["i"]]
        acc["i"] += 1
        res = b.process({q: fr[q] for q in range(S)}, cap)
        got = [res[q][0] for q in range(S)]
        assert not got or min(got) > 0, got
        acc["all_pts"] += sum(got)
        return sum(got), sum(res[q][3].reference_updated for q in range(S))

    t_w = time.perf_counter()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    warm_ms = 1000 * (time.perf_counter() - t_w)
    with ClockSampler(local_rank) as clk:
        ms_rank, outs = _timed_region(dist, step, args.steps)
    b.close()
    pts_rank = sum(o[0] for o in outs)
    value, mean_ms = aggregate(pts_rank, ms_rank / args.steps, args.steps, dist, "cuda")
    sums = torch.tensor([pts_rank / args.steps, sum(o[1] for o in outs), acc["all_pts"]], device="cuda",
                        dtype=torch.float64)
    all_ms_t = torch.tensor([warm_ms + ms_rank], device="cuda", dtype=torch.float64)
    if dist:
        dist.all_reduce(sums)
        dist.all_reduce(all_ms_t, op=dist.ReduceOp.MAX)
        dist.destroy_process_group()
    if rank != 0:
        return 0
    pts_step, updates, all_pts = (float(x) for x in sums.tolist())
    all_ms = float(all_ms_t.item())
    S = S_all
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"cfg3: {S} sequences of {n}x{n} speckle (own seeds), stretch 25 % + rotation 30 deg "
                               f"over 128 frames, noise 1.5, subset 21, step 6, window 21, update_interval "
                               f"{args.interval}; a step advances every sequence by one frame "
                               f"(semper_b200_inc_batch_process); frames {args.warmup + 1}..{total} timed after "
                               f"{args.warmup} warm-up frames",
                   "sequences": S, "frames_timed_per_sequence": args.steps, "reference_updates": int(updates),
                   "parallelism": f"the sequences split over {world} GPU(s)",
                   "points_per_step": pts_step, "frame_generation_s": round(gen_s, 1),
                   "l2": f"inputs larger than L2: each step reads {S} new {n * n >> 20} MiB frames and every "
                         f"session's planes"},
        "frames_per_s": S * 1000.0 / mean_ms,
        "from_frame1": {"frames": S * total, "points": int(all_pts), "ms": round(all_ms, 3),
                        "points_per_s": all_pts / (all_ms / 1000.0), "frames_per_s": S * total / (all_ms / 1000.0)},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": S * n * n,
                "d2h_bytes_per_step": int(pts_step) * 32},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def _init_dist(world, local_rank):
    """NCCL process group for N > 1 (None at N = 1), with a short timeout."""
    import torch

    torch.cuda.set_device(local_rank)
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist


def _timed_region(dist, fn, steps):
    """Runs fn() `steps` times between a barrier and a device synchronize on
    both sides; returns this rank's wall time in ms and fn's results."""
    import torch

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = [fn() for _ in range(steps)]
    torch.cuda.synchronize()
    ms = 1000 * (time.perf_counter() - t0)
    if dist:
        dist.barrier()
    return ms, out


def run_cfg4_seedings(args, rank):
    """The seedings of the large-deformation workload compared over its
    rotation distribution: args.pairs4 cfg4-large pairs (4096x4096, rotation
    ~U[0,180) deg, translation up to 60 px, 5 px random field, noise sigma 2;
    step 8, subset 41, window 41), each solved with every seeding: the
    lattice alone (the reference without a model), the global-motion
    estimate (the stand-in for the reference's AKAZE model), the proposal
    network first, and the rescue order (the estimate first, the network only
    where the lattice rejects the estimate). Per seeding and pair: K timed
    device-resident frames after W warm-up frames (CUDA events on the engine's
    stream), then K frames through semper_run from pinned host memory (e2e).
    A pair a seeding cannot solve contributes its time and no points. The
    line's value is the rescue order's."""
    if rank != 0:
        return 0
    import numpy as np
    import torch

    import semper_b200 as sb

    net = sb.Proposal.trained()
    seedings = ("lattice", "global", "learned", "rescue")
    acc = {s: {"pts": 0, "ms": 0.0, "e2e_ms": 0.0, "solved_pairs": 0, "per_pair": []} for s in seedings}
    gen_s = 0.0
    with ClockSampler(0) as clk:
        for pair in range(args.pairs4):
            t0 = time.perf_counter()
            ref, dfm, prm, warp, sim = sb.large_motion_pair(args.size, pair=pair)
            gen_s += time.perf_counter() - t0
            cap = (prm.rect_w // prm.step) * (prm.rect_h // prm.step) * 8
            d_def = torch.from_numpy(dfm).cuda()
            d_out = torch.empty(cap, dtype=torch.float32, device="cuda")
            h_frame = torch.from_numpy(dfm).pin_memory()
            h_out = torch.empty(cap, dtype=torch.float32).pin_memory().numpy()
            for s in seedings:
                eng = sb.Engine()
                assert eng.set_reference(ref) == 0
                if s in ("learned", "rescue"):
                    assert eng.set_proposal(net, True if s == "learned" else "rescue") == 0
                if s in ("lattice", "learned"):
                    eng.set_global_motion(False)
                for _ in range(1 + args.warmup):
                    rc, _ = eng.run_device(d_def, prm, d_out, cap)
                stream = torch.cuda.ExternalStream(eng.stream_handle())
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                ev0.record(stream)
                for _ in range(args.steps):
                    rc, _ = eng.run_device(d_def, prm, d_out, cap)
                ev1.record(stream)
                torch.cuda.synchronize()
                ms = ev0.elapsed_time(ev1)
                # e2e: one untimed call through semper_run first (its host
                # path sizes its buffers on first use), then K timed
                eng.run(h_frame.numpy(), prm, capacity=cap, out=h_out, copy=False)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for _ in range(args.steps):
                    rc_e, _, _ = eng.run(h_frame.numpy(), prm, capacity=cap, out=h_out, copy=False)
                e2e_ms = 1000 * (time.perf_counter() - t0)
                a = acc[s]
                a["pts"] += max(rc, 0) * args.steps
                a["ms"] += ms
                a["e2e_ms"] += e2e_ms
                a["solved_pairs"] += rc > 0
                a["per_pair"].append({"pair": pair, "rotation_deg": round(float(np.degrees(sim[0])), 1),
                                      "points": int(rc), "ms_per_frame": round(ms / args.steps, 3)})
                del eng
    out = {}
    for s in seedings:
        a = acc[s]
        out[s] = {"value": a["pts"] / (a["ms"] / 1000.0), "e2e": a["pts"] / (a["e2e_ms"] / 1000.0),
                  "unit": "points/s", "solved_pairs": int(a["solved_pairs"]), "pairs": args.pairs4,
                  "per_pair": a["per_pair"]}
    r = out["rescue"]
    frames = args.pairs4 * args.steps
    line = {
        "metric": METRIC, "value": r["value"], "unit": "points/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": acc["rescue"]["ms"] / frames, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"cfg4 seedings: {args.pairs4} large-deformation pairs (4096x4096, rotation "
                               f"~U[0,180) deg, translation up to 60 px, 5 px random field, noise sigma 2; step 8, "
                               f"subset 41, window 41), each solved with every seeding; value = the rescue order "
                               f"(global-motion estimate first, the proposal network where the lattice rejects "
                               f"it); a step is one frame of one pair",
                   "pair_generation_s": round(gen_s, 1),
                   "l2": "inputs larger than L2: reference planes 201 MB + deformed planes 201 MB per step"},
        "seedings": out,
        "e2e": {"value": r["e2e"], "unit": "points/s", "h2d_bytes_per_step": args.size * args.size,
                "d2h_bytes_per_step": int(acc["rescue"]["pts"] / frames * 32)},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_cfg2(args, rank, world=1, local_rank=0):
    """cfg2 (batched uneven solves): args.pairs independent pairs of side
    U{256..2048} with their own affine warps, masks, subsets and steps,
    solved concurrently through semper_b200_batch_run (host frames in, host
    points out). A step is one batch of every pair; the time is the host wall
    time of the call with the device idle on both sides."""
    import torch

    import semper_b200 as sb

    dist = _init_dist(world, local_rank)
    t0 = time.perf_counter()
    # N > 1: the fixed batch is split over the ranks (sb.shard, by cost),
    # each rank solving its share on its own GPU; no data crosses ranks
    all_jobs = sb.batch_job_params(args.pairs, seed=0)
    all_prm = [p for p, _ in all_jobs]
    mine = sb.shard([sb.job_cost(p) for p in all_prm], rank, world)
    jobs = sb.batch_jobs(args.pairs, seed=0, only=mine)
    gen_s = time.perf_counter() - t0
    b = sb.Batch(workers=args.workers)
    for _ in range(args.warmup):
        res = b.run(jobs)
    with ClockSampler(local_rank) as clk:
        ms_rank, outs = _timed_region(dist, lambda: b.run(jobs), args.steps)
    res = outs[-1]
    pts_rank = sum(sum(max(r[0], 0) for r in o) for o in outs)
    value, mean_ms = aggregate(pts_rank, ms_rank / args.steps, args.steps, dist, "cuda")
    pts_t = torch.tensor([pts_rank / args.steps], device="cuda", dtype=torch.float64)
    fail_t = torch.tensor([sum(1 for r in res if r[0] <= 0)], device="cuda", dtype=torch.float64)
    if dist:
        dist.all_reduce(pts_t)
        dist.all_reduce(fail_t)
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    nodes = sum((p.rect_w // p.step) * (p.rect_h // p.step) for p in all_prm)
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"cfg2: {args.pairs} independent pairs, side U{{256..2048}}, affine warps (|rot| <= 10 "
                               f"deg, stretch <= 3 %, shift <= 8 px), 1-3 circular mask holes removing U[0, 40 %], "
                               f"subset U{{15,21,31,41}}, step U{{4,8}}, window = subset; {args.workers} concurrent "
                               f"engines per GPU",
                   "parallelism": f"the batch split over {world} GPU(s) by cost (semper_b200.shard)",
                   "grid_nodes": nodes, "points_per_step": float(pts_t.item()),
                   "jobs_failed": int(fail_t.item()), "generation_s": round(gen_s, 1),
                   "timing": "host wall time of semper_b200_batch_run (frames from host memory, points to host "
                             "memory), device synchronised on both sides; value and e2e are the same measurement",
                   "l2": "inputs larger than L2: every pair's planes and pool are rebuilt per step"},
        "frames_per_s": args.pairs * 1000.0 / mean_ms,
        "e2e": {"value": value, "unit": "points/s",
                "h2d_bytes_per_step": int(sum(2 * p.rect_w * p.rect_h * (2 if m else 1) for p, m in all_jobs)),
                "d2h_bytes_per_step": int(pts_t.item() * 32)},
        "clocks": clk.summary(),
    }
    if not args.no_cpu and world == 1:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle

        small = sorted(jobs, key=lambda j: j["ref"].size)[: max(1, args.pairs // 16)]
        cpts, cdt = 0, 0.0
        for j in small:
            o = oracle.Oracle(False, kind="reference_flags")
            o.set_reference(j["ref"], j["mask"])
            p = [0, 0, j["ref"].shape[1], j["ref"].shape[0], j["prm"].step, j["prm"].subset_size,
                 j["prm"].strain_window, 0]
            t0 = time.perf_counter()
            rc, _, _ = o.run(j["dfm"], p, mask=j["mask"])
            cdt += time.perf_counter() - t0
            cpts += max(rc, 0)
        line["cpu_baseline"] = {"value": cpts / cdt, "unit": "points/s", "cores": len(os.sched_getaffinity(0)),
                                "kind": "port",
                                "sample": f"the {len(small)} smallest pairs, one cold solve each, {cdt:.1f} s"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-target", action="store_true",
                    help="cfg1 only: skip the nested target-settings measurement (step 8, subset 41)")
    ap.add_argument("--size", type=int, default=4096,
                    help="image edge (default 4096, the benchmark workload; smaller sizes are for profiling)")
    ap.add_argument("--workload", default="cfg1", choices=["cfg1", "cfg2", "cfg4-plain", "cfg4-large", "cfg4-learned", "cfg4-seedings",
                             "cfg3"],
                    help="cfg1 (the headline line), cfg2 (batched uneven pairs), cfg4-plain (the target "
                         "settings), cfg4-large (large deformation seeded by the global-motion estimate), "
                         "cfg4-learned (the same pair seeded by the proposal network), cfg4-seedings (every seeding "
                         "over several large-deformation pairs), cfg3 (batched incremental sequences)")
    ap.add_argument("--pairs", type=int, default=256, help="cfg2: pairs per batch")
    ap.add_argument("--workers", type=int, default=8, help="cfg2: concurrent engines")
    ap.add_argument("--interval", type=int, default=1, help="cfg3: the session's update_interval")
    ap.add_argument("--sequences", type=int, default=8, help="cfg3: sequences advanced together")
    ap.add_argument("--pairs4", type=int, default=8, help="cfg4-seedings: large-deformation pairs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.workload == "cfg3":
        return run_cfg3(args, rank, world, local_rank)
    if args.workload == "cfg2":
        return run_cfg2(args, rank, world, local_rank)
    if args.workload == "cfg4-seedings":
        return run_cfg4_seedings(args, rank)
    return run_b200(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
