#!/usr/bin/env python
"""Throughput of the B200 film-process render path (one JSON line on rank 0).

Workload (one step = one frame): the full optical print at 3840x2160 -- a float32
linear Rec.709 RGB synthetic frame (seeded smooth fields, prepare.synthetic_frame),
kodak_portra_400 -> kodak_portra_endura print route with every spatial stage on
(camera diffusion radius 0.5 % of the width, emulsion scatter/halation, spatial DIR
tail 200 um weight 0.03, density-space grain 35 mm format with fixed seeds over
synthetic noise of the production shapes), then capture development, 81-wavelength
print, scanner LUT, OkLch gamut and sRGB output -- rendered by fj_cuda_render, the
drop-in entry point. Frames are independent, so N GPUs run N replicas (weak scaling,
no collective on the data path).

  value   Mpix/s with the frame resident in HBM (CUDA events on the render stream
          around the timed frames, max over ranks);
  stages  device time per stage from the owner's stage events in the timed region;
  e2e     Mpix/s through the C-ABI with host buffers: pinned host frame -> H2D, render,
          D2H of the rendered frame, every step, frames pipelined over two copy streams;
  --impl reference  times the CPU restatement of the reference's render path (the
          reference has no CPU renderer) on all host threads, on the same 3840x2160
          frame and descriptors, one whole frame per step (diffusion in the
          reference's FFT form, FP64).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

WIDTH, HEIGHT = 3840, 2160
SEED = 20261203 + 2  # seed of the 4K precision-form configuration
METRIC = "4K full optical print render throughput (Mpix/s)"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="0 skips the CPU baseline leg")
    ap.add_argument("--width", type=int, default=WIDTH, help="frame width (profiling runs use small frames)")
    ap.add_argument("--height", type=int, default=HEIGHT)
    ap.add_argument("--next-rows", action="store_true",
                    help="workload variant: add highlight reconstruction and scanner post effects (glare, lens blur, "
                         "the production unsharp 0.7 px / 0.7)")
    ap.add_argument("--no-batch", action="store_true", help="skip the mixed-batch block")
    ap.add_argument("--precision", action="store_true",
                    help="instead of timing: one frame against the oracle's stage chain (CIEDE2000 of the output)")
    args = ap.parse_args()
    return args


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms during a region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi needs a moment before its first sample; start timing after it.
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:
                time.sleep(0.02)
            self.lines.clear()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "error": (self.lines[0][:200] if self.lines else "no nvidia-smi output")}
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": max(maxes), "reasons": sorted(reasons),
                "samples": len(mhz)}


def dist_setup(n):
    import torch

    if n <= 1:
        return 0, 1, None
    import datetime

    import torch.distributed as dist

    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    return rank, world, dist


def workload_config(W, H, next_rows: bool):
    """The `config` of both arms' JSON lines (identical, so the two lines name one workload)."""
    return {"workload": f"{W}x{H} full optical print (negative -> print -> scan)"
                        + (" + highlight reconstruction + scanner post effects + film/gate defects and weave"
                           if next_rows else ""),
            "recipe": "kodak_portra_400 -> kodak_portra_endura, Hanatos TC LUT, spatial DIR tail 200 um "
                      "w 0.03, camera diffusion r=0.5% W, scatter/halation, grain 35 mm, scanner LUT r=17, "
                      "OkLch gamut, sRGB",
            "frame_bytes": W * H * 12,
            "l2_policy": "inputs larger than L2 (99.5 MB frame in and out, ~0.7 GB of stage planes per frame)"}


def _cpu_frame(threads, W, H, next_rows):
    """One step of the CPU restatement: the whole frame (same seed and descriptors as
    the GPU arm) through the oracle's stage chain, diffusion in the FFT form."""
    __graft_entry__.package()
    from film_juicer_b200 import frame_records, prepare
    from oracle import frame as oframe

    recipe = prepare.PreparedRecipe.load(os.path.join(ROOT, "tests", "golden", "recipe_print.npz"))
    rec = workload_record(frame_records, recipe, W, H, next_rows)
    src = prepare.synthetic_frame(W, H, seed=SEED)
    return lambda: oframe.render_frame(rec, recipe, src, threads=threads, diffusion_form="fft")


def run_reference(args):
    """CPU restatement of the reference render path on all host threads, whole frames."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    W, H = args.width, args.height
    step = _cpu_frame(threads, W, H, args.next_rows)
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    per_step = statistics.median(times)
    mpix = W * H / per_step / 1e6
    sample = f"the whole {W}x{H} frame per step, median of {args.steps} steps"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(mpix, 4), "unit": "Mpix/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(W, H, args.next_rows),
        "cpu_baseline": {"value": round(mpix, 4), "unit": "Mpix/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(mpix, 4), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "threads": threads,
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(seconds: float, W, H, next_rows):
    """The oracle's whole-frame chain on the same frame, all host threads, whole frames
    until `seconds` have passed (at least one)."""
    threads = os.cpu_count() or 1
    step = _cpu_frame(threads, W, H, next_rows)
    n, t0 = 0, time.perf_counter()
    while n == 0 or time.perf_counter() - t0 < seconds:
        step()
        n += 1
    dt = time.perf_counter() - t0
    return {"value": round(W * H * n / dt / 1e6, 4), "unit": "Mpix/s", "cores": threads, "kind": "port",
            "sample": f"{n} whole {W}x{H} frame(s) in {dt:.1f} s"}


# Algorithmic work per stage per pixel of the frame (the roofline numerators), from the
# scope table's measurement row: compulsory HBM bytes of a minimal fused schedule (4 B
# per plane read or written per pixel), and for the print chain its arithmetic
# (2*81*3 density->spectral + 81 illuminant + 2*81*3 sensitivity FLOP and 81 EX2).
PRINT_FLOP_PER_PX = 2 * 81 * 3 + 81 + 2 * 81 * 3
PRINT_EX2_PER_PX = 81


def stage_models():
    return {
        "camera_exposure": ("hbm", 12 + 12),          # RGB in, 3 planes out
        "camera_diffusion": ("hbm", 24),              # 3 planes in, 3 planes out
        "scatter_halation": ("hbm", 24),              # 3 planes in, 3 planes out
        "spatial_dir": ("hbm", 12 + 24 + 24),         # source: carrier in, corrections + log raw out; blur
        "capture_density": ("hbm", 24 + 12),         # filtered corrections + log raw in, density out
        "grain": ("hbm", 24),                         # density in, density out
        "print_scan_output": ("spectral", 12 + 12),   # density in, RGB out; FMA / MUFU bound
    }


def stage_roofline(name, stage_ms, px, pk, sm_mhz):
    """Achieved work of one stage against its bound (measured HBM peak; FP32 FMA and
    MUFU EX2 rates at the sampled SM clock for the spectral chain)."""
    kind, per_px = stage_models()[name]
    stage_s = stage_ms * 1e-3
    if kind == "hbm":
        achieved = px * per_px / stage_s / 1e9
        return {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / pk["hbm_gbs"], 4), "bytes_per_px": per_px}
    clk = (sm_mhz or 1965.0) * 1e6
    fma_peak = 148 * 128 * 2 * clk / 1e12      # TFLOP/s
    mufu_peak = 148 * 16 * clk / 1e12          # T ex2/s
    flops = px * PRINT_FLOP_PER_PX / stage_s / 1e12
    ex2 = px * PRINT_EX2_PER_PX / stage_s / 1e12
    return {"bound": "fp32+mufu", "achieved": round(flops, 2), "peak": round(fma_peak, 1), "unit": "TFLOP/s",
            "frac": round(flops / fma_peak, 4), "ex2_per_s_T": round(ex2, 3), "ex2_peak_T": round(mufu_peak, 3),
            "ex2_frac": round(ex2 / mufu_peak, 4), "flop_per_px": PRINT_FLOP_PER_PX, "ex2_per_px": PRINT_EX2_PER_PX}


def workload_record(frame_records, recipe, W, H, next_rows: bool):
    """The bench frame; `next_rows` adds highlight reconstruction (protection 4, sharpness
    3, peak gain 1.5), scanner post effects (glare 0.3 % blurred 4 px, lens blur 0.8 px,
    unsharp 0.7 px amount 0.7) and film / gate defects with weave (the characterization's
    dust and scratch families at slot probabilities 0.02 / 0.05 / 0.01 / 0.02)."""
    if not next_rows:
        return frame_records.FrameRecord(recipe, W, H)
    from film_juicer_b200 import descriptors

    post = descriptors.scanner_post_record(glare_percent=0.3, glare_roughness=0.4, glare_blur_sigma_px=4.0,
                                           lens_blur_sigma_px=0.8, unsharp_sigma_px=0.7, unsharp_amount=0.7)
    boost = descriptors.highlight_boost_record(4.0, 3.0, 1.5)
    effects = descriptors.default_film_effects(W, H)
    return frame_records.FrameRecord(recipe, W, H, post=post, highlight_boost=boost, effects=effects)


def run_b200(args):
    import ctypes as C

    import numpy as np
    import torch

    rank, world, dist = dist_setup(args.gpus)
    if world == 1 and torch.cuda.is_available():
        torch.cuda.set_device(0)
    pkg = __graft_entry__.package()
    lib = pkg.load_library()
    from film_juicer_b200 import abi, frame_records, prepare, runtime

    dev = torch.cuda.current_device()
    W, H = args.width, args.height
    recipe = prepare.PreparedRecipe.load(os.path.join(ROOT, "tests", "golden", "recipe_print.npz"))
    record = workload_record(frame_records, recipe, W, H, args.next_rows)
    host = prepare.synthetic_frame(W, H, seed=SEED + rank)
    src = torch.from_numpy(host).to("cuda")
    dst = torch.empty_like(src)
    stream = torch.cuda.Stream()
    owner = runtime.Owner()
    err = abi.ErrorText()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident throughput ----
    # Exactly `steps` frames per timed region, bracketed by a barrier and a device
    # synchronise. The region is repeated so that the clock sampler (50 ms period)
    # sees at least ~2 s of rendering; ms_per_step is the median region / steps.
    for _ in range(args.warmup):
        owner.render(record, src, dst, stream=stream)
    stream.synchronize()
    t_est = time.perf_counter()
    owner.render(record, src, dst, stream=stream)
    stream.synchronize()
    est_ms = (time.perf_counter() - t_est) * 1e3
    regions = max(1, min(50, int(2000.0 / max(est_ms * args.steps, 1e-3)) + 1))
    if dist is not None:
        t = torch.tensor([regions], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        regions = int(t.item())
    lib.fjb_owner_stage_timing(owner.handle, 1, C.byref(err.buf))
    region_ms, launches = [], 0
    with ClockSampler(dev) as clocks:
        for _ in range(regions):
            barrier()
            torch.cuda.synchronize()
            launches0 = int(lib.fjb_kernel_launches())
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            for _ in range(args.steps):
                owner.render(record, src, dst, stream=stream)
            end.record(stream)
            end.synchronize()
            torch.cuda.synchronize()
            launches = int(lib.fjb_kernel_launches()) - launches0
            region_ms.append(start.elapsed_time(end))
    times = abi.FjbStageTimes()
    lib.fjb_owner_stage_times(owner.handle, C.byref(times), C.byref(err.buf))
    lib.fjb_owner_stage_timing(owner.handle, 0, C.byref(err.buf))
    barrier()
    ms = max_over_ranks(statistics.median(region_ms) / args.steps)
    px = W * H
    value = world * px / (ms * 1e-3) / 1e6
    stages = {}
    for i, name in enumerate(abi.FJB_STAGE_NAMES):
        if times.frames[i]:
            stages[name] = round(times.total_ms[i] / times.frames[i], 4)

    # ---- the print contraction's tensor-core forms (same frame, same timing rules) ----
    # The FP32 form above is the parity form and the headline value. The same K-step
    # regions are timed with the 81-wavelength contraction on the tensor cores (BF16
    # tiles, FP32 accumulation; transmittances as one BF16 or a hi + lo pair), and each
    # form's output is compared with the FP32 form's in CIEDE2000 on every 4th pixel of
    # every 4th row.
    forms = {}
    ref_out = dst.cpu().numpy()[::4, ::4] if rank == 0 else None
    for name, code in (("tensor", abi.FJB_PRINT_TENSOR), ("tensor_split", abi.FJB_PRINT_TENSOR_SPLIT)):
        owner.set_print_form(code)
        for _ in range(args.warmup):
            owner.render(record, src, dst, stream=stream)
        stream.synchronize()
        lib.fjb_owner_stage_timing(owner.handle, 1, C.byref(err.buf))
        f_ms = []
        for _ in range(regions):
            barrier()
            torch.cuda.synchronize()
            fa, fb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            fa.record(stream)
            for _ in range(args.steps):
                owner.render(record, src, dst, stream=stream)
            fb.record(stream)
            fb.synchronize()
            f_ms.append(fa.elapsed_time(fb))
        ftimes = abi.FjbStageTimes()
        lib.fjb_owner_stage_times(owner.handle, C.byref(ftimes), C.byref(err.buf))
        lib.fjb_owner_stage_timing(owner.handle, 0, C.byref(err.buf))
        barrier()
        fms = max_over_ranks(statistics.median(f_ms) / args.steps)
        pso = abi.FJB_STAGE_NAMES.index("print_scan_output")
        entry = {"value": round(world * W * H / (fms * 1e-3) / 1e6, 2), "ms_per_step": round(fms, 4),
                 "print_scan_output_ms": round(ftimes.total_ms[pso] / max(ftimes.frames[pso], 1), 4),
                 "frame_speedup_vs_fp32": round(ms / fms, 4)}
        if rank == 0:
            from oracle import color

            entry["delta_e00_vs_fp32"] = {k: round(v, 5) for k, v in
                                          color.delta_e_stats(dst.cpu().numpy()[::4, ::4], ref_out).items()}
        forms[name] = entry
    owner.set_print_form(abi.FJB_PRINT_FP32)
    owner.render(record, src, dst, stream=stream)
    stream.synchronize()

    # ---- differentiation: forward and adjoint of the fitting chain ----
    # 16 seeded 512 x 512 crops as one 8192 x 512 image (the chain is per pixel), the
    # bench's print recipe; the cotangent is the gradient of the mean squared error
    # against the recipe's own render. Forward = fjb_fit_forward, backward = fjb_fit_vjp
    # (which recomputes the forward); the pixel render of the same crops is timed
    # beside them. The crops (50 MB in, 50 MB of cotangent) fit in L2: these kernels
    # are issue-bound, so L2 residency does not change their time.
    diff = fit_block(torch, prepare, runtime, recipe, args, stream, barrier, max_over_ranks)
    batch = batch_block(torch, frame_records, prepare, owner, args, barrier, max_over_ranks) \
        if not args.no_batch else None

    # ---- end to end through the C-ABI with host buffers ----
    # Frames are pipelined as a host would: while frame i renders on the render stream,
    # frame i+1's pixels go up on a copy stream and frame i-1's result comes down on
    # another (two device frame buffers, pinned host buffers). Every step still copies
    # its whole input up and its whole output down inside the timed region.
    h_src = torch.from_numpy(host).pin_memory()
    h_dst = [torch.empty_like(h_src).pin_memory() for _ in range(2)]
    d_src = [src, torch.empty_like(src)]
    d_dst = [dst, torch.empty_like(dst)]
    cin, cout = torch.cuda.Stream(), torch.cuda.Stream()
    e_steps = max(3, min(args.steps, 30))

    def pipelined(n, t0=None, t1=None):
        ev = lambda: torch.cuda.Event()  # noqa: E731
        up, done, down = [ev(), ev()], [ev(), ev()], [ev(), ev()]
        if t0 is not None:
            t0.record(cin)
        with torch.cuda.stream(cin):
            d_src[0].copy_(h_src, non_blocking=True)
        up[0].record(cin)
        for i in range(n):
            b = i % 2
            if i + 1 < n:
                nb = (i + 1) % 2
                if i >= 1:
                    cin.wait_event(done[nb])  # frame i-1 has finished reading d_src[nb]
                with torch.cuda.stream(cin):
                    d_src[nb].copy_(h_src, non_blocking=True)
                up[nb].record(cin)
            stream.wait_event(up[b])
            if i >= 2:
                stream.wait_event(down[b])  # frame i-2's result has left d_dst[b]
            owner.render(record, d_src[b], d_dst[b], stream=stream)
            done[b].record(stream)
            cout.wait_event(done[b])
            with torch.cuda.stream(cout):
                h_dst[b].copy_(d_dst[b], non_blocking=True)
            down[b].record(cout)
        if t1 is not None:
            t1.record(cout)
        cout.synchronize()

    pipelined(3)
    barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pipelined(e_steps, e_start, e_end)
    barrier()
    e_ms = max_over_ranks(e_start.elapsed_time(e_end) / e_steps)
    e2e = world * px / (e_ms * 1e-3) / 1e6
    ok = bool(np.isfinite(h_dst[0].numpy()).all() and np.isfinite(h_dst[1].numpy()).all())

    if rank == 0:
        pk, pk_kind = peaks()
        clk = clocks.summary()
        models = stage_models()
        per_stage = {k: stage_roofline(k, stages[k], px, pk, clk.get("sm_mhz")) for k in stages if k in models}
        # the roofline object: the stage that takes the most device time
        dominant = max(per_stage, key=lambda k: stages[k])
        roof = dict(per_stage[dominant])
        roof["peak_source"] = pk_kind if roof["bound"] == "hbm" else "FP32 FMA / MUFU rates at the sampled SM clock"
        roof["kernel_stage"] = dominant
        roof["stage_ms"] = stages[dominant]
        traffic = None
        prof = os.path.join(ROOT, "profiles", "stage_traffic_4k.json")
        if os.path.exists(prof):
            with open(prof) as fh:
                traffic = json.load(fh).get(dominant, {}).get("dram_bytes_per_launch")
        roof["traffic"] = traffic
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(W, H, args.next_rows),
            "entry": "fj_cuda_render (C-ABI)",
            "replicas": world,
            "timed_regions": regions,
            "region_ms": [round(v, 3) for v in region_ms],
            "stages_ms": stages,
            "roofline": roof,
            "stages_roofline": {k: {"frac": v["frac"], "bound": v["bound"]} for k, v in per_stage.items()},
            "print_forms": {"fp32": {"value": round(value, 2), "ms_per_step": round(ms, 4),
                                     "print_scan_output_ms": stages.get("print_scan_output")}, **forms},
            "differentiation": diff,
            "batch": batch,
            "cpu_baseline": cpu_baseline(args.cpu_seconds, W, H, args.next_rows) if world == 1 and args.cpu_seconds > 0 else None,
            "e2e": {"value": round(e2e, 2), "unit": "Mpix/s", "h2d_bytes_per_step": int(h_src.numel() * 4),
                    "d2h_bytes_per_step": int(h_dst[0].numel() * 4), "steps": e_steps,
                    "schedule": "frames pipelined: H2D of frame i+1 and D2H of frame i-1 on copy streams "
                                "while frame i renders"},
            "gpu_launches": launches,
            "clocks": clk,
            "output_finite": ok,
        }
        print(json.dumps(line), flush=True)
    owner.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def fit_block(torch, prepare, runtime, recipe, args, stream, barrier, max_over_ranks):
    """Forward, adjoint and pixel-render times on the differentiation workload (16 seeded
    512 x 512 crops), K steps per timed region, median of 5 regions, max over ranks."""
    from film_juicer_b200 import fitting

    crops = [prepare.synthetic_frame(512, 512, seed=SEED + 100 + i) for i in range(16)]
    import numpy as np

    s = torch.from_numpy(np.ascontiguousarray(np.concatenate(crops, axis=0))).to("cuda")
    dr = runtime.DeviceRecipe(prepare.HostRecord(recipe), stream=stream)
    th0 = fitting.default_theta(dr)
    thp = th0.clone()
    thp[[0, 1, 2, 12]] += torch.tensor([0.1, -0.05, 0.08, -0.1], dtype=torch.float64)
    with torch.cuda.stream(stream):
        target = fitting.forward(dr, th0, s, stream=stream).clone()
        out = torch.empty_like(target)
        dst = torch.empty_like(s)
        gout = torch.empty(fitting.N_PARAMS, dtype=torch.float64, device="cuda")
    steps = max(3, min(args.steps, 50))

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        stream.synchronize()
        vals = []
        for _ in range(5):
            barrier()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(steps):
                fn()
            b.record(stream)
            b.synchronize()
            vals.append(a.elapsed_time(b) / steps)
        return max_over_ranks(statistics.median(vals))

    fwd = timed(lambda: fitting.forward(dr, thp, s, out, stream=stream))
    with torch.cuda.stream(stream):
        cot = (2.0 / out.numel()) * (out - target)
    bwd = timed(lambda: fitting.vjp(dr, thp, s, cot, gout, stream=stream))
    ren = timed(lambda: dr.render(s, dst, stream=stream))
    stream.synchronize()
    grad = gout.cpu()
    dr.close()
    px = s.shape[0] * s.shape[1]
    frame = frame_fit_block(torch, prepare, runtime, recipe, stream, th0, thp, timed)
    return {"workload": "16 x 512 x 512 seeded crops, print route, 13 parameters (exposure_ev BGR, film_gamma BGR, "
                        "print_gamma CMY, donor_k BGR, print_ev)",
            "forward_ms": round(fwd, 4), "adjoint_ms": round(bwd, 4), "fwd_bwd_ms": round(fwd + bwd, 4),
            "fwd_bwd_over_forward": round((fwd + bwd) / fwd, 3),
            "pixel_render_ms": round(ren, 4), "fwd_bwd_over_pixel_render": round((fwd + bwd) / ren, 3),
            "fwd_bwd_mpix_s": round(px / ((fwd + bwd) * 1e-3) / 1e6, 1),
            "gradient_finite": bool(torch.isfinite(grad).all()), "steps": steps, "regions": 5, "frame": frame}


def frame_fit_block(torch, prepare, runtime, recipe, stream, th0, thp, timed):
    """Whole-frame fitting: a 1920x1080 print frame with camera diffusion,
    scatter/halation and spatial DIR on (fitting.FrameFit): the forward (optics
    stages, DIR source, DIR filter, development) and the adjoint (13 parameters and the
    5 optics parameters: the development's adjoint, the filtered-correction cotangent
    through the DIR filter, the source stage's adjoint, the optics tangents), timed
    with CUDA events around the Python calls (host-side gaps included)."""
    from film_juicer_b200 import fitting, frame_records

    fw, fh = 1920, 1080
    rec = frame_records.FrameRecord(recipe, fw, fh, recipe_hash=0xF17, grain=False)
    dr = runtime.DeviceRecipe(rec.host, stream=stream)
    src = torch.from_numpy(prepare.synthetic_frame(fw, fh, seed=SEED + 150)).to("cuda")
    ff = fitting.FrameFit(dr, rec.host.h, src, stream=stream)
    opt = ff.optics_default()
    with torch.cuda.stream(stream):
        target = ff.forward(th0, opt).clone()
        out = torch.empty_like(target)
    fwd = timed(lambda: ff.forward(thp, opt, out=out))
    with torch.cuda.stream(stream):
        cot = (2.0 / out.numel()) * (out - target)
    grads = {}

    def adjoint():
        grads["g"] = ff.vjp(thp, opt, cot)

    bwd = timed(adjoint)
    g_theta, g_opt = grads["g"]
    ff.close()
    dr.close()
    return {"workload": "1920x1080 print frame, camera diffusion + scatter/halation + spatial DIR, 13 + 5 parameters",
            "forward_ms": round(fwd, 4), "adjoint_ms": round(bwd, 4), "fwd_bwd_ms": round(fwd + bwd, 4),
            "fwd_bwd_over_forward": round((fwd + bwd) / fwd, 3),
            "gradient_finite": bool(torch.isfinite(g_theta).all() and torch.isfinite(g_opt).all())}


BATCH_FRAMES = [(1920, 1080)] * 8 + [(3840, 2160)] * 4 + [(4096, 3072)] * 2
BATCH_RECIPES = [("recipe_print.npz", 0xB001), ("recipe_vision3_500t_2383.npz", 0xB002),
                 ("recipe_ektar100_endura.npz", 0xB003)]


def batch_block(torch, frame_records, prepare, owner, args, barrier, max_over_ranks):
    """The mixed batch: 8 x 1920x1080, 4 x 3840x2160 and 2 x 4096x3072 frames, three
    capture stocks on two print papers (assigned in turn), every spatial stage, through
    fjb_render_batch on one stream -- eagerly, and replayed from the captured CUDA graph
    (one launch per batch) -- with diffusion-form autotuning on (on the process's one
    owner, switched off again after). A step is one whole batch; CUDA events on the
    batch stream, median of the timed steps, max over ranks."""
    from film_juicer_b200 import grain_plan

    recipes = [(prepare.PreparedRecipe.load(os.path.join(ROOT, "tests", "golden", f)), h) for f, h in BATCH_RECIPES]
    noise = grain_plan.synthetic_noise()
    recs, srcs, dsts = [], [], []
    for i, (w, h) in enumerate(BATCH_FRAMES):
        rcp, rh = recipes[i % len(recipes)]
        recs.append(frame_records.FrameRecord(rcp, w, h, recipe_hash=rh, noise=noise))
        srcs.append(torch.from_numpy(prepare.synthetic_frame(w, h, seed=SEED + 200 + i)).to("cuda"))
        dsts.append(torch.empty_like(srcs[-1]))
    px = sum(w * h for w, h in BATCH_FRAMES)
    stream = torch.cuda.Stream()
    owner.set_autotune(True)
    steps = max(3, min(args.steps, 5))

    def timed(token):
        owner.render_batch(recs, srcs, dsts, stream, graph_token=token)  # warm-up (and capture)
        captured = owner.last_batch_text == ""
        vals = []
        for _ in range(steps):
            barrier()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            owner.render_batch(recs, srcs, dsts, stream, graph_token=token)
            b.record(stream)
            b.synchronize()
            vals.append(a.elapsed_time(b))
        return max_over_ranks(statistics.median(vals)), captured

    eager_ms, _ = timed(0)
    graph_ms, captured = timed(0xBA7C4)
    finite = all(bool(torch.isfinite(d).all()) for d in dsts)
    forms = {}
    for w, h in sorted(set(BATCH_FRAMES)):
        r = recs[BATCH_FRAMES.index((w, h))].host.h.optics.camera.radius_px
        f = owner.diffusion_form(w, h, r)
        forms[f"{w}x{h} r={r}"] = {0: "direct", 1: "fft"}.get(f, "undecided")
    owner.set_autotune(False)
    return {"workload": "8 x 1920x1080 + 4 x 3840x2160 + 2 x 4096x3072 full optical print frames, stocks "
                        "kodak_portra_400 / kodak_vision3_500t / kodak_ektar_100 on papers kodak_portra_endura / "
                        "kodak_2383, every spatial stage, one fjb_render_batch per step",
            "frames": len(BATCH_FRAMES), "mpix_per_batch": round(px / 1e6, 2),
            "value": round(px / (graph_ms * 1e-3) / 1e6, 2), "unit": "Mpix/s", "ms_per_batch": round(graph_ms, 3),
            "graph_captured": captured,
            "eager": {"value": round(px / (eager_ms * 1e-3) / 1e6, 2), "ms_per_batch": round(eager_ms, 3)},
            "diffusion_forms": forms, "steps": steps, "output_finite": finite}


def run_precision(args):
    """One frame through fj_cuda_render against the oracle's chain of the same stages
    (FP32/FP64 CPU restatement, all host threads): CIEDE2000 of the encoded output
    (p50 / p99 / max) and the largest absolute difference per encoded channel."""
    import numpy as np
    import torch

    __graft_entry__.package()
    from film_juicer_b200 import frame_records, prepare, runtime
    from oracle import color
    from oracle import frame as oframe

    W, H = args.width, args.height
    recipe = prepare.PreparedRecipe.load(os.path.join(ROOT, "tests", "golden", "recipe_print.npz"))
    record = frame_records.FrameRecord(recipe, W, H)
    host = np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=SEED))
    src = torch.from_numpy(host).to("cuda")
    dst = torch.empty_like(src)
    with runtime.Owner() as owner:
        owner.render(record, src, dst)
    got = dst.cpu().numpy()
    from film_juicer_b200 import staged as fstaged

    staged = fstaged.render_staged(record, src)
    t0 = time.perf_counter()
    ref_stages = {}
    want, _ = oframe.render_frame(record, recipe, host, threads=os.cpu_count() or 1, stages=ref_stages)
    t_oracle = time.perf_counter() - t0
    stats = color.delta_e_stats(got, want)
    per_stage = {}
    for name, planes in staged.items():
        ref = want if name == "output" else ref_stages[name]
        if name == "output":
            planes = [planes[..., c] for c in range(3)]
            ref = [ref[..., c] for c in range(3)]
        per_stage[name] = {"max_abs": float(max(np.abs(a - b).max() for a, b in zip(planes, ref))),
                           "mean_abs": float(np.mean([np.abs(a - b).mean() for a, b in zip(planes, ref)])),
                           "max_value": float(max(np.abs(b).max() for b in ref))}
    line = {"precision": {"workload": f"{W}x{H} full optical print through fj_cuda_render", "dtype": "f32",
                          "delta_e00_vs_oracle": {k: round(v, 6) for k, v in stats.items()},
                          "max_abs_encoded": float(np.abs(got - want).max()),
                          "mean_abs_encoded": float(np.abs(got - want).mean()),
                          "stages_vs_oracle": per_stage,
                          "oracle_seconds": round(t_oracle, 1), "oracle_threads": os.cpu_count()}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.precision:
        run_precision(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
