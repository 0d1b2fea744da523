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
          reference has no CPU renderer) on all host threads, on crops of the frame.
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
CROP = (384, 216)  # CPU sample: a crop of the frame with the 4K frame's descriptors
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
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
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


def _crop_workload(threads, crop=CROP):
    """The CPU sample: a crop of the 4K frame rendered by the oracle's chain with the 4K
    frame's descriptors (same pixel size, diffusion radius, grain)."""
    __graft_entry__.package()
    from film_juicer_b200 import frame_records, prepare
    from oracle import frame as oframe

    recipe = prepare.PreparedRecipe.load(os.path.join(ROOT, "tests", "golden", "recipe_print.npz"))
    w, h = crop
    rec = frame_records.FrameRecord(recipe, w, h, descriptor_width=WIDTH)
    src = prepare.synthetic_frame(WIDTH, HEIGHT, seed=SEED)[:h, :w].copy()
    return lambda: oframe.render_frame(rec, recipe, src, threads=threads)


def run_reference(args):
    """CPU restatement of the reference render path on all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    # crops shrink with the step count so that the whole run stays within minutes
    scale = min(1.0, (100.0 / max(args.steps, 1)) ** 0.5)
    crop = (max(96, int(CROP[0] * scale) // 8 * 8), max(54, int(CROP[1] * scale) // 2 * 2))
    step = _crop_workload(threads, crop)
    for _ in range(max(args.warmup, 1)):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    per_step = statistics.median(times)
    mpix = crop[0] * crop[1] / per_step / 1e6
    sample = (f"{crop[0]}x{crop[1]} crop of the 4K frame per step with the 4K descriptors, "
              f"median of {args.steps}")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(mpix, 4), "unit": "Mpix/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "full optical print, 3840x2160 frame, sampled as crops",
                   "recipe": "kodak_portra_400 -> kodak_portra_endura", "threads": threads},
        "cpu_baseline": {"value": round(mpix, 4), "unit": "Mpix/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(mpix, 4), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(seconds: float):
    """The oracle's whole-frame chain on crops of the frame, all host threads."""
    threads = os.cpu_count() or 1
    step = _crop_workload(threads)
    step()
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        step()
        n += 1
    dt = time.perf_counter() - t0
    return {"value": round(CROP[0] * CROP[1] * n / dt / 1e6, 4), "unit": "Mpix/s", "cores": threads,
            "kind": "port",
            "sample": f"{n} x ({CROP[0]}x{CROP[1]} crop of the 4K frame, 4K descriptors) in {dt:.1f} s"}


# Algorithmic work per stage per pixel of the frame (the roofline numerators):
# compulsory HBM bytes of a fused schedule (4 B per plane read or written), or FLOPs.
def stage_models(record):
    h = record.host.h
    r = h.optics.camera.radius_px
    return {
        "camera_exposure": ("hbm", 12 + 12),          # RGB in, 3 planes out
        "camera_diffusion": ("fp32", 3 * (2 * r + 1) ** 2 * 2.0),  # dense (2r+1)^2 PSF per channel
        "scatter_halation": ("hbm", 24 + 24),         # 3 planes in + out, in place, plus one temp round trip
        "spatial_dir": ("hbm", 12 + 36),              # carrier in; raw, filtered and log-raw planes out
        "capture_density": ("hbm", 12 + 24 + 12),     # carrier + spatial DIR planes in, density out
        "grain": ("hbm", 12 + 12),                    # density in, density out
        "print_scan_output": ("hbm", 12 + 12),        # density in, RGB out
    }


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
    for _ in range(args.warmup):
        owner.render(record, src, dst, stream=stream)
    stream.synchronize()
    lib.fjb_owner_stage_timing(owner.handle, 1, C.byref(err.buf))
    launches0 = int(lib.fjb_kernel_launches())
    barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            owner.render(record, src, dst, stream=stream)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    launches = int(lib.fjb_kernel_launches()) - launches0
    times = abi.FjbStageTimes()
    lib.fjb_owner_stage_times(owner.handle, C.byref(times), C.byref(err.buf))
    lib.fjb_owner_stage_timing(owner.handle, 0, C.byref(err.buf))
    barrier()
    ms = max_over_ranks(start.elapsed_time(end) / args.steps)
    px = W * H
    value = world * px / (ms * 1e-3) / 1e6
    stages = {}
    for i, name in enumerate(abi.FJB_STAGE_NAMES):
        if times.frames[i]:
            stages[name] = round(times.total_ms[i] / times.frames[i], 4)

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
        models = stage_models(record)
        # roofline of the stage that takes the most device time
        dominant = max((k for k in stages if k in models), key=lambda k: stages[k])
        kind, per_px = models[dominant]
        stage_s = stages[dominant] * 1e-3
        if kind == "hbm":
            achieved = px * per_px / stage_s / 1e9
            roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                    "frac": round(achieved / pk["hbm_gbs"], 4), "peak_source": pk_kind}
        else:
            # FP32 FMA pipe: 148 SMs x 128 lanes x 2 FLOP per clock at the sampled SM clock
            sm_mhz = clk.get("sm_mhz") or 1965.0
            peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
            achieved = px * per_px / stage_s / 1e12
            roof = {"bound": "fp32", "achieved": round(achieved, 2), "peak": round(peak, 1), "unit": "TFLOP/s",
                    "frac": round(achieved / peak, 4),
                    "peak_source": "nominal FP32 FMA rate at the sampled SM clock (no tensor or HBM bound applies)"}
        roof["kernel_stage"] = dominant
        roof["stage_ms"] = stages[dominant]
        traffic = None
        prof = os.path.join(ROOT, "profiles", "frame_stages_4k.json")
        if os.path.exists(prof):
            with open(prof) as fh:
                traffic = json.load(fh).get(dominant, {}).get("dram_bytes_per_launch")
        roof["traffic"] = traffic
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{W}x{H} full optical print through fj_cuda_render"
                                   + (" + highlight reconstruction + scanner post effects + film/gate defects and weave"
                                      if args.next_rows else ""),
                       "recipe": "kodak_portra_400 -> kodak_portra_endura, Hanatos TC LUT, spatial DIR tail 200 um "
                                 "w 0.03, camera diffusion r=0.5% W, scatter/halation, grain 35 mm, scanner LUT r=17, "
                                 "OkLch gamut, sRGB",
                       "frame_bytes": px * 12, "l2_policy": "inputs larger than L2 (99.5 MB frame in and out, "
                                                           "~0.7 GB of stage planes per frame)",
                       "parallelism": f"replicas x{world}"},
            "stages_ms": stages,
            "roofline": roof,
            "cpu_baseline": cpu_baseline(args.cpu_seconds) if world == 1 and args.cpu_seconds > 0 else None,
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
    t0 = time.perf_counter()
    want, _ = oframe.render_frame(record, recipe, host, threads=os.cpu_count() or 1)
    t_oracle = time.perf_counter() - t0
    stats = color.delta_e_stats(got, want)
    line = {"precision": {"workload": f"{W}x{H} full optical print through fj_cuda_render", "dtype": "f32",
                          "delta_e00_vs_oracle": {k: round(v, 6) for k, v in stats.items()},
                          "max_abs_encoded": float(np.abs(got - want).max()),
                          "mean_abs_encoded": float(np.abs(got - want).mean()),
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
