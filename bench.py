#!/usr/bin/env python3
"""Benchmark: frames/s of the splat frame pipeline at 1M splats, SH degree 3, 1920x1080.

A step renders one frame of a 120-frame orbit (radius 15 m, 3 degrees per frame) of a seeded
1M-splat SH3 scene through the C ABI: cull + project + SH + depth key, depth radix sort,
tile binning, stable tile sort, composite. The L2 is flushed (256 MiB memset) before every
step and each frame is timed on the device with CUDA events recorded on the renderer's own
stream. `e2e` repeats the steps through the public call a user makes (draw, then read the
RGBA8 image into pinned host memory) and times the host loop.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--bits 16|32] [--impl ours|reference]

N > 1 runs one independent replica per GPU (torchrun, one rank per GPU): the frame path has
no exchange step, so there is no collective in the data path; the max of the per-rank device
times gives the job time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "splatkit-ios_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "frames/s @1M-splat SH3 1080p"
SPLATS, WIDTH, HEIGHT, SH_DEGREE = 1_000_000, 1920, 1080, 3
ORBIT_FRAMES = 120
L2_FLUSH_BYTES = 256 << 20


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--bits", type=int, default=16, choices=(16, 32))
    p.add_argument("--impl", default="ours", choices=("ours", "reference"))
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batch", action="store_true", help="skip the 64-view batched comparison")
    p.add_argument("--no-serve", action="store_true", help="skip the serving comparison")
    p.add_argument("--no-lod", action="store_true", help="skip the LOD walk")
    p.add_argument("--sort-large-only", action="store_true",
                   help="only the 40M-key argsort measurement (one JSON object), e.g. as a profiling target")
    return p.parse_args(argv)


def workload_config(bits):
    return {"workload": f"{SPLATS // 1000}k-splat SH{SH_DEGREE} {WIDTH}x{HEIGHT}, {ORBIT_FRAMES}-frame "
                        "orbit r=15 m, one frame per step (plain per-frame path)",
            "splats": SPLATS, "sh_degree": SH_DEGREE, "width": WIDTH, "height": HEIGHT,
            "key_bits": bits, "scene": "synthetic PCG64 seed 0: positions U[-10,10]^3, "
            "log-scales N(-3,0.5), opacity sigmoid(N(0,1)), SH bands N(0,0.1)",
            "l2": "flushed between timed steps (256 MiB memset)", "parallelism": "replicas"}


def frame_inputs(step):
    from splatkit_b200 import camera

    view, eye = camera.orbit_view(step % ORBIT_FRAMES, radius=15.0, degrees_per_frame=3.0)
    proj = camera.perspective(math.radians(60.0), WIDTH / HEIGHT, 0.05, 200.0)
    return view, proj, eye


# ---- clocks sampled during the timed region ---------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.time() + 5.0  # the first sample arrives after nvidia-smi starts
            while not self.lines and time.time() < deadline:
                time.sleep(0.02)
            self.lines.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- algorithmic bytes per stage ---------------------------------------------------------------
def stage_bytes(stats, bits, n=SPLATS, width=WIDTH, height=HEIGHT, sh_words=24):
    v, inst, read = stats["draw_count"], stats["instances"], stats["instances_read"]
    cells = ((width + 31) // 32) * ((height + 31) // 32)
    blocks = (v + 1023) // 1024
    return {
        # 32 B record per source splat, the SH record (96 B at SH3, device stride) of each
        # survivor, then a 4 B key, a 32 B projected record and a 16 B tile span per survivor
        "cull": 32 * n + 4 * sh_words * v + 52 * v,
        # per pass read key(+value) and write key+value, the last pass skipping the key write (the
        # digit histogram is summed by the cull as it writes the keys): 56 B/key at 32 bits,
        # 24 B/key at 16 bits
        "sort": (56 if bits == 32 else 24) * v,
        # direct cell lists: count and emit each read order + span (20 B per survivor); the
        # per-block cell counts are written, read and turned into block starts (read again by
        # the emission): 3 x 4 B per (block, cell); 8 B range per cell; 4 B written per entry
        "bin": 40 * v + 12 * blocks * cells + 8 * cells + 4 * inst,
        # index + projected record per list entry read, RGBA8 image write
        "composite": 36 * read + width * height * 4,
    }


def traffic_from_profiles(stem):
    """DRAM bytes per launch from the committed ncu summary of this kernel, when present."""
    path = ROOT / "profiles" / f"{stem}.md"
    if path.exists():
        m = re.search(r"dram_bytes_per_launch_full_size:\s*([0-9.eE+]+)", path.read_text())
        if m:
            return float(m.group(1))
    return None


def instructions_from_profiles(stem):
    """Warp instructions per launch from the committed ncu summary of this kernel, when present."""
    path = ROOT / "profiles" / f"{stem}.md"
    if path.exists():
        m = re.search(r"warp instructions \(`smsp__inst_executed.sum`\) \| ([0-9.eE+]+)", path.read_text())
        if m:
            return float(m.group(1))
    return None


def issue_roofline(instructions, ms, sm_mhz, sms=148, schedulers=4):
    """The dominant kernel against instruction issue, the bound that applies to it: warp
    instructions per launch (its ncu summary) / live duration, against one warp instruction per
    scheduler per clock at the sampled SM clock."""
    if not instructions or not ms or not sm_mhz:
        return None
    achieved = instructions / (ms / 1000.0)
    peak = sms * schedulers * sm_mhz * 1e6
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "warp inst/s",
            "frac": achieved / peak, "instructions_per_launch": instructions}


def measured_peaks():
    """The HBM copy bandwidth measured on this pool's GPUs (GB/s) when the peaks file is present
    and readable, else the earlier measurement of 6650 GB/s."""
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(path.read_text())
        v = d["hbm_gbs"]
        if isinstance(v, dict):  # a record with its statistics
            v = next(v[k] for k in ("value", "median", "mean", "gbs") if k in v)
        v = float(v)
        if v > 0:
            return v, "measured"
    except (OSError, ValueError, KeyError, TypeError, StopIteration):
        pass
    return 6650.0, "fallback"


# ---- CPU baseline (oracle port of the path, all host threads) ----------------------------------
# ---- replicas (one process per GPU, no exchange step) ------------------------------------------
def replica_frame(step, rank):
    """The orbit frame a replica draws at a step: ranks start 37 frames apart."""
    return step + rank * 37


def max_over_ranks(value, world, device="cpu"):
    """The largest of every rank's value (the job's time is its slowest rank's); one rank: itself."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(steps, world, seconds):
    """Whole-job frames/s: every rank drew `steps` frames within the slowest rank's time."""
    return steps * world / seconds


def cpu_frame(cloud_packed, sh_packed, sh_stride, view, proj, eye, bits, threads, width=WIDTH,
              height=HEIGHT):
    from oracle.oracle import Oracle

    o = Oracle()
    cam = o.camera(view, proj, eye, width, height, 1.0)
    t0 = time.perf_counter()
    keys, pr = o.visibility(cam, cloud_packed, sh_packed, sh_stride, SH_DEGREE, bits,
                            [(0, len(cloud_packed))], threads=threads)
    t1 = time.perf_counter()
    order = o.radix_argsort(keys, bits, threads=threads)
    t2 = time.perf_counter()
    o.composite(pr, order, width, height, precision=32, threads=threads)
    t3 = time.perf_counter()
    return {"cull": t1 - t0, "sort": t2 - t1, "composite": t3 - t2, "total": t3 - t0,
            "visible": len(keys)}


def reference_packed_scene():
    """The workload's cloud packed by the reference's own packSplatRange / packShRange
    (splatkit-engine/src/rendering/GpuLayout.cpp:92-137, compiled into oracle/_ref): the CPU arm
    maps no library of the product. None when oracle/_ref is not built."""
    from oracle import oracle as oracle_mod
    from splatkit_b200 import synthetic  # numpy only: the product library stays unloaded

    if not oracle_mod.reference_available():
        return None
    ref = oracle_mod.Reference()
    cloud = synthetic.random_cloud(SPLATS, seed=0, sh_degree=SH_DEGREE)
    return ref.pack_splats(cloud), ref.pack_sh(cloud, SH_DEGREE), ref.sh_stride(SH_DEGREE)


def run_reference(args):
    """The reference arm: the reference has no CPU frame path (its frame runs only as Metal
    shaders), so it is the oracle port of the frame path (cull, LSD radix sort, FP32 composite) on
    every host core, fed the reference's own packed records."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    scene = reference_packed_scene()
    if scene is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's C++ "
                          "packing) is not built"}), flush=True)
        return
    packed, sh, stride = scene
    for step in range(args.warmup):
        cpu_frame(packed, sh, stride, *frame_inputs(step), args.bits, threads)
    times = []
    for step in range(args.steps):
        times.append(cpu_frame(packed, sh, stride, *frame_inputs(args.warmup + step), args.bits,
                               threads)["total"])
    total = sum(times)
    value = args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.bits),
            "cpu_baseline": {"value": value, "unit": "frames/s", "cores": threads, "kind": "port",
                             "sample": "every step is one full frame of the workload: cull "
                                       "1M splats (records packed by the reference's C++), LSD "
                                       "radix sort, FP32 composite 1920x1080"},
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---- our arm -----------------------------------------------------------------------------------
def run_ours(args):
    import torch

    import splatkit_b200 as sk
    from splatkit_b200 import synthetic

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    device = local if world > 1 else 0
    torch.cuda.set_device(device)

    cloud = synthetic.random_cloud(SPLATS, seed=0, sh_degree=SH_DEGREE)
    r = sk.Renderer(WIDTH, HEIGHT, device=device, image_format=sk.FORMAT_RGBA8, time_stages=True)
    r.apply_render_policy(sk.Policy(sort_depth_bits=args.bits))
    r.upload_world(cloud, SH_DEGREE)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{device}")

    def frame(step):
        view, proj, eye = frame_inputs(replica_frame(step, rank))
        r.draw(sk.Frame(view, proj, eye, [(0, SPLATS)], SH_DEGREE))

    for step in range(args.warmup):
        frame(step)
        r.wait_idle()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()

    stage_names = ("cull_ms", "sort_ms", "bin_ms", "composite_ms")
    per_frame, stages, stats_list = [], {k: [] for k in stage_names}, []
    # clocks are sampled over both timed loops (device-timed steps, then e2e)
    clocks = ClockSampler(device).__enter__()
    # the headline loop records only the frame's own events, so the stage kernels stay chained
    r.set_timing("frame")
    for step in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        frame(args.warmup + step)
        r.wait_idle()
        s = r.stats()
        per_frame.append(s["gpu_ms"])
        stats_list.append(s)
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(per_frame), world, f"cuda:{device}")
    if world > 1:
        torch.distributed.barrier()
    value = aggregate_rate(args.steps, world, total_ms / 1000.0)
    # the same frames again with an event pair around every stage, for the per-stage roofline
    r.set_timing(True)
    stage_stats = []
    for step in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        frame(args.warmup + step)
        r.wait_idle()
        s = r.stats()
        for k in stage_names:
            stages[k].append(s[k])
        stage_stats.append(s)  # fragments are counted in this pass only
    torch.cuda.synchronize()

    # the other depth-key width on the same frames (the workload compares 16- and 32-bit keys):
    # frame-timed, then per stage; the headline line's own width is restored afterwards
    other_bits = 32 if args.bits == 16 else 16
    other = time_key_width(r, frame, flush, other_bits, min(args.steps, 100), args.warmup)
    r.apply_render_policy(sk.Policy(sort_depth_bits=args.bits))

    # e2e: the public calls with every frame's image landing in pinned host memory, host-timed.
    # captureNextFrame form: each step requests the capture of its frame and draws it, then waits
    # for the previous step's image, whose copy overlapped this frame's drawing.
    # no GPU timing here: an application after throughput records no events (per-frame events
    # cost the pipelined loop about 10%)
    r.set_timing(False)
    host_images = [torch.empty((HEIGHT, WIDTH, 4), dtype=torch.uint8, pin_memory=True).numpy()
                   for _ in range(2)]
    def e2e_loop(first, steps):
        previous = None
        for step in range(steps):
            ticket = r.capture_next_frame(host_images[step % 2])
            frame(first + step)
            if previous is not None:
                r.wait_capture(previous)
            previous = ticket
        r.wait_capture(previous)
    e2e_loop(0, 3)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    e2e_loop(args.warmup, args.steps)
    e2e_s = time.perf_counter() - t0
    # the blocking form for comparison: draw, then read the image back before the next draw
    t0 = time.perf_counter()
    for step in range(args.steps):
        frame(args.warmup + step)
        r.read_image(sk.FORMAT_RGBA8, out=host_images[0])
    blocking_s = time.perf_counter() - t0
    clocks.__exit__(None, None, None)
    e2e_s = max_over_ranks(e2e_s, world, f"cuda:{device}")
    blocking_s = max_over_ranks(blocking_s, world, f"cuda:{device}")
    e2e_value = aggregate_rate(args.steps, world, e2e_s)
    blocking_value = aggregate_rate(args.steps, world, blocking_s)

    if rank == 0:
        mean = {k: float(np.mean(v)) for k, v in stages.items()}
        last = stats_list[-1]
        bytes_by_stage = {k: float(np.mean([stage_bytes(s, args.bits)[k] for s in stats_list]))
                          for k in ("cull", "sort", "bin", "composite")}
        dominant = max(("cull", "sort", "bin", "composite"), key=lambda k: mean[k + "_ms"])
        peak, peak_kind = measured_peaks()
        achieved = bytes_by_stage[dominant] / (mean[dominant + "_ms"] / 1000.0) / 1e9
        kernel_tag = {"cull": "visibility", "sort": "radix_sort", "bin": "cell_lists",
                      "composite": "composite"}[dominant]
        profile = {"cull": "visibility_1m_sh3_1080p", "sort": "radix_sort_scatter_depth_1m_sh3_1080p",
                   "bin": "cell_lists_emit_1m_sh3_1080p", "composite": "composite_1m_sh3_1080p"}[dominant]
        traffic = traffic_from_profiles(profile) if args.bits == 16 else None
        passes = 2 if args.bits == 16 else 4
        # visibility (with the depth keys' digit histogram), the depth sort's scatter passes, cell
        # lists (count, scan, emit), composite
        launches_per_frame = 1 + passes + 3 + 1
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(args.bits),
            "roofline": {"bound": "hbm", "kernel": kernel_tag, "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": bytes_by_stage[dominant],
                         "profile": f"profiles/{profile}.md"},
            "issue_roofline": issue_roofline(instructions_from_profiles(profile) if args.bits == 16 else None,
                                             mean[dominant + "_ms"], clocks.summary().get("sm_mhz")),
            "stages_ms": mean,
            "stage_timing": "a second pass over the same frames with events around each stage and fragment counting",
            "stage_gbs": {k: bytes_by_stage[k] / (mean[k + "_ms"] / 1000.0) / 1e9
                          for k in bytes_by_stage},
            "visible": last["draw_count"], "instances": last["instances"],
            "sort_keys_per_s": last["draw_count"] / (mean["sort_ms"] / 1000.0),
            "fragments_per_s": float(np.mean([s["fragments"] for s in stage_stats])) /
            (mean["composite_ms"] / 1000.0),
            "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": 208,
                    "d2h_bytes_per_step": WIDTH * HEIGHT * 4 + 64,
                    "how": "per step capture_next_frame into pinned memory + draw (camera 208 B "
                           "up), then wait for the previous step's image (8.3 MB down, copied "
                           "while this frame draws); the two frames in flight run on the "
                           "context's two frame streams and overlap on the device; no GPU "
                           "timing events; host-timed",
                    "blocking_read_image_frames_per_s": blocking_value},
            "clocks": clocks.summary(),
            "gpu_launches": launches_per_frame * args.steps,
        }
        line[f"bits{other_bits}"] = other
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.bits, args.warmup - 1, args.warmup)
        if world == 1 and not args.no_batch and args.bits == 16:
            line["batch64"] = measure_batch(r)
            line["sort_large"] = measure_sort_large()
        if world == 1 and not args.no_lod and args.bits == 16:
            line["lod_walk"] = measure_lod_walk()
        if world == 1 and not args.no_serve and args.bits == 16:
            line["served"] = measure_serve()
            line["served_lod"] = measure_serve_lod()
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def time_key_width(r, frame, flush, bits, steps, warmup):
    """Frames/s, per-stage device ms and GB/s, and sort keys/s of the workload with `bits`-bit
    depth keys: the same orbit frames as the headline loop, L2 flushed before each."""
    import torch

    import splatkit_b200 as sk

    r.apply_render_policy(sk.Policy(sort_depth_bits=bits))
    for step in range(3):
        frame(step)
        r.wait_idle()
    stage_names = ("cull_ms", "sort_ms", "bin_ms", "composite_ms")
    per_frame, stats_list, stages = [], [], {k: [] for k in stage_names}
    for timing in ("frame", True):
        r.set_timing(timing)
        for step in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            frame(warmup + step)
            r.wait_idle()
            s = r.stats()
            if timing == "frame":
                per_frame.append(s["gpu_ms"])
                stats_list.append(s)
            else:
                for k in stage_names:
                    stages[k].append(s[k])
    mean = {k: float(np.mean(v)) for k, v in stages.items()}
    bytes_by_stage = {k: float(np.mean([stage_bytes(s, bits)[k] for s in stats_list]))
                      for k in ("cull", "sort", "bin", "composite")}
    visible = float(np.mean([s["draw_count"] for s in stats_list]))
    return {"key_bits": bits, "steps": steps, "value": steps / (sum(per_frame) / 1000.0),
            "unit": "frames/s", "ms_per_step": float(np.mean(per_frame)), "stages_ms": mean,
            "stage_gbs": {k: bytes_by_stage[k] / (mean[k + "_ms"] / 1000.0) / 1e9
                          for k in bytes_by_stage},
            "sort_algorithmic_bytes": bytes_by_stage["sort"],
            "sort_keys_per_s": visible / (mean["sort_ms"] / 1000.0),
            "how": "device time per frame (frame events), then a second pass with per-stage "
                   "events; L2 flushed before every frame"}


def measure_sort_large(keys_n=40_000_000, reps=20):
    """The depth sort where HBM can bind: the argsort operator (sk_radix_argsort_device) over 40M
    keys (160 MB, above the 126 MB L2), 16-bit and 32-bit keys, device time per call with CUDA
    events on the sort's stream. Algorithmic bytes per key: 4 (one all-digit histogram read) + 12
    (first pass: read the key, write key and value) + 16 per middle pass + 12 (last pass, no key
    write): 28 B at 16 bits, 60 B at 32."""
    import torch

    import splatkit_b200 as sk

    dev = torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(40)
    out = {}
    peak, peak_kind = measured_peaks()
    for bits, per_key in ((16, 28), (32, 60)):
        hi = 1 << bits
        keys = torch.randint(0, hi, (keys_n,), device=dev, generator=gen, dtype=torch.int64)
        keys = (keys - (1 << 31) if bits == 32 else keys).to(torch.int32)
        count = torch.tensor([keys_n], dtype=torch.int32, device=dev)
        order = torch.empty(keys_n, dtype=torch.int32, device=dev)
        ws = torch.zeros(sk.sort_workspace_bytes(keys_n), dtype=torch.uint8, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream().cuda_stream
        sort_bits = bits

        def call():
            sk.radix_argsort_device(keys.data_ptr(), count.data_ptr(), keys_n, sort_bits, order.data_ptr(),
                                    ws.data_ptr(), ws.numel(), err.data_ptr(), stream)

        for _ in range(3):
            call()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(reps):
            call()
        end.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(end) / reps
        # spot check: the order sorts the keys stably
        k = keys.cpu().numpy().view(np.uint32)
        o = order.cpu().numpy()
        sorted_ok = bool(np.all(np.diff(k[o].astype(np.int64)) >= 0)) and int(err.item()) == 0
        gbs = per_key * keys_n / (ms / 1000.0) / 1e9
        out[f"bits{bits}"] = {"ms": ms, "keys_per_s": keys_n / (ms / 1000.0), "algorithmic_bytes_per_key": per_key,
                              "gbs": gbs, "frac": gbs / peak, "sorted": sorted_ok}
        del keys, order, ws
    out["peak_gbs"] = peak
    out["peak_kind"] = peak_kind
    out["workload"] = f"{keys_n} uniform random keys, stable argsort, {reps} back-to-back calls"
    return out


# ---- batched multi-view: 64 views of the 1M SH3 scene, mixed resolutions ----------------------
BATCH_VIEWS = 64
BATCH_SIZES = [(640, 480), (1280, 720), (1920, 1080)]


def batch_views(renderer, rotation_deg=0.0):
    import splatkit_b200 as sk
    from splatkit_b200 import camera as skcam

    rng = np.random.default_rng(64)
    sizes = [BATCH_SIZES[i] for i in rng.integers(0, len(BATCH_SIZES), BATCH_VIEWS)]
    views = []
    for i, (w, h) in enumerate(sizes):
        a = math.radians(360.0 * i / BATCH_VIEWS + rotation_deg)
        eye = np.array([15.0 * math.sin(a), 0.0, 15.0 * math.cos(a)], np.float32)
        view = skcam.look_at_view(eye, (0.0, 0.0, 0.0))
        proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 200.0)
        views.append(sk.BatchView(renderer, sk.Frame(view, proj, eye, [(0, SPLATS)], SH_DEGREE), w, h))
    return views


def measure_batch(renderer):
    """64 plain per-frame launches (draw + read back each) against the batched form (graph-captured
    submissions on two lanes, every image read back), same views, images compared bit for bit."""
    import torch

    import splatkit_b200 as sk

    views = batch_views(renderer)
    pinned = torch.empty(1920 * 1080 * 4, dtype=torch.uint8, pin_memory=True).numpy()
    plain_images = []
    for rounds in range(2):
        t0 = time.perf_counter()
        for v in views:
            renderer.resize(v.width, v.height)
            renderer.draw(v.frame)
            renderer.read_image(sk.FORMAT_RGBA8,
                                out=pinned[:v.width * v.height * 4].reshape(v.height, v.width, 4))
        plain_s = time.perf_counter() - t0
    for v in views:  # the reference images, outside the timed rounds
        renderer.resize(v.width, v.height)
        renderer.draw(v.frame)
        plain_images.append(renderer.read_image(sk.FORMAT_RGBA8))
    rounds = 8
    with sk.Batch(lanes=3, max_views=BATCH_VIEWS, use_graphs=True) as batch:
        tuning = batch.autotune(views)
        for k in range(2):
            batch.wait(batch.submit(batch_views(renderer, k)))
        t0 = time.perf_counter()
        tickets = [batch.submit(batch_views(renderer, k % 3)) for k in range(rounds)]
        for t in tickets[-int(tuning["lanes"]):]:  # each lane's last submission
            batch.wait(t)
        batch_s = time.perf_counter() - t0
        gpu_ms = batch.stats(tickets[-1])["gpu_ms"]
        check = batch.submit(views)
        same = all(np.array_equal(batch.read_image(check, i), plain_images[i]) for i in range(len(views)))
    plain_rate = len(views) / plain_s
    batch_rate = rounds * len(views) / batch_s
    return {"workload": "64 views of the 1M-splat SH3 scene on a 15 m circle, resolutions drawn "
                        "from {640x480, 1280x720, 1920x1080} (seed 64)",
            "plain_views_per_s": plain_rate, "batched_views_per_s": batch_rate,
            "speedup": batch_rate / plain_rate, "batched_gpu_ms_per_submission": gpu_ms,
            "images_identical": bool(same), "autotuned": tuning,
            "how": "plain: resize + draw + read_image per view; batched: autotuned (cell-list "
                   "construction, emission, radix tile, lanes of 3), then 8 submissions of 64 views, "
                   "CUDA-graph replay, every image copied back; host-timed"}


# ---- LOD walk: 6M leaves in 2000 clusters, 300 frames at 1920x1080 ----------------------------
def tree_build_call_seconds(sk, cloud, entry, reps=3):
    """Median time of one C-ABI tree build (with selection data) through `entry`, the tree freed
    after each call: the build alone, without the Python copies of the result."""
    import ctypes
    lib = sk.library()
    view = cloud.view()
    lo = np.ascontiguousarray(cloud.bounds_min, np.float32)
    hi = np.ascontiguousarray(cloud.bounds_max, np.float32)
    f32p = ctypes.POINTER(ctypes.c_float)
    times = []
    for _ in range(reps):
        handle = ctypes.c_void_p()
        t0 = time.perf_counter()
        st = getattr(lib, entry)(ctypes.byref(view), lo.ctypes.data_as(f32p), hi.ctypes.data_as(f32p),
                                 0, 0, 1, ctypes.byref(handle))
        times.append(time.perf_counter() - t0)
        if st != sk.SK_OK:
            raise sk.SplatError(st, entry)
        lib.sk_lod_tree_free(handle)
    return float(np.median(times))


def measure_lod_walk():
    """The LOD workload: 2000 anisotropic clusters of 3000 splats (centres in a 200 m box), the
    tree built on the GPU by the project's builder (the reference builder's layout), cut at
    1.5 px along a 300-frame walk (eye height 1.7 m, x from -90 to 90 m, looking +x)."""
    import splatkit_b200 as sk
    from splatkit_b200 import camera as skcam
    from splatkit_b200 import synthetic

    cloud = synthetic.clustered_cloud(2000, 3000, seed=0)
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min, cloud.bounds_max = pos.min(axis=0), pos.max(axis=0)
    sk.build_lod_tree(synthetic.random_cloud(1000, seed=1))  # loads the module
    t0 = time.perf_counter()
    tree = sk.build_lod_tree(cloud)
    build_s = time.perf_counter() - t0
    c_call_s = tree_build_call_seconds(sk, cloud, "sk_build_lod_tree_device")
    r = sk.Renderer(WIDTH, HEIGHT, image_format=sk.FORMAT_RGBA8, time_stages=True)
    r.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16))
    r.upload_lod_world(tree, 0, 4_000_000)
    proj = skcam.perspective(math.radians(60.0), WIDTH / HEIGHT, 0.05, 400.0)

    def frame(i):
        x = -90.0 + 180.0 * i / 299
        eye = np.array([x, 1.7, 0.0], np.float32)
        r.draw(sk.Frame(skcam.look_at_view(eye, (x + 10.0, 1.7, 0.0)), proj, eye, [], 0))

    for i in range(5):
        frame(i)
        r.wait_idle()
    gpu_ms, select_ms, cut = [], [], []
    for i in range(300):
        frame(i)
        r.wait_idle()
        s = r.stats()
        gpu_ms.append(s["gpu_ms"])
        select_ms.append(s["select_ms"])
        cut.append(s["selected_count"])
    r.close()
    return {"workload": "6M leaves (2000 clusters x 3000), GPU-built tree of "
                        f"{len(tree.layout)} nodes, 1.5 px cut, 300-frame walk at 1920x1080",
            "frames_per_s": 300 / (sum(gpu_ms) / 1000.0), "mean_gpu_ms": float(np.mean(gpu_ms)),
            "mean_select_ms": float(np.mean(select_ms)), "mean_cut_splats": float(np.mean(cut)),
            "tree_build_s": build_s, "tree_build_c_call_s": c_call_s,
            "tree_build_how": "tree_build_s: Python build_lod_tree with selection data (node arrays "
                              "returned as views); tree_build_c_call_s: the C-ABI call alone "
                              "(median of 3): keys, sort, levels and merges on the GPU, selection "
                              "data on the host threads"}


# ---- serving: Poisson requests over 8 resident scenes -----------------------------------------
SERVE_SCENES = [200_000, 500_000, 1_000_000, 2_000_000, 3_000_000, 4_000_000, 5_000_000, 6_000_000]
SERVE_SIZES = [(640, 480), (1280, 720), (1920, 1080), (2560, 1440), (3840, 2160)]


def serve_trace(count, rate, seed=2000):
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1e6 / rate, count))
    return arrivals, rng.integers(0, len(SERVE_SCENES), count), rng.integers(0, len(SERVE_SIZES), count), \
        rng.uniform(0.0, 360.0, count)


def run_served(renderers, frames, arrivals, max_queue_ms=0.0, lanes=2, max_batch_views=16,
               max_batch_splats=96_000_000):
    """Replays the trace through the continuous-batching server: completed requests over the wall
    time from the first arrival to the last completion, and the latency percentiles. One untimed
    replay of the same trace first, so that the lanes have grown to the trace's batches."""
    import splatkit_b200 as sk

    ring = [sk.HostImage(3840, 2160) for _ in range(96)]
    reqs = [sk.Request(scene, f, w, h, ring[i % len(ring)]) for i, (scene, f, w, h) in enumerate(frames)]
    with sk.Server(lanes=lanes, max_batch_views=max_batch_views, max_batch_splats=max_batch_splats,
                   max_queue_ms=max_queue_ms) as server:
        for r in renderers:
            server.add_scene(r)
        server.replay(reqs, arrivals)
        t0 = time.perf_counter()
        done = server.replay(reqs, arrivals)
        elapsed = time.perf_counter() - t0
    for x in ring:
        x.close()
    ok = [c for c in done if c["status"] == 0]
    lat = np.array([c["latency_ms"] for c in ok]) if ok else np.zeros(1)
    return {"offered_req_per_s": float(len(frames) / (arrivals[-1] * 1e-6)), "requests": len(frames),
            "served": len(ok), "served_req_per_s": len(ok) / elapsed,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_batch_views": float(np.mean([c["batch_views"] for c in ok])) if ok else 0.0}


def run_plain(renderers, frames, arrivals):
    """The same trace through the plain per-frame loop (resize, draw, blocking read back, one
    request at a time as it arrives): completed requests over the wall time from the first
    arrival to the last completion, as for the server, and the loop's busy-time capacity. Like
    the server, the loop first runs the trace once untimed."""
    import splatkit_b200 as sk

    pinned = sk.HostImage(3840, 2160)
    for scene, f, w, h in frames:
        r = renderers[scene]
        r.resize(w, h)
        r.draw(f)
        r.read_image(sk.FORMAT_RGBA8, out=pinned.array.reshape(-1)[:w * h * 4].reshape(h, w, 4))
    lat, busy = [], 0.0
    t0 = time.perf_counter()
    for i, (scene, f, w, h) in enumerate(frames):
        wait = arrivals[i] * 1e-6 - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        r = renderers[scene]
        b0 = time.perf_counter()
        r.resize(w, h)
        r.draw(f)
        r.read_image(sk.FORMAT_RGBA8, out=pinned.array.reshape(-1)[:w * h * 4].reshape(h, w, 4))
        end = time.perf_counter()
        busy += end - b0
        lat.append((end - t0) * 1e3 - arrivals[i] * 1e-3)
    elapsed = time.perf_counter() - t0
    pinned.close()
    lat = np.array(lat)
    return {"offered_req_per_s": float(len(frames) / (arrivals[-1] * 1e-6)), "requests": len(frames),
            "served_req_per_s": len(frames) / elapsed, "capacity_req_per_s": len(frames) / busy,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}


def measure_serve():
    """C5: requests at 2000/s (Poisson) over 8 resident scenes (0.2-6M splats, SH3), resolutions
    640x480..3840x2160, served with continuous batching, against the plain loop on the same trace."""
    import splatkit_b200 as sk
    from splatkit_b200 import camera as skcam
    from splatkit_b200 import synthetic

    renderers = []
    for i, n in enumerate(SERVE_SCENES):
        cloud = synthetic.random_cloud(n, seed=100 + i, sh_degree=SH_DEGREE)
        r = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8, time_stages=False)
        r.apply_render_policy(sk.Policy(sort_depth_bits=16))
        r.upload_world(cloud, SH_DEGREE)
        renderers.append(r)
        del cloud

    def trace(rate, count):
        arrivals, scene, size, angle = serve_trace(count, rate)
        frames = []
        for i in range(count):
            w, h = SERVE_SIZES[size[i]]
            a = math.radians(angle[i])
            eye = np.array([15.0 * math.sin(a), 0.0, 15.0 * math.cos(a)], np.float32)
            proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 200.0)
            f = sk.Frame(skcam.look_at_view(eye, (0.0, 0.0, 0.0)), proj, eye,
                         [(0, SERVE_SCENES[scene[i]])], SH_DEGREE)
            frames.append((int(scene[i]), f, w, h))
        return frames, arrivals

    busy_frames, busy_arrivals = trace(2000.0, 1000)
    light_frames, light_arrivals = trace(200.0, 300)
    out = {"workload": "8 resident scenes of 0.2-6M splats (SH3, 21.7M total), Poisson arrivals, "
                       "resolutions uniform over 640x480..3840x2160, cameras on a 15 m circle",
           "served_2000": run_served(renderers, busy_frames, busy_arrivals),
           "served_2000_shed_8ms": run_served(renderers, busy_frames, busy_arrivals, max_queue_ms=8.0),
           "served_200": run_served(renderers, light_frames, light_arrivals),
           "plain_2000": run_plain(renderers, busy_frames, busy_arrivals),
           "plain_200": run_plain(renderers, light_frames, light_arrivals)}
    out["throughput_vs_plain"] = out["served_2000"]["served_req_per_s"] / out["plain_2000"]["served_req_per_s"]
    out["how"] = ("both arms replay the same seeded trace in real time; req/s = completed requests / "
                  "wall time from the first arrival to the last completion")
    for r in renderers:
        r.close()
    return out


def measure_serve_lod():
    """LOD worlds served: the 6M-leaf walk tree (2000 clusters of 3000 splats, built on the GPU)
    as a resident LOD scene, requests from viewers anywhere on the walk path (eye height 1.7 m,
    x uniform in [-90, 90] m, looking +x), Poisson at 2000/s, resolutions 640x480..3840x2160; every
    request selects its cut (1.5 px, the scene's adaptive threshold carried from request to
    request) on the server's lanes. The plain loop draws the same trace one request at a time."""
    import splatkit_b200 as sk
    from splatkit_b200 import camera as skcam
    from splatkit_b200 import synthetic

    cloud = synthetic.clustered_cloud(2000, 3000, seed=0)
    pos = np.asarray(cloud.positions, np.float32)
    cloud.bounds_min, cloud.bounds_max = pos.min(axis=0), pos.max(axis=0)
    tree = sk.build_lod_tree(cloud)
    del cloud
    scene = sk.Renderer(64, 64, image_format=sk.FORMAT_RGBA8, time_stages=False)
    scene.apply_render_policy(sk.Policy(lod_error_pixels=1.5, sort_depth_bits=16))
    scene.upload_lod_world(tree, 0, 4_000_000)
    del tree
    rng = np.random.default_rng(3000)
    count = 600
    arrivals = np.cumsum(rng.exponential(1e6 / 2000.0, count))
    frames = []
    for i in range(count):
        w, h = SERVE_SIZES[int(rng.integers(0, len(SERVE_SIZES)))]
        x = float(rng.uniform(-90.0, 90.0))
        eye = np.array([x, 1.7, 0.0], np.float32)
        proj = skcam.perspective(math.radians(60.0), w / h, 0.05, 400.0)
        frames.append((0, sk.Frame(skcam.look_at_view(eye, (x + 10.0, 1.7, 0.0)), proj, eye, [], 0), w, h))
    out = {"workload": "the 6M-leaf walk tree as a LOD scene; viewers on the walk path, Poisson 2000/s, "
                       "resolutions uniform over 640x480..3840x2160, 1.5 px cut per request",
           "served_2000": run_served([scene], frames, arrivals, max_batch_splats=200_000_000),
           "plain_2000": run_plain([scene], frames, arrivals)}
    out["throughput_vs_plain"] = out["served_2000"]["served_req_per_s"] / out["plain_2000"]["served_req_per_s"]
    scene.close()
    return out


CPU_BASELINE_FRAMES = 8


def cpu_baseline(bits, warmup, first):
    """The oracle port of the frame path on every host core over the same orbit frames the timed
    loop starts with (one untimed warm-up frame first), records packed by the reference's C++."""
    threads = os.cpu_count() or 1
    scene = reference_packed_scene()
    if scene is None:
        return None
    packed, sh, stride = scene
    cpu_frame(packed, sh, stride, *frame_inputs(warmup), bits, threads)
    runs = [cpu_frame(packed, sh, stride, *frame_inputs(first + k), bits, threads)
            for k in range(CPU_BASELINE_FRAMES)]
    total = sum(t["total"] for t in runs)
    return {"value": CPU_BASELINE_FRAMES / total, "unit": "frames/s", "cores": threads, "kind": "port",
            "sample": f"{CPU_BASELINE_FRAMES} full frames of the workload (orbit frames {first}.."
                      f"{first + CPU_BASELINE_FRAMES - 1}: cull 1M, LSD radix sort, FP32 composite "
                      "1920x1080) on the oracle port, after one warm-up frame",
            "stages_s": {k: float(np.mean([t[k] for t in runs])) for k in ("cull", "sort", "composite")}}


def main():
    args = parse()
    if args.sort_large_only:
        print(json.dumps({"sort_large": measure_sort_large()}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
