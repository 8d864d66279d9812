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


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=60)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--bits", type=int, default=16, choices=(16, 32))
    p.add_argument("--impl", default="ours", choices=("ours", "reference"))
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


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
                 "--format=csv,noheader,nounits", "-lms", "100"],
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
    tiles = ((width + 15) // 16) * ((height + 15) // 16)
    return {
        # 32 B record per source splat, the SH record (96 B at SH3, device stride) of each
        # survivor, then a 4 B key, a 32 B projected record and a 16 B tile span per survivor
        "cull": 32 * n + 4 * sh_words * v + 52 * v,
        # one all-digit histogram read + per pass read key(+value) and write key+value; the
        # last pass skips the key write: 60 B/key at 32 bits, 28 B/key at 16 bits
        "sort": (60 if bits == 32 else 28) * v,
        # count and emit each read order + span (20 B per survivor), emit writes (tile, value);
        # the 16-bit tile sort reads the keys once for its histogram and moves 16 B per
        # instance per pass (sorted keys written too); ranges read the keys, write 8 B per tile
        "bin": 40 * v + 8 * inst + 4 * inst + 32 * inst + 4 * inst + 8 * tiles,
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


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        d = json.loads(path.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- CPU baseline (oracle port of the path, all host threads) ----------------------------------
def cpu_frame(cloud_packed, sh_packed, sh_stride, view, proj, eye, bits, threads, width=WIDTH,
              height=HEIGHT, pixel_rows=None):
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


def run_reference(args):
    """The reference arm: the oracle port of the frame path on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import splatkit_b200 as sk
    from splatkit_b200 import synthetic

    threads = os.cpu_count() or 1
    cloud = synthetic.random_cloud(SPLATS, seed=0, sh_degree=SH_DEGREE)
    packed = sk.pack_splats(cloud)
    sh = sk.pack_sh(cloud, SH_DEGREE)
    stride = sk.sh_device_stride(SH_DEGREE)
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
                                       "1M splats, LSD radix sort, FP32 composite 1920x1080"},
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
        view, proj, eye = frame_inputs(step + rank * 37)
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
    for step in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        frame(args.warmup + step)
        r.wait_idle()
        s = r.stats()
        per_frame.append(s["gpu_ms"])
        for k in stage_names:
            stages[k].append(s[k])
        stats_list.append(s)
    torch.cuda.synchronize()
    total_ms = float(sum(per_frame))
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
        torch.distributed.barrier()
    value = args.steps * world / (total_ms / 1000.0)

    # e2e: the public calls with the image read into pinned host memory, host-timed
    pinned = torch.empty((HEIGHT, WIDTH, 4), dtype=torch.uint8, pin_memory=True)
    host_image = pinned.numpy()
    for step in range(2):
        frame(step)
        r.read_image(sk.FORMAT_RGBA8, out=host_image)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for step in range(args.steps):
        frame(args.warmup + step)
        r.read_image(sk.FORMAT_RGBA8, out=host_image)
    e2e_s = time.perf_counter() - t0
    clocks.__exit__(None, None, None)
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = args.steps * world / e2e_s

    if rank == 0:
        mean = {k: float(np.mean(v)) for k, v in stages.items()}
        last = stats_list[-1]
        bytes_by_stage = {k: float(np.mean([stage_bytes(s, args.bits)[k] for s in stats_list]))
                          for k in ("cull", "sort", "bin", "composite")}
        dominant = max(("cull", "sort", "bin", "composite"), key=lambda k: mean[k + "_ms"])
        peak, peak_kind = measured_peaks()
        achieved = bytes_by_stage[dominant] / (mean[dominant + "_ms"] / 1000.0) / 1e9
        kernel_tag = {"cull": "visibility", "sort": "radix_sort", "bin": "binning",
                      "composite": "composite"}[dominant]
        profile = {"cull": "visibility_1m_sh3_1080p", "sort": "radix_sort_scatter_depth_1m_sh3_1080p",
                   "bin": "binning_emit_1m_sh3_1080p", "composite": "composite_1m_sh3_1080p"}[dominant]
        traffic = traffic_from_profiles(profile) if args.bits == 16 else None
        passes = 2 if args.bits == 16 else 4
        # visibility, depth sort (histogram + passes), bin count + emit, tile sort, ranges, composite
        launches_per_frame = 1 + (1 + passes) + 2 + 3 + 1 + 1
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
            "stages_ms": mean,
            "stage_gbs": {k: bytes_by_stage[k] / (mean[k + "_ms"] / 1000.0) / 1e9
                          for k in bytes_by_stage},
            "visible": last["draw_count"], "instances": last["instances"],
            "sort_keys_per_s": last["draw_count"] / (mean["sort_ms"] / 1000.0),
            "fragments_per_s": float(np.mean([s["fragments"] for s in stats_list])) /
            (mean["composite_ms"] / 1000.0),
            "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": 8,
                    "d2h_bytes_per_step": WIDTH * HEIGHT * 4 + 64},
            "clocks": clocks.summary(),
            "gpu_launches": launches_per_frame * args.steps,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(cloud, args.bits)
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def cpu_baseline(cloud, bits):
    import splatkit_b200 as sk

    threads = os.cpu_count() or 1
    packed = sk.pack_splats(cloud)
    sh = sk.pack_sh(cloud, SH_DEGREE)
    t = cpu_frame(packed, sh, sk.sh_device_stride(SH_DEGREE), *frame_inputs(0), bits, threads)
    return {"value": 1.0 / t["total"], "unit": "frames/s", "cores": threads, "kind": "port",
            "sample": "one full frame of the workload (cull 1M, radix sort, FP32 composite "
                      "1920x1080) on the oracle port",
            "stages_s": {k: t[k] for k in ("cull", "sort", "composite")}}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
