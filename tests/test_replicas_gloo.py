"""The bench's replica plumbing on two CPU ranks (gloo): the job time is the slowest rank's, the
aggregate rate counts every rank's frames, ranks draw different frames, and the reference arm
runs on rank 0 only, and the HBM peak is read from the peaks file when it is there. Frames are
independent, so there is no data-path collective to test."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_seconds = [2.0, 5.0][rank]
        slowest = bench.max_over_ranks(local_seconds, world)
        frames = [bench.replica_frame(step, rank) for step in range(10)]
        out.put((rank, slowest, bench.aggregate_rate(10, world, slowest), frames))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_draw_different_frames():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, slow0, rate0, frames0), (r1, slow1, rate1, frames1) = results
    assert slow0 == slow1 == 5.0
    assert rate0 == rate1 == pytest.approx(10 * 2 / 5.0)
    assert not set(frames0) & set(frames1)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    args = bench.parse(["--impl", "reference", "--steps", "1", "--warmup", "0"])
    bench.run_reference(args)  # returns at once on a non-zero rank
    assert capsys.readouterr().out == ""


def test_peaks_file_is_read_when_present_and_readable(tmp_path, monkeypatch):
    import bench
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_peaks() == (6650.0, "fallback")  # absent
    for text, expected in [('{"hbm_gbs": 7100.5}', (7100.5, "measured")),
                           ('{"hbm_gbs": {"value": 7000}}', (7000.0, "measured")),
                           ('{"bf16_tflops": 1590}', (6650.0, "fallback")),
                           ("not json", (6650.0, "fallback"))]:
        (tmp_path / "MEASURED_PEAKS.json").write_text(text)
        assert bench.measured_peaks() == expected
