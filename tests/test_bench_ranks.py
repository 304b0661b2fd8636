"""bench.py's multi-rank bookkeeping on CPU: two gloo ranks with different
timed regions agree on the slowest one, and the whole-job rate counts every
rank's frames (one replica per rank, no collective on the data path)."""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(100.0 + 25.0 * rank, dist, "cpu")
        out.put((rank, ms, bench.whole_job_rate(320, world, ms)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank_and_count_all_frames():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [125.0, 125.0]
    assert all(abs(r[2] - 2 * 320 / 0.125) < 1e-6 for r in results)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(REPO))
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_rate(16, 1, 20.0) == 800.0


def test_extras_option_rejects_unknown_names():
    """`--extras` takes a comma-separated subset of the extra workloads and
    refuses a name outside them before any device work."""
    import subprocess

    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--extras", "learned,nosuch"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "unknown extras ['nosuch']" in r.stderr
    sys.path.insert(0, str(REPO))
    import bench

    assert set(bench.EXTRAS) == {"reference_device", "distances", "learned", "mixed64", "serving"}


def test_streams_option_is_bounded_by_the_step():
    """Every encoder stream takes its own frames of the step, so `--streams`
    above the step's frame count is refused before any device work."""
    import subprocess

    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--streams", "24"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "--streams must be 1..16, got 24" in r.stderr


def test_reference_arm_prints_the_contract_line():
    """`--impl reference` times the CPU restatement on the host cores and
    prints one JSON line with the same metric as the GPU arm, a
    cpu_baseline describing the run and an e2e block without copies."""
    import json
    import subprocess

    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "4K frames/s" and line["unit"] == "frames/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["n_gpus"] == 1
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "frames/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
