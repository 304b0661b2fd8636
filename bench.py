#!/usr/bin/env python
"""4K NV12 -> JPEG XL VarDCT encode throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--streams S]

Workload: the seeded synthetic 3840x2160 NV12 frame (seed 0), distance 1.0,
the plain path (XYB, AQ, gaborish, transform selection, DCT, CfL, quantise,
histograms, prefix codes, packing, headers). One step encodes a batch of 16
device-resident copies of that frame, frame i on encoder i % S (S encoders,
each with its own CUDA stream and device arena, default 4); the 16 distinct
input buffers (199 MB) exceed the 126 MB L2, so no step reads its input from
L2.

value: frames/s over exactly K steps, CUDA events (start on the first
encoder's stream, the others wait on it and are joined back before the stop
event), barrier + synchronize on both sides, max over ranks (one process per
GPU, independent replicas: frames do not shard, so there is no collective).
p50/p99 frame latency and the frontend/entropy split: one encoder alone,
events around each stage of each frame.
e2e: the same metric through the public C ABI with host buffers, one host
thread per encoder: every frame is copied host->device from pinned memory,
encoded with cujpegxl_encoder_encode and its file copied back to pinned host
memory.
roofline: the fused frontend kernel, its algorithmic bytes per 4K frame over
its event-timed duration, against the measured HBM copy bandwidth.
--impl reference: the CPU encoder restated from the reference (the reference
has no CPU implementation of its device stages) run with every host core on
the same frame, rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

W_4K, H_4K = 3840, 2160
BATCH = 16
PUBLISHED_FPS = 15.0  # reference README.md:17, GTX 1080 Ti, 4K sustained


def frontend_algorithmic_bytes(w: int, h: int) -> int:
    """NV12 in; int16 AC, int32 DC, acs, int32 quant field, CfL maps out."""
    p = w * h
    b = p // 64
    t = ((w // 8 + 7) // 8) * ((h // 8 + 7) // 8)
    return int(1.5 * p) + 6 * p + 12 * b + 5 * b + 2 * t


def measured_peak() -> tuple[float, str]:
    f = REPO / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_value(key: str) -> float | None:
    """A per-launch figure of the 4K frontend launch from the committed ncu
    summary (lines `key: value`)."""
    f = REPO / "profiles" / "frontend_kernel_4k.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def profiled_traffic() -> float | None:
    """DRAM bytes per frontend launch at 4K."""
    return profiled_value("dram_bytes_per_launch_4k")


def sm_count() -> int:
    import torch

    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"bench_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        time.sleep(0.1)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self) -> dict:
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        try:
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 7:
                    continue
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
                for n, v in zip(names, parts[3:7]):
                    if v.lower() == "active":
                        reasons.add(n)
            self.path.unlink()
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value: float, pg, device: str) -> float:
    """The largest `value` over all ranks (each rank's device-timed region; the
    job lasts as long as its slowest rank). `pg` is torch.distributed or None."""
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, ms: float) -> float:
    """Units per second of the whole job: every rank processes the same number
    of independent units (replicas, weak scaling) within `ms`."""
    return world * units_per_rank / (ms / 1000.0)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(nv12, w, h, d, runs: int) -> dict:
    from oracle import api

    threads = os.cpu_count() or 1
    api.encode(nv12, w, h, d, threads)  # warm tables
    t0 = time.perf_counter()
    for _ in range(runs):
        api.encode(nv12, w, h, d, threads)
    dt = time.perf_counter() - t0
    return {"value": runs / dt, "unit": "frames/s", "cores": threads, "kind": "port",
            "sample": f"{runs} full {w}x{h} frames (seed 0, d={d}) through the CPU restatement, "
                      f"{threads} threads"}


def run_reference(args) -> None:
    world, rank, local = dist_setup()
    if rank != 0:
        return
    from cujpegxl_b200.synth import make_nv12
    from oracle import api

    nv12 = make_nv12(args.width, args.height, 0)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        api.encode(nv12, args.width, args.height, args.distance, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        api.encode(nv12, args.width, args.height, args.distance, threads)
        times.append(time.perf_counter() - t0)
    value = args.steps / sum(times)
    line = {
        "impl": "reference", "metric": "4K frames/s", "value": value, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": value / PUBLISHED_FPS, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{args.width}x{args.height} NV12 seed 0, d={args.distance}, plain VarDCT path",
                   "step": "one frame"},
        "cpu_baseline": {"value": value, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"one full {args.width}x{args.height} frame per step, {threads} threads"},
        "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import threading

    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    from cujpegxl_b200 import Encoder, _capi
    from cujpegxl_b200.synth import make_nv12

    W, H, d = args.width, args.height, args.distance
    S = args.streams
    nv12 = make_nv12(W, H, 0)
    luma_h = torch.from_numpy(nv12[: W * H].reshape(H, W).copy())
    chroma_h = torch.from_numpy(nv12[W * H:].reshape(H // 2, W).copy())
    frames = [(luma_h.cuda(), chroma_h.cuda()) for _ in range(BATCH)]
    torch.cuda.synchronize()

    # S encoders, each with its own CUDA stream and device arena; frame i of a
    # step goes to encoder i % S, so one frame's small entropy kernels overlap
    # another frame's frontend.
    encs = [Encoder(W, H, d, local) for _ in range(S)]
    streams = [torch.cuda.ExternalStream(e.stream()) for e in encs]
    kernels = int(_capi.lib().cujpegxl_b200_kernels_per_encode())

    def enqueue_step():
        for i, (lm, ch) in enumerate(frames):
            encs[i % S].enqueue(lm.data_ptr(), ch.data_ptr(), W, W)

    for _ in range(args.warmup):
        enqueue_step()
    size = encs[0].result()[0]
    for e in encs[1:]:
        e.result()

    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    joins = [torch.cuda.Event() for _ in streams]
    with ClockSampler(local) as clocks:
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        start.record(streams[0])
        for st in streams[1:]:
            st.wait_event(start)
        for _ in range(args.steps):
            enqueue_step()
        for ev, st in zip(joins[1:], streams[1:]):
            ev.record(st)
            streams[0].wait_event(ev)
        stop.record(streams[0])
        for e in encs:
            e.result()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
    total_ms = start.elapsed_time(stop)
    clock_summary = clocks.summary()
    clocks_mhz = clock_summary.get("sm_mhz")
    n = args.steps * BATCH
    total_ms = max_over_ranks(total_ms, pg, "cuda")
    value = whole_job_rate(n, world, total_ms)

    # Per-frame latency and the frontend/entropy split: one encoder alone,
    # events around each stage of each frame.
    enc, stream = encs[0], streams[0]
    ev_a = [torch.cuda.Event(enable_timing=True) for _ in range(BATCH + 1)]
    ev_b = [torch.cuda.Event(enable_timing=True) for _ in range(BATCH)]
    torch.cuda.synchronize()
    for i, (lm, ch) in enumerate(frames):
        ev_a[i].record(stream)
        enc.enqueue_stages(lm.data_ptr(), ch.data_ptr(), W, W, 1)
        ev_b[i].record(stream)
        enc.enqueue_stages(lm.data_ptr(), ch.data_ptr(), W, W, 2)
    ev_a[BATCH].record(stream)
    enc.result()
    torch.cuda.synchronize()
    front = [ev_a[i].elapsed_time(ev_b[i]) for i in range(BATCH)]
    frame_ms = [ev_a[i].elapsed_time(ev_a[i + 1]) for i in range(BATCH)]

    # End to end through the C ABI with host buffers, one host thread per
    # encoder: pinned host NV12 -> device, cujpegxl_encoder_encode, file -> host.
    pinned_l = luma_h.pin_memory()
    pinned_c = chroma_h.pin_memory()
    out_cap = 64 << 20
    outs = [torch.empty(out_cap, dtype=torch.uint8).pin_memory() for _ in range(S)]
    e2e_n = max(args.steps, 4) * S
    d2h = [0] * S

    def e2e_worker(j: int, count: int, gate: torch.cuda.Event | None, done: torch.cuda.Event | None):
        e, st, (dl, dc) = encs[j], streams[j], frames[j]
        with torch.cuda.stream(st):
            if gate is not None:
                st.wait_event(gate)
            for _ in range(count):
                dl.copy_(pinned_l, non_blocking=True)
                dc.copy_(pinned_c, non_blocking=True)
                d2h[j] = e.encode_device_into(dl.data_ptr(), dc.data_ptr(), W, W, outs[j].data_ptr(), out_cap)
            if done is not None:
                done.record(st)

    for j in range(S):
        e2e_worker(j, 2, None, None)
    e0 = torch.cuda.Event(enable_timing=True)
    dones = [torch.cuda.Event(enable_timing=True) for _ in range(S)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0.record(streams[0])
    workers = [threading.Thread(target=e2e_worker, args=(j, e2e_n // S, e0, dones[j])) for j in range(S)]
    for t in workers:
        t.start()
    for t in workers:
        t.join()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(max(e0.elapsed_time(dn) for dn in dones), pg, "cuda")
    e2e = whole_job_rate((e2e_n // S) * S, world, e2e_ms)

    # The same step with learned transform decisions (the shipped network at
    # its default margin, split only): device-resident throughput, the
    # frontend stage with the network's inference in front of it, and the
    # share of regions the network decided.
    from cujpegxl_b200.acsnet import DEFAULT_MARGIN, DEFAULT_WEIGHTS, SPLIT, AcsNet

    net = AcsNet.load(device_ordinal=local)
    for e in encs:
        e.set_acsnet(net, DEFAULT_MARGIN, SPLIT)
    for _ in range(args.warmup):
        enqueue_step()
    for e in encs:
        e.result()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    l0 = torch.cuda.Event(enable_timing=True)
    l1 = torch.cuda.Event(enable_timing=True)
    l0.record(streams[0])
    for st in streams[1:]:
        st.wait_event(l0)
    for _ in range(args.steps):
        enqueue_step()
    for ev, st in zip(joins[1:], streams[1:]):
        ev.record(st)
        streams[0].wait_event(ev)
    l1.record(streams[0])
    for e in encs:
        e.result()
    torch.cuda.synchronize()
    learned_ms = max_over_ranks(l0.elapsed_time(l1), pg, "cuda")
    lf = []
    for lm, ch in frames:
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        enc.enqueue_stages(lm.data_ptr(), ch.data_ptr(), W, W, 1)
        b.record(stream)
        lf.append((a, b))
    enc.result()
    torch.cuda.synchronize()
    learned_front = statistics.mean(a.elapsed_time(b) for a, b in lf)
    decided, regions = enc.acsnet_stats()
    learned_data = enc.encode_device(frames[0][0].data_ptr(), frames[0][1].data_ptr(), W, W) if rank == 0 else b""
    for e in encs:
        e.set_acsnet(None)
    net.close()

    front_ms = statistics.mean(front)
    alg = frontend_algorithmic_bytes(W, H)
    achieved = alg / (front_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peak()
    sorted_ms = sorted(frame_ms)
    p50 = sorted_ms[len(sorted_ms) // 2]
    p99 = sorted_ms[min(len(sorted_ms) - 1, int(round(0.99 * (len(sorted_ms) - 1))))]
    in_bytes = BATCH * W * H * 3 // 2
    # The frontend is bound by instruction issue, not HBM: warp instructions
    # per launch (one-pass ncu count at 4K, committed with the DRAM figure)
    # over the event-timed duration, against 4 issue slots per SM per clock.
    inst = profiled_value("warp_instructions_per_launch_4k") if (W, H) == (W_4K, H_4K) else None
    issue = None
    if inst is not None and clocks_mhz is not None:
        peak_issue = sm_count() * 4 * clocks_mhz * 1e6
        issue = {"achieved": inst / (front_ms / 1000.0), "peak": peak_issue, "unit": "warp instructions/s",
                 "frac": inst / (front_ms / 1000.0) / peak_issue,
                 "basis": "smsp__inst_executed.sum per 4K frontend launch / event-timed launch; peak = SMs x 4 "
                          "schedulers x median SM clock under load"}

    if rank == 0:
        from cujpegxl_b200.decode import psnr_y

        data = encs[0].encode_device(frames[0][0].data_ptr(), frames[0][1].data_ptr(), W, W)
        quality = {"psnr_y_db": psnr_y(nv12, data), "bpp": 8.0 * len(data) / (W * H),
                   "decoder": "in-repo subset decoder, plain dequantisation, BT.709 Y' against the input luma"}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(nv12, W, H, d, args.cpu_runs)
        l2 = (f"{BATCH} distinct input buffers ({in_bytes / 1e6:.0f} MB) "
              + ("exceed the 126 MB L2" if in_bytes > 126e6 else "fit in the 126 MB L2"))
        line = {
            "metric": "4K frames/s", "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / PUBLISHED_FPS, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{W}x{H} NV12 seed 0, d={d}, plain VarDCT path",
                       "step": f"{BATCH} device-resident frames over {S} encoder streams",
                       "width": W, "height": H, "distance": d, "l2": l2,
                       "parallelism": f"{world} independent replica(s), {S} streams each"},
            "mp_per_s": value * W * H / 1e6,
            "bytes_per_frame": size, "bpp": 8.0 * size / (W * H), "quality": quality,
            "p50_frame_ms": p50, "p99_frame_ms": p99, "latency": "one encoder alone, per frame",
            "frontend_ms": front_ms, "entropy_ms": statistics.mean(frame_ms) - front_ms,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic(),
                         "kernel": "frontend_kernel", "algorithmic_bytes": alg, "peak_kind": peak_kind},
            "sm_issue": issue,
            "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": W * H * 3 // 2,
                    "d2h_bytes_per_step": max(d2h) + 32, "step": f"one frame, {S} host threads"},
            "gpu_launches": kernels * n,
            "clocks": clock_summary,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        report = json.loads(DEFAULT_WEIGHTS.with_suffix(".json").read_text())
        lq = psnr_y(nv12, learned_data)
        line["learned"] = {
            "fps": whole_job_rate(n, world, learned_ms), "unit": "frames/s", "frontend_ms": learned_front,
            "decided_regions": decided, "regions": regions, "margin": DEFAULT_MARGIN,
            "bpp": 8.0 * len(learned_data) / (W * H), "psnr_y_db": lq,
            "bpp_delta_pct": 100.0 * (len(learned_data) / len(data) - 1.0),
            "psnr_delta_db": lq - quality["psnr_y_db"],
            "bpp_delta_at_equal_psnr_pct": {
                f"{r['frame']} d={r['distance']}": round(r["bpp_delta_at_equal_psnr_pct"], 3)
                for r in report["codec_split"]},
            "basis": "same step with the shipped network attached (split decisions, margin 0.2); the "
                     "equal-PSNR bpp changes are from the weights' training report (held-out frames)",
        }
        print(json.dumps(line), flush=True)
    # Torch's allocators record events on the streams their blocks were used
    # on when they are freed, so release every torch object that touched the
    # encoders' streams before the encoders destroy those streams.
    torch.cuda.synchronize()
    del frames, pinned_l, pinned_c, outs, ev_a, ev_b, start, stop, e0, dones, joins, stream, streams
    import gc

    gc.collect()
    torch.cuda.synchronize()
    for e in encs:
        e.close()
    if pg:
        pg.destroy_process_group()


MIXED64 = ([(1280, 720)] * 16 + [(1920, 1080)] * 16 + [(2560, 1440)] * 16 + [(3840, 2160)] * 8
           + [(4096, 2160)] * 8)


def run_batch(args) -> None:
    """The 64-frame uneven-resolution batch (16 x 720p, 16 x 1080p, 16 x 1440p,
    8 x 3840x2160, 8 x 4096x2160; frame i from seed i, d=1.0): one CUDA graph
    launch per step through cujpegxl_b200_batch_encode."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from cujpegxl_b200 import Batch
    from cujpegxl_b200.synth import make_nv12

    d = args.distance
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as pool:
        nvs = list(pool.map(lambda i: make_nv12(MIXED64[i][0], MIXED64[i][1], i), range(len(MIXED64))))
    dev = [torch.from_numpy(nv).cuda() for nv in nvs]
    torch.cuda.synchronize()
    inputs = [(t.data_ptr(), t.data_ptr() + w * h, w, w) for t, (w, h) in zip(dev, MIXED64)]
    batch = Batch([(w, h, d) for w, h in MIXED64], local)
    for _ in range(args.warmup):
        batch.encode(inputs)
        batch.sync()
    stream = torch.cuda.ExternalStream(batch.stream())
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        batch.encode(inputs)
    stop.record(stream)
    sizes = batch.sync()
    torch.cuda.synchronize()
    dt = start.elapsed_time(stop) / 1000.0
    n = args.steps * len(MIXED64)
    mp = sum(w * h for w, h in MIXED64) * args.steps / 1e6

    # The same batch with learned transform decisions (the shipped network,
    # split and quant field, margin 0.2): the graph is captured and tuned
    # again, then timed the same way.
    from cujpegxl_b200.acsnet import DEFAULT_MARGIN, QF, SPLIT, AcsNet

    net = AcsNet.load(device_ordinal=local)
    batch.set_acsnet(net, DEFAULT_MARGIN, SPLIT | QF)
    for _ in range(args.warmup):
        batch.encode(inputs)
        batch.sync()
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        batch.encode(inputs)
    stop.record(stream)
    lsizes = batch.sync()
    torch.cuda.synchronize()
    ldt = start.elapsed_time(stop) / 1000.0
    learned = {"value": n / ldt, "unit": "frames/s", "mp_per_s": mp / ldt, "bytes_per_step": sum(lsizes),
               "lanes": batch.lanes, "decisions": "split and quant field, margin 0.2"}
    batch.set_acsnet(None)
    net.close()
    if rank == 0:
        print(json.dumps({
            "metric": "mixed-resolution batch frames/s", "value": n / dt, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "64 frames: 16x1280x720, 16x1920x1080, 16x2560x1440, 8x3840x2160, "
                                   f"8x4096x2160, frame i seed i, d={d}",
                       "step": "one CUDA graph launch of the whole batch", "lanes": batch.lanes},
            "mp_per_s": mp / dt, "bytes_per_step": sum(sizes),
            "timing": "CUDA events on the batch's stream around K graph launches (each ends with the "
                      "device-to-host copy of every frame's size)",
            "learned": learned,
        }), flush=True)
    torch.cuda.synchronize()
    del start, stop, stream
    batch.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=W_4K)
    ap.add_argument("--height", type=int, default=H_4K)
    ap.add_argument("--distance", type=float, default=1.0)
    ap.add_argument("--cpu-runs", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--streams", type=int, default=4, help="encoders (CUDA streams) per GPU")
    ap.add_argument("--workload", default="4k", choices=["4k", "mixed64"],
                    help="mixed64: the 64-frame uneven-resolution batch in one graph launch per step")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "mixed64":
        run_batch(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
