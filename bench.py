#!/usr/bin/env python
"""4K NV12 -> JPEG XL VarDCT encode throughput on B200, with every workload of
the benchmark set measured in the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--streams S]
                    [--no-extras | --extras NAME,...] [--workload 4k|mixed64]

Headline (`value`): the seeded synthetic 3840x2160 NV12 frame (seed 0),
distance 1.0, the plain path (XYB, AQ, gaborish, transform selection, DCT,
CfL, quantise, histograms, prefix codes, packing, headers). One step encodes
a batch of 16 device-resident copies of that frame, frame i on encoder i % S
(S encoders, each with its own CUDA stream and device arena, default 12); the
16 distinct input buffers (199 MB) exceed the 126 MB L2, so no step reads its
input from L2. frames/s over exactly K steps, CUDA events (start on the first
encoder's stream, the others wait on it and are joined back before the stop
event), barrier + synchronize on both sides, max over ranks (one process per
GPU, independent replicas: frames do not shard, so there is no collective).

latency: one encoder alone, 128 frames back to back, events around each
frame (and its frontend stage); n/mean/stddev/min/p50/p99/max as the
reference's benchmark prints them (tools/benchmark/encode_bench.cc:376-390).
e2e: the same metric through the reference's C ABI with host buffers, one
host thread per encoder: every frame is copied host->device from pinned
memory, encoded with cujpegxl_encoder_encode and its file copied back to
pinned host memory.
roofline: the fused frontend kernel, its algorithmic bytes per 4K frame over
its event-timed duration, against the measured HBM copy bandwidth.

Extras (N = 1, rank 0; --no-extras skips them, --extras a,b runs a subset),
each timed in this run:
  distances: the 4K frame at d = 0.5, 2 and 4 (frames/s over the same step,
    bpp, PSNR-Y through the in-repo decoder);
  learned: the 4K step with the shipped transform-decision network (split
    only, and split + quant field), and the bpp change at equal PSNR-Y against
    the plain heuristic at d = 1 and 2 on held-out frames (log-bpp
    interpolated over the network's encodes at d x 0.8 .. 1.25);
  mixed64: the 64-frame uneven-resolution batch in one launch per step,
    plain and learned;
  serving: the 8-stream serving workload (2 x 4K@30, 4 x 1080p@60,
    2 x 720p@60, Poisson arrivals, 40 GB budget) at 1x for 3 s (>= 1000
    frames) and at rising speeds until it no longer keeps up, plain and
    learned; p50/p99 latency and sustained frames/s, and the fastest speed
    whose p99 stays within 8 ms.
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
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

W_4K, H_4K = 3840, 2160
BATCH = 16
LATENCY_FRAMES = 128
EXTRAS = ("reference_device", "distances", "learned", "mixed64", "serving")
PUBLISHED_FPS = 15.0  # reference README.md:17, GTX 1080 Ti, 4K sustained
HELD_OUT = [(3840, 2160, 0), (1920, 1080, 424242)]  # frames outside the network's training and validation seeds
P99_TARGET_MS = 8.0  # serving-loop latency target per 4K frame


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
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"bench_clocks_{os.getpid()}_{id(self)}.csv"

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


def psnr_many(pairs: list[tuple[np.ndarray, bytes]]) -> list[float]:
    """PSNR-Y of each (nv12, file) through the in-repo decoder, decoded on every
    host core at once (the decoder releases the interpreter while it runs)."""
    from cujpegxl_b200.decode import psnr_y

    with ThreadPoolExecutor(max_workers=max(1, min(len(pairs), os.cpu_count() or 1))) as pool:
        return list(pool.map(lambda p: psnr_y(p[0], p[1]), pairs))


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


class Step:
    """S encoders over one set of device frames; one step = BATCH frames,
    frame i on encoder i % S."""

    def __init__(self, encs, frames, W, H):
        import torch

        self.encs, self.frames, self.W, self.H = encs, frames, W, H
        self.streams = [torch.cuda.ExternalStream(e.stream()) for e in encs]
        self.joins = [torch.cuda.Event() for _ in encs]

    def enqueue(self):
        S = len(self.encs)
        for i, (lm, ch) in enumerate(self.frames):
            self.encs[i % S].enqueue(lm.data_ptr(), ch.data_ptr(), self.W, self.W)

    def drain(self):
        for e in self.encs:
            e.result()

    def timed(self, steps: int, warmup: int, pg=None) -> float:
        """ms for `steps` steps after `warmup` untimed ones, CUDA events on the
        first stream (the others fork from and join into it)."""
        import torch

        for _ in range(warmup):
            self.enqueue()
        self.drain()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        start.record(self.streams[0])
        for st in self.streams[1:]:
            st.wait_event(start)
        for _ in range(steps):
            self.enqueue()
        for ev, st in zip(self.joins[1:], self.streams[1:]):
            ev.record(st)
            self.streams[0].wait_event(ev)
        stop.record(self.streams[0])
        self.drain()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        return start.elapsed_time(stop)

    def stage_times(self, n: int) -> tuple[list[float], list[float]]:
        """(frontend ms, whole-frame ms) of n frames on the first encoder alone."""
        import torch

        enc, stream = self.encs[0], self.streams[0]
        ev_a = [torch.cuda.Event(enable_timing=True) for _ in range(n + 1)]
        ev_b = [torch.cuda.Event(enable_timing=True) for _ in range(n)]
        torch.cuda.synchronize()
        for i in range(n):
            lm, ch = self.frames[i % len(self.frames)]
            ev_a[i].record(stream)
            enc.enqueue_stages(lm.data_ptr(), ch.data_ptr(), self.W, self.W, 1)
            ev_b[i].record(stream)
            enc.enqueue_stages(lm.data_ptr(), ch.data_ptr(), self.W, self.W, 2)
        ev_a[n].record(stream)
        enc.result()
        torch.cuda.synchronize()
        return ([ev_a[i].elapsed_time(ev_b[i]) for i in range(n)],
                [ev_a[i].elapsed_time(ev_a[i + 1]) for i in range(n)])


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
    from cujpegxl_b200.serve import latency_stats
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
    step = Step(encs, frames, W, H)
    streams = step.streams
    kernels = int(_capi.lib().cujpegxl_b200_kernels_per_encode())

    with ClockSampler(local) as clocks:
        total_ms = step.timed(args.steps, args.warmup, pg)
    clock_summary = clocks.summary()
    clocks_mhz = clock_summary.get("sm_mhz")
    size = encs[0].result()[0]
    n = args.steps * BATCH
    total_ms = max_over_ranks(total_ms, pg, "cuda")
    value = whole_job_rate(n, world, total_ms)

    # Per-frame latency and the frontend/entropy split: one encoder alone.
    front, frame_ms = step.stage_times(LATENCY_FRAMES)

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
    e2e_bytes = bytes(outs[0][:d2h[0]].numpy())

    front_ms = statistics.mean(front)
    alg = frontend_algorithmic_bytes(W, H)
    achieved = alg / (front_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peak()
    lat = latency_stats(frame_ms)
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

    line = None
    if rank == 0:
        from cujpegxl_b200.decode import psnr_y

        data = encs[0].encode_device(frames[0][0].data_ptr(), frames[0][1].data_ptr(), W, W)
        if e2e_bytes != data:
            raise AssertionError("the end-to-end file differs from the device-resident encode")
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
            "p50_frame_ms": lat["p50"], "p99_frame_ms": lat["p99"],
            "latency": dict(lat, unit="ms", basis=f"one encoder alone, {LATENCY_FRAMES} frames back to back, "
                                                  "CUDA events around each frame"),
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

    extras = rank == 0 and world == 1 and not args.no_extras
    want = set(args.extras.split(",")) if extras else set()
    if "reference_device" in want:
        line["reference_device"] = bench_reference_device(step, args)
    if "distances" in want:
        line["distances"] = bench_distances(step, nv12, args)
    if "learned" in want:
        line["learned"] = bench_learned(step, nv12, data, quality, args, local)
    # Torch's allocators record events on the streams their blocks were used
    # on when they are freed, so release every torch object that touched the
    # encoders' streams before the encoders destroy those streams.
    torch.cuda.synchronize()
    del frames, pinned_l, pinned_c, outs, e0, dones, streams, step
    import gc

    gc.collect()
    torch.cuda.synchronize()
    for e in encs:
        e.close()
    if "mixed64" in want:
        line["mixed64"] = bench_mixed64(args, local, value)
    if "serving" in want:
        line["serving"] = bench_serving(args, local)
    if line is not None:
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def bench_reference_device(step: Step, args) -> dict | None:
    """The reference's own device stages on the same 4K frame, timed per call
    (CUDA events on the legacy default stream around each entry point, which
    launches its kernels there and synchronises the device before returning):
    nv12_to_xyb (src/xyb.cu), the fused adaptive-quantisation kernel
    (src/frontend_fused.cu encode_frontend) and XYB + inverse gaborish + the
    variable DCT (src/frontend_transform.cu) on this encoder's transform
    decisions. The reference's selection, CfL, quantiser and entropy coder are
    not built (src/transform_select.cu, src/frontend_quantize.cu and
    src/entropy.cu do not compile with nvcc)."""
    import ctypes

    import torch

    lib_path = REPO / "oracle" / "_ref" / "libjxlref_gpu.so"
    if not lib_path.exists():
        return None
    L = ctypes.CDLL(str(lib_path))
    U = ctypes.c_size_t
    L.refgpu_nv12_to_xyb.argtypes = [U, U, U, U, U, U, U]
    L.refgpu_encode_frontend.argtypes = [U, U, U, U, U, U, ctypes.c_float, U]
    L.refgpu_frontend_transform.argtypes = [U, U, U, U, U, U, ctypes.c_float, U, U, U]
    W, H = step.W, step.H
    nb = (W // 8) * (H // 8)
    lm, ch = step.frames[0]
    acs = torch.from_numpy(step.encs[0].read_planes(keys=("acs",))["acs"]).cuda()
    xyb = torch.empty(3 * W * H, dtype=torch.float32, device="cuda")
    qf = torch.empty(nb, dtype=torch.int32, device="cuda")
    coef = torch.empty(3 * nb * 64, dtype=torch.float16, device="cuda")
    acs_out = torch.empty(nb, dtype=torch.int8, device="cuda")
    calls = {
        "nv12_to_xyb": lambda: L.refgpu_nv12_to_xyb(lm.data_ptr(), W, ch.data_ptr(), W, W, H, xyb.data_ptr()),
        "aq_field": lambda: L.refgpu_encode_frontend(lm.data_ptr(), W, ch.data_ptr(), W, W, H, args.distance,
                                                     qf.data_ptr()),
        "xyb_gaborish_dct": lambda: L.refgpu_frontend_transform(lm.data_ptr(), W, ch.data_ptr(), W, W, H,
                                                                args.distance, coef.data_ptr(), acs_out.data_ptr(),
                                                                acs.data_ptr()),
    }
    out = {}
    stream = torch.cuda.default_stream()
    for name, fn in calls.items():
        times = []
        for i in range(3 + 10):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            if fn() != 1:
                raise RuntimeError(f"reference {name} failed")
            b.record(stream)
            torch.cuda.synchronize()
            if i >= 3:
                times.append(a.elapsed_time(b))
        out[name + "_ms"] = statistics.median(times)
    out["sum_ms"] = sum(out.values())
    out["basis"] = ("the reference's device entry points built from its sources for sm_100a, median of 10 calls "
                    "after 3; each call includes its own allocation, texture set-up and device synchronise")
    return out


def bench_distances(step: Step, nv12, args) -> dict:
    """The headline step at d = 0.5, 2 and 4 (d = 1 is the headline)."""
    W, H = step.W, step.H
    out = {}
    pairs = []
    for d in (0.5, 2.0, 4.0):
        for e in step.encs:
            e.configure(W, H, d)
        steps = max(3, args.steps // 2)
        ms = step.timed(steps, args.warmup)
        front, frame_ms = step.stage_times(16)
        data = step.encs[0].encode_device(step.frames[0][0].data_ptr(), step.frames[0][1].data_ptr(), W, W)
        pairs.append((nv12, data))
        out[str(d)] = {"fps": steps * BATCH / (ms / 1000.0), "steps": steps, "bpp": 8.0 * len(data) / (W * H),
                       "frontend_ms": statistics.mean(front), "frame_ms": statistics.mean(frame_ms)}
    for (k, v), p in zip(out.items(), psnr_many(pairs)):
        v["psnr_y_db"] = p
    for e in step.encs:
        e.configure(W, H, args.distance)
    return out


def bench_learned(step: Step, nv12, plain_data: bytes, quality: dict, args, device: int) -> dict:
    """The headline step with the shipped network attached, and the live
    equal-PSNR bpp change on held-out frames."""
    from cujpegxl_b200 import Encoder
    from cujpegxl_b200.acsnet import DEFAULT_MARGIN, QF, SPLIT, AcsNet
    from cujpegxl_b200.synth import make_nv12

    W, H = step.W, step.H
    net = AcsNet.load(device_ordinal=device)
    res = {"margin": DEFAULT_MARGIN, "unit": "frames/s"}
    pairs = []
    try:
        for name, flags in (("split", SPLIT), ("split_qf", SPLIT | QF)):
            for e in step.encs:
                e.set_acsnet(net, DEFAULT_MARGIN, flags)
            ms = step.timed(args.steps, args.warmup)
            front, _ = step.stage_times(16)
            data = step.encs[0].encode_device(step.frames[0][0].data_ptr(), step.frames[0][1].data_ptr(), W, W)
            decided, regions = step.encs[0].acsnet_stats()
            res[name] = {"fps": args.steps * BATCH / (ms / 1000.0), "frontend_ms": statistics.mean(front),
                         "decided_regions": decided, "regions": regions, "bpp": 8.0 * len(data) / (W * H),
                         "bpp_delta_pct": 100.0 * (len(data) / len(plain_data) - 1.0)}
            pairs.append((nv12, data))
        for e in step.encs:
            e.set_acsnet(None)
        for (name, v), p in zip([(k, res[k]) for k in ("split", "split_qf")], psnr_many(pairs)):
            v["psnr_y_db"] = p
            v["psnr_delta_db"] = p - quality["psnr_y_db"]

        # Equal-PSNR bpp change, measured now: per held-out frame and distance,
        # the plain encode and the network's encodes at d x 0.8 .. 1.25.
        scales = (0.8, 0.9, 1.0, 1.12, 1.25)
        jobs = []   # (key, nv12, data, bpp, kind)
        for (w, h, seed) in HELD_OUT:
            nv = make_nv12(w, h, seed)
            for d in (1.0, 2.0):
                key = f"{w}x{h}#{seed} d={d}"
                with Encoder(w, h, d, device) as enc:
                    data = enc.encode_host(nv)
                jobs.append((key, nv, data, 8.0 * len(data) / (w * h), "plain"))
                for s in scales:
                    with Encoder(w, h, d * s, device) as enc:
                        enc.set_acsnet(net, DEFAULT_MARGIN, SPLIT | QF)
                        data = enc.encode_host(nv)
                        enc.set_acsnet(None)
                    jobs.append((key, nv, data, 8.0 * len(data) / (w * h), s))
        psnrs = psnr_many([(j[1], j[2]) for j in jobs])
        table = {}
        for (key, _, _, bpp, kind), p in zip(jobs, psnrs):
            t = table.setdefault(key, {"curve": []})
            if kind == "plain":
                t["bpp_plain"], t["psnr_plain"] = bpp, p
            else:
                t["curve"].append((kind, bpp, p))
        for key, t in table.items():
            ps = np.array([c[2] for c in t["curve"]])
            lb = np.log(np.array([c[1] for c in t["curve"]]))
            order = np.argsort(ps)
            pp = t["psnr_plain"]
            at = float(np.exp(np.interp(pp, ps[order], lb[order]))) if ps.min() <= pp <= ps.max() else float("nan")
            mid = [c for c in t["curve"] if c[0] == 1.0][0]
            t.update(bpp_learned=mid[1], psnr_learned=mid[2],
                     bpp_delta_at_equal_psnr_pct=100.0 * (at / t["bpp_plain"] - 1.0))
            del t["curve"]
        res["equal_psnr"] = table
        res["equal_psnr_basis"] = ("measured in this run: split + quant-field decisions, margin 0.2, held-out "
                                   "seeds; log-bpp interpolated at the plain encode's PSNR-Y over the network's "
                                   "encodes at d x 0.8, 0.9, 1, 1.12, 1.25")
    finally:
        for e in step.encs:
            e.set_acsnet(None)
        net.close()
    return res


MIXED64 = ([(1280, 720)] * 16 + [(1920, 1080)] * 16 + [(2560, 1440)] * 16 + [(3840, 2160)] * 8
           + [(4096, 2160)] * 8)


def mixed64_frames(device: int):
    import torch

    from cujpegxl_b200.synth import make_nv12

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as pool:
        nvs = list(pool.map(lambda i: make_nv12(MIXED64[i][0], MIXED64[i][1], i), range(len(MIXED64))))
    dev = [torch.from_numpy(nv).cuda(device) for nv in nvs]
    torch.cuda.synchronize()
    inputs = [(t.data_ptr(), t.data_ptr() + w * h, w, w) for t, (w, h) in zip(dev, MIXED64)]
    return dev, inputs


def time_batch(batch, inputs, steps: int, warmup: int) -> tuple[float, list[int]]:
    import torch

    for _ in range(warmup):
        batch.encode(inputs)
        batch.sync()
    stream = torch.cuda.ExternalStream(batch.stream())
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(steps):
        batch.encode(inputs)
    stop.record(stream)
    sizes = batch.sync()
    torch.cuda.synchronize()
    return start.elapsed_time(stop), sizes


def bench_mixed64(args, device: int, single_fps: float) -> dict:
    """The 64-frame uneven-resolution batch (16 x 720p, 16 x 1080p, 16 x 1440p,
    8 x 3840x2160, 8 x 4096x2160; frame i from seed i, d=1.0), one launch
    per step, plain then learned (split and quant field, margin 0.2)."""
    from cujpegxl_b200 import Batch
    from cujpegxl_b200.acsnet import DEFAULT_MARGIN, QF, SPLIT, AcsNet

    dev, inputs = mixed64_frames(device)
    steps = max(3, args.steps // 2)
    mp = sum(w * h for w, h in MIXED64) / 1e6
    res = {"frames": len(MIXED64), "steps": steps, "distance": 1.0,
           "workload": "16x1280x720, 16x1920x1080, 16x2560x1440, 8x3840x2160, 8x4096x2160, frame i seed i",
           "timing": "CUDA events on the batch's stream around K launches"}
    with Batch([(w, h, 1.0) for w, h in MIXED64], device) as batch:
        ms, sizes = time_batch(batch, inputs, steps, args.warmup)
        res["plain"] = {"fps": steps * len(MIXED64) / (ms / 1000.0), "mp_per_s": steps * mp / (ms / 1000.0),
                        "bytes_per_step": sum(sizes), "schedule": batch.schedule()}
        net = AcsNet.load(device_ordinal=device)
        batch.set_acsnet(net, DEFAULT_MARGIN, SPLIT | QF)
        ms, sizes = time_batch(batch, inputs, steps, args.warmup)
        res["learned"] = {"fps": steps * len(MIXED64) / (ms / 1000.0), "mp_per_s": steps * mp / (ms / 1000.0),
                          "bytes_per_step": sum(sizes), "schedule": batch.schedule(),
                          "decisions": "split and quant field, margin 0.2"}
        batch.set_acsnet(None)
        net.close()
    res["single_frame_plain_4k_fps"] = single_fps
    del dev
    return res


def bench_serving(args, device: int) -> dict:
    """The 8-stream serving workload, plain and learned: 1x for 3 s, then
    rising speeds (2x .. 12x) for 1.5 s each until a run no longer keeps up
    (every offered frame done within 0.1 s of the last arrival); reports the
    fastest run that kept up and the fastest whose p99 stayed within 8 ms."""
    from cujpegxl_b200.acsnet import QF, SPLIT, AcsNet
    from cujpegxl_b200.serve import DEFAULT_STREAMS, AdmissionError, Server

    def one(net) -> dict:
        srv = Server(device, 40e9, depth=2, net=net, net_flags=SPLIT | QF, frames=4)
        try:
            rejected = []
            for i, spec in enumerate(DEFAULT_STREAMS):
                try:
                    srv.admit(spec, seed=i)
                except AdmissionError as e:
                    rejected.append(str(e))
            srv.run(0.3, seed=99, speed=1.0)   # warm-up
            base = srv.run(3.0, seed=0, speed=1.0)
            trim = lambda r: None if r is None else {k: r[k] for k in (
                "speed", "duration_s", "offered_frames", "frames", "wall_s", "kept_up", "sustained_fps",
                "sustained_mp_per_s", "p50_ms", "p99_ms", "latency_ms", "clock_offset_bound_ms")}
            sweep = []
            for speed in (2.0, 4.0, 6.0, 8.0, 10.0, 12.0):
                r = srv.run(1.5, seed=int(speed), speed=speed)
                sweep.append(r)
                if not r["kept_up"]:
                    break
            kept = [r for r in sweep if r["kept_up"]]
            within = [r for r in kept if r["p99_ms"] is not None and r["p99_ms"] <= P99_TARGET_MS]
            return {"at_1x": trim(base), "fastest_kept_up": trim(kept[-1] if kept else None),
                    "fastest_p99_within_8ms": trim(within[-1] if within else None),
                    "sweep": [{k: r[k] for k in ("speed", "frames", "kept_up", "sustained_fps", "p50_ms", "p99_ms")}
                              for r in sweep],
                    "rejected": rejected, "device_bytes_admitted": base["device_bytes_admitted"]}
        finally:
            srv.close()

    res = {"workload": "2x3840x2160@30, 4x1920x1080@60, 2x1280x720@60 frames/s, Poisson arrivals, "
                       "4 distinct seeded frames per stream, 2 slots per stream, 40 GB budget, d=1.0",
           "latency_basis": "arrival (host clock) to the file in host memory (device event)"}
    res["plain"] = one(None)
    net = AcsNet.load(device_ordinal=device)
    try:
        res["learned"] = one(net)
    finally:
        net.close()
    return res


def run_batch(args) -> None:
    """The 64-frame uneven-resolution batch as the headline line."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    r = bench_mixed64(args, local, float("nan"))
    if rank == 0:
        print(json.dumps({
            "metric": "mixed-resolution batch frames/s", "value": r["plain"]["fps"], "unit": "frames/s",
            "n_gpus": world, "steps": r["steps"], "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": r["workload"], "step": "one launch of the whole batch"}, "mixed64": r,
        }), flush=True)


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
    ap.add_argument("--no-extras", action="store_true",
                    help="only the headline line: skip the distance, learned, batch and serving workloads")
    ap.add_argument("--extras", default=",".join(EXTRAS),
                    help="comma-separated subset of the extra workloads to run (default: all of them)")
    ap.add_argument("--streams", type=int, default=12,
                    help=f"encoders (CUDA streams) per GPU, 1..{BATCH} (each takes frames of the {BATCH}-frame step)")
    ap.add_argument("--workload", default="4k", choices=["4k", "mixed64"],
                    help="mixed64: the 64-frame uneven-resolution batch as the headline")
    args = ap.parse_args()
    unknown = set(args.extras.split(",")) - set(EXTRAS)
    if unknown:
        ap.error(f"unknown extras {sorted(unknown)}; choose from {list(EXTRAS)}")
    if not 1 <= args.streams <= BATCH:
        ap.error(f"--streams must be 1..{BATCH}, got {args.streams}")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "mixed64":
        run_batch(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
