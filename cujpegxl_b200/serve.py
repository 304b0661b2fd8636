"""Continuous serving loop: live NV12 streams encoded as their frames arrive.

    python -m cujpegxl_b200.serve [--duration S] [--speed K] [--budget-gb G] [--seed N] [--learned]

Each admitted stream gets `depth` encoder slots (an encoder with its own CUDA
stream and device arena, a device frame buffer and a page-locked host output
buffer). A frame is scheduled the moment it arrives and a slot of its stream
is free; nothing waits to form a batch, and frames of all streams run
concurrently on their slots' streams (the GPU interleaves their kernels). Per
frame: the pinned host frame is copied to the device, encoded with the C ABI's
asynchronous entry point, and its file copied back into the slot's host
buffer by cujpegxl_b200_encoder_enqueue_readback (a kernel that reads the
file size on the device, so the three steps run back to back with no host
round trip); a CUDA event marks the end. A frame's latency is that event's
device time minus the frame's arrival time, both measured from one start
point: the start event is recorded and synchronised before the host clock
starts, so device times lead host times by at most the measured
`clock_offset_bound_ms`.

Every stream owns `frames` distinct seeded frames (frame k of stream i from
seed frame_seed(i, k)) and arrival n carries frame n mod `frames`, so the
loop never re-encodes one fixed input. With `verify=True` the SHA-256 of
every delivered file is kept, so a caller can compare each against the file
of the same frame encoded alone.

Admission: a stream is admitted only if the device memory its slots hold
(cujpegxl_b200_encoder_memory, plus the frame buffers) fits in what remains of
the budget; otherwise AdmissionError and nothing of it stays allocated.

The default workload is 2 x 3840x2160 at 30 frames/s, 4 x 1920x1080 at 60 and
2 x 1280x720 at 60, Poisson arrivals (seed 0), distance 1.0, a 40 GB budget.
`--speed K` scales every stream's rate by K to find the sustained throughput.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class StreamSpec:
    name: str
    width: int
    height: int
    fps: float
    distance: float = 1.0


DEFAULT_STREAMS = (
    [StreamSpec(f"uhd30-{i}", 3840, 2160, 30.0) for i in range(2)]
    + [StreamSpec(f"fhd60-{i}", 1920, 1080, 60.0) for i in range(4)]
    + [StreamSpec(f"hd60-{i}", 1280, 720, 60.0) for i in range(2)]
)


def frame_seed(stream_seed: int, k: int) -> int:
    """Seed of frame k of the stream admitted with `stream_seed`."""
    return 1_000_000 + 1000 * stream_seed + k


class AdmissionError(RuntimeError):
    pass


def poisson_arrivals(rate: float, duration: float, rng: np.random.Generator) -> np.ndarray:
    """Arrival times in [0, duration) of a Poisson process with `rate` per second."""
    if rate <= 0 or duration <= 0:
        return np.zeros(0)
    n = int(rate * duration * 2 + 32)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    while t[-1] < duration:
        t = np.concatenate([t, t[-1] + np.cumsum(rng.exponential(1.0 / rate, n))])
    return t[t < duration]


class Budget:
    """Device-memory admission budget."""

    def __init__(self, total_bytes: int):
        self.total = int(total_bytes)
        self.used = 0

    def reserve(self, nbytes: int) -> bool:
        if self.used + nbytes > self.total:
            return False
        self.used += nbytes
        return True

    def release(self, nbytes: int) -> None:
        self.used = max(0, self.used - nbytes)


def percentile(values: list[float], q: float) -> float | None:
    """The value at sorted index round-half-away(q/100 * (n - 1)), the rule of
    the reference's benchmark (tools/benchmark/encode_bench.cc:310-316)."""
    if not values:
        return None
    s = sorted(values)
    return s[min(len(s) - 1, int(math.floor(q / 100.0 * (len(s) - 1) + 0.5)))]


def latency_stats(values: list[float]) -> dict:
    """n, mean, stddev (n - 1), min, p50, p99, max: the statistics the
    reference's benchmark prints (tools/benchmark/encode_bench.cc:376-390)."""
    if not values:
        return {"n": 0}
    a = np.asarray(values, np.float64)
    return {"n": int(a.size), "mean": float(a.mean()), "stddev": float(a.std(ddof=1)) if a.size > 1 else 0.0,
            "min": float(a.min()), "p50": percentile(values, 50), "p99": percentile(values, 99),
            "max": float(a.max())}


@dataclass
class _Slot:
    enc: object
    stream: object
    luma: object
    chroma: object
    out: object          # page-locked host output buffer (torch uint8)
    words: object        # page-locked {size, status} written by the readback
    done: object = None
    arrival_ms: float = 0.0
    frame: int = 0
    busy: bool = False


@dataclass
class _Stream:
    spec: StreamSpec
    slots: list
    frames: list         # [(pinned luma, pinned chroma)] distinct seeded frames
    seeds: list
    reserved: int
    next_frame: int = 0
    queue: deque = field(default_factory=deque)
    latencies: list = field(default_factory=list)
    sizes: list = field(default_factory=list)
    digests: list = field(default_factory=list)   # (frame index, sha256 hex)


class Server:
    def __init__(self, device: int = 0, budget_bytes: float = 40e9, depth: int = 2, net=None,
                 margin: float = 0.2, net_flags: int = 1, frames: int = 4, out_capacity: int = 8 << 20):
        """net: an acsnet.AcsNet for learned transform decisions (owned by the
        caller), attached to every encoder with `margin` and `net_flags`.
        frames: distinct seeded frames per stream. out_capacity: host output
        buffer per slot (larger files are read back in a second copy)."""
        import torch

        from . import Encoder  # noqa: F401  (fails loudly if the library is missing)
        from . import _capi

        self.torch = torch
        self._L = _capi.lib()
        self.device = device
        self.budget = Budget(int(budget_bytes))
        self.depth = depth
        self.net, self.margin, self.net_flags = net, margin, net_flags
        self.frames_per_stream = frames
        self.out_capacity = out_capacity
        self.streams: list[_Stream] = []
        torch.cuda.set_device(device)

    def admit(self, spec: StreamSpec, seed: int = 0) -> int:
        """Allocates the stream's slots; raises AdmissionError if they do not fit."""
        from concurrent.futures import ThreadPoolExecutor

        from . import Encoder
        from .synth import make_nv12

        torch = self.torch
        w, h = spec.width, spec.height
        slots: list[_Slot] = []
        reserved = 0
        try:
            for _ in range(self.depth):
                enc = Encoder(w, h, spec.distance, self.device)
                if self.net is not None:
                    enc.set_acsnet(self.net, self.margin, self.net_flags)
                dev_bytes, _ = enc.memory()
                need = dev_bytes + w * h * 3 // 2
                if not self.budget.reserve(need):
                    enc.close()
                    raise AdmissionError(f"{spec.name}: {need / 1e9:.2f} GB more than the "
                                         f"{(self.budget.total - self.budget.used) / 1e9:.2f} GB left")
                reserved += need
                slots.append(_Slot(enc, torch.cuda.ExternalStream(enc.stream()),
                                   torch.empty((h, w), dtype=torch.uint8, device="cuda"),
                                   torch.empty((h // 2, w), dtype=torch.uint8, device="cuda"),
                                   torch.empty(self.out_capacity, dtype=torch.uint8).pin_memory(),
                                   torch.zeros(2, dtype=torch.int64).pin_memory()))
        except AdmissionError:
            self.budget.release(reserved)
            for s in slots:
                s.enc.close()
            raise
        seeds = [frame_seed(seed, k) for k in range(self.frames_per_stream)]
        with ThreadPoolExecutor(max_workers=len(seeds)) as pool:
            nvs = list(pool.map(lambda s: make_nv12(w, h, s), seeds))
        frames = [(torch.from_numpy(nv[: w * h].reshape(h, w).copy()).pin_memory(),
                   torch.from_numpy(nv[w * h:].reshape(h // 2, w).copy()).pin_memory()) for nv in nvs]
        self.streams.append(_Stream(spec, slots, frames, seeds, reserved))
        return len(self.streams) - 1

    def _launch(self, st: _Stream, slot: _Slot, arrival_ms: float) -> None:
        torch = self.torch
        w = st.spec.width
        k = st.next_frame % len(st.frames)
        st.next_frame += 1
        host_luma, host_chroma = st.frames[k]
        with torch.cuda.stream(slot.stream):
            slot.luma.copy_(host_luma, non_blocking=True)
            slot.chroma.copy_(host_chroma, non_blocking=True)
        slot.enc.enqueue(slot.luma.data_ptr(), slot.chroma.data_ptr(), w, w)
        self._readback(slot, slot.out)
        slot.done = torch.cuda.Event(enable_timing=True)
        slot.done.record(slot.stream)
        slot.arrival_ms = arrival_ms
        slot.frame = k
        slot.busy = True

    def _readback(self, slot: _Slot, out) -> None:
        from ._capi import check

        check("encoder_enqueue_readback", self._L.cujpegxl_b200_encoder_enqueue_readback(
            slot.enc.handle, out.data_ptr(), out.numel(), slot.words.data_ptr()))

    def _collect(self, st: _Stream, slot: _Slot, start, verify: bool) -> None:
        size, status = int(slot.words[0]), int(slot.words[1])
        if status == 2:
            raise RuntimeError(f"{st.spec.name}: encode failed")
        out = slot.out
        if status == 1:
            # Larger than the slot's buffer: a second copy into a buffer that fits.
            out = self.torch.empty(size, dtype=self.torch.uint8).pin_memory()
            self._readback(slot, out)
            self.torch.cuda.synchronize(self.device)
        st.latencies.append(start.elapsed_time(slot.done) - slot.arrival_ms)
        st.sizes.append(size)
        if verify:
            st.digests.append((slot.frame, hashlib.sha256(out[:size].numpy().tobytes()).hexdigest()))

    def run(self, duration: float, seed: int = 0, speed: float = 1.0, verify: bool = False) -> dict:
        torch = self.torch
        rng = np.random.Generator(np.random.PCG64(seed))
        events = []
        for i, st in enumerate(self.streams):
            st.queue.clear()
            st.latencies.clear()
            st.sizes.clear()
            st.digests.clear()
            st.next_frame = 0
            for t in poisson_arrivals(st.spec.fps * speed, duration, rng):
                events.append((float(t), i))
        events.sort()
        offered = len(events)
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        t_before = time.perf_counter()
        start.record(self.streams[0].slots[0].stream)
        start.synchronize()
        t0 = time.perf_counter()
        offset_bound_ms = 1000.0 * (t0 - t_before)
        k = 0
        in_flight = 0
        while k < len(events) or in_flight or any(st.queue for st in self.streams):
            now = time.perf_counter() - t0
            while k < len(events) and events[k][0] <= now:
                self.streams[events[k][1]].queue.append(1000.0 * events[k][0])
                k += 1
            progressed = False
            for st in self.streams:
                for slot in st.slots:
                    if slot.busy and slot.done.query():
                        self._collect(st, slot, start, verify)
                        slot.busy = False
                        in_flight -= 1
                        progressed = True
                    if not slot.busy and st.queue:
                        self._launch(st, slot, st.queue.popleft())
                        in_flight += 1
                        progressed = True
            if not progressed:
                time.sleep(0.0001)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        all_lat = [x for st in self.streams for x in st.latencies]
        done = len(all_lat)
        per = {}
        for st in self.streams:
            per[st.spec.name] = {"width": st.spec.width, "height": st.spec.height,
                                 "offered_fps": st.spec.fps * speed, "frames": len(st.latencies),
                                 "p50_ms": percentile(st.latencies, 50), "p99_ms": percentile(st.latencies, 99),
                                 "mean_bytes": float(np.mean(st.sizes)) if st.sizes else None}
            if verify:
                per[st.spec.name]["digests"] = list(st.digests)
                per[st.spec.name]["frame_seeds"] = list(st.seeds)
        mp = sum(st.spec.width * st.spec.height * len(st.latencies) for st in self.streams) / 1e6
        return {"duration_s": duration, "speed": speed, "offered_frames": offered, "frames": done,
                "wall_s": wall, "kept_up": done == offered and wall <= duration + 0.1,
                "sustained_fps": done / wall, "sustained_mp_per_s": mp / wall,
                "p50_ms": percentile(all_lat, 50), "p99_ms": percentile(all_lat, 99),
                "latency_ms": latency_stats(all_lat),
                "clock_offset_bound_ms": offset_bound_ms,
                "latency_basis": "device event at the end of the file's copy to host memory minus the host "
                                 "arrival time, both from one start point; the device clock leads the host "
                                 "clock by at most clock_offset_bound_ms",
                "device_bytes_admitted": self.budget.used, "streams": per}

    def close(self) -> None:
        # Torch's pinned-memory allocator records events on every stream a
        # pinned block was copied on when the block is freed, so every torch
        # object that touched an encoder's stream goes before that stream.
        import gc

        self.torch.cuda.synchronize()
        for st in self.streams:
            st.frames = []
            for slot in st.slots:
                slot.done = None
                slot.stream = None
                slot.luma = None
                slot.chroma = None
                slot.out = None
                slot.words = None
        gc.collect()
        self.torch.cuda.synchronize()
        for st in self.streams:
            for slot in st.slots:
                slot.enc.close()
            self.budget.release(st.reserved)
        self.streams.clear()


def serve_workload(duration: float, speed: float, seed: int = 0, device: int = 0, budget_bytes: float = 40e9,
                   depth: int = 2, net=None, net_flags: int = 1, frames: int = 4) -> dict:
    """Admits the default 8-stream workload (stream i from seed i), runs it
    once at `speed`, and returns the result with the refused streams."""
    srv = Server(device, budget_bytes, depth, net, net_flags=net_flags, frames=frames)
    rejected = []
    try:
        for i, spec in enumerate(DEFAULT_STREAMS):
            try:
                srv.admit(spec, seed=i)
            except AdmissionError as e:
                rejected.append(str(e))
        result = srv.run(duration, seed=seed, speed=speed)
    finally:
        srv.close()
    result["rejected"] = rejected
    return result


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--duration", type=float, default=5.0)
    ap.add_argument("--speed", type=float, default=1.0)
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--depth", type=int, default=2)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--frames", type=int, default=4, help="distinct seeded frames per stream")
    ap.add_argument("--learned", action="store_true", help="learned transform decisions (shipped weights)")
    args = ap.parse_args()
    net = None
    if args.learned:
        from .acsnet import QF, SPLIT, AcsNet
        net = AcsNet.load(device_ordinal=args.device)
    result = serve_workload(args.duration, args.speed, args.seed, args.device, args.budget_gb * 1e9, args.depth,
                            net, (SPLIT | QF) if net is not None else 1, args.frames)
    print(json.dumps(result), flush=True)
    if net is not None:
        net.close()


if __name__ == "__main__":
    main()
