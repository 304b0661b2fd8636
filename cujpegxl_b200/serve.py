"""Continuous serving loop: live NV12 streams encoded as their frames arrive.

    python -m cujpegxl_b200.serve [--duration S] [--speed K] [--budget-gb G] [--seed N]

Each admitted stream gets `depth` encoder slots (an encoder with its own CUDA
stream and device arena, plus a device frame buffer). A frame is scheduled the
moment it arrives and a slot of its stream is free; nothing waits to form a
batch, and frames of all streams run concurrently on their slots' streams (the
GPU interleaves their kernels). Per frame: the pinned host frame is copied to
the device, encoded with the C ABI's asynchronous entry point, and the end of
the encode is marked with a CUDA event; latency is that event's device time
minus the frame's arrival time, both measured from one start event.

Admission: a stream is admitted only if the device memory its slots hold
(cujpegxl_b200_encoder_memory, plus the frame buffers) fits in what remains of
the budget; otherwise AdmissionError and nothing of it stays allocated.

The default workload is 2 x 3840x2160 at 30 frames/s, 4 x 1920x1080 at 60 and
2 x 1280x720 at 60, Poisson arrivals (seed 0), distance 1.0, a 40 GB budget.
`--speed K` scales every stream's rate by K to find the sustained throughput.
"""

from __future__ import annotations

import argparse
import json
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
    if not values:
        return None
    s = sorted(values)
    return s[min(len(s) - 1, int(round(q / 100.0 * (len(s) - 1))))]


@dataclass
class _Slot:
    enc: object
    stream: object
    luma: object
    chroma: object
    done: object = None
    arrival_ms: float = 0.0
    busy: bool = False


@dataclass
class _Stream:
    spec: StreamSpec
    slots: list
    host_luma: object
    host_chroma: object
    reserved: int
    queue: deque = field(default_factory=deque)
    latencies: list = field(default_factory=list)
    sizes: list = field(default_factory=list)


class Server:
    def __init__(self, device: int = 0, budget_bytes: float = 40e9, depth: int = 2, net=None,
                 margin: float = 0.2, net_flags: int = 1):
        """net: an acsnet.AcsNet for learned transform decisions (owned by the
        caller), attached to every encoder with `margin` and `net_flags`."""
        import torch

        from . import Encoder  # noqa: F401  (fails loudly if the library is missing)

        self.torch = torch
        self.device = device
        self.budget = Budget(int(budget_bytes))
        self.depth = depth
        self.net, self.margin, self.net_flags = net, margin, net_flags
        self.streams: list[_Stream] = []
        torch.cuda.set_device(device)

    def admit(self, spec: StreamSpec, seed: int = 0) -> int:
        """Allocates the stream's slots; raises AdmissionError if they do not fit."""
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
                                   torch.empty((h // 2, w), dtype=torch.uint8, device="cuda")))
        except AdmissionError:
            self.budget.release(reserved)
            for s in slots:
                s.enc.close()
            raise
        nv = make_nv12(w, h, seed)
        host_luma = torch.from_numpy(nv[: w * h].reshape(h, w).copy()).pin_memory()
        host_chroma = torch.from_numpy(nv[w * h:].reshape(h // 2, w).copy()).pin_memory()
        self.streams.append(_Stream(spec, slots, host_luma, host_chroma, reserved))
        return len(self.streams) - 1

    def _launch(self, st: _Stream, slot: _Slot, arrival_ms: float) -> None:
        torch = self.torch
        w = st.spec.width
        with torch.cuda.stream(slot.stream):
            slot.luma.copy_(st.host_luma, non_blocking=True)
            slot.chroma.copy_(st.host_chroma, non_blocking=True)
        slot.enc.enqueue(slot.luma.data_ptr(), slot.chroma.data_ptr(), w, w)
        slot.done = torch.cuda.Event(enable_timing=True)
        slot.done.record(slot.stream)
        slot.arrival_ms = arrival_ms
        slot.busy = True

    def run(self, duration: float, seed: int = 0, speed: float = 1.0) -> dict:
        torch = self.torch
        rng = np.random.Generator(np.random.PCG64(seed))
        events = []
        for i, st in enumerate(self.streams):
            st.queue.clear()
            st.latencies.clear()
            st.sizes.clear()
            for t in poisson_arrivals(st.spec.fps * speed, duration, rng):
                events.append((float(t), i))
        events.sort()
        offered = len(events)
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record(self.streams[0].slots[0].stream)
        t0 = time.perf_counter()
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
                        st.latencies.append(start.elapsed_time(slot.done) - slot.arrival_ms)
                        st.sizes.append(slot.enc.result()[0])
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
        mp = sum(st.spec.width * st.spec.height * len(st.latencies) for st in self.streams) / 1e6
        return {"duration_s": duration, "speed": speed, "offered_frames": offered, "frames": done,
                "sustained_fps": done / wall, "sustained_mp_per_s": mp / wall,
                "p50_ms": percentile(all_lat, 50), "p99_ms": percentile(all_lat, 99),
                "device_bytes_admitted": self.budget.used, "streams": per}

    def close(self) -> None:
        # Torch's pinned-memory allocator records events on every stream a
        # pinned block was copied on when the block is freed, so every torch
        # object that touched an encoder's stream goes before that stream.
        import gc

        self.torch.cuda.synchronize()
        for st in self.streams:
            st.host_luma = None
            st.host_chroma = None
            for slot in st.slots:
                slot.done = None
                slot.stream = None
                slot.luma = None
                slot.chroma = None
        gc.collect()
        self.torch.cuda.synchronize()
        for st in self.streams:
            for slot in st.slots:
                slot.enc.close()
            self.budget.release(st.reserved)
        self.streams.clear()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--duration", type=float, default=5.0)
    ap.add_argument("--speed", type=float, default=1.0)
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--depth", type=int, default=2)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--learned", action="store_true", help="learned transform decisions (shipped weights)")
    args = ap.parse_args()
    net = None
    if args.learned:
        from .acsnet import AcsNet
        net = AcsNet.load(device_ordinal=args.device)
    srv = Server(args.device, args.budget_gb * 1e9, args.depth, net)
    rejected = []
    for i, spec in enumerate(DEFAULT_STREAMS):
        try:
            srv.admit(spec, seed=i)
        except AdmissionError as e:
            rejected.append(str(e))
    result = srv.run(args.duration, seed=args.seed, speed=args.speed)
    result["rejected"] = rejected
    print(json.dumps(result), flush=True)
    srv.close()
    if net is not None:
        net.close()


if __name__ == "__main__":
    main()
