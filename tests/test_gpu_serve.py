"""The serving loop on the GPU: every arriving frame of every admitted stream
is encoded and delivered to host memory, each delivered file is byte for
byte the file that the same frame gives when encoded alone (plain and with
learned decisions), and a stream that does not fit the budget is refused
without leaking its allocations."""

from __future__ import annotations

import hashlib

import pytest

from cujpegxl_b200 import Encoder
from cujpegxl_b200.serve import AdmissionError, Server, StreamSpec
from cujpegxl_b200.synth import make_nv12

from .gpu_util import device_nv12

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("learned", [False, True])
def test_each_served_file_equals_the_frame_encoded_alone(learned):
    """Frames of three streams (two geometries, two distances) overlap on the
    device; every delivered file's SHA-256 equals that of the same seeded
    frame encoded by a lone encoder with the same settings."""
    from cujpegxl_b200.acsnet import QF, SPLIT, AcsNet
    net = AcsNet.load() if learned else None
    flags = SPLIT | QF
    specs = [StreamSpec("a", 512, 384, 150.0), StreamSpec("b", 264, 264, 250.0, 2.0),
             StreamSpec("c", 640, 480, 150.0, 0.5)]
    srv = Server(0, 8e9, depth=2, net=net, net_flags=flags, frames=3)
    try:
        for i, s in enumerate(specs):
            srv.admit(s, seed=i)
        r = srv.run(0.6, seed=0, verify=True)
        assert r["frames"] == r["offered_frames"] > 0
        assert 0 <= r["clock_offset_bound_ms"] < 50
        for s in specs:
            st = r["streams"][s.name]
            assert st["frames"] == len(st["digests"]) > 3
            expected = {}
            for k, seed in enumerate(st["frame_seeds"]):
                nv = make_nv12(s.width, s.height, seed)
                keep, luma, chroma, lp, cp = device_nv12(nv, s.width, s.height)
                with Encoder(s.width, s.height, s.distance) as enc:
                    if net is not None:
                        enc.set_acsnet(net, 0.2, flags)
                    expected[k] = hashlib.sha256(enc.encode_device(luma, chroma, lp, cp)).hexdigest()
                    enc.set_acsnet(None)
            assert len(set(expected.values())) == len(expected), "the stream's frames must differ"
            seen = set()
            for k, digest in st["digests"]:
                assert digest == expected[k], (s.name, k)
                seen.add(k)
            assert seen == set(expected), "every distinct frame of the stream was served"
            assert st["p99_ms"] >= st["p50_ms"] > 0
    finally:
        srv.close()
        if net is not None:
            net.close()


def test_large_files_take_the_second_copy():
    """A slot buffer smaller than the file: the file is still delivered whole."""
    specs = [StreamSpec("small-buffer", 512, 384, 100.0)]
    srv = Server(0, 8e9, depth=1, frames=2, out_capacity=4096)
    try:
        srv.admit(specs[0], seed=5)
        r = srv.run(0.2, seed=1, verify=True)
        st = r["streams"]["small-buffer"]
        assert st["frames"] == r["offered_frames"] > 0
        nv = make_nv12(512, 384, st["frame_seeds"][0])
        keep, luma, chroma, lp, cp = device_nv12(nv, 512, 384)
        with Encoder(512, 384, 1.0) as enc:
            data = enc.encode_device(luma, chroma, lp, cp)
        assert len(data) > 4096
        assert all(d == hashlib.sha256(data).hexdigest() for k, d in st["digests"] if k == 0)
    finally:
        srv.close()


def test_admission_refuses_what_does_not_fit():
    srv = Server(0, 16e6, depth=2)
    try:
        with pytest.raises(AdmissionError):
            srv.admit(StreamSpec("big", 1920, 1080, 30.0))
        assert srv.budget.used == 0 and not srv.streams
    finally:
        srv.close()
