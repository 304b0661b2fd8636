"""The serving loop on the GPU: every arriving frame of every admitted stream
is encoded, each output equals the single-encoder file of that stream's
frame, and a stream that does not fit the budget is refused without leaking
its allocations."""

from __future__ import annotations

import pytest

from cujpegxl_b200 import Encoder
from cujpegxl_b200.serve import AdmissionError, Server, StreamSpec
from cujpegxl_b200.synth import make_nv12

from .gpu_util import device_nv12

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("learned", [False, True])
def test_serving_loop_encodes_every_frame(learned):
    """With learned decisions too: every frame in the mix equals the file the
    same network gives that frame alone."""
    from cujpegxl_b200.acsnet import AcsNet
    net = AcsNet.load() if learned else None
    specs = [StreamSpec("a", 512, 384, 120.0), StreamSpec("b", 264, 264, 200.0, 2.0)]
    srv = Server(0, 8e9, depth=2, net=net)
    try:
        for i, s in enumerate(specs):
            srv.admit(s, seed=i)
        r = srv.run(0.5, seed=0)
        assert r["frames"] == r["offered_frames"] > 0
        for i, s in enumerate(specs):
            nv = make_nv12(s.width, s.height, i)
            keep, luma, chroma, lp, cp = device_nv12(nv, s.width, s.height)
            with Encoder(s.width, s.height, s.distance) as enc:
                if net is not None:
                    enc.set_acsnet(net)
                size = len(enc.encode_device(luma, chroma, lp, cp))
                if net is not None:
                    assert enc.acsnet_stats()[0] > 0
                enc.set_acsnet(None)
            st = r["streams"][s.name]
            assert st["frames"] > 0 and st["mean_bytes"] == size
            assert st["p99_ms"] >= st["p50_ms"] > 0
    finally:
        srv.close()
        if net is not None:
            net.close()


def test_admission_refuses_what_does_not_fit():
    srv = Server(0, 16e6, depth=2)
    try:
        with pytest.raises(AdmissionError):
            srv.admit(StreamSpec("big", 1920, 1080, 30.0))
        assert srv.budget.used == 0 and not srv.streams
    finally:
        srv.close()
