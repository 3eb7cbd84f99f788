"""Serving loop host side, no GPU: settings validation through the C ABI,
the request-stream generator and the latency summaries."""

import ctypes as C

import numpy as np
import pytest

import blade_volume_b200 as bv
from blade_volume_b200 import serving


def new_server_status(**kw):
    s = bv.ServerSettings()
    s.hbm_budget_bytes = kw.get("budget", 1 << 30)
    s.mode = kw.get("mode", bv.SERVE_BATCHED)
    s.max_batch_views = kw.get("views", 0)
    s.slots = kw.get("slots", 0)
    s.weight_threshold = kw.get("threshold", 1e-3)
    h = C.c_void_p()
    st = bv.load_library().bv_server_new(C.byref(s), C.byref(h))
    if st == 0:
        bv.load_library().bv_server_destroy(h)
    return st


@pytest.mark.parametrize("kw", [dict(mode=7), dict(views=5000), dict(slots=9), dict(budget=0),
                                dict(threshold=float("nan"))])
def test_bad_settings_are_refused_before_any_device_work(kw):
    assert new_server_status(**kw) == 1  # BV_ERR_INVALID_ARGUMENT


def test_null_arguments():
    L = bv.load_library()
    assert L.bv_server_new(None, None) == 1
    assert L.bv_server_start(None) == 1
    assert L.bv_server_submit(None, None, None) == 1
    res = bv.RequestResult()
    assert L.bv_server_wait(None, 1, 0.0, C.byref(res)) == 1
    L.bv_server_destroy(None)


def test_abi_struct_sizes():
    # the C layouts (x86-64): settings 56, request 112, result 184, stats 88 bytes
    assert C.sizeof(bv.ServerSettings) == 56
    assert C.sizeof(bv.RequestC) == 112
    assert C.sizeof(bv.RequestResult) == 184
    assert C.sizeof(bv.ServerStats) == 104


def test_poisson_stream_statistics():
    specs = serving.poisson_stream(rate=200.0, count=4000, n_scenes=4, seed=1)
    gaps = np.diff([0.0] + [s.arrival for s in specs])
    assert abs(gaps.mean() - 1 / 200.0) < 0.05 / 200.0
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05  # exponential: cv = 1
    fb = np.mean([s.fwdbwd for s in specs])
    assert 0.08 < fb < 0.12
    views = np.array([s.views for s in specs])
    assert views.min() == 1 and views.max() == 16
    res = {(s.width, s.height) for s in specs}
    assert res == set(serving.RESOLUTIONS)
    assert {s.scene for s in specs} == {0, 1, 2, 3}
    assert all(len(s.cameras) == s.views for s in specs[:50])
    # reproducible
    again = serving.poisson_stream(rate=200.0, count=10, n_scenes=4, seed=1)
    assert [s.arrival for s in again] == [s.arrival for s in specs[:10]]


def test_percentile():
    assert serving.percentile([], 50) is None
    v = list(range(1, 101))
    assert serving.percentile(v, 50) == pytest.approx(50.5)
    assert serving.percentile(v, 99) == pytest.approx(99.01)


class _FakeServer:
    """Stands in for bv.Server on the host: a clock that advances 1 ms per
    read, frames that land 4 ms after submission plus one 16 ms period per
    frame, and training requests that run 50 ms."""

    def __init__(self):
        self.now = 100.0
        self.reqs = {}

    def clock(self):
        self.now += 1e-3
        return self.now

    def submit(self, scene, cams, w, h, out=None, target=None, loss=None, frame_done=None):
        rid = len(self.reqs)
        t = self.now
        if target is None:
            frame_done[:] = t + 0.004 + 0.016 * np.arange(len(frame_done))
            done = float(frame_done[-1])
        else:
            frame_done[:] = t + 0.05
            done = t + 0.05
        self.reqs[rid] = dict(status=0, start_s=t, done_s=done)
        return rid

    def wait(self, rid, timeout):
        return self.reqs[rid]


class _FakeBuffers:
    def request_args(self, spec):
        return dict(target=np.zeros(1)) if spec.fwdbwd else dict(out=np.zeros(1))


def test_run_stream_paces_frames_and_keeps_training_out_of_frame_figures():
    cams = []
    specs = [serving.RequestSpec(arrival=0.002 * i, scene=0, width=1920, height=1080,
                                 views=4, fwdbwd=(i % 3 == 2), cameras=cams)
             for i in range(9)]
    r = serving.run_stream(_FakeServer(), specs, _FakeBuffers(), frame_period_s=0.016)
    hd = r["per_resolution"]["1920x1080"]
    # 6 render requests of 4 frames; the 3 training requests are not frames
    assert hd["frame"]["n"] == 24 and hd["first_frame"]["n"] == 6
    assert r["per_resolution_fwdbwd"]["1920x1080"]["n"] == 3
    # each frame lands 4 ms after its request was submitted plus k periods:
    # paced latency is that 4 ms plus the submission's lag behind arrival
    assert 3.9 < hd["paced_frame"]["p50_ms"] < 8.0
    assert hd["paced_frame"]["p99_ms"] < 8.0
    assert hd["frame"]["p99_ms"] > 48.0  # the last frames, 3 periods later
    # training work: 3 x 4 x 1080p rays over 50 ms each
    want = 3 * 4 * 1920 * 1080 / (3 * 0.05) / 1e6
    assert abs(r["fwdbwd_service_mrays_per_s"] - want) < 1e-6 * want
