"""Serving loop (bv_server_*) on the GPU.

Every render frame must be bit-identical to what the tracer's own
dispatch_batch renders for the same camera (which the walk tests pin to the
oracle bit for bit), whether the request is served alone or in a mix with
other scenes, resolutions and forward+backward requests, in batched or plain
mode, with or without graph replay, and whether its frames share one batch or
are split over several.  Forward+backward requests: colours bit-identical to
bv_forward_backward, loss and gradients equal up to the order of the FP32
atomic additions (1e-5 relative to the table's largest entry).
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402

pytestmark = pytest.mark.gpu

SIZES = [(64, 48), (37, 29), (96, 96), (8, 4), (130, 70)]


@pytest.fixture(scope="module")
def models():
    return [scenes.radfoam_ball(n, seed=s, sh_degree=3) for n, s in ((3000, 1), (6000, 2), (1500, 3))]


@pytest.fixture(scope="module")
def reference_tracers(models):
    ts = [bv.RadFoamGpuTracer(m, max_steps=1024, weight_threshold=1e-3) for m in models]
    yield ts
    for t in ts:
        t.deinit()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def make_requests(n_scenes, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        w, h = SIZES[int(rng.integers(len(SIZES)))]
        views = int(rng.integers(1, 5))
        cams = scenes.sphere_cameras(views, 3.0, int(rng.integers(1 << 20)), math.radians(55.0),
                                     w / h, 100.0)
        reqs.append(dict(scene=int(rng.integers(n_scenes)), cams=cams, w=w, h=h))
    return reqs


def expected(tracers, req):
    img = tracers[req["scene"]].render(req["cams"], req["w"], req["h"])
    torch.cuda.synchronize()
    return img.cpu().numpy()


def new_server(models, budget=2 << 30, **kw):
    kw.setdefault("max_train_rays", 1 << 20)
    s = bv.Server(budget, **kw)
    for m in models:
        s.add_scene(m)
    s.start()
    return s


def serve(server, reqs):
    outs, ids = [], []
    for r in reqs:
        out = np.full((len(r["cams"]), r["h"], r["w"], 4), np.nan, np.float32)
        fd = np.zeros(len(r["cams"]))
        ids.append(server.submit(r["scene"], r["cams"], r["w"], r["h"], out=out, frame_done=fd))
        outs.append((out, fd))
    results = [server.wait(i, 120.0) for i in ids]
    return outs, results


@pytest.mark.parametrize("kw", [dict(), dict(max_batch_rays=10240, slots=3),
                                dict(use_graphs=False), dict(mode="plain"),
                                dict(mode="plain_batch")],
                         ids=["batched", "split-batches", "no-graphs", "plain", "plain-batch"])
def test_mixed_stream_matches_tracer(models, reference_tracers, kw):
    reqs = make_requests(len(models), 24, seed=11)
    server = new_server(models, **kw)
    try:
        outs, results = serve(server, reqs)
        st = server.stats()
    finally:
        server.close()
    for r, (out, fd), res in zip(reqs, outs, results):
        assert res["status"] == 0, res["message"]
        ref = expected(reference_tracers, r)
        assert np.array_equal(bits(out), bits(ref)), (r["scene"], r["w"], r["h"])
        assert res["submit_s"] <= res["admit_s"] <= res["start_s"] <= res["done_s"]
        assert np.all(fd > 0) and np.all(fd <= res["done_s"] + 1e-9)
    assert st["requests_done"] == len(reqs)
    assert st["frames_done"] == sum(len(r["cams"]) for r in reqs)
    if kw.get("mode") is None:
        assert st["batches"] >= 1
        if kw.get("max_batch_rays") == 10240:
            assert st["batches"] > len(reqs) // 2  # frames spread over many batches
        if kw.get("use_graphs", True):
            assert st["graph_launches"] == st["batches"]


def test_same_alone_and_in_mix(models, reference_tracers):
    reqs = make_requests(len(models), 12, seed=5)
    server = new_server(models)
    try:
        mixed, _ = serve(server, reqs)
        alone = [serve(server, [r])[0][0] for r in reqs]
    finally:
        server.close()
    for (m, _), (a, _) in zip(mixed, alone):
        assert np.array_equal(bits(m), bits(a))


@pytest.mark.parametrize("chunk,rec", [(0, 0), (1024, 0), (1024, 3), (0, None)],
                         ids=["one-launch-pair", "chunks-of-1024-rays", "3-step-record",
                              "no-record"])
def test_forward_backward_requests_in_the_mix(models, reference_tracers, chunk, rec):
    """chunk: the server's training launch pairs cover at most this many
    work items (0: its default, larger than these requests); rec: the steps
    per ray of the step record the server lends (0: automatic, 3: the replay
    searches past the third step, None: it searches every step); the results
    are the tracer's own."""
    w, h = 48, 40
    cams = scenes.sphere_cameras(3, 3.0, 9, math.radians(55.0), w / h, 100.0)
    target = np.random.default_rng(2).random((3, h, w, 3)).astype(np.float32)
    # the tracer's own gradient call
    t = reference_tracers[0]
    g_ref = t.new_grads()
    tgt_dev = torch.from_numpy(target).cuda()
    rgb_ref = torch.zeros((3, h, w, 3), dtype=torch.float32, device="cuda")
    loss_ref = t.forward_backward(cams, w, h, tgt_dev, g_ref, rgb_out=rgb_ref,
                                  weight_threshold=0.0, max_dt=50.0)
    torch.cuda.synchronize()
    server = new_server(models, train_chunk_rays=chunk, train_record_steps=rec)
    try:
        renders = make_requests(len(models), 10, seed=3)
        ids = []
        outs = []
        for r in renders[:5]:
            out = np.zeros((len(r["cams"]), r["h"], r["w"], 4), np.float32)
            ids.append(server.submit(r["scene"], r["cams"], r["w"], r["h"], out=out))
            outs.append(out)
        g = t.new_grads()
        torch.cuda.synchronize()  # the server works on streams of its own
        rgb = np.zeros((3, h, w, 3), np.float32)
        loss = np.zeros(1, np.float32)
        fid = server.submit(0, cams, w, h, out=rgb, target=target, loss=loss, grads=g,
                            weight_threshold=0.0, max_dt=50.0)
        for r in renders[5:]:
            out = np.zeros((len(r["cams"]), r["h"], r["w"], 4), np.float32)
            ids.append(server.submit(r["scene"], r["cams"], r["w"], r["h"], out=out))
            outs.append(out)
        res = server.wait(fid, 120.0)
        for i in ids:
            assert server.wait(i, 120.0)["status"] == 0
    finally:
        server.close()
    assert res["status"] == 0, res["message"]
    assert np.array_equal(bits(rgb), bits(rgb_ref.cpu().numpy()))
    assert abs(float(loss[0]) - float(loss_ref)) <= 1e-5 * abs(float(loss_ref))
    for k in g_ref:
        a, b = g[k].cpu().numpy(), g_ref[k].cpu().numpy()
        scale = max(float(np.abs(b).max()), 1e-30)
        assert float(np.abs(a - b).max()) <= 1e-5 * scale, k
    for r, out in zip(renders, outs):
        assert np.array_equal(bits(out), bits(expected(reference_tracers, r)))


def test_scene_gradient_tables_accumulate(models):
    server = bv.Server(1 << 30, max_train_rays=1 << 20)
    server.add_scene(models[2], gradients=True)
    server.start()
    try:
        w = h = 32
        cams = scenes.sphere_cameras(2, 3.0, 4, math.radians(55.0), 1.0, 100.0)
        target = np.zeros((2, h, w, 3), np.float32)
        loss = np.zeros(1, np.float32)
        res = server.wait(server.submit(0, cams, w, h, target=target, loss=loss), 60.0)
        assert res["status"] == 0, res["message"]
        assert loss[0] > 0
        g = server.scene_grads(0)
        assert g.d_density_dev and g.d_sh_dev and g.d_positions_dev
    finally:
        server.close()


def test_admission_under_a_small_budget(models, reference_tracers):
    # no training step record: the resident bytes then do not depend on the budget
    probe = new_server(models, budget=1 << 30, train_record_steps=None)
    resident = probe.stats()["resident_bytes"]
    probe.close()
    reqs = make_requests(len(models), 16, seed=21)
    biggest = max(len(r["cams"]) * r["w"] * r["h"] * 16 for r in reqs)
    arena_want = 2 * biggest + 4096
    server = new_server(models, budget=resident + arena_want, train_record_steps=None)
    try:
        st0 = server.stats()
        assert st0["arena_bytes"] <= arena_want
        outs, results = serve(server, reqs)
        st = server.stats()
        with pytest.raises(bv.BvError) as e:  # can never fit
            big = scenes.sphere_cameras(4, 3.0, 1, 1.0, 1.0, 100.0)
            server.submit(0, big, 512, 512, out=np.zeros((4, 512, 512, 4), np.float32))
        assert e.value.status == 4
    finally:
        server.close()
    assert st["arena_peak_bytes"] <= st["arena_bytes"]
    assert st["admission_waits"] > 0
    for r, (out, _), res in zip(reqs, outs, results):
        assert res["status"] == 0
        assert np.array_equal(bits(out), bits(expected(reference_tracers, r)))


def test_rejects_bad_requests(models):
    server = bv.Server(1 << 30, max_batch_rays=4096, max_train_rays=1 << 20)
    with pytest.raises(bv.BvError):
        server.submit(0, scenes.sphere_cameras(1, 3.0, 1, 1.0, 1.0, 100.0), 8, 8,
                      out=np.zeros((1, 8, 8, 4), np.float32))  # not started
    server.add_scene(models[0])
    with pytest.raises(bv.BvError):  # mixed SH degree
        server.add_scene(scenes.radfoam_ball(500, seed=1, sh_degree=1))
    server.start()
    try:
        cam = scenes.sphere_cameras(1, 3.0, 1, 1.0, 1.0, 100.0)
        with pytest.raises(bv.BvError):
            server.submit(5, cam, 8, 8, out=np.zeros((1, 8, 8, 4), np.float32))
        with pytest.raises(bv.BvError):  # frame above max_batch_rays
            server.submit(0, cam, 128, 128, out=np.zeros((1, 128, 128, 4), np.float32))
        with pytest.raises(bv.BvError):  # scene keeps no gradient tables
            server.submit(0, cam, 8, 8, target=np.zeros((1, 8, 8, 3), np.float32),
                          loss=np.zeros(1, np.float32))
        with pytest.raises(bv.BvError):
            server.wait(12345, 0.1)
    finally:
        server.close()
    with pytest.raises(bv.BvError):
        bv.Server(1 << 30, train_record_steps=257)


def test_cancel_withdraws_requests_and_returns_their_arena_bytes(models, reference_tracers):
    """Requests queued behind a small arena are withdrawn: each finishes with
    BV_ERR_CANCELLED (or, if it had already finished, with its own status
    and a correct image), the arena holds no bytes once everything is done,
    and cancelling a finished request changes nothing."""
    probe = new_server(models, budget=1 << 30)
    resident = probe.stats()["resident_bytes"]
    probe.close()
    w = h = 256
    frame = 4 * w * h * 16
    server = new_server(models, budget=resident + 2 * frame + 4096)
    try:
        reqs = []
        for i in range(10):
            cams = scenes.sphere_cameras(4, 3.0, 40 + i, math.radians(55.0), 1.0, 100.0)
            reqs.append(dict(scene=i % len(models), cams=cams, w=w, h=h))
        outs, ids = [], []
        for r in reqs:
            out = np.zeros((4, h, w, 4), np.float32)
            ids.append(server.submit(r["scene"], r["cams"], w, h, out=out))
            outs.append(out)
        for rid in ids[2:]:
            server.cancel(rid)
        results = [server.wait(rid, 120.0) for rid in ids]
        st = server.stats()
        done = server.submit(0, reqs[0]["cams"][:1], 8, 8, out=np.zeros((1, 8, 8, 4), np.float32))
        res_done = server.wait(done, 60.0)
        with pytest.raises(bv.BvError):
            server.cancel(done)  # forgotten once waited for
    finally:
        server.close()
    assert res_done["status"] == 0
    statuses = [r["status"] for r in results]
    assert set(statuses) <= {0, bv.BV_ERR_CANCELLED}, statuses
    assert statuses[0] == 0 and statuses[1] == 0
    assert statuses.count(bv.BV_ERR_CANCELLED) >= 4
    assert st["requests_cancelled"] == statuses.count(bv.BV_ERR_CANCELLED)
    assert st["arena_used_bytes"] == 0
    for r, out, res in zip(reqs, outs, results):
        if res["status"] == 0:
            assert np.array_equal(bits(out), bits(expected(reference_tracers, r)))
