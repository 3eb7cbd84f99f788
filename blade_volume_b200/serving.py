"""Request streams for the serving loop (:class:`blade_volume_b200.Server`).

The workload: several resident RadFoam scenes; requests arrive as a Poisson
process; each picks a scene and a resolution uniformly, 1-16 views, and a
tenth of them ask for forward+backward with an L2 loss against a target
image.  :func:`run_stream` submits every request at its arrival time (on the
server's clock), waits for all of them and reports aggregate Mrays/s and
p50/p99 latencies, each measured from the request's scheduled arrival:
  request      until every output of the request is on the host;
  first_frame  until its first frame (view) is on the host;
  frame        until each frame is on the host (one sample per frame);
  frame_interval  the time a viewer of the request waits for each frame: the
               first frame from arrival, every later one from the frame
               before it (frames in the order they landed);
  paced_frame  a streamed request: frame k is asked for k frame periods
               after arrival (the server's deadline for it is one period
               later), and its latency runs from then until it is on the
               host (negative when it landed ahead of being asked for).
Frame figures cover render requests; a forward+backward request's colours
land with its gradients, so it counts in request latency only.  Its work is
summarised as Mrays/s over the stream's span and over the time from its
first launch to its outputs (service Mrays/s).

Host buffers: each resolution has one pinned output sink and one pinned
target, shared by every request of that resolution (the outputs overwrite
one another).  The copies are real, full-size device-to-host transfers;
only their destination is shared, so that a long stream needs no pinned
memory per request.  Correctness of every frame is the business of the
serving tests, which give each request its own buffers.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import scenes

RESOLUTIONS: Tuple[Tuple[int, int], ...] = ((256, 256), (512, 512), (1280, 720), (1920, 1080))
SERVE_SCENE_SITES: Tuple[int, ...] = (65536, 262144, 524288, 1048576)


@dataclass
class RequestSpec:
    arrival: float            # seconds after the stream starts
    scene: int
    width: int
    height: int
    views: int
    fwdbwd: bool
    cameras: List[scenes.Camera] = field(default_factory=list)

    @property
    def rays(self) -> int:
        return self.views * self.width * self.height


def poisson_stream(rate: float, count: int, n_scenes: int, seed: int,
                   resolutions: Sequence[Tuple[int, int]] = RESOLUTIONS, max_views: int = 16,
                   fwdbwd_fraction: float = 0.1) -> List[RequestSpec]:
    """``count`` requests with exponential inter-arrival gaps of mean 1/rate."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        views = int(rng.integers(1, max_views + 1))
        cams = scenes.sphere_cameras(views, 3.0, int(rng.integers(1 << 30)), math.radians(60.0),
                                     w / h, 100.0)
        out.append(RequestSpec(arrival=t, scene=int(rng.integers(n_scenes)), width=w, height=h,
                               views=views, fwdbwd=bool(rng.random() < fwdbwd_fraction),
                               cameras=cams))
    return out


def build_scene(args) -> scenes.PointCloudModel:
    n, seed = args
    return scenes.radfoam_ball(n, seed=seed, sh_degree=3)


def serving_scenes(sites: Sequence[int] = SERVE_SCENE_SITES, processes: int = 4):
    """The resident scenes: RadFoam balls (uniform unit ball, lognormal(0,1)
    density, SH degree 3 FP32) with seeds 1..len(sites).  Built in spawned
    worker processes (safe before or after CUDA is initialised)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    jobs = [(n, i + 1) for i, n in enumerate(sites)]
    if processes <= 1:
        return [build_scene(j) for j in jobs]
    with cf.ProcessPoolExecutor(max_workers=min(processes, len(jobs)),
                                mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(build_scene, jobs))


class HostBuffers:
    """Pinned per-resolution output sinks and targets (see module notes)."""

    def __init__(self, resolutions=RESOLUTIONS, max_views: int = 16, seed: int = 7):
        import torch

        rng = np.random.default_rng(seed)
        self.out: Dict[Tuple[int, int], object] = {}
        self.rgb: Dict[Tuple[int, int], object] = {}
        self.target: Dict[Tuple[int, int], object] = {}
        self.loss = torch.zeros(1, dtype=torch.float32).pin_memory()
        for w, h in resolutions:
            self.out[(w, h)] = torch.empty((max_views, h, w, 4), dtype=torch.float32,
                                           pin_memory=True)
            self.rgb[(w, h)] = torch.empty((max_views, h, w, 3), dtype=torch.float32,
                                           pin_memory=True)
            tgt = torch.from_numpy(rng.random((max_views, h, w, 3), dtype=np.float32))
            self.target[(w, h)] = tgt.pin_memory()

    def request_args(self, spec: RequestSpec) -> dict:
        key = (spec.width, spec.height)
        if spec.fwdbwd:
            return dict(out=self.rgb[key][: spec.views], target=self.target[key][: spec.views],
                        loss=self.loss)
        return dict(out=self.out[key][: spec.views])


def percentile(values, q: float) -> Optional[float]:
    if len(values) == 0:
        return None
    return float(np.percentile(np.asarray(values, dtype=np.float64), q))


def run_stream(server, specs: Sequence[RequestSpec], bufs: HostBuffers,
               timeout: float = 600.0, frame_period_s: float = 0.016) -> dict:
    """Submit every request at its arrival time, wait for all, summarise.
    frame_period_s: the server's frame period (frame k of a request is asked
    for k periods after its arrival)."""
    t0 = server.clock() + 0.01
    sub = []
    for spec in specs:
        due = t0 + spec.arrival
        while True:
            d = due - server.clock()
            if d <= 0:
                break
            time.sleep(d if d > 2e-4 else 0.0)
        frame_done = np.zeros(spec.views, dtype=np.float64)
        rid = server.submit(spec.scene, spec.cameras, spec.width, spec.height,
                            frame_done=frame_done, **bufs.request_args(spec))
        sub.append((rid, spec, due, frame_done))
    lat, frame_lat, first_lat, gaps, paced_lat = [], [], [], [], []
    fwdbwd_rays = 0
    fwdbwd_busy = 0.0
    per_res: Dict[str, Dict[str, list]] = {}
    per_res_fb: Dict[str, list] = {}
    per_kind: Dict[str, list] = {"render": [], "fwdbwd": []}
    rays = 0
    end = t0
    failures = 0
    for rid, spec, due, frame_done in sub:
        r = server.wait(rid, timeout)
        if r["status"] != 0:
            failures += 1
            continue
        rays += spec.rays
        end = max(end, r["done_s"])
        key = f"{spec.width}x{spec.height}"
        lat.append(r["done_s"] - due)
        per_kind["fwdbwd" if spec.fwdbwd else "render"].append(r["done_s"] - due)
        if spec.fwdbwd:
            # a training request's colours land with its gradients: no frames
            fwdbwd_rays += spec.rays
            fwdbwd_busy += r["done_s"] - r["start_s"]
            per_res_fb.setdefault(key, []).append(r["done_s"] - due)
            continue
        d = per_res.setdefault(key, dict(request=[], frame=[], first_frame=[],
                                         frame_interval=[], paced_frame=[]))
        d["request"].append(r["done_s"] - due)
        f = [float(x) - due for x in frame_done]
        frame_lat.extend(f)
        d["frame"].extend(f)
        first_lat.append(min(f))
        d["first_frame"].append(min(f))
        landed = sorted(f)
        g = [landed[0]] + [b - a for a, b in zip(landed, landed[1:])]
        gaps.extend(g)
        d["frame_interval"].extend(g)
        paced = [x - k * frame_period_s for k, x in enumerate(f)]
        paced_lat.extend(paced)
        d["paced_frame"].extend(paced)
    span = end - t0
    ms = 1e3

    def pct(v):
        return dict(p50_ms=None if not v else percentile(v, 50) * ms,
                    p99_ms=None if not v else percentile(v, 99) * ms, n=len(v))

    return dict(requests=len(specs), failures=failures, rays=rays, span_s=span,
                mrays_per_s=rays / span / 1e6 if span > 0 else None,
                fwdbwd_mrays_per_s=fwdbwd_rays / span / 1e6 if span > 0 else None,
                fwdbwd_service_mrays_per_s=(fwdbwd_rays / fwdbwd_busy / 1e6
                                            if fwdbwd_busy > 0 else None),
                request_latency=pct(lat), first_frame_latency=pct(first_lat),
                frame_latency=pct(frame_lat), frame_interval=pct(gaps),
                paced_frame_latency=pct(paced_lat),
                per_kind={k: pct(v) for k, v in per_kind.items()},
                per_resolution={k: {m: pct(x) for m, x in v.items()}
                                for k, v in sorted(per_res.items())},
                per_resolution_fwdbwd={k: pct(v) for k, v in sorted(per_res_fb.items())},
                offered_rate=len(specs) / specs[-1].arrival if specs else None)
