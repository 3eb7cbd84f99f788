"""Multi-rank data-parallel step on CPU (world size 2, gloo over 127.0.0.1).

Each rank differentiates its own views (blade_volume_b200.dist.rank_cameras)
with the FP64 gradient oracle standing in for the device kernel, then the
ranks sum their gradient tables with blade_volume_b200.dist.allreduce_grads,
the one exchange of the training step.  The summed tables must equal the
per-rank gradients added up in one process, and max_over_ranks must return
the slowest rank's time.
"""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as tdist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import dist as bvdist  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402

WORLD = 2
SIDE = 24
VIEWS = 2


def scene():
    return scenes.radfoam_ball(768, seed=11, sh_degree=1, jitter=0.0)


def rank_grads(model, rank):
    om = O.OracleModel.from_scene(model)
    cams = bvdist.rank_cameras(VIEWS, rank)
    target = np.full((VIEWS, SIDE, SIDE, 3), 0.3, np.float32)
    g = O.forward_backward(om, cams, SIDE, SIDE, target=target, threads=1)
    return {k: g[k] for k in ("d_density", "d_sh", "d_pos")}


def worker(rank, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    tdist.init_process_group("gloo", rank=rank, world_size=WORLD,
                             timeout=__import__("datetime").timedelta(seconds=60))
    try:
        g = rank_grads(scene(), rank)
        # a plain dict of tables: packed into one bucket, one collective
        tables = {k: torch.from_numpy(np.array(v, copy=True).reshape(-1)) for k, v in g.items()}
        bvdist.allreduce_grads(tables, tdist)
        # a tracer's tables (views of one flat buffer): the buffer is reduced
        flat = bv._grad_tables(len(g["d_density"]), len(g["d_sh"]) // len(g["d_density"]),
                               False, device="cpu")
        for k, v in g.items():
            flat[k].copy_(torch.from_numpy(np.ascontiguousarray(v).reshape(-1)).float())
        bvdist.allreduce_grads(flat, tdist)
        slowest = bvdist.max_over_ranks([10.0 + rank, 5.0 - rank], tdist, "cpu")
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), slowest=np.array(slowest),
                 **{k: v.numpy() for k, v in tables.items()},
                 **{"flat_" + k: v.numpy() for k, v in flat.items()})
    finally:
        tdist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gradient_allreduce_across_two_gloo_ranks(tmp_path):
    mp.start_processes(worker, args=(free_port(), str(tmp_path)), nprocs=WORLD, join=True,
                       start_method="spawn")
    model = scene()
    want = [rank_grads(model, r) for r in range(WORLD)]
    for r in range(WORLD):
        got = np.load(tmp_path / f"rank{r}.npz")
        assert list(got["slowest"]) == [11.0, 5.0]
        for k in ("d_density", "d_sh", "d_pos"):
            total = sum(np.asarray(w[k]).reshape(-1) for w in want)
            assert np.abs(total).max() > 0
            np.testing.assert_allclose(got[k], total, rtol=1e-12, atol=1e-15)
            np.testing.assert_allclose(got["flat_" + k], total.astype(np.float32), rtol=1e-6,
                                       atol=1e-6 * np.abs(total).max())
    # the ranks rendered different views: their gradients differ
    assert not np.allclose(want[0]["d_density"], want[1]["d_density"])
