"""The multi-rank bench path on the CPU: two processes joined by a gloo
process group, each walking its own ray batch of the terrain workload (a
small grid here) over a replicated scene, as `bench.py --gpus N` does with
one rank per GPU. Checks that every rank's batch has the workload's size and
two ray kinds and differs from the others', that the only collective is the
max of the step time, and that each rank's answers equal a single-process
run of the same batch (sharding exchanges no data). The walks are the
oracle's: the CUDA path's multi-rank run differs only in the device."""
import hashlib
import json
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import bench  # noqa: E402
import oracle as O  # noqa: E402
from spatial_query_b200 import scenes  # noqa: E402

NX, NY = 64, 32


def _scene():
    return scenes.terrain_scene(seed=1, nx=NX, ny=NY)


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = _scene()
        rays = bench.rank_rays(s, rank)
        hits = O.Scene("tris", 3, s["prims"]).nearest(rays, s["max_toi"], threads=1)
        digest = [None] * world
        dist.all_gather_object(digest, hashlib.sha256(rays.tobytes()).hexdigest())
        step_ms = 1.5 + rank  # a stand-in step time per rank
        slowest = bench.max_over_ranks(step_ms, dist)
        np.save(os.path.join(out_dir, f"leaf{rank}.npy"), hits.leaf)
        np.save(os.path.join(out_dir, f"toi{rank}.npy"), hits.toi)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"n": int(rays.shape[0]), "digests": digest, "slowest": slowest}, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


@pytest.mark.timeout(300)
def test_two_gloo_ranks_walk_their_own_batches(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    s = _scene()
    n = s["rays"].shape[0]
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert all(r["n"] == n for r in res)
    assert res[0]["digests"][0] != res[0]["digests"][1]  # distinct batches
    assert all(r["slowest"] == 2.5 for r in res)  # max over ranks on every rank
    sc = O.Scene("tris", 3, s["prims"])
    for r in range(world):
        rays = bench.rank_rays(s, r)
        if r > 0:  # the same two kinds: coherent half pointing down, then isotropic
            assert (rays[: n // 2, 5] < -0.99).all()
            assert (rays[n // 2:, 5] > 0).any()
        ref = sc.nearest(rays, s["max_toi"], threads=1)
        assert np.array_equal(np.load(tmp_path / f"leaf{r}.npy"), ref.leaf)
        assert np.array_equal(np.load(tmp_path / f"toi{r}.npy").view(np.uint32), ref.toi.view(np.uint32))
        assert (ref.leaf != O.NO_HIT).mean() > 0.3


def test_one_process_needs_no_group():
    assert bench.max_over_ranks(3.25) == 3.25
    s = _scene()
    assert bench.rank_rays(s, 0) is s["rays"]
