"""The multi-rank path (replicas + one FP64 film reduction) with world_size 2 on gloo (CPU).

Each rank renders the same scene with the oracle (the CPU checker stands in for
the GPU renderer here) using its own random streams; combine_films must return
the mean of the two films on rank 0, and that mean must agree statistically with
a single render of twice the samples.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT, golden_scene


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, path, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import oracle
    from wurstrenderer_b200.distributed import combine_films, max_over_ranks, rank_seed
    sc = oracle.OracleScene(path)
    img, sec, _ = sc.render(spp=64, salt=rank_seed(5, rank), threads=1)
    np.save(os.path.join(out_dir, "rank%d.npy" % rank), img)
    film = torch.from_numpy(img.copy())
    combine_films(film, world, dist)
    t = max_over_ranks(sec, world, dist)
    if rank == 0:
        np.save(os.path.join(out_dir, "combined.npy"), film.numpy())
        np.save(os.path.join(out_dir, "tmax.npy"), np.array([t]))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_reduce_to_the_mean(tmp_path):
    path, _ = golden_scene("cornell")
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, path, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    comb = np.load(tmp_path / "combined.npy")
    assert not np.array_equal(r0, r1)                 # distinct random streams per rank
    assert np.allclose(comb, (r0 + r1) / 2.0, rtol=1e-12, atol=1e-15)
    assert np.load(tmp_path / "tmax.npy")[0] > 0
    ref = np.load(os.path.join(ROOT, "tests", "golden", "cornell_ref_hi_a.npy")).astype(np.float64)
    assert abs(comb.mean() / ref.mean() - 1.0) < 0.03


def test_rank_seeds_distinct():
    from wurstrenderer_b200.distributed import rank_seed
    seeds = {rank_seed(7, r) for r in range(64)}
    assert len(seeds) == 64
    assert rank_seed(7, 0) == 7
