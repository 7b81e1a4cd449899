"""The multi-rank host logic on CPU: world_size 2 over gloo.  The per-rank
tile analysis is a stand-in that returns records at positions inside the
tiles it is given (no GPU here); the test checks the round-robin shares, the
tile assignment by position, and that rank 0 gathers every record in the
single-process tile order."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from peakpatch_b200 import distributed as D

NTILE, DCORE, NF = 2, 100.0, 33


def _fake_run(tiles):
    """records of each tile: positions inside its core, a field encoding the tile"""
    out = []
    for (it, jt, kt) in tiles:
        c = np.array([(it - 1.5) * DCORE, (jt - 1.5) * DCORE, (kt - 1.5) * DCORE])
        rng = np.random.default_rng(it + 10 * jt + 100 * kt)
        m = 3 + it + jt + kt
        r = np.zeros((m, NF), np.float32)
        r[:, :3] = c + rng.uniform(-0.49 * DCORE, 0.49 * DCORE, (m, 3))
        r[:, 10] = it + 10 * jt + 100 * kt
        r[:, 11] = np.arange(m)
        out.append(r)
    return np.concatenate(out) if out else np.zeros((0, NF), np.float32)


def _worker(rank, world, port, result_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = D.run_multitile_sharded(_fake_run, NTILE, DCORE, NF)
        if rank == 0:
            np.save(result_path, got)
        else:
            assert got is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_and_tile_assignment():
    tiles = D.tile_list(2)
    assert tiles[:3] == [(1, 1, 1), (2, 1, 1), (1, 2, 1)] and len(tiles) == 8
    a, b = D.shard_tiles(tiles, 0, 2), D.shard_tiles(tiles, 1, 2)
    assert sorted(a + b) == sorted(tiles) and not set(a) & set(b)
    rec = _fake_run(tiles)
    t = D.tile_of_records(rec, NTILE, DCORE)
    assert np.array_equal(t[:, 0] + 10 * t[:, 1] + 100 * t[:, 2], rec[:, 10].astype(int))
    with pytest.raises(ValueError):
        D.shard_tiles(tiles, 2, 2)


def test_two_ranks_gather_the_single_process_catalogue(tmp_path):
    path = str(tmp_path / "cat.npy")
    mp.start_processes(_worker, args=(2, _free_port(), path), nprocs=2, join=True, start_method="spawn")
    got = np.load(path)
    ref = _fake_run(D.tile_list(NTILE))
    assert got.shape == ref.shape and got.tobytes() == ref.tobytes()
