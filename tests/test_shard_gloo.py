"""World-size-2 test of the sharded search's host path on CPU (gloo): each
rank scans its shard of subjects (the oracle stands in for the device scan,
since this runs without a GPU), rank 0 gathers and merges, and the merged
answer equals one unsharded scan."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from blastp_b200 import shard, synth


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    m = oracle.load_fixture_matrix()
    w = synth.shape1(m, n_subjects=1500, qlen=120)
    q = w.queries[0]
    b = shard.shard_bounds(w.db.offsets, world)
    res, off = shard.local_database(w.db.residues, w.db.offsets, int(b[rank]), int(b[rank + 1]))
    table = oracle.build_table(q, m, 11)
    part = oracle.scan(res, off, q, table, m, [(0, 16, 41)], threads=1)
    merged = shard.gather_to_rank0(part, rank, world)
    if rank == 0:
        np.savez(os.path.join(out_dir, "merged.npz"), c=merged[0], o=merged[1], h=merged[2])
    dist.barrier()
    dist.destroy_process_group()


def test_shard_bounds_balance_residues():
    rng = np.random.default_rng(0)
    lens = rng.integers(1, 1000, size=5000)
    off = np.concatenate([[0], np.cumsum(lens)])
    for world in (1, 2, 3, 8):
        b = shard.shard_bounds(off, world)
        assert b[0] == 0 and b[-1] == 5000 and np.all(np.diff(b) >= 0)
        share = np.diff(off[b]) / off[-1]
        assert np.all(np.abs(share - 1.0 / world) < 0.01)
    assert shard.shard_bounds(np.zeros(1, np.int64), 4).tolist() == [0, 0, 0, 0, 0]


def test_merge_concatenates_csr():
    a = (np.array([[1, 0, 1]]), np.array([5, 7]), np.arange(12).reshape(2, 6))
    b = (np.array([[0, 0, 0], [2, 1, 1]]), np.array([0, 0, 1]), np.arange(6).reshape(1, 6))
    c, o, h = shard.merge([a, b])
    assert c.tolist() == [[1, 0, 1], [0, 0, 0], [2, 1, 1]]
    assert o.tolist() == [0, 2, 2, 3]
    assert h.shape == (3, 6)


def test_two_ranks_gloo_equal_unsharded(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    z = np.load(tmp_path / "merged.npz")
    m = oracle.load_fixture_matrix()
    w = synth.shape1(m, n_subjects=1500, qlen=120)
    q = w.queries[0]
    c, o, h = oracle.scan(w.db.residues, w.db.offsets, q, oracle.build_table(q, m, 11), m, [(0, 16, 41)],
                          threads=1)
    assert np.array_equal(z["c"], c)
    assert np.array_equal(z["o"], o)
    assert np.array_equal(z["h"], h)
