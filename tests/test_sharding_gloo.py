"""Host logic of the multi-GPU path on CPU: two gloo ranks each search their
contiguous shard (scored by the CPU oracle, standing in for a device shard),
all-gather the per-shard top-k and merge. The merged result must equal one
search over the union, ids and scores, including tie order."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from vectorcache_b200.sharded import merge_topk, shard_bounds


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, db, q, calib, bits, k, out):
    import torch.distributed as dist

    from oracle.oracle import Oracle
    from vectorcache_b200.sharded import allgather_merge

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        orc = Oracle()
        shift, scale = orc.fit_calibration(calib, bits)  # same sample on every rank
        b, e = shard_bounds(db.shape[0], world, rank)
        packed, alpha = orc.encode(db[b:e], bits, shift, scale)
        s, i = orc.search_flat(q, bits, packed, alpha, k, shift, scale)
        s = torch.from_numpy(s)
        i = torch.from_numpy(i.astype(np.int64)) + b
        ms, mi = allgather_merge(s, i, k)
        if rank == 0:
            out["scores"] = ms.numpy()
            out["ids"] = mi.numpy()
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_equal_one_index(oracle):
    from vectorcache_b200.synthetic import power_law

    dim, bits, n, nq, k = 128, 4, 3001, 9, 12
    db = power_law(n, dim, seed=3)
    db[2000] = db[17]  # duplicate vector across the shard boundary: equal scores, id order decides
    q = power_law(nq, dim, seed=4)
    calib = db[:500]
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank_main, args=(2, _free_port(), db, q, calib, bits, k, out), nprocs=2,
                       join=True, start_method="spawn")
    shift, scale = oracle.fit_calibration(calib, bits)
    packed, alpha = oracle.encode(db, bits, shift, scale)
    want_s, want_i = oracle.search_flat(q, bits, packed, alpha, k, shift, scale)
    assert np.array_equal(out["ids"], want_i.astype(np.int64))
    assert np.array_equal(out["scores"].view(np.uint32), want_s.view(np.uint32))


class OracleShardIndex:
    """The CPU oracle behind the TurboQuantIndex methods ShardedIndex calls
    (calibrate / add / prepare / search_device), standing in for a device
    shard on CPU."""

    def __init__(self, bits):
        from oracle.oracle import Oracle

        self.orc = Oracle()
        self.bits = bits
        self.shift = self.scale = None
        self.rows = []

    def calibrate(self, sample):
        self.shift, self.scale = self.orc.fit_calibration(np.asarray(sample, np.float32), self.bits)

    def add(self, vectors):
        self.rows.append(np.asarray(vectors, np.float32))

    def prepare(self):
        x = np.concatenate(self.rows)
        self.packed, self.alpha = self.orc.encode(x, self.bits, self.shift, self.scale)

    def search_device(self, q, k, out_s, out_i, stream=None):
        s, i = self.orc.search_flat(q.numpy(), self.bits, self.packed, self.alpha, k, self.shift, self.scale)
        ke = s.shape[1]
        out_s.view(-1)[: s.size] = torch.from_numpy(s.reshape(-1))
        out_i.view(-1)[: i.size] = torch.from_numpy(i.reshape(-1).astype(np.int64))
        return ke


def _bench_path_rank(rank, world, port, shards, q, n_calib, bits, k, out):
    """The benchmark's multi-GPU path: rank 0's first rows broadcast as the one
    calibration sample, each rank's own shard, ids offset by rank * shard
    size, one all-gather merge."""
    import torch.distributed as dist

    from vectorcache_b200.sharded import ShardedIndex

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        db = shards[rank]
        shard = ShardedIndex(db.shape[1], bits, device=0, shard_base=rank * shards[0].shape[0],
                             index=OracleShardIndex(bits))
        sample = torch.from_numpy(db[:n_calib].copy()) if rank == 0 else torch.zeros((n_calib, db.shape[1]))
        shard.calibrate_shared(sample)
        shard.add(db)
        shard.prepare()
        ms, mi = shard.search_device(torch.from_numpy(q), k)
        out[f"scores{rank}"] = ms.numpy()
        out[f"ids{rank}"] = mi.numpy()
    finally:
        dist.destroy_process_group()


def test_bench_sharded_path_equals_one_index(oracle):
    """Two ranks with different shards (different seeds, as the benchmark
    generates them) and one broadcast calibration: both ranks return the top-k
    of one index over the union, calibrated on rank 0's first rows."""
    from vectorcache_b200.synthetic import power_law

    dim, bits, n, nq, k, n_calib = 128, 4, 2000, 7, 10, 400
    shards = [power_law(n, dim, seed=1000 + r) for r in range(2)]
    shards[1][5] = shards[0][11]  # equal scores across the shards: the lower id wins
    q = power_law(nq, dim, seed=7)
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_bench_path_rank, args=(2, _free_port(), shards, q, n_calib, bits, k, out), nprocs=2,
                       join=True, start_method="spawn")
    union = np.concatenate(shards)
    shift, scale = oracle.fit_calibration(shards[0][:n_calib], bits)
    packed, alpha = oracle.encode(union, bits, shift, scale)
    want_s, want_i = oracle.search_flat(q, bits, packed, alpha, k, shift, scale)
    for r in range(2):
        assert np.array_equal(out[f"ids{r}"], want_i.astype(np.int64))
        assert np.array_equal(out[f"scores{r}"].view(np.uint32), want_s.view(np.uint32))


def test_merge_topk_order():
    s = torch.tensor([[1.0, 3.0, 3.0, 2.0, 3.0]])
    i = torch.tensor([[9, 7, 2, 5, 4]])
    ms, mi = merge_topk(s, i, 4)
    assert mi.tolist() == [[2, 4, 7, 5]]
    assert ms.tolist() == [[3.0, 3.0, 3.0, 2.0]]


def test_shard_bounds_cover():
    for n in (1, 7, 1000, 1001):
        for w in (1, 2, 3, 8):
            parts = [shard_bounds(n, w, r) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
