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
