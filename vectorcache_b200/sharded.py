"""Multi-GPU sharding of the flat index: one process per GPU, each holding a
contiguous shard of the vectors (ids offset by the shard base).

Vectors are encoded independently, so with one shared TQ+ calibration every
shard scores a query exactly as a single index over the union would. The only
exchange is one all-gather of the per-shard top-k lists (nq x k scores and ids
per rank, a few hundred KB), after which every rank merges them by score
descending, equal scores by lower id — the reference's merge order
(merge_search_results, src/search/search.cpp:1551-1600). The result is
identical to searching the union on one GPU.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def merge_topk(scores: torch.Tensor, ids: torch.Tensor, k: int) -> tuple[torch.Tensor, torch.Tensor]:
    """Best k of each row: score descending, equal scores by lower id.

    Two stable sorts: ids ascending first, then scores descending keeps the id
    order among equal scores.
    """
    order = torch.argsort(ids, dim=1, stable=True)
    s = torch.gather(scores, 1, order)
    i = torch.gather(ids, 1, order)
    order = torch.argsort(s, dim=1, descending=True, stable=True)
    s = torch.gather(s, 1, order)
    i = torch.gather(i, 1, order)
    return s[:, :k].contiguous(), i[:, :k].contiguous()


def allgather_merge(scores: torch.Tensor, ids: torch.Tensor, k: int, group=None):
    """All-gather the per-rank top-k (global ids) and merge them on every rank."""
    world = dist.get_world_size(group)
    if world == 1:
        return scores, ids
    gs = [torch.empty_like(scores) for _ in range(world)]
    gi = [torch.empty_like(ids) for _ in range(world)]
    dist.all_gather(gs, scores.contiguous(), group=group)
    dist.all_gather(gi, ids.contiguous(), group=group)
    return merge_topk(torch.cat(gs, dim=1), torch.cat(gi, dim=1), k)


def shard_bounds(n_total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous [begin, end) of the vectors rank `rank` holds."""
    per = (n_total + world - 1) // world
    b = min(n_total, rank * per)
    return b, min(n_total, b + per)


def _world(group) -> int:
    return dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1


class ShardedIndex:
    """One shard of a flat index spread over the ranks of a process group.

    Every rank calls the same methods in the same order (collective calls):
    `calibrate_shared` (one broadcast), `add*`, `prepare`, then any number of
    `search_device` calls (one all-gather each). `index` defaults to a
    TurboQuantIndex on `device`; any object with the same calibrate / add /
    prepare / search_device methods serves (the CPU tests pass one backed by
    the oracle).
    """

    def __init__(self, dim: int, bits: int, device: int, shard_base: int, group=None, index=None):
        if index is None:
            from . import TurboQuantIndex

            index = TurboQuantIndex(dim, bits, device=device)
        self.index = index
        self.dim = int(dim)
        self.base = int(shard_base)
        self.group = group

    def calibrate(self, sample) -> None:
        """Calibrate on host rows; the caller passes the same sample on every
        rank, so all shards share one TQ+ calibration."""
        self.index.calibrate(sample)

    def calibrate_shared(self, sample: torch.Tensor, src: int = 0) -> None:
        """Broadcast rank `src`'s sample rows (every rank passes a tensor of the
        same shape, dtype and device) and calibrate on them: one TQ+ shift /
        scale for every shard, so the shards score exactly like one index
        over their union."""
        if _world(self.group) > 1:
            dist.broadcast(sample, src, group=self.group)
        if sample.is_cuda:
            self.index.calibrate_device(sample)
        else:
            self.index.calibrate(sample.numpy())

    def add(self, vectors) -> None:
        self.index.add(vectors)

    def add_device(self, d_vectors) -> None:
        self.index.add_device(d_vectors)

    def prepare(self) -> None:
        self.index.prepare()

    def search_device(self, d_queries: torch.Tensor, k: int, out_scores=None, out_ids=None, stream=None):
        """This shard's top-k (ids offset by the shard base), all-gathered and
        merged: every rank returns the top-k of the union. With one rank the
        rows hold k_eff = min(k, n) entries; with several, k entries, ending
        in (-inf, 2^63 - 1) when the union holds fewer than k vectors."""
        nq = d_queries.shape[0]
        dev = d_queries.device
        s = out_scores if out_scores is not None else torch.empty((nq, k), dtype=torch.float32, device=dev)
        i = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int64, device=dev)
        ke = self.index.search_device(d_queries, k, s, i, stream=stream)
        if ke < k:  # rows were written with stride k_eff = min(k, shard size)
            s = s.reshape(-1)[: nq * ke].view(nq, ke)
            i = i.reshape(-1)[: nq * ke].view(nq, ke)
        i = i + self.base
        if _world(self.group) == 1:
            return s, i
        if ke < k:  # equal shapes on every rank for the all-gather
            pad_s = torch.full((nq, k - ke), float("-inf"), dtype=torch.float32, device=dev)
            pad_i = torch.full((nq, k - ke), torch.iinfo(torch.int64).max, dtype=torch.int64, device=dev)
            s, i = torch.cat([s, pad_s], 1), torch.cat([i, pad_i], 1)
        return allgather_merge(s, i, k, self.group)
