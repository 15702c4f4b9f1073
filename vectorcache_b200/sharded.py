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


class ShardedIndex:
    """One shard of a flat index spread over the ranks of a process group.

    Every rank calls the same methods in the same order (collective calls).
    """

    def __init__(self, dim: int, bits: int, device: int, shard_base: int, group=None):
        from . import TurboQuantIndex

        self.index = TurboQuantIndex(dim, bits, device=device)
        self.base = int(shard_base)
        self.group = group
        self.device = torch.device("cuda", device)

    def calibrate(self, sample) -> None:
        """The same sample on every rank, so all shards share one calibration."""
        self.index.calibrate(sample)

    def add(self, vectors) -> None:
        self.index.add(vectors)

    def prepare(self) -> None:
        self.index.prepare()

    def search_device(self, d_queries: torch.Tensor, k: int, stream=None):
        nq = d_queries.shape[0]
        s = torch.empty((nq, k), dtype=torch.float32, device=self.device)
        i = torch.empty((nq, k), dtype=torch.int64, device=self.device)
        ke = self.index.search_device(d_queries, k, s, i, stream=stream)
        s, i = s[:, :ke], i[:, :ke] + self.base
        return allgather_merge(s, i, k, self.group)
