"""Several GPUs: pairs are independent, so a batch shards into contiguous pair ranges, one
per rank (one process per GPU), and the only exchange is the FP64 all-reduce of the summed
gradient (K*N*N + 4K doubles) -- no collective on the data path.

    rank_range = shard_pairs(off_a, off_b, world, rank)       # balanced by DP cells
    batch = SeqPairBatch.from_codes(... the rank's pairs ...)
    batch.score_and_grad()
    g = allreduce_grad(batch.compute_grad())                  # torch.distributed, any backend
"""
from __future__ import annotations

import numpy as np

from .params import AlignParams


def shard_pairs(off_a, off_b, world: int, rank: int) -> tuple[int, int]:
    """[start, end) of ``rank``'s contiguous pair range: the ranges split the batch's total
    DP cells (len(a) * len(b) summed) as evenly as contiguous cuts allow."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"nwgrad: bad rank {rank} of {world}")
    oa = np.asarray(off_a, np.int64)
    ob = np.asarray(off_b, np.int64)
    n = oa.size - 1
    cells = np.diff(oa).astype(np.float64) * np.diff(ob).astype(np.float64) + 1.0   # +1: empty pairs count
    cum = np.concatenate([[0.0], np.cumsum(cells)])
    total = cum[-1]
    cut = lambda r: int(np.searchsorted(cum, total * r / world, side="left")) if r < world else n  # noqa: E731
    lo, hi = cut(rank), cut(rank + 1)
    return min(lo, n), min(max(hi, lo), n)


def allreduce_grad(g: AlignParams, group=None, device=None) -> AlignParams:
    """The sum over ranks of a gradient (FP64, torch.distributed all-reduce on ``device``:
    a CUDA device for NCCL, the CPU for gloo)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return g
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
            else torch.device("cpu")
    K, N = g.num_sets, g.alphabet_obj.size
    flat = np.concatenate([np.ascontiguousarray(g.matrices).reshape(-1), np.ascontiguousarray(g.gaps).reshape(-1)])
    t = torch.from_numpy(flat).to(device)
    dist.all_reduce(t, group=group)
    v = t.cpu().numpy()
    return AlignParams._make(v[:K * N * N].reshape(K, N, N).copy(), v[K * N * N:].reshape(K, 4).copy(),
                             g.alphabet_obj)
