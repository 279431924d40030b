"""Multi-GPU plumbing of the mapping path (one process per GPU).

The path shards two ways (no exchange on the data path for the first):
  * by reads: every rank maps its own read batch against a replica of the
    index -- weak scaling; only timings are reduced (max over ranks);
  * by index columns: rank r holds columns [lo_r, hi_r); each rank computes
    its local top-k, and one all-gather of G x k (value, column) candidates
    per read followed by a merge gives the global top-k.  The merge order is
    the engine's total order (value descending, ties by ascending global
    column), so the sharded result equals the single-GPU result exactly.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def max_over_ranks(values, group=None, device=None):
    """Element-wise max of a list of floats across ranks (timings)."""
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(x) for x in t.tolist()]


def shard_bounds(N: int, world: int, rank: int):
    """Contiguous column range [lo, hi) of `rank` (balanced to within one)."""
    q, r = divmod(N, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def merge_topk(vals: torch.Tensor, locs: torch.Tensor, k: int):
    """Merge candidate lists (nb, C) -> top-k (nb, k): value descending, ties
    by ascending 1-based column; empty slots (loc 0, -inf) sort last."""
    key_loc = torch.where(locs > 0, locs.to(torch.int64), torch.full_like(locs, 2 ** 62, dtype=torch.int64))
    # stable two-key sort: first by column, then (stable) by value descending
    o1 = torch.argsort(key_loc, dim=1, stable=True)
    v1 = torch.gather(vals, 1, o1)
    o2 = torch.argsort(-v1, dim=1, stable=True)
    order = torch.gather(o1, 1, o2)[:, :k]
    return torch.gather(vals, 1, order), torch.gather(locs, 1, order)


def merge_topk_lists(vals: torch.Tensor, locs: torch.Tensor, lists: int, k: int, stream=None):
    """merge_topk of `lists` sorted k-lists per row laid side by side, on the
    GPU with the library's merge kernel (r2m_merge_topk_lists)."""
    from ._lib import check, lib, ptr, stream_handle
    nb = vals.shape[0]
    vals = vals.contiguous()
    locs = locs.to(torch.int32).contiguous()
    ov = torch.empty((nb, k), dtype=torch.float32, device=vals.device)
    ol = torch.empty((nb, k), dtype=torch.int32, device=vals.device)
    check(lib().r2m_merge_topk_lists(ptr(vals), ptr(locs), lists, nb, vals.shape[1] // lists, k, ptr(ov), ptr(ol),
                                     stream_handle(stream)))
    return ov, ol


def scale_rows(vals: torch.Tensor, scaleA: torch.Tensor) -> torch.Tensor:
    """Apply per-row scales after a merge (empty slots stay -inf).  Scaled
    scores rank by the value before the row scale -- a shared positive
    factor can round two different values to one -- so a sharded search runs
    its shards with a unit row scale, merges, then scales once; the result
    equals the single-engine search bit for bit."""
    return torch.where(torch.isneginf(vals), vals, vals * scaleA[:, None])


def gather_shard_topk(vals: torch.Tensor, locs: torch.Tensor, col_lo: int, k: int, group=None):
    """All-gather every rank's local top-k (local 1-based ids shifted by its
    shard offset) and merge them into the global top-k on every rank: on
    CUDA tensors with the library's merge kernel, otherwise with torch."""
    g = torch.where(locs > 0, locs + col_lo, locs)
    world = dist.get_world_size(group)
    vs = [torch.empty_like(vals) for _ in range(world)]
    ls = [torch.empty_like(g) for _ in range(world)]
    dist.all_gather(vs, vals.contiguous(), group=group)
    dist.all_gather(ls, g.contiguous(), group=group)
    cat_v, cat_l = torch.cat(vs, dim=1), torch.cat(ls, dim=1)
    if cat_v.is_cuda and world <= 32:
        return merge_topk_lists(cat_v, cat_l, world, k)
    return merge_topk(cat_v, cat_l, k)
