"""Exact k = 2 Hamming search over a database sharded across GPUs, one process
per GPU (torch.distributed; NCCL on GPUs, gloo on CPU).

Each rank holds one contiguous block of database rows and searches it with the
library's exact matcher (orbx_match_knn2).  The ranks then exchange their
per-query top-2 (distance, global row index) pairs with one all-gather, 16
bytes per query per rank.  Every rank merges the world_size x 2 candidates of
each query into the global top-2 by (distance, index), the order the
single-GPU search uses, so the result equals orbx_match_knn2 over the whole
database bit for bit.  A row lives in exactly one shard, so no candidate is
counted twice.  Missing entries are (0xFFFFFFFF, -1), as in orbx_match_knn2.

This is the database-row sharding of the matching workloads (65536 x 65536
matching and the learned proposal's exact search).  The 1080p pair itself
runs as independent replicas and needs no exchange.
"""
import torch

NO_DIST = 0xFFFFFFFF
_NONE_KEY = 1 << 62


def shard_rows(n, world, rank):
    """Rows [begin, end) of an n-row database held by `rank` of `world`:
    contiguous blocks whose sizes differ by at most one."""
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def merge_knn2(dist, idx):
    """dist, idx: (W, nq, 2) integer tensors of per-shard top-2 pairs with
    global row indices (idx < 0: none).  Returns (dist2, idx2) of shape (nq, 2),
    int64, the two smallest (distance, index) pairs per query."""
    dist = dist.to(torch.int64)
    idx = idx.to(torch.int64)
    W, nq, _ = dist.shape
    key = torch.where(idx < 0, torch.full_like(dist, _NONE_KEY), (dist << 32) | idx)
    key = key.permute(1, 0, 2).reshape(nq, 2 * W)
    top = torch.topk(key, 2, dim=1, largest=False, sorted=True).values
    none = top >= _NONE_KEY
    d = torch.where(none, torch.full_like(top, NO_DIST), top >> 32)
    i = torch.where(none, torch.full_like(top, -1), top & 0xFFFFFFFF)
    return d, i


def gather_merge_knn2(dist_local, idx_global, group=None):
    """Collective: every rank passes its (nq, 2) local top-2 with global row
    indices (the same nq on every rank); every rank gets the merged (nq, 2)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    d = dist_local.to(torch.int64).contiguous()
    i = idx_global.to(torch.int64).contiguous()
    gd = [torch.empty_like(d) for _ in range(world)]
    gi = [torch.empty_like(i) for _ in range(world)]
    dist.all_gather(gd, d, group=group)
    dist.all_gather(gi, i, group=group)
    return merge_knn2(torch.stack(gd), torch.stack(gi))


def knn2_sharded(ctx, q, db_local, row_offset, mode=None, group=None):
    """k = 2 search of the uint8 (nq, 32) queries `q` against this rank's
    database block `db_local` (rows row_offset .. of the whole database), merged
    over all ranks.  q and db_local are CUDA tensors on this rank's GPU; every
    rank passes the same queries.  Returns (dist2, idx2) as int64 (nq, 2)."""
    import orbx

    d, i = orbx.knn2(ctx, q, db_local, orbx.MATCH_IMMA if mode is None else mode)
    ctx.sync()  # the exchange runs on torch's stream, the search on the context's
    gi = torch.where(i >= 0, i.to(torch.int64) + int(row_offset), torch.full_like(i, -1, dtype=torch.int64))
    return gather_merge_knn2(d, gi, group)
