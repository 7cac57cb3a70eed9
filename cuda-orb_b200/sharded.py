"""Exact k = 2 Hamming search over a database sharded across GPUs, one process
per GPU (torch.distributed; NCCL on GPUs, gloo on CPU).

Each rank holds one contiguous block of database rows and searches it with the
library's exact matcher (orbx_match_knn2).  Each rank packs its per-query
top-2 as two 64-bit keys, (distance << 32) | global row index, and the ranks
exchange them with one all-gather: 16 bytes per query per rank.  Every rank
keeps the two smallest of the world_size x 2 keys of each query, which is the
(distance, index) order the single-GPU search uses, so the result equals
orbx_match_knn2 over the whole database bit for bit.  A row lives in exactly
one shard, so no candidate is counted twice.  Results have the types and
sentinels of orbx.knn2: int32 distances (0xFFFFFFFF, i.e. -1, when missing)
and int32 indices (-1 when missing).

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


def pack_keys(dist, idx):
    """(..., 2) distances (any integer type; 0xFFFFFFFF or -1 when missing) and
    global indices (< 0 when missing) -> int64 keys (distance << 32) | index,
    with a key above every real one for a missing entry."""
    d = dist.to(torch.int64) & 0xFFFFFFFF
    i = idx.to(torch.int64)
    return torch.where(i < 0, torch.full_like(d, _NONE_KEY), (d << 32) | (i & 0xFFFFFFFF))


def merge_keys(keys):
    """keys: (W, nq, 2) int64 packed per-shard top-2.  Returns (dist2, idx2) of
    shape (nq, 2), int32, the two smallest (distance, index) pairs per query."""
    W, nq, _ = keys.shape
    k = keys.permute(1, 0, 2).reshape(nq, 2 * W)
    top = torch.topk(k, 2, dim=1, largest=False, sorted=True).values
    none = top >= _NONE_KEY
    d = torch.where(none, torch.full_like(top, -1), top >> 32).to(torch.int32)
    i = torch.where(none, torch.full_like(top, -1), top & 0xFFFFFFFF).to(torch.int32)
    return d, i


def merge_knn2(dist, idx):
    """dist, idx: (W, nq, 2) per-shard top-2 pairs with global row indices
    (idx < 0: none).  Returns the merged (dist2, idx2), int32, as merge_keys."""
    return merge_keys(pack_keys(dist, idx))


def gather_merge_knn2(dist_local, idx_global, group=None):
    """Collective: every rank passes its (nq, 2) local top-2 with global row
    indices (the same nq on every rank); every rank gets the merged (nq, 2).
    One all-gather of the packed keys, 16 bytes per query per rank."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    keys = pack_keys(dist_local, idx_global).contiguous()
    nq = keys.shape[0]
    out = torch.empty((world * nq, 2), dtype=torch.int64, device=keys.device)
    dist.all_gather_into_tensor(out, keys, group=group)
    return merge_keys(out.view(world, nq, 2))


def knn2_sharded(ctx, q, db_local, row_offset, mode=None, group=None):
    """k = 2 search of the uint8 (nq, 32) queries `q` against this rank's
    database block `db_local` (rows row_offset .. of the whole database), merged
    over all ranks.  q and db_local are CUDA tensors on this rank's GPU; every
    rank passes the same queries.  Returns (dist2, idx2) as int32 (nq, 2), the
    types of orbx.knn2."""
    import orbx

    d, i = orbx.knn2(ctx, q, db_local, orbx.MATCH_IMMA if mode is None else mode)
    ctx.sync()  # the exchange runs on torch's stream, the search on the context's
    gi = torch.where(i >= 0, i.to(torch.int64) + int(row_offset), torch.full_like(i, -1, dtype=torch.int64))
    return gather_merge_knn2(d, gi, group)
