"""Database-sharded k = 2 search (cuda-orb_b200/sharded.py) without a GPU: the
merge of per-shard top-2 pairs, and the all-gather exchange on gloo with 2 and
3 ranks (127.0.0.1).  Each rank's local search is the CPU oracle on its shard,
in place of the GPU matcher; the merged result must equal the oracle over the
whole database bit for bit, including exact ties between rows of different
shards (the smaller global index wins) and empty shards."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import sharded
from oracle import oracle as O


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _data(n_db, n_q, seed):
    rng = np.random.Generator(np.random.PCG64(0x0C4400 + seed))
    db = rng.integers(0, 256, size=(n_db, 32), dtype=np.uint8)
    if n_db >= 8:
        # copies of early rows near the end: equal distances across shard boundaries
        db[-3:] = db[:3]
    q = rng.integers(0, 256, size=(n_q, 32), dtype=np.uint8)
    if n_db >= 8:
        q[:3] = db[:3]
        q[3:6] = db[:3] ^ np.uint8(1)
    return db, q


def test_shard_rows_cover_the_database():
    for n in (0, 1, 7, 65536, 1048577):
        for world in (1, 2, 3, 8):
            spans = [sharded.shard_rows(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1


def test_merge_knn2_orders_by_distance_then_index():
    # two shards, three queries
    d = torch.tensor([[[5, 9], [3, 3], [sharded.NO_DIST, sharded.NO_DIST]],
                      [[5, 6], [2, 7], [sharded.NO_DIST, sharded.NO_DIST]]])
    i = torch.tensor([[[10, 11], [0, 1], [-1, -1]],
                      [[4, 20], [30, 31], [-1, -1]]])
    md, mi = sharded.merge_knn2(d, i)
    # the types and sentinels of orbx.knn2: int32, missing distance 0xFFFFFFFF (-1 as int32)
    assert md.dtype == torch.int32 and mi.dtype == torch.int32
    assert md.tolist() == [[5, 5], [2, 3], [-1, -1]]
    assert mi.tolist() == [[4, 10], [30, 0], [-1, -1]]
    assert md.numpy().view(np.uint32)[2].tolist() == [sharded.NO_DIST, sharded.NO_DIST]


def test_merge_knn2_one_missing_second():
    # a query with one candidate in one shard and none in the other
    d = torch.tensor([[[7, -1]], [[-1, -1]]], dtype=torch.int32)
    i = torch.tensor([[[3, -1]], [[-1, -1]]], dtype=torch.int32)
    md, mi = sharded.merge_knn2(d, i)
    assert md.tolist() == [[7, -1]] and mi.tolist() == [[3, -1]]


def test_packed_key_is_16_bytes_per_query():
    keys = sharded.pack_keys(torch.zeros((10, 2), dtype=torch.int32), torch.zeros((10, 2), dtype=torch.int32))
    assert keys.dtype == torch.int64 and keys.numel() * keys.element_size() == 16 * 10


def _rank_main(rank, world, port, n_db, n_q, seed, out):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        db, q = _data(n_db, n_q, seed)
        b, e = sharded.shard_rows(n_db, world, rank)
        ld, li = O.knn2(q, db[b:e])
        gi = np.where(li >= 0, li.astype(np.int64) + b, -1)
        # the local search's own types: uint32 bits in int32 distances, int32 indices
        md, mi = sharded.gather_merge_knn2(torch.from_numpy(ld.view(np.int32)), torch.from_numpy(gi))
        assert md.dtype == torch.int32 and mi.dtype == torch.int32
        out[rank] = (md.numpy().view(np.uint32).tolist(), mi.numpy().tolist())
        dist.barrier()
    finally:
        dist.destroy_process_group()


# (2, 3, ...) and (3, 2, ...): fewer database rows than world_size x 2, so some
# queries have a missing second neighbour and some shards are empty
@pytest.mark.parametrize("world,n_db,n_q,seed", [(2, 1000, 64, 1), (3, 1001, 50, 2), (2, 1, 5, 3), (3, 2, 4, 4),
                                                 (2, 3, 6, 5)])
def test_sharded_knn2_gloo_equals_whole_database(world, n_db, n_q, seed):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_db, n_q, seed, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    db, q = _data(n_db, n_q, seed)
    ed, ei = O.knn2(q, db)
    for r in range(world):
        d, i = out[r]
        assert np.array_equal(np.array(d, dtype=np.uint32), ed), r
        assert np.array_equal(np.array(i, dtype=np.int32), ei), r
