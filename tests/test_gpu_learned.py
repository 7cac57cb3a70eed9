"""The learned matching proposal (orbx_learned_*, orbx_gemm_bf16) on the GPU:
the tcgen05 BF16 GEMM against a PyTorch fp32 reference, the MLP gradients
against the CPU FP64 oracle (oracle/mlp_oracle.py), k-majority clustering
layout, search exactness (all-fallback search equals exact brute force,
probed results are consistent Hamming distances), recall, and the LSH
ablation on clustered descriptors."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import orbx  # noqa: E402
from oracle import mlp_oracle as MO  # noqa: E402


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = orbx.Context(0)
    yield c
    c.close()


def clustered(n_db, n_q, n_centers=512, p_db=0.12, p_q=0.04, seed=0):
    """Database rows = random centers with bits flipped at p_db; queries = random
    database rows with bits flipped at p_q."""
    rng = np.random.Generator(np.random.PCG64(0x0C4100 + seed))
    centers = rng.integers(0, 2, size=(n_centers, 256), dtype=np.uint8)
    cid = rng.integers(0, n_centers, size=n_db)
    bits = centers[cid] ^ (rng.uniform(size=(n_db, 256)) < p_db).astype(np.uint8)
    src = rng.integers(0, n_db, size=n_q)
    qbits = bits[src] ^ (rng.uniform(size=(n_q, 256)) < p_q).astype(np.uint8)
    return np.packbits(bits, axis=1), np.packbits(qbits, axis=1)


def bf16_tensor(shape, gen, scale=1.0):
    return (torch.randn(shape, generator=gen) * scale).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 512, 320), (512, 4096, 512)])
def test_gemm_f32_vs_torch(ctx, M, N, K):
    g = torch.Generator().manual_seed(M + N + K)
    a, b = bf16_tensor((M, K), g), bf16_tensor((N, K), g)
    bias = torch.randn(N, generator=g).cuda()
    ref = a.float() @ b.float().T + bias
    out = orbx.gemm_bf16(ctx, a, b, orbx.GEMM_F32, bias=bias)
    ctx.sync()
    # fp32 accumulation of exact bf16 products: only the summation order differs
    assert torch.allclose(out, ref, rtol=1e-5, atol=1e-4 * K ** 0.5)


def test_gemm_split_k(ctx):
    g = torch.Generator().manual_seed(7)
    a, b = bf16_tensor((256, 1024), g), bf16_tensor((512, 1024), g)
    out = orbx.gemm_bf16(ctx, a, b, orbx.GEMM_F32, splits=4)
    ctx.sync()
    ref = a.float() @ b.float().T
    assert out.shape == (4, 256, 512)
    assert torch.allclose(out.sum(0), ref, rtol=1e-5, atol=1e-2)
    # each split is the product over its quarter of K
    q = 1024 // 4
    for s in range(4):
        part = a[:, s * q:(s + 1) * q].float() @ b[:, s * q:(s + 1) * q].float().T
        assert torch.allclose(out[s], part, rtol=1e-5, atol=5e-3)


def test_gemm_bf16_epilogues(ctx):
    g = torch.Generator().manual_seed(11)
    M, N, K = 256, 512, 256
    a, b = bf16_tensor((M, K), g), bf16_tensor((N, K), g)
    bias = torch.randn(N, generator=g).cuda()
    ref = a.float() @ b.float().T
    relu = orbx.gemm_bf16(ctx, a, b, orbx.GEMM_BIAS_RELU_BF16, bias=bias)
    plain = orbx.gemm_bf16(ctx, a, b, orbx.GEMM_BF16, bias=bias)
    aux = bf16_tensor((M, N), g)
    aux[:, ::7] = 0
    masked = orbx.gemm_bf16(ctx, a, b, orbx.GEMM_MASK_BF16, aux=aux)
    ctx.sync()
    tol = dict(rtol=2 ** -7, atol=1e-3)
    assert torch.allclose(relu.float(), torch.relu(ref + bias), **tol)
    assert torch.allclose(plain.float(), ref + bias, **tol)
    assert torch.allclose(masked.float(), ref * (aux.float() > 0), **tol)
    assert bool((masked[:, ::7] == 0).all())


def test_gemm_top8(ctx):
    g = torch.Generator().manual_seed(13)
    M, N, K = 256, 1024, 512
    a, b = bf16_tensor((M, K), g), bf16_tensor((N, K), g)
    bias = torch.randn(N, generator=g).cuda()
    keys = orbx.gemm_bf16(ctx, a, b, orbx.GEMM_TOP8, bias=bias)
    ctx.sync()
    ref = (a.float() @ b.float().T + bias).cpu().numpy()
    k = keys.cpu().numpy().astype(np.uint32)  # (M, N / 128, 8)
    cols = 4095 - (k & 0xFFF).astype(np.int64)
    for t in range(N // 128):
        tile = ref[:, t * 128:(t + 1) * 128]
        kth = np.sort(tile, axis=1)[:, -8]
        got = np.take_along_axis(ref, cols[:, t, :], axis=1)
        assert np.all((cols[:, t, :] >= t * 128) & (cols[:, t, :] < (t + 1) * 128))
        # every returned column is at least the tile's 8th largest (keys keep ~2^-11 of the logit)
        assert np.all(got >= kth[:, None] - 1e-3 * np.abs(kth[:, None]) - 1e-3)
        # descending, distinct
        assert np.all(np.diff(k[:, t, :].astype(np.int64), axis=1) < 0)


def _top8_row_sets(N):
    """Column sets of GEMM_TOP8_ROW's lists for N columns."""
    tiles = N // 256
    parts = 2 if tiles % 2 == 0 else 1
    tpi = tiles // parts
    return [np.concatenate([np.arange(256 * t + 128 * h, 256 * t + 128 * h + 128) for t in range(p * tpi, (p + 1) * tpi)])
            for p in range(parts) for h in range(2)]


@pytest.mark.parametrize("N", [1024, 768, 4096])
def test_gemm_top8_row(ctx, N):
    g = torch.Generator().manual_seed(17)
    M, K = 384, 512
    a, b = bf16_tensor((M, K), g), bf16_tensor((N, K), g)
    bias = torch.randn(N, generator=g).cuda()
    keys = orbx.gemm_bf16(ctx, a, b, orbx.GEMM_TOP8_ROW, bias=bias)
    ctx.sync()
    ref = (a.float() @ b.float().T + bias).cpu().numpy()
    k = keys.cpu().numpy().astype(np.uint32)  # (M, lists, 8)
    sets = _top8_row_sets(N)
    assert k.shape == (M, len(sets), 8) == (M, orbx.gemm_top_lists(N), 8)
    cols = 4095 - (k & 0xFFF).astype(np.int64)
    for l, cs in enumerate(sets):
        assert np.all(np.isin(cols[:, l, :], cs))
        kth = np.sort(ref[:, cs], axis=1)[:, -8]
        got = np.take_along_axis(ref, cols[:, l, :], axis=1)
        assert np.all(got >= kth[:, None] - 1e-3 * np.abs(kth[:, None]) - 1e-3)
        assert np.all(np.diff(k[:, l, :].astype(np.int64), axis=1) < 0)
    # the best 8 keys over all lists are the row's 8 largest logits
    allk = np.sort(k.reshape(M, -1).astype(np.int64), axis=1)[:, ::-1][:, :8]
    top_cols = 4095 - (allk & 0xFFF)
    kth = np.sort(ref, axis=1)[:, -8]
    assert np.all(np.take_along_axis(ref, top_cols, axis=1) >= kth[:, None] - 1e-3 * np.abs(kth[:, None]) - 1e-3)


@pytest.fixture(scope="module")
def small_index(ctx):
    db, q = clustered(16384, 4096, seed=1)
    train = clustered(16384, 8192, seed=1)[1][4096:]  # other noisy copies of the same database
    p = orbx.learned_params(n_clusters=256, hidden=512, epochs=10, batch=512, kmeans_iters=12, lr=1e-3)
    tdb, tq, ttr = (torch.from_numpy(x).cuda() for x in (db, q, train))
    idx = orbx.LearnedIndex(ctx, tdb, ttr, p)
    yield idx, db, q, tdb, tq
    idx.close()


def test_kmeans_layout(small_index):
    idx, db, *_ = small_index
    ex = idx.export(weights=False)
    # spill 2: every row is listed in its nearest and its second-nearest cluster
    counts = np.diff(ex["offsets"])
    assert ex["offsets"][0] == 0 and ex["offsets"][-1] == 2 * len(db)
    assert np.all(counts >= np.bincount(ex["assign"], minlength=256))
    st = idx.stats()
    assert st["kmeans_iters"] >= 1 and st["largest_cluster"] == counts.max()


def test_training_reduces_loss(small_index):
    st = small_index[0].stats()
    assert st["epochs"] == 10
    assert st["loss"][-1] < st["loss"][0]
    assert st["accuracy"][-1] > 0.5


def test_gradients_vs_fp64_oracle(ctx, small_index):
    idx, db, q, tdb, tq = small_index
    rng = np.random.Generator(np.random.PCG64(0x0C4200))
    n = 256
    x = q[:n]
    labels = rng.integers(0, 256, size=n).astype(np.int32)
    loss, g = idx.gradients(tq[:n].contiguous(), torch.from_numpy(labels).cuda())
    w = idx.export()
    ref_loss, ref = MO.forward_backward(x, labels, w["w1"], w["b1"], w["w2"], w["b2"], bf16=False)
    _, ref16 = MO.forward_backward(x, labels, w["w1"], w["b1"], w["w2"], w["b2"], bf16=True)
    assert abs(loss - ref_loss) < 1e-3 * max(1.0, abs(ref_loss))
    for k in ("w1", "b1", "w2", "b2"):
        err = np.linalg.norm(g[k] - ref[k]) / np.linalg.norm(ref[k])
        err16 = np.linalg.norm(g[k] - ref16[k]) / np.linalg.norm(ref16[k])
        assert err < 2e-2, (k, err)      # against exact FP64 arithmetic
        assert err16 < 5e-3, (k, err16)  # against FP64 with the GPU's bf16 roundings


def test_search_all_fallback_is_exact(ctx, small_index):
    idx, db, q, tdb, tq = small_index
    idx.set_margin(3.0e38)
    try:
        d, i, m, fb = idx.search(tq)
        ed, ei = orbx.knn2(ctx, tq, tdb, orbx.MATCH_IMMA)
        ctx.sync()
        assert int(fb.item()) == len(q)
        assert torch.equal(d, ed) and torch.equal(i, ei)
    finally:
        idx.set_margin(0.0)


def _check_consistent(q, db, d, i):
    d, i = d.cpu().numpy(), i.cpu().numpy()
    ok = i[:, 0] >= 0
    qb = np.unpackbits(q[ok], axis=1)
    rb = np.unpackbits(db[i[ok, 0]], axis=1)
    assert np.array_equal((qb != rb).sum(1), d[ok, 0])
    return d, i


def test_search_recall_and_margin(ctx, small_index):
    idx, db, q, tdb, tq = small_index
    d, i, m, fb = idx.search(tq)
    ctx.sync()
    assert int(fb.item()) == 0  # margin 0 never falls back
    d, i = _check_consistent(q, db, d, i)
    ed, ei = MO.knn1_bruteforce(q, db)
    assert np.all(d[:, 0] >= ed)
    recall = float(np.mean(d[:, 0] == ed))
    assert recall > 0.9, recall
    # queries below a margin threshold go to exact search: recall can only rise
    mm = m.cpu().numpy()
    thr = float(np.quantile(mm, 0.2))
    idx.set_margin(thr)
    try:
        d2, i2, _, fb2 = idx.search(tq)
        ctx.sync()
        n_fb = int(fb2.item())
        assert n_fb == int(np.sum(mm < thr))
        d2, _ = _check_consistent(q, db, d2, i2)
        assert np.all(d2[:, 0] >= ed)
        assert np.all(d2[mm < thr, 0] == ed[mm < thr])
        assert float(np.mean(d2[:, 0] == ed)) >= recall
    finally:
        idx.set_margin(0.0)


def test_lsh_ablation(ctx, small_index):
    idx, db, q, tdb, tq = small_index
    d, i, _, _ = idx.search(tq)
    p = orbx.learned_params(proposal=orbx.PROPOSAL_LSH, lsh_bits=8, n_clusters=256)
    lsh = orbx.LearnedIndex(ctx, tdb, None, p)
    try:
        ld, li, _, lfb = lsh.search(tq)
        ctx.sync()
        assert int(lfb.item()) == 0
        ld, _ = _check_consistent(q, db, ld, li)
        ed, _ = MO.knn1_bruteforce(q, db)
        r_mlp = float(np.mean(d.cpu().numpy()[:, 0] == ed))
        r_lsh = float(np.mean(ld[:, 0] == ed))
        assert r_mlp > r_lsh, (r_mlp, r_lsh)
    finally:
        lsh.close()


def test_centroid_init_is_nearest_centroid(ctx):
    """With no training, the centroid-initialised MLP scores clusters by their
    Hamming distance: logit_c = 0.25 * (256 - 2 * Hamming(x, centroid_c))."""
    db, q = clustered(8192, 512, n_centers=64, seed=3)
    p = orbx.learned_params(n_clusters=256, hidden=512, epochs=0, batch=128, kmeans_iters=8, spill=1)
    tdb, tq = torch.from_numpy(db).cuda(), torch.from_numpy(q).cuda()
    idx = orbx.LearnedIndex(ctx, tdb, tq[:128].contiguous(), p)
    try:
        w = idx.export()
        x = MO.pm1(q)
        logits = np.maximum(x @ w["w1"].T.astype(np.float64) + w["b1"], 0) @ w["w2"].T.astype(np.float64) + w["b2"]
        # recover the centroid signs from W2 and compare with the scores
        s = np.sign(w["w2"][:, :256])
        assert np.all(np.abs(w["w2"][:, :256]) == 0.25) and np.array_equal(w["w2"][:, 256:512], -w["w2"][:, :256])
        ham = (256 - x @ s.T) / 2
        assert np.allclose(logits, 0.25 * (256 - 2 * ham))
        ex = idx.export(weights=False)
        assert ex["offsets"][-1] == len(db)  # spill 1: each row once
    finally:
        idx.close()


def test_spill_and_synthetic_rows_and_distance_rule(ctx):
    db, q = clustered(16384, 2048, seed=4)
    tdb, tq = torch.from_numpy(db).cuda(), torch.from_numpy(q).cuda()
    ed, _ = MO.knn1_bruteforce(q, db)
    rec = {}
    for spill in (1, 2):
        p = orbx.learned_params(n_clusters=256, hidden=512, epochs=2, batch=512, kmeans_iters=8, spill=spill,
                                synth_train=4096, flip_lo=0.02, flip_hi=0.08)
        idx = orbx.LearnedIndex(ctx, tdb, tq[:512].contiguous(), p)
        try:
            d, i, m, fb = idx.search(tq)
            ctx.sync()
            d, i = _check_consistent(q, db, d, i)
            rec[spill] = float(np.mean(d[:, 0] == ed))
            # no duplicate row in the k = 2 result even when a row is listed twice
            assert np.all((i[:, 0] != i[:, 1]) | (i[:, 0] < 0))
            if spill == 2:
                thr = int(np.quantile(d[:, 0], 0.7))
                idx.set_max_distance(thr)
                d2, i2, _, fb2 = idx.search(tq)
                ctx.sync()
                d2, _ = _check_consistent(q, db, d2, i2)
                far = d[:, 0] > thr
                assert int(fb2.item()) == int(far.sum())
                assert np.array_equal(d2[far, 0], ed[far])
                assert np.array_equal(d2[~far, 0], d[~far, 0])
        finally:
            idx.close()
    assert rec[2] >= rec[1], rec


# ---------------------------------------------------------------- checkpoints
CKPT_HEAD = 16 + 4 * (20 + 136)  # magic, version, size; 20 parameter words; the statistics words


def _ckpt_centroids(blob, C):
    return np.frombuffer(blob, dtype=np.uint8, count=C * 32, offset=CKPT_HEAD).reshape(C, 32)


def _hamming(a, b):
    ab = np.unpackbits(a, axis=1).astype(np.int32)
    bb = np.unpackbits(b, axis=1).astype(np.int32)
    return ab.sum(1)[:, None] + bb.sum(1)[None, :] - 2 * (ab @ bb.T)


def _same_search(ctx, a, b, tq):
    ra, rb = a.search(tq), b.search(tq)
    ctx.sync()
    for x, y in zip(ra, rb):
        assert torch.equal(x, y)


def test_checkpoint_round_trip(ctx, small_index):
    """save -> load over the same database: identical lists, weights and search."""
    idx, db, q, tdb, tq = small_index
    blob = idx.save()
    p = orbx.LearnedParams.from_buffer_copy(idx.params)
    assert len(blob) == CKPT_HEAD + 256 * 32 + 512 * 256 * 2 + 512 * 4 + 256 * 512 * 2 + 256 * 4 + 8
    re = orbx.LearnedIndex.load(ctx, blob, tdb)
    try:
        for f in ("proposal", "n_clusters", "hidden", "n_probe", "spill", "seed", "max_distance", "lr", "margin",
                  "rerank", "label_mode"):
            assert getattr(re.params, f) == getattr(p, f), f
        st, rst = idx.stats(), re.stats()
        assert rst["loss"] == st["loss"] and rst["largest_cluster"] == st["largest_cluster"]
        a, b = idx.export(), re.export()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        _same_search(ctx, idx, re, tq)
        # with a margin threshold part of the queries go to exact search in both
        for m in (1.0, 3.0e38):
            idx.set_margin(m)
            re.set_margin(m)
            _same_search(ctx, idx, re, tq)
        # saving the loaded index gives the same checkpoint apart from its build times
        re.set_margin(p.margin)
        blob2 = re.save()
        bt = 16 + 4 * (20 + 4 + 64 + 64)
        assert len(blob2) == len(blob) and blob2[:bt] == blob[:bt] and blob2[bt + 16:-8] == blob[bt + 16:-8]
    finally:
        idx.set_margin(0.0)
        re.close()


def test_checkpoint_over_new_database(ctx, small_index):
    """load over another database lists each row under its two nearest saved
    centroids (exact Hamming, ties to the smaller index) and searches it."""
    idx, *_ = small_index
    blob = idx.save()
    cent = _ckpt_centroids(blob, 256)
    db2, q2 = clustered(12000, 2048, seed=7)
    tdb2, tq2 = torch.from_numpy(db2).cuda(), torch.from_numpy(q2).cuda()
    re = orbx.LearnedIndex.load(ctx, blob, tdb2)
    try:
        ex = re.export(weights=False)
        d = _hamming(db2, cent).astype(np.int64)
        order = np.argsort(d * 256 + np.arange(256)[None, :], axis=1)
        assert np.array_equal(ex["assign"], order[:, 0])
        counts = np.bincount(order[:, 0], minlength=256) + np.bincount(order[:, 1], minlength=256)
        assert np.array_equal(np.diff(ex["offsets"]), counts)
        assert re.stats()["largest_cluster"] == counts.max()
        dd, ii, _, fb = re.search(tq2)
        ctx.sync()
        assert int(fb.item()) == 0
        _check_consistent(q2, db2, dd, ii)
        re.set_margin(3.0e38)
        dd, ii, _, fb = re.search(tq2)
        ed, ei = orbx.knn2(ctx, tq2, tdb2, orbx.MATCH_IMMA)
        ctx.sync()
        assert int(fb.item()) == len(q2) and torch.equal(dd, ed) and torch.equal(ii, ei)
    finally:
        re.close()


def test_checkpoint_lsh(ctx, small_index):
    _, db, q, tdb, tq = small_index
    p = orbx.learned_params(proposal=orbx.PROPOSAL_LSH, lsh_bits=8, n_clusters=256)
    lsh = orbx.LearnedIndex(ctx, tdb, None, p)
    try:
        blob = lsh.save()
        assert len(blob) == CKPT_HEAD + 256 * 256 * 2 + 8
        re = orbx.LearnedIndex.load(ctx, blob, tdb)
        try:
            a, b = lsh.export(), re.export()
            assert np.array_equal(a["assign"], b["assign"]) and np.array_equal(a["offsets"], b["offsets"])
            _same_search(ctx, lsh, re, tq)
        finally:
            re.close()
    finally:
        lsh.close()


def test_checkpoint_rejects_damaged_bytes(ctx, small_index):
    idx, db, q, tdb, tq = small_index
    blob = bytearray(idx.save())
    cases = {"truncated": bytes(blob[:-1]), "empty": b"\0" * 8}
    for name, off in (("magic", 0), ("version", 8), ("size", 12), ("params", 20), ("weights", CKPT_HEAD + 9000),
                      ("hash", len(blob) - 1)):
        bad = bytearray(blob)
        bad[off] ^= 0x10
        cases[name] = bytes(bad)
    for name, bad in cases.items():
        with pytest.raises(orbx.OrbxError) as e:
            orbx.LearnedIndex.load(ctx, bad, tdb)
        assert e.value.status == orbx.ORBX_ERR_ARG, name
    with pytest.raises(orbx.OrbxError):
        orbx.LearnedIndex.load(ctx, bytes(blob), tdb[:0])


# ---------------------------------------------------------------- rerank forms
def _both_forms(ctx, idx, tq):
    out = {}
    for form in (orbx.RERANK_TENSOR, orbx.RERANK_POPC):
        idx.set_rerank(form)
        out[form] = idx.search(tq)
        ctx.sync()
    idx.set_rerank(orbx.RERANK_TENSOR)
    return out[orbx.RERANK_TENSOR], out[orbx.RERANK_POPC]


def test_rerank_forms_agree(ctx, small_index):
    """The int8 tensor-core rerank and the XOR-popc rerank give the same top-2
    (distance, index) for every query, at margin 0 and with part of the queries
    sent to exact search."""
    idx, db, q, tdb, tq = small_index
    for m in (0.0, 1.0):
        idx.set_margin(m)
        try:
            t, p = _both_forms(ctx, idx, tq)
        finally:
            idx.set_margin(0.0)
        for x, y in zip(t, p):
            assert torch.equal(x, y)
    d, i = _check_consistent(q, db, t[0], t[1])
    # the second neighbour is a consistent distance too, ordered after the first
    ok = i[:, 1] >= 0
    qb = np.unpackbits(q[ok], axis=1)
    rb = np.unpackbits(db[i[ok, 1]], axis=1)
    assert np.array_equal((qb != rb).sum(1), d[ok, 1])
    assert np.all((d[ok, 1] > d[ok, 0]) | ((d[ok, 1] == d[ok, 0]) & (i[ok, 1] > i[ok, 0])))


def test_rerank_forms_ties_and_ragged_clusters(ctx):
    """Many exact ties (rows duplicated in the database), clusters of every size
    from empty to several 256-row tiles, queries that probe one cluster many
    times over: both forms agree, and they find the exact nearest row whenever
    it is listed in a probed cluster."""
    rng = np.random.Generator(np.random.PCG64(0x0C4300))
    base, _ = clustered(6000, 1, n_centers=96, p_db=0.1, seed=9)
    # near-copies of one row make a cluster of several tiles; exact duplicates give equal distances
    hub = np.unpackbits(np.repeat(base[:1], 1500, axis=0), axis=1) ^ (rng.uniform(size=(1500, 256)) < 0.005)
    db = np.concatenate([base, np.packbits(hub.astype(np.uint8), axis=1), base[rng.integers(0, len(base), 1500)]])
    db = db[rng.permutation(len(db))]
    q = db[rng.integers(0, len(db), 3000)].copy()
    flips = (rng.uniform(size=(len(q), 256)) < 0.03).astype(np.uint8)
    q = np.packbits(np.unpackbits(q, axis=1) ^ flips, axis=1)
    q = np.concatenate([q, q[:5]])  # a ragged query count
    tdb, tq = torch.from_numpy(db).cuda(), torch.from_numpy(q).cuda()
    for spill in (1, 2):
        p = orbx.learned_params(n_clusters=256, hidden=512, epochs=1, batch=512, kmeans_iters=6, spill=spill)
        idx = orbx.LearnedIndex(ctx, tdb, tq[:512].contiguous(), p)
        try:
            sizes = np.diff(idx.export(weights=False)["offsets"])
            assert sizes.min() < 64 and sizes.max() > 512, (sizes.min(), sizes.max())
            t, pp = _both_forms(ctx, idx, tq)
            for x, y in zip(t, pp):
                assert torch.equal(x, y)
            _check_consistent(q, db, t[0], t[1])
        finally:
            idx.close()


def _cpu_spill_counts(db, cent, s):
    """Each row's clusters as spill >= 3 chooses them: the 8 nearest of every 128
    centroids by (distance, index), then the best s of those."""
    key = _hamming(db, cent).astype(np.int64) * 4096 + np.arange(cent.shape[0])[None, :]
    cand = np.concatenate([np.sort(key[:, t:t + 128], axis=1)[:, :8] for t in range(0, cent.shape[0], 128)], axis=1)
    best = np.sort(cand, axis=1)[:, :s] % 4096
    return np.bincount(best.reshape(-1), minlength=cent.shape[0])


@pytest.mark.parametrize("spill", [3, 8, 12])
def test_wide_spill_lists_and_recall(ctx, spill):
    db, q = clustered(16384, 2048, seed=11)
    tdb, tq = torch.from_numpy(db).cuda(), torch.from_numpy(q).cuda()
    p = orbx.learned_params(n_clusters=256, hidden=512, epochs=1, batch=512, kmeans_iters=8, spill=spill)
    idx = orbx.LearnedIndex(ctx, tdb, tq[:512].contiguous(), p)
    try:
        ex = idx.export(weights=False)
        cent = _ckpt_centroids(idx.save(), 256)
        counts = np.diff(ex["offsets"])
        assert ex["offsets"][-1] == spill * len(db)
        assert np.array_equal(counts, _cpu_spill_counts(db, cent, spill))
        t, pp = _both_forms(ctx, idx, tq)
        for x, y in zip(t, pp):
            assert torch.equal(x, y)
        d, _ = _check_consistent(q, db, t[0], t[1])
        ed, _ = MO.knn1_bruteforce(q, db)
        recall = float(np.mean(d[:, 0] == ed))
        # spill 2 on the same data and clustering for comparison: wider lists find more
        p2 = orbx.learned_params(n_clusters=256, hidden=512, epochs=1, batch=512, kmeans_iters=8, spill=2)
        idx2 = orbx.LearnedIndex(ctx, tdb, tq[:512].contiguous(), p2)
        try:
            d2, i2, _, _ = idx2.search(tq)
            ctx.sync()
            r2 = float(np.mean(d2.cpu().numpy()[:, 0] == ed))
        finally:
            idx2.close()
        assert recall >= r2, (recall, r2)
    finally:
        idx.close()


# ---------------------------------------------------------------- label sets
def test_listed_labels(ctx):
    """ORBX_LABEL_LISTED trains on the softmax mass of the nearest row's listed
    clusters.  With spill 1 that set is the nearest cluster alone, so training
    equals ORBX_LABEL_NEAREST weight for weight; with spill 4 the set loss
    falls over the epochs and the search stays exact in the rows it scans."""
    db, q = clustered(16384, 2048, seed=21)
    tdb, tq = torch.from_numpy(db).cuda(), torch.from_numpy(q).cuda()
    train = tq[:1024].contiguous()
    base = dict(n_clusters=256, hidden=512, epochs=3, batch=512, kmeans_iters=6)
    w = {}
    for mode in (orbx.LABEL_NEAREST, orbx.LABEL_LISTED):
        idx = orbx.LearnedIndex(ctx, tdb, train, orbx.learned_params(spill=1, label_mode=mode, **base))
        try:
            w[mode] = idx.export()
        finally:
            idx.close()
    for k in ("w1", "b1", "w2", "b2"):
        assert np.array_equal(w[orbx.LABEL_NEAREST][k], w[orbx.LABEL_LISTED][k]), k
    idx = orbx.LearnedIndex(ctx, tdb, train, orbx.learned_params(spill=4, label_mode=orbx.LABEL_LISTED, **base))
    try:
        st = idx.stats()
        assert st["loss"][-1] < st["loss"][0], st["loss"]
        d, i, _, _ = idx.search(tq)
        ctx.sync()
        _check_consistent(q, db, d, i)
    finally:
        idx.close()
