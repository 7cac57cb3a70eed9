"""Parity of the sm_100a library (through its C ABI) with the reference.

Checkers: the CPU oracle (oracle/), the golden fixtures produced by the
reference CUDA build (tests/golden/), and, when oracle/_ref/libref_orb.so is
present, the reference build itself run live on the same inputs.  Integer and
byte outputs are compared bit-exactly, floats by their bit patterns.
"""
import numpy as np
import pytest

from conftest import canon_order

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import orbx  # noqa: E402
import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import refharness as R  # noqa: E402


def f32bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = orbx.Context(0, orbx.make_params(max_pts=10000))
    yield c
    c.close()


def run_frame(ctx, img, w, h, compute_desc=True):
    d = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    bufs = orbx.detect_and_compute(ctx, d, w, h, compute_desc=compute_desc)
    ctx.sync()
    pts, desc = bufs.to_host()
    return pts, desc


def ref_sincos(angles):
    if R.available():
        R.lib()
        return R.sincos(angles)
    return None


def check_against_golden_image(ctx, g, img_key, prefix, params):
    w, h = int(g["w"]), int(g["h"])
    ctx.init(params)
    pts, desc = run_frame(ctx, g[img_key], w, h)
    gpts = g[prefix + "points"]
    order = canon_order(gpts)
    gp = gpts[order]
    assert len(pts) == len(gp)
    # the library emits raster order, which is the canonical order
    assert np.array_equal(canon_order(pts), np.arange(len(pts)))
    for f in ("x", "y", "octave"):
        assert np.array_equal(pts[f], gp[f]), f
    assert np.array_equal(f32bits(pts["score"]), f32bits(gp["score"]))
    assert np.array_equal(f32bits(pts["angle"]), f32bits(gp["angle"]))
    assert np.array_equal(desc, g[prefix + "desc"][order])
    return pts, desc


@pytest.mark.parametrize("name", ["pair_320x240_s1.npz", "pair_640x480_s2.npz"])
@pytest.mark.parametrize("img", ["A", "B"])
def test_golden_pairs(ctx, golden, name, img):
    g = golden(name)
    check_against_golden_image(ctx, g, "img" + img, img + "_", orbx.make_params(max_pts=10000))


def test_golden_internal_buffers(ctx, golden):
    g = golden("pair_320x240_s1.npz")
    w, h = int(g["w"]), int(g["h"])
    ctx.init(orbx.make_params(max_pts=10000))
    run_frame(ctx, g["imgA"], w, h)
    dbg = ctx.debug_buffers(w, h)
    assert np.array_equal(dbg["pyr"], g["A_pyr_raw"])
    assert np.array_equal(dbg["blur"], g["A_pyr_blur"])
    nz = np.nonzero(dbg["vmap"])[0]
    assert np.array_equal(nz, g["A_map_idx"])
    assert np.array_equal(f32bits(dbg["vmap"][nz]), f32bits(g["A_map_score"]))
    assert np.array_equal(dbg["layer"][nz], g["A_map_layer"])


@pytest.mark.parametrize("case,score,wta,patch", [("fast", 1, 2, 31), ("wta3", 0, 3, 31), ("wta4", 0, 4, 31),
                                                  ("patch25", 0, 2, 25)])
def test_golden_variants(ctx, golden, case, score, wta, patch):
    g = golden("variants_320x240.npz")
    params = orbx.make_params(max_pts=4000, score_type=score, wta_k=wta, patch_size=patch)
    check_against_golden_image(ctx, g, "img", case + "_", params)


def test_cap_keeps_first_in_raster_order(ctx, golden):
    g = golden("cap_320x240.npz")
    w, h = int(g["w"]), int(g["h"])
    cap = int(g["cap"])
    ctx.init(orbx.make_params(max_pts=cap))
    pts, desc = run_frame(ctx, g["img"], w, h)
    full = g["full_points"][canon_order(g["full_points"])]
    assert len(pts) == cap == int(g["cap_num_pts"])
    assert np.array_equal(pts["x"], full["x"][:cap]) and np.array_equal(pts["y"], full["y"][:cap])
    dbg = ctx.debug_buffers(w, h)
    assert dbg["total"] == len(full)


@pytest.mark.parametrize("w,h,seed", [(1920, 1080, 0), (333, 257, 7), (1280, 720, 5), (3840, 2160, 9),
                                      (1024, 1024, 11)])
def test_against_oracle_sizes(ctx, w, h, seed):
    """Whole pipeline vs the oracle on fresh seeds; descriptors use the GPU's
    __sinf/__cosf via the reference build when present, else only keypoints,
    scores and angles are compared plus descriptors on the shared-sign subset."""
    a, b, _ = synth.make_pair(w, h, seed)
    ctx.init(orbx.make_params(max_pts=20000))
    for img in (a, b):
        pts, desc = run_frame(ctx, img, w, h)
        ref = O.detect_and_compute(img, w, h, max_pts=20000, sincos=ref_sincos if R.available() else None)
        rp = ref["points"]
        assert len(pts) == len(rp) == ref["total"]
        for f in ("x", "y", "octave"):
            assert np.array_equal(pts[f], rp[f]), f
        assert np.array_equal(f32bits(pts["score"]), f32bits(rp["score"]))
        assert np.array_equal(f32bits(pts["angle"]), f32bits(rp["angle"]))
        if R.available():
            assert np.array_equal(desc, ref["desc"])
        else:
            # libm sin/cos differ from __sinf/__cosf in the last bits; rows must still mostly agree
            same = np.all(desc == ref["desc"], axis=1).mean()
            assert same > 0.99


@pytest.mark.parametrize("w,h,seed,nms_rows", [(640, 480, 3, 0), (1280, 720, 4, 0), (1280, 720, 4, 16)])
def test_dense_corners_vs_oracle(ctx, w, h, seed, nms_rows):
    """Uniform noise in the top half (corners at a large share of its pixels),
    the synthetic scene below.  NMS strips whose window holds more set bits
    than its shared-memory stage check their centres in rounds over global
    memory, the others from the stage; both must give the oracle's keypoints."""
    img, _, _ = synth.make_pair(w, h, seed)
    rng = np.random.default_rng(seed)
    img = img.copy()
    img[: h // 2] = rng.integers(0, 256, size=(h // 2, img.shape[1]), dtype=np.uint8)
    cap = w * h // 4
    ctx.init(orbx.make_params(max_pts=cap))
    if nms_rows:
        t = ctx.get_tuning()
        t.nms_rows = nms_rows
        ctx.set_tuning(t)
    pts, desc = run_frame(ctx, img, w, h)
    ref = O.detect_and_compute(img, w, h, max_pts=cap, sincos=ref_sincos if R.available() else None)
    rp = ref["points"]
    assert ref["total"] > 2048  # far more set bits than one strip's stage holds
    assert len(pts) == len(rp) == ref["total"]
    for f in ("x", "y", "octave"):
        assert np.array_equal(pts[f], rp[f]), f
    assert np.array_equal(f32bits(pts["score"]), f32bits(rp["score"]))
    assert np.array_equal(f32bits(pts["angle"]), f32bits(rp["angle"]))
    if R.available():
        assert np.array_equal(desc, ref["desc"])


@pytest.mark.skipif(not R.available(), reason="reference build not present")
@pytest.mark.parametrize("w,h,seed", [(1920, 1080, 0), (640, 480, 21)])
def test_against_reference_build_live(ctx, w, h, seed):
    """The reference CUDA build (race-free blur) on the same inputs, same GPU."""
    a, b, _ = synth.make_pair(w, h, seed)
    ctx.init(orbx.make_params(max_pts=10000))
    R.init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1, max_pts=10000)
    descs = []
    for img in (a, b):
        pts, desc = run_frame(ctx, img, w, h)
        st = R.stages(img, w, h, 10000, race_free=True)
        order = canon_order(st["points"])
        rp = st["points"][order]
        assert len(pts) == len(rp)
        for f in ("x", "y", "octave"):
            assert np.array_equal(pts[f], rp[f])
        assert np.array_equal(f32bits(pts["score"]), f32bits(rp["score"]))
        assert np.array_equal(f32bits(pts["angle"]), f32bits(rp["angle"]))
        assert np.array_equal(desc, st["desc"][order])
        descs.append((desc, st["desc"][order]))
    # matching: same descriptor sets in the same order -> identical match/distance
    m_ref, d_ref = R.hmatch(descs[0][1], descs[1][1])
    m_o, d_o = O.match(descs[0][0], descs[1][0])
    assert np.array_equal(m_ref, m_o) and np.array_equal(d_ref, d_o)


def _match_gpu(ctx, d1, d2, mode=orbx.MATCH_POPC):
    n1, n2 = len(d1), len(d2)
    pts = torch.zeros((max(n1, 1), 7), dtype=torch.int32, device="cuda")
    t1 = torch.from_numpy(np.ascontiguousarray(d1)).cuda() if n1 else torch.zeros((1, 32), dtype=torch.uint8,
                                                                                  device="cuda")
    t2 = torch.from_numpy(np.ascontiguousarray(d2)).cuda() if n2 else None
    cnt = torch.tensor([n1, n2], dtype=torch.int32, device="cuda")
    ctx.match_ptr(pts, cnt[0:1].data_ptr(), t1, cnt[1:2].data_ptr(), t2, n1, n2, mode)
    ctx.sync()
    p = pts[:n1].cpu().numpy()
    return p[:, 5].copy(), p[:, 6].copy()


@pytest.mark.parametrize("mode", [orbx.MATCH_POPC, orbx.MATCH_IMMA])
def test_match_kat(ctx, golden, mode):
    g = golden("match_kat.npz")
    for name in g["names"]:
        name = str(name)
        m, d = _match_gpu(ctx, g[name + "_q"], g[name + "_db"], mode)
        assert np.array_equal(m, g[name + "_match"]), name
        assert np.array_equal(d, g[name + "_dist"]), name


@pytest.mark.parametrize("mode", [orbx.MATCH_POPC, orbx.MATCH_IMMA])
@pytest.mark.parametrize("name", ["pair_320x240_s1.npz", "pair_640x480_s2.npz"])
def test_match_golden_pairs(ctx, golden, name, mode):
    g = golden(name)
    m, d = _match_gpu(ctx, g["A_desc"], g["B_desc"], mode)
    assert np.array_equal(m, g["match_rf"]) and np.array_equal(d, g["dist_rf"])


@pytest.mark.parametrize("mode", [orbx.MATCH_POPC, orbx.MATCH_IMMA])
@pytest.mark.parametrize("nq,ndb", [(1, 1), (5, 0), (127, 129), (1000, 1000), (3000, 200), (200, 70000),
                                    (4096, 16384), (333, 257)])
def test_knn2_vs_oracle(ctx, nq, ndb, mode):
    db, q, _ = synth.match_workload(max(ndb, 1), nq, seed=nq * 7 + ndb)
    db = db[:ndb]
    dist, idx = orbx.knn2(ctx, torch.from_numpy(q).cuda(), torch.from_numpy(db).cuda() if ndb else
                          torch.zeros((0, 32), dtype=torch.uint8, device="cuda"), mode)
    ctx.sync()
    od, oi = O.knn2(q, db)
    assert np.array_equal(dist.cpu().numpy().view(np.uint32), od)
    assert np.array_equal(idx.cpu().numpy(), oi)


@pytest.mark.parametrize("mode", [orbx.MATCH_POPC, orbx.MATCH_IMMA])
def test_knn2_full_size_sampled(ctx, mode):
    """65536 x 65536 (the matching-only workload) on the GPU; a seeded sample of
    2048 queries is checked against the oracle, and every planted near-duplicate
    query must find its source row."""
    db, q, src = synth.match_workload(65536, 65536, seed=0)
    dist, idx = orbx.knn2(ctx, torch.from_numpy(q).cuda(), torch.from_numpy(db).cuda(), mode)
    ctx.sync()
    dist = dist.cpu().numpy().view(np.uint32)
    idx = idx.cpu().numpy()
    rng = np.random.default_rng(5)
    sample = np.sort(rng.choice(65536, 2048, replace=False))
    od, oi = O.knn2(q[sample], db)
    assert np.array_equal(dist[sample], od) and np.array_equal(idx[sample], oi)
    half = len(src)
    assert np.mean(idx[:half, 0] == src) > 0.999
    assert np.all(dist[:, 0] <= dist[:, 1])


def test_imma_equals_popc_full_size(ctx):
    """Both matcher forms on the 65536 x 65536 workload: identical distances and indices."""
    db, q, _ = synth.match_workload(65536, 65536, seed=1)
    tq, tdb = torch.from_numpy(q).cuda(), torch.from_numpy(db).cuda()
    d0, i0 = orbx.knn2(ctx, tq, tdb, orbx.MATCH_POPC)
    d1, i1 = orbx.knn2(ctx, tq, tdb, orbx.MATCH_IMMA)
    ctx.sync()
    assert torch.equal(d0, d1) and torch.equal(i0, i1)


@pytest.mark.parametrize("mode", [orbx.MATCH_POPC, orbx.MATCH_IMMA])
def test_pair_api_matches_single_calls(ctx, mode):
    w, h = 1280, 720
    a, b, _ = synth.make_pair(w, h, 3)
    ctx.init(orbx.make_params(max_pts=10000))
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    A = orbx.FrameBuffers(10000)
    B = orbx.FrameBuffers(10000)
    for _ in range(3):  # first call captures the graph, later calls replay it
        ctx.pair_ptr(da, db, w, h, a.shape[1], A.points, A.desc, A.count, B.points, B.desc, B.count, mode)
        ctx.sync()
        pa, desc_a = A.to_host()
        pb, desc_b = B.to_host()
        sa, sda = run_frame(ctx, a, w, h)
        sb, sdb = run_frame(ctx, b, w, h)
        for f in ("x", "y", "octave"):
            assert np.array_equal(pa[f], sa[f]) and np.array_equal(pb[f], sb[f])
        assert np.array_equal(desc_a, sda) and np.array_equal(desc_b, sdb)
        m, d = O.match(desc_a, desc_b)
        assert np.array_equal(pa["match"], m) and np.array_equal(pa["distance"], d)


def test_determinism_repeat(ctx):
    w, h = 1920, 1080
    a, _, _ = synth.make_pair(w, h, 1)
    ctx.init(orbx.make_params(max_pts=10000))
    first = run_frame(ctx, a, w, h)
    for _ in range(5):
        again = run_frame(ctx, a, w, h)
        assert np.array_equal(first[0], again[0]) and np.array_equal(first[1], again[1])


def test_flat_image_has_no_keypoints(ctx):
    w, h = 640, 480
    img = np.full((h, 640), 128, dtype=np.uint8)
    ctx.init(orbx.make_params(max_pts=1000))
    pts, desc = run_frame(ctx, img, w, h)
    assert len(pts) == 0


def test_wider_pitch_same_result(ctx):
    w, h = 640, 480
    a, _, _ = synth.make_pair(w, h, 4)
    ctx.init(orbx.make_params(max_pts=10000))
    base = run_frame(ctx, a, w, h)
    wide = np.zeros((h, 1024), dtype=np.uint8)
    wide[:, :w] = a[:, :w]
    d = torch.from_numpy(wide).cuda()
    bufs = orbx.detect_and_compute(ctx, d, w, h)
    ctx.sync()
    pts, desc = bufs.to_host()
    assert np.array_equal(pts, base[0]) and np.array_equal(desc, base[1])


def test_size_errors(ctx):
    ctx.init(orbx.make_params(max_pts=100))
    d = torch.zeros((60, 128), dtype=torch.uint8, device="cuda")
    bufs = orbx.FrameBuffers(100)
    with pytest.raises(orbx.OrbxError) as e:
        ctx.detect_and_compute_ptr(d, 70, 60, 128, bufs.points, bufs.desc, bufs.count)
    assert e.value.status == 3
    with pytest.raises(orbx.OrbxError):
        ctx.detect_and_compute_ptr(d, 70, 60, 60, bufs.points, bufs.desc, bufs.count)  # pitch < w
