"""Batched frame pairs (orbx_batch_pairs): many pairs of mixed resolution and
keypoint caps, in five shared launches or in one persistent launch with a
device work queue, must give, pair by pair, exactly what orbx_pair gives on
that pair alone and what the oracle gives; the autotuner must keep results
unchanged.  The 64-pair workload (resolutions 320x240 .. 3840x2160, caps
U[500, 10000]) is checked pair by pair against the oracle, and one of its pairs
against the reference build itself."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import orbx  # noqa: E402
import synth  # noqa: E402
from conftest import canon_order  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import refharness as R  # noqa: E402

PAIRS = [(320, 240, 500), (640, 480, 10000), (1280, 720, 3000), (333, 257, 200), (1920, 1080, 10000),
         (3840, 2160, 8000), (640, 480, 64), (1024, 1024, 5000)]


@pytest.fixture(scope="module")
def batch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pairs = []
    for k, (w, h, cap) in enumerate(PAIRS):
        a, b, _ = synth.make_pair(w, h, seed=100 + k)
        pairs.append((a, b, w, h, cap))
    return pairs


def _single(ctx, a, b, w, h, cap):
    ctx.init(orbx.make_params(max_pts=cap))
    A, B = orbx.FrameBuffers(cap), orbx.FrameBuffers(cap)
    ctx.pair_ptr(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), w, h, a.shape[1], A.points, A.desc,
                 A.count, B.points, B.desc, B.count)
    ctx.sync()
    return A.to_host() + B.to_host()


def _check_against_single(ctx_single, pb, pairs):
    for i, (a, b, w, h, cap) in enumerate(pairs):
        got = pb.results(i)
        want = _single(ctx_single, a, b, w, h, cap)
        for g, e in zip(got, want):
            assert np.array_equal(g, e), (i, w, h, cap)
        assert len(got[0]) <= cap
        m, d = O.match(got[1], got[3])
        assert np.array_equal(got[0]["match"], m) and np.array_equal(got[0]["distance"], d)


def test_batch_equals_single_pairs(batch):
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    single = orbx.Context(0, orbx.make_params(max_pts=10000))
    pb = orbx.PairBatch(batch)
    for _ in range(2):  # capture, then replay
        ctx.batch_pairs(pb)
        ctx.sync()
        _check_against_single(single, pb, batch)
    ctx.close()
    single.close()


def test_autotune_keeps_results(batch):
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    single = orbx.Context(0, orbx.make_params(max_pts=10000))
    pb = orbx.PairBatch(batch[:5])
    t, ms = ctx.autotune_pairs(pb, reps=2)
    assert ms > 0 and 1 <= t.nms_rows <= 16
    assert ctx.get_tuning().as_dict() == t.as_dict()
    ctx.batch_pairs(pb)
    ctx.sync()
    _check_against_single(single, pb, batch[:5])
    ctx.close()
    single.close()


@pytest.mark.parametrize("rows", [1, 2, 8, 16])
def test_nms_strip_heights_agree(batch, rows):
    a, b, w, h, cap = batch[4]
    ctx = orbx.Context(0, orbx.make_params(max_pts=cap))
    t = ctx.get_tuning()
    t.nms_rows = rows
    ctx.set_tuning(t)
    got = _single(ctx, a, b, w, h, cap)
    ref = _single(orbx.Context(0, orbx.make_params(max_pts=cap)), a, b, w, h, cap)
    for g, e in zip(got, ref):
        assert np.array_equal(g, e)
    ctx.close()


def _set_form(ctx, form, group=0, bps=0, rows=0):
    t = ctx.get_tuning()
    t.batch_form = form
    t.persist_group = group
    t.persist_blocks_per_sm = bps
    t.persist_row_deps = rows
    ctx.set_tuning(t)


@pytest.mark.parametrize("group,bps,rows", [(0, 0, 0), (2, 1, 0), (4, 0, 0), (0, 0, 1), (0, 1, 1)])
def test_persistent_batch_equals_single_pairs(batch, group, bps, rows):
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    single = orbx.Context(0, orbx.make_params(max_pts=10000))
    _set_form(ctx, 1, group, bps, rows)
    pb = orbx.PairBatch(batch)
    for _ in range(3):  # capture, then replays (counters and strip words reset each time)
        ctx.batch_pairs(pb)
        assert ctx.sync() is None
        _check_against_single(single, pb, batch)
    ctx.close()
    single.close()


def _sincos():
    if R.available():
        R.lib()
        return R.sincos
    return None


@pytest.fixture(scope="module")
def batch64():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pairs = []
    for k, (w, h, cap) in enumerate(synth.batch_layout()):
        a, b, _ = synth.make_pair(w, h, seed=1000 + k)
        pairs.append((a, b, w, h, cap))
    return pairs


@pytest.mark.parametrize("form", [0, 1])
def test_batch64_against_oracle(batch64, form):
    """The 64-pair workload in one batch: every pair's keypoints (first cap in
    raster order), descriptors and matches equal the oracle's."""
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    _set_form(ctx, form)
    pb = orbx.PairBatch(batch64)
    ctx.batch_pairs(pb)
    ctx.sync()
    sc = _sincos()
    for i, (a, b, w, h, cap) in enumerate(batch64):
        pa, da, pbb, db = pb.results(i)
        for pts, desc, img in ((pa, da, a), (pbb, db, b)):
            ref = O.detect_and_compute(img, w, h, max_pts=cap, sincos=sc)
            rp = ref["points"]
            assert len(pts) == len(rp) == min(cap, ref["total"]), (i, w, h, cap)
            for f in ("x", "y", "octave"):
                assert np.array_equal(pts[f], rp[f]), (i, f)
            assert np.array_equal(pts["score"].view(np.uint32), rp["score"].view(np.uint32)), i
            assert np.array_equal(pts["angle"].view(np.uint32), rp["angle"].view(np.uint32)), i
            if sc is not None:
                assert np.array_equal(desc, ref["desc"]), i
        m, d = O.match(da, db)
        assert np.array_equal(pa["match"], m) and np.array_equal(pa["distance"], d), i
    ctx.close()


@pytest.mark.skipif(not R.available(), reason="reference build not present")
def test_batch64_pair_against_reference_build(batch64):
    """One pair of the 64-pair batch (the first 1280x720 one) against the
    reference build (race-free blur) run on the same images."""
    i = next(k for k, p in enumerate(batch64) if p[2] == 1280)
    a, b, w, h, cap = batch64[i]
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    _set_form(ctx, 1)
    pb = orbx.PairBatch(batch64)
    ctx.batch_pairs(pb)
    ctx.sync()
    pa, da, pbb, db = pb.results(i)
    R.init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1, max_pts=20000)
    for pts, desc, img in ((pa, da, a), (pbb, db, b)):
        st = R.stages(img, w, h, 20000, race_free=True)
        o = canon_order(st["points"])
        rp = st["points"][o][:cap]
        assert len(pts) == len(rp)
        for f in ("x", "y", "octave"):
            assert np.array_equal(pts[f], rp[f])
        assert np.array_equal(pts["score"].view(np.uint32), rp["score"].view(np.uint32))
        assert np.array_equal(pts["angle"].view(np.uint32), rp["angle"].view(np.uint32))
        assert np.array_equal(desc, st["desc"][o][:cap])
    ctx.close()


def test_bounded_wait_times_out_and_context_recovers(batch):
    """A device wait on a counter that nothing sets gives up after its bound and
    the call reports ORBX_ERR_TIMEOUT; the same context then runs a batch in the
    persistent form normally."""
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    assert ctx.selftest_wait_timeout(2000) == orbx.ORBX_ERR_TIMEOUT
    assert ctx.selftest_wait_timeout(2000) == orbx.ORBX_ERR_TIMEOUT  # the error word was cleared in between
    _set_form(ctx, 1)
    pb = orbx.PairBatch(batch[:3])
    ctx.batch_pairs(pb)
    ctx.sync()
    single = orbx.Context(0, orbx.make_params(max_pts=10000))
    _check_against_single(single, pb, batch[:3])
    ctx.close()
    single.close()


def test_wait_timeout_tuning_is_validated():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = orbx.Context(0, orbx.make_params(max_pts=1000))
    t = ctx.get_tuning()
    assert t.wait_timeout_us == 1000000 and t.batch_form == 0
    t.wait_timeout_us = 0
    with pytest.raises(orbx.OrbxError):
        ctx.set_tuning(t)
    ctx.close()


@pytest.mark.parametrize("rows", [0, 1])
@pytest.mark.parametrize("w,h,seed,cap", [(1920, 1080, 7, 10000), (333, 257, 8, 200), (3840, 2160, 9, 10000)])
def test_pair_persistent_form_equals_five_launches(w, h, seed, cap, rows):
    """orbx_pair as one persistent launch (per-frame or row-level stage
    dependencies) gives exactly the five-launch results."""
    a, b, _ = synth.make_pair(w, h, seed=seed)
    five = orbx.Context(0, orbx.make_params(max_pts=cap))
    pers = orbx.Context(0, orbx.make_params(max_pts=cap))
    t = pers.get_tuning()
    t.pair_form = 1
    t.persist_row_deps = rows
    pers.set_tuning(t)
    want = _single(five, a, b, w, h, cap)
    for _ in range(3):
        got = _single(pers, a, b, w, h, cap)
        for g, e in zip(got, want):
            assert np.array_equal(g, e)
    five.close()
    pers.close()


@pytest.mark.parametrize("shape", [1, 2, 3])
def test_pyramid_tile_shapes_agree(batch, shape):
    """Every pyramid + blur tile shape of the five-launch form gives the same
    batch results (pair by pair equal to orbx_pair with the default shape)."""
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    single = orbx.Context(0, orbx.make_params(max_pts=10000))
    t = ctx.get_tuning()
    t.pyr_tile = shape
    ctx.set_tuning(t)
    pb = orbx.PairBatch(batch)
    ctx.batch_pairs(pb)
    ctx.sync()
    _check_against_single(single, pb, batch)
    ctx.close()
    single.close()
