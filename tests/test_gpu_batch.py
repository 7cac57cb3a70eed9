"""Batched frame pairs (orbx_batch_pairs): many pairs of mixed resolution and
keypoint caps in shared launches must give, pair by pair, exactly what
orbx_pair gives on that pair alone; the autotuner must keep results unchanged."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import orbx  # noqa: E402
import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

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
