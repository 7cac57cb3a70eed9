"""Workloads run through both builds of the library by tests/test_gpu_bounds.py.

run(orbx, synth) drives the loaded library (normal or bounds-checked, chosen
by ORBX_CHECKED when orbx is imported) over the pair, batch, host-buffer and
k = 2 entry points, and returns every output as numpy arrays keyed by case,
plus, in the checked build, the bounds record read after each case.

Run as a script (ORBX_CHECKED=1 python tests/bounds_cases.py OUT.npz) it saves
that dictionary, so the bounds-checked library runs in a process of its own.
"""
import os
import sys

import numpy as np

# (w, h, pitch, max_pts, params): odd sizes, padded pitches, binding caps, 4K
PAIRS = [
    (333, 257, 333, 200, {}),
    (1000, 701, 1012, 10000, {}),
    (1920, 1080, 1920, 10000, {}),
    (3840, 2160, 3840, 8000, {}),
    (640, 480, 640, 64, {}),
    (640, 480, 640, 5000, {"wta_k": 3}),
    (640, 480, 640, 5000, {"wta_k": 4}),
    (640, 480, 640, 5000, {"patch_size": 25}),
    (640, 480, 640, 5000, {"score_type": 1}),
]
BATCH = [(320, 240, 500), (1280, 720, 3000), (333, 257, 200), (1920, 1080, 10000), (640, 480, 64)]


def _padded(img, w, pitch):
    """The first w columns of a generated image, in rows of `pitch` bytes (padding 0x5A)."""
    out = np.full((img.shape[0], pitch), 0x5A, dtype=np.uint8)
    out[:, :w] = img[:, :w]
    return out


def _report(ctx, out, key):
    if ctx is not None and _checked():
        out[key + ".bounds"] = np.array(ctx.bounds_report(), dtype=np.int64)


def _checked():
    import orbx

    return orbx.CHECKED


def run(orbx, synth, torch):
    out = {}
    # pairs, five-launch form, and the 1080p pair as one persistent launch
    for k, (w, h, pitch, cap, kw) in enumerate(PAIRS):
        a, b, _ = synth.make_pair(w, h, seed=700 + k)
        a, b = _padded(a, w, pitch), _padded(b, w, pitch)
        forms = [0, 1] if (w, h) == (1920, 1080) else [0]
        for form in forms:
            ctx = orbx.Context(0, orbx.make_params(max_pts=cap, **kw))
            if form:
                t = ctx.get_tuning()
                t.pair_form = 1
                ctx.set_tuning(t)
            A, B = orbx.FrameBuffers(cap), orbx.FrameBuffers(cap)
            ctx.pair_ptr(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), w, h, pitch, A.points, A.desc,
                         A.count, B.points, B.desc, B.count)
            ctx.sync()
            key = f"pair{k}_form{form}"
            pa, da = A.to_host()
            pb, db = B.to_host()
            out[key + ".pa"], out[key + ".da"] = pa.view(np.int32).reshape(-1, 7), da
            out[key + ".pb"], out[key + ".db"] = pb.view(np.int32).reshape(-1, 7), db
            _report(ctx, out, key)
            ctx.close()
    # batches: five shared launches and one persistent launch
    pairs = []
    for k, (w, h, cap) in enumerate(BATCH):
        a, b, _ = synth.make_pair(w, h, seed=800 + k)
        pairs.append((a, b, w, h, cap))
    for form in (0, 1):
        ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
        t = ctx.get_tuning()
        t.batch_form = form
        ctx.set_tuning(t)
        pb_ = orbx.PairBatch(pairs)
        ctx.batch_pairs(pb_)
        ctx.sync()
        for i in range(len(pairs)):
            pa, da, pb, db = pb_.results(i)
            key = f"batch{form}_{i}"
            out[key + ".pa"], out[key + ".da"] = pa.view(np.int32).reshape(-1, 7), da
            out[key + ".pb"], out[key + ".db"] = pb.view(np.int32).reshape(-1, 7), db
        _report(ctx, out, f"batch{form}")
        ctx.close()
    # host buffers in and out: two streams (pageable images, then pinned ones
    # replayed from a graph) and banded uploads into one persistent launch
    w, h = 1280, 720
    a, b, _ = synth.make_pair(w, h, seed=900)
    pinned = [torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in (a, b)]
    for name, bands, src in (("host", 0, (np.ascontiguousarray(a), np.ascontiguousarray(b))),
                             ("hostpinned", 0, tuple(t.data_ptr() for t in pinned)),
                             ("hostbands", 4, tuple(t.data_ptr() for t in pinned))):
        ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
        t = ctx.get_tuning()
        t.upload_bands = bands
        ctx.set_tuning(t)
        hpa = np.zeros((10000, 7), np.int32)
        hpb = np.zeros((10000, 7), np.int32)
        hna, hnb = np.zeros(1, np.int32), np.zeros(1, np.int32)
        hda, hdb = np.zeros((10000, 32), np.uint8), np.zeros((10000, 32), np.uint8)
        for _ in range(2):
            ctx.pair_host(src[0], src[1], w, h, a.shape[1], hpa, hna, hpb, hnb, hda, hdb)
        na, nb = int(hna[0]), int(hnb[0])
        out[name + ".pa"], out[name + ".da"] = hpa[:na].copy(), hda[:na].copy()
        out[name + ".pb"], out[name + ".db"] = hpb[:nb].copy(), hdb[:nb].copy()
        _report(ctx, out, name)
        ctx.close()
    # one frame (orbx_detect_and_compute) at an odd width and unaligned pitch
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    img = _padded(a, 1277, 1277)
    bufs = orbx.detect_and_compute(ctx, torch.from_numpy(img).cuda(), 1277, h)
    ctx.sync()
    p1, d1 = bufs.to_host()
    out["single.p"], out["single.d"] = p1.view(np.int32).reshape(-1, 7), d1
    _report(ctx, out, "single")
    # k = 2 lists, popcount form, ragged sizes
    rng = np.random.default_rng(901)
    q = torch.from_numpy(rng.integers(0, 256, (1000, 32), dtype=np.uint8)).cuda()
    d = torch.from_numpy(rng.integers(0, 256, (777, 32), dtype=np.uint8)).cuda()
    dist, idx = orbx.knn2(ctx, q, d, orbx.MATCH_POPC)
    ctx.sync()
    out["knn2.dist"], out["knn2.idx"] = dist.cpu().numpy(), idx.cpu().numpy()
    _report(ctx, out, "knn2")
    ctx.close()
    return out


def run_slack(orbx, synth, torch):
    """Checked build only: a 333 x 257 pair whose image extents, as checked,
    end two rows early.  The pyramid's reads of those rows must be reported."""
    w, h = 333, 257
    a, b, _ = synth.make_pair(w, h, seed=950)
    ctx = orbx.Context(0, orbx.make_params(max_pts=2000))
    ctx.bounds_set_slack(2 * a.shape[1])
    A, B = orbx.FrameBuffers(2000), orbx.FrameBuffers(2000)
    ctx.pair_ptr(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), w, h, a.shape[1], A.points, A.desc,
                 A.count, B.points, B.desc, B.count)
    ctx.sync()
    rep = ctx.bounds_report()
    ctx.close()
    return np.array(rep, dtype=np.int64)


if __name__ == "__main__":
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "cuda-orb_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch

    import orbx
    import synth

    assert orbx.CHECKED and orbx.lib().orbx_bounds_checked() == 1, "needs ORBX_CHECKED=1"
    res = run(orbx, synth, torch)
    res["slack.bounds"] = run_slack(orbx, synth, torch)
    np.savez(sys.argv[1], **res)
    print("bounds cases:", len(res), "arrays")
