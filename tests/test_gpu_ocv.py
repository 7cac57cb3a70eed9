"""OpenCV-compatible mode (orbx_ocv_detect_and_compute) against cv2.ORB on the
same synthetic images.  The mode follows cv::ORB's published algorithm, not
its code, so the comparison is statistical: keypoint counts per level, level-0
positions (the level-0 image is shared, so FAST + NMS + the two retains should
mostly pick the same pixels), angles and descriptors at the shared positions,
and the matching rate under the known homography of a warped pair."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
cv2 = pytest.importorskip("cv2")
pytestmark = pytest.mark.gpu

import orbx  # noqa: E402
import synth  # noqa: E402

NF = 2000


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = orbx.Context(0)
    yield c
    c.close()


def _ours(ctx, img, w, h, **kw):
    p = orbx.ocv_params(nfeatures=NF, **kw)
    return orbx.ocv_detect_and_compute(ctx, torch.from_numpy(img).cuda(), w, h, p)


def _cv(img, w, h, fast=False):
    orb = cv2.ORB_create(nfeatures=NF, scaleFactor=1.2, nlevels=8, edgeThreshold=31, patchSize=31, fastThreshold=20,
                         WTA_K=2, scoreType=cv2.ORB_FAST_SCORE if fast else cv2.ORB_HARRIS_SCORE)
    kps, desc = orb.detectAndCompute(np.ascontiguousarray(img[:, :w]), None)
    return kps, desc


def test_counts_positions_angles_descriptors(ctx):
    a, _, _ = synth.make_pair(640, 480, seed=51)
    k, d = _ours(ctx, a, 640, 480)
    ck, cd = _cv(a, 640, 480)
    assert abs(len(k) - len(ck)) <= 0.03 * len(ck), (len(k), len(ck))
    ours_lv = np.bincount(k["octave"], minlength=8)
    cv_lv = np.bincount([p.octave for p in ck], minlength=8)
    assert np.all(np.abs(ours_lv - cv_lv) <= np.maximum(0.05 * cv_lv, 5)), (ours_lv, cv_lv)
    # level 0: same image, same detector
    cv0 = {(int(round(p.pt[0])), int(round(p.pt[1]))): i for i, p in enumerate(ck) if p.octave == 0}
    ours0 = [(int(round(x)), int(round(y)), i) for i, (x, y, o) in enumerate(zip(k["x"], k["y"], k["octave"])) if o == 0]
    shared = [(i, cv0[(x, y)]) for x, y, i in ours0 if (x, y) in cv0]
    assert len(shared) >= 0.95 * len(ours0), (len(shared), len(ours0))
    dang = np.array([abs((k["angle"][i] - ck[j].angle + 180.0) % 360.0 - 180.0) for i, j in shared])
    assert np.mean(dang < 1.0) >= 0.98, np.percentile(dang, [50, 90, 99])
    ham = np.array([int(np.unpackbits(d[i] ^ cd[j]).sum()) for i, j in shared])
    assert np.median(ham) <= 2 and np.percentile(ham, 90) <= 8, np.percentile(ham, [50, 90])


def _inlier_rate(ka, da, kb, db, H):
    bf = cv2.BFMatcher(cv2.NORM_HAMMING, crossCheck=True)
    m = bf.match(da, db)
    if not m:
        return 0.0
    pa = np.array([ka[x.queryIdx] for x in m], dtype=np.float64)
    pb = np.array([kb[x.trainIdx] for x in m], dtype=np.float64)
    proj = (H @ np.c_[pa, np.ones(len(pa))].T).T
    proj = proj[:, :2] / proj[:, 2:3]
    return float(np.mean(np.linalg.norm(proj - pb, axis=1) < 3.0))


def test_matching_rate_under_homography(ctx):
    a, b, H = synth.make_pair(640, 480, seed=52)
    ka, da = _ours(ctx, a, 640, 480)
    kb, db = _ours(ctx, b, 640, 480)
    cka, cda = _cv(a, 640, 480)
    ckb, cdb = _cv(b, 640, 480)
    ours = _inlier_rate(np.c_[ka["x"], ka["y"]], da, np.c_[kb["x"], kb["y"]], db, H)
    ref = _inlier_rate(np.array([p.pt for p in cka]), cda, np.array([p.pt for p in ckb]), cdb, H)
    assert ours >= 0.85 * ref, (ours, ref)


def test_deterministic_and_fast_score_mode(ctx):
    a, _, _ = synth.make_pair(640, 480, seed=53)
    k1, d1 = _ours(ctx, a, 640, 480)
    k2, d2 = _ours(ctx, a, 640, 480)
    assert np.array_equal(k1, k2) and np.array_equal(d1, d2)
    # within a level, keypoints come in decreasing score order
    for lv in range(8):
        r = k1["response"][k1["octave"] == lv]
        assert np.all(np.diff(r) <= 0)
    kf, df = _ours(ctx, a, 640, 480, score_type=1)
    ck, _ = _cv(a, 640, 480, fast=True)
    assert abs(len(kf) - len(ck)) <= 0.1 * len(ck), (len(kf), len(ck))
    assert np.all(kf["response"] >= 20)
