"""The FP64 side-oracle and the exception counts of the parity report, on CPU.

The reference computes Harris scores (orbd.cu:651-669) and angles
(orbd.cu:986-1036) in FP32.  The FP64 restatement of the same formulas must
agree with the reference build's own values (the golden fixtures) within
1e-5 relative, with the absolute floors stated in oracle/oracle.py.  The
exception flags (rounding ties, octave-straddling patches) are checked on
planted cases where the answer is known by construction.
"""
import numpy as np
import pytest

from conftest import canon_order
from oracle import oracle as O

PAIRS = ["pair_320x240_s1.npz", "pair_640x480_s2.npz"]


@pytest.mark.parametrize("name", PAIRS)
@pytest.mark.parametrize("img", ["A", "B"])
def test_reference_scores_and_angles_within_fp64_tolerance(golden, name, img):
    g = golden(name)
    w, h = int(g["w"]), int(g["h"])
    pts = g[img + "_points"]
    rep = O.fp64_check(g["img" + img], w, h, pts, g[img + "_sin"], g[img + "_cos"])
    print(name, img, {k: v for k, v in rep.items() if k != "flags"})
    assert rep["keypoints"] == len(pts) > 0
    assert rep["harris_fail"] == 0 and rep["harris_term_bound_fail"] == 0
    assert rep["angle_fail"] == 0


def test_harris_floor_is_the_float_rounding_bound():
    # |A| <= 2^31 and B <= 2^32: the floor is 2^-22 (|A| + 0.04 B) scale^4 at its largest
    s4 = (1.0 / 7140.0) ** 4
    assert O.HARRIS_ABS_FLOOR == pytest.approx(2.0 ** -22 * (2.0 ** 31 + 0.04 * 2.0 ** 32) * s4)
    assert 2e-13 < O.HARRIS_ABS_FLOOR < 2.2e-13


def test_fp64_angle_matches_float_polynomial_on_a_ramp():
    # a horizontal ramp: m01 = 0, m10 > 0 -> angle 0; a vertical ramp -> pi/2
    w, h = 320, 240
    img = np.zeros((h, 384), dtype=np.uint8)
    img[:, :w] = (np.arange(w) % 256).astype(np.uint8)[None, :]
    n, oszp = O.layout(w, h)
    store, _ = O.pyramid(img, w, h, n, oszp)
    pts = np.zeros(1, dtype=O.ORB_POINT_DTYPE)
    pts["x"], pts["y"] = 100, 100
    a64 = O.angle_f64(store, n, oszp, pts)
    a32 = O.angle(store, n, oszp, pts.copy())["angle"]
    assert a64[0] == 0.0 and a32[0] == 0.0
    img2 = np.zeros((h, 384), dtype=np.uint8)
    img2[:, :w] = np.arange(h, dtype=np.uint8)[:, None]
    store2, _ = O.pyramid(img2, w, h, n, oszp)
    a64 = O.angle_f64(store2, n, oszp, pts)
    assert abs(a64[0] - np.pi / 2) < 1e-12


def test_tie_flag_on_planted_rotation():
    # cos = 0.5 exactly puts the pattern point (1, 0) on x = 0.5: a rounding tie
    n, oszp = O.layout(640, 480)
    pts = np.zeros(2, dtype=O.ORB_POINT_DTYPE)
    pts["x"], pts["y"] = 320, 240
    pat = np.array([[1, 0], [2, 2]], dtype=np.int32)
    s = np.array([np.float32(np.sqrt(0.75)), 0.0], dtype=np.float32)
    c = np.array([0.5, 1.0], dtype=np.float32)
    f = O.exception_flags(n, oszp, pts, s, c, pat)
    assert f[0] & O.TIE and not f[1] & O.TIE


def test_straddle_flags_at_coarse_octave_border():
    # level 0 keeps 31 px from the border; at octave 3 that is 3 px, so the
    # radius-15 disc and the 13-px pattern leave the octave
    w, h = 1920, 1080
    n, oszp = O.layout(w, h)
    pts = np.zeros(3, dtype=O.ORB_POINT_DTYPE)
    pts["x"] = [31, 960, 960]
    pts["y"] = [540, 540, 31]
    pts["octave"] = [3, 0, 0]
    pat = O.pattern(31, 2)
    s = np.zeros(3, dtype=np.float32)
    c = np.ones(3, dtype=np.float32)
    f = O.exception_flags(n, oszp, pts, s, c, pat)
    assert f[0] & O.STRADDLE_ANGLE and f[0] & O.STRADDLE_DESC
    assert f[1] == 0
    # 31 px from the top at octave 0: the disc (15) and pattern (13) stay inside
    assert not f[2] & (O.STRADDLE_ANGLE | O.STRADDLE_DESC)


@pytest.mark.parametrize("name", PAIRS)
def test_blur_race_count_from_golden(golden, name):
    """Descriptors of the stock reference (in-place blur, orbd.cu:1756) against
    the race-free build: keypoints and angles agree, and the rows that differ
    are counted (they depend on block scheduling)."""
    g = golden(name)
    for img in ("A", "B"):
        rf = g[img + "_points"]
        st = g[img + "_stock_points"]
        o1, o2 = canon_order(rf), canon_order(st)
        assert np.array_equal(rf["x"][o1], st["x"][o2]) and np.array_equal(rf["y"][o1], st["y"][o2])
        assert np.array_equal(rf["angle"][o1].view(np.uint32), st["angle"][o2].view(np.uint32))
        diff = np.any(g[img + "_desc"][o1] != g[img + "_stock_desc"][o2], axis=1)
        print(name, img, "blur-race descriptor rows", int(diff.sum()), "of", len(diff))
        assert O.blur_race_rows(g[img + "_desc"][o1], g[img + "_stock_desc"][o2]) == int(diff.sum())
