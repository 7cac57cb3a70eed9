"""ctypes wrapper of oracle/liborb_oracle.so, the CPU restatement of CUDA-ORB.

TEST INFRASTRUCTURE ONLY: the checker for the sm_100a library.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg may use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborb_oracle.so")
GUARD = 256 * 1024

ORB_POINT_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("octave", "<i4"), ("score", "<f4"),
                            ("angle", "<f4"), ("match", "<i4"), ("distance", "<i4")])

# Floating-point contraction variants of the reference build (nvcc -fmad=true),
# fixed against the reference's own outputs (tests/test_oracle_golden.py):
#  Harris: f(A) - 0.04f*f(B) fused, B converted as unsigned 32-bit (mode 3);
#  blur:   k0*t0 + k1*t1 as fma(k0, t0, k1*t1), then k2, k3 fused (mode 6), both passes;
#  rotate: x*c - y*s as fma(x, c, -(y*s)) and x*s + y*c as fma(x, s, y*c) (mode 1, 1),
#          the same first-product fusing rule; the golden data has no sample that
#          separates the rotation forms.
HARRIS_FMA = 3
BLUR_FMA_H = 6
BLUR_FMA_V = 6
ROT_X = 1
ROT_Y = 1

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oo_fast_atan2.restype = ctypes.c_float
        _lib.oo_fast_atan2.argtypes = [ctypes.c_float, ctypes.c_float]
        _lib.oo_harris_scale.restype = ctypes.c_float
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def threads():
    return int(lib().oo_threads())


def layout(w, h, noctaves=8):
    buf = np.zeros(64, dtype=np.int32)
    n = lib().oo_layout(w, h, noctaves, _p(buf))
    oszp = buf[:5 * n + 1].copy()
    return n, oszp


def split(oszp, n):
    return {"osizes": oszp[0:n], "widths": oszp[n:2 * n], "heights": oszp[2 * n:3 * n],
            "pitchs": oszp[3 * n:4 * n], "offsets": oszp[4 * n:5 * n + 1]}


def guarded(nbytes):
    """Zeroed buffer with GUARD bytes before and after; returns (storage, view)."""
    store = np.zeros(GUARD + nbytes + GUARD, dtype=np.uint8)
    return store, store[GUARD:GUARD + nbytes]


def _gp(store):
    return ctypes.c_void_p(store.ctypes.data + GUARD)


def fast_lut(t):
    lut = np.zeros(512, dtype=np.uint8)
    lib().oo_fast_lut(t, _p(lut))
    return lut


def umax(patch_size=31):
    u = np.zeros(32, dtype=np.int32)
    lib().oo_umax(patch_size, _p(u))
    return u[:patch_size // 2 + 2].copy()


def gauss_kernel():
    k = np.zeros(4, dtype=np.float32)
    lib().oo_gauss_kernel(_p(k))
    return k


def pattern(patch_size=31, wta_k=2):
    buf = np.zeros(1024, dtype=np.int32)
    cnt = lib().oo_pattern(patch_size, wta_k, _p(buf))
    return buf[:2 * cnt].reshape(cnt, 2).copy()


def fast_atan2(y, x):
    return lib().oo_fast_atan2(float(y), float(x))


def pyramid(img, w, h, n, oszp):
    lay = split(oszp, n)
    store, view = guarded(int(lay["offsets"][-1]))
    img = np.ascontiguousarray(img)
    lib().oo_pyramid(_p(img), int(lay["pitchs"][0]), _gp(store), _p(oszp), n)
    return store, view


def score_map(pyr_store, n, oszp, threshold=20, harris=True, harris_fma=None):
    lay = split(oszp, n)
    npx = int(lay["osizes"][0])
    vmap = np.zeros(npx, dtype=np.float32)
    layer = np.zeros(npx, dtype=np.int32)
    hf = HARRIS_FMA if harris_fma is None else harris_fma
    lib().oo_score_map(_gp(pyr_store), _p(oszp), n, threshold, int(harris), hf, _p(vmap), _p(layer))
    return vmap, layer


def nms(vmap, layer, n, oszp, border=31, cap=1 << 22):
    out = np.zeros(cap, dtype=ORB_POINT_DTYPE)
    cnt = lib().oo_nms(_p(vmap), _p(layer), _p(oszp), n, border, _p(out), cap)
    return out[:min(cnt, cap)].copy(), cnt


def angle(pyr_store, n, oszp, pts, patch_size=31):
    pts = np.ascontiguousarray(pts)
    lib().oo_angle(_gp(pyr_store), _p(oszp), n, _p(pts), len(pts), patch_size)
    return pts


def blur(pyr_store, n, oszp, fma_h=None, fma_v=None):
    lay = split(oszp, n)
    store, view = guarded(int(lay["offsets"][-1]))
    lib().oo_blur(_gp(pyr_store), _gp(store), _p(oszp), n, BLUR_FMA_H if fma_h is None else fma_h,
                  BLUR_FMA_V if fma_v is None else fma_v)
    return store, view


def describe(blur_store, n, oszp, pts, sinv, cosv, pat=None, wta_k=2, rot_x=None, rot_y=None):
    if pat is None:
        pat = pattern(31, wta_k)
    pat = np.ascontiguousarray(pat, dtype=np.int32)
    pts = np.ascontiguousarray(pts)
    desc = np.zeros((len(pts), 32), dtype=np.uint8)
    s = np.ascontiguousarray(sinv, dtype=np.float32)
    c = np.ascontiguousarray(cosv, dtype=np.float32)
    lib().oo_describe(_gp(blur_store), _p(oszp), n, _p(pts), len(pts), _p(s), _p(c), _p(pat), wta_k,
                      ROT_X if rot_x is None else rot_x, ROT_Y if rot_y is None else rot_y, _p(desc))
    return desc


def sincos_host(angles):
    """libm sin/cos stand-in for the GPU's __sinf/__cosf when no GPU values are given."""
    a = np.asarray(angles, dtype=np.float32)
    return np.sin(a.astype(np.float64)).astype(np.float32), np.cos(a.astype(np.float64)).astype(np.float32)


def match(d1, d2):
    d1 = np.ascontiguousarray(d1, dtype=np.uint8)
    d2 = np.ascontiguousarray(d2, dtype=np.uint8)
    m = np.zeros(max(len(d1), 1), dtype=np.int32)
    d = np.zeros(max(len(d1), 1), dtype=np.int32)
    lib().oo_match(_p(d1), len(d1), _p(d2) if len(d2) else None, len(d2), _p(m), _p(d))
    return m[:len(d1)], d[:len(d1)]


def knn2(q, db):
    q = np.ascontiguousarray(q, dtype=np.uint8)
    db = np.ascontiguousarray(db, dtype=np.uint8)
    dist = np.zeros((max(len(q), 1), 2), dtype=np.uint32)
    idx = np.zeros((max(len(q), 1), 2), dtype=np.int32)
    lib().oo_knn2(_p(q), len(q), _p(db) if len(db) else None, len(db), _p(dist), _p(idx))
    return dist[:len(q)], idx[:len(q)]


def detect_and_compute(img, w, h, noctaves=8, edge=31, wta_k=2, harris=True, patch=31, fast_thr=20,
                       max_pts=10000, sincos=None):
    """Whole per-image pipeline.  Returns points in raster order (the first
    max_pts survivors), descriptors, and the total survivor count.  sincos(angles)
    supplies the GPU __sinf/__cosf values; the libm stand-in is used otherwise."""
    n, oszp = layout(w, h, noctaves)
    if n <= 0:
        raise ValueError("image too small")
    pyr_store, _ = pyramid(img, w, h, n, oszp)
    vmap, layer = score_map(pyr_store, n, oszp, fast_thr, harris)
    pts, total = nms(vmap, layer, n, oszp, edge, cap=max(max_pts, 1))
    pts = pts[:max_pts]
    pts = angle(pyr_store, n, oszp, pts, patch)
    bstore, _ = blur(pyr_store, n, oszp)
    s, c = (sincos or sincos_host)(pts["angle"])
    pat = pattern(patch, wta_k)
    desc = describe(bstore, n, oszp, pts, s, c, pat, wta_k)
    return {"points": pts, "desc": desc, "total": total, "n": n, "oszp": oszp, "sin": s, "cos": c}


# ---------------------------------------------------------------------------
# FP64 side-oracle and the exception counts of the parity report.
# ---------------------------------------------------------------------------

# Tolerances of the FP64 comparison.  Harris: 1e-5 relative, plus an absolute
# floor for the cancellation of A - 0.04 B.  The float path rounds A and B to
# 24 bits before they cancel, so its absolute error is below
# 2^-22 * (|A| + 0.04 B) * scale^4 (four times the rounding of the two terms);
# over every possible int32 term pair that is at most HARRIS_ABS_FLOOR.
# Angle: 1e-5 relative with an absolute floor of 2^-20 rad (four float ulps of
# pi); the folds pi/2 - r and pi - r never cancel (r <= pi/4 and r <= pi/2).
FP64_REL_TOL = 1e-5
HARRIS_TERM_FLOOR = 2.0 ** -22
HARRIS_ABS_FLOOR = 2.0 ** -22 * (2.0 ** 31 + 0.04 * 2.0 ** 32) * (1.0 / (4 * 7 * 255.0)) ** 4
ANGLE_ABS_FLOOR = 2.0 ** -20
TIE_EPS = 1e-4
TIE, STRADDLE_ANGLE, STRADDLE_DESC = 1, 2, 4


def harris_f64(pyr_store, n, oszp, pts):
    """FP64 Harris at each keypoint; returns (score, |A| scale^4, 0.04 B scale^4)."""
    pts = np.ascontiguousarray(pts)
    score = np.zeros(max(len(pts), 1), dtype=np.float64)
    terms = np.zeros((max(len(pts), 1), 2), dtype=np.float64)
    lib().oo_harris_f64(_gp(pyr_store), _p(oszp), n, _p(pts), len(pts), _p(score), _p(terms))
    return score[:len(pts)], terms[:len(pts), 0], terms[:len(pts), 1]


def angle_f64(pyr_store, n, oszp, pts, patch_size=31):
    pts = np.ascontiguousarray(pts)
    ang = np.zeros(max(len(pts), 1), dtype=np.float64)
    lib().oo_angle_f64(_gp(pyr_store), _p(oszp), n, _p(pts), len(pts), patch_size, _p(ang))
    return ang[:len(pts)]


def exception_flags(n, oszp, pts, sinv, cosv, pat, patch_size=31, tie_eps=TIE_EPS):
    pts = np.ascontiguousarray(pts)
    pat = np.ascontiguousarray(pat, dtype=np.int32)
    s = np.ascontiguousarray(sinv, dtype=np.float32)
    c = np.ascontiguousarray(cosv, dtype=np.float32)
    flags = np.zeros(max(len(pts), 1), dtype=np.int32)
    lib().oo_exception_flags(_p(oszp), n, _p(pts), len(pts), _p(s), _p(c), _p(pat), len(pat), patch_size,
                             ctypes.c_double(tie_eps), _p(flags))
    return flags[:len(pts)]


def fp64_check(img, w, h, pts, sinv, cosv, noctaves=8, patch=31, wta_k=2, harris=True):
    """Compare GPU keypoint scores and angles (float32) with the FP64 side-oracle
    and count the keypoints the parity report lists.  Returns a dict of counts and
    the largest relative errors; 'harris_fail' and 'angle_fail' count keypoints
    outside tolerance (rel 1e-5 or the absolute floor)."""
    n, oszp = layout(w, h, noctaves)
    pyr_store, _ = pyramid(img, w, h, n, oszp)
    pts = np.ascontiguousarray(pts)
    out = {"keypoints": int(len(pts))}
    if harris:
        s64, ta, tb = harris_f64(pyr_store, n, oszp, pts)
        g = pts["score"].astype(np.float64)
        err = np.abs(g - s64)
        rel_ok = err <= FP64_REL_TOL * np.abs(s64)
        ok = err <= FP64_REL_TOL * np.abs(s64) + HARRIS_ABS_FLOOR
        # the per-keypoint bound the fixed floor comes from, checked too
        term_ok = err <= FP64_REL_TOL * np.abs(s64) + HARRIS_TERM_FLOOR * (ta + tb)
        rel = np.where(s64 != 0, err / np.maximum(np.abs(s64), 1e-300), 0.0)
        out.update(harris_fail=int((~ok).sum()), harris_needs_floor=int((ok & ~rel_ok).sum()),
                   harris_term_bound_fail=int((~term_ok).sum()),
                   harris_max_rel=float(rel[rel_ok].max()) if rel_ok.any() else 0.0,
                   harris_max_abs=float(err.max()) if len(err) else 0.0)
    a64 = angle_f64(pyr_store, n, oszp, pts, patch)
    ga = pts["angle"].astype(np.float64)
    both_nan = np.isnan(ga) & np.isnan(a64)
    aerr = np.where(both_nan, 0.0, np.abs(ga - a64))
    arel_ok = both_nan | (aerr <= FP64_REL_TOL * np.abs(a64))
    aok = both_nan | (aerr <= FP64_REL_TOL * np.abs(a64) + ANGLE_ABS_FLOOR)
    arel = np.where(np.abs(a64) > 0, aerr / np.maximum(np.abs(a64), 1e-300), 0.0)
    out.update(angle_fail=int((~aok).sum()), angle_needs_floor=int((aok & ~arel_ok).sum()),
               angle_max_rel=float(np.nanmax(arel[arel_ok])) if arel_ok.any() else 0.0,
               angle_max_abs=float(np.nanmax(aerr)) if len(aerr) else 0.0, angle_nan=int(both_nan.sum()))
    flags = exception_flags(n, oszp, pts, sinv, cosv, pattern(patch, wta_k), patch)
    out.update(rounding_tie=int(((flags & TIE) != 0).sum()),
               straddle_angle=int(((flags & STRADDLE_ANGLE) != 0).sum()),
               straddle_desc=int(((flags & STRADDLE_DESC) != 0).sum()),
               straddle_any=int(((flags & (STRADDLE_ANGLE | STRADDLE_DESC)) != 0).sum()))
    out["flags"] = flags
    return out


def blur_race_rows(desc_race_free, desc_stock):
    """Descriptor rows (same keypoint order) that differ between the race-free
    build and the stock reference, whose in-place blur (orbd.cu:1756) lets
    neighbouring blocks overwrite halo pixels before they are read."""
    a = np.asarray(desc_race_free)
    b = np.asarray(desc_stock)
    if len(a) == 0:
        return 0
    return int(np.any(a != b, axis=1).sum())
