"""ctypes wrapper of oracle/_ref/libref_orb.so (the reference CUDA-ORB build).

TEST INFRASTRUCTURE: used by tests/, tests/golden/make_golden.py and the
reference arm of bench.py only.  The library is the reference's own orbd.cu and
orb.cpp compiled for sm_100a plus oracle/ref_harness.cu; it runs on a GPU.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_orb.so")

# OrbPoint (orb_structures.h:8-17): int x, y, octave; float score, angle; int match, distance.
ORB_POINT_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("octave", "<i4"), ("score", "<f4"),
                            ("angle", "<f4"), ("match", "<i4"), ("distance", "<i4")])

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference build missing: {LIB_PATH} (run `make -C oracle ref`)")
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def align_up(a, b):
    return (a + b - 1) // b * b


_state = {"noctaves": 8}


def init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1, max_pts=10000):
    _check(lib().ref_init(noctaves, edge, wta_k, score_type, patch, fast_thr, retain_topn, max_pts), "ref_init")
    _state["noctaves"] = noctaves
    return max_pts


def layout():
    n = ctypes.c_int(0)
    buf = np.zeros(64, dtype=np.int32)
    cnt = lib().ref_layout(ctypes.byref(n), _p(buf), 64)
    no = n.value
    osz = buf[:cnt]
    return {"n": no, "osizes": osz[0:no].copy(), "widths": osz[no:2 * no].copy(),
            "heights": osz[2 * no:3 * no].copy(), "pitchs": osz[3 * no:4 * no].copy(),
            "offsets": osz[4 * no:5 * no + 1].copy()}


def detect(slot, img, w, h, max_pts):
    """Stock Orbor::detectAndCompute. img: uint8 (h, align_up(w,128))."""
    img = np.ascontiguousarray(img)
    pts = np.zeros(max_pts, dtype=ORB_POINT_DTYPE)
    desc = np.zeros((max_pts, 32), dtype=np.uint8)
    n = ctypes.c_int(0)
    raw = ctypes.c_uint(0)
    _check(lib().ref_detect(slot, _p(img), w, h, ctypes.byref(n), ctypes.byref(raw), _p(pts), _p(desc)), "ref_detect")
    k = n.value
    return {"num_pts": k, "raw_counter": raw.value, "points": pts[:k].copy(), "desc": desc[:k].copy()}


def match_slots(n1):
    m = np.zeros(max(n1, 1), dtype=np.int32)
    d = np.zeros(max(n1, 1), dtype=np.int32)
    _check(lib().ref_match_slots(_p(m), _p(d)), "ref_match_slots")
    return m[:n1], d[:n1]


def stages(img, w, h, max_pts, race_free=True):
    """Lower-API pipeline with intermediate dumps (see ref_harness.cu:ref_stages)."""
    img = np.ascontiguousarray(img)
    lay = layout_for(w, h, noctaves=_state["noctaves"])
    obytes = int(lay["offsets"][-1])
    vbytes = int(lay["osizes"][0]) * 8
    pyr_raw = np.zeros(obytes, dtype=np.uint8)
    pyr_blur = np.zeros(obytes, dtype=np.uint8)
    vmem = np.zeros(vbytes // 4, dtype=np.float32)
    pts = np.zeros(max_pts, dtype=ORB_POINT_DTYPE)
    desc = np.zeros((max_pts, 32), dtype=np.uint8)
    sinv = np.zeros(max_pts, dtype=np.float32)
    cosv = np.zeros(max_pts, dtype=np.float32)
    sizes = np.zeros(3, dtype=np.int64)
    n = ctypes.c_int(0)
    raw = ctypes.c_uint(0)
    _check(lib().ref_stages(_p(img), w, h, int(race_free), ctypes.byref(n), ctypes.byref(raw), _p(pyr_raw),
                            _p(vmem), _p(pyr_blur), _p(pts), _p(desc), _p(sinv), _p(cosv), _p(sizes)),
           "ref_stages")
    assert sizes[0] == obytes and sizes[1] == vbytes, (sizes, obytes, vbytes)
    k = n.value
    npx = int(lay["osizes"][0])
    return {"num_pts": k, "raw_counter": raw.value, "pyr_raw": pyr_raw, "pyr_blur": pyr_blur,
            "vmap": vmem[:npx].copy(), "layer": vmem[npx:].view(np.int32).copy(),
            "points": pts[:k].copy(), "desc": desc[:k].copy(), "sin": sinv[:k].copy(), "cos": cosv[:k].copy(),
            "layout": lay}


def layout_for(w, h, noctaves=8):
    """Pyramid layout as Orbor::updateParam computes it (orb.cpp:145-191)."""
    m = min(w, h) // 80
    # (int)log2f(m) + 1: the integer part of log2 of a small positive int
    no = min(noctaves, m.bit_length()) if m > 0 else 0
    widths, heights, pitchs, osizes, offsets = [w], [h], [align_up(w, 128)], [], [0]
    for j in range(1, no):
        widths.append(widths[-1] >> 1)
        heights.append(heights[-1] >> 1)
        pitchs.append(align_up(widths[-1], 128))
    for j in range(no):
        osizes.append(heights[j] * pitchs[j])
        offsets.append(offsets[-1] + osizes[-1])
    return {"n": no, "osizes": np.array(osizes), "widths": np.array(widths), "heights": np.array(heights),
            "pitchs": np.array(pitchs), "offsets": np.array(offsets)}


def sincos(angles):
    a = np.ascontiguousarray(angles, dtype=np.float32)
    s = np.zeros_like(a)
    c = np.zeros_like(a)
    _check(lib().ref_sincos(_p(a), len(a), _p(s), _p(c)), "ref_sincos")
    return s, c


def hmatch(d1, d2):
    d1 = np.ascontiguousarray(d1, dtype=np.uint8)
    d2 = np.ascontiguousarray(d2, dtype=np.uint8)
    n1, n2 = len(d1), len(d2)
    m = np.zeros(max(n1, 1), dtype=np.int32)
    d = np.zeros(max(n1, 1), dtype=np.int32)
    _check(lib().ref_hmatch(_p(d1), n1, _p(d2) if n2 else None, n2, _p(m), _p(d)), "ref_hmatch")
    return m[:n1], d[:n1]


def time_pair(a, b, w, h, warmup, iters):
    ms = ctypes.c_float(0)
    na = ctypes.c_int(0)
    nb = ctypes.c_int(0)
    _check(lib().ref_time_pair(_p(np.ascontiguousarray(a)), _p(np.ascontiguousarray(b)), w, h, warmup, iters,
                               ctypes.byref(ms), ctypes.byref(na), ctypes.byref(nb)), "ref_time_pair")
    return ms.value, na.value, nb.value


def time_hmatch(d1, d2, warmup, iters):
    ms = ctypes.c_float(0)
    d1 = np.ascontiguousarray(d1, dtype=np.uint8)
    d2 = np.ascontiguousarray(d2, dtype=np.uint8)
    _check(lib().ref_time_hmatch(_p(d1), len(d1), _p(d2), len(d2), warmup, iters, ctypes.byref(ms)),
           "ref_time_hmatch")
    return ms.value
