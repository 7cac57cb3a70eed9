"""Python binding of liborbx.so (include/orbx.h), the sm_100a ORB library.

Device memory comes from torch tensors; the library itself is the CUDA code in
csrc/.  There is no CPU path: if the shared library is missing or fails to
load, import raises.

Keypoints are int32 tensors of shape (max_pts, 7) laid out as orb::OrbPoint
(x, y, octave, score, angle, match, distance; score and angle are float32 bits).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# ORBX_CHECKED=1 loads the bounds-checked build (build.py --checked) instead:
# same entry points, each kernel access tested against its buffer's extent.
CHECKED = os.environ.get("ORBX_CHECKED", "0") == "1"
LIB_PATH = os.path.join(HERE, "liborbx_checked.so" if CHECKED else "liborbx.so")

ORBX_OK = 0
ORBX_ERR_ARG, ORBX_ERR_CUDA, ORBX_ERR_SIZE, ORBX_ERR_STATE, ORBX_ERR_TIMEOUT, ORBX_ERR_NOMEM = 1, 2, 3, 4, 5, 6
MATCH_POPC = 0
MATCH_IMMA = 1
MATCH_AUTO = 2
HARRIS_SCORE = 0
FAST_SCORE = 1

POINT_FIELDS = ("x", "y", "octave", "score", "angle", "match", "distance")
ORB_POINT_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("octave", "<i4"), ("score", "<f4"),
                            ("angle", "<f4"), ("match", "<i4"), ("distance", "<i4")])


class OrbxError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


class Params(ctypes.Structure):
    _fields_ = [("noctaves", ctypes.c_int), ("edge_threshold", ctypes.c_int), ("wta_k", ctypes.c_int),
                ("score_type", ctypes.c_int), ("patch_size", ctypes.c_int), ("fast_threshold", ctypes.c_int),
                ("retain_topn", ctypes.c_int), ("max_pts", ctypes.c_int)]


class Image(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("w", ctypes.c_int), ("h", ctypes.c_int), ("pitch", ctypes.c_int)]


class FrameOut(ctypes.Structure):
    _fields_ = [("points", ctypes.c_void_p), ("desc", ctypes.c_void_p), ("num_pts", ctypes.c_void_p),
                ("max_pts", ctypes.c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("nms_rows", ctypes.c_int), ("describe_blocks_per_sm", ctypes.c_int),
                ("match_blocks_per_sm", ctypes.c_int), ("match_blocks_per_pair", ctypes.c_int),
                ("batch_form", ctypes.c_int), ("persist_group", ctypes.c_int),
                ("persist_blocks_per_sm", ctypes.c_int), ("wait_timeout_us", ctypes.c_int),
                ("upload_bands", ctypes.c_int), ("pair_form", ctypes.c_int), ("pyr_tile", ctypes.c_int),
                ("persist_row_deps", ctypes.c_int), ("host_overlap", ctypes.c_int)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{os.path.basename(LIB_PATH)} not built: run "
                              f"`python {os.path.join(HERE, 'build.py')}{' --checked' if CHECKED else ''}`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32 = ctypes.c_void_p, ctypes.c_int
        L.orbx_version.restype = ctypes.c_char_p
        L.orbx_status_string.restype = ctypes.c_char_p
        L.orbx_status_string.argtypes = [i32]
        L.orbx_create.argtypes = [ctypes.POINTER(vp), i32]
        L.orbx_destroy.argtypes = [vp]
        L.orbx_set_stream.argtypes = [vp, vp]
        L.orbx_get_stream.argtypes = [vp]
        L.orbx_get_stream.restype = vp
        L.orbx_sync.argtypes = [vp]
        L.orbx_default_params.argtypes = [ctypes.POINTER(Params)]
        L.orbx_init.argtypes = [vp, ctypes.POINTER(Params)]
        L.orbx_layout.argtypes = [i32, i32, i32, vp, i32]
        L.orbx_detect_and_compute.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp, i32]
        L.orbx_match.argtypes = [vp, vp, vp, vp, vp, vp, i32, i32, i32]
        L.orbx_match_knn2.argtypes = [vp, vp, i32, vp, i32, vp, vp, i32]
        L.orbx_match_knn2_static.argtypes = [vp, i32, vp, i32, vp, vp, vp]
        L.orbx_pair.argtypes = [vp, vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32]
        L.orbx_debug_buffers.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orbx_pair_host.argtypes = [vp, vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32]
        L.orbx_profile_pair_host.argtypes = [vp, vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32, vp]
        L.orbx_profile_pair.argtypes = [vp, vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32, vp]
        L.orbx_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.orbx_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.orbx_batch_pairs.argtypes = [vp, i32, ctypes.POINTER(Image), ctypes.POINTER(Image),
                                       ctypes.POINTER(FrameOut), ctypes.POINTER(FrameOut), i32]
        L.orbx_autotune_pairs.argtypes = [vp, i32, ctypes.POINTER(Image), ctypes.POINTER(Image),
                                          ctypes.POINTER(FrameOut), ctypes.POINTER(FrameOut), i32,
                                          ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_float)]
        L.orbx_autotune_pairs_forms.argtypes = [vp, i32, ctypes.POINTER(Image), ctypes.POINTER(Image),
                                                ctypes.POINTER(FrameOut), ctypes.POINTER(FrameOut), i32, i32,
                                                ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_float)]
        L.orbx_selftest_wait_timeout.argtypes = [vp, i32]
        L.orbx_bounds_checked.argtypes = []
        L.orbx_bounds_report.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.orbx_bounds_set_slack.argtypes = [vp, ctypes.c_longlong]
        L.orbx_profile_batch.argtypes = [vp, i32, ctypes.POINTER(Image), ctypes.POINTER(Image),
                                         ctypes.POINTER(FrameOut), ctypes.POINTER(FrameOut), vp]
        L.orbx_learned_default_params.argtypes = [ctypes.POINTER(LearnedParams)]
        L.orbx_learned_build.argtypes = [vp, ctypes.POINTER(LearnedParams), vp, i32, vp, i32, ctypes.POINTER(vp)]
        L.orbx_learned_search.argtypes = [vp, vp, vp, i32, vp, vp, vp, vp]
        L.orbx_learned_set_margin.argtypes = [vp, ctypes.c_float]
        L.orbx_learned_set_max_distance.argtypes = [vp, i32]
        L.orbx_learned_set_rerank.argtypes = [vp, i32]
        L.orbx_learned_probe_pairs.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_ulonglong)]
        L.orbx_learned_profile_search.argtypes = [vp, vp, vp, i32, vp, vp, vp]
        L.orbx_learned_get_stats.argtypes = [vp, ctypes.POINTER(LearnedStats)]
        L.orbx_learned_export.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        L.orbx_learned_gradients.argtypes = [vp, vp, vp, vp, i32, vp, vp, vp, vp, vp]
        L.orbx_learned_save.argtypes = [vp, vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.orbx_learned_load.argtypes = [vp, vp, ctypes.c_size_t, vp, i32, ctypes.POINTER(vp)]
        L.orbx_learned_get_params.argtypes = [vp, ctypes.POINTER(LearnedParams)]
        L.orbx_learned_destroy.argtypes = [vp]
        L.orbx_gemm_bf16.argtypes = [vp, vp, vp, i32, i32, i32, vp, i32, i32, vp, vp]
        L.orbx_upload_image.argtypes = [vp, vp, i32, i32, i32, vp, i32]
        L.orbx_ocv_default_params.argtypes = [ctypes.POINTER(OcvParams)]
        L.orbx_ocv_detect_and_compute.argtypes = [vp, ctypes.POINTER(OcvParams), vp, i32, i32, i32, vp, vp, vp, i32]
        L.orbx_download_points.argtypes = [vp, vp, i32, vp, i32]
        L.orbx_selftest_pi_minus.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.orbx_selftest_pi_minus.restype = ctypes.c_longlong
        _lib = L
    return _lib


FIELDS_KEYPOINT, FIELDS_MATCH = 1, 2
class OcvParams(ctypes.Structure):
    _fields_ = [("nfeatures", ctypes.c_int), ("scale_factor", ctypes.c_float), ("nlevels", ctypes.c_int),
                ("edge_threshold", ctypes.c_int), ("score_type", ctypes.c_int), ("patch_size", ctypes.c_int),
                ("fast_threshold", ctypes.c_int)]


OCV_KEYPOINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("size", "<f4"), ("angle", "<f4"),
                               ("response", "<f4"), ("octave", "<i4")])


def ocv_params(**kw):
    p = OcvParams()
    _check(lib().orbx_ocv_default_params(ctypes.byref(p)), "orbx_ocv_default_params")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def ocv_detect_and_compute(ctx, img, w, h, params=None, cap=None):
    """OpenCV-compatible mode on a uint8 CUDA image (h, pitch).  Returns host
    (keypoints as OCV_KEYPOINT_DTYPE, descriptors (n, 32) uint8)."""
    torch = _torch()
    params = params if params is not None else ocv_params()
    cap = cap if cap is not None else params.nfeatures
    kps = torch.zeros((cap, 6), dtype=torch.int32, device=img.device)
    desc = torch.zeros((cap, 32), dtype=torch.uint8, device=img.device)
    n = torch.zeros(1, dtype=torch.int32, device=img.device)
    _check(lib().orbx_ocv_detect_and_compute(ctx.h, ctypes.byref(params), _ptr(img), w, h, img.shape[1], _ptr(kps),
                                             _ptr(desc), _ptr(n), cap), "orbx_ocv_detect_and_compute")
    ctx.sync()
    k = int(n.item())
    return kps[:k].cpu().numpy().copy().view(OCV_KEYPOINT_DTYPE).reshape(k), desc[:k].cpu().numpy().copy()


PROPOSAL_MLP, PROPOSAL_LSH = 0, 1
RERANK_TENSOR, RERANK_POPC = 0, 1
LABEL_NEAREST, LABEL_LISTED = 0, 1
INIT_CENTROIDS, INIT_RANDOM = 0, 1
GEMM_F32, GEMM_BIAS_RELU_BF16, GEMM_MASK_BF16, GEMM_BF16, GEMM_TOP8, GEMM_TOP8_ROW = 0, 1, 2, 3, 4, 5


def gemm_top_lists(n):
    """Key lists per row of GEMM_TOP8_ROW for n columns."""
    return 4 if (n // 256) % 2 == 0 else 2


class LearnedParams(ctypes.Structure):
    _fields_ = [("proposal", ctypes.c_int), ("n_clusters", ctypes.c_int), ("hidden", ctypes.c_int),
                ("n_probe", ctypes.c_int), ("kmeans_iters", ctypes.c_int), ("epochs", ctypes.c_int),
                ("batch", ctypes.c_int), ("lr", ctypes.c_float), ("margin", ctypes.c_float),
                ("lsh_bits", ctypes.c_int), ("seed", ctypes.c_ulonglong), ("max_distance", ctypes.c_int),
                ("spill", ctypes.c_int), ("init", ctypes.c_int), ("synth_train", ctypes.c_int),
                ("flip_lo", ctypes.c_float), ("flip_hi", ctypes.c_float), ("rerank", ctypes.c_int),
                ("label_mode", ctypes.c_int)]


class LearnedStats(ctypes.Structure):
    _fields_ = [("kmeans_iters_run", ctypes.c_int), ("kmeans_last_moved", ctypes.c_int),
                ("largest_cluster", ctypes.c_int), ("epochs_run", ctypes.c_int),
                ("loss", ctypes.c_float * 64), ("accuracy", ctypes.c_float * 64), ("build_ms", ctypes.c_float * 4)]

    def to_dict(self):
        e = self.epochs_run
        return {"kmeans_iters": self.kmeans_iters_run, "kmeans_last_moved": self.kmeans_last_moved,
                "largest_cluster": self.largest_cluster, "epochs": e,
                "loss": [round(float(x), 4) for x in self.loss[:e]],
                "accuracy": [round(float(x), 4) for x in self.accuracy[:e]],
                "build_ms": {k: round(float(v), 2) for k, v in zip(("cluster", "labels", "train", "total"),
                                                                    self.build_ms)}}


def learned_params(**kw):
    p = LearnedParams()
    _check(lib().orbx_learned_default_params(ctypes.byref(p)), "orbx_learned_default_params")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def status_string(status):
    return lib().orbx_status_string(int(status)).decode()


def version():
    return lib().orbx_version().decode()


def _check(status, what):
    if status != ORBX_OK:
        raise OrbxError(status, what)


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def layout(w, h, noctaves=8):
    buf = np.zeros(64, dtype=np.int32)
    n = lib().orbx_layout(w, h, noctaves, buf.ctypes.data, 64)
    if n < 0:
        raise OrbxError(-n, "orbx_layout")
    return n, buf[:5 * n + 1].copy()


def default_params():
    p = Params()
    _check(lib().orbx_default_params(ctypes.byref(p)), "orbx_default_params")
    return p


def make_params(noctaves=8, edge_threshold=31, wta_k=2, score_type=HARRIS_SCORE, patch_size=31, fast_threshold=20,
                retain_topn=-1, max_pts=10000):
    return Params(noctaves, edge_threshold, wta_k, score_type, patch_size, fast_threshold, retain_topn, max_pts)


class Context:
    """An orbx context: tables, workspaces and a CUDA stream on one device."""

    def __init__(self, device=0, params=None, stream=None):
        h = ctypes.c_void_p()
        _check(lib().orbx_create(ctypes.byref(h), device), "orbx_create")
        self.h = h
        self.device = device
        self.params = None
        if stream is not None:
            self.set_stream(stream)
        if params is not None:
            self.init(params)

    def close(self):
        if self.h:
            lib().orbx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _check(lib().orbx_set_stream(self.h, handle), "orbx_set_stream")

    @property
    def stream_handle(self):
        return lib().orbx_get_stream(self.h)

    def init(self, params):
        _check(lib().orbx_init(self.h, ctypes.byref(params)), "orbx_init")
        self.params = params

    def sync(self):
        _check(lib().orbx_sync(self.h), "orbx_sync")

    # -- raw pointer entry points -------------------------------------------
    def detect_and_compute_ptr(self, d_img, w, h, pitch, d_points, d_desc, d_count, compute_desc=True):
        _check(lib().orbx_detect_and_compute(self.h, _ptr(d_img), w, h, pitch, _ptr(d_points), _ptr(d_desc),
                                             _ptr(d_count), int(bool(compute_desc))), "orbx_detect_and_compute")

    def match_ptr(self, d_points1, d_n1, d_desc1, d_n2, d_desc2, n1_cap, n2_cap, mode=MATCH_POPC):
        _check(lib().orbx_match(self.h, _ptr(d_points1), _ptr(d_n1), _ptr(d_desc1), _ptr(d_n2), _ptr(d_desc2),
                                n1_cap, n2_cap, mode), "orbx_match")

    def upload_image(self, h_img, w, h, h_pitch, d_img, d_pitch):
        """h_img: numpy uint8 array or pinned torch tensor (h, h_pitch); d_img: CUDA tensor (h, d_pitch)."""
        hp = h_img.ctypes.data if hasattr(h_img, "ctypes") else h_img.data_ptr()
        _check(lib().orbx_upload_image(self.h, hp, w, h, h_pitch, _ptr(d_img), d_pitch), "orbx_upload_image")

    def download_points(self, d_pts, n, h_pts, fields=3):
        """h_pts: numpy array of ORB_POINT_DTYPE (updated in place, other fields kept)."""
        _check(lib().orbx_download_points(self.h, _ptr(d_pts), n, h_pts.ctypes.data, fields), "orbx_download_points")

    def knn2_ptr(self, d_q, nq, d_db, ndb, d_dist2, d_idx2, mode=MATCH_POPC):
        _check(lib().orbx_match_knn2(self.h, _ptr(d_q), nq, _ptr(d_db), ndb, _ptr(d_dist2), _ptr(d_idx2), mode),
               "orbx_match_knn2")

    def pair_ptr(self, d_a, d_b, w, h, pitch, pa, da, na, pb, db, nb, mode=MATCH_POPC):
        _check(lib().orbx_pair(self.h, _ptr(d_a), _ptr(d_b), w, h, pitch, _ptr(pa), _ptr(da), _ptr(na), _ptr(pb),
                               _ptr(db), _ptr(nb), mode), "orbx_pair")

    def pair_host(self, a, b, w, h, pitch, pts_a, n_a, pts_b, n_b, desc_a=None, desc_b=None, mode=MATCH_POPC):
        """Host-buffer pair call; a/b/pts/n/desc are host pointers (ints) or numpy arrays."""
        def hp(x):
            if x is None or isinstance(x, int):
                return x
            if hasattr(x, "ctypes"):
                return x.ctypes.data
            return x.data_ptr()
        _check(lib().orbx_pair_host(self.h, hp(a), hp(b), w, h, pitch, hp(pts_a), hp(n_a), hp(pts_b), hp(n_b),
                                    hp(desc_a), hp(desc_b), mode), "orbx_pair_host")

    def profile_pair_host(self, a, b, w, h, pitch, pts_a, n_a, pts_b, n_b, desc_a=None, desc_b=None,
                          mode=MATCH_POPC):
        """orbx_pair_host with phase times: dict of ms (events: upload, kernels, export
        ends from the start; host: enqueue, wait, copy-out, wall)."""
        def hp(x):
            if x is None or isinstance(x, int):
                return x
            if hasattr(x, "ctypes"):
                return x.ctypes.data
            return x.data_ptr()
        ms = np.zeros(7, dtype=np.float32)
        _check(lib().orbx_profile_pair_host(self.h, hp(a), hp(b), w, h, pitch, hp(pts_a), hp(n_a), hp(pts_b),
                                            hp(n_b), hp(desc_a), hp(desc_b), mode,
                                            ms.ctypes.data_as(ctypes.c_void_p)), "orbx_profile_pair_host")
        keys = ("upload_end", "kernels_end", "export_end", "host_enqueue", "host_wait", "host_copy_out",
                "host_wall")
        return {k: float(v) for k, v in zip(keys, ms)}

    def profile_pair(self, d_a, d_b, w, h, pitch, pa, da, na, pb, db, nb, mode=MATCH_POPC):
        ms = np.zeros(5, dtype=np.float32)
        _check(lib().orbx_profile_pair(self.h, _ptr(d_a), _ptr(d_b), w, h, pitch, _ptr(pa), _ptr(da), _ptr(na),
                                       _ptr(pb), _ptr(db), _ptr(nb), mode, ms.ctypes.data), "orbx_profile_pair")
        return ms

    def get_tuning(self):
        t = Tuning()
        _check(lib().orbx_get_tuning(self.h, ctypes.byref(t)), "orbx_get_tuning")
        return t

    def set_tuning(self, t):
        _check(lib().orbx_set_tuning(self.h, ctypes.byref(t)), "orbx_set_tuning")

    def batch_pairs(self, batch, mode=MATCH_POPC):
        """batch: a PairBatch (device images and outputs).  Asynchronous."""
        _check(lib().orbx_batch_pairs(self.h, batch.n, batch.ia, batch.ib, batch.oa, batch.ob, mode),
               "orbx_batch_pairs")

    def profile_batch(self, batch):
        ms = np.zeros(5, dtype=np.float32)
        _check(lib().orbx_profile_batch(self.h, batch.n, batch.ia, batch.ib, batch.oa, batch.ob, ms.ctypes.data),
               "orbx_profile_batch")
        return ms

    def autotune_pairs(self, batch, reps=3):
        t = Tuning()
        ms = ctypes.c_float(0)
        _check(lib().orbx_autotune_pairs(self.h, batch.n, batch.ia, batch.ib, batch.oa, batch.ob, reps,
                                         ctypes.byref(t), ctypes.byref(ms)), "orbx_autotune_pairs")
        return t, ms.value

    def autotune_pairs_forms(self, batch, forms, reps=3):
        """forms: 1 = five launches, 2 = persistent, 3 = both."""
        t = Tuning()
        ms = ctypes.c_float(0)
        _check(lib().orbx_autotune_pairs_forms(self.h, batch.n, batch.ia, batch.ib, batch.oa, batch.ob, reps, forms,
                                               ctypes.byref(t), ctypes.byref(ms)), "orbx_autotune_pairs_forms")
        return t, ms.value

    def selftest_wait_timeout(self, timeout_us):
        """Returns the status of a device wait on a counter nothing sets (ORBX_ERR_TIMEOUT expected)."""
        return int(lib().orbx_selftest_wait_timeout(self.h, int(timeout_us)))

    def bounds_report(self):
        """Bounds-checked build: (skipped accesses, site of the first, its offset,
        its buffer's extent) since the last report; clears the record."""
        out = (ctypes.c_longlong * 4)()
        _check(lib().orbx_bounds_report(self.h, out), "orbx_bounds_report")
        return tuple(int(v) for v in out)

    def bounds_set_slack(self, nbytes):
        """Bounds-checked build: later frames' image extents, as checked, end nbytes early."""
        _check(lib().orbx_bounds_set_slack(self.h, int(nbytes)), "orbx_bounds_set_slack")

    def debug_buffers(self, w, h):
        n, oszp = layout(w, h, self.params.noctaves)
        obytes = int(oszp[5 * n])
        npx = int(oszp[0])
        pyr = np.zeros(obytes, dtype=np.uint8)
        blur = np.zeros(obytes, dtype=np.uint8)
        vmap = np.zeros(npx, dtype=np.float32)
        layer = np.zeros(npx, dtype=np.int32)
        total = np.zeros(1, dtype=np.int32)
        _check(lib().orbx_debug_buffers(self.h, pyr.ctypes.data, blur.ctypes.data, vmap.ctypes.data,
                                        layer.ctypes.data, total.ctypes.data), "orbx_debug_buffers")
        return {"pyr": pyr, "blur": blur, "vmap": vmap, "layer": layer, "total": int(total[0]), "n": n,
                "oszp": oszp}


# -- torch conveniences -------------------------------------------------------
def _torch():
    import torch
    return torch


class FrameBuffers:
    """Device buffers for one image's keypoints, descriptors and count."""

    def __init__(self, max_pts, device="cuda"):
        torch = _torch()
        self.max_pts = max_pts
        self.points = torch.zeros((max_pts, 7), dtype=torch.int32, device=device)
        self.desc = torch.zeros((max_pts, 32), dtype=torch.uint8, device=device)
        self.count = torch.zeros(1, dtype=torch.int32, device=device)

    def to_host(self):
        n = int(self.count.item())
        pts = self.points[:n].cpu().numpy().copy().view(ORB_POINT_DTYPE).reshape(n)
        return pts, self.desc[:n].cpu().numpy().copy()


def detect_and_compute(ctx, img, w, h, bufs=None, compute_desc=True):
    """img: uint8 CUDA tensor of shape (h, pitch).  Returns FrameBuffers (asynchronous)."""
    if bufs is None:
        bufs = FrameBuffers(ctx.params.max_pts, img.device)
    ctx.detect_and_compute_ptr(img, w, h, img.shape[1], bufs.points, bufs.desc, bufs.count, compute_desc)
    return bufs


def knn2(ctx, q, db, mode=MATCH_POPC):
    """q, db: uint8 CUDA tensors (n, 32).  Returns (dist2 uint32 as int64, idx2 int32) CUDA tensors."""
    torch = _torch()
    nq, ndb = q.shape[0], db.shape[0]
    dist = torch.empty((nq, 2), dtype=torch.int32, device=q.device)
    idx = torch.empty((nq, 2), dtype=torch.int32, device=q.device)
    ctx.knn2_ptr(q, nq, db if ndb else None, ndb, dist, idx, mode)
    return dist, idx


STATIC_MAX_QUERIES = 16384  # ORBX_STATIC_MAX_QUERIES


def knn2_static_ptr(d_q, nq, d_db, ndb, d_dist2, d_idx2, stream=None):
    """orbx_match_knn2_static on the current device; stream is a raw cudaStream_t (int) or None."""
    _check(lib().orbx_match_knn2_static(_ptr(d_q), nq, _ptr(d_db), ndb, _ptr(d_dist2), _ptr(d_idx2), stream),
           "orbx_match_knn2_static")


class LearnedIndex:
    """orbx_learned_*: a trained proposal index over a device database.

    db, train: uint8 CUDA tensors (n, 32); the index keeps its own copy of db."""

    def __init__(self, ctx, db, train=None, params=None):
        self.ctx = ctx
        self.params = params if params is not None else learned_params()
        h = ctypes.c_void_p()
        ntrain = 0 if train is None else train.shape[0]
        _check(lib().orbx_learned_build(ctx.h, ctypes.byref(self.params), _ptr(db), db.shape[0], _ptr(train), ntrain,
                                        ctypes.byref(h)), "orbx_learned_build")
        self.h = h
        self.ndb = db.shape[0]

    @classmethod
    def load(cls, ctx, data, db):
        """An index from save()'s bytes over the uint8 CUDA database db (n, 32),
        listed again under the saved centroids or buckets; no training."""
        self = cls.__new__(cls)
        self.ctx = ctx
        h = ctypes.c_void_p()
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        _check(lib().orbx_learned_load(ctx.h, buf, len(data), _ptr(db), db.shape[0], ctypes.byref(h)),
               "orbx_learned_load")
        self.h = h
        self.ndb = db.shape[0]
        self.params = LearnedParams()
        _check(lib().orbx_learned_get_params(self.h, ctypes.byref(self.params)), "orbx_learned_get_params")
        return self

    def save(self):
        """The checkpoint as bytes (parameters, statistics, centroids, search weights)."""
        need = ctypes.c_size_t()
        _check(lib().orbx_learned_save(self.ctx.h, self.h, None, 0, ctypes.byref(need)), "orbx_learned_save")
        buf = ctypes.create_string_buffer(need.value)
        _check(lib().orbx_learned_save(self.ctx.h, self.h, buf, need.value, ctypes.byref(need)), "orbx_learned_save")
        return buf.raw

    def close(self):
        if getattr(self, "h", None):
            lib().orbx_learned_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_margin(self, m):
        self.params.margin = float(m)
        _check(lib().orbx_learned_set_margin(self.h, float(m)), "orbx_learned_set_margin")

    def set_max_distance(self, d):
        self.params.max_distance = int(d)
        _check(lib().orbx_learned_set_max_distance(self.h, int(d)), "orbx_learned_set_max_distance")

    def set_rerank(self, form):
        self.params.rerank = int(form)
        _check(lib().orbx_learned_set_rerank(self.h, int(form)), "orbx_learned_set_rerank")

    def probe_pairs(self):
        """(query, row) pairs the last search's rerank scanned (synchronises)."""
        v = ctypes.c_ulonglong()
        _check(lib().orbx_learned_probe_pairs(self.ctx.h, self.h, ctypes.byref(v)), "orbx_learned_probe_pairs")
        return int(v.value)

    def stats(self):
        st = LearnedStats()
        _check(lib().orbx_learned_get_stats(self.h, ctypes.byref(st)), "orbx_learned_get_stats")
        return st.to_dict()

    def search_ptr(self, d_q, nq, d_dist2, d_idx2, d_margin=None, d_fb=None):
        _check(lib().orbx_learned_search(self.ctx.h, self.h, _ptr(d_q), nq, _ptr(d_dist2), _ptr(d_idx2),
                                         _ptr(d_margin), _ptr(d_fb)), "orbx_learned_search")

    def profile_search(self, q, dist, idx):
        """Per-phase device ms: proposal, lists, rerank, merge, fallback (synchronises)."""
        ms = np.zeros(5, dtype=np.float32)
        _check(lib().orbx_learned_profile_search(self.ctx.h, self.h, _ptr(q), q.shape[0], _ptr(dist), _ptr(idx),
                                                 ms.ctypes.data), "orbx_learned_profile_search")
        return ms

    def search(self, q):
        """Returns (dist2, idx2, margin, fallback_count tensor) as CUDA tensors."""
        torch = _torch()
        nq = q.shape[0]
        dist = torch.empty((nq, 2), dtype=torch.int32, device=q.device)
        idx = torch.empty((nq, 2), dtype=torch.int32, device=q.device)
        margin = torch.empty(nq, dtype=torch.float32, device=q.device)
        fb = torch.zeros(1, dtype=torch.int32, device=q.device)
        self.search_ptr(q, nq, dist, idx, margin, fb)
        return dist, idx, margin, fb

    def export(self, weights=True):
        p = self.params
        assign = np.zeros(self.ndb, dtype=np.int32)
        offsets = np.zeros(p.n_clusters + 1, dtype=np.int32)
        out = {"assign": assign, "offsets": offsets}
        args = [None] * 4
        if weights and p.proposal == PROPOSAL_MLP:
            out["w1"] = np.zeros((p.hidden, 256), dtype=np.float32)
            out["b1"] = np.zeros(p.hidden, dtype=np.float32)
            out["w2"] = np.zeros((p.n_clusters, p.hidden), dtype=np.float32)
            out["b2"] = np.zeros(p.n_clusters, dtype=np.float32)
            args = [out[k].ctypes.data for k in ("w1", "b1", "w2", "b2")]
        _check(lib().orbx_learned_export(self.ctx.h, self.h, assign.ctypes.data, offsets.ctypes.data, *args),
               "orbx_learned_export")
        return out

    def gradients(self, x, labels):
        """x: uint8 CUDA (n, 32), labels: int32 CUDA (n,).  Returns loss and fp32 host gradients."""
        p = self.params
        n = x.shape[0]
        g = {"w1": np.zeros((p.hidden, 256), dtype=np.float32), "b1": np.zeros(p.hidden, dtype=np.float32),
             "w2": np.zeros((p.n_clusters, p.hidden), dtype=np.float32), "b2": np.zeros(p.n_clusters, dtype=np.float32)}
        loss = ctypes.c_float()
        _check(lib().orbx_learned_gradients(self.ctx.h, self.h, _ptr(x), _ptr(labels), n, ctypes.byref(loss),
                                            *[g[k].ctypes.data for k in ("w1", "b1", "w2", "b2")]),
               "orbx_learned_gradients")
        return float(loss.value), g


def gemm_bf16(ctx, a, b, mode=GEMM_F32, bias=None, splits=1, aux=None):
    """C = a @ b.T on the tcgen05 BF16 GEMM; a (M, K), b (N, K) bf16 CUDA tensors."""
    torch = _torch()
    M, K = a.shape
    N = b.shape[0]
    if mode == GEMM_F32:
        out = torch.empty((splits, M, N) if splits > 1 else (M, N), dtype=torch.float32, device=a.device)
    elif mode == GEMM_TOP8:
        out = torch.empty((M, N // 128, 8), dtype=torch.int32, device=a.device)
    elif mode == GEMM_TOP8_ROW:
        out = torch.empty((M, gemm_top_lists(N), 8), dtype=torch.int32, device=a.device)
    else:
        out = torch.empty((M, N), dtype=torch.bfloat16, device=a.device)
    _check(lib().orbx_gemm_bf16(ctx.h, _ptr(a), _ptr(b), M, N, K, _ptr(bias), mode, splits, _ptr(out), _ptr(aux)),
           "orbx_gemm_bf16")
    return out


class PairBatch:
    """Device images and output buffers for orbx_batch_pairs.

    pairs: list of (img_a, img_b, w, h, max_pts) with uint8 host arrays of shape
    (h, pitch); images are copied to the device once."""

    def __init__(self, pairs, device="cuda"):
        torch = _torch()
        self.n = len(pairs)
        self.ia = (Image * self.n)()
        self.ib = (Image * self.n)()
        self.oa = (FrameOut * self.n)()
        self.ob = (FrameOut * self.n)()
        self.imgs, self.outs, self.shapes = [], [], []
        for i, (a, b, w, h, cap) in enumerate(pairs):
            da = torch.from_numpy(np.ascontiguousarray(a)).to(device)
            db = torch.from_numpy(np.ascontiguousarray(b)).to(device)
            A, B = FrameBuffers(cap, device), FrameBuffers(cap, device)
            self.imgs.append((da, db))
            self.outs.append((A, B))
            self.shapes.append((w, h, cap))
            self.ia[i] = Image(da.data_ptr(), w, h, a.shape[1])
            self.ib[i] = Image(db.data_ptr(), w, h, b.shape[1])
            self.oa[i] = FrameOut(A.points.data_ptr(), A.desc.data_ptr(), A.count.data_ptr(), cap)
            self.ob[i] = FrameOut(B.points.data_ptr(), B.desc.data_ptr(), B.count.data_ptr(), cap)

    def results(self, i):
        A, B = self.outs[i]
        pa, da = A.to_host()
        pb, db = B.to_host()
        return pa, da, pb, db
