#!/usr/bin/env python
"""Benchmark of the sm_100a ORB library on one 1920x1080 frame pair.

A step is one frame pair: detect + describe both images and match A -> B
(noctaves 8 -> 4 levels at 1080p, edge 31, FAST 20, Harris score, patch 31,
WTA_K 2, at most 10000 keypoints per image), synthetic images from the seeded
generator in cuda-orb_b200/synth.py.  The L2 cache is flushed (256 MiB write)
before every timed step; each step is timed with CUDA events on the library's
stream.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl orbx|reference]

Prints one JSON line (rank 0).  Under torchrun every rank runs its own replica
(there is no exchange between frame pairs) and the reported time is the max
over ranks.  --impl reference runs the reference CUDA-ORB build
(oracle/_ref/libref_orb.so, the reference's own orbd.cu/orb.cpp compiled for
sm_100a) through its Orbor API on the same pair and GPU.
"""
import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuda-orb_b200"))
sys.path.insert(0, ROOT)

METRIC = "ms/1080p pair detect+match; Hamming match-pairs/s exact vs learned @recall>=0.99"
W, H = 1920, 1080
MAX_PTS = 10000
L2_FLUSH_BYTES = 256 << 20
POPC_PER_CLK_PER_SM = 16  # 32-bit population count results per clock per SM
SMS = 148

# DRAM bytes per launch measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum,
# cold cache) on the same workloads (the committed ncu summaries of the 1080p
# pair and of 65536 x 65536 matching); kernels without a capture report None.
# Warp instructions per launch of the five pair kernels (ncu smsp__inst_executed.sum
# on the same 1080p pair, the committed summary of the pair's kernels): the
# instruction roofline beside the HBM one, since these kernels are issue- and
# latency-bound.
NCU_WARP_INST = {"pyramid_blur": 9089420, "detect": 11898158, "nms": 3933009, "describe": 2286742,
                 "match": 2037180}
ISSUE_PER_CLK_PER_SM = 4  # warp instructions issued per clock per SM (one per scheduler)

NCU_TRAFFIC = {"k_pyramid_blur": 4167808, "k_detect": 5666176, "k_nms": 1543552, "k_describe<2>": 5689856,
               "k_match_popc": 99584, "k_match_imma": 33602560}


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=["orbx", "reference"], default="orbx")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-match-bench", action="store_true")
    p.add_argument("--no-e2e-variants", action="store_true",
                   help="pair workload: skip the upload-banding variants of the end-to-end call (their "
                        "second stream cannot overlap the launch under a profiler that serialises work)")
    p.add_argument("--no-learned-bench", action="store_true",
                   help="pair workload: skip the learned-proposal summary (about 20 s on rank 0)")
    p.add_argument("--workload", choices=["pair1080", "match65536", "batch64", "learned"], default="pair1080",
                   help="pair1080: the 1920x1080 pair (default); match65536: k=2 matching only; "
                        "batch64: 64 pairs of mixed resolution and caps in one batch; "
                        "learned: learned-proposal k=2 search, 131072 queries x 1048576 database rows")
    p.add_argument("--learned-spill", type=int, default=8,
                   help="learned: clusters each database row is listed in (1..16)")
    p.add_argument("--learned-epochs", type=int, default=3, help="learned: training epochs")
    p.add_argument("--learned-labels", choices=["nearest", "listed"], default="listed",
                   help="learned: training target, the nearest row's cluster or all clusters it is listed in")
    p.add_argument("--learned-scale", type=float, default=1.0,
                   help="learned: fraction of the database / query / training sizes (tests use < 1)")
    p.add_argument("--match-mode", choices=["imma", "popc"], default="imma")
    p.add_argument("--no-autotune", action="store_true", help="batch64: keep the default launch shapes")
    return p.parse_args(argv)


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value, world):
    """Max of a float over all ranks (the whole-job time)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, world):
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, interval_ms=50):
        self.gpu = gpu_index
        self.interval = interval_ms
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 f"-lms={self.interval}"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
        time.sleep(0.15)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [r for r in csv.reader(io.StringIO(out)) if len(r) >= 9]
        sm = []
        smax = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# per-kernel algorithmic bytes / work for the pair (two frames)
# ---------------------------------------------------------------------------
def stage_work(oszp, n, na, nb):
    h0 = int(oszp[2 * n])
    p0 = int(oszp[3 * n])
    obytes = int(oszp[5 * n])
    npx = h0 * p0
    nk = na + nb
    return {
        # input read once, raw and blurred pyramids written
        "pyramid_blur": 2 * (npx + 2 * obytes),
        # raw pyramid read, occupancy bits + sparse score/octave of the survivors written
        # (corners that NMS removes are not counted: a lower bound)
        "detect": 2 * (obytes + npx // 8) + nk * 5,
        # occupancy bits and survivors' score/octave read, keypoints written
        "nms": 2 * (npx // 8) + nk * (5 + 28),
        # per keypoint: point, 31x31 disc, 512 samples, angle + 32-byte descriptor
        "describe": nk * (28 + 961 + 512 + 4 + 32),
    }


def pair_config(n, na, nb):
    """The pair workload's config, printed identically by both arms."""
    return {"workload": "1920x1080 uint8 pair: detect+describe A and B, match A->B",
            "levels": n, "noctaves_requested": 8, "fast_threshold": 20, "edge": 31, "wta_k": 2,
            "score": "harris", "patch": 31, "max_pts": MAX_PTS, "keypoints": [na, nb],
            "l2": "flushed (256 MiB write) before every timed step", "parallelism": "replicas"}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return pk, "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# ---------------------------------------------------------------------------
# CPU baselines
# ---------------------------------------------------------------------------
def cpu_baseline_port(a, b, budget_s=12.0, max_reps=20):
    """The oracle (CPU restatement) on the same pair, on this host's cores."""
    from oracle import oracle as O

    times = []
    t_end = time.time() + budget_s
    while len(times) < max_reps and (not times or time.time() < t_end):
        t0 = time.perf_counter()
        ra = O.detect_and_compute(a, W, H, max_pts=MAX_PTS)
        rb = O.detect_and_compute(b, W, H, max_pts=MAX_PTS)
        O.match(ra["desc"], rb["desc"])
        times.append(time.perf_counter() - t0)
    return {"value": 1000.0 * statistics.median(times), "unit": "ms", "cores": O.threads(), "kind": "port",
            "sample": f"{len(times)} runs of the full 1920x1080 pair (detect+describe A and B, match A->B) "
                      f"by the oracle restatement, median"}


def parity_report(a, b, pa, da, pb, db):
    """Check of the timed pair's output (outside every timed region), run with
    the CPU baseline: bit-exactness with the oracle (given the reference build's
    __sinf/__cosf when present) and with the live reference build, Harris
    scores and angles against the FP64 side-oracle (1e-5 relative, absolute
    floors in oracle/oracle.py), and the counted exceptions: rotation rounding
    ties, patches that leave their octave, and descriptors the stock
    reference's in-place blur race changes."""
    from oracle import oracle as O
    from oracle import refharness as R

    have_ref = R.available()
    sincos = None
    if have_ref:
        R.lib()
        sincos = R.sincos
    rep = {"sin_cos": "reference build __sinf/__cosf" if have_ref else "libm (reference build absent)",
           "fp64_rel_tol": O.FP64_REL_TOL, "harris_abs_floor": O.HARRIS_ABS_FLOOR,
           "angle_abs_floor": O.ANGLE_ABS_FLOOR, "tie_eps": O.TIE_EPS, "frames": {}}
    for name, img, pts, desc in (("A", a, pa, da), ("B", b, pb, db)):
        ref = O.detect_and_compute(img, W, H, max_pts=MAX_PTS, sincos=sincos)
        fr = {"keypoints": int(len(pts)),
              "points_bit_exact_vs_oracle": bool(len(pts) == len(ref["points"]) and
                                                 np.array_equal(pts[["x", "y", "octave"]],
                                                                ref["points"][["x", "y", "octave"]]) and
                                                 np.array_equal(pts["score"].view(np.uint32),
                                                                ref["points"]["score"].view(np.uint32)) and
                                                 np.array_equal(pts["angle"].view(np.uint32),
                                                                ref["points"]["angle"].view(np.uint32))),
              "desc_rows_differing_vs_oracle": int(np.any(desc != ref["desc"], axis=1).sum())
              if desc.shape == ref["desc"].shape else -1}
        chk = O.fp64_check(img, W, H, pts, ref["sin"], ref["cos"])
        flags = chk.pop("flags")
        fr.update({k: v for k, v in chk.items() if k != "keypoints"})
        if have_ref:
            # rows whose bits change when libm sin/cos replace __sinf/__cosf: these
            # are the rotation-sensitive keypoints, and should carry the tie flag
            alt = O.detect_and_compute(img, W, H, max_pts=MAX_PTS)
            if alt["desc"].shape == ref["desc"].shape:
                sens = np.any(alt["desc"] != ref["desc"], axis=1)
                fr["desc_rows_sensitive_to_sincos"] = int(sens.sum())
                fr["of_which_flagged_tie"] = int((sens & ((flags & O.TIE) != 0)).sum())
        if have_ref:
            # the reference build live on the same image: race-free form (A') and stock form (A)
            R.init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1,
                   max_pts=MAX_PTS)
            rf = R.stages(img, W, H, MAX_PTS, race_free=True)
            st = R.stages(img, W, H, MAX_PTS, race_free=False)
            o1 = np.lexsort((rf["points"]["x"], rf["points"]["y"]))
            o2 = np.lexsort((st["points"]["x"], st["points"]["y"]))
            rpts = rf["points"][o1]
            fr["bit_exact_vs_reference_build"] = bool(
                len(rpts) == len(pts) and np.array_equal(pts[["x", "y", "octave"]], rpts[["x", "y", "octave"]])
                and np.array_equal(pts["score"].view(np.uint32), rpts["score"].view(np.uint32))
                and np.array_equal(pts["angle"].view(np.uint32), rpts["angle"].view(np.uint32))
                and np.array_equal(desc, rf["desc"][o1]))
            fr["blur_race_desc_rows"] = O.blur_race_rows(rf["desc"][o1], st["desc"][o2])
        rep["frames"][name] = fr
    m, d = O.match(da, db)
    rep["matches_bit_exact_vs_oracle"] = bool(np.array_equal(pa["match"], m) and np.array_equal(pa["distance"], d))
    return rep


def cpu_baseline_opencv_c0(budget_s=6.0):
    """OpenCV's own ORB + BFMatcher on the 640x480 pair (5000 keypoints, 8
    levels, scale 1.2), on all host cores and on one thread: the comparison the
    reference's demo makes on the host (main.cpp:274-336)."""
    try:
        import cv2
    except ImportError:
        return {"unavailable": "cv2 not importable on this host"}
    import synth

    a, b, _ = synth.make_pair(640, 480, seed=0)
    ia, ib = np.ascontiguousarray(a[:, :640]), np.ascontiguousarray(b[:, :640])
    out = {"workload": "640x480 uint8 pair, cv2.ORB(5000, 1.2, 8 levels, FAST 20) + BFMatcher knn k=2"}
    all_cores = len(os.sched_getaffinity(0))
    for key, cores in (("all_cores", all_cores), ("one_thread", 1)):
        cv2.setNumThreads(cores)
        orb = cv2.ORB_create(nfeatures=5000, scaleFactor=1.2, nlevels=8, edgeThreshold=31, patchSize=31,
                             fastThreshold=20, WTA_K=2)
        bf = cv2.BFMatcher(cv2.NORM_HAMMING)
        times = []
        t_end = time.time() + budget_s
        while len(times) < 50 and (not times or time.time() < t_end):
            t0 = time.perf_counter()
            ka, da = orb.detectAndCompute(ia, None)
            kb, db = orb.detectAndCompute(ib, None)
            if da is not None and db is not None:
                bf.knnMatch(da, db, k=2)
            times.append(time.perf_counter() - t0)
        out[key] = {"value": 1000.0 * statistics.median(times), "unit": "ms", "cores": cores,
                    "runs": len(times), "keypoints": [len(ka), len(kb)]}
    cv2.setNumThreads(all_cores)
    return out


def cpu_baseline_opencv(a, b, budget_s=8.0):
    """OpenCV cv2.ORB + BFMatcher(NORM_HAMMING) knnMatch k=2 on the host (its own algorithm, for context)."""
    try:
        import cv2
    except ImportError:
        return {"unavailable": "cv2 not importable on this host"}
    cores = len(os.sched_getaffinity(0))
    cv2.setNumThreads(cores)
    orb = cv2.ORB_create(nfeatures=MAX_PTS, scaleFactor=1.2, nlevels=8, edgeThreshold=31, patchSize=31,
                         fastThreshold=20, WTA_K=2)
    bf = cv2.BFMatcher(cv2.NORM_HAMMING)
    ia, ib = np.ascontiguousarray(a[:, :W]), np.ascontiguousarray(b[:, :W])
    times = []
    t_end = time.time() + budget_s
    nka = nkb = 0
    while len(times) < 20 and (not times or time.time() < t_end):
        t0 = time.perf_counter()
        ka, da = orb.detectAndCompute(ia, None)
        kb, db = orb.detectAndCompute(ib, None)
        if da is not None and db is not None:
            bf.knnMatch(da, db, k=2)
        times.append(time.perf_counter() - t0)
        nka, nkb = len(ka), len(kb)
    return {"value": 1000.0 * statistics.median(times), "unit": "ms", "cores": cores,
            "kind": "opencv", "keypoints": [nka, nkb],
            "sample": f"{len(times)} runs, cv2 {cv2.__version__} ORB(10000, 1.2, 8 levels) + BFMatcher knn k=2"}


# ---------------------------------------------------------------------------
# the library arm
# ---------------------------------------------------------------------------
def run_orbx(args, world, rank, local):
    import torch

    import orbx
    import synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    a, b, _ = synth.make_pair(W, H, seed=rank)
    pitch = a.shape[1]
    stream = torch.cuda.Stream(device=dev)
    ctx = orbx.Context(local, orbx.make_params(noctaves=8, edge_threshold=31, wta_k=2, score_type=0, patch_size=31,
                                               fast_threshold=20, max_pts=MAX_PTS), stream=stream)
    da = torch.from_numpy(a).to(dev)
    db = torch.from_numpy(b).to(dev)
    A, B = orbx.FrameBuffers(MAX_PTS, dev), orbx.FrameBuffers(MAX_PTS, dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def step():
        ctx.pair_ptr(da, db, W, H, pitch, A.points, A.desc, A.count, B.points, B.desc, B.count)

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
        stream.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        sampler = ClockSampler(local)
        if rank == 0:
            sampler.start()
        barrier(world)
        torch.cuda.synchronize(dev)
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            step()
            ends[k].record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        clocks = sampler.stop() if rank == 0 else None
        step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    local_total = sum(step_ms)
    total_ms = max_over_ranks(local_total, world)
    na, nb = int(A.count.item()), int(B.count.item())
    matched = int((A.points[:na, 5] >= 0).sum().item())
    host_pa, host_da = A.to_host()
    host_pb, host_db = B.to_host()

    # the same pair with the int8 tcgen05 matcher (the other exact form)
    imma_ms = []
    with torch.cuda.stream(stream):
        for _ in range(3):
            ctx.pair_ptr(da, db, W, H, pitch, A.points, A.desc, A.count, B.points, B.desc, B.count,
                         orbx.MATCH_IMMA)
        for _ in range(min(args.steps, 100)):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.pair_ptr(da, db, W, H, pitch, A.points, A.desc, A.count, B.points, B.desc, B.count,
                         orbx.MATCH_IMMA)
            e1.record(stream)
            e1.synchronize()
            imma_ms.append(e0.elapsed_time(e1))
    imma_pa, _ = A.to_host()

    # both forms of the device-resident pair: five graph-replayed launches and
    # one persistent launch with a device work queue
    pair_forms = {}
    keep_t = ctx.get_tuning()
    for name, form, rows in (("five_launch", 0, 0), ("persistent", 1, 0), ("persistent_row_deps", 1, 1)):
        t = ctx.get_tuning()
        t.pair_form = form
        t.persist_row_deps = rows
        ctx.set_tuning(t)
        f_ms = []
        with torch.cuda.stream(stream):
            for _ in range(3):
                step()
            for _ in range(min(args.steps, 100)):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step()
                e1.record(stream)
                e1.synchronize()
                f_ms.append(e0.elapsed_time(e1))
        fa, fda = A.to_host()
        pair_forms[name] = {"ms": statistics.median(f_ms),
                            "equal_to_timed_run": bool(np.array_equal(fa, host_pa) and np.array_equal(fda, host_da))}
    ctx.set_tuning(keep_t)
    pair_imma = {"ms": statistics.median(imma_ms), "steps": len(imma_ms),
                 "matches_equal_popc": bool(np.array_equal(imma_pa["match"], host_pa["match"]) and
                                            np.array_equal(imma_pa["distance"], host_pa["distance"]))}

    # end to end through the host-buffer C ABI call, pinned host images
    ha = torch.from_numpy(a).pin_memory()
    hb = torch.from_numpy(b).pin_memory()
    hpa = np.zeros((MAX_PTS, 7), dtype=np.int32)
    hpb = np.zeros((MAX_PTS, 7), dtype=np.int32)
    hna = np.zeros(1, dtype=np.int32)
    hnb = np.zeros(1, dtype=np.int32)
    e2e_steps = min(max(args.steps, 200), 300)  # host-side noise: at least 200 samples

    def e2e_run(bands, steps, rows=0, streams=0):
        """CUDA-event and host wall times of orbx_pair_host with the given upload overlap."""
        t = ctx.get_tuning()
        keep = (t.upload_bands, t.persist_row_deps, t.host_overlap)
        if bands is not None:
            t.upload_bands = bands
            t.persist_row_deps = rows
            t.host_overlap = streams
            ctx.set_tuning(t)
        with torch.cuda.stream(stream):
            for _ in range(3):
                ctx.pair_host(ha.data_ptr(), hb.data_ptr(), W, H, pitch, hpa, hna, hpb, hnb)
            ev_ms, wall_ms = [], []
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            barrier(world)
            for _ in range(steps):
                flush.zero_()
                stream.synchronize()
                t0 = time.perf_counter()
                ev0.record(stream)
                ctx.pair_host(ha.data_ptr(), hb.data_ptr(), W, H, pitch, hpa, hna, hpb, hnb)
                ev1.record(stream)
                wall_ms.append(1000.0 * (time.perf_counter() - t0))
                ev1.synchronize()
                ev_ms.append(ev0.elapsed_time(ev1))
            barrier(world)
        if bands is not None:
            t.upload_bands, t.persist_row_deps, t.host_overlap = keep
            ctx.set_tuning(t)
        return ev_ms, wall_ms

    _t = ctx.get_tuning()
    ctx_overlap = {"upload_bands": int(_t.upload_bands), "host_overlap": int(_t.host_overlap)}
    e_ms, e_wall = e2e_run(None, e2e_steps)
    e2e_total = max_over_ranks(sum(e_ms), world)
    e2e_variants = {}
    variants = ((0, 0, 0), (0, 0, 1), (2, 0, 0), (4, 0, 0), (8, 0, 0), (4, 1, 0))
    for bands, rows, streams in (() if args.no_e2e_variants else variants):
        name = ("two_streams" if streams else f"bands_{bands}") + ("_row_deps" if rows else "")
        v_ev, v_wall = e2e_run(bands, min(e2e_steps, 50), rows, streams)
        e2e_variants[name] = {"ms": statistics.median(v_ev), "host_wall_ms": statistics.median(v_wall)}
        # where the time goes: CUDA events between the phases and host clocks
        t = ctx.get_tuning()
        keep_b = (t.upload_bands, t.persist_row_deps, t.host_overlap)
        t.upload_bands = bands
        t.persist_row_deps = rows
        t.host_overlap = streams
        ctx.set_tuning(t)
        phases = []
        with torch.cuda.stream(stream):
            for _ in range(min(e2e_steps, 30)):
                flush.zero_()
                stream.synchronize()
                phases.append(ctx.profile_pair_host(ha.data_ptr(), hb.data_ptr(), W, H, pitch, hpa, hna, hpb, hnb))
        t.upload_bands, t.persist_row_deps, t.host_overlap = keep_b
        ctx.set_tuning(t)
        e2e_variants[name]["phases_ms"] = {k: statistics.median(p[k] for p in phases) for k in phases[0]}
    h2d = 2 * H * pitch
    d2h = 8 + (int(hna[0]) + int(hnb[0])) * 28

    # per-kernel times (events between the five launches, same inputs, L2 flushed)
    prof_steps = min(args.steps, 100)
    with torch.cuda.stream(stream):
        acc = np.zeros(5)
        for _ in range(prof_steps):
            flush.zero_()
            acc += ctx.profile_pair(da, db, W, H, pitch, A.points, A.desc, A.count, B.points, B.desc, B.count)
    stage_ms = acc / prof_steps
    names = ["pyramid_blur", "detect", "nms", "describe", "match"]
    n, oszp = orbx.layout(W, H, 8)
    work = stage_work(oszp, n, na, nb)
    peaks, peak_kind = load_peaks()
    kernels = {}
    clk_hz = ((clocks or {}).get("sm_mhz") or 1965.0) * 1e6
    for i, nm in enumerate(names):
        ent = {"ms": float(stage_ms[i])}
        if nm in work:
            ent["bytes"] = work[nm]
            ent["gbs"] = work[nm] / (stage_ms[i] * 1e-3) / 1e9
        else:
            ent["popc_ops"] = na * nb * 8
        if nm in NCU_WARP_INST:
            # instruction roofline: warp instructions per level-0 pixel of the pair,
            # and the fraction of the SMs' issue slots they fill in the live time
            inst = NCU_WARP_INST[nm]
            ent["warp_inst"] = inst
            ent["warp_inst_per_l0_pixel"] = inst / (2.0 * W * H)
            ent["issue_slot_frac"] = inst / (ISSUE_PER_CLK_PER_SM * SMS * clk_hz * stage_ms[i] * 1e-3)
        kernels[nm] = ent
    dom = max(names, key=lambda k: kernels[k]["ms"])
    if dom == "match":
        clock_mhz = (clocks or {}).get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        peak_ops = SMS * POPC_PER_CLK_PER_SM * peaks.get("sm_max_mhz", 1965.0) * 1e6
        ach = kernels["match"]["popc_ops"] / (stage_ms[4] * 1e-3)
        roofline = {"kernel": "k_match_popc", "bound": "int", "achieved": ach / 1e12, "peak": peak_ops / 1e12,
                    "unit": "Tpopc/s", "frac": ach / peak_ops, "traffic": NCU_TRAFFIC.get("k_match_popc"),
                    "peak_kind": "derived: 148 SMs x 16 popc/clk x max SM clock", "clock_mhz": clock_mhz}
    else:
        kname = {"pyramid_blur": "k_pyramid_blur", "detect": "k_detect", "nms": "k_nms",
                 "describe": "k_describe<2>"}[dom]
        ach = kernels[dom]["gbs"]
        roofline = {"kernel": kname, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": ach / peaks["hbm_gbs"], "traffic": NCU_TRAFFIC.get(kname),
                    "peak_kind": f"{peak_kind} hbm_gbs", "algorithmic_bytes": work[dom]}

    match_bench = None
    if not args.no_match_bench and rank == 0:
        match_bench = bench_knn2(ctx, stream, dev, peaks)

    result = None
    if rank == 0:
        steps_all = args.steps * world
        value = total_ms / steps_all
        result = {
            "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded blobs + polygons + noise, homography-warped partner; cuda-orb_b200/synth.py)",
            "config": pair_config(n, na, nb),
            "impl_detail": {"matcher": "XOR-popc", "graph": "one CUDA graph per pair (5 kernels)",
                            "matches": matched},
            "e2e": {"value": e2e_total / (e2e_steps * world), "unit": "ms", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "median_ms": statistics.median(e_ms), "steps": e2e_steps,
                    "host_wall_ms_median": statistics.median(e_wall),
                    "overlap": ctx_overlap,
                    "how": "orbx_pair_host: pinned host images in, host keypoints/matches out, CUDA events",
                    "variants": e2e_variants},
            "gpu_launches": 5 * args.steps,
            "roofline": roofline,
            "kernels": kernels,
            "pair_int8_tcgen05_matcher": pair_imma,
            "pair_forms": pair_forms,
            "clocks": clocks,
        }
        if match_bench:
            result["match_65536"] = match_bench
    ctx.close()
    return result, (a, b), (host_pa, host_da, host_pb, host_db)


def bench_knn2(ctx, stream, dev, peaks):
    """Matching only: 65536 queries x 65536 database rows, k = 2, both exact forms."""
    import torch

    import orbx
    import synth

    dbh, qh, _ = synth.match_workload(65536, 65536, seed=0)
    q = torch.from_numpy(qh).to(dev)
    db = torch.from_numpy(dbh).to(dev)
    pairs = 65536.0 * 65536.0
    out = {}
    with torch.cuda.stream(stream):
        res = {}
        for name, mode in (("xor_popc", orbx.MATCH_POPC), ("int8_tcgen05", orbx.MATCH_IMMA)):
            res[name] = orbx.knn2(ctx, q, db, mode)
            ctx.sync()
            ms = []
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                orbx.knn2(ctx, q, db, mode)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            out[name] = {"ms": statistics.median(ms), "pairs_per_s": pairs / (statistics.median(ms) * 1e-3)}
        same = bool(torch.equal(res["xor_popc"][0], res["int8_tcgen05"][0]) and
                    torch.equal(res["xor_popc"][1], res["int8_tcgen05"][1]))
    popc_peak = SMS * POPC_PER_CLK_PER_SM * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 8
    out["xor_popc"].update({"roofline_pairs_per_s": popc_peak, "frac": out["xor_popc"]["pairs_per_s"] / popc_peak,
                            "peak_kind": "derived: 148 SMs x 16 popc/clk x max SM clock / 8 popc per pair"})
    ops = pairs * 512.0  # 256 int8 multiply-adds per pair, 2 ops each
    t = out["int8_tcgen05"]["ms"] * 1e-3
    i8_measured = 2.0 * peaks.get("bf16_tflops", 1590.0) * 1e12
    out["int8_tcgen05"].update({"tops": ops / t / 1e12, "peak_tops_measured_bf16x2": i8_measured / 1e12,
                                "frac_of_measured": ops / t / i8_measured, "peak_tops_nominal_dense": 4500.0,
                                "frac_of_nominal": ops / t / 4.5e15,
                                "note": "int8 dense peak taken as 2x the measured cuBLAS bf16 peak; includes the "
                                        "+-1 expansion of both 65536 x 32-byte sets"})
    out["bit_exact_popc_vs_tcgen05"] = same
    return out


# ---------------------------------------------------------------------------
# the reference arm
# ---------------------------------------------------------------------------
def run_reference(args, world, rank, local):
    if rank != 0:
        return None
    from oracle import refharness as R

    if not R.available():
        return {"impl": "reference", "unavailable": "reference build oracle/_ref/libref_orb.so not built"}
    import torch

    import synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    a, b, _ = synth.make_pair(W, H, seed=rank)
    R.init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1, max_pts=MAX_PTS)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    steps = min(args.steps, 300)

    R.time_pair(a, b, W, H, max(args.warmup, 3), 1)
    ms = []
    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t, na, nb = R.time_pair(a, b, W, H, 0, 1)
        ms.append(t)
    clocks = sampler.stop()
    # The harness zero-fills every reference allocation with its guards (the
    # reference reads outside its buffers by design); per pair that adds two
    # fills of the descriptor block plus 512 KiB.  Their cost, timed alone:
    fill = torch.empty((na * 32 + 512 * 1024), dtype=torch.uint8, device=dev)
    fill_ms = []
    for _ in range(50):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fill.zero_()
        fill[: nb * 32 + 512 * 1024].zero_()
        e1.record()
        e1.synchronize()
        fill_ms.append(e0.elapsed_time(e1))
    value = sum(ms) / len(ms)
    lay = R.layout_for(W, H, 8)
    return {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": value, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "impl": "reference",
        "data": "synthetic (same generator and seed as the library arm)",
        "config": pair_config(int(lay["n"]), na, nb),
        "impl_detail": {"api": "Orbor::detectAndCompute A and B, Orbor::match A->B (orb.cpp:57-113)",
                        "harness_zero_fill_ms_est": statistics.median(fill_ms),
                        "note": "includes the harness's zero-fill of each descriptor allocation and its guards; "
                                "harness_zero_fill_ms_est is that fill's cost per pair, timed alone"},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": "ms", "cores": 1, "kind": "reference",
                         "sample": f"{steps} pairs through the reference CUDA build (its orbd.cu/orb.cpp compiled "
                                   f"for sm_100a, oracle/_ref) on cuda:{local}; the reference has no CPU "
                                   f"implementation of the path, so its own GPU build is the arm"},
        "clocks": clocks,
    }


def run_match_workload(args, world, rank, local):
    """k = 2 Hamming matching only: 65536 queries x 65536 database rows (uniform
    256-bit rows, half the queries near-duplicates with p = 0.05 bit flips), L2
    flushed before each step; metric match-pairs/s."""
    import torch

    import orbx
    import synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dbh, qh, _ = synth.match_workload(65536, 65536, seed=rank)
    q = torch.from_numpy(qh).to(dev)
    db = torch.from_numpy(dbh).to(dev)
    stream = torch.cuda.Stream(device=dev)
    ctx = orbx.Context(local, orbx.make_params(max_pts=1000), stream=stream)
    mode = orbx.MATCH_IMMA if args.match_mode == "imma" else orbx.MATCH_POPC
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    steps = max(1, min(args.steps, 200))
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            orbx.knn2(ctx, q, db, mode)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        barrier(world)
        torch.cuda.synchronize(dev)
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            orbx.knn2(ctx, q, db, mode)
            e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
    total_ms = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in ev), world)
    ctx.close()
    if rank != 0:
        return None
    pairs = 65536.0 * 65536.0 * world
    peaks, peak_kind = load_peaks()
    ms1 = total_ms / steps
    if mode == orbx.MATCH_IMMA:
        # 512 int8 ops per pair (256 multiply-adds); the dense int8 rate is twice bf16
        ach = 65536.0 * 65536.0 * 512 / (ms1 * 1e-3) / 1e12
        roof = {"kernel": "k_match_imma", "bound": "tensor", "achieved": ach, "peak": 2 * peaks["bf16_tflops"],
                "unit": "TOP/s (int8)", "frac": ach / (2 * peaks["bf16_tflops"]),
                "traffic": NCU_TRAFFIC.get("k_match_imma"),
                "peak_kind": f"{peak_kind}: 2 x bf16_tflops (int8 dense rate is twice bf16)"}
    else:
        peak_pairs = SMS * POPC_PER_CLK_PER_SM * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 8
        ach = 65536.0 * 65536.0 / (ms1 * 1e-3)
        roof = {"kernel": "k_match_popc", "bound": "int", "achieved": ach / 1e12, "peak": peak_pairs / 1e12,
                "unit": "Tpairs/s", "frac": ach / peak_pairs, "traffic": None,
                "peak_kind": "derived: 148 SMs x 16 popc/clk x max SM clock / 8 popc per pair"}
    cpu = cpu_baseline_knn2(qh, dbh, budget_s=8.0)
    return {"metric": "Hamming match-pairs/s (exact, k=2, 65536 x 65536)", "value": pairs * steps / (total_ms * 1e-3),
            "unit": "pairs/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": total_ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8" if mode == orbx.MATCH_IMMA else "u32", "data": "synthetic (cuda-orb_b200/synth.py)",
            "config": {"workload": f"k=2 matching 65536 x 65536, {args.match_mode} form",
                       "l2": "flushed before every step"},
            "roofline": roof, "cpu_baseline": cpu,
            "gpu_launches": 3 * steps if mode == orbx.MATCH_IMMA else steps}


def run_batch_workload(args, world, rank, local):
    """64 frame pairs of mixed resolution and caps: detect + describe every image
    and match every pair, either in five shared launches or in one persistent
    launch with a device work queue (each replayed from one CUDA graph), each
    form autotuned; the faster form is the reported value.  Beside it, the
    reference build run pair by pair on the same pairs (rank 0)."""
    import torch

    import orbx
    import synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    layout = synth.batch_layout()
    pairs = []
    for k, (w, h, cap) in enumerate(layout):
        a, b, _ = synth.make_pair(w, h, seed=1000 * rank + k)
        pairs.append((a, b, w, h, cap))
    stream = torch.cuda.Stream(device=dev)
    ctx = orbx.Context(local, orbx.make_params(max_pts=10000), stream=stream)
    pb = orbx.PairBatch(pairs, dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    steps = max(1, min(args.steps, 200))

    def timed(tuning):
        ctx.set_tuning(tuning)
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 3)):
                ctx.batch_pairs(pb)
            ctx.sync()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            barrier(world)
            torch.cuda.synchronize(dev)
            for e0, e1 in ev:
                flush.zero_()
                e0.record(stream)
                ctx.batch_pairs(pb)
                e1.record(stream)
            torch.cuda.synchronize(dev)
            barrier(world)
        ctx.sync()
        return max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in ev), world) / steps

    forms = {}
    with torch.cuda.stream(stream):
        for name, mask in (("five_launch", 1), ("persistent", 2)):
            if args.no_autotune:
                t = ctx.get_tuning()
                t.batch_form = 0 if mask == 1 else 1
                tms = None
            else:
                t, tms = ctx.autotune_pairs_forms(pb, mask, reps=3)
            forms[name] = {"tuning": t.as_dict(), "autotune_ms": tms}
    sampler = ClockSampler(local)
    if rank == 0:
        sampler.start()
    for name in forms:
        forms[name]["ms"] = timed(orbx.Tuning(**forms[name]["tuning"]))
    clocks = sampler.stop() if rank == 0 else None
    best = min(forms, key=lambda k: forms[k]["ms"])
    ms = forms[best]["ms"]
    ctx.set_tuning(orbx.Tuning(**forms[best]["tuning"]))
    with torch.cuda.stream(stream):
        acc = np.zeros(5)
        for _ in range(10):
            flush.zero_()
            acc += ctx.profile_batch(pb)
        stage_ms = acc / 10
        ctx.batch_pairs(pb)
        ctx.sync()
    nkp = 0
    in_bytes = 0
    for i, (a, b, w, h, cap) in enumerate(pairs):
        A, B = pb.outs[i]
        nkp += int(A.count.item()) + int(B.count.item())
        in_bytes += 2 * w * h
    ctx.close()
    if rank != 0:
        return None
    # The reference build is not run on this workload: its angleIC (orbd.cu:1001-1010)
    # reads keypoints up to the raw survivor count when the cap binds, past the
    # points NMS wrote, and on this workload's binding caps that faulted the GPU
    # (illegal memory access reported at orbd.cu:1727).
    ref = {"unavailable": "the reference build reads past its keypoint array when the cap binds "
                          "(angleIC, orbd.cu:1001-1010) and faulted with an illegal memory access on this "
                          "workload; not run again"}
    # algorithmic bytes per batch: every image read once, 28 + 32 bytes out per keypoint
    alg = in_bytes + nkp * 60
    peaks, peak_kind = load_peaks()
    gbs = alg / (ms * 1e-3) / 1e9
    return {"metric": "ms per batch of 64 frame pairs (detect+describe+match)", "value": ms, "unit": "ms",
            "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (cuda-orb_b200/synth.py)",
            "config": {"workload": "64 pairs, resolutions uniform over 320x240..3840x2160, caps U[500,10000]",
                       "pixels": in_bytes, "keypoints": nkp, "l2": "flushed before every step",
                       "form": best},
            "forms": forms,
            "pairs_per_s": 64 * 1000.0 / ms,
            "reference_pair_by_pair": ref,
            "roofline": {"kernel": "whole batch", "bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": gbs / peaks["hbm_gbs"], "algorithmic_bytes": alg,
                         "peak_kind": f"{peak_kind} hbm_gbs"},
            "kernels_five_launch": {k: {"ms": float(v)} for k, v in
                                    zip(["pyramid_blur", "detect", "nms", "describe", "match"], stage_ms)},
            "gpu_launches": (1 if best == "persistent" else 5) * steps, "clocks": clocks}


LEARNED_SIZES = {"db": 1 << 20, "q": 131072, "train": 262144, "cal": 32768}
LEARNED_RECALL = 0.99
LEARNED_CAL_TARGET = 0.992  # calibration target, above the reported bar to cover held-out variance


def learned_view_ids(i, short):
    """Views of learned-proposal image i that are still needed: 0 = query, 1 =
    training (every 3rd image), 2 = calibration (every 24th image)."""
    v = []
    if short["q"]:
        v.append(0)
    if i % 3 == 1 and short["train"]:
        v.append(1)
    if i % 24 == 5 and short["cal"]:
        v.append(2)
    return v


def learned_descriptors(ctx, dev, sizes, workers=None):
    """Pipeline descriptors of the learned-proposal workload: the database from
    images A (1024 x 1024, seeds from synth.LEARNED_IMAGE_SEED), queries from view
    0 of the first images, training and calibration rows from other warped views.
    Images come from a spawned process pool in index order, so the sets are the
    same for every run."""
    import multiprocessing as mp

    import torch

    import orbx
    import synth

    workers = workers or max(1, min(32, len(os.sched_getaffinity(0))))
    got = {k: [] for k in sizes}
    cnt = {k: 0 for k in sizes}
    bufs = orbx.FrameBuffers(MAX_PTS, dev)
    chunk = 4 * workers
    i = 0
    n_images = 0
    with mp.get_context("spawn").Pool(workers) as pool:
        while any(cnt[k] < sizes[k] for k in sizes):
            short = {k: cnt[k] < sizes[k] for k in sizes}
            jobs = [(j, learned_view_ids(j, short)) for j in range(i, i + chunk)]
            if not short["db"]:
                jobs = [jb for jb in jobs if jb[1]]
            for (j, views), (a, vs) in zip(jobs, pool.imap(synth.learned_image_set, jobs)):
                n_images += 1
                for key, img in [("db", a)] + [({0: "q", 1: "train", 2: "cal"}[v], x) for v, x in zip(views, vs)]:
                    if cnt[key] >= sizes[key]:
                        continue
                    t = torch.from_numpy(img).to(dev)
                    orbx.detect_and_compute(ctx, t, 1024, 1024, bufs=bufs)
                    ctx.sync()
                    n = min(int(bufs.count.item()), sizes[key] - cnt[key])
                    got[key].append(bufs.desc[:n].clone())
                    cnt[key] += n
            i += chunk
    return {k: torch.cat(v) for k, v in got.items()}, n_images


def calibrate_margin(margin, correct, target):
    """Smallest margin threshold whose fallback set (margins below it) lifts the
    recall of the calibration queries to at least target."""
    order = np.argsort(margin, kind="stable")
    m = margin[order]
    c = correct[order].astype(np.int64)
    n = len(m)
    suffix = np.concatenate([np.cumsum(c[::-1])[::-1], [0]])  # correct among order[k:]
    k = np.arange(n + 1)
    ok = (k + suffix) >= target * n
    kstar = int(np.argmax(ok))
    return (float(m[kstar]) if kstar < n else float("inf")), kstar / n


def calibrate_fallback(margin, dstar, correct, target, max_dists=None):
    """Fallback rule with the fewest fallbacks that lifts the calibration recall to
    target: a query falls back when its margin is below tau_m or its best probed
    distance is above tau_d.  Returns (tau_m, tau_d, fallback fraction)."""
    n = len(margin)
    best = (float("inf"), 256, 1.0)
    cands = sorted(set(int(x) for x in np.unique(np.minimum(dstar, 256)))) + [256]
    if max_dists is not None:
        cands = list(max_dists)
    for td in cands:
        far = dstar > td
        keep = ~far
        m, c = margin[keep], correct[keep]
        n_far = int(far.sum())
        order = np.argsort(m, kind="stable")
        cs = c[order].astype(np.int64)
        suffix = np.concatenate([np.cumsum(cs[::-1])[::-1], [0]])
        k = np.arange(len(cs) + 1)
        ok = (n_far + k + suffix) >= target * n
        if not ok.any():
            continue
        kstar = int(np.argmax(ok))
        frac = (n_far + kstar) / n
        if frac < best[2]:
            tm = float(m[order][kstar]) if kstar < len(cs) else float("inf")
            best = (tm if kstar > 0 else float("-inf"), td, frac)
    return best


def run_learned_workload(args, world, rank, local, with_cpu=True):
    """Learned-proposal k = 2 search: 131072 queries against 1048576 database
    rows, all pipeline descriptors of synthetic 1024 x 1024 images (queries from
    warped copies).  The MLP index is built and trained on the GPU, its fallback
    margin calibrated on held-out queries for recall@1 >= 0.99, then the search
    is timed against exact int8 tensor-core brute force over the same sets."""
    import torch

    import orbx

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sizes = {k: max(1024, int(v * args.learned_scale)) // 128 * 128 for k, v in LEARNED_SIZES.items()}
    stream = torch.cuda.Stream(device=dev)
    ctx = orbx.Context(local, orbx.make_params(max_pts=MAX_PTS), stream=stream)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    peaks, peak_kind = load_peaks()
    t0 = time.time()
    with torch.cuda.stream(stream):
        data, n_images = learned_descriptors(ctx, dev, sizes)
    gen_s = time.time() - t0
    q, db, train, cal = data["q"], data["db"], data["train"], data["cal"]
    nq, ndb = q.shape[0], db.shape[0]
    steps = max(1, min(args.steps, 50))
    warm = max(args.warmup, 3)

    def timed(fn, n):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        torch.cuda.synchronize(dev)
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            fn()
            e1.record(stream)
        torch.cuda.synchronize(dev)
        return [e0.elapsed_time(e1) for e0, e1 in ev]

    with torch.cuda.stream(stream):
        # exact brute force: the reference's matcher semantics (k = 2 over every row)
        for _ in range(2):
            ex_d, ex_i = orbx.knn2(ctx, q, db, orbx.MATCH_IMMA)
        exact_ms = timed(lambda: orbx.knn2(ctx, q, db, orbx.MATCH_IMMA), min(steps, 5))
        ex_d1 = ex_d[:, 0].cpu().numpy()
        cal_d, _ = orbx.knn2(ctx, cal, db, orbx.MATCH_IMMA)
        cal_d1 = cal_d[:, 0].cpu().numpy()
        # build: clustering + labels + training on the GPU
        label_mode = orbx.LABEL_LISTED if args.learned_labels == "listed" else orbx.LABEL_NEAREST
        lp = orbx.learned_params(synth_train=sizes["train"], flip_lo=0.08, flip_hi=0.2, spill=args.learned_spill,
                                 label_mode=label_mode, epochs=args.learned_epochs)
        tb = time.time()
        index = orbx.LearnedIndex(ctx, db, train, lp)
        build_wall_s = time.time() - tb
        build = index.stats()

        def no_fallback(ix, queries):
            ix.set_margin(float("-inf"))
            ix.set_max_distance(1 << 20)
            dd, _, mm, _ = ix.search(queries)
            torch.cuda.synchronize(dev)
            return dd[:, 0].cpu().numpy(), mm.cpu().numpy()

        # calibrate the fallback rule on held-out queries
        cd, cm = no_fallback(index, cal)
        tau_m, tau_d, cal_fb = calibrate_fallback(cm, cd, cd == cal_d1, LEARNED_CAL_TARGET)
        # proposal alone (no fallback) on the test queries, for the ablation
        qd0, _ = no_fallback(index, q)
        recall_mlp_only = float(np.mean(qd0 == ex_d1))
        index.set_margin(tau_m)
        index.set_max_distance(tau_d)
        dist = torch.empty((nq, 2), dtype=torch.int32, device=dev)
        idx = torch.empty((nq, 2), dtype=torch.int32, device=dev)
        fbc = torch.zeros(1, dtype=torch.int32, device=dev)
        for _ in range(warm):
            index.search_ptr(q, nq, dist, idx, None, fbc)
        sampler = ClockSampler(local)
        sampler.start()
        learned_ms = timed(lambda: index.search_ptr(q, nq, dist, idx, None, fbc), steps)
        clocks = sampler.stop()
        recall = float(np.mean(dist[:, 0].cpu().numpy() == ex_d1))
        n_fb = int(fbc.item())
        prof = np.zeros(5)
        for _ in range(5):
            flush.zero_()
            prof += index.profile_search(q, dist, idx)
        prof /= 5
        probe_pairs = index.probe_pairs()
        # the same search with the XOR-popc rerank, for comparison
        index.set_rerank(orbx.RERANK_POPC)
        prof_popc = np.zeros(5)
        for _ in range(3):
            flush.zero_()
            prof_popc += index.profile_search(q, dist, idx)
        prof_popc /= 3
        index.set_rerank(orbx.RERANK_TENSOR)
        # other operating points of the same index: (calibration target, recall, fallback, ms)
        curve = []
        for tgt in (0.9, 0.95, 0.98):
            tm, td, _ = calibrate_fallback(cm, cd, cd == cal_d1, tgt)
            index.set_margin(tm)
            index.set_max_distance(td)
            ms = statistics.median(timed(lambda: index.search_ptr(q, nq, dist, idx, None, fbc), min(steps, 10)))
            curve.append({"calibration_target": tgt, "recall_at_1": float(np.mean(dist[:, 0].cpu().numpy() == ex_d1)),
                          "fallback_fraction": int(fbc.item()) / nq, "ms": ms})
        index.set_margin(tau_m)
        index.set_max_distance(tau_d)
        # end to end through the public API: queries from pinned host memory, results back to the host
        hq = q.cpu().pin_memory()
        hd = torch.empty((nq, 2), dtype=torch.int32).pin_memory()
        hi = torch.empty((nq, 2), dtype=torch.int32).pin_memory()
        qd = torch.empty_like(q)

        def e2e():
            qd.copy_(hq, non_blocking=True)
            index.search_ptr(qd, nq, dist, idx, None, None)
            hd.copy_(dist, non_blocking=True)
            hi.copy_(idx, non_blocking=True)

        for _ in range(warm):
            e2e()
        e2e_ms = timed(e2e, steps)
        index.close()
        # without training: the same clustering probed by nearest centroids, alone
        # and with the fallback rule calibrated for it the same way, timed alike
        cen = orbx.LearnedIndex(ctx, db, train, orbx.learned_params(epochs=0, spill=args.learned_spill))
        recall_centroid = float(np.mean(no_fallback(cen, q)[0] == ex_d1))
        ccd, ccm = no_fallback(cen, cal)
        c_tm, c_td, c_cal_fb = calibrate_fallback(ccm, ccd, ccd == cal_d1, LEARNED_CAL_TARGET)
        cen.set_margin(c_tm)
        cen.set_max_distance(c_td)
        c_fbc = torch.zeros(1, dtype=torch.int32, device=dev)
        for _ in range(warm):
            cen.search_ptr(q, nq, dist, idx, None, c_fbc)
        cen_ms = timed(lambda: cen.search_ptr(q, nq, dist, idx, None, c_fbc), steps)
        untrained = {"recall_at_1": float(np.mean(dist[:, 0].cpu().numpy() == ex_d1)),
                     "fallback_fraction": int(c_fbc.item()) / nq, "calibration_fallback_fraction": c_cal_fb,
                     "ms": sum(cen_ms) / len(cen_ms)}
        cen.close()
        # the other training target, same data and schedule
        other = orbx.LABEL_NEAREST if label_mode == orbx.LABEL_LISTED else orbx.LABEL_LISTED
        alt = orbx.LearnedIndex(ctx, db, train, orbx.learned_params(synth_train=sizes["train"], flip_lo=0.08,
                                                                    flip_hi=0.2, spill=args.learned_spill,
                                                                    label_mode=other, epochs=args.learned_epochs))
        recall_other_labels = float(np.mean(no_fallback(alt, q)[0] == ex_d1))
        alt.close()
        # non-learned proposal at the same probe budget: random-projection buckets
        lsh = orbx.LearnedIndex(ctx, db, None, orbx.learned_params(proposal=orbx.PROPOSAL_LSH, lsh_bits=12,
                                                                    n_clusters=4096))
        ld, _, _, _ = lsh.search(q)
        for _ in range(2):
            lsh.search(q)
        lsh_ms = timed(lambda: lsh.search(q), min(steps, 10))
        recall_lsh = float(np.mean(ld[:, 0].cpu().numpy() == ex_d1))
        lsh.close()
    ctx.close()
    t_exact = statistics.median(exact_ms)
    t_learned = sum(learned_ms) / len(learned_ms)
    pairs = float(nq) * float(ndb)
    cpu = cpu_baseline_knn2(q.cpu().numpy(), db.cpu().numpy()) if with_cpu else None
    phases = dict(zip(["proposal", "probe_lists", "rerank", "merge", "fallback"], prof.tolist()))
    # Roofline of the dominant phase.  The fallback is exact int8 tensor-core matching
    # (512 ops per pair, bound: twice the measured bf16 rate); the proposal is the MLP
    # (2 * (256 * 512 + 512 * 4096) FLOPs per query, bf16 tensor bound).
    mlp_flop = 2.0 * (256 * 512 + 512 * 4096) * nq
    top = max(("fallback", "proposal", "rerank"), key=lambda k: phases[k])
    if top == "fallback":
        ops = float(n_fb) * ndb * 512.0
        achieved = ops / (phases["fallback"] * 1e-3) / 1e12
        roof = {"kernel": "k_match_imma (exact fallback)", "bound": "tensor", "achieved": achieved,
                "peak": 2.0 * peaks["bf16_tflops"], "unit": "TOP/s (int8)",
                "frac": achieved / (2.0 * peaks["bf16_tflops"]), "traffic": None,
                "peak_kind": f"{peak_kind}: 2 x bf16_tflops (int8 dense rate is twice bf16)"}
    elif top == "rerank":
        ops = float(probe_pairs) * 512.0
        achieved = ops / (phases["rerank"] * 1e-3) / 1e12
        roof = {"kernel": "k_rerank_imma (probe rerank)", "bound": "tensor", "achieved": achieved,
                "peak": 2.0 * peaks["bf16_tflops"], "unit": "TOP/s (int8)",
                "frac": achieved / (2.0 * peaks["bf16_tflops"]), "traffic": None,
                "peak_kind": f"{peak_kind}: 2 x bf16_tflops (int8 dense rate is twice bf16)",
                "algorithmic": "512 int8 ops per scanned (query, row) pair"}
    else:
        achieved = mlp_flop / (phases["proposal"] * 1e-3) / 1e12
        roof = {"kernel": "k_gemm_bf16 (MLP proposal phase)", "bound": "tensor", "achieved": achieved,
                "peak": peaks["bf16_tflops"], "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops"],
                "traffic": None, "peak_kind": f"{peak_kind} bf16_tflops"}
    proposal_tflops = mlp_flop / (phases["proposal"] * 1e-3) / 1e12
    return {"metric": "Hamming match-pairs/s (learned proposal, recall@1 >= 0.99, 131072 x 1048576)",
            "value": pairs / (t_learned * 1e-3), "unit": "pairs/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": t_learned, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16+u32",
            "data": f"synthetic: pipeline descriptors of {n_images} generated 1024x1024 images",
            "config": {"workload": "learned-proposal k=2 search", "queries": nq, "database": ndb,
                       "train_rows": train.shape[0], "calibration_rows": cal.shape[0],
                       "n_clusters": 4096, "hidden": 512, "n_probe": 8, "spill": args.learned_spill,
                       "labels": args.learned_labels, "epochs": args.learned_epochs,
                       "rerank": "int8 tcgen05", "l2": "flushed before every step"},
            "recall_at_1": recall, "recall_target": LEARNED_RECALL,
            "fallback_rule": {"margin_below": tau_m, "distance_above": tau_d},
            "fallback_fraction": n_fb / nq, "calibration_fallback_fraction": cal_fb,
            "exact": {"ms": t_exact, "pairs_per_s": pairs / (t_exact * 1e-3), "form": "int8 tcgen05"},
            "speedup_vs_exact": t_exact / t_learned,
            "operating_points": [dict(c, speedup_vs_exact=t_exact / c["ms"]) for c in curve],
            "ablation": {"recall_mlp_no_fallback": recall_mlp_only,
                         "labels": args.learned_labels, "epochs": args.learned_epochs,
                         "recall_mlp_other_labels_no_fallback": recall_other_labels,
                         "recall_nearest_centroid_no_fallback": recall_centroid,
                         "nearest_centroid_calibrated": dict(untrained, speedup_vs_exact=t_exact / untrained["ms"]),
                         "recall_lsh_no_fallback": recall_lsh,
                         "lsh_ms": statistics.median(lsh_ms), "lsh": "12 random-projection bits, 8 probes"},
            "phases_ms": phases, "proposal_tflops": proposal_tflops, "roofline": roof,
            "rerank": {"pairs_scanned": probe_pairs, "pairs_per_query": probe_pairs / nq,
                       "tensor_pairs_per_s": probe_pairs / (phases["rerank"] * 1e-3),
                       "popc_ms": float(prof_popc[2]),
                       "popc_pairs_per_s": probe_pairs / (float(prof_popc[2]) * 1e-3)},
            "build": build, "build_wall_s": build_wall_s, "generate_s": gen_s,
            "e2e": {"value": pairs / (statistics.median(e2e_ms) * 1e-3), "unit": "pairs/s",
                    "h2d_bytes_per_step": nq * 32, "d2h_bytes_per_step": nq * 16},
            "cpu_baseline": cpu, "peaks": {"kind": peak_kind},
            "gpu_launches": 12 * steps, "clocks": clocks}


def learned_summary(args, world, rank, local):
    """The learned-proposal workload (131072 x 1048576 k = 2 search at recall@1
    >= 0.99) reduced to its headline figures, for the default bench line."""
    la = parse_args(["--workload", "learned", "--steps", str(min(args.steps, 20)), "--warmup", "3"])
    r = run_learned_workload(la, world, rank, local, with_cpu=False)
    keep = ("metric", "value", "unit", "ms_per_step", "recall_at_1", "recall_target", "fallback_fraction",
            "speedup_vs_exact", "exact", "phases_ms", "rerank", "roofline", "ablation", "config", "clocks")
    return {k: r[k] for k in keep if k in r}


def cpu_baseline_knn2(q, db, budget_s=10.0):
    """Exact k = 2 brute force of the oracle's C port (one thread) on a sample of queries."""
    from oracle import oracle as O

    n = 16
    t0 = time.time()
    done = 0
    while time.time() - t0 < budget_s and done < 4096:
        O.knn2(q[done:done + n], db)
        done += n
        n = min(2 * n, 256)
    dt = time.time() - t0
    return {"value": done * float(len(db)) / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
            "sample": f"{done} queries x {len(db)} rows, exact k=2 (oracle/orb_oracle.c)"}


def main(argv=None):
    args = parse_args(argv)
    world, rank, local = dist_setup()
    if args.workload == "learned":
        res = run_learned_workload(args, world, rank, local) if rank == 0 else None
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload in ("match65536", "batch64"):
        res = (run_match_workload if args.workload == "match65536" else run_batch_workload)(args, world, rank, local)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        res = run_reference(args, world, rank, local)
    else:
        res, imgs, outs = run_orbx(args, world, rank, local)
        if rank == 0 and not args.no_learned_bench:
            res["learned_proposal"] = learned_summary(args, world, rank, local)
        if rank == 0 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline_port(*imgs)
            res["parity_report"] = parity_report(imgs[0], imgs[1], *outs)
            res["cpu_opencv"] = cpu_baseline_opencv(*imgs)
            res["cpu_opencv_640x480"] = cpu_baseline_opencv_c0()
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
