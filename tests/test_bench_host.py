"""Host-side logic of bench.py without a GPU: the multi-rank plumbing on
gloo (world size 2, 127.0.0.1), the per-kernel work model and the clock
parser."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    # per-rank step times differ; the job time is the slowest rank
    t_max = bench.max_over_ranks(10.0 + 5.0 * rank, w)
    t_sum = bench.sum_over_ranks(1.0, w)
    out[rank] = (t_max, t_sum)
    import torch.distributed as dist

    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_gloo_world2():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert out[0] == out[1] == (15.0, 2.0)


def test_single_rank_helpers():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.sum_over_ranks(2.0, 1) == 2.0


def test_stage_work_1080p():
    import orbx

    n, oszp = orbx.layout(1920, 1080, 8)
    work = bench.stage_work(oszp, n, 1000, 1200)
    assert work["pyramid_blur"] == 2 * (1080 * 1920 + 2 * 2799360)
    assert work["detect"] == 2 * (2799360 + 1080 * 1920 // 8) + 2200 * 5
    assert work["nms"] == 2 * (1080 * 1920 // 8) + 2200 * 33
    assert work["describe"] == 2200 * (28 + 961 + 512 + 36)


def test_clock_sampler_parses_reasons(monkeypatch):
    class FakeProc:
        def terminate(self):
            pass

        def communicate(self, timeout=None):
            rows = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
                    "0, 1890, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
                    "0, 1900, 1965, 995.2, 0x4, Not Active, Not Active, Not Active, Active"]
            return "\n".join(rows) + "\n", ""

    s = bench.ClockSampler(0)
    s.proc = FakeProc()
    c = s.stop()
    assert c["samples"] == 3 and c["sm_mhz"] == 1900.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]


def test_peaks_file_or_fallback():
    pk, kind = bench.load_peaks()
    assert kind in ("measured", "fallback")
    assert pk["hbm_gbs"] > 1000


def test_calibrate_margin():
    # 10 queries; the proposal is wrong on the three with the smallest margins
    margin = np.array([0.1, 5.0, 0.2, 3.0, 4.0, 0.3, 6.0, 7.0, 8.0, 9.0])
    correct = np.array([0, 1, 0, 1, 1, 0, 1, 1, 1, 1], dtype=bool)
    tau, frac = bench.calibrate_margin(margin, correct, 0.99)
    assert tau == 3.0 and frac == 0.3      # the three wrong ones fall back
    tau, frac = bench.calibrate_margin(margin, correct, 0.7)
    assert tau == 0.1 and frac == 0.0      # already at 0.7
    tau, frac = bench.calibrate_margin(margin, np.zeros(10, dtype=bool), 0.99)
    assert tau == float("inf") and frac == 1.0


def test_learned_view_ids():
    short = {"db": True, "q": True, "train": True, "cal": True}
    assert bench.learned_view_ids(1, short) == [0, 1]
    assert bench.learned_view_ids(6, short) == [0]
    assert bench.learned_view_ids(5, short) == [0, 2]
    short["q"] = False
    assert bench.learned_view_ids(4, short) == [1]


def test_calibrate_fallback_uses_distance():
    # wrong answers all have a large best distance but ordinary margins
    rng = np.random.Generator(np.random.PCG64(3))
    n = 1000
    margin = rng.uniform(0, 10, n)
    dstar = rng.integers(10, 40, n)
    correct = np.ones(n, dtype=bool)
    bad = rng.choice(n, 50, replace=False)
    correct[bad] = False
    dstar[bad] = rng.integers(60, 80, 50)
    tm, td, frac = bench.calibrate_fallback(margin, dstar, correct, 0.99)
    # only wrong answers need to fall back: at most the 5% that are wrong, all by distance
    assert td >= 40 and frac <= 0.05 + 1e-9
    fb = (margin < tm) | (dstar > td)
    assert (fb.sum() + (correct & ~fb).sum()) / n >= 0.99


def test_bench_names_are_defined():
    """Every name bench.py reads is defined, imported or a builtin (a guard
    against a definition lost in an edit; the bench only runs on a GPU box)."""
    import ast
    import builtins

    src = open(os.path.join(os.path.dirname(__file__), "..", "bench.py")).read()
    tree = ast.parse(src)
    defined = {n.id for n in ast.walk(tree) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Store)}
    defined |= {n.name for n in ast.walk(tree) if isinstance(n, (ast.FunctionDef, ast.ClassDef))}
    defined |= {a.asname or a.name.split(".")[0] for n in ast.walk(tree) if isinstance(n, (ast.Import, ast.ImportFrom))
                for a in n.names}
    defined |= {a.arg for n in ast.walk(tree) if isinstance(n, ast.arguments) for a in n.args + n.kwonlyargs}
    used = {n.id for n in ast.walk(tree) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load)}
    assert sorted(u for u in used - defined if not hasattr(builtins, u) and u != "__file__") == []
