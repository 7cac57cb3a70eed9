"""The C++ drop-in API (include/orb.h, include/orbd.h) driven by a compiled
C++ program (tests/cxx/orbor_dropin.cpp) that follows the reference demo's
call sequence and the lower-level orbd.h pipeline on caller-owned buffers.
Both must give exactly what the C ABI gives (which the parity tests pin to
the reference), and the matches must equal the oracle's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import orbx  # noqa: E402
import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "orbor_dropin.cpp")
PT = orbx.ORB_POINT_DTYPE


@pytest.fixture(scope="module")
def dropin_exe(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("cxx") / "orbor_dropin")
    cuda = "/usr/local/cuda"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I",
                           os.path.join(cuda, "include"), SRC, "-o", out, "-L", os.path.dirname(orbx.LIB_PATH),
                           "-lorbx", "-L", os.path.join(cuda, "lib64"), "-lcudart",
                           "-Wl,-rpath," + os.path.dirname(orbx.LIB_PATH), "-Wl,-rpath," + os.path.join(cuda, "lib64")])
    return out


def _read(f, dtype, n):
    a = np.frombuffer(f.read(np.dtype(dtype).itemsize * n), dtype=dtype)
    assert len(a) == n
    return a


def _read_result(f):
    n = int(_read(f, np.int32, 1)[0])
    if n == 0:
        return np.zeros(0, dtype=PT), np.zeros((0, 32), dtype=np.uint8)
    pts = _read(f, PT, n).copy()
    desc = _read(f, np.uint8, 32 * n).reshape(n, 32).copy()
    return pts, desc


@pytest.mark.parametrize("w,h,seed", [(640, 480, 31), (1920, 1080, 32)])
def test_orbor_and_lower_api_dropin(dropin_exe, tmp_path, w, h, seed):
    a, b, _ = synth.make_pair(w, h, seed)
    pa, pb, po = tmp_path / "a.raw", tmp_path / "b.raw", tmp_path / "out.bin"
    a.tofile(pa)
    b.tofile(pb)
    subprocess.check_call([dropin_exe, str(w), str(h), str(pa), str(pb), str(po), "10000"],
                          stdout=subprocess.DEVNULL)
    with open(po, "rb") as f:
        A, dA = _read_result(f)
        B, dB = _read_result(f)
        md = _read(f, np.int32, 2 * len(A)).reshape(-1, 2)
        LA, ldA = _read_result(f)
        LB, ldB = _read_result(f)
    # the C ABI on the same images
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    for img, pts, desc, lpts, ldesc in ((a, A, dA, LA, ldA), (b, B, dB, LB, ldB)):
        bufs = orbx.detect_and_compute(ctx, torch.from_numpy(img).cuda(), w, h)
        ctx.sync()
        cp, cd = bufs.to_host()
        for f_ in ("x", "y", "octave", "score", "angle"):
            assert np.array_equal(pts[f_], cp[f_]), f_
            assert np.array_equal(lpts[f_], cp[f_]), f_
        assert np.array_equal(desc, cd) and np.array_equal(ldesc, cd)
    ctx.close()
    m, d = O.match(dA, dB)
    assert np.array_equal(md[:, 0], m) and np.array_equal(md[:, 1], d)
