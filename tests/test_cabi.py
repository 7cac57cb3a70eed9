"""The C ABI library without a GPU: it loads, exports every symbol that
include/orbx.h declares, and its host-side logic agrees with the oracle."""
import os
import re
import subprocess
import threading

import numpy as np
import pytest

import orbx
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "orbx.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"ORBX_API\s+[\w\s\*]+?\b(orbx_\w+)\s*\(", text)))


def exported_symbols(path=None):
    out = subprocess.check_output(["nm", "-D", "--defined-only", path or orbx.LIB_PATH]).decode()
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_loads():
    assert orbx.version().startswith("orbx")
    assert orbx.status_string(0) == "ok"


def test_exports_every_declared_symbol():
    decl = declared_symbols()
    assert len(decl) >= 15
    exp = exported_symbols()
    missing = [s for s in decl if s not in exp]
    assert not missing, missing


def test_checked_build_exports_every_declared_symbol():
    """The bounds-checked variant (build.py --checked) is a drop-in for the
    normal library: same entry points, and it says which build it is."""
    import ctypes

    path = os.path.join(ROOT, "cuda-orb_b200", "liborbx_checked.so")
    if not os.path.exists(path):
        pytest.fail("liborbx_checked.so not built (python cuda-orb_b200/build.py --checked)")
    exp = exported_symbols(path)
    missing = [s for s in declared_symbols() if s not in exp]
    assert not missing, missing
    assert ctypes.CDLL(path).orbx_bounds_checked() == 1
    assert orbx.lib().orbx_bounds_checked() == (1 if orbx.CHECKED else 0)


def test_cxx_api_symbols_exported():
    exp = exported_symbols()
    for sym in ("_ZN3orb5Orbor4initEiiiNS_9ScoreTypeEiiii", "_ZN3orb5Orbor16detectAndComputeEPhRNS_7OrbDataE4int3PPvb",
                "_ZN3orb5Orbor5matchERNS_7OrbDataES2_PhS3_", "_ZN3orb19hFastDectectWithNMSEPhS0_PfRNS_7OrbDataEPiiiib",
                "_ZN3orb6hMatchERNS_7OrbDataES1_PhS2_"):
        assert sym in exp, sym


@pytest.mark.parametrize("w,h", [(320, 240), (640, 480), (1920, 1080), (3840, 2160), (1280, 720), (1024, 1024),
                                 (333, 257), (80, 80), (5000, 4000)])
def test_layout_matches_oracle(w, h):
    n_o, oszp_o = O.layout(w, h)
    if n_o > 5:
        with pytest.raises(orbx.OrbxError):
            orbx.layout(w, h)
        return
    n, oszp = orbx.layout(w, h)
    assert n == n_o and np.array_equal(oszp, oszp_o)


def test_layout_rejects_tiny_images():
    with pytest.raises(orbx.OrbxError) as e:
        orbx.layout(79, 300)
    assert e.value.status == 3


def test_pi_fold_exhaustive():
    """(float)(M_PI - (double)r) computed in integer arithmetic, for every float
    r in [0, 2), equals the double computation (dFastAtan2, orbd.cu:995)."""
    L = orbx.lib()
    nt = 8
    res = [None] * nt
    top = 0x40000000

    def run(i):
        res[i] = L.orbx_selftest_pi_minus(i * (top // nt), (i + 1) * (top // nt))

    th = [threading.Thread(target=run, args=(i,)) for i in range(nt)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert sum(res) == 0


def test_create_without_gpu_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    with pytest.raises(orbx.OrbxError) as e:
        orbx.Context(0)
    assert e.value.status == 2


def test_every_binding_call_has_argtypes():
    """Each C entry point the Python binding calls declares its argument types:
    without them ctypes passes Python ints as 32-bit C ints, truncating pointers."""
    src = open(os.path.join(os.path.dirname(__file__), "..", "cuda-orb_b200", "orbx.py")).read()
    called = set(re.findall(r"lib\(\)\.(orbx_\w+)\(", src)) | set(re.findall(r"\bL\.(orbx_\w+)\(", src))
    typed = set(re.findall(r"L\.(orbx_\w+)\.argtypes", src))
    no_args = {"orbx_version"}  # takes no arguments
    assert called - typed - no_args == set()
