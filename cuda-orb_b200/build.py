"""Build liborbx.so (the sm_100a ORB library) in place with nvcc.

    python cuda-orb_b200/build.py [--force] [--checked]

Compiles every CUDA source under csrc/ for sm_100a only and links one shared
library next to this file: the C ABI of include/orbx.h and the C++ API of
include/orb.h / include/orbd.h.  --checked builds the bounds-checked variant
instead, liborbx_checked.so: the same sources with -DORBX_BOUNDS_CHECK, whose
kernels test each global access against its buffer's extent and report the
ones outside it (orbx_bounds_report) instead of making them.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liborbx.so")
LIB_CHECKED = os.path.join(HERE, "liborbx_checked.so")
SOURCES = ["orbx_api.cu", "orbx_detect.cu", "orbx_describe.cu", "orbx_match.cu", "orbx_match_imma.cu",
           "orb_compat.cu", "orbx_static.cu", "orbx_gemm.cu", "orbx_learned.cu", "orbx_learned_api.cu",
           "orbx_hostio.cu", "orbx_ocv.cu", "orbx_persist.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def _inputs():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    files.append(os.path.join(HERE, "..", "include", "orbx.h"))
    files += [os.path.join(HERE, "..", "include", f) for f in ("orb.h", "orbd.h", "orb_structures.h", "cuda_utils.h")]
    return files


def up_to_date(lib=LIB):
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force=False, verbose=False, checked=False):
    lib = LIB_CHECKED if checked else LIB
    if not force and up_to_date(lib):
        return lib
    objdir = os.path.join(HERE, "_build_checked" if checked else "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    flags = FLAGS + (["-DORBX_BOUNDS_CHECK"] if checked else [])
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [NVCC] + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out.decode(errors='replace')}")
    tmp = lib + ".tmp"
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + objs
    subprocess.check_call(cmd)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
