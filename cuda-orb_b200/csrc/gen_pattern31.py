"""Generate ``orb_pattern31.h``: the 256 rBRIEF point pairs for a 31x31 patch.

The descriptor bits are defined by this fixed table (OpenCV's ``bit_pattern_31_``,
which CUDA-ORB embeds at orbd.cu:97-354 and uploads in ``setPattern``,
orbd.cu:95-375).  Bit-exact descriptors need the identical table, so it is read
out of the reference source instead of being retyped, and written in this
project's own compact layout (int8 point pairs, no comments).

Usage:  python gen_pattern31.py path/to/orbd.cu
        (or set ORB_REFERENCE_SRC to the reference's orbd.cu)
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def read_pattern(src_path):
    text = open(src_path, "r", encoding="utf-8", errors="replace").read()
    start = text.index("bit_pattern_31_[256 * 4] = {")
    end = text.index("};", start)
    body = text[start + len("bit_pattern_31_[256 * 4] = {"):end]
    body = re.sub(r"/\*.*?\*/", " ", body, flags=re.S)
    vals = [int(v) for v in re.findall(r"-?\d+", body)]
    if len(vals) != 1024:
        raise ValueError(f"expected 1024 integers, found {len(vals)}")
    return vals


def render(vals):
    lines = [
        "// Generated by gen_pattern31.py -- do not edit.",
        "// 512 sampling points (x, y) of the 256 rBRIEF tests for a 31x31 patch;",
        "// test i compares point 2i against point 2i+1.",
        "#pragma once",
        "static const signed char kOrbPattern31[512][2] = {",
    ]
    for i in range(0, 1024, 16):
        chunk = vals[i:i + 16]
        pairs = ", ".join(f"{{{chunk[j]},{chunk[j + 1]}}}" for j in range(0, 16, 2))
        lines.append("    " + pairs + ",")
    lines.append("};")
    return "\n".join(lines) + "\n"


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ORB_REFERENCE_SRC")
    if not src:
        sys.exit("usage: gen_pattern31.py path/to/orbd.cu (or set ORB_REFERENCE_SRC)")
    vals = read_pattern(src)
    out = os.path.join(HERE, "orb_pattern31.h")
    with open(out, "w") as f:
        f.write(render(vals))
    print(f"wrote {out} ({len(vals) // 2} points)")


if __name__ == "__main__":
    main()
