"""TEST INFRASTRUCTURE ONLY: patched copies of the reference's depth-path
sources for comparator builds at other hypothesis counts and ranges.

The reference compiles its hypothesis count and inverse-depth range in:
DEPTH_NUM 64 (include/quadmap/pixel_cost.cuh:4), MIN_INV_DEPTH 0.01 and
STEP_INV_DEPTH = (MAX - MIN) / 63.0 (include/quadmap/stereo_parameter.cuh:5-7),
and its host code launches the per-hypothesis kernels with 64-thread blocks
(src/bpextract.cu:70, 105, 123; the cost launches live in the replay driver).
A variant `d<N>_lo<MIN>` copies the sources the comparator includes into an
output tree (never into the repository) and changes exactly these:

* DEPTH_NUM -> N, MIN_INV_DEPTH -> MIN, the step's divisor 63.0 -> N - 1;
* bp_extract's message-upsampling and BP blocks take DEPTH_NUM threads
  instead of 64;
* cost_distribute reads its hypothesis from threadIdx.z + blockIdx.z *
  blockDim.z and bp_extract launches DEPTH_NUM / 64 blocks in z (a block may
  have at most 64 threads in z); for N = 64 this is the reference's launch.

Every substitution must match the expected number of times, otherwise the
script fails: a changed reference tree is reported, never half-patched.

    python oracle/refpatch.py --ref <reference tree> --variant d128_lo0.02 --out <dir>
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import sys

SOURCES = ["seed_init.cu", "lsd_semidense.cu", "quadtree.cu", "depth_extract.cu", "bpextract.cu",
           "depth_upsample.cu", "depth_fusion.cu"]
HEADERS = ["pixel_cost.cuh", "stereo_parameter.cuh"]


def parse_variant(v):
    m = re.fullmatch(r"d(\d+)_lo([0-9.]+)", v)
    if not m:
        raise SystemExit("variant must look like d128_lo0.02, got %r" % v)
    n = int(m.group(1))
    if n < 2 or n & (n - 1) or n > 1024:
        raise SystemExit("the reference's tree reductions need a power-of-two DEPTH_NUM")
    return n, m.group(2)


def sub(text, old, new, count, what):
    found = text.count(old)
    if found != count:
        raise SystemExit("refpatch: %s: expected %d occurrence(s) of %r, found %d"
                         % (what, count, old, found))
    return text.replace(old, new)


def patch(ref, variant, out):
    n, lo = parse_variant(variant)
    inc = os.path.join(out, "include", "quadmap")
    src = os.path.join(out, "src")
    os.makedirs(inc, exist_ok=True)
    os.makedirs(src, exist_ok=True)
    for f in SOURCES:
        shutil.copyfile(os.path.join(ref, "src", f), os.path.join(src, f))
    for f in HEADERS:
        shutil.copyfile(os.path.join(ref, "include", "quadmap", f), os.path.join(inc, f))

    p = os.path.join(inc, "pixel_cost.cuh")
    t = open(p).read()
    t = sub(t, "#define DEPTH_NUM 64", "#define DEPTH_NUM %d" % n, 1, p)
    open(p, "w").write(t)

    p = os.path.join(inc, "stereo_parameter.cuh")
    t = open(p).read()
    t = sub(t, "#define MIN_INV_DEPTH 0.01", "#define MIN_INV_DEPTH %s" % lo, 1, p)
    t = sub(t, "(MAX_INV_DEPTH-MIN_INV_DEPTH)/63.0", "(MAX_INV_DEPTH-MIN_INV_DEPTH)/%d.0" % (n - 1),
            1, p)
    open(p, "w").write(t)

    p = os.path.join(src, "bpextract.cu")
    t = open(p).read()
    t = sub(t, "hier_block.z = 64;", "hier_block.z = 64;\n    hier_grid.z = DEPTH_NUM / 64;", 1, p)
    t = sub(t, "const int depth_id = threadIdx.z;",
            "const int depth_id = threadIdx.z + blockIdx.z * blockDim.z;", 1, p)
    t = sub(t, "message_up_block.x = 64;", "message_up_block.x = DEPTH_NUM;", 1, p)
    t = sub(t, "bp_block.y = 64;", "bp_block.y = DEPTH_NUM;", 1, p)
    open(p, "w").write(t)
    return n, lo


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    ap.add_argument("--variant", required=True)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    n, lo = patch(a.ref, a.variant, a.out)
    print("refpatch: %s -> DEPTH_NUM %d, MIN_INV_DEPTH %s, step divisor %d.0" % (a.out, n, lo, n - 1))


if __name__ == "__main__":
    sys.exit(main())
