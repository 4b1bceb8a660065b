"""Generates the golden fixtures of tests/golden/ by running the reference's
own CUDA kernels (oracle/_ref/libqm_ref.so, built from the reference sources
by `make -C oracle ref`) on seeded synthetic inputs.  Needs a GPU:

    python tests/golden/make_golden.py OUT_DIR

Each fixture stores the inputs (u8 images, poses, camera) and the reference
outputs: quadtree levels, cost volume, winning labels (recovered from the
final BP messages with the reference's argmin tie rule), sparse BP depths,
upsampled depth, and for the fusion fixture two fusion steps.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refbuild  # noqa: E402
from oracle.oracle import slots_from_ring  # noqa: E402
from open_quadtree_mapping_b200 import synthetic as syn  # noqa: E402


def extract_case(stream, W, H, keep_messages):
    f = 460.0 * W / 752.0
    kf = syn.make_keyframe(stream, W=W, H=H, fx=f, fy=f, F=11)
    cam = (kf.fx, kf.fy, kf.cx, kf.cy)
    r = refbuild.extract(kf.ref, kf.meas, kf.T_meas_ref, cam, nslots=5)
    labels = refbuild.labels_from_messages(r["cost"], r["messages"], r["levels"], W, H)
    used = int(max(slots_from_ring(5))) + 1
    out = dict(ref=kf.ref, ring=kf.meas[:used], T_ring_ref=kf.T_meas_ref[:used],
               cam=np.array(cam, np.float32), slots=np.array(slots_from_ring(5), np.int32),
               levels=r["levels"].astype(np.uint8), cost=r["cost"], labels=labels,
               sparse=r["sparse"], dense=r["dense"])
    if keep_messages:
        out["messages"] = r["messages"]
    return out, kf


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    small, _ = extract_case(31, 64, 48, keep_messages=True)
    np.savez_compressed(os.path.join(out_dir, "ref_extract_64x48.npz"), **small)
    mid, kf = extract_case(32, 160, 128, keep_messages=False)
    np.savez_compressed(os.path.join(out_dir, "ref_extract_160x128.npz"), **mid)
    # fusion: two steps on the mid case's upsampled depth
    cam = tuple(mid["cam"])
    seeds0 = np.zeros((128, 160, 4), np.float32)
    T1 = np.eye(3, 4, dtype=np.float32).reshape(12)
    d1, s1, t1 = refbuild.fuse(mid["dense"], seeds0, T1, cam)
    T2 = np.eye(3, 4, dtype=np.float32)
    T2[0, 3] = 0.03
    T2[2, 3] = -0.02
    d2, s2, t2 = refbuild.fuse(mid["dense"], s1, T2.reshape(12), cam)
    np.savez_compressed(os.path.join(out_dir, "ref_fuse_160x128.npz"), dense=mid["dense"],
                        cam=mid["cam"], T1=T1, T2=T2.reshape(12), fused1=d1, seeds1=s1,
                        table1=t1, fused2=d2, seeds2=s2, table2=t2)
    # larger case: level map, labels, sparse and dense only
    big, _ = extract_case(33, 320, 240, keep_messages=False)
    del big["cost"]
    np.savez_compressed(os.path.join(out_dir, "ref_extract_320x240.npz"), **big)
    print("wrote", sorted(os.listdir(out_dir)))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
