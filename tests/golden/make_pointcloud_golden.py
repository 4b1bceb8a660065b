"""Generates tests/golden/ref_pointcloud_160x128.npz: the point cloud of
Publisher::publishPointCloud (publisher.cpp:146-163) evaluated with the
reference's own host arithmetic (oracle/_ref/libqm_ref_host.so, built by
`make -C oracle ref-host` from the reference headers), no GPU needed:

    python tests/golden/make_pointcloud_golden.py OUT_DIR

Input: the reference's upsampled depth of the 160x128 extraction fixture,
with holes (-1), depths on both sides of the 0.1 cut and NaNs planted, its
reference image, and a rigid T_world_ref.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HOST_LIB = os.path.join(ROOT, "oracle", "_ref", "libqm_ref_host.so")


def reference_point_cloud(depth, ref, cam, T):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-host"], check=True)
    L = ctypes.CDLL(HOST_LIB)
    L.qmref_point_cloud.restype = ctypes.c_int
    H, W = depth.shape
    out = np.zeros((H * W, 4), np.float32)
    T = np.ascontiguousarray(T, np.float32).reshape(12)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    n = L.qmref_point_cloud(p(depth), p(ref), W, H, *[ctypes.c_float(v) for v in cam], p(T),
                            p(out))
    return out[:n].copy()


def main(out_dir):
    src = np.load(os.path.join(ROOT, "tests", "golden", "ref_extract_160x128.npz"))
    depth = np.ascontiguousarray(src["dense"], np.float32).copy()
    ref = np.ascontiguousarray(src["ref"], np.uint8)
    cam = tuple(float(v) for v in src["cam"])
    rng = np.random.default_rng(77)
    H, W = depth.shape
    holes = rng.random((H, W)) < 0.2
    depth[holes] = -1.0
    idx = rng.choice(H * W, 64, replace=False)
    flat = depth.reshape(-1)
    flat[idx[:16]] = np.float32(0.1)
    flat[idx[16:32]] = np.nextafter(np.float32(0.1), np.float32(0))
    flat[idx[32:40]] = np.nan
    flat[idx[40:48]] = 0.0
    flat[idx[48:64]] = rng.uniform(0.05, 0.15, 16).astype(np.float32)
    c, s = np.cos(0.3), np.sin(0.3)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]]) @ \
        np.array([[1.0, 0.0, 0.0], [0.0, np.cos(-0.2), -np.sin(-0.2)],
                  [0.0, np.sin(-0.2), np.cos(-0.2)]])
    T = np.concatenate([R, [[1.25], [-0.5], [2.0]]], axis=1).astype(np.float32)
    pts = reference_point_cloud(depth, ref, cam, T)
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "ref_pointcloud_160x128.npz"), depth=depth,
                        ref=ref, cam=np.array(cam, np.float32), T_world_ref=T.reshape(12),
                        points=pts)
    print("points:", len(pts))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
