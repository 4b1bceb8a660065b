"""Generates tests/golden/ref_semidense_160x128.npz by running the
reference's own semi-dense tracker kernels (lsd_semidense.cu, seed_init.cu,
compiled from the reference sources into oracle/_ref/libqm_ref.so by
`make -C oracle ref`) over a seeded synthetic 24-frame sequence, with the
host sequence of SeedMatrix::add_frames (first frame, updates, keyframe
switches).  Needs a GPU:

    python tests/golden/make_semidense_golden.py OUT_DIR

Stores the frames, poses, camera, the per-frame step modes, the debug image
after every frame and the seeds after the last frame.  The reference's
regularisation and hole filling run in place and its propagation and
projection resolve collisions by scheduling, so two runs of the reference
itself may differ in a few pixels.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refbuild  # noqa: E402
from open_quadtree_mapping_b200 import synthetic as syn  # noqa: E402


def main(out_dir):
    W, H, n = 160, 128, 24
    f = 460.0 * W / 752.0
    imgs, Ts, _ = syn.make_sequence(41, n, W=W, H=H, fx=f, fy=f)
    cam = (f, f, W / 2.0, H / 2.0)
    debug, seeds, modes = refbuild.semidense(imgs, Ts, cam)
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "ref_semidense_160x128.npz"),
                        frames=np.asarray(imgs, np.uint8), T_cur_world=np.asarray(Ts, np.float32),
                        cam=np.array(cam, np.float32), modes=modes, debug=debug, seeds=seeds)
    print("modes", modes.tolist(), "projected per frame", [int((d > 0).sum()) for d in debug])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
