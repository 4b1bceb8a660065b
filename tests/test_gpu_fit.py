"""Fitting the BP penalties and the per-pixel upsampling weight factors to
ray-cast ground truth (the differentiable configuration: 8 keyframes of
752x480, 64 hypotheses, 5 measurement frames, readout temperature 0.05, L1
loss on the fused depth): a few Adam steps lower the loss."""
import numpy as np
import pytest
import torch

from conftest import cam_of, keyframe
from open_quadtree_mapping_b200.params import Params

pytestmark = pytest.mark.gpu


def test_fit_lowers_l1_loss(gpu):
    from open_quadtree_mapping_b200 import diff
    W, H = 752, 480
    p = Params.for_range(64, 0.5, 50.0)
    rng = np.random.default_rng(3)
    kfs = []
    for s in range(8):
        kf = keyframe(20 + s, W, H, 5)
        gt = kf.gt_depth.astype(np.float32)
        seeds = np.zeros((H, W, 4), np.float32)
        seeds[..., 0], seeds[..., 1] = 30.0, 5.0
        seeds[..., 2] = gt * (1.0 + 0.05 * rng.standard_normal((H, W)))
        seeds[..., 3] = 4.0
        kfs.append(diff.Keyframe(
            ref=torch.from_numpy(kf.ref).to(gpu),
            slots=[torch.from_numpy(np.ascontiguousarray(m)).to(gpu) for m in kf.meas],
            T_slot_ref=kf.T_meas_ref, cam=cam_of(kf),
            seeds=torch.from_numpy(seeds).to(gpu),
            T_fuse=np.eye(3, 4, dtype=np.float32).reshape(12),
            gt=torch.from_numpy(gt).to(gpu)).prepare(p))
    pen, omegas, hist = diff.fit(kfs, p, steps=8)
    assert all(np.isfinite(hist))
    assert hist[-1] < hist[0], hist
    assert torch.all(pen > 0)
    assert all(torch.isfinite(om).all() for om in omegas)
