"""Poses that are not rigid transforms are rejected before any work.

The cost kernel gathers measurement pixels without clamping: it relies on
every measurement pose being finite with bounded rotation rows (|r00| +
|r01| <= 1.5 and |r10| + |r11| <= 1.5, which every rotation satisfies), so
that the rotated 3x3 patch of a projection that passed the bounds test stays
inside the image.  The C-ABI checks this on the host: qm_cost_volume for its
slot poses, qm_depthmap_add_frame / qm_batch_add_frames / qm_batch_submit
for the frame poses the slot poses are made from.  A rejected call returns
QM_ERR_INVALID_ARG, launches nothing and changes no state: a stream fed a
bad pose in between continues exactly like a twin that never saw it.
"""
import ctypes

import numpy as np
import pytest

from conftest import has_gpu, sequence
from open_quadtree_mapping_b200 import _lib
from open_quadtree_mapping_b200.params import Params, QmParamsC

W, H = 160, 128
F_PX = 460.0 * W / 752.0


def _bad_poses(T):
    """NaN, +inf, -inf, a rotation scaled by 2 and a shear, each derived from
    a good world->camera (or slot) pose T (12 floats)."""
    out = []
    for k, v in ((3, np.nan), (5, np.inf), (10, -np.inf)):
        b = np.array(T, np.float32).reshape(12)
        b[k] = v
        out.append(b)
    b = np.array(T, np.float32).reshape(12)
    b[[0, 1, 2, 4, 5, 6, 8, 9, 10]] *= 2.0
    out.append(b)
    # a shear that lifts |r00| + |r01| above the bound, whatever the rotation
    b = np.array(T, np.float32).reshape(12)
    b[1] += np.float32(1.6) * (np.float32(1.0) if b[1] >= 0 else np.float32(-1.0))
    out.append(b)
    return out


@pytest.mark.skipif(has_gpu(), reason="host-side check without a device; "
                                      "the GPU test below covers the device case")
def test_cost_volume_rejects_bad_slot_poses_on_the_host():
    """Rejected before anything touches the device: without a GPU the call
    still answers QM_ERR_INVALID_ARG (not a CUDA error).  The buffers are
    host memory and are never dereferenced."""
    L = _lib.lib()
    ref = np.zeros((H, W), np.uint8)
    levels = np.full((H, W), 2, np.uint8)
    slot = np.zeros((H, W), np.uint8)
    cost = np.zeros((H // 4, W // 4, 64), np.float32)
    cam = _lib.QmCamera(F_PX, F_PX, W / 2.0, H / 2.0)
    pc = QmParamsC.from_params(Params())
    good = np.eye(3, 4, dtype=np.float32).reshape(12)
    for bad in _bad_poses(good):
        T = np.stack([good, bad, good]).astype(np.float32)
        ptrs = (ctypes.c_void_p * 3)(*[slot.ctypes.data] * 3)
        st = L.qm_cost_volume(ref.ctypes.data, W, W, H, ctypes.byref(cam), levels.ctypes.data,
                              3, ptrs, W, T.ctypes.data, ctypes.byref(pc), cost.ctypes.data,
                              None)
        assert st == _lib.QM_ERR_INVALID_ARG, (bad, L.qm_last_error())
        assert b"rigid" in L.qm_last_error()


@pytest.mark.gpu
def test_cost_volume_rejects_bad_slot_poses(gpu):
    import torch
    from open_quadtree_mapping_b200 import stages
    from conftest import keyframe, cam_of
    kf = keyframe(21, W, H, 11)
    ref = torch.from_numpy(kf.ref).to(gpu)
    levels = stages.quadtree(ref)
    slots = [torch.from_numpy(kf.meas[k]).to(gpu) for k in (0, 0, 1)]
    T = np.array(kf.T_meas_ref[[0, 0, 1]], np.float32)
    good = stages.cost_volume(ref, levels, slots, T, cam_of(kf))
    for bad in _bad_poses(T[2]):
        Tb = T.copy()
        Tb[2] = bad
        with pytest.raises(_lib.QmError) as e:
            stages.cost_volume(ref, levels, slots, Tb, cam_of(kf))
        assert e.value.status == _lib.QM_ERR_INVALID_ARG
    again = stages.cost_volume(ref, levels, slots, T, cam_of(kf))
    assert torch.equal(good, again)


@pytest.mark.gpu
def test_facade_rejects_bad_frame_poses_without_state_change(gpu):
    from open_quadtree_mapping_b200.depthmap import Depthmap
    imgs, Ts, _ = sequence(1, 15, W, H)
    p = Params.for_range(64, 0.5, 50.0)
    dm = Depthmap(W, H, F_PX, W / 2.0, F_PX, H / 2.0, params=p)
    twin = Depthmap(W, H, F_PX, W / 2.0, F_PX, H / 2.0, params=p)
    for i in range(15):
        if i in (0, 6, 13):  # before the first frame, in the ring phase, when dense
            for bad in _bad_poses(Ts[i]):
                with pytest.raises(_lib.QmError) as e:
                    dm.add_frames(imgs[i], bad)
                assert e.value.status == _lib.QM_ERR_INVALID_ARG
        assert dm.add_frames(imgs[i], Ts[i]) == twin.add_frames(imgs[i], Ts[i])
    assert np.array_equal(dm.getDepthmap(), twin.getDepthmap())
    assert np.array_equal(dm.getDebugmap(), twin.getDebugmap())


@pytest.mark.gpu
def test_batch_rejects_a_bad_pose_in_any_stream(gpu):
    """One bad pose among three streams rejects the whole call (add_frames and
    submit alike); no stream advances."""
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    seqs = [sequence(s, 14, W, H) for s in (2, 3, 4)]
    p = Params.for_range(64, 0.5, 50.0)
    desc = dict(width=W, height=H, fx=F_PX, fy=F_PX, cx=W / 2.0, cy=H / 2.0)
    b = BatchDepthmap([desc] * 3, params=p)
    twin = BatchDepthmap([desc] * 3, params=p)
    for i in range(14):
        imgs = [s[0][i] for s in seqs]
        poses = [s[1][i] for s in seqs]
        if i in (0, 12):
            for k in range(3):
                for bad in _bad_poses(poses[k]):
                    bp = list(poses)
                    bp[k] = bad
                    with pytest.raises(_lib.QmError) as e:
                        b.add_frames(imgs, bp)
                    assert e.value.status == _lib.QM_ERR_INVALID_ARG
                    with pytest.raises(_lib.QmError) as e:
                        b.submit(imgs, bp)
                    assert e.value.status == _lib.QM_ERR_INVALID_ARG
        assert b.add_frames(imgs, poses) == twin.add_frames(imgs, poses)
    for k in range(3):
        assert np.array_equal(b.get_depth(k), twin.get_depth(k))
