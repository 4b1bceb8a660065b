"""GPU parity of the stage entry points (through the C-ABI) against the oracle.

IEEE arithmetic mode: levels, costs, final BP messages, labels and sparse
depths are bit-exact with the fp32 oracle; the upsampled depth (FP64
elimination on the GPU) is within 1e-5 relative of the fp32 oracle and
within 2e-6 of the fp64 oracle; the fused depth (FP64 update) within 1e-6 of
the fp64 oracle.  Reference arithmetic mode (fast-math, the default): levels
exact, costs/labels agree except at projections within a fast-math error of
a rounding boundary.
"""
import numpy as np
import pytest
import torch

from conftest import cam_of, keyframe
from open_quadtree_mapping_b200.params import ARITH_IEEE, ARITH_REFERENCE, Params

pytestmark = pytest.mark.gpu

UPSAMPLE_RTOL_F32 = 1e-5   # vs the fp32 oracle (the reference's order)
UPSAMPLE_RTOL_F64 = 2e-6   # vs the fp64 oracle
FUSE_RTOL_F64 = 1e-6


def _gpu_extract(kf, p, gpu, slots=None, T=None):
    from open_quadtree_mapping_b200 import stages
    ref = torch.from_numpy(kf.ref).to(gpu)
    slots = kf.meas if slots is None else slots
    T = kf.T_meas_ref if T is None else T
    s = [torch.from_numpy(np.ascontiguousarray(m)).to(gpu) for m in slots]
    g = stages.extract_depth(ref, s, T, cam_of(kf), p, want_messages=True)
    torch.cuda.synchronize()
    return {k: (v.cpu().numpy() if v is not None else None) for k, v in g.items()}


CASES = [
    # W, H, D, F, stream
    (160, 128, 64, 5, 3),
    (752, 480, 64, 5, 0),
    (320, 240, 48, 3, 4),
    (320, 240, 96, 2, 5),
    (256, 192, 128, 1, 6),
    (256, 192, 32, 10, 7),
]


@pytest.mark.parametrize("W,H,D,F,stream", CASES)
def test_ieee_bit_exact_vs_oracle(W, H, D, F, stream, oracle_mod, gpu):
    kf = keyframe(stream, W, H, F)
    p = Params.for_range(D, 0.5, 50.0, arith=ARITH_IEEE)
    g = _gpu_extract(kf, p, gpu)
    o = oracle_mod.extract_depth(kf.ref, kf.meas, kf.T_meas_ref, cam_of(kf), p,
                                 want_messages=True)
    assert np.array_equal(g["levels"], o["levels"])
    assert np.array_equal(g["cost"], o["cost"])
    assert np.array_equal(g["messages"], o["messages"])
    assert np.array_equal(g["labels"], o["labels"])
    assert np.array_equal(g["sparse"], o["sparse"])
    d32 = o["dense"]
    d64 = oracle_mod.upsample(o["sparse"].astype(np.float64), kf.ref, p)
    assert np.allclose(g["dense"], d32, rtol=UPSAMPLE_RTOL_F32, atol=0)
    assert np.allclose(g["dense"], d64, rtol=UPSAMPLE_RTOL_F64, atol=0)


@pytest.mark.parametrize("W,H,D,F,stream", CASES[:2])
def test_reference_mode_agrees_with_oracle(W, H, D, F, stream, oracle_mod, gpu):
    kf = keyframe(stream, W, H, F)
    p = Params.for_range(D, 0.5, 50.0, arith=ARITH_REFERENCE)
    g = _gpu_extract(kf, p, gpu)
    o = oracle_mod.extract_depth(kf.ref, kf.meas, kf.T_meas_ref, cam_of(kf), p)
    assert np.array_equal(g["levels"], o["levels"])
    # fast-math divisions differ from IEEE in the last bits; a rounded
    # projection near a .5 boundary changes one SAD term
    close = np.isclose(g["cost"], o["cost"], rtol=1e-6, atol=1e-9).mean()
    assert close > 0.999, close
    node = o["labels"] >= 0
    assert np.array_equal(g["labels"] >= 0, node)
    agree = (g["labels"][node] == o["labels"][node]).mean()
    assert agree > 0.99, agree


def test_quadtree_odd_sizes(oracle_mod, gpu):
    from open_quadtree_mapping_b200 import stages
    rng = np.random.default_rng(11)
    for (H, W) in [(1080 // 4, 1920 // 4), (37, 53), (8, 8), (100, 30)]:
        base = rng.integers(0, 40, (H, W)).astype(np.uint8)
        img = np.where(rng.random((H, W)) < 0.02, 255, base).astype(np.uint8)
        for p in (Params(), Params(qt_max_level=5, qt_min_level=0), Params(qt_threshold=3.5)):
            lv = stages.quadtree(torch.from_numpy(img).to(gpu), p).cpu().numpy()
            assert np.array_equal(lv, oracle_mod.quadtree(img, p))


def test_all_slots_out_of_view_and_identity(oracle_mod, gpu):
    kf = keyframe(3, 160, 128, 2)
    p = Params.for_range(64, 0.5, 50.0, arith=ARITH_IEEE)
    far = np.eye(3, 4, dtype=np.float32)
    far[0, 3] = 1e4
    ident = np.eye(3, 4, dtype=np.float32)
    T = np.stack([far.reshape(12), ident.reshape(12)])
    g = _gpu_extract(kf, p, gpu, slots=[kf.meas[0], kf.ref], T=T)
    o = oracle_mod.extract_depth(kf.ref, [kf.meas[0], kf.ref], T, cam_of(kf), p,
                                 want_messages=True)
    assert np.array_equal(g["cost"], o["cost"])
    assert np.array_equal(g["labels"], o["labels"])


def test_textureless_image(oracle_mod, gpu):
    """A flat image: every pixel at the top quadtree level, few nodes."""
    kf = keyframe(3, 160, 128, 3)
    flat = np.full_like(kf.ref, 90)
    p = Params.for_range(64, 0.5, 50.0, arith=ARITH_IEEE)
    g = _gpu_extract(kf, p, gpu, slots=[flat] * 3)
    from open_quadtree_mapping_b200 import stages
    lv = stages.quadtree(torch.from_numpy(flat).to(gpu), p).cpu().numpy()
    assert (lv == 4).all()
    assert np.isfinite(g["dense"]).all()


def test_fuse_vs_oracle(oracle_mod, gpu):
    """Twenty fusion steps on a real keyframe (nineteen static, then a small
    motion): table bit-exact (IEEE transform), fused depth and seeds within
    FP64 tolerance of the oracle's FP64 update on the same float seeds.  The
    first outputs are all -1: the prior inlier ratio starts at 0.5 and only
    passes 0.6 after ~15 consistent updates (depth_fusion.cu:175-210)."""
    from open_quadtree_mapping_b200 import stages
    kf = keyframe(3, 160, 128, 3)
    p = Params.for_range(64, 0.5, 50.0, arith=ARITH_IEEE)
    cam = cam_of(kf)
    o = oracle_mod.extract_depth(kf.ref, kf.meas, kf.T_meas_ref, cam, p)
    dense = o["dense"].astype(np.float32)
    seeds = np.zeros((128, 160, 4), np.float32)
    valid = []
    for step in range(20):
        T = np.eye(3, 4, dtype=np.float32)
        if step == 19:
            T[0, 3] = 0.02
        T = T.reshape(12)
        gd, _, gs, gt = stages.fuse(torch.from_numpy(dense).to(gpu),
                                    torch.from_numpy(seeds).to(gpu), T, cam, p)
        od, os_, ot, _ = oracle_mod.fuse(dense.astype(np.float64), seeds, T, cam)
        assert np.array_equal(gt.cpu().numpy(), ot), step
        gd = gd.cpu().numpy()
        assert np.array_equal(gd > 0, od > 0), step
        assert np.allclose(gd, od, rtol=FUSE_RTOL_F64), step
        gs = gs.cpu().numpy()
        assert np.allclose(gs, os_, rtol=FUSE_RTOL_F64, atol=1e-9), step
        valid.append((gd > 0).mean())
        seeds = gs
    assert valid[0] == 0.0
    assert max(valid) > 0.3, valid


_UPSAMPLE_CHILD = r"""
import sys, numpy as np, torch
from open_quadtree_mapping_b200 import stages
from open_quadtree_mapping_b200.params import ARITH_IEEE, Params
z = np.load(sys.argv[1])
dev = torch.device("cuda:0")
d = stages.upsample(torch.from_numpy(z["sparse"]).to(dev), torch.from_numpy(z["img"]).to(dev),
                    Params(arith=ARITH_IEEE))
np.save(sys.argv[2], d.cpu().numpy())
"""


def _sparse_case(W, H, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:H, 0:W]
    img = (128 + 60 * np.sin(xx / 37.0) * np.cos(yy / 23.0)
           + rng.normal(0, 8, (H, W))).clip(0, 255).astype(np.uint8)
    sparse = np.where(rng.random((H, W)) < 0.05, rng.uniform(0.5, 20.0, (H, W)), 0.0)
    return img, sparse.astype(np.float32)


def test_upsample_long_lines_in_fresh_process(oracle_mod, gpu, tmp_path):
    """Lines of 1280 and 720 samples need more than 48 KB of dynamic shared
    memory: the stage call must opt in by itself, in a process where no depth
    engine was ever created."""
    import subprocess
    import sys
    W, H = 1280, 720
    img, sparse = _sparse_case(W, H, 5)
    np.savez(tmp_path / "in.npz", img=img, sparse=sparse)
    root = str(__import__("pathlib").Path(__file__).resolve().parents[1])
    subprocess.run([sys.executable, "-c", _UPSAMPLE_CHILD, str(tmp_path / "in.npz"),
                    str(tmp_path / "out.npy")], check=True, cwd=root, timeout=300)
    g = np.load(tmp_path / "out.npy")
    p = Params(arith=ARITH_IEEE)
    d64 = oracle_mod.upsample(sparse.astype(np.float64), img, p)
    assert np.allclose(g, d64, rtol=UPSAMPLE_RTOL_F64, atol=0)


def test_invalid_arguments_are_rejected(gpu):
    import ctypes
    from open_quadtree_mapping_b200 import _lib
    L = _lib.lib()
    p = _lib.default_params()
    assert L.qm_quadtree(None, 0, 4, 4, ctypes.byref(p), None, None) == _lib.QM_ERR_INVALID_ARG
    p.num_hyp = 50
    buf = torch.zeros(64 * 64, dtype=torch.uint8, device=gpu)
    assert L.qm_quadtree(ctypes.c_void_p(buf.data_ptr()), 64, 64, 64, ctypes.byref(p),
                         ctypes.c_void_p(buf.data_ptr()), None) == _lib.QM_ERR_INVALID_ARG
    assert "num_hyp" in _lib.last_error()
    p = _lib.default_params()
    nbytes = ctypes.c_size_t()
    assert L.qm_bp_workspace_size(64, 64, ctypes.byref(p), ctypes.byref(nbytes)) == 0
    assert L.qm_bp_extract(ctypes.c_void_p(buf.data_ptr()), 64, 64, ctypes.c_void_p(buf.data_ptr()),
                           ctypes.byref(p), ctypes.c_void_p(buf.data_ptr()), None, None,
                           ctypes.c_void_p(buf.data_ptr()), 16, None) == _lib.QM_ERR_WORKSPACE


@pytest.mark.parametrize("arith", [ARITH_IEEE, ARITH_REFERENCE])
def test_cost_volume_into_unaligned_buffer(arith, gpu):
    """The cost kernel stores four hypotheses at a time where the output is
    16-byte aligned and one at a time where it is not; a caller's buffer
    offset by one float gets the same volume as an aligned one."""
    from open_quadtree_mapping_b200 import stages
    kf = keyframe(2, 320, 240, 4)
    p = Params.for_range(48, 0.5, 50.0, arith=arith)
    ref = torch.from_numpy(kf.ref).to(gpu)
    slots = [torch.from_numpy(np.ascontiguousarray(m)).to(gpu) for m in kf.meas]
    levels = stages.quadtree(ref, p)
    aligned = stages.cost_volume(ref, levels, slots, kf.T_meas_ref, cam_of(kf), p)
    shape = tuple(aligned.shape)
    buf = torch.full((aligned.numel() + 1,), float("nan"), dtype=torch.float32, device=gpu)
    view = buf[1:].view(shape)
    assert view.data_ptr() % 16 == 4
    got = stages.cost_volume(ref, levels, slots, kf.T_meas_ref, cam_of(kf), p, out=view)
    torch.cuda.synchronize()
    assert got.data_ptr() == view.data_ptr()
    assert torch.isnan(buf[0])
    assert torch.equal(got, aligned)
