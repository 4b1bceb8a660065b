"""qm_upsample_noalloc (static device scratch, no workspace) against
qm_upsample (caller workspace), both through the C-ABI.

Both entry points launch the same row and column solvers, so their outputs
agree to the last bit; the tolerance below (1e-6 relative) only leaves room
for a different launch order of the same arithmetic.  Two calls in a row
check that the shared scratch needs no clearing between calls.
"""
import ctypes

import numpy as np
import pytest
import torch

from open_quadtree_mapping_b200 import _lib
from open_quadtree_mapping_b200.params import ARITH_IEEE, ARITH_REFERENCE, Params, QmParamsC

pytestmark = pytest.mark.gpu

RTOL = 1e-6
MAX_PIXELS = 1 << 20


def _case(W, H, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:H, 0:W]
    img = (120 + 70 * np.sin(xx / 29.0 + seed) * np.cos(yy / 19.0)
           + rng.normal(0, 10, (H, W))).clip(0, 255).astype(np.uint8)
    sparse = np.where(rng.random((H, W)) < 0.06, rng.uniform(0.5, 30.0, (H, W)), 0.0)
    return img, sparse.astype(np.float32)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _with_workspace(sparse, img, params, stream):
    H, W = img.shape
    dense = torch.empty((H, W), dtype=torch.float32, device=img.device)
    n = ctypes.c_size_t()
    _lib.check(_lib.lib().qm_upsample_workspace_size(W, H, ctypes.byref(n)))
    ws = torch.empty(n.value, dtype=torch.uint8, device=img.device)
    pc = QmParamsC.from_params(params)
    _lib.check(_lib.lib().qm_upsample(_p(sparse), _p(img), W, W, H, ctypes.byref(pc), _p(dense),
                                      _p(ws), n.value, stream))
    return dense


def _no_alloc(sparse, img, params, dense, stream):
    H, W = img.shape
    pc = QmParamsC.from_params(params)
    return _lib.lib().qm_upsample_noalloc(_p(sparse), _p(img), W, W, H, ctypes.byref(pc),
                                          _p(dense), stream)


@pytest.mark.parametrize("W,H,arith", [(752, 480, ARITH_REFERENCE), (1024, 1024, ARITH_IEEE),
                                       (160, 128, ARITH_IEEE)])
def test_no_alloc_matches_workspace_entry(W, H, arith, gpu):
    dev = gpu
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    params = Params(arith=arith)
    outs = []
    for seed in (1, 2):  # two calls in a row, different inputs
        img_h, sparse_h = _case(W, H, seed + W)
        img = torch.from_numpy(img_h).to(dev)
        sparse = torch.from_numpy(sparse_h).to(dev)
        dense = torch.full((H, W), float("nan"), dtype=torch.float32, device=dev)
        st = _no_alloc(sparse, img, params, dense, stream)
        assert st == 0, _lib.lib().qm_last_error()
        want = _with_workspace(sparse, img, params, stream)
        torch.cuda.synchronize()
        got = dense.cpu().numpy()
        ref = want.cpu().numpy()
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=0)
        outs.append(got)
    assert not np.array_equal(outs[0], outs[1])


def test_no_alloc_calls_leave_free_device_memory_unchanged(gpu):
    """After a first call (the per-device set-up), back-to-back calls on one
    stream allocate no device memory: the driver's free-memory count stays
    the same.  The workspace entry's reference output is computed after the
    loop, so nothing else allocates in between."""
    dev = gpu
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    params = Params(arith=ARITH_IEEE)
    W, H = 752, 480
    img_h, sparse_h = _case(W, H, 7)
    img = torch.from_numpy(img_h).to(dev)
    sparse = torch.from_numpy(sparse_h).to(dev)
    dense = torch.empty((H, W), dtype=torch.float32, device=dev)
    assert _no_alloc(sparse, img, params, dense, stream) == 0, _lib.lib().qm_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(8):
        assert _no_alloc(sparse, img, params, dense, stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    got = dense.cpu().numpy()
    want = _with_workspace(sparse, img, params, stream).cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=0)


def test_no_alloc_call_captured_in_graph_after_setup(gpu):
    """The documented set-up order: one eager call on the device first, then
    a later call can be captured into a CUDA graph (global capture mode, so
    any call that is unsafe during capture would fail the capture).  The
    replayed graph, on new inputs copied into the captured buffers, gives
    the eager result for those inputs."""
    dev = gpu
    params = Params(arith=ARITH_REFERENCE)
    W, H = 752, 480
    img_h, sparse_h = _case(W, H, 11)
    img = torch.from_numpy(img_h).to(dev)
    sparse = torch.from_numpy(sparse_h).to(dev)
    dense = torch.full((H, W), float("nan"), dtype=torch.float32, device=dev)
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        st = ctypes.c_void_p(side.cuda_stream)
        assert _no_alloc(sparse, img, params, dense, st) == 0, _lib.lib().qm_last_error()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cap = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = _no_alloc(sparse, img, params, dense, cap)
    assert rc == 0, _lib.lib().qm_last_error()
    img2_h, sparse2_h = _case(W, H, 12)
    img.copy_(torch.from_numpy(img2_h))
    sparse.copy_(torch.from_numpy(sparse2_h))
    dense.fill_(float("nan"))
    g.replay()
    torch.cuda.synchronize()
    got = dense.cpu().numpy()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    want = _with_workspace(sparse, img, params, stream).cpu().numpy()
    assert np.isfinite(got).all()
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=0)
    del g


def test_no_alloc_rejects_oversize_and_bad_shapes(gpu):
    dev = gpu
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    params = Params()
    # 2048 x 1024 is within the solvers' limits but above the scratch
    W, H = 2048, 1024
    assert W * H > MAX_PIXELS
    img = torch.zeros((H, W), dtype=torch.uint8, device=dev)
    sparse = torch.zeros((H, W), dtype=torch.float32, device=dev)
    dense = torch.zeros((H, W), dtype=torch.float32, device=dev)
    st = _no_alloc(sparse, img, params, dense, stream)
    assert st == _lib.QM_ERR_INVALID_ARG
    assert b"exceeds the static scratch" in _lib.lib().qm_last_error()
    # width not a multiple of 16
    img = torch.zeros((64, 100), dtype=torch.uint8, device=dev)
    sparse = torch.zeros((64, 100), dtype=torch.float32, device=dev)
    dense = torch.zeros((64, 100), dtype=torch.float32, device=dev)
    assert _no_alloc(sparse, img, params, dense, stream) == _lib.QM_ERR_INVALID_ARG
    torch.cuda.synchronize()
