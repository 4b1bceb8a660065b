"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (qm_oracle.cpp).

Used by tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and
the reference arm) as the checker; the product never imports this module.
Images are numpy arrays (H, W) uint8; costs (ch, cw, D); messages
(4, ch, cw, D) in the order up, down, left, right.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from open_quadtree_mapping_b200.params import Params, QmParamsC

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libqm_oracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libqm_ref.so")

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _real(dtype):
    return np.float32 if np.dtype(dtype) == np.float32 else np.float64


def quadtree(img: np.ndarray, params: Params = Params()) -> np.ndarray:
    img = np.ascontiguousarray(img, dtype=np.uint8)
    H, W = img.shape
    out = np.zeros((H, W), np.int32)
    pc = QmParamsC.from_params(params)
    lib().orc_quadtree(_p(img), W, H, ctypes.byref(pc), _p(out))
    return out


def cost_volume(ref, levels, slot_imgs, T_slot_ref, cam, params: Params = Params(),
                dtype=np.float32):
    """Cost volume (ch, cw, D) and visited-cell mask (ch, cw).

    slot_imgs: (F, H, W) u8 measurement images, one per slot (duplicates
    allowed); T_slot_ref: (F, 12) f32 row-major T_slot<-ref; cam = (fx, fy,
    cx, cy)."""
    ref = np.ascontiguousarray(ref, np.uint8)
    H, W = ref.shape
    levels = np.ascontiguousarray(levels, np.int32)
    slots = [np.ascontiguousarray(s, np.uint8) for s in slot_imgs]
    ptrs = (ctypes.c_void_p * len(slots))(*[s.ctypes.data for s in slots])
    T = np.ascontiguousarray(T_slot_ref, np.float32).reshape(-1, 12)
    R = _real(dtype)
    D = params.num_hyp
    cost = np.zeros((H // 4, W // 4, D), R)
    valid = np.zeros((H // 4, W // 4), np.int32)
    pc = QmParamsC.from_params(params)
    fn = lib().orc_cost_f32 if R == np.float32 else lib().orc_cost_f64
    fx, fy, cx, cy = [ctypes.c_float(v) for v in cam]
    fn(_p(ref), W, H, _p(levels), len(slots), ptrs, _p(T), fx, fy, cx, cy, ctypes.byref(pc),
       _p(cost), _p(valid))
    return cost, valid


def bp_extract(cost, W, H, levels, params: Params = Params(), sparse=None, want_messages=False):
    """Hierarchical BP + extraction.  Returns (labels (ch, cw) int32 with -1 at
    non-node cells, sparse depth (H, W), messages or None)."""
    R = _real(cost.dtype)
    cost = np.ascontiguousarray(cost, R)
    ch, cw, D = cost.shape
    levels = np.ascontiguousarray(levels, np.int32)
    labels = np.zeros((ch, cw), np.int32)
    sp = np.zeros((H, W), R) if sparse is None else np.array(sparse, dtype=R, copy=True)
    msgs = np.zeros((4, ch, cw, D), R) if want_messages else None
    pc = QmParamsC.from_params(params)
    fn = lib().orc_bp_f32 if R == np.float32 else lib().orc_bp_f64
    fn(_p(cost), W, H, _p(levels), ctypes.byref(pc), _p(labels), _p(sp),
       _p(msgs) if msgs is not None else None)
    return labels, sp, msgs


def upsample(sparse, img, params: Params = Params(), dense=None):
    R = _real(sparse.dtype)
    sparse = np.ascontiguousarray(sparse, R)
    img = np.ascontiguousarray(img, np.uint8)
    H, W = img.shape
    out = np.zeros((H, W), R) if dense is None else np.array(dense, dtype=R, copy=True)
    pc = QmParamsC.from_params(params)
    fn = lib().orc_upsample_f32 if R == np.float32 else lib().orc_upsample_f64
    fn(_p(sparse), _p(img), W, H, ctypes.byref(pc), _p(out))
    return out


def bp_soft(cost, W, H, levels, params: Params, tau: float):
    """FP64 hierarchical BP with the softened readout of the differentiable
    path (disparity = sum softmax(-belief/tau) d).  Returns sparse (H, W)."""
    cost = np.ascontiguousarray(cost, np.float64)
    ch, cw, D = cost.shape
    levels = np.ascontiguousarray(levels, np.int32)
    labels = np.zeros((ch, cw), np.int32)
    sp = np.zeros((H, W), np.float64)
    pc = QmParamsC.from_params(params)
    lib().orc_bp_soft_f64(_p(cost), W, H, _p(levels), ctypes.byref(pc), ctypes.c_double(tau),
                          _p(labels), _p(sp))
    return sp


def upsample_w(sparse, img, params: Params, omega):
    """FP64 upsampling with per-pixel edge-weight factors omega (H, W)."""
    sparse = np.ascontiguousarray(sparse, np.float64)
    img = np.ascontiguousarray(img, np.uint8)
    omega = np.ascontiguousarray(omega, np.float64)
    H, W = img.shape
    out = np.zeros((H, W), np.float64)
    pc = QmParamsC.from_params(params)
    lib().orc_upsample_w_f64(_p(sparse), _p(img), W, H, ctypes.byref(pc), _p(omega), _p(out))
    return out


def upsample_weights(img, params: Params = Params()):
    img = np.ascontiguousarray(img, np.uint8)
    H, W = img.shape
    row_w = np.zeros((H, W + 1), np.float32)
    col_w = np.zeros((H + 1, W), np.float32)
    pc = QmParamsC.from_params(params)
    lib().orc_upsample_weights_f32(_p(img), W, H, ctypes.byref(pc), _p(row_w), _p(col_w))
    return row_w, col_w


def fuse(depth, seeds, T_income_last, cam):
    """Bayesian fusion.  Returns (fused depth, new seeds (H, W, 4), table,
    contested mask)."""
    R = _real(depth.dtype)
    depth = np.ascontiguousarray(depth, R)
    H, W = depth.shape
    seeds = np.ascontiguousarray(seeds, np.float32).reshape(H, W, 4)
    T = np.ascontiguousarray(T_income_last, np.float32).reshape(12)
    out = np.zeros((H, W), R)
    new_seeds = np.zeros((H, W, 4), R)
    table = np.zeros((H, W), np.int32)
    contested = np.zeros((H, W), np.uint8)
    fn = lib().orc_fuse_f32 if R == np.float32 else lib().orc_fuse_f64
    fx, fy, cx, cy = [ctypes.c_float(v) for v in cam]
    fn(_p(depth), _p(seeds), _p(T), fx, fy, cx, cy, W, H, _p(out), _p(new_seeds), _p(table),
       _p(contested))
    return out, new_seeds, table, contested


def point_cloud(depth, ref, cam, T_world_ref):
    """Point cloud of a depth map (publisher.cpp:146-163): (N, 4) float32
    rows (x, y, z, intensity) in row-major pixel order."""
    depth = np.ascontiguousarray(depth, np.float32)
    H, W = depth.shape
    ref = np.ascontiguousarray(ref, np.uint8)
    T = np.ascontiguousarray(T_world_ref, np.float32).reshape(12)
    out = np.zeros((H * W, 4), np.float32)
    fn = lib().orc_point_cloud
    fn.restype = ctypes.c_int
    fx, fy, cx, cy = [ctypes.c_float(v) for v in cam]
    n = fn(_p(depth), _p(ref), W, H, fx, fy, cx, cy, _p(T), _p(out))
    return out[:n].copy()


SD_INIT, SD_UPDATE, SD_SWITCH = 1, 2, 3


def sd_step(key, inc, cam, T_income_key, mode, trk, dep):
    """One semi-dense step (qm_oracle_semidense.cpp).  key / inc: (H, W)
    uint8 (key None for SD_INIT); trk / dep: (H, W, 4) float32, updated in
    place.  Returns the debug image (H, W) float32."""
    inc = np.ascontiguousarray(inc, np.uint8)
    H, W = inc.shape
    key = None if key is None else np.ascontiguousarray(key, np.uint8)
    T = np.ascontiguousarray(T_income_key, np.float32).reshape(12)
    assert trk.dtype == np.float32 and trk.flags.c_contiguous and trk.shape == (H, W, 4)
    assert dep.dtype == np.float32 and dep.flags.c_contiguous and dep.shape == (H, W, 4)
    debug = np.zeros((H, W), np.float32)
    fx, fy, cx, cy = [ctypes.c_float(v) for v in cam]
    lib().orc_sd_step(W, H, fx, fy, cx, cy, _p(key) if key is not None else None, _p(inc),
                      _p(T), int(mode), _p(trk), _p(dep), _p(debug))
    return debug


def sd_sample(img, uv):
    """The oracle's bilinear texture emulation (8-bit fractional weights,
    clamp) of a u8 image at (n, 2) unnormalised coordinates."""
    img = np.ascontiguousarray(img, np.uint8)
    H, W = img.shape
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    out = np.zeros(len(uv), np.float32)
    lib().orc_sd_sample(_p(img), W, H, _p(uv), len(uv), _p(out))
    return out


def slots_from_ring(n_slots: int):
    """Ring index read by measurement slot f: floor(age/10 * f) with the age
    table all zero, i.e. age clamped to 9 (depth_extract.cu:153-166)."""
    return [int(9 / 10.0 * f) for f in range(n_slots)]


def extract_depth(ref, slot_imgs, T_slot_ref, cam, params: Params = Params(), dtype=np.float32,
                  sparse=None, want_messages=False):
    """quadtree -> cost -> BP/extract -> upsample, as SeedMatrix::extract_depth
    (seed_matrix.cu:448-551).  Returns a dict of every intermediate."""
    H, W = ref.shape
    levels = quadtree(ref, params)
    cost, valid = cost_volume(ref, levels, slot_imgs, T_slot_ref, cam, params, dtype)
    labels, sp, msgs = bp_extract(cost, W, H, levels, params, sparse=sparse,
                                  want_messages=want_messages)
    dense = upsample(sp, ref, params)
    return dict(levels=levels, cost=cost, valid=valid, labels=labels, sparse=sp,
                messages=msgs, dense=dense)
