"""Stage entry points on torch CUDA tensors (qm_quadtree, qm_cost_volume,
qm_bp_extract, qm_upsample, qm_fuse in include/qm_capi.h).

torch provides the device memory and the stream; the work is done by
libqm_b200.so.  Every call is asynchronous on torch's current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .params import Params, QmParamsC


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _pc(params: Params) -> QmParamsC:
    return QmParamsC.from_params(params)


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _need(t: torch.Tensor, dtype, name):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise ValueError("%s must be a contiguous CUDA %s tensor" % (name, dtype))


def quadtree(img: torch.Tensor, params: Params = Params()) -> torch.Tensor:
    _need(img, torch.uint8, "img")
    H, W = img.shape
    levels = torch.empty((H, W), dtype=torch.uint8, device=img.device)
    pc = _pc(params)
    _lib.check(_lib.lib().qm_quadtree(_ptr(img), W, W, H, ctypes.byref(pc), _ptr(levels),
                                      _stream()))
    return levels


def cost_volume(ref: torch.Tensor, levels: torch.Tensor, slots, T_slot_ref, cam,
                params: Params = Params(), out: torch.Tensor | None = None) -> torch.Tensor:
    """slots: list of (H, W) uint8 CUDA tensors; T_slot_ref: (F, 12) host
    floats; cam = (fx, fy, cx, cy).  Returns the (H/4, W/4, D) cost volume,
    written into `out` when given (contiguous float32 of that shape)."""
    _need(ref, torch.uint8, "ref")
    _need(levels, torch.uint8, "levels")
    H, W = ref.shape
    F = len(slots)
    for s in slots:
        _need(s, torch.uint8, "slot")
    ptrs = (ctypes.c_void_p * F)(*[s.data_ptr() for s in slots])
    T = np.ascontiguousarray(np.asarray(T_slot_ref, dtype=np.float32).reshape(F, 12))
    shape = (H // 4, W // 4, params.num_hyp)
    if out is None:
        cost = torch.empty(shape, dtype=torch.float32, device=ref.device)
    else:
        _need(out, torch.float32, "out")
        if tuple(out.shape) != shape:
            raise ValueError("out must have shape %s" % (shape,))
        cost = out
    c = _lib.QmCamera(*[float(v) for v in cam])
    pc = _pc(params)
    _lib.check(_lib.lib().qm_cost_volume(_ptr(ref), W, W, H, ctypes.byref(c), _ptr(levels), F,
                                         ptrs, W, T.ctypes.data, ctypes.byref(pc), _ptr(cost),
                                         _stream()))
    return cost


def bp_extract(cost: torch.Tensor, W: int, H: int, levels: torch.Tensor,
               params: Params = Params(), sparse: torch.Tensor | None = None,
               want_messages: bool = False):
    """Returns (sparse (H, W) f32, labels (H/4, W/4) int32, messages or None)."""
    _need(cost, torch.float32, "cost")
    _need(levels, torch.uint8, "levels")
    dev = cost.device
    if sparse is None:
        sparse = torch.zeros((H, W), dtype=torch.float32, device=dev)
    labels = torch.empty((H // 4, W // 4), dtype=torch.int32, device=dev)
    msgs = (torch.empty((4, H // 4, W // 4, params.num_hyp), dtype=torch.float32, device=dev)
            if want_messages else None)
    pc = _pc(params)
    nbytes = ctypes.c_size_t()
    _lib.check(_lib.lib().qm_bp_workspace_size(W, H, ctypes.byref(pc), ctypes.byref(nbytes)))
    ws = torch.empty(max(1, nbytes.value), dtype=torch.uint8, device=dev)
    _lib.check(_lib.lib().qm_bp_extract(_ptr(cost), W, H, _ptr(levels), ctypes.byref(pc),
                                        _ptr(sparse), _ptr(labels),
                                        _ptr(msgs) if msgs is not None else None, _ptr(ws),
                                        nbytes.value, _stream()))
    return sparse, labels, msgs


def upsample(sparse: torch.Tensor, img: torch.Tensor, params: Params = Params()) -> torch.Tensor:
    _need(sparse, torch.float32, "sparse")
    _need(img, torch.uint8, "img")
    H, W = img.shape
    dense = torch.empty((H, W), dtype=torch.float32, device=img.device)
    nbytes = ctypes.c_size_t()
    _lib.check(_lib.lib().qm_upsample_workspace_size(W, H, ctypes.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=img.device)
    pc = _pc(params)
    _lib.check(_lib.lib().qm_upsample(_ptr(sparse), _ptr(img), W, W, H, ctypes.byref(pc),
                                      _ptr(dense), _ptr(ws), nbytes.value, _stream()))
    return dense


def fuse(depth: torch.Tensor, seeds: torch.Tensor, T_income_last, cam,
         params: Params = Params()):
    """depth (H, W) f32 and seeds (H, W, 4) f32 CUDA tensors.  Returns
    (fused depth, transformed previous seeds, new seeds, table); the inputs
    are not modified."""
    _need(depth, torch.float32, "depth")
    _need(seeds, torch.float32, "seeds")
    H, W = depth.shape
    d = depth.clone()
    s_in = seeds.clone()
    s_out = torch.empty_like(seeds)
    table = torch.empty((H, W), dtype=torch.int32, device=depth.device)
    nbytes = ctypes.c_size_t()
    _lib.check(_lib.lib().qm_fuse_workspace_size(W, H, ctypes.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=depth.device)
    T = np.ascontiguousarray(np.asarray(T_income_last, dtype=np.float32).reshape(12))
    c = _lib.QmCamera(*[float(v) for v in cam])
    pc = _pc(params)
    _lib.check(_lib.lib().qm_fuse(_ptr(d), _ptr(s_in), _ptr(s_out), T.ctypes.data,
                                  ctypes.byref(c), W, H, ctypes.byref(pc), _ptr(table), _ptr(ws),
                                  nbytes.value, _stream()))
    return d, s_in, s_out, table


def point_cloud(depth: torch.Tensor, ref: torch.Tensor, cam, T_world_ref) -> torch.Tensor:
    """Point cloud of a depth map (publisher.cpp:146-163): depth (H, W) f32
    and ref (H, W) u8 CUDA tensors (row strides may exceed W); returns the
    (N, 4) f32 CUDA tensor of (x, y, z, intensity) rows in pixel order."""
    if not (isinstance(depth, torch.Tensor) and depth.is_cuda and depth.dtype == torch.float32
            and depth.dim() == 2 and depth.stride(1) == 1):
        raise ValueError("depth must be a row-major CUDA float32 tensor")
    if not (isinstance(ref, torch.Tensor) and ref.is_cuda and ref.dtype == torch.uint8
            and ref.dim() == 2 and ref.stride(1) == 1):
        raise ValueError("ref must be a row-major CUDA uint8 tensor")
    H, W = depth.shape
    pts = torch.empty((H * W, 4), dtype=torch.float32, device=depth.device)
    count = torch.zeros(1, dtype=torch.int32, device=depth.device)
    nbytes = ctypes.c_size_t()
    _lib.check(_lib.lib().qm_point_cloud_workspace_size(W, H, ctypes.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=depth.device)
    T = np.ascontiguousarray(np.asarray(T_world_ref, dtype=np.float32).reshape(12))
    c = _lib.QmCamera(*[float(v) for v in cam])
    _lib.check(_lib.lib().qm_point_cloud(_ptr(depth), depth.stride(0), _ptr(ref), ref.stride(0),
                                         W, H, ctypes.byref(c), T.ctypes.data, _ptr(pts),
                                         _ptr(count), _ptr(ws), nbytes.value, _stream()))
    return pts[:int(count.item())]


SD_INIT, SD_UPDATE, SD_SWITCH = 1, 2, 3


def semidense_step(key, inc, cam, T_income_key, mode, trk, dep, arith=0):
    """One semi-dense tracker step (qm_semidense_step).  key / inc: (H, W)
    uint8 CUDA tensors (key may be None for SD_INIT); trk / dep: (H, W, 4)
    float32 CUDA tensors updated in place.  Returns the (H, W) float32 debug
    image (projected depths of the confident seeds, 0 elsewhere)."""
    _need(inc, torch.uint8, "inc")
    _need(trk, torch.float32, "trk")
    _need(dep, torch.float32, "dep")
    if key is not None:
        _need(key, torch.uint8, "key")
    H, W = inc.shape
    debug = torch.empty((H, W), dtype=torch.float32, device=inc.device)
    nbytes = ctypes.c_size_t()
    _lib.check(_lib.lib().qm_semidense_workspace_size(W, H, ctypes.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=inc.device)
    T = np.ascontiguousarray(np.asarray(T_income_key, dtype=np.float32).reshape(12))
    c = _lib.QmCamera(*[float(v) for v in cam])
    _lib.check(_lib.lib().qm_semidense_step(
        _ptr(key) if key is not None else None, _ptr(inc), W, H, ctypes.byref(c), T.ctypes.data,
        int(mode), int(arith), _ptr(trk), _ptr(dep), _ptr(debug), _ptr(ws), nbytes.value,
        _stream()))
    return debug


def extract_depth(ref, slots, T_slot_ref, cam, params: Params = Params(),
                  want_messages=False):
    """quadtree -> cost -> BP/extraction -> upsampling on one keyframe."""
    H, W = ref.shape
    levels = quadtree(ref, params)
    cost = cost_volume(ref, levels, slots, T_slot_ref, cam, params)
    sparse, labels, msgs = bp_extract(cost, W, H, levels, params, want_messages=want_messages)
    dense = upsample(sparse, ref, params)
    return dict(levels=levels, cost=cost, labels=labels, sparse=sparse, messages=msgs,
                dense=dense)
