"""Differentiable depth pipeline: torch.autograd.Function wrappers over the
adjoint kernels of libqm_b200.so (qm_bp_soft_*, qm_upsample_w_*,
qm_fuse_backward in include/qm_capi.h).

The pipeline of one keyframe, as a function of the fitted parameters:

    cost (no gradient) -> SoftBP(P1, P2) -> sparse depth at node pixels
    -> UpsampleW(sparse, omega) -> dense depth
    -> Fuse(dense; previous seeds, pose) -> fused depth (-1 where not valid)

SoftBP replaces the hard argmin of the extraction (bpextract.cu:314-372) by
a softmax over the beliefs with temperature tau; UpsampleW multiplies every
inner edge weight of the upsampling systems (depth_upsample.cu:58-93) by a
per-pixel factor omega.  The hard-argmin plain pipeline stays the product
path; this module serves fitting P1, P2 and omega to ground-truth depth
(`fit` below).  All work happens on the GPU through the C-ABI; torch
provides device memory, streams and autograd.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _lib, stages
from .params import Params, QmParamsC


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _with_penalties(params: Params, pen: torch.Tensor) -> Params:
    p1, p2 = (float(v) for v in pen.detach().cpu().tolist())
    return dataclasses.replace(params, P1=p1, P2=p2)


class SoftBP(torch.autograd.Function):
    """sparse = SoftBP.apply(penalties, cost, levels, params, tau, fp64=False).

    penalties: (2,) float64 tensor (P1, P2); cost: (H/4, W/4, D) float32 CUDA;
    levels: (H, W) uint8 CUDA quadtree levels.  Returns (H, W) float32 with
    the soft-readout depth at (4x, 4y) of every node cell, 0 elsewhere.
    fp64: run the BP, the readout and the adjoint in FP64 (qm_bp_soft64_*),
    the gradient-check mode; the default FP32 path is the fitting path."""

    @staticmethod
    def forward(ctx, penalties, cost, levels, params: Params, tau: float, fp64: bool = False):
        H, W = levels.shape
        p = _with_penalties(params, penalties)
        pc = QmParamsC.from_params(p)
        L = _lib.lib()
        ws_size, fwd = ((L.qm_bp_soft64_workspace_size, L.qm_bp_soft64_forward) if fp64 else
                        (L.qm_bp_soft_workspace_size, L.qm_bp_soft_forward))
        n = ctypes.c_size_t()
        _lib.check(ws_size(W, H, ctypes.byref(pc), ctypes.byref(n)))
        ws = torch.empty(n.value, dtype=torch.uint8, device=cost.device)
        sparse = torch.empty((H, W), dtype=torch.float32, device=cost.device)
        _lib.check(fwd(_ptr(cost), W, H, _ptr(levels), ctypes.byref(pc), ctypes.c_float(tau),
                       _ptr(sparse), _ptr(ws), n.value, _stream()))
        ctx.state = (cost, levels, p, tau, ws, penalties.dtype, penalties.device, fp64)
        return sparse

    @staticmethod
    def backward(ctx, g_sparse):
        cost, levels, p, tau, ws, dtype, device, fp64 = ctx.state
        H, W = levels.shape
        g = g_sparse.contiguous().to(torch.float32)
        gp = torch.empty(2, dtype=torch.float64, device=cost.device)
        pc = QmParamsC.from_params(p)
        L = _lib.lib()
        bwd = L.qm_bp_soft64_backward if fp64 else L.qm_bp_soft_backward
        _lib.check(bwd(_ptr(cost), W, H, _ptr(levels), ctypes.byref(pc), ctypes.c_float(tau),
                       _ptr(g), _ptr(gp), _ptr(ws), ws.numel(), _stream()))
        return gp.to(device=device, dtype=dtype), None, None, None, None, None


class UpsampleW(torch.autograd.Function):
    """dense = UpsampleW.apply(sparse, omega, img, params): the edge-aware
    upsampling with per-pixel edge-weight factors omega (FP64 line solves)."""

    @staticmethod
    def forward(ctx, sparse, omega, img, params: Params):
        H, W = img.shape
        pc = QmParamsC.from_params(params)
        n = ctypes.c_size_t()
        _lib.check(_lib.lib().qm_upsample_w_workspace_size(W, H, ctypes.byref(n)))
        ws = torch.empty(n.value, dtype=torch.uint8, device=img.device)
        sp = sparse.contiguous().to(torch.float32)
        om = omega.contiguous().to(torch.float32)
        dense = torch.empty((H, W), dtype=torch.float32, device=img.device)
        _lib.check(_lib.lib().qm_upsample_w_forward(_ptr(sp), _ptr(img), W, W, H,
                                                    ctypes.byref(pc), _ptr(om), _ptr(dense),
                                                    _ptr(ws), n.value, _stream()))
        ctx.state = (img, om, params, ws, omega.dtype)
        return dense

    @staticmethod
    def backward(ctx, g_dense):
        img, om, params, ws, odtype = ctx.state
        H, W = img.shape
        g = g_dense.contiguous().to(torch.float32)
        g_sp = torch.empty((H, W), dtype=torch.float32, device=img.device)
        g_om = torch.empty((H, W), dtype=torch.float32, device=img.device)
        pc = QmParamsC.from_params(params)
        _lib.check(_lib.lib().qm_upsample_w_backward(_ptr(img), W, W, H, ctypes.byref(pc),
                                                     _ptr(om), _ptr(g), _ptr(g_sp), _ptr(g_om),
                                                     _ptr(ws), ws.numel(), _stream()))
        return g_sp, g_om.to(odtype), None, None


class Fuse(torch.autograd.Function):
    """fused = Fuse.apply(dense, seeds, T_income_last, cam, params): the
    Bayesian fusion of qm_fuse (seeds (H, W, 4) of the previous result are
    not modified); differentiable in the upsampled depth."""

    @staticmethod
    def forward(ctx, dense, seeds, T_income_last, cam, params: Params):
        d_in = dense.detach().contiguous().to(torch.float32)
        fused, s_t, _, table = stages.fuse(d_in, seeds.contiguous(), T_income_last, cam, params)
        ctx.state = (d_in, s_t, table)
        return fused

    @staticmethod
    def backward(ctx, g_fused):
        d_in, s_t, table = ctx.state
        H, W = d_in.shape
        g = g_fused.contiguous().to(torch.float32)
        g_d = torch.empty((H, W), dtype=torch.float32, device=d_in.device)
        _lib.check(_lib.lib().qm_fuse_backward(_ptr(d_in), _ptr(s_t), _ptr(table), W, H, _ptr(g),
                                               _ptr(g_d), _stream()))
        return g_d, None, None, None, None


@dataclasses.dataclass
class Keyframe:
    """One training keyframe: reference image, measurement images and poses,
    the previous fusion state and the ground-truth depth (all (H, W))."""
    ref: torch.Tensor            # uint8 CUDA
    slots: list                  # uint8 CUDA images
    T_slot_ref: np.ndarray       # (F, 12)
    cam: tuple                   # fx, fy, cx, cy
    seeds: torch.Tensor          # (H, W, 4) float32 CUDA, previous seeds
    T_fuse: np.ndarray           # 12 floats, T_income<-lastfuse
    gt: torch.Tensor             # float32 CUDA ground-truth depth
    levels: torch.Tensor | None = None
    cost: torch.Tensor | None = None

    def prepare(self, params: Params):
        """Quadtree and cost volume (no parameters): computed once."""
        if self.cost is None:
            self.levels = stages.quadtree(self.ref, params)
            self.cost = stages.cost_volume(self.ref, self.levels, self.slots, self.T_slot_ref,
                                           self.cam, params)
        return self


def forward_keyframe(kf: Keyframe, penalties, omega, params: Params, tau: float = 0.05,
                     fp64: bool = False):
    """Fused depth of one keyframe as a differentiable function of
    penalties (P1, P2) and omega (fp64: the soft BP in its FP64
    gradient-check mode)."""
    kf.prepare(params)
    sparse = SoftBP.apply(penalties, kf.cost, kf.levels, params, tau, fp64)
    dense = UpsampleW.apply(sparse, omega, kf.ref, params)
    return Fuse.apply(dense, kf.seeds, kf.T_fuse, kf.cam, params)


def l1_loss(fused, gt):
    """Mean absolute error over the pixels where fusion and ground truth are
    both valid."""
    mask = ((fused > 0) & (gt > 0)).to(fused.dtype)
    return (torch.abs(fused - gt) * mask).sum() / mask.sum().clamp(min=1.0)


def batch_loss(kfs, penalties, omegas, params: Params, tau: float = 0.05):
    return sum(l1_loss(forward_keyframe(kf, penalties, om, params, tau), kf.gt)
               for kf, om in zip(kfs, omegas)) / len(kfs)


def fit(kfs, params: Params, steps: int = 20, lr_pen: float = 1e-4, lr_omega: float = 2e-2,
        tau: float = 0.05):
    """Fits (P1, P2) and one omega map per keyframe by Adam on the batch L1
    loss (Adam moves every parameter by about its learning rate per step, so
    lr_pen is small against the default penalties 0.003 / 0.01).  Returns
    (penalties, omegas, loss history)."""
    dev = kfs[0].ref.device
    pen = torch.tensor([params.P1, params.P2], dtype=torch.float64, requires_grad=True)
    omegas = [torch.ones(kf.ref.shape, dtype=torch.float32, device=dev, requires_grad=True)
              for kf in kfs]
    opt = torch.optim.Adam([{"params": [pen], "lr": lr_pen},
                            {"params": omegas, "lr": lr_omega}])
    hist = []
    for _ in range(steps):
        opt.zero_grad()
        loss = batch_loss(kfs, pen, omegas, params, tau)
        loss.backward()
        opt.step()
        with torch.no_grad():
            pen.clamp_(min=1e-6)
            for om in omegas:
                om.clamp_(min=0.0)
        hist.append(float(loss.detach()))
    return pen.detach(), [om.detach() for om in omegas], hist
