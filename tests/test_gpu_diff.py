"""Differentiable path on the GPU (qm_bp_soft_*, qm_upsample_w_*,
qm_fuse_backward through the C-ABI) against FP64 central finite differences
of the oracle (h = 1e-6) on a 64x48 keyframe, and against FP64 torch autograd
of the same formulas.

Tolerances: per stage, gradients within 1e-4 relative (to the largest
component of the gradient) of the FP64 references; forward values within
1e-4 relative of the FP64 oracle (the GPU runs BP and the readout in FP32,
the line solves and the fusion update in FP64).  End to end through the FP32
BP the bound is 1e-3 (see E2E_RTOL); with the soft BP in its FP64
gradient-check mode (qm_bp_soft64_*) end to end is held to 1e-4.
"""
import dataclasses

import numpy as np
import pytest
import torch

from conftest import cam_of, keyframe
from open_quadtree_mapping_b200.params import ARITH_IEEE, Params

pytestmark = pytest.mark.gpu

W, H = 64, 48
TAU = 0.05
FD_H = 1e-6
GRAD_RTOL = 1e-4
# End to end, the FP32 BP forward is the limit: the readout divides the
# beliefs by tau = 0.05, so message rounding (~1e-7 of the beliefs) moves the
# soft depths by ~1e-5 relative, and the FP64 references run an FP64 BP.
E2E_RTOL = 1e-3
FWD_RTOL = 1e-4


def _params(**kw):
    return Params.for_range(64, 0.5, 50.0, arith=ARITH_IEEE, **kw)


@pytest.fixture(scope="module")
def case(gpu, oracle_mod):
    from open_quadtree_mapping_b200 import stages
    kf = keyframe(3, W, H, 5)
    p = _params()
    ref = torch.from_numpy(kf.ref).to(gpu)
    slots = [torch.from_numpy(np.ascontiguousarray(m)).to(gpu) for m in kf.meas]
    levels = stages.quadtree(ref, p)
    cost = stages.cost_volume(ref, levels, slots, kf.T_meas_ref, cam_of(kf), p)
    rng = np.random.default_rng(7)
    gt = kf.gt_depth.astype(np.float32)
    # a prior that fusion accepts (inlier ratio 30/35): the ground truth with
    # 3 % noise and a variance wide enough (25 m^2) that the coarse depth of
    # this small image does not reset it
    seeds = np.zeros((H, W, 4), np.float32)
    seeds[..., 0] = 30.0
    seeds[..., 1] = 5.0
    seeds[..., 2] = gt * (1.0 + 0.03 * rng.standard_normal((H, W)))
    seeds[..., 3] = 25.0
    T_id = np.eye(3, 4, dtype=np.float32).reshape(12)
    return dict(kf=kf, p=p, ref=ref, levels=levels, cost=cost, gt=gt, seeds=seeds, T=T_id,
                rng=rng, dev=gpu)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def _soft(case, pen, fp64=False):
    from open_quadtree_mapping_b200.diff import SoftBP
    return SoftBP.apply(pen, case["cost"], case["levels"], case["p"], TAU, fp64)


def _oracle_soft(case, oracle_mod, P1, P2):
    p = dataclasses.replace(case["p"], P1=P1, P2=P2)
    cost = case["cost"].cpu().numpy().astype(np.float64)
    return oracle_mod.bp_soft(cost, W, H, case["levels"].cpu().numpy(), p, TAU)


@pytest.mark.parametrize("fp64,rtol", [(False, FWD_RTOL), (True, 1e-6)])
def test_soft_bp_forward_matches_fp64_oracle(case, oracle_mod, fp64, rtol):
    """FP32 soft BP within 1e-4 of the FP64 oracle; the FP64 mode to the
    float rounding of its output (1e-6)."""
    p = case["p"]
    pen = torch.tensor([p.P1, p.P2], dtype=torch.float64)
    g = _soft(case, pen, fp64).cpu().numpy()
    o = _oracle_soft(case, oracle_mod, p.P1, p.P2)
    node = o > 0
    assert node.sum() > 20
    assert np.array_equal(g > 0, node)
    assert _rel(g[node], o[node]) < rtol


def _torch_soft(case, P1, P2):
    from bp_torch_ref import soft_bp
    cost = torch.from_numpy(case["cost"].cpu().numpy().astype(np.float64))
    return soft_bp(cost, case["levels"].cpu().numpy().astype(np.int64), case["p"], P1, P2, TAU)


def test_soft_bp_penalty_gradients(case, oracle_mod):
    """dL/dP1, dL/dP2 of a linear functional of the soft readout.  The loss
    is piecewise linear in the penalties with kinks closer together than the
    FD step (every min-sum selection switches at some P), so central
    differences at h = 1e-6 average the slopes of several pieces; the exact
    gradient is checked against FP64 autograd of the same forward, and the
    differences only to the spread that the kinks leave."""
    p = case["p"]
    R = case["rng"].standard_normal((H, W))
    pen = torch.tensor([p.P1, p.P2], dtype=torch.float64, requires_grad=True)
    sparse = _soft(case, pen)
    (sparse.double() * torch.from_numpy(R).to(sparse.device)).sum().backward()
    got = pen.grad.numpy()
    assert np.all(np.isfinite(got))
    P1 = torch.tensor(p.P1, dtype=torch.float64, requires_grad=True)
    P2 = torch.tensor(p.P2, dtype=torch.float64, requires_grad=True)
    (_torch_soft(case, P1, P2) * torch.from_numpy(R)).sum().backward()
    ref = np.array([P1.grad.item(), P2.grad.item()])
    assert _rel(got, ref) < GRAD_RTOL, (got, ref)
    fd = []
    for k in range(2):
        vals = []
        for sgn in (1, -1):
            q = [p.P1, p.P2]
            q[k] += sgn * FD_H
            vals.append((_oracle_soft(case, oracle_mod, *q) * R).sum())
        fd.append((vals[0] - vals[1]) / (2 * FD_H))
    assert _rel(got, fd) < 0.25, (got, fd)


def test_upsample_w_gradients_vs_fd(case, oracle_mod):
    from open_quadtree_mapping_b200.diff import UpsampleW
    p, dev, rng = case["p"], case["dev"], case["rng"]
    sparse = _oracle_soft(case, oracle_mod, p.P1, p.P2).astype(np.float32)
    omega = (1.0 + 0.2 * rng.standard_normal((H, W))).clip(0.2, 2.0).astype(np.float32)
    R = rng.standard_normal((H, W))
    sp_t = torch.from_numpy(sparse).to(dev).requires_grad_(True)
    om_t = torch.from_numpy(omega).to(dev).requires_grad_(True)
    dense = UpsampleW.apply(sp_t, om_t, case["ref"], p)
    o = case["kf"].ref
    d64 = oracle_mod.upsample_w(sparse.astype(np.float64), o, p, omega.astype(np.float64))
    assert _rel(dense.detach().cpu().numpy(), d64) < FWD_RTOL
    (dense.double() * torch.from_numpy(R).to(dev)).sum().backward()
    g_sp = sp_t.grad.cpu().numpy()
    g_om = om_t.grad.cpu().numpy()

    def L(sp, om):
        return (oracle_mod.upsample_w(sp, o, p, om) * R).sum()

    nodes = np.argwhere(sparse > 0)
    picks_sp = nodes[rng.choice(len(nodes), 8, replace=False)]
    picks_om = np.stack([rng.integers(1, H, 8), rng.integers(1, W, 8)], 1)
    fd_sp, fd_om = [], []
    for (y, x) in picks_sp:
        vals = []
        for sgn in (1, -1):
            sp = sparse.astype(np.float64)
            sp[y, x] += sgn * FD_H
            vals.append(L(sp, omega.astype(np.float64)))
        fd_sp.append((vals[0] - vals[1]) / (2 * FD_H))
    for (y, x) in picks_om:
        vals = []
        for sgn in (1, -1):
            om = omega.astype(np.float64)
            om[y, x] += sgn * FD_H
            vals.append(L(sparse.astype(np.float64), om))
        fd_om.append((vals[0] - vals[1]) / (2 * FD_H))
    assert _rel(g_sp[tuple(picks_sp.T)], fd_sp) < GRAD_RTOL
    assert _rel(g_om[tuple(picks_om.T)], fd_om) < GRAD_RTOL


def test_upsample_w_gradients_vs_autograd(case, oracle_mod):
    """The adjoint against torch autograd through dense FP64 solves of the
    same row and column systems."""
    from open_quadtree_mapping_b200.diff import UpsampleW
    p, dev, rng = case["p"], case["dev"], case["rng"]
    sparse = _oracle_soft(case, oracle_mod, p.P1, p.P2).astype(np.float32)
    omega = (1.0 + 0.2 * rng.standard_normal((H, W))).clip(0.2, 2.0).astype(np.float32)
    R = torch.from_numpy(rng.standard_normal((H, W))).double()
    sp_t = torch.from_numpy(sparse).to(dev).requires_grad_(True)
    om_t = torch.from_numpy(omega).to(dev).requires_grad_(True)
    (UpsampleW.apply(sp_t, om_t, case["ref"], p).double() * R.to(dev)).sum().backward()

    sp = torch.from_numpy(sparse.astype(np.float64)).requires_grad_(True)
    om = torch.from_numpy(omega.astype(np.float64)).requires_grad_(True)
    (_torch_upsample(case["kf"].ref, sp, om, p) * R).sum().backward()
    assert _rel(sp_t.grad.cpu().numpy()[sparse > 0], sp.grad.numpy()[sparse > 0]) < 1e-5
    assert _rel(om_t.grad.cpu().numpy(), om.grad.numpy()) < 1e-5


def _torch_upsample(ref, sp, om, p):
    """The weighted upsampling as dense FP64 solves (both line lengths here
    are multiples of 16, so both closing weights are 0)."""
    img = torch.from_numpy(ref.astype(np.float64))
    lam, sig = p.up_lambda, p.up_sigma

    def solve(w_inner, rhs):
        # lines along the last axis; w_inner[..., k] = weight of edge (k-1, k)
        n = rhs.shape[-1]
        w = torch.cat([torch.zeros_like(w_inner[..., :1]), w_inner[..., 1:],
                       torch.zeros_like(w_inner[..., :1])], -1)  # w[0] = w[n] = 0
        diag = 1.0 + lam * (w[..., :n] + w[..., 1:])
        A = torch.diag_embed(diag) - lam * torch.diag_embed(w[..., 1:n], 1) \
            - lam * torch.diag_embed(w[..., 1:n], -1)
        return torch.linalg.solve(A, rhs.unsqueeze(-1)).squeeze(-1)

    e_row = torch.exp(-(img[:, 1:] - img[:, :-1]) ** 2 / sig)
    e_col = torch.exp(-(img[1:, :] - img[:-1, :]) ** 2 / sig)
    w_row = torch.cat([torch.zeros(H, 1, dtype=torch.float64), om[:, 1:] * e_row], 1)
    w_col = torch.cat([torch.zeros(1, W, dtype=torch.float64), om[1:, :] * e_col], 0)
    ind = (sp > 0).double()
    sd, si = solve(w_row, sp), solve(w_row, ind)
    td, ti = solve(w_col.T, sd.T).T, solve(w_col.T, si.T).T
    return td / ti


def _torch_fuse(dep, prior_t, table):
    """fuse_currentmap (depth_fusion.cu:146-213) in FP64 torch, with the
    priors the GPU fusion gathered (transformed seeds, table)."""
    t = torch.from_numpy(table.astype(np.int64))
    s = torch.from_numpy(prior_t.reshape(-1, 4).astype(np.float64))[t.reshape(-1)]
    s = s.reshape(H, W, 4)
    has = t > 0
    unc = torch.clamp(dep * 0.2, min=0.5) ** 2
    unc = torch.where(dep <= 0, torch.full_like(dep, 1e9), unc)
    a = torch.where(has, s[..., 0], torch.full_like(dep, 10.0))
    b = torch.where(has, s[..., 1], torch.full_like(dep, 10.0))
    mu = torch.where(has, s[..., 2], dep)
    s2 = torch.where(has, s[..., 3], torch.full_like(dep, 2500.0))
    reset = (dep - mu) ** 2 > unc + s2
    a = torch.where(reset, torch.full_like(dep, 10.0), a)
    b = torch.where(reset, torch.full_like(dep, 10.0), b)
    mu = torch.where(reset, dep, mu)
    s2 = torch.where(reset, torch.full_like(dep, 2500.0), s2)
    var = unc + s2
    new_mu = (dep * s2 + mu * unc) / var
    pdf = torch.exp(-(dep - mu) ** 2 / (2 * var)) / torch.sqrt(2 * np.pi * var)
    ratio = a / (a + b)
    c1 = ratio * pdf
    c2 = b / (a + b) / 50.0
    norm = c1 + c2
    mu_p = (c1 / norm) * new_mu + (c2 / norm) * mu
    return torch.where(ratio > 0.6, mu_p, torch.full_like(dep, -1.0))


def _fused(case, oracle_mod, dense64):
    kf = case["kf"]
    out, _, _, _ = oracle_mod.fuse(dense64, case["seeds"], case["T"], cam_of(kf))
    return out


def test_fuse_gradient_vs_fd(case, oracle_mod):
    from open_quadtree_mapping_b200.diff import Fuse, UpsampleW
    p, dev, rng = case["p"], case["dev"], case["rng"]
    sparse = _oracle_soft(case, oracle_mod, p.P1, p.P2).astype(np.float32)
    dense = UpsampleW.apply(torch.from_numpy(sparse).to(dev),
                            torch.ones((H, W), device=dev), case["ref"], p).detach()
    d_t = dense.clone().requires_grad_(True)
    seeds = torch.from_numpy(case["seeds"]).to(dev)
    fused = Fuse.apply(d_t, seeds, case["T"], cam_of(case["kf"]), p)
    R = rng.standard_normal((H, W))
    valid = (fused > 0).cpu().numpy()
    assert valid.mean() > 0.2
    (fused.double() * torch.from_numpy(R).to(dev)).sum().backward()
    g = d_t.grad.cpu().numpy()
    d64 = dense.cpu().numpy().astype(np.float64)
    # the update is per pixel, so one perturbation of every pixel gives the
    # whole diagonal
    fp = _fused(case, oracle_mod, d64 + FD_H)
    fm = _fused(case, oracle_mod, d64 - FD_H)
    ok = valid & (fp > 0) & (fm > 0)
    fd = (fp - fm) / (2 * FD_H) * R
    assert _rel(g[ok], fd[ok]) < GRAD_RTOL
    assert np.all(g[~valid] == 0)


@pytest.mark.parametrize("fp64,rtol", [(False, E2E_RTOL), (True, GRAD_RTOL)])
def test_pipeline_gradients(case, oracle_mod, fp64, rtol):
    """End to end through autograd: L1 of the fused depth against the ground
    truth.  Gradients for (P1, P2) and omega against FP64 torch autograd of
    the same pipeline; for omega (smooth) also against FP64 finite
    differences (h = 1e-6) of the oracle pipeline.  FP32 soft BP within
    1e-3, the FP64 gradient-check mode within 1e-4."""
    from open_quadtree_mapping_b200 import diff
    p, dev, rng = case["p"], case["dev"], case["rng"]
    kf = case["kf"]
    K = diff.Keyframe(ref=case["ref"], slots=None, T_slot_ref=None, cam=cam_of(kf),
                      seeds=torch.from_numpy(case["seeds"]).to(dev), T_fuse=case["T"],
                      gt=torch.from_numpy(case["gt"]).to(dev), levels=case["levels"],
                      cost=case["cost"])
    omega = (1.0 + 0.1 * rng.standard_normal((H, W))).astype(np.float32)
    pen = torch.tensor([p.P1, p.P2], dtype=torch.float64, requires_grad=True)
    om = torch.from_numpy(omega).to(dev).requires_grad_(True)
    fused = diff.forward_keyframe(K, pen, om, p, TAU, fp64)
    loss = diff.l1_loss(fused, K.gt)
    loss.backward()
    g_pen = pen.grad.numpy()
    g_om = om.grad.cpu().numpy()
    gt = case["gt"].astype(np.float64)
    mask = (fused.detach().cpu().numpy() > 0) & (gt > 0)
    cost64 = case["cost"].cpu().numpy().astype(np.float64)
    lv = case["levels"].cpu().numpy()

    def L(P1, P2, om64):
        q = dataclasses.replace(p, P1=P1, P2=P2)
        sp = oracle_mod.bp_soft(cost64, W, H, lv, q, TAU)
        dn = oracle_mod.upsample_w(sp, kf.ref, q, om64)
        f = _fused(case, oracle_mod, dn)
        return (np.abs(f - gt) * mask).sum() / mask.sum()

    om64 = omega.astype(np.float64)
    picks = np.stack([rng.integers(1, H, 6), rng.integers(1, W, 6)], 1)
    fd_om = []
    for (y, x) in picks:
        a, b = om64.copy(), om64.copy()
        a[y, x] += FD_H
        b[y, x] -= FD_H
        fd_om.append((L(p.P1, p.P2, a) - L(p.P1, p.P2, b)) / (2 * FD_H))
    assert mask.sum() > 100
    assert _rel(g_om[tuple(picks.T)], fd_om) < rtol, (g_om[tuple(picks.T)], fd_om)
    # FP64 autograd of the whole pipeline, with the fusion's table and
    # transformed seeds (they do not depend on the current depth)
    from open_quadtree_mapping_b200 import stages
    _, s_t, _, table = stages.fuse(fused.detach() * 0 + 1, K.seeds, K.T_fuse, K.cam, p)
    P1 = torch.tensor(p.P1, dtype=torch.float64, requires_grad=True)
    P2 = torch.tensor(p.P2, dtype=torch.float64, requires_grad=True)
    omr = torch.from_numpy(om64).requires_grad_(True)
    f_ref = _torch_fuse(_torch_upsample(kf.ref, _torch_soft(case, P1, P2), omr, p),
                        s_t.cpu().numpy(), table.cpu().numpy())
    m = torch.from_numpy(mask.astype(np.float64))
    ((f_ref - torch.from_numpy(gt)).abs() * m).sum().div(m.sum()).backward()
    assert _rel(g_pen, [P1.grad.item(), P2.grad.item()]) < rtol, \
        (g_pen, P1.grad.item(), P2.grad.item())
    assert _rel(g_om, omr.grad.numpy()) < rtol
