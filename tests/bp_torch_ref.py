"""FP64 torch restatement of the hierarchical BP with the softened readout,
for autograd gradient references (test infrastructure).

Follows the oracle's bp_extract (oracle/qm_oracle.cpp, after
bpextract.cu:37-395 of the reference): cost pyramid by 2x2 sums, messages
copied down from the parent level (zeros at the coarsest level), red-black
half-sweeps with the quadtree skip test on the pre-checkerboard column, and
at level 0 a softmax readout over the beliefs at node cells.  Every cell
update is vectorised; cells that a half-sweep does not update keep their
messages through torch.where, so autograd follows exactly the forward's
dependencies (min takes the gradient to the selected argument).
"""
import numpy as np
import torch

UP, DOWN, LEFT, RIGHT = 0, 1, 2, 3


def _shift(t, dy, dx):
    """out[y, x] = t[y + dy, x + dx], zero outside."""
    out = torch.zeros_like(t)
    h, w = t.shape[:2]
    ys = slice(max(0, -dy), min(h, h - dy))
    xs = slice(max(0, -dx), min(w, w - dx))
    yt = slice(max(0, dy), min(h, h + dy))
    xt = slice(max(0, dx), min(w, w + dx))
    out[ys, xs] = t[yt, xt]
    return out


def soft_bp(cost, levels, params, P1, P2, tau):
    """cost (ch, cw, D) float64 tensor, levels (H, W) numpy int, P1 / P2
    float64 scalar tensors.  Returns the sparse depth (H, W) tensor."""
    H, W = levels.shape
    D = cost.shape[-1]
    L = params.bp_levels
    data = [cost]
    for _ in range(1, L):
        a = data[-1]
        h, w = a.shape[:2]
        ph, pw = (h + 1) // 2, (w + 1) // 2
        b = torch.zeros((ph, pw, D), dtype=a.dtype)
        for j in range(2):
            for i in range(2):
                sub = a[j::2, i::2]
                b[:sub.shape[0], :sub.shape[1]] = b[:sub.shape[0], :sub.shape[1]] + sub
        data.append(b)
    msgs = None
    for l in range(L - 1, -1, -1):
        h, w = data[l].shape[:2]
        if msgs is None:
            m = [torch.zeros((h, w, D), dtype=cost.dtype) for _ in range(4)]
        else:
            yy = torch.arange(h) // 2
            xx = torch.arange(w) // 2
            m = [p[yy][:, xx] for p in msgs]
        ys = torch.arange(h)[:, None].expand(h, w)
        xs = torch.arange(w)[None, :].expand(h, w)
        ilev = l + 2
        if ilev <= params.qt_max_level:
            size = 1 << ilev
            sx = np.minimum((xs.numpy() >> 1) * size, W - 1)
            sy = np.minimum(ys.numpy() * size, H - 1)
            keep = torch.from_numpy(levels[sy, sx] <= ilev)
        else:
            keep = torch.ones((h, w), dtype=torch.bool)
        has_u = (ys > 0)[..., None]
        has_d = (ys < h - 1)[..., None]
        has_l = (xs > 0)[..., None]
        has_r = (xs < w - 1)[..., None]
        dpos = torch.arange(D)
        for it in range(params.bp_iters[l]):
            parity = it & 1
            upd = (keep & ((xs & 1) == ((ys + parity) & 1)))[..., None]
            fu = _shift(m[DOWN], -1, 0)   # message of the upper neighbour
            fd = _shift(m[UP], 1, 0)
            fl = _shift(m[RIGHT], 0, -1)
            fr = _shift(m[LEFT], 0, 1)
            zero = torch.zeros_like(fu)
            fu, fd = torch.where(has_u, fu, zero), torch.where(has_d, fd, zero)
            fl, fr = torch.where(has_l, fl, zero), torch.where(has_r, fr, zero)
            new = []
            for dr in range(4):
                hv = data[l].clone()
                if dr != UP:
                    hv = hv + fu
                if dr != DOWN:
                    hv = hv + fd
                if dr != LEFT:
                    hv = hv + fl
                if dr != RIGHT:
                    hv = hv + fr
                big = torch.full_like(hv[..., :1], float("inf"))
                prev = torch.cat([big, hv[..., :-1]], -1) + P1
                nxt = torch.cat([hv[..., 1:], big], -1) + P1
                mv = torch.minimum(torch.minimum(hv, prev), nxt)
                mv = torch.minimum(mv, hv.min(-1, keepdim=True).values + P2)
                new.append(mv - mv.mean(-1, keepdim=True))
            m = [torch.where(upd, new[dr], m[dr]) for dr in range(4)]
        msgs = m
    # soft readout at level-0 node cells
    h, w = data[0].shape[:2]
    b = data[0] + _shift(msgs[RIGHT], 0, -1) + _shift(msgs[LEFT], 0, 1) \
        + _shift(msgs[DOWN], -1, 0) + _shift(msgs[UP], 1, 0)
    p = torch.softmax(-b / tau, -1)
    disp = (p * torch.arange(D, dtype=b.dtype)).sum(-1)
    depth = 1.0 / (params.inv_depth_step * disp + params.min_inv_depth)
    out = torch.zeros((H, W), dtype=cost.dtype)
    for y in range(h):
        for x in range(w):
            lvl = levels[min(y * 4, H - 1), min(x * 4, W - 1)]
            size = 1 << int(lvl)
            if (x * 4) % size == 0 and (y * 4) % size == 0:
                out[y * 4, x * 4] = depth[y, x]
    return out
