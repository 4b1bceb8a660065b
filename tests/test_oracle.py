"""CPU checks of the oracle itself (properties the reference's algorithm must
have).  The oracle's parity with the reference kernels is pinned by
tests/test_golden.py."""
import numpy as np
import pytest
from scipy.linalg import solve_banded

from conftest import cam_of, keyframe
from open_quadtree_mapping_b200.params import Params


def test_quadtree_uniform_and_noise(oracle_mod):
    p = Params()
    flat = np.full((64, 96), 77, np.uint8)
    assert (oracle_mod.quadtree(flat, p) == 4).all()
    rng = np.random.default_rng(0)
    noise = rng.integers(0, 256, (64, 96), dtype=np.uint8)
    lv = oracle_mod.quadtree(noise, p)
    assert (lv == 2).mean() > 0.99  # clamped minimum level


def test_quadtree_threshold_and_children(oracle_mod):
    p = Params()
    img = np.full((32, 32), 100, np.uint8)
    # one 4x4 block with a deviation of exactly 10 from its mean stays approved
    img[0:4, 0:4] = np.array([[100, 120], [100, 100]]).repeat(2, 0).repeat(2, 1)[:4, :4]
    lv = oracle_mod.quadtree(img, p)
    assert lv.shape == img.shape
    # a 2x2 block {0,0,0,14}: fails its own test (14 - 3.5 > 10) while the
    # 4x4 block around it would pass on its own; the child failure must cap
    # the 4x4 block's pixels below level 2 -> clamp to 2
    img2 = np.full((16, 16), 7, np.uint8)
    img2[0:2, 0:2] = [[0, 0], [0, 14]]
    img2[2:4, 0:4] = 7
    lv2 = oracle_mod.quadtree(img2, p)
    assert (lv2[0:4, 0:4] == 2).all()
    # the other 8x8 quadrants are uniform -> level 3 (16x16 block fails)
    assert (lv2[8:16, 8:16] == 3).all()
    # incomplete blocks at the border: height 20 -> bottom rows cannot reach 4
    img3 = np.full((20, 32), 50, np.uint8)
    lv3 = oracle_mod.quadtree(img3, p)
    assert (lv3[:16] == 4).all() and (lv3[16:20] == 2).all()


def test_cost_identity_pose_is_zero(oracle_mod):
    kf = keyframe(0, 160, 128)
    p = Params.for_range(64, 0.5, 50.0)
    lv = oracle_mod.quadtree(kf.ref, p)
    T = np.tile(np.eye(3, 4, dtype=np.float32).reshape(1, 12), (3, 1))
    cost, valid = oracle_mod.cost_volume(kf.ref, lv, [kf.ref] * 3, T, cam_of(kf), p)
    assert valid.sum() > 0
    assert (cost[valid == 1] == 0).all()
    # border cells and non-node cells are zero
    assert (cost[0] == 0).all() and (cost[:, 0] == 0).all()


def test_cost_out_of_view_is_100_over_d(oracle_mod):
    kf = keyframe(0, 160, 128)
    p = Params.for_range(64, 0.5, 50.0)
    lv = oracle_mod.quadtree(kf.ref, p)
    T = np.eye(3, 4, dtype=np.float32)
    T[0, 3] = 1e4  # moved far sideways: nothing projects into the image
    cost, valid = oracle_mod.cost_volume(kf.ref, lv, [kf.ref], T.reshape(1, 12), cam_of(kf), p)
    # 100 for no valid slot, divided by the writer count (the hypothesis count)
    assert (cost[valid == 1] == np.float32(100) / np.float32(64)).all()


def _tree_sum(v):
    v = list(v)
    n = 1
    while n < len(v):
        n *= 2
    v += [0.0] * (n - len(v))
    v = np.array(v, np.float32)
    s = n // 2
    while s > 0:
        v[:s] = v[:s] + v[s:2 * s]
        s //= 2
    return v[0]


def test_bp_clear_minimum_and_normalised_messages(oracle_mod):
    W, H, D = 128, 96, 64
    p = Params(num_hyp=D)
    lv = np.full((H, W), 2, np.int32)
    cost = np.ones((H // 4, W // 4, D), np.float32)
    cost[:, :, 17] = 0.0
    labels, sparse, msgs = oracle_mod.bp_extract(cost, W, H, lv, p, want_messages=True)
    assert (labels == 17).all()
    # every written message is mean-normalised with the reference's tree sum
    m = msgs[0, 5, 7]
    assert abs(_tree_sum(m)) < 1e-5
    # node pixels get 1/(min + step*disparity)
    d = sparse[0:H:4, 0:W:4]
    assert np.isfinite(d).all() and (d > 0).all()


def test_bp_skip_keeps_coarse_messages(oracle_mod):
    """Level-0 cells whose quadtree sample is coarser than the level are not
    updated (bpextract.cu:214-220)."""
    W, H, D = 128, 96, 64
    p = Params(num_hyp=D)
    rng = np.random.default_rng(1)
    cost = rng.random((H // 4, W // 4, D)).astype(np.float32)
    lv_fine = np.full((H, W), 2, np.int32)
    lv_coarse = np.full((H, W), 4, np.int32)
    la, _, ma = oracle_mod.bp_extract(cost, W, H, lv_fine, p, want_messages=True)
    lb, _, mb = oracle_mod.bp_extract(cost, W, H, lv_coarse, p, want_messages=True)
    assert not np.array_equal(ma, mb)
    # level 4 everywhere: only cells at multiples of 16 px are node origins
    assert (lb >= 0).sum() == ((W // 16) * (H // 16))


def _thomas_dense(w, r, lam):
    """Solve (I + lam*L_w) s = r with a banded solver; w[k] joins k-1 and k."""
    n = len(r)
    wl = np.array([0.0] + list(w[1:n]))
    wr = np.array(list(w[1:n + 1]))
    ab = np.zeros((3, n))
    ab[0, 1:] = -lam * wr[:-1]
    ab[1, :] = 1.0 + lam * (wl + wr)
    ab[2, :-1] = -lam * wl[1:]
    return solve_banded((1, 1), ab, r)


def test_upsample_matches_banded_solve(oracle_mod):
    kf = keyframe(0, 64, 48)
    p = Params()
    rng = np.random.default_rng(3)
    sparse = np.zeros((48, 64), np.float64)
    mask = rng.random(sparse.shape) < 0.08
    sparse[mask] = rng.uniform(0.5, 8.0, mask.sum())
    dense = oracle_mod.upsample(sparse, kf.ref, p)
    # weights in double (the fp64 oracle keeps them unrounded); W=64 and
    # H=48 are multiples of 16, so the closing weights are 0
    I = kf.ref.astype(np.float64)
    row_w = np.zeros((48, 65))
    row_w[:, 1:64] = np.exp(-np.diff(I, axis=1) ** 2 / p.up_sigma)
    col_w = np.zeros((49, 64))
    col_w[1:48, :] = np.exp(-np.diff(I, axis=0) ** 2 / p.up_sigma)
    lam = p.up_lambda
    ind = (sparse > 0).astype(np.float64)
    rd = np.stack([_thomas_dense(row_w[y], sparse[y], lam) for y in range(48)])
    ri = np.stack([_thomas_dense(row_w[y], ind[y], lam) for y in range(48)])
    cd = np.stack([_thomas_dense(col_w[:, x], rd[:, x], lam) for x in range(64)], 1)
    ci = np.stack([_thomas_dense(col_w[:, x], ri[:, x], lam) for x in range(64)], 1)
    ref = cd / ci
    assert np.allclose(dense, ref, rtol=1e-10, atol=0)


def test_upsample_weight_grid_quirk(oracle_mod):
    """row_w(W, .) = 1 when W % 16 != 0, else 0; col_w(., H) likewise."""
    img = np.random.default_rng(0).integers(0, 255, (40, 72), dtype=np.uint8)
    rw, cw = oracle_mod.upsample_weights(img, Params())
    assert (rw[:, 72] == 1).all() and (cw[40, :] == 1).all()
    img2 = np.random.default_rng(0).integers(0, 255, (48, 64), dtype=np.uint8)
    rw2, cw2 = oracle_mod.upsample_weights(img2, Params())
    assert (rw2[:, 64] == 0).all() and (cw2[48, :] == 0).all()
    assert (rw2[:, 0] == 0).all() and (cw2[0, :] == 0).all()


def test_fuse_first_frame_is_invalid(oracle_mod):
    """Zero seeds: every prior is (10, 10), ratio 0.5 <= 0.6 -> output -1."""
    kf = keyframe(0, 64, 48)
    depth = np.full((48, 64), 3.0, np.float32)
    seeds = np.zeros((48, 64, 4), np.float32)
    out, new, table, contested = oracle_mod.fuse(depth, seeds, np.eye(3, 4), cam_of(kf))
    assert (out == -1).all()
    assert (table == 0).all() and not contested.any()
    assert np.allclose(new[..., 2], 3.0, rtol=1e-6)


def test_fuse_identity_keeps_pixels(oracle_mod):
    """With an identity motion every good seed lands on its own pixel."""
    kf = keyframe(0, 64, 48)
    depth = np.full((48, 64), 3.0, np.float32)
    seeds = np.zeros((48, 64, 4), np.float32)
    seeds[..., 0] = 30.0
    seeds[..., 1] = 5.0
    seeds[..., 2] = 3.0
    seeds[..., 3] = 0.01
    out, new, table, contested = oracle_mod.fuse(depth, seeds, np.eye(3, 4), cam_of(kf))
    idx = np.arange(48 * 64).reshape(48, 64)
    ok = ~contested.astype(bool)
    assert (table[ok][1:] == idx[ok][1:]).all()
    assert np.allclose(out[1:, 1:], 3.0, rtol=1e-5)
