"""The oracle pinned against the reference's own kernels.

tests/golden/*.npz are dumps of the reference's CUDA kernels (built from its
sources for sm_100a with -use_fast_math, run on a B200 by
tests/golden/make_golden.py) on seeded synthetic inputs.  The oracle uses
IEEE arithmetic where the reference build uses fast-math divisions and
rsqrtf, so: levels, node masks and fusion tables are bit-exact; costs agree
to the last bits except where a rounded projection falls within a fast-math
error of a .5 boundary (a handful of cells); labels agree except at those.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from open_quadtree_mapping_b200.params import Params

EXTRACT = ["ref_extract_64x48", "ref_extract_160x128", "ref_extract_320x240"]


def _load(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail("missing golden fixture %s" % path)
    return np.load(path)


@pytest.mark.parametrize("name", EXTRACT)
def test_oracle_extract_vs_reference_kernels(name, oracle_mod):
    z = _load(name)
    ref = z["ref"]
    slots = [z["ring"][k] for k in z["slots"]]
    T = z["T_ring_ref"][z["slots"]]
    cam = tuple(float(c) for c in z["cam"])
    o = oracle_mod.extract_depth(ref, slots, T, cam, Params(), want_messages=True)
    assert np.array_equal(o["levels"], z["levels"])
    if "cost" in z.files:
        rc = z["cost"]
        close = np.isclose(o["cost"], rc, rtol=1e-6, atol=1e-9)
        assert close.mean() > 0.999, close.mean()  # elements off by a straddle
        assert np.abs(o["cost"] - rc).max() < 1e-2
    lab = z["labels"]
    node = lab >= 0
    assert np.array_equal(o["labels"] >= 0, node)
    agree = (o["labels"][node] == lab[node]).mean()
    assert agree > 0.999, agree
    sp = z["sparse"]
    m = sp != 0
    assert np.array_equal(o["sparse"] != 0, m)
    rel = np.abs(o["sparse"][m] - sp[m]) / sp[m]
    # a straddle-affected cost moves the parabola of its cell
    assert np.mean(rel < 1e-6) > 0.99
    d = z["dense"]
    fin = np.isfinite(d)
    assert np.array_equal(np.isfinite(o["dense"]), fin)
    reld = np.abs(o["dense"][fin] - d[fin]) / np.abs(d[fin])
    assert np.percentile(reld, 99) < 1e-4
    assert np.median(reld) < 1e-6
    if "messages" in z.files:
        assert np.allclose(o["messages"], z["messages"], rtol=0, atol=1e-6)


def test_oracle_fuse_vs_reference_kernels(oracle_mod):
    z = _load("ref_fuse_160x128")
    cam = tuple(float(c) for c in z["cam"])
    dense = z["dense"].astype(np.float32)
    d1, s1, t1, c1 = oracle_mod.fuse(dense, np.zeros((128, 160, 4), np.float32), z["T1"], cam)
    assert np.array_equal(d1, z["fused1"])
    assert np.array_equal(t1, z["table1"])
    assert np.allclose(s1, z["seeds1"], rtol=2e-5, atol=1e-7)
    d2, s2, t2, c2 = oracle_mod.fuse(dense, z["seeds1"], z["T2"], cam)
    ok = c2 == 0
    assert ok.mean() > 0.9
    assert np.array_equal(t2[ok], z["table2"][ok])
    assert np.array_equal(d2[ok], z["fused2"][ok])
    assert np.allclose(s2[ok], z["seeds2"][ok], rtol=2e-5, atol=1e-7)


def test_oracle_point_cloud_vs_reference_host_arithmetic(oracle_mod):
    """tests/golden/ref_pointcloud_160x128.npz holds the publisher's point
    cloud evaluated with the reference's own helper_math.h / se3.cuh host
    arithmetic (tests/golden/make_pointcloud_golden.py): the oracle matches
    it bit for bit, NaN depths (kept by the reference's `< 0.1` test) and the
    0.1 cut included."""
    z = _load("ref_pointcloud_160x128")
    pts = oracle_mod.point_cloud(z["depth"], z["ref"], tuple(float(c) for c in z["cam"]),
                                 z["T_world_ref"])
    want = z["points"]
    assert len(want) > 1000 and np.isnan(want[:, 0]).sum() == 8
    assert pts.shape == want.shape
    assert np.array_equal(pts.view(np.uint32), want.view(np.uint32))


def test_oracle_semidense_vs_reference_kernels(oracle_mod):
    """tests/golden/ref_semidense_160x128.npz: the reference's own semi-dense
    tracker kernels over 24 frames (tests/golden/make_semidense_golden.py).
    The reference's hole filling and regularisation run in place and its
    collisions resolve by scheduling: two runs of the reference itself share
    only ~25 % bit-identical projected depths by frame 23 (93 % of the
    projected pixels in common, median relative difference 2e-5).  The
    oracle is deterministic (Jacobi passes, nearest-wins collisions) and
    IEEE, with the texture unit's bilinear arithmetic; it must follow the
    same step modes and stay close: up to the first keyframe switch 99 % of
    the projected pixels in common with a median relative difference near
    1e-6, later frames drifting slowly (79 % / 2e-3 by frame 23)."""
    from oracle.policy import PolicyReplay
    z = _load("ref_semidense_160x128")
    frames, Ts = z["frames"], z["T_cur_world"]
    cam = tuple(float(c) for c in z["cam"])
    H, W = frames.shape[1:]
    pol = PolicyReplay()
    trk = np.zeros((H, W, 4), np.float32)
    dep = np.zeros((H, W, 4), np.float32)
    for i in range(len(frames)):
        r = pol.add(i, Ts[i])
        assert r["sd_mode"] == z["modes"][i], i
        k = r["sd_key"]
        d = oracle_mod.sd_step(frames[k] if k is not None else None, frames[i], cam, r["sd_T"],
                               r["sd_mode"], trk, dep)
        ref = z["debug"][i]
        either = (d > 0) | (ref > 0)
        both = (d > 0) & (ref > 0)
        if not either.any():
            continue
        overlap = both.sum() / either.sum()
        rel = np.median(np.abs(d[both] - ref[both]) / ref[both])
        if i <= 6:  # up to the first keyframe switch (propagation races)
            assert overlap > 0.985 and rel < 1e-5, (i, overlap, rel)
        assert overlap > 0.7 and rel < 1e-2, (i, overlap, rel)
    assert ((trk[..., 0] > 0) == (z["seeds"][..., 0] > 0)).mean() > 0.95
