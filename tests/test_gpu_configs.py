"""The workloads the reference is measured on, at their full sizes.

* Large keyframe: 1920x1080 (fx = fy = 1150), 128 hypotheses, 20 distinct
  measurement frames, 5-level quadtree.  IEEE arithmetic: levels, cost
  volume, labels and sparse depths bit-exact with the oracle; upsampled depth
  within 1e-5 relative of the FP64 oracle for 99.9 % of the pixels and
  1e-4 for all.
* Video sequence: one stream at 1280x720 (fx = fy = 780), 64 hypotheses,
  10 measurement slots, 30 frames with Bayesian fusion across keyframes,
  IEEE arithmetic, against an oracle replay of the same frame policy: debug
  map (sparse BP depths) bit-exact on every dense frame; fused depth and
  variance within 1e-5 relative at the 99th percentile.
* Uneven batch: 16 streams (6 at 640x480, 6 at 752x480, 4 at 1280x720), 3-10
  measurement frames and 48/64/96 hypotheses per stream, one launch per
  stage: every stream's fused depth bit-identical to the same stream run
  alone.

Frames are rendered in a process pool (spawn start: the test process has a
CUDA context).
"""
import multiprocessing as mp

import numpy as np
import pytest
import torch

from open_quadtree_mapping_b200.params import ARITH_IEEE, Params

pytestmark = pytest.mark.gpu

UPSAMPLE_RTOL = 1e-5
FUSE_RTOL = 1e-5


def _render(args):
    from open_quadtree_mapping_b200 import synthetic as syn
    seed, T, W, H, f = args
    img, gt = syn.render(syn.make_scene(seed), T, W, H, f, f, W / 2.0, H / 2.0)
    return img, gt


def _render_all(jobs):
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(8, len(jobs))) as pool:
        return pool.map(_render, jobs)


def test_large_keyframe_vs_oracle(oracle_mod, gpu):
    from open_quadtree_mapping_b200 import stages
    from open_quadtree_mapping_b200 import synthetic as syn
    W, H, f, F, s = 1920, 1080, 1150.0, 20, 9
    traj = syn.make_trajectory(2000 + s, F + 1)
    frames = _render_all([(1000 + s, traj[k], W, H, f) for k in range(F + 1)])
    ref = frames[F][0]
    meas = [frames[F - 1 - k][0] for k in range(F)]
    T = np.stack([(syn.inv_se3(traj[F - 1 - k]) @ traj[F])[:3, :4].reshape(-1)
                  for k in range(F)]).astype(np.float32)
    cam = (f, f, W / 2.0, H / 2.0)
    p = Params.for_range(128, 0.5, 50.0, arith=ARITH_IEEE, qt_max_level=5)
    oracle_mod.set_threads(8)
    o = oracle_mod.extract_depth(ref, meas, T, cam, p)
    g = stages.extract_depth(torch.from_numpy(ref).to(gpu),
                             [torch.from_numpy(np.ascontiguousarray(m)).to(gpu) for m in meas],
                             T, cam, p)
    g = {k: (v.cpu().numpy() if v is not None else None) for k, v in g.items()}
    assert (o["levels"] == 5).any()  # the 5-level quadtree is exercised
    assert np.array_equal(g["levels"], o["levels"])
    assert np.array_equal(g["cost"], o["cost"])
    assert np.array_equal(g["labels"], o["labels"])
    assert np.array_equal(g["sparse"], o["sparse"])
    # upsampled depth against the FP64 oracle on the same sparse depths: the
    # GPU eliminates with FP64 pivots and FP32 right-hand sides over lines of
    # 1920 and 1080 samples
    d64 = oracle_mod.upsample(o["sparse"].astype(np.float64), ref, p)
    ok = np.isfinite(d64) & (d64 > 0)
    assert ok.mean() > 0.9
    rel = np.abs(g["dense"][ok] - d64[ok]) / d64[ok]
    stats = (np.percentile(rel, 99.9), rel.max())
    assert stats[0] < UPSAMPLE_RTOL and stats[1] < 10 * UPSAMPLE_RTOL, stats


def test_video_720p_sequence_vs_oracle_replay(oracle_mod, gpu):
    """The 720p, 10-slot, 30-frame sequence through the batched engine (one
    stream; the facade is fixed at the reference's 5 slots) against the
    oracle replaying the same frame policy: quadtree, cost, BP and
    extraction in IEEE arithmetic equal the oracle bit for bit, so the debug
    map must too; the upsampled depth (FP32 right-hand sides here, FP64 in
    the replay) and the FP64 fusion then agree within FUSE_RTOL."""
    from open_quadtree_mapping_b200 import synthetic as syn
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    from oracle.policy import PolicyReplay
    W, H, f, F, n, s = 1280, 720, 780.0, 10, 30, 41
    traj = syn.make_trajectory(2000 + s, n)
    imgs = _render_all([(1000 + s, traj[i], W, H, f) for i in range(n)])
    imgs = [im for im, _ in imgs]
    Ts = [np.ascontiguousarray(syn.inv_se3(traj[i])[:3, :4].reshape(-1), np.float32)
          for i in range(n)]
    cam = (f, f, W / 2.0, H / 2.0)
    p = Params(arith=ARITH_IEEE)
    b = BatchDepthmap([dict(width=W, height=H, fx=f, fy=f, cx=W / 2.0, cy=H / 2.0, num_hyp=64,
                            num_slots=F)], params=p)
    pol = PolicyReplay(num_slots=F)
    oracle_mod.set_threads(8)
    seeds = np.zeros((H, W, 4), np.float32)
    n_dense = n_valid = n_oracle_valid = 0
    worst_depth = worst_var = 0.0
    for i in range(n):
        has = b.add_frames([imgs[i]], [Ts[i]])[0]
        r = pol.add(i, Ts[i])
        assert has == (r["outcome"] in ("first", "dense")), (i, r["outcome"])
        if r["outcome"] != "dense":
            continue
        n_dense += 1
        o = oracle_mod.extract_depth(imgs[i], [imgs[k] for k in r["slots"]], r["T_slots"], cam,
                                     p)
        assert np.array_equal(b.get_debug(0), o["sparse"]), i
        dense64 = oracle_mod.upsample(o["sparse"].astype(np.float64), imgs[i], p)
        fused, new_seeds, _, _ = oracle_mod.fuse(dense64, seeds, r["T_fuse"], cam)
        seeds = new_seeds.astype(np.float32)
        depth = b.get_depth(0)
        var = b.get_variance(0)
        valid = fused > 0
        n_oracle_valid += valid.sum()
        assert (depth > 0).mean() == pytest.approx(valid.mean(), abs=2e-3), i
        both = valid & (depth > 0)
        n_valid += both.sum()
        if both.any():
            rel = np.abs(depth[both] - fused[both]) / fused[both]
            worst_depth = max(worst_depth, float(np.percentile(rel, 99)))
        # the variance of every seed the update wrote, valid or not
        upd = new_seeds[..., 3] > 0
        relv = np.abs(var[upd] - new_seeds[..., 3][upd]) / new_seeds[..., 3][upd]
        worst_var = max(worst_var, float(np.percentile(relv, 99)))
    assert n_dense >= 15
    assert n_oracle_valid > 0
    assert n_valid == pytest.approx(n_oracle_valid, rel=0.01, abs=50)
    assert worst_depth < FUSE_RTOL and worst_var < FUSE_RTOL, (worst_depth, worst_var)


def test_uneven_16_stream_batch_equals_single_streams(gpu):
    from open_quadtree_mapping_b200 import synthetic as syn
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    sizes = {(640, 480): 460.0 * 640 / 752, (752, 480): 460.0, (1280, 720): 780.0}
    n_frames = 13
    seqs = {}
    jobs = []
    for k, (W, H) in enumerate(sizes):
        traj = syn.make_trajectory(2100 + k, n_frames)
        # the renderer takes camera->world poses; the API takes world->camera
        jobs += [(1100 + k, traj[i], W, H, sizes[(W, H)]) for i in range(n_frames)]
        seqs[(W, H)] = [np.ascontiguousarray(syn.inv_se3(traj[i])[:3, :4], np.float32)
                        for i in range(n_frames)]
    frames = _render_all(jobs)
    imgs = {}
    for k, (W, H) in enumerate(sizes):
        imgs[(W, H)] = [frames[k * n_frames + i][0] for i in range(n_frames)]
    rng = np.random.default_rng(16)
    layout = [(640, 480)] * 6 + [(752, 480)] * 6 + [(1280, 720)] * 4
    descs = []
    for (W, H) in layout:
        descs.append(dict(width=W, height=H, fx=sizes[(W, H)], fy=sizes[(W, H)], cx=W / 2.0,
                          cy=H / 2.0, num_hyp=int(rng.choice([48, 64, 96])),
                          num_slots=int(rng.integers(3, 11))))
    p = Params.for_range(64, 0.5, 50.0)
    batch = BatchDepthmap(descs, params=p)
    singles = [BatchDepthmap([d], params=p) for d in descs]
    for i in range(n_frames):
        frame = [imgs[sz][i] for sz in layout]
        poses = [seqs[sz][i] for sz in layout]
        hb = batch.add_frames(frame, poses)
        for k in range(len(layout)):
            assert singles[k].add_frames([frame[k]], [poses[k]])[0] == hb[k]
    assert all(hb)
    for k in range(len(layout)):
        assert np.array_equal(batch.get_depth(k), singles[k].get_depth(0)), k
        assert np.array_equal(batch.get_debug(k), singles[k].get_debug(0)), k
