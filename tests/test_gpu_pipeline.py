"""GPU tests of the Depthmap facade and the batched multi-stream path, all
through the C-ABI (libqm_b200.so)."""
import numpy as np
import pytest

from conftest import sequence
from open_quadtree_mapping_b200.params import ARITH_IEEE, Params
from oracle.policy import PolicyReplay

pytestmark = pytest.mark.gpu

W, H = 160, 128
F_PX = 460.0 * W / 752.0


def _stream_kw(W=W, H=H, f=F_PX, **kw):
    d = dict(width=W, height=H, fx=f, fy=f, cx=W / 2.0, cy=H / 2.0)
    d.update(kw)
    return d


def test_facade_matches_oracle_replay(oracle_mod, gpu):
    """Depthmap over a 16-frame sequence: has_result flags follow the frame
    policy, the debug map (sparse BP depths) is bit-exact with the oracle in
    IEEE mode, and the fused depth agrees with an oracle replay."""
    from open_quadtree_mapping_b200.depthmap import Depthmap
    n_frames = 40
    imgs, Ts, gts = sequence(1, n_frames, W, H)
    p = Params(arith=ARITH_IEEE)  # the reference's hypothesis range
    dm = Depthmap(W, H, F_PX, W / 2.0, F_PX, H / 2.0, semi2dense_ratio=1, params=p)
    pol = PolicyReplay(num_slots=5)
    cam = (F_PX, F_PX, W / 2.0, H / 2.0)
    seeds = np.zeros((H, W, 4), np.float32)
    n_dense = 0
    n_valid = 0
    n_oracle_valid = 0
    for i in range(n_frames):
        has = dm.add_frames(imgs[i], Ts[i])
        r = pol.add(i, Ts[i])
        assert has == (r["outcome"] in ("first", "dense")), (i, r["outcome"])
        if r["outcome"] == "first":
            assert (dm.getDepthmap() == 0).all()
            continue
        if r["outcome"] != "dense":
            continue
        n_dense += 1
        slots = [imgs[k] for k in r["slots"]]
        o = oracle_mod.extract_depth(imgs[i], slots, r["T_slots"], cam, p)
        debug = dm.getDebugmap()
        assert np.array_equal(debug, o["sparse"])
        dense64 = oracle_mod.upsample(o["sparse"].astype(np.float64), imgs[i], p)
        fused, new_seeds, _, contested = oracle_mod.fuse(dense64, seeds, r["T_fuse"], cam)
        seeds = new_seeds.astype(np.float32)
        depth = dm.getDepthmap()
        valid = fused > 0
        n_oracle_valid += valid.sum()
        # fused variance: sigma^2 of the new seeds where both fused the pixel
        var = dm.getVariancemap()
        ok = valid & (depth > 0)
        if ok.any():
            ov = new_seeds[..., 3][ok]
            rel = np.abs(var[ok] - ov) / np.maximum(np.abs(ov), 1e-6)
            assert np.percentile(rel, 99) < 1e-4, np.percentile(rel, 99)
        assert (depth > 0).mean() == pytest.approx(valid.mean(), abs=2e-3)
        both = valid & (depth > 0)
        n_valid += both.sum()
        if both.any():
            rel = np.abs(depth[both] - fused[both]) / fused[both]
            assert np.percentile(rel, 99) < 1e-5, np.percentile(rel, 99)
        assert np.array_equal(dm.getReferenceImage(), imgs[i])
        T_wr = dm.getT_world_ref()
        from oracle.policy import se3_inv
        assert np.array_equal(T_wr.reshape(12), se3_inv(Ts[i]))
    assert n_dense >= 20
    # the fused output turns valid only after ~15 consistent updates
    assert n_valid == pytest.approx(n_oracle_valid, rel=0.01, abs=50)


def test_batch_equals_plain_and_graph_equals_eager(gpu):
    """Three streams run batched (one launch per stage, graph replay) give
    bit-identical maps to three single-stream runs, to eager launches, to
    other BP job groupings and branch counts, and with the coarse BP levels
    swept per launch or all levels in the cluster launch."""
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    seqs = [sequence(s, 14, W, H) for s in (2, 3, 4)]
    p = Params.for_range(64, 0.5, 50.0)
    batch = BatchDepthmap([_stream_kw()] * 3, params=p)
    eager = BatchDepthmap([_stream_kw()] * 3, params=p)
    eager.set_graphs(False)
    # BP job ranges: one stream per range, and all streams in one range
    split = BatchDepthmap([_stream_kw()] * 3, params=p)
    split.set_group_bytes(1)
    whole = BatchDepthmap([_stream_kw()] * 3, params=p)
    whole.set_group_bytes(0)
    # one launch sequence over all streams (the default runs two concurrent
    # branches over the halves of the streams)
    branched = BatchDepthmap([_stream_kw()] * 3, params=p)
    branched.set_branches(1)
    # the coarse BP levels one launch per half-sweep (the reference's launch
    # sequence), and every level in the cluster launch (extraction included)
    coarse_off = BatchDepthmap([_stream_kw()] * 3, params=p)
    coarse_off.set_coarse_bp(0)
    coarse_all = BatchDepthmap([_stream_kw()] * 3, params=p)
    coarse_all.set_coarse_bp(1 << 30)
    # branches staggered behind each other's cost volume instead of started
    # together, and three branches
    staggered = BatchDepthmap([_stream_kw()] * 3, params=p)
    staggered.set_stagger(True)
    three = BatchDepthmap([_stream_kw()] * 3, params=p)
    three.set_branches(3)
    singles = [BatchDepthmap([_stream_kw()], params=p) for _ in range(3)]
    for i in range(14):
        imgs = [s[0][i] for s in seqs]
        poses = [s[1][i] for s in seqs]
        hb = batch.add_frames(imgs, poses)
        he = eager.add_frames(imgs, poses)
        assert split.add_frames(imgs, poses) == hb
        assert whole.add_frames(imgs, poses) == hb
        assert branched.add_frames(imgs, poses) == hb
        assert coarse_off.add_frames(imgs, poses) == hb
        assert coarse_all.add_frames(imgs, poses) == hb
        assert staggered.add_frames(imgs, poses) == hb
        assert three.add_frames(imgs, poses) == hb
        hs = [singles[k].add_frames([imgs[k]], [poses[k]])[0] for k in range(3)]
        assert hb == he == hs
        if all(hb) and i > 0:
            together = batch.get_depths()
            for k in range(3):
                a = batch.get_depth(k)
                assert np.array_equal(a, together[k])
                assert np.array_equal(a, eager.get_depth(k))
                assert np.array_equal(a, split.get_depth(k))
                assert np.array_equal(a, whole.get_depth(k))
                assert np.array_equal(a, branched.get_depth(k))
                assert np.array_equal(a, coarse_off.get_depth(k))
                assert np.array_equal(a, coarse_all.get_depth(k))
                assert np.array_equal(a, staggered.get_depth(k))
                assert np.array_equal(a, three.get_depth(k))
                assert np.array_equal(batch.get_debug(k), coarse_off.get_debug(k))
                assert np.array_equal(a, singles[k].get_depth(0))
                assert np.array_equal(batch.get_debug(k), singles[k].get_debug(0))
    assert batch.last_launches() > 0


def test_submit_pipeline_equals_add_frames(gpu):
    """qm_batch_submit (two steps in flight, uploads and downloads on their
    own streams) gives the same flags and bit-identical depth maps as the
    synchronous add_frames + get_depths, frame by frame."""
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    seqs = [sequence(s, 16, W, H) for s in (5, 6, 7)]
    p = Params.for_range(64, 0.5, 50.0)
    sync = BatchDepthmap([_stream_kw()] * 3, params=p)
    pipe = BatchDepthmap([_stream_kw()] * 3, params=p)
    want, got = [], []
    for i in range(16):
        imgs = [s[0][i] for s in seqs]
        poses = [s[1][i] for s in seqs]
        hs = sync.add_frames(imgs, poses)
        want.append((hs, [d.copy() for d in sync.get_depths()]))
        outs = [np.full((H, W), np.nan, np.float32) for _ in range(3)]
        hp = pipe.submit(imgs, poses, outs=outs)
        got.append((hp, outs))
    pipe.wait()
    for (hs, ds), (hp, outs) in zip(want, got):
        assert hs == hp
        for k in range(3):
            if hp[k]:
                assert np.array_equal(ds[k], outs[k])
            else:
                assert np.isnan(outs[k]).all()  # nothing downloaded
    # the synchronous getters wait for submitted work by themselves
    imgs = [s[0][15] for s in seqs]
    pipe.submit(imgs, [s[1][15] for s in seqs])
    sync.add_frames(imgs, [s[1][15] for s in seqs])
    for k in range(3):
        assert np.array_equal(pipe.get_depth(k), sync.get_depth(k))


def test_uneven_batch_equals_per_stream(gpu):
    """Streams of different sizes, hypothesis and slot counts in one batch."""
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    shapes = [(160, 128, 64, 5), (192, 144, 48, 3), (128, 96, 96, 7), (160, 120, 32, 2)]
    seqs = [sequence(10 + k, 13, w, h) for k, (w, h, _, _) in enumerate(shapes)]
    p = Params.for_range(64, 0.5, 50.0)
    descs = [_stream_kw(W=w, H=h, f=460.0 * w / 752.0, num_hyp=d, num_slots=f)
             for (w, h, d, f) in shapes]
    batch = BatchDepthmap(descs, params=p)
    batch.set_group_bytes(3 << 20)  # ranges of one or two streams
    singles = [BatchDepthmap([d], params=p) for d in descs]
    for i in range(13):
        imgs = [s[0][i] for s in seqs]
        poses = [s[1][i] for s in seqs]
        hb = batch.add_frames(imgs, poses)
        for k in range(len(shapes)):
            assert singles[k].add_frames([imgs[k]], [poses[k]])[0] == hb[k]
    for k in range(len(shapes)):
        assert np.array_equal(batch.get_depth(k), singles[k].get_depth(0))
        assert np.array_equal(batch.get_debug(k), singles[k].get_debug(0))
    batch.run_resident()


def test_semi2dense_ratio_and_resident_errors(gpu):
    from open_quadtree_mapping_b200 import _lib
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    imgs, Ts, _ = sequence(5, 16, W, H)
    b = BatchDepthmap([_stream_kw(semi2dense_ratio=3)], params=Params())
    with pytest.raises(_lib.QmError) as e:
        b.run_resident()
    assert e.value.status == _lib.QM_ERR_STATE
    flags = [b.add_frames([imgs[i]], [Ts[i]])[0] for i in range(16)]
    assert flags[0]
    # only multiples of the ratio can produce a depth map
    for i, f in enumerate(flags[1:], start=2):
        if i % 3 != 0:
            assert not f
    with pytest.raises(_lib.QmError):
        BatchDepthmap([_stream_kw(W=100)], params=Params())


@pytest.mark.parametrize("iters", [(1, 0, 3, 2), (2, 1, 0, 5)])
def test_short_bp_iterations_match_oracle(oracle_mod, gpu, iters):
    """Levels with fewer than two half-sweeps take the separate
    message-inheritance pass, levels with two or more let their first two
    half-sweeps write the inherited messages: with counts of 0, 1, 2, 3 and
    5 across the levels the batched pipeline's node depths (the debug map)
    stay bit-exact with the oracle in IEEE mode."""
    from open_quadtree_mapping_b200.depthmap import Depthmap
    n_frames = 15
    imgs, Ts, _ = sequence(2, n_frames, W, H)
    p = Params(arith=ARITH_IEEE, bp_iters=iters)
    dm = Depthmap(W, H, F_PX, W / 2.0, F_PX, H / 2.0, semi2dense_ratio=1, params=p)
    pol = PolicyReplay(num_slots=5)
    cam = (F_PX, F_PX, W / 2.0, H / 2.0)
    n_dense = 0
    for i in range(n_frames):
        has = dm.add_frames(imgs[i], Ts[i])
        r = pol.add(i, Ts[i])
        assert has == (r["outcome"] in ("first", "dense")), (i, r["outcome"])
        if r["outcome"] != "dense":
            continue
        n_dense += 1
        slots = [imgs[k] for k in r["slots"]]
        o = oracle_mod.extract_depth(imgs[i], slots, r["T_slots"], cam, p)
        assert np.array_equal(dm.getDebugmap(), o["sparse"]), i
    assert n_dense >= 3
