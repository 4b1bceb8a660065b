"""Throughput and latency of the depth pipeline on the other measured workloads.

    python -m open_quadtree_mapping_b200.workloads [--only NAME ...] [--steps K]

Prints one JSON line per workload (seeded synthetic ray-cast scenes):

* video720: one 1280x720 stream (fx=fy=780), 64 hypotheses, 10 measurement
  slots, 30 frames through the Depthmap facade with fusion; per-frame
  latency through the C-ABI (host frame in, fused depth out) p50/p99 over the
  frames that produce a map, and the device time of one dense frame.
* uneven16: 16 streams in one batch (6 x 640x480, 6 x 752x480, 4 x 1280x720)
  with 3-10 slots and 48/64/96 hypotheses per stream: maps/s of the resident
  batched pipeline and end to end (pinned host frames in, depth maps out).
* large1080: 8 streams of 1920x1080 (fx=fy=1150), 128 hypotheses, 20 slots,
  5-level quadtree: maps/s, p50/p99 of the batch-step latency, end to end.
* diff8: 8 keyframes of 752x480 through the differentiable pipeline (soft
  readout tau=0.05, weighted upsampling, fusion, L1 loss): forward +
  backward per batch.
* semidense32: 32 streams of 752x480 end to end with and without the
  semi-dense tracker (its cost per stream and frame).

Per-step latencies flush the L2 (a 256 MiB write) before every timed step;
back-to-back throughput runs use working sets larger than the L2.

Under torchrun (`python -m torch.distributed.run --nproc-per-node N -m
open_quadtree_mapping_b200.workloads --only uneven16 large1080`) the batch
workloads place their streams over the N GPUs (sharding.ShardedBatch) and
report the max over ranks of the step times.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import time

import numpy as np


def render_sequences(specs, n_frames, procs=8):
    """specs: [(seq_id, W, H, f)].  Returns {seq_id: (imgs, T_curr_world)}
    with frames rendered in a spawn pool (call before any CUDA work)."""
    from . import synthetic as syn
    jobs, meta = [], []
    for sid, W, H, f in specs:
        traj = syn.make_trajectory(2000 + sid, n_frames)
        for i in range(n_frames):
            jobs.append((1000 + sid, traj[i], W, H, f))
        meta.append((sid, traj))
    with mp.get_context("spawn").Pool(procs) as pool:
        imgs = pool.map(syn.render_frame, jobs)
    out = {}
    for k, (sid, traj) in enumerate(meta):
        frames = imgs[k * n_frames:(k + 1) * n_frames]
        poses = [np.ascontiguousarray(syn.inv_se3(traj[i])[:3, :4], np.float32).reshape(12)
                 for i in range(n_frames)]
        out[sid] = (frames, poses)
    return out


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs), q)) if xs else None


class _Timer:
    def __init__(self, torch, stream_ptr):
        self.torch = torch
        self.ext = torch.cuda.ExternalStream(stream_ptr)
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step_ms(self, fn, flush=True):
        t = self.torch
        if flush:
            self.flush.fill_(1)
        t.cuda.synchronize()
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        e0.record(self.ext)
        fn()
        e1.record(self.ext)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def run_ms(self, fn, steps):
        t = self.torch
        t.cuda.synchronize()
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        e0.record(self.ext)
        for _ in range(steps):
            fn()
        e1.record(self.ext)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps


def _dist():
    """(world, rank, local rank) from the torchrun environment; with more
    than one process the NCCL group is set up (one process per GPU)."""
    import os
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        if not dist.is_initialized():
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def _batch_workload(name, descs, seqs, layout, params, steps, warm_frames, extra):
    """One batch workload.  Under torchrun the streams are placed over the
    ranks (sharding.ShardedBatch, no data crosses ranks) and the step times
    are the max over ranks; maps/s counts every rank's streams."""
    import torch

    from .sharding import ShardedBatch, max_over_ranks
    world, rank, local = _dist()
    S = len(descs)
    shard = ShardedBatch(descs, rank, world, params=params, device=local)
    batch = shard.batch
    layout = [layout[i] for i in shard.mine]
    pinned = {}
    for k, sid in enumerate(layout):
        for i, img in enumerate(seqs[sid][0]):
            key = (sid, i)
            if key not in pinned:
                t = torch.empty(img.shape, dtype=torch.uint8, pin_memory=True)
                t.numpy()[:] = img
                pinned[key] = t.numpy()

    def frame(i):
        return ([pinned[(sid, i)] for sid in layout], [seqs[sid][1][i] for sid in layout])

    for i in range(warm_frames):
        has = batch.add_frames(*frame(i))
    assert all(has), "every stream must have produced a depth map"
    tm = _Timer(torch, batch.stream_ptr())
    for _ in range(3):
        batch.run_resident()
    ms = tm.run_ms(batch.run_resident, steps)
    lat = [tm.step_ms(batch.run_resident) for _ in range(steps)]
    # end to end: pinned frames in, fused depth maps out (pipelined submit)
    outs = [[torch.empty(seqs[sid][0][0].shape, dtype=torch.float32,
                         pin_memory=True).numpy() for sid in layout] for _ in range(2)]
    n_frames = len(seqs[layout[0]][0])
    cyc = list(range(warm_frames, n_frames)) or [n_frames - 1]
    for j in range(3):
        batch.submit(*frame(cyc[j % len(cyc)]), outs=outs[j % 2])
    batch.wait()
    t0 = time.perf_counter()
    for j in range(steps):
        batch.submit(*frame(cyc[j % len(cyc)]), outs=outs[j % 2])
    batch.wait()
    e2e_ms = 1000.0 * (time.perf_counter() - t0) / steps
    prof = {k: round(v[0], 4) for k, v in batch.profile().items()}
    ms = max_over_ranks(ms)
    e2e_ms = max_over_ranks(e2e_ms)
    lat = [max_over_ranks(x) for x in lat]
    line = {"workload": name, "streams": S, "gpus": world,
            "maps_per_s": round(S / (ms * 1e-3), 2),
            "kernel_ms_eager": prof,
            "ms_per_step": round(ms, 4),
            "step_latency_ms": {"p50": round(_pct(lat, 50), 4), "p99": round(_pct(lat, 99), 4),
                                "l2": "flushed before every step"},
            "e2e_maps_per_s": round(S / (e2e_ms * 1e-3), 2), "e2e_ms_per_step": round(e2e_ms, 3),
            "launch_shapes": batch.get_tune(), "launches_per_step": batch.last_launches()}
    line.update(extra)
    batch.close()
    return line


def video720(steps):
    import torch

    from .depthmap import BatchDepthmap
    from .params import Params
    W, H, f = 1280, 720, 780.0
    seqs = render_sequences([(70, W, H, f)], 30)
    imgs, poses = seqs[70]
    p = Params.for_range(64, 0.5, 50.0)
    b = BatchDepthmap([dict(width=W, height=H, fx=f, fy=f, cx=W / 2.0, cy=H / 2.0,
                            num_hyp=64, num_slots=10)], params=p)
    lat = []
    depth = np.empty((H, W), np.float32)
    for i in range(30):
        t0 = time.perf_counter()
        has = b.add_frames([imgs[i]], [poses[i]])[0]
        if has:
            depth = b.get_depth(0)
            lat.append(1000.0 * (time.perf_counter() - t0))
    tm = _Timer(torch, b.stream_ptr())
    for _ in range(3):
        b.run_resident()
    dev = [tm.step_ms(b.run_resident) for _ in range(steps)]
    b.close()
    return {"workload": "video720", "streams": 1, "frames": 30, "dense_frames": len(lat),
            "frame_latency_ms_e2e": {"p50": round(_pct(lat, 50), 3),
                                     "p99": round(_pct(lat, 99), 3)},
            "device_ms_per_frame": {"p50": round(_pct(dev, 50), 4),
                                    "p99": round(_pct(dev, 99), 4),
                                    "l2": "flushed before every frame"},
            "valid_fused_fraction": round(float((depth > 0).mean()), 4),
            "config": "1280x720, fx=fy=780, 64 hyp, 10 slots, fusion on; latency = "
                      "add_frames + get_depth through the C-ABI per frame with a result"}


def uneven16(steps):
    from .params import Params
    sizes = {(640, 480): 460.0 * 640 / 752, (752, 480): 460.0, (1280, 720): 780.0}
    specs = [(80 + k, W, H, f) for k, ((W, H), f) in enumerate(sizes.items())]
    seqs = render_sequences(specs, 21)
    rng = np.random.default_rng(16)
    layout_sz = [(640, 480)] * 6 + [(752, 480)] * 6 + [(1280, 720)] * 4
    sid_of = {(W, H): sid for sid, W, H, _ in specs}
    layout = [sid_of[sz] for sz in layout_sz]
    descs = [dict(width=W, height=H, fx=sizes[(W, H)], fy=sizes[(W, H)], cx=W / 2.0,
                  cy=H / 2.0, num_hyp=int(rng.choice([48, 64, 96])),
                  num_slots=int(rng.integers(3, 11))) for (W, H) in layout_sz]
    return _batch_workload("uneven16", descs, seqs, layout, Params.for_range(64, 0.5, 50.0),
                           steps, 13, {"config": "6x640x480 + 6x752x480 + 4x1280x720, "
                                                 "48/64/96 hyp, 3-10 slots"})


def large1080(steps):
    from .params import Params
    W, H, f = 1920, 1080, 1150.0
    specs = [(90, W, H, f), (91, W, H, f)]
    seqs = render_sequences(specs, 24)
    layout = [90, 91] * 4
    descs = [dict(width=W, height=H, fx=f, fy=f, cx=W / 2.0, cy=H / 2.0, num_hyp=128,
                  num_slots=20)] * 8
    p = Params.for_range(128, 0.5, 50.0, qt_max_level=5)
    return _batch_workload("large1080", descs, seqs, layout, p, steps, 22,
                           {"config": "8x1920x1080, fx=fy=1150, 128 hyp, 20 slots, "
                                      "5-level quadtree (ring of 21 frames: 19 distinct "
                                      "slot frames)"})


def diff8(steps):
    import torch

    from . import diff
    from . import synthetic as syn
    from .params import Params
    W, H = 752, 480
    p = Params.for_range(64, 0.5, 50.0)
    rng = np.random.default_rng(3)
    kfs = []
    for s in range(8):
        kf = syn.make_keyframe(20 + s, W=W, H=H, fx=460.0, fy=460.0, F=5)
        gt = kf.gt_depth.astype(np.float32)
        seeds = np.zeros((H, W, 4), np.float32)
        seeds[..., 0], seeds[..., 1] = 30.0, 5.0
        seeds[..., 2] = gt * (1.0 + 0.05 * rng.standard_normal((H, W)))
        seeds[..., 3] = 4.0
        kfs.append(diff.Keyframe(
            ref=torch.from_numpy(kf.ref).cuda(),
            slots=[torch.from_numpy(np.ascontiguousarray(m)).cuda() for m in kf.meas],
            T_slot_ref=kf.T_meas_ref, cam=(kf.fx, kf.fy, kf.cx, kf.cy),
            seeds=torch.from_numpy(seeds).cuda(),
            T_fuse=np.eye(3, 4, dtype=np.float32).reshape(12),
            gt=torch.from_numpy(gt).cuda()).prepare(p))
    pen = torch.tensor([p.P1, p.P2], dtype=torch.float64, requires_grad=True)
    omegas = [torch.ones((H, W), dtype=torch.float32, device="cuda", requires_grad=True)
              for _ in kfs]

    def fwd_bwd():
        for om in omegas:
            om.grad = None
        pen.grad = None
        loss = diff.batch_loss(kfs, pen, omegas, p, 0.05)
        loss.backward()
        return loss

    for _ in range(2):
        fwd_bwd()
    torch.cuda.synchronize()
    t = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fwd_bwd()
        torch.cuda.synchronize()
        t.append(1000.0 * (time.perf_counter() - t0))
    return {"workload": "diff8", "keyframes": 8,
            "ms_per_batch_fwd_bwd": {"p50": round(_pct(t, 50), 3), "p99": round(_pct(t, 99), 3)},
            "keyframes_per_s": round(8 / (_pct(t, 50) * 1e-3), 2),
            "config": "8x752x480, 64 hyp, 5 slots, tau=0.05, gradients for P1, P2 and "
                      "per-pixel omega"}


def semidense32(steps):
    """32 streams of 752x480 (64 hypotheses, 5 slots) end to end through
    the pipelined API with and without the semi-dense tracker; every frame
    of every stream runs the tracker, so its cost per frame is the
    difference."""
    import torch

    from .depthmap import BatchDepthmap
    from .params import Params
    W, H, f = 752, 480, 460.0
    seqs = render_sequences([(60, W, H, f), (61, W, H, f)], 21)
    layout = [60, 61] * 16
    p = Params.for_range(64, 0.5, 50.0)
    desc = dict(width=W, height=H, fx=f, fy=f, cx=W / 2.0, cy=H / 2.0, num_hyp=64, num_slots=5)
    out = {}
    for on in (False, True):
        b = BatchDepthmap([desc] * 32, params=p)
        b.set_semidense(on)
        pinned = {}
        for sid in (60, 61):
            for i, img in enumerate(seqs[sid][0]):
                t = torch.empty(img.shape, dtype=torch.uint8, pin_memory=True)
                t.numpy()[:] = img
                pinned[(sid, i)] = t.numpy()
        outs = [[torch.empty((H, W), dtype=torch.float32, pin_memory=True).numpy()
                 for _ in layout] for _ in range(2)]

        def frame(i):
            return ([pinned[(sid, i)] for sid in layout], [seqs[sid][1][i] for sid in layout])

        for i in range(13):
            b.add_frames(*frame(i))
        for j in range(3):
            b.submit(*frame(13 + j % 8), outs=outs[j % 2])
        b.wait()
        t0 = time.perf_counter()
        for j in range(steps):
            b.submit(*frame(13 + j % 8), outs=outs[j % 2])
        b.wait()
        out["on" if on else "off"] = 1000.0 * (time.perf_counter() - t0) / steps
        b.close()
    return {"workload": "semidense32", "streams": 32,
            "e2e_ms_per_step": {"without_tracker": round(out["off"], 3),
                                "with_tracker": round(out["on"], 3)},
            "tracker_ms_per_stream_frame": round((out["on"] - out["off"]) / 32, 4),
            "config": "32x752x480, 64 hyp, 5 slots; every step = one frame of every stream"}


WORKLOADS = {"video720": video720, "uneven16": uneven16, "large1080": large1080,
             "diff8": diff8, "semidense32": semidense32}


SHARDED = ("uneven16", "large1080")


def main():
    """Under torchrun (one process per GPU) only the batch workloads run,
    their streams placed over the GPUs; rank 0 prints."""
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=list(WORKLOADS))
    ap.add_argument("--steps", type=int, default=20)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    for name in args.only:
        if world > 1 and name not in SHARDED:
            continue
        line = WORKLOADS[name](args.steps)
        if rank == 0:
            print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
