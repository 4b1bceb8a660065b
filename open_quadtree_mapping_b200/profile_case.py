"""A small, self-contained run of the batched pipeline for profiler captures.

    python -m open_quadtree_mapping_b200.profile_case --streams 4 --runs 3
    python -m open_quadtree_mapping_b200.profile_case --large --streams 2 --runs 1
    ncu --profile-from-start off ... python -m open_quadtree_mapping_b200.profile_case \
        --streams 4 --runs 1 --eager --profile-range   # only the timed run

Feeds S synthetic streams (default 752x480, 64 hypotheses, 5 slots; with
--large 1920x1080, fx=fy=1150, 128 hypotheses, 20 slots, 5-level quadtree)
until every stream produces a depth map, then replays the resident dense
pipeline R more times.  Sized so that a kernel-level capture (ncu -k ... -c
...) stays well under a few GB of device memory; prints the device time per
run.
"""
from __future__ import annotations

import argparse
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--runs", type=int, default=3)
    ap.add_argument("--eager", action="store_true", help="launch stage by stage, no graph")
    ap.add_argument("--large", action="store_true",
                    help="1920x1080, 128 hypotheses, 20 slots, 5-level quadtree")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the timed runs with cudaProfilerStart/Stop (for ncu "
                         "--profile-from-start off: only those runs' launches are captured)")
    args = ap.parse_args()

    import torch

    from . import synthetic
    from .depthmap import BatchDepthmap
    from .params import Params

    if args.large:
        W, H, F, D, slots, n_frames = 1920, 1080, 1150.0, 128, 20, 22
        params = Params.for_range(D, 0.5, 50.0, qt_max_level=5)
    else:
        W, H, F, D, slots, n_frames = 752, 480, 460.0, 64, 5, 13
        params = Params.for_range(D, 0.5, 50.0)
    imgs, Ts, _ = synthetic.make_sequence(4000, n_frames, W=W, H=H, fx=F, fy=F)
    desc = dict(width=W, height=H, fx=F, fy=F, cx=W / 2.0, cy=H / 2.0, num_hyp=D,
                num_slots=slots)
    b = BatchDepthmap([desc] * args.streams, params=params)
    if args.eager:
        b.set_graphs(False)
    for i in range(n_frames):
        has = b.add_frames([imgs[i]] * args.streams, [Ts[i]] * args.streams)
    assert all(has)
    ext = torch.cuda.ExternalStream(b.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if args.profile_range:
        torch.cuda.cudart().cudaProfilerStart()
    t0 = time.perf_counter()
    e0.record(ext)
    for _ in range(args.runs):
        b.run_resident()
    e1.record(ext)
    e1.synchronize()
    if args.profile_range:
        torch.cuda.cudart().cudaProfilerStop()
    print("streams=%d runs=%d device_ms_per_run=%.4f wall_ms_per_run=%.4f launches_per_run=%d"
          % (args.streams, args.runs, e0.elapsed_time(e1) / args.runs,
             1000.0 * (time.perf_counter() - t0) / args.runs, b.last_launches()))


if __name__ == "__main__":
    main()
