#!/usr/bin/env python
"""Depth-maps/s of the per-keyframe depth pipeline on B200.

Workload (the reference's plain configuration): 752x480 u8 keyframes,
pinhole fx=fy=460, c=(376, 240), 64 inverse-depth hypotheses uniform in
[1/50, 1/0.5] m^-1, 5 measurement slots (the reference's launch,
seed_matrix.cu:505, slot f reads ring frame floor(0.9 f)), seeded synthetic
ray-cast room scenes.  A step is one dense-pipeline pass (quadtree, cost
volume, hierarchical BP, extraction, upsampling, fusion) over S camera
streams, i.e. S depth maps; value = S * n_gpus / step time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--streams S]
    python bench.py --impl reference ...   # the CPU restatement (oracle port)

Multi-GPU: one process per GPU (torchrun); every rank owns S streams of its
own (weak scaling), no collective on the data path; the step time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H = 752, 480
FX = FY = 460.0
CX, CY = 376.0, 240.0
D = 64
SLOTS = 5
MIN_DEPTH, MAX_DEPTH = 0.5, 50.0
WARM_FRAMES = 13       # frame 13 is the first with more than 10 ring frames
CYCLE_FRAMES = 8       # frames fed round-robin in the end-to-end steps
METRIC = "depth-maps/s @752x480x64 hyp batched vs plain, 1 B200, same error; HBM % peak"
WORKLOAD = ("752x480 u8 keyframes, 64 inverse-depth hypotheses in [1/50, 1/0.5] m^-1, "
            "5 measurement slots, fx=fy=460, synthetic ray-cast room (seeded)")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.skip = 0

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "25"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def wait_first_sample(self, timeout=3.0):
        """Blocks until the sampler has written a line (nvidia-smi start-up
        takes a moment), so that the timed region that follows is sampled."""
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < timeout:
            try:
                if os.path.getsize(self.path) > 0:
                    return
            except OSError:
                pass
            time.sleep(0.02)

    def mark(self):
        """Samples written before this call are left out of the summary."""
        try:
            with open(self.path) as f:
                self.skip = sum(1 for _ in f)
        except Exception:
            self.skip = 0

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            lines = open(self.path).readlines()
            # the samples of the timed region (and the last one before it, so
            # that a short region still has one)
            for line in lines[max(0, self.skip - 1):]:
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def render_streams(n_distinct, seed_base):
    from open_quadtree_mapping_b200 import synthetic as syn
    seqs = []
    for k in range(n_distinct):
        imgs, Ts, _ = syn.make_sequence(seed_base + k, WARM_FRAMES + CYCLE_FRAMES, W=W, H=H,
                                        fx=FX, fy=FY, cx=CX, cy=CY)
        seqs.append((imgs, Ts))
    return seqs


def bp_updated_cells(levels, params):
    """Cells each BP half-sweep updates, per level and colour (the quadtree
    skip of bpextract.cu:214-220 removes the rest)."""
    out = []
    w, h = W // 4, H // 4
    for l in range(params.bp_levels):
        hw = (w + 1) // 2
        bx = np.arange(hw)[None, :]
        y = np.arange(h)[:, None]
        ilev = l + 2
        if ilev <= params.qt_max_level:
            size = 1 << ilev
            sx = np.minimum(bx * size, W - 1)
            sy = np.minimum(y * size, H - 1)
            keep = levels[sy, sx] <= ilev
        else:
            keep = np.ones((h, hw), bool)
        counts = []
        for parity in (0, 1):
            x = 2 * bx + ((y + parity) & 1)
            counts.append(int((keep & (x < w)).sum()))
        out.append((w, h, counts))
        w, h = (w + 1) // 2, (h + 1) // 2
    return out


def algorithmic_bytes(levels_list, params):
    """Algorithmic bytes per kernel kind for one step (all streams): every
    kernel reads its logical inputs once and writes its outputs once (images
    u8, costs/messages/depth f32, seeds 16 B)."""
    P = W * H
    C = (W // 4) * (H // 4)
    by = {k: 0.0 for k in ("quadtree", "cost", "pyramid", "msg_init", "bp_sweep", "extract",
                           "row_solve", "col_solve", "fuse_transform", "fuse_fill",
                           "fuse_update")}
    for lv in levels_list:
        cells = bp_updated_cells(lv, params)
        # levels written, the debug depth cleared
        by["quadtree"] += P * (1 + 4) + P
        by["cost"] += P * (1 + SLOTS) + C + 4 * C * D
        sizes = [(w * h) for (w, h, _) in cells]
        for l in range(1, params.bp_levels):
            by["pyramid"] += 4 * D * (sizes[l - 1] + sizes[l])
        # message inheritance writes the four messages of the cells the
        # quadtree test skips (copied from the parent level, zeros at the
        # top); at a level with two or more half-sweeps the first two sweeps
        # write them, otherwise a separate pass does
        for l, (w, h, counts) in enumerate(cells):
            skipped = w * h - counts[0] - counts[1]
            kind = "bp_sweep" if params.bp_iters[l] >= 2 else "msg_init"
            by[kind] += 16 * D * skipped * (2 if l + 1 < params.bp_levels else 1)
        for l, (w, h, counts) in enumerate(cells):
            it = params.bp_iters[l]
            n = sum(counts[i & 1] for i in range(it))
            by["bp_sweep"] += 36 * D * n
        by["extract"] += C * (20 * D + 4)
        # both solves derive the smoothness weights from the image in-kernel;
        # the row solve also resets the fusion keys
        by["row_solve"] += P * (4 + 1 + 8 + 8)
        by["col_solve"] += P * (8 + 1 + 4)
        by["fuse_transform"] += P * 32
        # hole filling runs inside the update: depth, key and source seed
        # read, depth and seed written
        by["fuse_update"] += P * (4 + 8 + 16 + 4 + 16)
    return by


def dram_traffic(kind, streams):
    """DRAM bytes (read + write) per launch of kernel kind `kind` from the
    committed ncu capture (profiles/: a few launches per BP level of the
    4-stream case of this workload), scaled by the stream count the bench
    runs.  (None, reason) if absent."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_bp_752x480x64_4streams.json")
    try:
        with open(path) as f:
            cap = json.load(f)
        per = cap["kernels"][kind]["dram_bytes_per_launch"]
    except Exception:
        return None, "no capture for this kernel"
    scale = streams / float(cap["streams"])
    src = "ncu capture, %d streams (profiles/%s)" % (cap["streams"], os.path.basename(path))
    if scale != 1.0:
        src += ", scaled by %d/%d streams" % (streams, cap["streams"])
    return int(per * scale), src


def cpu_baseline(kf_imgs, kf_Ts, budget_s=12.0):
    """The oracle (C++ restatement of the reference kernels) on the host cores:
    extract + fuse of full 752x480 keyframes, as many as fit in budget_s."""
    from oracle import oracle
    from open_quadtree_mapping_b200.params import Params
    from oracle.policy import PolicyReplay
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    p = Params.for_range(D, MIN_DEPTH, MAX_DEPTH)
    pol = PolicyReplay(num_slots=SLOTS)
    jobs = []
    for i in range(len(kf_imgs)):
        r = pol.add(i, kf_Ts[i])
        if r["outcome"] == "dense":
            jobs.append((i, r))
    cam = (FX, FY, CX, CY)
    seeds = np.zeros((H, W, 4), np.float32)
    done = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < budget_s or done < 2:
        i, r = jobs[done % len(jobs)]
        o = oracle.extract_depth(kf_imgs[i], [kf_imgs[k] for k in r["slots"]], r["T_slots"],
                                 cam, p)
        _, seeds, _, _ = oracle.fuse(o["dense"], seeds.astype(np.float32), r["T_fuse"], cam)
        done += 1
        if done >= 200:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "depth-maps/s", "cores": threads, "kind": "port",
            "sample": "%d keyframes of the same workload (752x480, D=64, 5 slots), extract + "
                      "fusion, oracle fp32 C++ port on %d host threads, %.1f s" % (done, threads, dt)}


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    seqs = render_streams(1, 7000)
    imgs, Ts = seqs[0]
    log("reference arm: oracle port on host cores")
    # warmup steps, then K timed steps; each step is a bounded sample of the
    # workload (one full keyframe extract + fusion on all host threads)
    from oracle import oracle
    from open_quadtree_mapping_b200.params import Params
    from oracle.policy import PolicyReplay
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    p = Params.for_range(D, MIN_DEPTH, MAX_DEPTH)
    pol = PolicyReplay(num_slots=SLOTS)
    jobs = [(i, r) for i in range(len(imgs)) for r in [pol.add(i, Ts[i])] if r["outcome"] == "dense"]
    cam = (FX, FY, CX, CY)
    seeds = np.zeros((H, W, 4), np.float32)

    def step(k):
        nonlocal seeds
        i, r = jobs[k % len(jobs)]
        o = oracle.extract_depth(imgs[i], [imgs[q] for q in r["slots"]], r["T_slots"], cam, p)
        _, s, _, _ = oracle.fuse(o["dense"], seeds, r["T_fuse"], cam)
        seeds = s.astype(np.float32)

    for k in range(args.warmup):
        step(k)
    t0 = time.perf_counter()
    for k in range(args.steps):
        step(k)
    dt = time.perf_counter() - t0
    value = args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "depth-maps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "maps_per_step": 1},
            "cpu_baseline": {"value": value, "unit": "depth-maps/s", "cores": threads,
                             "kind": "port",
                             "sample": "one 752x480 keyframe (extract + fusion) per step on "
                                       "%d host threads; the reference's path is CUDA-only, "
                                       "so its CPU implementation is the oracle's C++ port"
                                       % threads},
            "e2e": {"value": value, "unit": "depth-maps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_cuda_time(imgs, Ts):
    """The reference's own CUDA kernels (oracle/_ref) on this GPU, per keyframe,
    with its per-frame allocations and synchronisations."""
    try:
        from oracle import refbuild
        if not refbuild.available():
            return None
        from oracle.policy import PolicyReplay, se3_inv, se3_mul
        # the ring the reference's extract_depth sees at the first dense frame
        pol = PolicyReplay(num_slots=SLOTS)
        i = WARM_FRAMES - 1
        for k in range(i):
            pol.add(k, Ts[k])
        ring = [fid for fid, _ in pol.ring]
        if len(ring) <= 10:
            return None
        inv = se3_inv(Ts[i])
        T_ring = np.stack([se3_mul(Ts[k], inv) for k in ring])
        ms = refbuild.time_frames(imgs[i], imgs[ring], T_ring, (FX, FY, CX, CY), nslots=SLOTS,
                                  warmup=3, iters=10)
        return {"value": 1000.0 / ms, "unit": "depth-maps/s", "ms_per_map": ms,
                "what": "the reference's CUDA kernels built from its sources for sm_100a "
                        "(-O3 -use_fast_math), extract_depth + fuse_output_depth with its "
                        "allocations and syncs, one keyframe at a time"}
    except Exception as e:  # informational only
        log("reference CUDA timing failed:", e)
        return None


def accuracy_vs_fp64(imgs, Ts, params):
    """The error the throughput is measured at: one keyframe of the workload
    (the first dense frame of stream 0) through the library's stage calls in
    the benchmarked arithmetic, against the FP64 oracle on the same inputs:
    relative error of the upsampled depth (p50 / p99 over valid pixels) and
    the share of node cells whose BP label differs."""
    import torch
    from oracle import oracle
    from oracle.policy import PolicyReplay
    from open_quadtree_mapping_b200 import stages
    pol = PolicyReplay(num_slots=SLOTS)
    r = None
    for i in range(WARM_FRAMES):
        r = pol.add(i, Ts[i])
    if r is None or r["outcome"] != "dense":
        return None
    i = WARM_FRAMES - 1
    cam = (FX, FY, CX, CY)
    slots = [imgs[k] for k in r["slots"]]
    dev = torch.device("cuda")
    g = stages.extract_depth(torch.from_numpy(np.ascontiguousarray(imgs[i])).to(dev),
                             [torch.from_numpy(np.ascontiguousarray(m)).to(dev) for m in slots],
                             r["T_slots"], cam, params)
    oracle.set_threads(os.cpu_count() or 1)
    o = oracle.extract_depth(imgs[i], slots, r["T_slots"], cam, params, dtype=np.float64)
    dense, ref = g["dense"].cpu().numpy(), o["dense"]
    ok = np.isfinite(ref) & (ref > 0) & np.isfinite(dense)
    rel = np.abs(dense[ok] - ref[ok]) / ref[ok]
    lab_g, lab_o = g["labels"].cpu().numpy(), o["labels"]
    node = lab_o >= 0
    return {"dense_rel_err_p50": float(np.percentile(rel, 50)),
            "dense_rel_err_p99": float(np.percentile(rel, 99)),
            "label_mismatch_frac": float((lab_g[node] != lab_o[node]).mean()),
            "what": "stream 0's first dense keyframe, library stage calls (the benchmarked "
                    "arithmetic) vs the FP64 oracle on the same inputs"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--streams", type=int, default=32, help="camera streams per GPU")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--distinct", type=int, default=2, help="distinct rendered sequences")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

    import torch
    from open_quadtree_mapping_b200 import build_ext
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    from open_quadtree_mapping_b200.params import Params
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    if rank == 0 and not build_ext.up_to_date():
        build_ext.build()
    if pg:
        pg.barrier()

    S = args.streams
    params = Params.for_range(D, MIN_DEPTH, MAX_DEPTH)
    t0 = time.time()
    seqs = render_streams(args.distinct, 3000)
    log("rank %d: rendered %d sequences in %.1f s" % (rank, len(seqs), time.time() - t0))
    desc = dict(width=W, height=H, fx=FX, fy=FY, cx=CX, cy=CY, num_hyp=D, num_slots=SLOTS)
    # S * world global streams placed over the ranks by estimated bytes (equal
    # streams: round-robin, S per rank); global stream g replays sequence
    # g % distinct
    from open_quadtree_mapping_b200.sharding import ShardedBatch
    shard = ShardedBatch([desc] * (S * world), rank, world, params=params, device=local)
    batch = shard.batch
    seq_of = [g % len(seqs) for g in shard.mine]
    assert len(seq_of) == S
    # pinned host frames, one per (distinct sequence, frame)
    pinned = {}
    for k, (imgs, _) in enumerate(seqs):
        for i in range(len(imgs)):
            t = torch.empty((H, W), dtype=torch.uint8, pin_memory=True)
            t.numpy()[:] = imgs[i]
            pinned[(k, i)] = t
    # two sets of pinned depth outputs: the pipelined API keeps two steps in
    # flight, step j downloading into set j % 2
    out_pinned = [[torch.empty((H, W), dtype=torch.float32, pin_memory=True) for _ in range(S)]
                  for _ in range(2)]

    def feed(i):
        imgs = [pinned[(seq_of[s], i)].numpy() for s in range(S)]
        poses = [seqs[seq_of[s]][1][i] for s in range(S)]
        return batch.add_frames(imgs, poses)

    for i in range(WARM_FRAMES):
        has = feed(i)
    assert all(has), "every stream must produce a depth map after %d frames" % WARM_FRAMES
    launches_per_step = batch.last_launches()
    tune = batch.get_tune()  # launch shapes the autotuner chose on the first dense frame
    ext = torch.cuda.ExternalStream(batch.stream_ptr())

    # ---- device-resident batched steps (value)
    for _ in range(args.warmup):
        batch.run_resident()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        clk.wait_first_sample()
        clk.mark()
        e0.record(ext)
        for _ in range(args.steps):
            batch.run_resident()
        e1.record(ext)
        e1.synchronize()
    torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / args.steps
    clocks = clk.summary()

    # ---- end-to-end: host frames in, host depth out, through the C-ABI
    # (qm_batch_submit: every step uploads its S frames from pinned memory
    # and downloads its S fused depth maps into pinned memory; the uploads
    # and downloads overlap the neighbouring steps' pipelines; the timed
    # region ends when the last download has landed)
    out_np = [[t.numpy() for t in ts] for ts in out_pinned]

    def e2e_step(j):
        i = WARM_FRAMES + (j % CYCLE_FRAMES)
        imgs = [pinned[(seq_of[s], i)].numpy() for s in range(S)]
        poses = [seqs[seq_of[s]][1][i] for s in range(S)]
        has = batch.submit(imgs, poses, outs=out_np[j % 2])
        # every step must yield S depth maps: a frame the policy skipped
        # would download nothing and inflate the rate
        assert all(has), "e2e step %d: a stream produced no depth map" % j

    for j in range(args.warmup):
        e2e_step(j)
    batch.wait()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for j in range(args.steps):
        e2e_step(j)
    batch.wait()
    torch.cuda.synchronize()
    e2e_ms = 1000.0 * (time.perf_counter() - t1) / args.steps

    # ---- max over ranks
    if pg:
        t = torch.tensor([ms_step, e2e_ms], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_step, e2e_ms = float(t[0]), float(t[1])

    # ---- per-kernel profile (eager launches with events) for the roofline
    prof = batch.profile()
    # the quadtree levels of the profiled frames (for the cells the BP
    # actually updates), from the library's own quadtree kernel
    from open_quadtree_mapping_b200 import stages
    lv_by_seq = {k: stages.quadtree(torch.from_numpy(np.ascontiguousarray(
        seqs[k][0][WARM_FRAMES - 1])).cuda(), params).cpu().numpy() for k in range(len(seqs))}
    levels_list = [lv_by_seq[seq_of[s]] for s in range(S)]
    alg = algorithmic_bytes(levels_list, params)
    peak, peak_kind = measured_hbm_peak()
    kinds = {}
    for k, (ms, n) in prof.items():
        gbs = alg[k] / (ms * 1e-3) / 1e9 if ms > 0 else None
        kinds[k] = {"ms": round(ms, 4), "launches": n, "alg_MB": round(alg[k] / 1e6, 2),
                    "GBs": round(gbs, 1) if gbs else None}
    dom = max(prof, key=lambda k: prof[k][0])
    dms, dn = prof[dom]
    achieved = alg[dom] / (dms * 1e-3) / 1e9
    traffic, traffic_src = dram_traffic(dom, S)
    # the whole pipeline against the same peak: every kernel's algorithmic
    # bytes per step over the device-timed step, and the rate the step would
    # reach if it moved those bytes at the peak
    alg_step = sum(alg.values())
    pipeline = {"alg_GB_per_step": round(alg_step / 1e9, 4),
                "achieved_GBs": round(alg_step / (ms_step * 1e-3) / 1e9, 1),
                "frac": round(alg_step / (ms_step * 1e-3) / 1e9 / peak, 4),
                "hbm_ceiling_maps_per_s": round(S / (alg_step / (peak * 1e9)), 1),
                "what": "all kernels' algorithmic bytes per step / ms_per_step, of the "
                        "measured copy peak; the ceiling is the rate at that peak"}
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "traffic_source": traffic_src, "peak_source": peak_kind,
                "per_launch_alg_bytes": alg[dom] / max(dn, 1),
                "avg_launch_ms": dms / max(dn, 1),
                "timing": "CUDA events around every launch of one eager run on the "
                          "library's stream, right after the timed region"}

    # ---- plain per-frame path: one stream, launched stage by stage
    plain = BatchDepthmap([desc], params=params, device=local)
    plain.set_graphs(False)
    for i in range(WARM_FRAMES):
        plain.add_frames([seqs[0][0][i]], [seqs[0][1][i]])
    pext = torch.cuda.ExternalStream(plain.stream_ptr())
    for _ in range(args.warmup):
        plain.run_resident()
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(pext)
    for _ in range(args.steps):
        plain.run_resident()
    p1.record(pext)
    p1.synchronize()
    plain_ms = p0.elapsed_time(p1) / args.steps
    plain.close()

    if rank != 0:
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    # ---- the baseline leg (rank 0 at N=1 only): the CPU port of the
    # reference on the host cores, the reference's own kernels on this GPU,
    # and the error this run's arithmetic is measured at against the FP64
    # oracle
    cpu = ref_cuda = accuracy = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_baseline(seqs[0][0], seqs[0][1])
        ref_cuda = reference_cuda_time(seqs[0][0], seqs[0][1])
        try:
            accuracy = accuracy_vs_fp64(seqs[0][0], seqs[0][1], params)
        except Exception as e:  # informational only
            log("accuracy check failed:", e)

    value = S * world / (ms_step * 1e-3)
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "depth-maps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "streams_per_gpu": S, "global_batch": S * world,
                   "maps_per_step": S * world,
                   "parallelism": "streams placed per GPU by estimated bytes (sharding.ShardedBatch)",
                   "launch_shapes": tune,
                   "l2": "inputs larger than L2: per-GPU working set %.1f GB per step"
                         % (S * 0.08)},
        "e2e": {"value": round(S * world / (e2e_ms * 1e-3), 2), "unit": "depth-maps/s",
                "h2d_bytes_per_step": S * (W * H + 48),
                "d2h_bytes_per_step": S * W * H * 4, "ms_per_step": round(e2e_ms, 3)},
        "plain": {"value": round(1.0 / (plain_ms * 1e-3), 2), "unit": "depth-maps/s",
                  "ms_per_map": round(plain_ms, 4),
                  "what": "one stream, stage-by-stage launches, no graph"},
        "batched_vs_plain": round(value / world / (1.0 / (plain_ms * 1e-3)), 2),
        "roofline": roofline, "pipeline_frac": pipeline["frac"], "pipeline": pipeline,
        "kernels": kinds,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "reference_cuda_kernels": ref_cuda,
        "accuracy": accuracy,
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
