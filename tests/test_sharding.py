"""Multi-process (gloo, CPU) checks of the stream sharding used for N GPUs:
every rank computes the same placement, the placement covers every stream
once and balances bytes, and the max-over-ranks reduction bench.py uses
returns the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from open_quadtree_mapping_b200.sharding import assign_streams, map_bytes


def test_assign_streams_balanced():
    descs = [(640, 480, 64)] * 6 + [(752, 480, 64)] * 6 + [(1280, 720, 96)] * 4
    costs = [map_bytes(w, h, d) for (w, h, d) in descs]
    for world in (1, 2, 4, 8):
        parts = assign_streams(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(descs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-6
    # equal streams are dealt round-robin
    assert assign_streams([1.0] * 6, 3) == [[0, 3], [1, 4], [2, 5]]


def test_map_bytes_cfg1():
    # about 300 MB per 752x480x64 map, dominated by the BP half-sweeps
    b = map_bytes(752, 480, 64)
    assert 2.5e8 < b < 3.5e8


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _FakeBatch:
    """Stands in for BatchDepthmap: records its streams and answers flags."""

    def __init__(self, descs, params=None, device=0):
        self.descs = descs

    def add_frames(self, imgs, poses):
        assert len(imgs) == len(poses) == len(self.descs)
        return [img["stream"] % 2 == 0 for img in imgs]

    def submit(self, imgs, poses, outs=None):
        return self.add_frames(imgs, poses)

    def close(self):
        pass


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from open_quadtree_mapping_b200.sharding import assign_streams, map_bytes, max_over_ranks
    costs = [map_bytes(752, 480, 64)] * 5 + [map_bytes(1280, 720, 64)] * 3
    mine = assign_streams(costs, world)[rank]
    slowest = max_over_ranks(10.0 + rank)
    # the sharded driver over the uneven 16-stream layout: this rank's batch
    # gets its placed streams' descriptors, and frames fed as global lists
    # reach the right streams
    from open_quadtree_mapping_b200.sharding import ShardedBatch
    descs = ([dict(width=640, height=480, num_hyp=48, num_slots=3)] * 6 +
             [dict(width=752, height=480, num_hyp=64, num_slots=5)] * 6 +
             [dict(width=1280, height=720, num_hyp=96, num_slots=10)] * 4)
    sb = ShardedBatch(descs, rank, world, batch_factory=_FakeBatch)
    frames = [{"stream": i} for i in range(16)]
    flags = sb.add_frames(frames, [None] * 16)
    sub = sb.submit(frames, [None] * 16)
    assert [d for d in sb.batch.descs] == [descs[i] for i in sb.mine]
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, slowest, sb.mine, flags, sub))


def test_two_rank_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts = [r[1] for r in res]
    assert sorted(parts[0] + parts[1]) == list(range(8))
    assert not set(parts[0]) & set(parts[1])
    assert all(r[2] == 11.0 for r in res)
    sharded = [r[3] for r in res]
    assert sorted(sharded[0] + sharded[1]) == list(range(16))
    for r in res:
        assert r[4] == {i: i % 2 == 0 for i in r[3]} == r[5]
