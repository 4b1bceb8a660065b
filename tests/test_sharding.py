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


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from open_quadtree_mapping_b200.sharding import assign_streams, map_bytes, max_over_ranks
    costs = [map_bytes(752, 480, 64)] * 5 + [map_bytes(1280, 720, 64)] * 3
    mine = assign_streams(costs, world)[rank]
    slowest = max_over_ranks(10.0 + rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, slowest))


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
