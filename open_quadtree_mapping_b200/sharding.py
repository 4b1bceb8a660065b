"""Multi-GPU placement of camera streams.

Streams (and their keyframes) share no state, so the path shards by stream:
one process per GPU, each owning a disjoint set of streams, with no
collective on the data path.  Streams are placed greedily by their estimated
bytes per depth map (largest first onto the least-loaded GPU), which is
round-robin for equal streams.  The only collective is the max over ranks of
a measured time (bench.py) or an optional metrics gather.
"""
from __future__ import annotations


def map_bytes(width: int, height: int, num_hyp: int = 64, num_slots: int = 5,
              bp_levels: int = 4, bp_iters=(4, 10, 10, 10)) -> float:
    """Algorithmic bytes of one depth map (every stage reads its inputs and
    writes its outputs once; BP counts 9*D*4 bytes per cell per half-sweep
    over half of each level's cells)."""
    P = width * height
    D = num_hyp
    w, h = width // 4, height // 4
    sizes = []
    for _ in range(bp_levels):
        sizes.append((w, h))
        w, h = (w + 1) // 2, (h + 1) // 2
    C = sizes[0][0] * sizes[0][1]
    b = 2 * P + P * (1 + num_slots) + C + 4 * C * D
    for l in range(1, bp_levels):
        b += 4 * D * (sizes[l - 1][0] * sizes[l - 1][1] + sizes[l][0] * sizes[l][1])
    b += 16 * D * sizes[-1][0] * sizes[-1][1]
    for l in range(bp_levels - 1):
        b += 16 * D * (sizes[l + 1][0] * sizes[l + 1][1] + sizes[l][0] * sizes[l][1])
    for l, (sw, sh) in enumerate(sizes):
        b += bp_iters[l] * ((sw + 1) // 2) * sh * 36 * D
    b += C * (20 * D + 4) + 25 * P + 52 * P
    return float(b)


def assign_streams(costs, world: int):
    """Greedy placement: returns `world` lists of stream indices."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value: float, group=None) -> float:
    """Max of a per-rank scalar over the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
