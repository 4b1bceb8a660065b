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


def desc_bytes(d: dict) -> float:
    """map_bytes of a stream descriptor (width, height, num_hyp, num_slots)."""
    return map_bytes(int(d["width"]), int(d["height"]), int(d.get("num_hyp") or 64),
                     int(d.get("num_slots") or 5))


class ShardedBatch:
    """This rank's share of a global list of camera streams.

    Every rank builds the same placement (assign_streams over the streams'
    estimated bytes), owns the streams placed on it as one batch on its own
    GPU, and is fed the global per-tick frame lists: add_frames / submit take
    one image and pose per GLOBAL stream and pass this rank's on.  Flags and
    depth maps are keyed by global stream index.  No data crosses ranks.

    batch_factory(descs, params=..., device=...) builds the per-rank batch
    (default: BatchDepthmap); tests pass a stand-in."""

    def __init__(self, descs, rank: int, world: int, params=None, device: int = 0,
                 batch_factory=None):
        if not 0 <= rank < world:
            raise ValueError("rank %d outside world %d" % (rank, world))
        self.n = len(descs)
        self.mine = assign_streams([desc_bytes(d) for d in descs], world)[rank]
        if batch_factory is None:
            from .depthmap import BatchDepthmap as batch_factory
        self.batch = (batch_factory([descs[i] for i in self.mine], params=params, device=device)
                      if self.mine else None)

    def _pick(self, xs):
        if len(xs) != self.n:
            raise ValueError("expected %d per-stream entries, got %d" % (self.n, len(xs)))
        return [xs[i] for i in self.mine]

    def add_frames(self, imgs, poses) -> dict:
        if self.batch is None:
            return {}
        return dict(zip(self.mine, self.batch.add_frames(self._pick(imgs), self._pick(poses))))

    def submit(self, imgs, poses, outs=None) -> dict:
        if self.batch is None:
            return {}
        has = self.batch.submit(self._pick(imgs), self._pick(poses),
                                outs=self._pick(outs) if outs is not None else None)
        return dict(zip(self.mine, has))

    def get_depth(self, i):
        return self.batch.get_depth(self.mine.index(i))

    def close(self):
        if self.batch is not None:
            self.batch.close()

