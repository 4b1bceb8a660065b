"""Launch-shape autotuner of the batched engine (qm_batch_set_autotune /
qm_batch_set_tune / qm_batch_get_tune), through the C-ABI.

The BP half-sweep, extraction, row-solve and column-solve kernels take their
block shape at launch, the cost kernel its register budget (resident blocks
per SM); whatever shapes are chosen, every fused depth and debug map is
bit-identical."""
import numpy as np
import pytest

from conftest import sequence
from open_quadtree_mapping_b200.params import Params

pytestmark = pytest.mark.gpu

SHAPES = [(160, 128, 64, 5), (192, 144, 48, 3), (128, 96, 96, 7), (160, 120, 32, 2)]
FIXED = [
    dict(sweep_warps=4, extract_warps=16, row_warps=1, col_lines=8, cost_blocks=3),
    dict(sweep_warps=16, extract_warps=4, row_warps=4, col_lines=2, cost_blocks=4),
    dict(sweep_warps=8, extract_warps=8, row_warps=2, col_lines=4, cost_blocks=5),
]


def _descs():
    return [dict(width=w, height=h, fx=460.0 * w / 752.0, fy=460.0 * w / 752.0, cx=w / 2.0,
                 cy=h / 2.0, num_hyp=d, num_slots=f) for (w, h, d, f) in SHAPES]


def test_results_do_not_depend_on_launch_shapes(gpu):
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    seqs = [sequence(20 + k, 13, w, h) for k, (w, h, _, _) in enumerate(SHAPES)]
    p = Params.for_range(64, 0.5, 50.0)
    tuned = BatchDepthmap(_descs(), params=p)  # autotune is the default
    fixed = []
    for t in FIXED:
        b = BatchDepthmap(_descs(), params=p)
        b.set_tune(**t)
        fixed.append(b)
    eager = BatchDepthmap(_descs(), params=p)
    eager.set_graphs(False)
    eager.set_tune(**FIXED[0])
    for i in range(13):
        imgs = [s[0][i] for s in seqs]
        poses = [s[1][i] for s in seqs]
        h = tuned.add_frames(imgs, poses)
        for b in fixed + [eager]:
            assert b.add_frames(imgs, poses) == h
        if all(h) and i > 0:
            for k in range(len(SHAPES)):
                want = tuned.get_depth(k)
                for b in fixed + [eager]:
                    assert np.array_equal(b.get_depth(k), want)
                    assert np.array_equal(b.get_debug(k), tuned.get_debug(k))
    t = tuned.get_tune()
    assert t["sweep_warps"] in (4, 8, 16) and t["extract_warps"] in (4, 8, 16)
    assert t["row_warps"] in (1, 2, 4) and t["col_lines"] in (2, 4, 8)
    assert t["cost_blocks"] in (3, 4, 5)
    for b, want in zip(fixed, FIXED):
        assert b.get_tune() == want
    # switching back to autotune re-plans and still gives the same maps
    fixed[0].set_autotune(True)
    fixed[0].run_resident()
    tuned.run_resident()
    for k in range(len(SHAPES)):
        assert np.array_equal(fixed[0].get_depth(k), tuned.get_depth(k))


def test_invalid_launch_shapes_are_rejected(gpu):
    from open_quadtree_mapping_b200 import _lib
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    b = BatchDepthmap(_descs()[:1], params=Params.for_range(64, 0.5, 50.0))
    for bad in (dict(sweep_warps=5), dict(extract_warps=32), dict(row_warps=3),
                dict(col_lines=16), dict(cost_blocks=6), dict(cost_blocks=2)):
        with pytest.raises(_lib.QmError):
            b.set_tune(**bad)
    # lines of 4096 samples (the longest rows): at 13 bytes of shared memory
    # per sample even four rows per block fit a block's 227 KB
    wide = BatchDepthmap([dict(width=4096, height=64, fx=2000.0, fy=2000.0, cx=2048.0, cy=32.0,
                               num_hyp=32, num_slots=1)], params=Params.for_range(32, 0.5, 50.0))
    wide.set_tune(row_warps=4)
    wide.set_tune(row_warps=2)
    # a cost budget of 0 (a qm_tune filled with the four block shapes only)
    # selects the default instead of being rejected
    wide.set_tune(cost_blocks=0)
