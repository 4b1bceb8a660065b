"""Point cloud of a fused depth map (Publisher::publishPointCloud,
publisher.cpp:129-166) on the GPU, through the C-ABI: bit-identical to the
oracle and to the golden cloud made with the reference's own host
arithmetic, point order included."""
import numpy as np
import pytest
import torch

from conftest import GOLDEN, sequence
from open_quadtree_mapping_b200.params import Params

pytestmark = pytest.mark.gpu


def _same(a, b):
    """Bit-identical, except that any NaN matches any NaN (the device writes
    its canonical NaN where the host propagates the input's payload)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and
                np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


def _gpu_cloud(depth, ref, cam, T, dev, pad=0):
    from open_quadtree_mapping_b200 import stages
    H, W = depth.shape
    d = torch.full((H, W + pad), -5.0, dtype=torch.float32, device=dev)[:, :W]
    d.copy_(torch.from_numpy(np.ascontiguousarray(depth)))
    r = torch.zeros((H, W + 3 * pad), dtype=torch.uint8, device=dev)[:, :W]
    r.copy_(torch.from_numpy(np.ascontiguousarray(ref)))
    return stages.point_cloud(d, r, cam, T).cpu().numpy()


def test_point_cloud_matches_golden(gpu):
    z = np.load(GOLDEN + "/ref_pointcloud_160x128.npz")
    cam = tuple(float(c) for c in z["cam"])
    for pad in (0, 7):
        pts = _gpu_cloud(z["depth"], z["ref"], cam, z["T_world_ref"], gpu, pad)
        assert _same(pts, z["points"]), pad


@pytest.mark.parametrize("W,H,frac", [(64, 48, 0.0), (64, 48, 1.0), (100, 37, 0.5),
                                      (752, 480, 0.7), (1920, 1080, 0.6), (4096, 2048, 0.3)])
def test_point_cloud_matches_oracle(oracle_mod, gpu, W, H, frac):
    rng = np.random.default_rng(W * 7 + H)
    depth = rng.uniform(0.2, 40.0, (H, W)).astype(np.float32)
    depth[rng.random((H, W)) >= frac] = -1.0
    ref = rng.integers(0, 256, (H, W), dtype=np.uint8)
    cam = (0.6 * W, 0.6 * W, W / 2.0 - 0.25, H / 2.0 + 0.5)
    a = 0.4
    T = np.array([[np.cos(a), 0.0, np.sin(a), 3.0], [0.0, 1.0, 0.0, -1.0],
                  [-np.sin(a), 0.0, np.cos(a), 0.25]], np.float32)
    want = oracle_mod.point_cloud(depth, ref, cam, T)
    got = _gpu_cloud(depth, ref, cam, T, gpu)
    assert _same(got, want)


def test_facade_point_cloud(oracle_mod, gpu):
    """Depthmap.getPointCloud on the facade's own last result equals the
    oracle's cloud of getDepthmap / getReferenceImage / getT_world_ref."""
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap, Depthmap
    W, H = 160, 128
    f = 460.0 * W / 752.0
    imgs, Ts, _ = sequence(3, 40, W, H)
    dm = Depthmap(W, H, f, W / 2.0, f, H / 2.0, params=Params.for_range(64, 0.5, 50.0))
    batch = BatchDepthmap([dict(width=W, height=H, fx=f, fy=f, cx=W / 2.0, cy=H / 2.0)] * 2,
                          params=Params.for_range(64, 0.5, 50.0))
    n_points = []
    for i in range(40):
        has = dm.add_frames(imgs[i], Ts[i])
        batch.add_frames([imgs[i]] * 2, [Ts[i]] * 2)
        if has:
            want = oracle_mod.point_cloud(dm.getDepthmap(), dm.getReferenceImage(),
                                          (f, f, W / 2.0, H / 2.0), dm.getT_world_ref())
            got = dm.getPointCloud()
            assert _same(got, want)
            assert _same(batch.get_point_cloud(1), want)
            n_points.append(len(got))
    assert max(n_points) > 0  # fused depth became valid somewhere


def test_point_cloud_rejects_small_workspace(gpu):
    import ctypes
    from open_quadtree_mapping_b200 import _lib
    H, W = 48, 64
    depth = torch.ones((H, W), dtype=torch.float32, device=gpu)
    ref = torch.zeros((H, W), dtype=torch.uint8, device=gpu)
    pts = torch.empty((H * W, 4), dtype=torch.float32, device=gpu)
    count = torch.zeros(1, dtype=torch.int32, device=gpu)
    need = ctypes.c_size_t()
    _lib.check(_lib.lib().qm_point_cloud_workspace_size(W, H, ctypes.byref(need)))
    ws = torch.empty(need.value, dtype=torch.uint8, device=gpu)
    c = _lib.QmCamera(50.0, 50.0, 32.0, 24.0)
    T = np.ascontiguousarray(np.eye(3, 4, dtype=np.float32).reshape(12))
    st = _lib.lib().qm_point_cloud(depth.data_ptr(), W, ref.data_ptr(), W, W, H, ctypes.byref(c),
                                   T.ctypes.data, pts.data_ptr(), count.data_ptr(), ws.data_ptr(),
                                   need.value - 1, None)
    assert st != 0
    st = _lib.lib().qm_point_cloud(depth.data_ptr(), W - 1, ref.data_ptr(), W, W, H,
                                   ctypes.byref(c), T.ctypes.data, pts.data_ptr(),
                                   count.data_ptr(), ws.data_ptr(), need.value, None)
    assert st != 0  # depth stride below the width
