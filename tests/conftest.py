import functools
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@functools.lru_cache(maxsize=None)
def keyframe(stream: int, W: int, H: int, F: int = 5, f: float | None = None):
    """Seeded synthetic keyframe (scene 1000+stream, trajectory 2000+stream)."""
    from open_quadtree_mapping_b200 import synthetic as syn
    fx = f if f is not None else 460.0 * W / 752.0
    return syn.make_keyframe(stream, W=W, H=H, fx=fx, fy=fx, F=F)


@functools.lru_cache(maxsize=None)
def sequence(stream: int, n: int, W: int, H: int, f: float | None = None):
    from open_quadtree_mapping_b200 import synthetic as syn
    fx = f if f is not None else 460.0 * W / 752.0
    return syn.make_sequence(stream, n, W=W, H=H, fx=fx, fy=fx)


def cam_of(kf):
    return (kf.fx, kf.fy, kf.cx, kf.cy)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    oracle.set_threads(min(8, os.cpu_count() or 1))
    return oracle


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("needs a CUDA GPU")
    import torch
    from open_quadtree_mapping_b200 import build_ext
    build_ext.build()
    return torch.device("cuda:0")
