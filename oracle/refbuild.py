"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the reference comparator
(oracle/_ref/libqm_ref.so: the reference's own CUDA kernels built from its
sources by `make -C oracle ref`; oracle/_ref/libqm_ref_<variant>.so: the
same kernels from patched copies at other hypothesis counts and ranges,
`make -C oracle ref-variants`, see oracle/refpatch.py).  Runs on a GPU only.
Used by tests/, tests/golden/make_golden.py and bench.py's reference-kernel
timing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .oracle import REF_LIB_PATH

F32P = ctypes.POINTER(ctypes.c_float)
REF_DIR = os.path.dirname(REF_LIB_PATH)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class Comparator:
    """One comparator build: the reference's kernels as compiled (DEPTH_NUM
    64, inverse depth [0.01, 2.0]) or a patched variant (oracle/refpatch.py)."""

    def __init__(self, path):
        self.path = path
        self._lib = None

    def available(self) -> bool:
        return os.path.exists(self.path)

    def lib(self):
        if self._lib is None:
            if not self.available():
                raise RuntimeError("reference comparator not built: make -C oracle "
                                   "ref-if-present (%s)" % os.path.basename(self.path))
            L = ctypes.CDLL(self.path)
            f = ctypes.c_float
            p = ctypes.c_void_p
            L.qmref_extract.restype = ctypes.c_int
            L.qmref_extract.argtypes = [ctypes.c_int, ctypes.c_int, f, f, f, f, p, ctypes.c_int,
                                        p, p, ctypes.c_int, p, p, p, p, p]
            L.qmref_fuse.restype = ctypes.c_int
            L.qmref_fuse.argtypes = [ctypes.c_int, ctypes.c_int, f, f, f, f, p, p, p, p]
            L.qmref_tex_sample.restype = ctypes.c_int
            L.qmref_tex_sample.argtypes = [ctypes.c_int, ctypes.c_int, p, p, ctypes.c_int, p]
            L.qmref_semidense.restype = ctypes.c_int
            L.qmref_semidense.argtypes = [ctypes.c_int, ctypes.c_int, f, f, f, f, ctypes.c_int,
                                          p, p, p, p, p]
            L.qmref_time_frames.restype = ctypes.c_int
            L.qmref_time_frames.argtypes = [ctypes.c_int, ctypes.c_int, f, f, f, f, p,
                                            ctypes.c_int, p, p, ctypes.c_int, p, ctypes.c_int,
                                            ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
            L.qmref_depth_num.restype = ctypes.c_int
            L.qmref_depth_num.argtypes = []
            L.qmref_min_inv_depth.restype = ctypes.c_double
            L.qmref_min_inv_depth.argtypes = []
            L.qmref_inv_depth_step.restype = ctypes.c_double
            L.qmref_inv_depth_step.argtypes = []
            self._lib = L
        return self._lib

    @property
    def depth_num(self) -> int:
        return int(self.lib().qmref_depth_num())

    @property
    def min_inv_depth(self) -> float:
        return float(self.lib().qmref_min_inv_depth())

    @property
    def inv_depth_step(self) -> float:
        return float(self.lib().qmref_inv_depth_step())

    def extract(self, income_u8, ring_u8, T_frame_income, cam, nslots=5, debug_in=None,
                want_messages=True):
        """SeedMatrix::extract_depth with the reference kernels.  ring_u8: (n,
        H, W) most recent first; T_frame_income: (n, 12)."""
        D = self.depth_num
        income = np.ascontiguousarray(income_u8, np.float32)
        H, W = income.shape
        ring = np.ascontiguousarray(np.asarray(ring_u8, np.float32))
        n = ring.shape[0]
        T = np.ascontiguousarray(np.asarray(T_frame_income, np.float32).reshape(n, 12))
        debug = (np.zeros((H, W), np.float32) if debug_in is None
                 else np.array(debug_in, np.float32, copy=True))
        levels = np.zeros((H, W), np.int32)
        cost = np.zeros((H // 4, W // 4, D), np.float32)
        msgs = np.zeros((4, H // 4, W // 4, D), np.float32) if want_messages else None
        dense = np.zeros((H, W), np.float32)
        fx, fy, cx, cy = [ctypes.c_float(v) for v in cam]
        rc = self.lib().qmref_extract(W, H, fx, fy, cx, cy, _p(income), n, _p(ring), _p(T),
                                      nslots, _p(debug), _p(levels), _p(cost), _p(msgs),
                                      _p(dense))
        if rc != 0:
            raise RuntimeError("qmref_extract failed: %d" % rc)
        return dict(levels=levels, cost=cost, messages=msgs, sparse=debug, dense=dense)

    def fuse(self, depth, seeds, T_income_last, cam):
        depth = np.array(depth, np.float32, copy=True)
        H, W = depth.shape
        seeds = np.array(seeds, np.float32, copy=True).reshape(H, W, 4)
        T = np.ascontiguousarray(np.asarray(T_income_last, np.float32).reshape(12))
        table = np.zeros((H, W), np.int32)
        fx, fy, cx, cy = [ctypes.c_float(v) for v in cam]
        rc = self.lib().qmref_fuse(W, H, fx, fy, cx, cy, _p(depth), _p(seeds), _p(T), _p(table))
        if rc != 0:
            raise RuntimeError("qmref_fuse failed: %d" % rc)
        return depth, seeds, table

    def time_frames(self, income_u8, ring_u8, T_frame_income, cam, nslots=5, warmup=2,
                    iters=10):
        income = np.ascontiguousarray(income_u8, np.float32)
        H, W = income.shape
        ring = np.ascontiguousarray(np.asarray(ring_u8, np.float32))
        n = ring.shape[0]
        T = np.ascontiguousarray(np.asarray(T_frame_income, np.float32).reshape(n, 12))
        T_last = np.ascontiguousarray(np.eye(3, 4, dtype=np.float32).reshape(12))
        ms = ctypes.c_double()
        fx, fy, cx, cy = [ctypes.c_float(v) for v in cam]
        rc = self.lib().qmref_time_frames(W, H, fx, fy, cx, cy, _p(income), n, _p(ring), _p(T),
                                          nslots, _p(T_last), warmup, iters, ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError("qmref_time_frames failed: %d" % rc)
        return ms.value

    def semidense(self, frames, T_cur_world, cam):
        """The reference's semi-dense tracker over a frame sequence
        (qmref_semidense): frames (n, H, W) u8, T_cur_world (n, 12).  Returns
        (debug (n, H, W) f32, seeds (H, W, 8) f32 after the last frame, modes
        (n,) int32)."""
        frames = np.ascontiguousarray(frames, np.float32)
        n, H, W = frames.shape
        T = np.ascontiguousarray(T_cur_world, np.float32).reshape(n, 12)
        debug = np.zeros((n, H, W), np.float32)
        seeds = np.zeros((H, W, 8), np.float32)
        modes = np.zeros(n, np.int32)
        fx, fy, cx, cy = [float(v) for v in cam]
        rc = self.lib().qmref_semidense(W, H, fx, fy, cx, cy, n, _p(frames), _p(T), _p(debug),
                                        _p(seeds), _p(modes))
        if rc != 0:
            raise RuntimeError("qmref_semidense failed: %d" % rc)
        return debug, seeds, modes

    def tex_sample(self, img, uv):
        """Texture-unit bilinear samples of a u8 image (as float texels) at
        the (n, 2) unnormalised coordinates uv (qmref_tex_sample)."""
        img = np.ascontiguousarray(img, np.float32)
        H, W = img.shape
        uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
        out = np.zeros(len(uv), np.float32)
        rc = self.lib().qmref_tex_sample(W, H, _p(img), _p(uv), len(uv), _p(out))
        if rc != 0:
            raise RuntimeError("qmref_tex_sample failed: %d" % rc)
        return out


_default = Comparator(REF_LIB_PATH)
DEPTH_NUM = 64


def variant(name: str) -> Comparator:
    """A patched comparator build, e.g. variant("d128_lo0.02"): 128
    hypotheses over inverse depth [0.02, 2.0] (make -C oracle ref-variants)."""
    return Comparator(os.path.join(REF_DIR, "libqm_ref_%s.so" % name))


def available() -> bool:
    return _default.available()


def lib():
    return _default.lib()


def extract(*a, **k):
    return _default.extract(*a, **k)


def fuse(*a, **k):
    return _default.fuse(*a, **k)


def time_frames(*a, **k):
    return _default.time_frames(*a, **k)


def semidense(*a, **k):
    return _default.semidense(*a, **k)


def tex_sample(*a, **k):
    return _default.tex_sample(*a, **k)


def _tree_argmin(b):
    """Stride-halving argmin over the last axis with the right element winning
    only when strictly smaller (bpextract.cu:347-355)."""
    v = b.copy()
    idx = np.broadcast_to(np.arange(b.shape[-1]), b.shape).copy()
    s = b.shape[-1] // 2
    while s > 0:
        take = v[..., s:2 * s] < v[..., :s]
        v[..., :s] = np.where(take, v[..., s:2 * s], v[..., :s])
        idx[..., :s] = np.where(take, idx[..., s:2 * s], idx[..., :s])
        s //= 2
    return idx[..., 0]


def labels_from_messages(cost, msgs, levels, W, H):
    """Winning labels of depth_extract (bpextract.cu:314-372) from the cost
    volume and the final level-0 messages (up, down, left, right), -1 at
    cells that are not node origins."""
    ch, cw, D = cost.shape
    up, down, left, right = msgs
    b = cost.astype(np.float32).copy()
    b[:, 1:] += right[:, :-1]
    b[:, :-1] += left[:, 1:]
    b[1:, :] += down[:-1, :]
    b[:-1, :] += up[1:, :]
    lab = _tree_argmin(b).astype(np.int32)
    ys = np.minimum(np.arange(ch) * 4, H - 1)
    xs = np.minimum(np.arange(cw) * 4, W - 1)
    size = 1 << levels[np.ix_(ys, xs)]
    node = ((np.arange(cw)[None, :] * 4) % size == 0) & ((np.arange(ch)[:, None] * 4) % size == 0)
    return np.where(node, lab, -1).astype(np.int32)
