"""Algorithm parameters of the depth pipeline, with the reference's values.

The reference compiles every constant in (stereo_parameter.cuh:2-42,
pixel_cost.cuh:4, bpextract.cu:41-45,222-223, quadtree.cu:40,59,74,
depth_upsample.cu, depth_fusion.cu:13-15).  Here they are one runtime struct,
`qm_params` in include/qm_capi.h; this module mirrors it for Python callers.
"""
from __future__ import annotations

import ctypes
import dataclasses

ARITH_REFERENCE = 0  # fast-math arithmetic of the reference build (-use_fast_math)
ARITH_IEEE = 1       # IEEE-rounded arithmetic; equals the CPU oracle bit for bit

MAX_BP_LEVELS = 8


@dataclasses.dataclass
class Params:
    num_hyp: int = 64                 # pixel_cost.cuh:4 DEPTH_NUM
    min_inv_depth: float = 0.01       # stereo_parameter.cuh:5 MIN_INV_DEPTH
    inv_depth_step: float = (2.0 - 0.01) / 63.0  # stereo_parameter.cuh:7 STEP_INV_DEPTH
    P1: float = 0.003                 # bpextract.cu:222
    P2: float = 0.01                  # bpextract.cu:223
    bp_levels: int = 4                # bpextract.cu:41
    bp_iters: tuple = (4, 10, 10, 10) # bpextract.cu:45, fine -> coarse
    qt_max_level: int = 4             # quadtree.cu:40
    qt_min_level: int = 2             # quadtree.cu:74
    qt_threshold: float = 10.0        # quadtree.cu:59
    up_sigma: float = 400.0           # stereo_parameter.cuh upsample_sigma
    up_lambda: float = 10.0           # stereo_parameter.cuh upsample_lambda
    arith: int = ARITH_REFERENCE

    @staticmethod
    def for_range(num_hyp: int, min_depth: float, max_depth: float, **kw) -> "Params":
        """Hypotheses uniform in inverse depth over [1/max_depth, 1/min_depth]."""
        lo = 1.0 / max_depth
        hi = 1.0 / min_depth
        return Params(num_hyp=num_hyp, min_inv_depth=lo,
                      inv_depth_step=(hi - lo) / float(num_hyp - 1), **kw)

    def hyp_depths(self):
        return [1.0 / (self.inv_depth_step * d + self.min_inv_depth) for d in range(self.num_hyp)]


class QmParamsC(ctypes.Structure):
    """ctypes mirror of `qm_params` (include/qm_capi.h)."""
    _fields_ = [
        ("num_hyp", ctypes.c_int),
        ("min_inv_depth", ctypes.c_double),
        ("inv_depth_step", ctypes.c_double),
        ("P1", ctypes.c_float),
        ("P2", ctypes.c_float),
        ("bp_levels", ctypes.c_int),
        ("bp_iters", ctypes.c_int * MAX_BP_LEVELS),
        ("qt_max_level", ctypes.c_int),
        ("qt_min_level", ctypes.c_int),
        ("qt_threshold", ctypes.c_float),
        ("up_sigma", ctypes.c_double),
        ("up_lambda", ctypes.c_double),
        ("arith", ctypes.c_int),
    ]

    @classmethod
    def from_params(cls, p: Params) -> "QmParamsC":
        c = cls()
        c.num_hyp = p.num_hyp
        c.min_inv_depth = p.min_inv_depth
        c.inv_depth_step = p.inv_depth_step
        c.P1 = p.P1
        c.P2 = p.P2
        c.bp_levels = p.bp_levels
        for i in range(MAX_BP_LEVELS):
            c.bp_iters[i] = p.bp_iters[i] if i < len(p.bp_iters) else 0
        c.qt_max_level = p.qt_max_level
        c.qt_min_level = p.qt_min_level
        c.qt_threshold = p.qt_threshold
        c.up_sigma = p.up_sigma
        c.up_lambda = p.up_lambda
        c.arith = p.arith
        return c
