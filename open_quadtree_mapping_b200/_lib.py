"""ctypes binding of libqm_b200.so (include/qm_capi.h).

The library is the only compute path: loading fails loudly when it has not
been built (run `python -m open_quadtree_mapping_b200.build_ext`).
"""
from __future__ import annotations

import ctypes
import os
import re

from .build_ext import LIB_PATH, ROOT
from .params import QmParamsC

HEADER = os.path.join(ROOT, "include", "qm_capi.h")

QM_OK = 0
QM_ERR_INVALID_ARG = 1
QM_ERR_CUDA = 2
QM_ERR_NO_MEMORY = 3
QM_ERR_STATE = 4
QM_ERR_TIMEOUT = 5
QM_ERR_WORKSPACE = 6

_lib = None


class QmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("qm status %d: %s" % (status, msg))
        self.status = status


class QmCamera(ctypes.Structure):
    _fields_ = [("fx", ctypes.c_float), ("fy", ctypes.c_float),
                ("cx", ctypes.c_float), ("cy", ctypes.c_float)]


class QmStreamDesc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("cam", QmCamera),
                ("num_hyp", ctypes.c_int), ("num_slots", ctypes.c_int),
                ("semi2dense_ratio", ctypes.c_int)]


def declared_symbols():
    """Function names declared in include/qm_capi.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qm_[A-Za-z0-9_]+)\s*\(", text)))


_P = ctypes.c_void_p
_I = ctypes.c_int
_S = ctypes.c_size_t
_F = ctypes.c_float

_SIGS = {
    "qm_params_default": (None, [ctypes.POINTER(QmParamsC)]),
    "qm_last_error": (ctypes.c_char_p, []),
    "qm_version": (_I, []),
    "qm_depthmap_create": (_I, [ctypes.POINTER(_P), _I, _I, _F, _F, _F, _F, _I,
                                ctypes.POINTER(QmParamsC), _I]),
    "qm_depthmap_destroy": (_I, [_P]),
    "qm_depthmap_add_frame": (_I, [_P, _P, _S, _P, ctypes.POINTER(_I)]),
    "qm_depthmap_get_depth": (_I, [_P, _P, _S]),
    "qm_depthmap_get_debug": (_I, [_P, _P, _S]),
    "qm_depthmap_get_reference": (_I, [_P, _P, _S]),
    "qm_depthmap_get_variance": (_I, [_P, _P, _S]),
    "qm_depthmap_get_point_cloud": (_I, [_P, _P, _S, ctypes.POINTER(_I)]),
    "qm_depthmap_get_T_world_ref": (_I, [_P, _P]),
    "qm_depthmap_get_camera": (_I, [_P, ctypes.POINTER(QmCamera), ctypes.POINTER(_I),
                                    ctypes.POINTER(_I)]),
    "qm_batch_create": (_I, [ctypes.POINTER(_P), _I, ctypes.POINTER(QmStreamDesc),
                             ctypes.POINTER(QmParamsC), _I]),
    "qm_batch_destroy": (_I, [_P]),
    "qm_batch_add_frames": (_I, [_P, _P, _P, _P, _P]),
    "qm_batch_get_depth": (_I, [_P, _I, _P, _S]),
    "qm_batch_submit": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "qm_batch_wait": (_I, [_P]),
    "qm_batch_get_debug": (_I, [_P, _I, _P, _S]),
    "qm_batch_get_variance": (_I, [_P, _I, _P, _S]),
    "qm_batch_get_point_cloud": (_I, [_P, _I, _P, _S, ctypes.POINTER(_I)]),
    "qm_batch_get_depths": (_I, [_P, _I, _P, _P, _P]),
    "qm_batch_run_resident": (_I, [_P]),
    "qm_batch_device_depth": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "qm_batch_set_graphs": (_I, [_P, _I]),
    "qm_batch_set_semidense": (_I, [_P, _I]),
    "qm_batch_set_branches": (_I, [_P, _I]),
    "qm_depthmap_set_semidense": (_I, [_P, _I]),
    "qm_batch_set_group_bytes": (_I, [_P, _S]),
    "qm_batch_set_coarse_bp": (_I, [_P, _I]),
    "qm_batch_set_stagger": (_I, [_P, _I]),
    "qm_batch_set_autotune": (_I, [_P, _I]),
    "qm_batch_set_tune": (_I, [_P, ctypes.POINTER(_I)]),
    "qm_batch_get_tune": (_I, [_P, ctypes.POINTER(_I)]),
    "qm_batch_last_launches": (_I, [_P, ctypes.POINTER(_I)]),
    "qm_batch_stream": (_I, [_P, ctypes.POINTER(_P)]),
    "qm_batch_profile": (_I, [_P, ctypes.POINTER(_F), ctypes.POINTER(_I)]),
    "qm_quadtree": (_I, [_P, _S, _I, _I, ctypes.POINTER(QmParamsC), _P, _P]),
    "qm_cost_volume": (_I, [_P, _S, _I, _I, ctypes.POINTER(QmCamera), _P, _I, _P, _S, _P,
                            ctypes.POINTER(QmParamsC), _P, _P]),
    "qm_bp_workspace_size": (_I, [_I, _I, ctypes.POINTER(QmParamsC), ctypes.POINTER(_S)]),
    "qm_bp_extract": (_I, [_P, _I, _I, _P, ctypes.POINTER(QmParamsC), _P, _P, _P, _P, _S, _P]),
    "qm_upsample_workspace_size": (_I, [_I, _I, ctypes.POINTER(_S)]),
    "qm_upsample": (_I, [_P, _P, _S, _I, _I, ctypes.POINTER(QmParamsC), _P, _P, _S, _P]),
    "qm_upsample_noalloc": (_I, [_P, _P, _S, _I, _I, ctypes.POINTER(QmParamsC), _P, _P]),
    "qm_fuse_workspace_size": (_I, [_I, _I, ctypes.POINTER(_S)]),
    "qm_point_cloud_workspace_size": (_I, [_I, _I, ctypes.POINTER(_S)]),
    "qm_semidense_workspace_size": (_I, [_I, _I, ctypes.POINTER(_S)]),
    "qm_semidense_step": (_I, [_P, _P, _I, _I, ctypes.POINTER(QmCamera), _P, _I, _I, _P, _P, _P,
                               _P, _S, _P]),
    "qm_point_cloud": (_I, [_P, _S, _P, _S, _I, _I, ctypes.POINTER(QmCamera), _P, _P, _P, _P,
                            _S, _P]),
    "qm_fuse": (_I, [_P, _P, _P, _P, ctypes.POINTER(QmCamera), _I, _I,
                     ctypes.POINTER(QmParamsC), _P, _P, _S, _P]),
    "qm_bp_soft_workspace_size": (_I, [_I, _I, ctypes.POINTER(QmParamsC), ctypes.POINTER(_S)]),
    "qm_bp_soft_forward": (_I, [_P, _I, _I, _P, ctypes.POINTER(QmParamsC), _F, _P, _P, _S, _P]),
    "qm_bp_soft_backward": (_I, [_P, _I, _I, _P, ctypes.POINTER(QmParamsC), _F, _P, _P, _P, _S,
                                 _P]),
    "qm_bp_soft64_workspace_size": (_I, [_I, _I, ctypes.POINTER(QmParamsC), ctypes.POINTER(_S)]),
    "qm_bp_soft64_forward": (_I, [_P, _I, _I, _P, ctypes.POINTER(QmParamsC), _F, _P, _P, _S, _P]),
    "qm_bp_soft64_backward": (_I, [_P, _I, _I, _P, ctypes.POINTER(QmParamsC), _F, _P, _P, _P, _S,
                                 _P]),
    "qm_upsample_w_workspace_size": (_I, [_I, _I, ctypes.POINTER(_S)]),
    "qm_upsample_w_forward": (_I, [_P, _P, _S, _I, _I, ctypes.POINTER(QmParamsC), _P, _P, _P,
                                   _S, _P]),
    "qm_upsample_w_backward": (_I, [_P, _S, _I, _I, ctypes.POINTER(QmParamsC), _P, _P, _P, _P,
                                    _P, _S, _P]),
    "qm_fuse_backward": (_I, [_P, _P, _P, _I, _I, _P, _P, _P]),
}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libqm_b200.so is not built (%s); run `python -m "
                "open_quadtree_mapping_b200.build_ext`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    m = lib().qm_last_error()
    return m.decode() if m else ""


def check(status: int) -> None:
    if status != QM_OK:
        raise QmError(status, last_error())


def default_params() -> QmParamsC:
    p = QmParamsC()
    lib().qm_params_default(ctypes.byref(p))
    return p
