"""CPU checks of the C-ABI library: it loads, exports every symbol that
include/qm_capi.h declares, and rejects bad arguments before touching CUDA."""
import ctypes
import subprocess

import pytest

from conftest import has_gpu
from open_quadtree_mapping_b200 import _lib, build_ext
from open_quadtree_mapping_b200.params import Params, QmParamsC


@pytest.fixture(scope="module")
def L():
    build_ext.build()
    return _lib.lib()


def test_exports_every_declared_symbol(L):
    declared = _lib.declared_symbols()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", build_ext.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:
        assert hasattr(L, s)
    # every declared symbol has a ctypes signature
    assert set(declared) <= set(_lib._SIGS)


def test_build_targets_sm100a_only():
    assert build_ext.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_default_params_match_reference_constants(L):
    p = _lib.default_params()
    d = Params()
    assert p.num_hyp == d.num_hyp == 64
    assert p.min_inv_depth == d.min_inv_depth == 0.01
    assert p.inv_depth_step == d.inv_depth_step == (2.0 - 0.01) / 63.0
    assert list(p.bp_iters)[:4] == [4, 10, 10, 10]
    assert (p.qt_max_level, p.qt_min_level, p.qt_threshold) == (4, 2, 10.0)
    assert abs(p.P1 - 0.003) < 1e-9 and abs(p.P2 - 0.01) < 1e-9
    assert (p.up_sigma, p.up_lambda) == (400.0, 10.0)
    assert ctypes.sizeof(QmParamsC) == ctypes.sizeof(p)


def test_tune_fields_match_header():
    """The Python binding passes qm_tune as a plain int array in field order:
    the header's struct must list exactly those int fields, in that order."""
    import re
    from open_quadtree_mapping_b200.depthmap import BatchDepthmap
    text = open(_lib.HEADER).read()
    body = re.search(r"typedef struct qm_tune\s*\{(.*?)\}\s*qm_tune;", text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        assert decl.startswith("int "), decl
        fields += [f.strip() for f in decl[4:].split(",")]
    assert tuple(fields) == BatchDepthmap.TUNE_FIELDS


def test_invalid_arguments_without_gpu(L):
    p = _lib.default_params()
    assert L.qm_quadtree(None, 0, 2, 2, ctypes.byref(p), None, None) == _lib.QM_ERR_INVALID_ARG
    assert "image size" in _lib.last_error()
    bad = _lib.default_params()
    bad.num_hyp = 63
    n = ctypes.c_size_t()
    assert L.qm_bp_workspace_size(64, 64, ctypes.byref(bad), ctypes.byref(n)) == \
        _lib.QM_ERR_INVALID_ARG
    bad = _lib.default_params()
    bad.qt_max_level = 9
    assert L.qm_bp_workspace_size(64, 64, ctypes.byref(bad), ctypes.byref(n)) == \
        _lib.QM_ERR_INVALID_ARG
    assert L.qm_bp_workspace_size(64, 64, ctypes.byref(p), ctypes.byref(n)) == _lib.QM_OK
    assert n.value > 0
    assert L.qm_upsample_workspace_size(752, 480, ctypes.byref(n)) == _lib.QM_OK
    assert n.value >= 752 * 480 * 8  # the row-pass result, float2 per pixel
    h = ctypes.c_void_p()
    assert L.qm_depthmap_create(None, 64, 64, 1, 1, 1, 1, 1, None, 0) == _lib.QM_ERR_INVALID_ARG
    assert L.qm_depthmap_create(ctypes.byref(h), 64, 64, 50, 32, 50, 32, 0, None, 0) != _lib.QM_OK
    assert L.qm_depthmap_add_frame(None, None, 0, None, None) == _lib.QM_ERR_INVALID_ARG
    assert L.qm_batch_create(ctypes.byref(h), 0, None, None, 0) == _lib.QM_ERR_INVALID_ARG


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_reports_cuda_error(L):
    h = ctypes.c_void_p()
    rc = L.qm_depthmap_create(ctypes.byref(h), 64, 64, 50.0, 32.0, 50.0, 32.0, 1, None, 0)
    assert rc == _lib.QM_ERR_CUDA
    assert _lib.last_error()
    assert not h.value
