"""The C++ drop-in header (include/qm_depthmap.hpp, the quadmap::Depthmap API)
compiles and links against libqm_b200.so with a plain g++; on a GPU it runs a
short sequence to depth maps, without one it reports the CUDA error."""
import os
import subprocess

import pytest

from conftest import ROOT, has_gpu
from open_quadtree_mapping_b200 import build_ext


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    build_ext.build()
    out = str(tmp_path_factory.mktemp("cpp") / "depthmap_smoke")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "depthmap_smoke.cpp"),
                    "-L", build_ext.OUT_DIR, "-lqm_b200", "-Wl,-rpath," + build_ext.OUT_DIR,
                    "-o", out], check=True)
    return out


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_cpp_dropin_without_gpu(exe):
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 3, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_dropin_on_gpu(exe):
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "results=" in r.stdout
