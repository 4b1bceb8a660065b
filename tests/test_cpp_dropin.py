"""The C++ drop-in header (include/qm_depthmap.hpp, the quadmap::Depthmap API)
compiles and links against libqm_b200.so with a plain g++; on a GPU it runs a
short sequence to depth maps, without one it reports the CUDA error.

tests/cpp/ros_caller.cpp holds the reference's own callers' statements (ROS
node construction and frame callback, publisher getters and point-cloud
loop) and is built with QM_WITH_OPENCV over a minimal cv::Mat stand-in
(tests/cpp/cvstub), so the OpenCV overloads compile and run too.  When the
environment variable QM_REFERENCE_TREE names the reference's source tree,
the same file is also compiled against the reference's own SE3 type."""
import os
import subprocess

import pytest

from conftest import ROOT, has_gpu
from open_quadtree_mapping_b200 import build_ext

CXX = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include")]
CV_STUB = ["-DQM_WITH_OPENCV", "-I", os.path.join(ROOT, "tests", "cpp", "cvstub")]


def _link(src, out, extra=()):
    subprocess.run(CXX + list(extra) + [os.path.join(ROOT, "tests", "cpp", src),
                                        "-L", build_ext.OUT_DIR, "-lqm_b200",
                                        "-Wl,-rpath," + build_ext.OUT_DIR, "-o", out],
                   check=True)
    return out


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    build_ext.build()
    return _link("depthmap_smoke.cpp", str(tmp_path_factory.mktemp("cpp") / "depthmap_smoke"))


@pytest.fixture(scope="module")
def ros_exe(tmp_path_factory):
    build_ext.build()
    return _link("ros_caller.cpp", str(tmp_path_factory.mktemp("cpp") / "ros_caller"), CV_STUB)


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_cpp_dropin_without_gpu(exe):
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 3, r.stdout + r.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_reference_callers_compile_without_gpu(ros_exe):
    r = subprocess.run([ros_exe], capture_output=True, text=True)
    assert r.returncode == 3, r.stdout + r.stderr


def test_reference_callers_compile_with_reference_se3(tmp_path):
    tree = os.environ.get("QM_REFERENCE_TREE")
    if not tree or not os.path.isdir(os.path.join(tree, "include", "quadmap")):
        pytest.skip("QM_REFERENCE_TREE does not name the reference's source tree")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(CXX + CV_STUB + ["-DQM_TEST_REFERENCE_SE3", "-I", os.path.join(cuda, "include"),
                                    "-I", os.path.join(tree, "include"), "-fsyntax-only",
                                    os.path.join(ROOT, "tests", "cpp", "ros_caller.cpp")],
                   check=True)


@pytest.mark.gpu
def test_cpp_dropin_on_gpu(exe):
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "results=" in r.stdout


@pytest.mark.gpu
def test_reference_callers_run_on_gpu(ros_exe):
    """The callers' statements run unchanged: 40 frames of a textured plane
    give depth maps, the pose getter converts to SE3<float> with the value
    the facade stores, and the fused map yields cloud points on the plane."""
    r = subprocess.run([ros_exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
