"""The C++ host layer (mikroptim_b200/host): reference-shaped SystemBatchHost / ResidualLayout /
VariableSet / TraceEngine (RESIDUALS, MERIT, prefilter, EVAL) / PsfEngine / DeviceFdJacobian /
DeviceAdjointJacobian / DeviceNormalEquations / optimize_lm_gpu (with paraxial constraints on the
device) over the C ABI.

CPU: the layer builds, exports its classes, and the test driver (tests/cpp/test_host.cpp)
compiles and links against it and the oracle. GPU: the driver traces, differentiates and
optimises a singlet batch and checks every result against the oracle bit for bit.
"""

import os
import shutil
import subprocess

import pytest

from mikroptim_b200 import build as mbuild
import oracle.pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "cpp", "_build")
DRIVER = os.path.join(OUT, "test_host")


def build_driver() -> str:
    mbuild.build()
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(HERE, "cpp", "test_host.cpp")
    cuda = mbuild.CUDA_HOME
    cmd = [shutil.which("g++") or "g++", "-std=c++20", "-O2", "-Wall", src, "-o", DRIVER,
           "-I", os.path.join(ROOT, "include"), "-I", mbuild.HOST_DIR,
           "-I", os.path.join(ROOT, "oracle"), "-I", os.path.join(cuda, "include"),
           "-L", mbuild.HERE, "-lmikroptim_b200_host", "-lmikroptim_b200",
           "-L", os.path.dirname(po.PORT_LIB), "-l:" + os.path.basename(po.PORT_LIB),
           "-L", os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath," + mbuild.HERE, "-Wl,-rpath," + os.path.dirname(po.PORT_LIB),
           "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    if os.path.exists(po.REF_LIB):  # the reference's CPU build: extra-row checks against it
        cmd += ["-DMKB_HAVE_REF", "-L", os.path.dirname(po.REF_LIB),
                "-l:" + os.path.basename(po.REF_LIB),
                "-Wl,-rpath," + os.path.dirname(po.REF_LIB)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return DRIVER


def test_host_layer_builds_and_exports_classes():
    lib = mbuild.build_host()
    syms = subprocess.run(["nm", "-DC", lib], capture_output=True, text=True).stdout
    for name in ("mkb::SystemBatchHost::validate_values", "mkb::ResidualLayout::plan",
                 "mkb::VariableSet::VariableSet", "mkb::cuda::TraceEngine::run",
                 "mkb::cuda::DeviceFdJacobian::compute", "mkb::cuda::DeviceAdjointJacobian::compute",
                 "mkb::cuda::DeviceNormalEquations::compute", "mkb::cuda::optimize_lm_gpu",
                 "mkb::cuda::TraceEngine::prefilter_variants", "mkb::cuda::TraceEngine::evaluate",
                 "mkb::LmOptions::c_struct", "mkb::cuda::PsfEngine::compute",
                 "mkb::cuda::make_psf_pupils"):
        assert name in syms, name


def test_host_driver_compiles_and_links():
    assert os.access(build_driver(), os.X_OK)


@pytest.mark.gpu
def test_host_driver_matches_oracle_bitwise():
    res = subprocess.run([build_driver()], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "checks passed" in res.stdout
