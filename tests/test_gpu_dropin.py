"""GPU: the reference's own C++ classes (WassersteinRegression, liblbfgs'
regress_both) instantiated on the CUDA KernelType of include/wdl_kernels.hpp,
checked against the same classes on the reference's Gaussian2DKernel.  The
program (oracle/dropin_demo.cpp) is built where the reference sources exist;
its binary travels prebuilt in oracle/_ref/."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
DEMO = os.path.join(ROOT, "oracle", "_ref", "dropin_demo")


@pytest.mark.skipif(not os.path.exists(DEMO), reason="oracle/_ref/dropin_demo not built")
def test_reference_classes_on_cuda_kerneltype():
    r = subprocess.run([DEMO], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
