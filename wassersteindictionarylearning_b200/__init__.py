"""B200-native Sinkhorn-barycenter hot path of Wasserstein dictionary learning.

The compute lives in ``lib/libwdl_b200.so`` (CUDA, sm_100a) behind the C ABI of
``include/wdl.h``; this package is the Python mirror of the reference's
KernelType / Problem / WassersteinRegression interface over that ABI.
"""
from ._lib import WdlError, build, lib  # noqa: F401
from .kernels import (CudaGaussian2DKernel, CudaGaussian3DKernel,  # noqa: F401
                      CudaLogSignArrayGaussian2DKernel)
from .regression import (LOSS_KL, LOSS_QUADRATIC, LOSS_TV, LOSS_WASSERSTEIN,  # noqa: F401
                         Problem, WassersteinBarycenter, WassersteinRegression)
