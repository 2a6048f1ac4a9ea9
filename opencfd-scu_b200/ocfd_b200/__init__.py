"""Host-side mirror of the OpenCFD-SCU RHS-path interface (B200 build).

The product is the C-ABI library ``libocfd_b200.so`` (CUDA kernels for
sm_100a behind ``include/ocfd_b200.h``); this package binds it with ctypes and
carries the case-file formats the reference reads.
"""
from . import formats, cases  # noqa: F401
