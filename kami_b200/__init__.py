"""kami_b200 -- a B200-native (sm_100a) implementation of the KAMI
block-GEMM / block-SpGEMM path, behind the C ABI of include/kami.h.

``kami_b200.api`` is the Python mirror of that ABI over torch CUDA tensors.
"""
from ._lib import KamiError, load  # noqa: F401

__version__ = "0.1.0"
