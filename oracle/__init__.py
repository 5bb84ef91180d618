"""CPU oracle for the KAMI block-GEMM / block-SpGEMM path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` may import this package, and only as the
checker.  The product (``kami_b200``) never imports it.
"""
from .oracle import *  # noqa: F401,F403
