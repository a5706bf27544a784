"""parafaft_b200 — a B200-native transform backend for ParaFaFT.

The product is native code: ``include/b200fft.h`` (C ABI of the sm_100a
kernels in ``csrc/``) and ``include/fft_backend_b200.hpp`` (``B200Backend<T>``,
the ParaFaFT backend). This package builds them in-tree (``build``) and binds
them for Python callers (``native``).
"""
from . import native  # noqa: F401

__all__ = ["native"]
