"""B200 (sm_100a) implementation of ANQI's reverse-kNN hot path.

``anqi.formats`` reads and writes every prefix file of the reference;
``anqi._lib.Context`` drives the CUDA kernels of libanqi.so through the C ABI
declared in include/anqi.h.
"""
from . import formats  # noqa: F401
