"""B200-native (sm_100a) light-transport passes of the hdRestir render delegate.

The product is the CUDA library behind include/hdrestir.h
(``libhdrestir_b200.so``); this package builds it, binds it with ctypes and
mirrors the reference's pass interface on top of it.
"""
from .abi import HdrError  # noqa: F401
