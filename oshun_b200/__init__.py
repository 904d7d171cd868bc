"""oshun_b200 — B200 (sm_100a) implementation of OSHUN's RK4 Vlasov-Maxwell
stage and Fokker-Planck collision step behind a C ABI (include/oshun_b200.h).

The product is liboshun_b200.so (built from csrc/ by ``build.py``); ``abi``
is its ctypes binding and ``host/oshun.hpp`` the C++ mirror of the
reference's operator classes.  Nothing here falls back to a CPU path.
"""
from .abi import Batch, Handle, OshunError, load, OSHUN_FP64, OSHUN_FP32_SPLIT, OSHUN_FLAG_FIX_YADV_CHAIN, OSHUN_FLAG_IMPLICIT_EE  # noqa: F401
