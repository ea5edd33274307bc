"""B200 (sm_100a) engine for CudaMONSEL's electron-transport hot path.

The C ABI (include/cudamonsel_b200.h, libcudamonsel_b200.so) is the product
boundary; ``capi.Engine`` binds it from Python, ``scenes`` builds scenes in the
reference's terms and ``stats`` states errors between runs.
"""
from . import capi, data, scenes, stats  # noqa: F401
from .capi import PREC_FP32, PREC_FP64, CMError, Engine  # noqa: F401

__all__ = ["capi", "data", "scenes", "stats", "Engine", "CMError", "PREC_FP32", "PREC_FP64"]
