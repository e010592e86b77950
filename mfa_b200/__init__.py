"""mfa_b200: B200 (sm_100a) implementation of mfa's per-timestep force and
integration loop, behind the reference's subroutine interface.

The compute path is libmfa_gpu.so (hand-written CUDA, C ABI in
include/mfa_gpu.h).  This package holds the host side: the ctypes binding,
the derivation of run constants, configuration generators and the ``System``
class that mirrors the reference's per-step subroutines.
"""
from . import _abi
from ._abi import FP64, MIXED, MfaError, MfaParams, MfaScalars
from .params import Spec, derive

__all__ = ["_abi", "FP64", "MIXED", "MfaError", "MfaParams", "MfaScalars", "Spec", "derive",
           "System", "Batch", "from_config"]


def __getattr__(name):
    # the System class needs the CUDA library; load it lazily so that the
    # parameter and configuration helpers import without a GPU build present
    if name in ("System", "Batch", "from_config"):
        import importlib
        return getattr(importlib.import_module(".api", __name__), name)
    raise AttributeError(name)
