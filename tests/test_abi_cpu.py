"""The C-ABI library loads without a GPU, exports every entry point that
include/mfa_gpu.h declares, and its structs match the ctypes mirrors.  Only
argument-validation paths (which return before any CUDA call) are exercised."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from mfa_b200 import _abi
from mfa_b200.params import Spec, derive

HEADER = os.path.join(ROOT, "include", "mfa_gpu.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(mfa_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(mfa_\w+)", out))
    for n in names:
        assert n in exported, n
        assert hasattr(lib, n)
        assert n in _abi.SIGNATURES, f"{n} missing from the ctypes mirror"


def test_struct_sizes_match_header():
    lib = _abi.load()
    pb, sb = C.c_int32(0), C.c_int32(0)
    assert lib.mfa_abi_sizes(C.byref(pb), C.byref(sb)) == 0
    assert pb.value == C.sizeof(_abi.MfaParams)
    assert sb.value == C.sizeof(_abi.MfaScalars)
    assert lib.mfa_abi_version() == 1


def test_status_strings():
    lib = _abi.load()
    for s in range(0, 10):
        assert len(lib.mfa_status_string(s)) > 0


def _spec(n=4):
    return Spec(n_part=n, boundary=(10.0, 10.0, 10.0), n_type=1)


def test_init_rejects_bad_arguments_before_touching_the_device():
    lib = _abi.load()
    p = derive(_spec())
    r0 = np.zeros((4, 3))
    t = np.ones(4, dtype=np.int32)
    m = np.ones(4)
    ctx = C.c_void_p()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    # type outside 1..n_type
    bad_t = np.array([1, 2, 1, 1], dtype=np.int32)
    assert lib.mfa_init(C.byref(p), _abi.MIXED, -1, dp(r0), None, None, ip(bad_t), dp(m), None, None,
                        C.byref(ctx)) == _abi.ERR_ARGS
    # non-positive mass
    bad_m = np.array([1.0, 0.0, 1.0, 1.0])
    assert lib.mfa_init(C.byref(p), _abi.MIXED, -1, dp(r0), None, None, ip(t), dp(bad_m), None, None,
                        C.byref(ctx)) == _abi.ERR_ARGS
    # unknown precision
    assert lib.mfa_init(C.byref(p), 7, -1, dp(r0), None, None, ip(t), dp(m), None, None,
                        C.byref(ctx)) == _abi.ERR_ARGS
    # charged without charges
    pc = p.copy()
    pc.charged = 1
    assert lib.mfa_init(C.byref(pc), _abi.MIXED, -1, dp(r0), None, None, ip(t), dp(m), None, None,
                        C.byref(ctx)) == _abi.ERR_ARGS
    # chain topology larger than the particle count
    pt = p.copy()
    pt.n_mon, pt.n_chain = 3, 2
    assert lib.mfa_init(C.byref(pt), _abi.MIXED, -1, dp(r0), None, None, ip(t), dp(m), None, None,
                        C.byref(ctx)) == _abi.ERR_ARGS
    # delta_bin outside -1..1
    pd = p.copy()
    pd.delta_bin[0] = 2
    assert lib.mfa_init(C.byref(pd), _abi.MIXED, -1, dp(r0), None, None, ip(t), dp(m), None, None,
                        C.byref(ctx)) == _abi.ERR_ARGS
    # null context handles
    for fn in ("mfa_verlet_positions", "mfa_binning", "mfa_fluid_fluid", "mfa_intra_molec",
               "mfa_verlet_velocities", "mfa_zero_forces", "mfa_finalize", "mfa_sync"):
        assert getattr(lib, fn)(None) == _abi.ERR_ARGS


def test_product_package_does_not_reference_the_oracle():
    pkg = os.path.join(ROOT, "mfa_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in txt.lower(), f


@pytest.mark.parametrize("n_bin", [(1 << 17 + 1, 1, 1), (1 << 16, 1 << 16, 1 << 16),
                                   (2 ** 31 - 1, 2 ** 31 - 1, 2 ** 31 - 1), (64, 64, 64)])
def test_noalloc_binning_rejects_grids_beyond_capacity_before_any_cuda_call(n_bin):
    """Each n_bin factor and each partial product is checked against the fixed
    131,072-cell capacity before the product is formed, so three large values
    cannot wrap the cell count past the check.  The rejection comes before any
    CUDA call (no GPU here: a call that got further would fail with
    MFA_ERR_CUDA instead); the buffers are never touched."""
    lib = _abi.load()
    dummy = np.zeros(16, dtype=np.int32)
    r0 = np.zeros((1, 3))
    b = (C.c_double * 3)(10.0, 10.0, 10.0)
    nb = (C.c_int32 * 3)(*n_bin)
    ptr = C.c_void_p(dummy.ctypes.data)
    rc = lib.mfa_bin_cells_noalloc(C.c_void_p(r0.ctypes.data), 1, b, nb, 0, ptr, ptr, ptr, None)
    assert rc == _abi.ERR_CAPACITY
