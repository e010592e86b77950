"""The allocation-free binning entry point (mfa_bin_cells_noalloc).

It serves callers that must not allocate device memory -- programs that own
all of the GPU's memory through their own pools, or that call at a point where
an allocation's implicit synchronisation is not acceptable.  Here it is called
through the C ABI with caller-owned device buffers and checked against the cell
assignment of the regular entry point (mfa_binning), on two calls in a row with
different positions (the second call reuses the library's fixed scratch array).
This file is collected last so that a failure here never hides another test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mfa_b200 import _abi, configs
from mfa_b200.api import System

pytestmark = pytest.mark.gpu


def noalloc_binning(r0, boundary, n_bin, rule):
    lib = _abi.load()
    n = r0.shape[0]
    ncell = int(np.prod(n_bin))
    dev_r0 = torch.from_numpy(np.ascontiguousarray(r0, dtype=np.float64)).cuda()
    cell_of = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    cell_start = torch.full((ncell + 1,), -7, dtype=torch.int32, device="cuda")
    ids = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    b = (C.c_double * 3)(*[float(x) for x in boundary])
    nb = (C.c_int32 * 3)(*[int(x) for x in n_bin])
    rc = lib.mfa_bin_cells_noalloc(C.c_void_p(dev_r0.data_ptr()), n, b, nb, rule,
                                   C.c_void_p(cell_of.data_ptr()), C.c_void_p(cell_start.data_ptr()),
                                   C.c_void_p(ids.data_ptr()), None)
    return rc, cell_of.cpu().numpy(), cell_start.cpu().numpy(), ids.cpu().numpy()


def regular_binning(cfg, r0, rule):
    g = System(cfg.params, r0, cfg.v, cfg.a_type, cfg.mass, precision=_abi.MIXED)
    if rule == 0:
        g.binning()
    else:
        g.my_binning()
    cell, _, _ = g.debug_lists(1)
    g.close()
    return cell


@pytest.mark.parametrize("rule", [0, 1])
def test_noalloc_binning_matches_regular_binning_twice(rule):
    cfg = configs.melt(seed=21)
    p = cfg.params
    boundary = [p.boundary[d] for d in range(3)]
    n_bin = [p.n_bin[d] for d in range(3)]
    ncell = int(np.prod(n_bin))
    shifted = np.mod(cfg.r0 + np.array([3.7, -1.3, 5.9]), np.array(boundary))
    for r0 in (cfg.r0, shifted):
        ref = regular_binning(cfg, r0, rule)
        rc, cell, start, ids = noalloc_binning(r0, boundary, n_bin, rule)
        assert rc == _abi.OK
        assert (cell == ref).all()                                   # integer work: exact
        assert (np.diff(start) == np.bincount(ref, minlength=ncell)).all()
        assert start[0] == 0 and start[-1] == cfg.n
        assert (ids == np.lexsort((np.arange(cfg.n), ref))).all()   # by cell, then id


def test_noalloc_binning_rejects_grids_beyond_its_capacity():
    cfg = configs.melt(seed=22, n_chain=4, n_mon=8)
    rc, _, _, _ = noalloc_binning(cfg.r0, [cfg.params.boundary[d] for d in range(3)], (64, 64, 64), 0)
    assert rc == _abi.ERR_CAPACITY
