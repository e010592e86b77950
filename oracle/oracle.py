"""TEST INFRASTRUCTURE: ctypes binding of the oracle (oracle/liboracle.so).

The oracle is the CPU FP64 restatement of the reference's per-step routines
(see mfa_oracle.h).  Only the tests, the smoke check and the CPU-baseline leg
of the benchmark use it, as the checker; the product never imports it.
Parity: unpinned by reference data (no Fortran compiler, no golden vectors in
the reference for this path).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> str:
    subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        import sys
        sys.path.insert(0, os.path.dirname(HERE))
        from mfa_b200._abi import MfaParams, MfaScalars  # struct layout only
        lib = C.CDLL(LIB)
        P, DP, IP = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
        sig = {
            "orc_create": (C.c_int, [C.POINTER(MfaParams), DP, DP, DP, IP, DP, DP, IP, C.c_int, C.c_int,
                                     C.c_int, C.POINTER(P)]),
            "orc_destroy": (None, [P]),
            "orc_set_step": (None, [P, C.c_int64]),
            "orc_get_step": (C.c_int64, [P]),
            "orc_verlet_positions": (None, [P]),
            "orc_check_skin": (C.c_int, [P]),
            "orc_binning": (C.c_int, [P]),
            "orc_my_binning": (C.c_int, [P]),
            "orc_zero_forces": (None, [P]),
            "orc_fluid_fluid": (None, [P]),
            "orc_fluid_wall": (None, [P, C.c_int]),
            "orc_intra_molec": (None, [P]),
            "orc_bending": (None, [P, C.c_int]),
            "orc_ewald_k": (C.c_int, [P, C.c_int]),
            "orc_dipolar_correction": (None, [P]),
            "orc_verlet_velocities": (None, [P]),
            "orc_external_force": (None, [P, C.c_int, C.c_double]),
            "orc_orientation": (C.c_double, [P, C.c_int, C.c_double, C.c_double]),
            "orc_set_dpd_vv": (None, [P, C.c_int]),
            "orc_new_dpd_fd": (None, [P]),
            "orc_md_step": (C.c_int, [P]),
            "orc_check_fluid_fluid": (C.c_double, [P]),
            "orc_get_state": (None, [P, DP, DP, DP, DP, IP]),
            "orc_set_state": (None, [P, DP, DP, DP, DP, IP]),
            "orc_get_scalars": (None, [P, C.POINTER(MfaScalars)]),
            "orc_get_lists": (None, [P, IP, IP, IP]),
            "orc_get_kvecs": (C.c_int, [P, DP, C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


class Oracle:
    """The reference's per-step routines on the CPU, same names as mfa_b200.System."""

    def __init__(self, params, r0, v, a_type, mass, q=None, a=None, mic=None,
                 bin_cap: int = 300, list_cap: int = 256, rng_mode: int = 0, bin_type: int = 0):
        self.lib = load()
        self.bin_type = bin_type      # BIN_TYPE: 0 binning, 1 my_binning
        self.params = params
        self.n = int(params.n_part)
        self._keep = [np.ascontiguousarray(x, dtype=dt).reshape(shape) if x is not None else None
                      for x, dt, shape in ((r0, np.float64, (self.n, 3)), (v, np.float64, (self.n, 3)),
                                           (a, np.float64, (self.n, 3)), (a_type, np.int32, (self.n,)),
                                           (mass, np.float64, (self.n,)), (q, np.float64, (self.n,)),
                                           (mic, np.int32, (self.n, 3)))]
        r0, v, a, t, m, qq, mc = self._keep
        self.mass = m
        self.bin_cap, self.list_cap = bin_cap, list_cap
        ptr = C.c_void_p()
        rc = self.lib.orc_create(C.byref(params), _dp(r0), _dp(v), _dp(a), _ip(t), _dp(m), _dp(qq),
                                 _ip(mc), bin_cap, list_cap, rng_mode, C.byref(ptr))
        if rc != 0:
            raise RuntimeError(f"orc_create failed: {rc}")
        self.ptr = ptr
        self.ncell = int(params.n_bin[0] * params.n_bin[1] * params.n_bin[2])

    def __del__(self):
        if getattr(self, "ptr", None):
            self.lib.orc_destroy(self.ptr)
            self.ptr = None

    def set_step(self, t):
        self.lib.orc_set_step(self.ptr, int(t))

    def verlet_positions(self):
        self.lib.orc_verlet_positions(self.ptr)

    def check_skin(self):
        return int(self.lib.orc_check_skin(self.ptr))

    def binning(self):
        rc = self.lib.orc_binning(self.ptr)
        if rc:
            raise RuntimeError(f"orc_binning: {rc}")

    def my_binning(self):
        rc = self.lib.orc_my_binning(self.ptr)
        if rc:
            raise RuntimeError(f"orc_my_binning: {rc}")

    def zero_forces(self):
        self.lib.orc_zero_forces(self.ptr)

    def fluid_fluid(self):
        self.lib.orc_fluid_fluid(self.ptr)

    def fluid_wall(self, t):
        self.lib.orc_fluid_wall(self.ptr, int(t))

    def intra_molec(self):
        self.lib.orc_intra_molec(self.ptr)

    def bending(self, mode):
        self.lib.orc_bending(self.ptr, int(mode))

    def ewald_k(self, mode):
        rc = self.lib.orc_ewald_k(self.ptr, int(mode))
        if rc:
            raise RuntimeError(f"orc_ewald_k: {rc}")

    def dipolar_correction(self):
        self.lib.orc_dipolar_correction(self.ptr)

    def verlet_velocities(self):
        self.lib.orc_verlet_velocities(self.ptr)

    def external_force(self, mode, k_elastic):
        self.lib.orc_external_force(self.ptr, int(mode), float(k_elastic))

    def orientation(self, mode, k_or, alpha_or=0.0):
        """Adds the orientation forces; returns v_or."""
        return float(self.lib.orc_orientation(self.ptr, int(mode), float(k_or), float(alpha_or)))

    def set_dpd_vv(self, on=True):
        self.lib.orc_set_dpd_vv(self.ptr, int(bool(on)))

    def new_dpd_fd(self):
        self.lib.orc_new_dpd_fd(self.ptr)

    def init_forces(self):
        p = self.params
        if p.charged:
            self.ewald_k(0)
        if self.bin_type == 1:
            self.my_binning()
        else:
            self.binning()
        self.zero_forces()
        self.fluid_fluid()
        if p.symmetry == 0 and p.wall in (2, 3, 4):
            self.fluid_wall(p.wall)
        self.intra_molec()
        st = self.state()
        self.set_state(a=st["force"] / self.mass[:, None])

    def md_step(self):
        rc = self.lib.orc_md_step(self.ptr)
        if rc:
            raise RuntimeError(f"orc_md_step: {rc}")

    def check_fluid_fluid(self):
        return float(self.lib.orc_check_fluid_fluid(self.ptr))

    def state(self):
        n = self.n
        out = {k: np.empty((n, 3)) for k in ("r0", "v", "a", "force")}
        out["mic"] = np.empty((n, 3), dtype=np.int32)
        self.lib.orc_get_state(self.ptr, _dp(out["r0"]), _dp(out["v"]), _dp(out["a"]),
                               _dp(out["force"]), _ip(out["mic"]))
        return out

    def set_state(self, r0=None, v=None, a=None, force=None, mic=None):
        conv = [None if x is None else np.ascontiguousarray(x, dtype=dt).reshape(self.n, 3)
                for x, dt in ((r0, np.float64), (v, np.float64), (a, np.float64), (force, np.float64),
                              (mic, np.int32))]
        self.lib.orc_set_state(self.ptr, _dp(conv[0]), _dp(conv[1]), _dp(conv[2]), _dp(conv[3]),
                               _ip(conv[4]))

    def scalars(self):
        from mfa_b200._abi import MfaScalars
        s = MfaScalars()
        self.lib.orc_get_scalars(self.ptr, C.byref(s))
        return s.as_dict()

    def lists(self):
        cell = np.empty(self.n, dtype=np.int32)
        bf = np.empty(self.ncell * (self.bin_cap + 1), dtype=np.int32)
        ff = np.empty(self.n * (self.list_cap + 1), dtype=np.int32)
        self.lib.orc_get_lists(self.ptr, _ip(cell), _ip(bf), _ip(ff))
        return cell, bf.reshape(self.bin_cap + 1, self.ncell), ff.reshape(self.n, self.list_cap + 1)

    def kvecs(self, max_k=100000):
        out = np.empty((max_k, 3))
        nk = self.lib.orc_get_kvecs(self.ptr, _dp(out), max_k)
        return out[:nk].copy()


def pair_multiset_half(ff_list: np.ndarray) -> np.ndarray:
    """Unordered pairs of the reference's half list (ff_list(0:cap, n), 1-based)."""
    rows = []
    for i in range(ff_list.shape[0]):
        c = ff_list[i, 0]
        for j in ff_list[i, 1:c + 1]:
            a, b = (i + 1, int(j)) if i + 1 < j else (int(j), i + 1)
            rows.append((a, b))
    arr = np.array(rows, dtype=np.int64).reshape(-1, 2)
    return arr[np.lexsort((arr[:, 1], arr[:, 0]))]


def pair_multiset_rows(counts: np.ndarray, nbr: np.ndarray) -> np.ndarray:
    """Unordered pairs of every entry of a list given as (counts, nbr), ids
    1-based: one (min, max) row per entry, repeats kept."""
    n = counts.shape[0]
    ii = np.repeat(np.arange(1, n + 1), counts)
    mask = np.arange(nbr.shape[1])[None, :] < counts[:, None]
    jj = nbr[mask]
    arr = np.stack([np.minimum(ii, jj), np.maximum(ii, jj)], axis=1).astype(np.int64)
    return arr[np.lexsort((arr[:, 1], arr[:, 0]))]


def pair_multiset_full(counts: np.ndarray, nbr: np.ndarray) -> np.ndarray:
    """Unordered pairs of a full list (each pair in both rows); keeps i < j entries."""
    n = counts.shape[0]
    ii = np.repeat(np.arange(1, n + 1), counts)
    mask = np.arange(nbr.shape[1])[None, :] < counts[:, None]
    jj = nbr[mask]
    keep = ii < jj
    arr = np.stack([ii[keep], jj[keep]], axis=1).astype(np.int64)
    return arr[np.lexsort((arr[:, 1], arr[:, 0]))]


def derive_params(n_type, eps, sigma_ii, k_chain_in, r_chain, dt, temp, friction, k_bend, alpha_eq,
                  a_w, sigma_w, boundary, skin, brush_heads=False, wall93=False, binning_rule=0,
                  n_bin_in=(1, 1, 1), n_bin_init=None):
    """The oracle's own restatement of the init-time derived constants."""
    from mfa_b200._abi import MfaParams, MAX_TYPES

    class Inputs(C.Structure):
        _fields_ = [("n_type", C.c_int32), ("eps", C.c_double * (MAX_TYPES * MAX_TYPES)),
                    ("sigma_ii", C.c_double * MAX_TYPES),
                    ("k_chain_in", C.c_double), ("r_chain", C.c_double), ("dt", C.c_double),
                    ("temp", C.c_double), ("friction", C.c_double), ("k_bend", C.c_double),
                    ("alpha_eq", C.c_double), ("a_w", C.c_double), ("sigma_w", C.c_double),
                    ("boundary", C.c_double * 3), ("skin", C.c_double),
                    ("brush_heads", C.c_int32), ("wall93", C.c_int32), ("binning_rule", C.c_int32),
                    ("n_bin_in", C.c_int32 * 3), ("n_bin_init", C.c_int32 * 3)]

    lib = load()
    lib.orc_derive_params.restype = None
    lib.orc_derive_params.argtypes = [C.POINTER(Inputs), C.POINTER(MfaParams)]
    inp = Inputs()
    inp.n_type = n_type
    e = np.asarray(eps, dtype=np.float64)
    for i in range(n_type):
        inp.sigma_ii[i] = sigma_ii[i]
        for j in range(n_type):
            inp.eps[i * MAX_TYPES + j] = e[i, j]
    inp.k_chain_in, inp.r_chain, inp.dt, inp.temp, inp.friction = k_chain_in, r_chain, dt, temp, friction
    inp.k_bend, inp.alpha_eq, inp.a_w, inp.sigma_w, inp.skin = k_bend, alpha_eq, a_w, sigma_w, skin
    for d in range(3):
        inp.boundary[d] = boundary[d]
        inp.n_bin_in[d] = n_bin_in[d]
    inp.brush_heads, inp.wall93, inp.binning_rule = int(brush_heads), int(wall93), binning_rule
    out = MfaParams()
    nbi = n_bin_init
    if nbi is None:
        # delta_bin from the final n_bin when no separate initial value is given
        tmp = MfaParams()
        for d in range(3):
            inp.n_bin_init[d] = 3
        lib.orc_derive_params(C.byref(inp), C.byref(tmp))
        nbi = [tmp.n_bin[d] for d in range(3)]
    for d in range(3):
        inp.n_bin_init[d] = nbi[d]
    lib.orc_derive_params(C.byref(inp), C.byref(out))
    return out
