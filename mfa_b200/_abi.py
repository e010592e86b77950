"""ctypes mirror of include/mfa_gpu.h and the loader of libmfa_gpu.so.

The shared library is built in-tree (``mfa_b200/libmfa_gpu.so``) by
``mfa_b200/csrc/Makefile``.  There is no fallback: if the library is missing
or cannot be loaded, importing the product API raises.
"""
from __future__ import annotations

import ctypes as C
import os

MAX_TYPES = 8
T2 = MAX_TYPES * MAX_TYPES

# status codes (mfa_status)
OK = 0
ERR_ARGS = 1
ERR_CUDA = 2
ERR_CELL_RANGE = 3
ERR_NEIGH_OVERFLOW = 4
ERR_NONFINITE = 5
ERR_TIMEOUT = 6
ERR_NOMEM = 7
ERR_STATE = 8
ERR_UNSUPPORTED = 9
ERR_CAPACITY = 10

FP64 = 0
MIXED = 1

Q_EWALD_REAL_IN_LJ = 0x1
Q_WALL_ENERGY_AW = 0x2

THERMO_DPD = 0
THERMO_LGV = 1
THERMO_NONE = 2

NOISE_GAUSS = 0
NOISE_UNIFORM = 1

R0, V, A, F, MIC = 0x01, 0x02, 0x04, 0x08, 0x10


class MfaParams(C.Structure):
    """struct mfa_params (field order and types must match the header)."""

    _fields_ = [
        ("n_part", C.c_int32), ("n_type", C.c_int32),
        ("n_mon", C.c_int32), ("n_chain", C.c_int32),
        ("n_mon_d", C.c_int32), ("n_chain_d", C.c_int32),
        ("symmetry", C.c_int32), ("thermostat", C.c_int32), ("dpd_weight", C.c_int32),
        ("wall", C.c_int32), ("charged", C.c_int32), ("bending", C.c_int32),
        ("force_switch_on", C.c_int32), ("pin_heads", C.c_int32), ("quirks", C.c_int32),
        ("noise", C.c_int32),
        ("boundary", C.c_double * 3),
        ("n_bin", C.c_int32 * 3), ("delta_bin", C.c_int32 * 3), ("pad0", C.c_int32),
        ("range_2", C.c_double * T2), ("epsil", C.c_double * T2), ("sigma_2", C.c_double * T2),
        ("e_shift", C.c_double * T2), ("inv_range_2", C.c_double * T2),
        ("skin", C.c_double), ("skin_2", C.c_double),
        ("dt", C.c_double), ("temp", C.c_double), ("friction", C.c_double), ("sig", C.c_double),
        ("k_chain", C.c_double), ("k_ring", C.c_double), ("r_chain_2", C.c_double),
        ("inv_r_chain_2", C.c_double), ("fene_clamp", C.c_double),
        ("k_bend", C.c_double), ("alpha_eq", C.c_double),
        ("a_wall", C.c_double * MAX_TYPES), ("sigma_wall", C.c_double * MAX_TYPES),
        ("a_w", C.c_double), ("z_space_wall", C.c_double), ("z_head", C.c_double),
        ("wall_cut", C.c_double), ("va_spring_twall", C.c_double * 3),
        ("r_2_min_init", C.c_double), ("r_2_min_time", C.c_double), ("s_time", C.c_int64),
        ("alpha_c", C.c_double), ("sqrt_alpha", C.c_double), ("inv_sqrt_pi", C.c_double),
        ("pi", C.c_double), ("ewald_rc_2", C.c_double),
        ("n_kmax", C.c_int32), ("pad1", C.c_int32),
        ("seed", C.c_uint64),
    ]

    def copy(self) -> "MfaParams":
        out = MfaParams()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(MfaParams))
        return out


class MfaScalars(C.Structure):
    """struct mfa_scalars."""

    _fields_ = [
        ("v_fluid_fluid", C.c_double), ("v_fluid_wall", C.c_double),
        ("v_intra_molec", C.c_double), ("v_bend", C.c_double), ("v_coul", C.c_double),
        ("t_fluid", C.c_double), ("v_total", C.c_double), ("e_total", C.c_double),
        ("virial", C.c_double), ("i_time", C.c_int64),
        ("f_skin", C.c_int32), ("n_rebuilds", C.c_int32), ("max_neigh", C.c_int32),
        ("max_cell", C.c_int32), ("fene_clamped", C.c_int32), ("error_bits", C.c_int32),
        ("kernel_launches", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class MfaObservables(C.Structure):
    """struct mfa_observables."""

    _fields_ = [("r_g2_brush", C.c_double * 3), ("r_g2_melt", C.c_double * 3), ("momentum", C.c_double * 3)]


# every entry point declared in include/mfa_gpu.h: name -> (restype, argtypes)
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)
SIGNATURES = {
    "mfa_init": (C.c_int, [C.POINTER(MfaParams), C.c_int, C.c_int, _DP, _DP, _DP, _IP, _DP, _DP, _IP,
                           C.POINTER(_P)]),
    "mfa_finalize": (C.c_int, [_P]),
    "mfa_abi_version": (C.c_int, []),
    "mfa_abi_sizes": (C.c_int, [_IP, _IP]),
    "mfa_status_string": (C.c_char_p, [C.c_int]),
    "mfa_set_step": (C.c_int, [_P, C.c_int64]),
    "mfa_verlet_positions": (C.c_int, [_P]),
    "mfa_check_skin": (C.c_int, [_P, _IP]),
    "mfa_binning": (C.c_int, [_P]),
    "mfa_my_binning": (C.c_int, [_P]),
    "mfa_zero_forces": (C.c_int, [_P]),
    "mfa_fluid_fluid": (C.c_int, [_P]),
    "mfa_pair_forces": (C.c_int, [_P]),
    "mfa_forces": (C.c_int, [_P]),
    "mfa_fluid_wall": (C.c_int, [_P, C.c_int32]),
    "mfa_intra_molec": (C.c_int, [_P]),
    "mfa_bending": (C.c_int, [_P, C.c_int32]),
    "mfa_ewald_k": (C.c_int, [_P, C.c_int32]),
    "mfa_dipolar_correction": (C.c_int, [_P]),
    "mfa_verlet_velocities": (C.c_int, [_P]),
    "mfa_external_force": (C.c_int, [_P, C.c_int32, C.c_double]),
    "mfa_orientation": (C.c_int, [_P, C.c_int32, C.c_double, C.c_double, _DP]),
    "mfa_set_dpd_vv": (C.c_int, [_P, C.c_int32]),
    "mfa_new_dpd_fd": (C.c_int, [_P]),
    "mfa_step": (C.c_int, [_P, C.c_int32]),
    "mfa_set_energy_log": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "mfa_read_energy_log": (C.c_int, [_P, _DP, C.c_int32, _IP]),
    "mfa_fetch_energy_log": (C.c_int, [_P, _DP, C.c_int32, C.c_int32]),
    "mfa_get_scalars": (C.c_int, [_P, C.POINTER(MfaScalars)]),
    "mfa_observe": (C.c_int, [_P, C.POINTER(MfaObservables)]),
    "mfa_observe_ends": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mfa_histogram_z": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "mfa_download": (C.c_int, [_P, C.c_uint32, _DP, _DP, _DP, _DP, _IP]),
    "mfa_upload": (C.c_int, [_P, C.c_uint32, _DP, _DP, _DP, _DP, _IP]),
    "mfa_sync": (C.c_int, [_P]),
    "mfa_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "mfa_set_pair_queue": (C.c_int, [_P, C.c_int32]),
    "mfa_set_pair_split": (C.c_int, [_P, C.c_int32]),
    "mfa_get_pair_split": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "mfa_set_pair_shape": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    "mfa_set_cells": (C.c_int, [_P, _IP, C.c_double]),
    "mfa_bin_cells_noalloc": (C.c_int, [C.c_void_p, C.c_int32, _DP, _IP, C.c_int32, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]),
    "mfa_debug_lists": (C.c_int, [_P, _IP, _IP, _IP, C.c_int32]),
    "mfa_debug_kvecs": (C.c_int, [_P, _IP, _DP, C.c_int32]),
    "mfa_batch_create": (C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(_P)]),
    "mfa_batch_step": (C.c_int, [_P, C.c_int32]),
    "mfa_batch_sync": (C.c_int, [_P]),
    "mfa_batch_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "mfa_batch_launches": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "mfa_batch_destroy": (C.c_int, [_P]),
    "mfa_trajectory_observable": (C.c_int, [_P, C.c_int32, _DP]),
    "mfa_adjoint": (C.c_int, [_P, C.c_int32, C.c_int32, _DP]),
}

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmfa_gpu.so")
_lib = None


class MfaError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = load().mfa_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{where}: status {status} ({msg})")


def load() -> C.CDLL:
    """Load libmfa_gpu.so (raises if it is absent: there is no CPU fallback)."""
    global _lib
    if _lib is None:
        # MFA_LIB: another build of the same library (same ABI), e.g. one made
        # with different compile-time options
        path = os.environ.get("MFA_LIB", LIB_PATH)
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing; build it with `make -C mfa_b200/csrc`")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.mfa_abi_version() != 1:
            raise ImportError("libmfa_gpu.so ABI version mismatch")
        _lib = lib
    return _lib


def check(status: int, where: str) -> None:
    if status != OK:
        raise MfaError(status, where)
