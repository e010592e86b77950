"""Derived run constants, as the reference's init routines compute them.

The reference reads raw inputs (mfa_input, system_input) and derives the
constants the hot path uses in init_params.f90:395-845, init_config.f90:217-246
and make_binning_boxes.f90:14-64.  A Fortran shim passes those module
variables straight into ``mfa_params``; in Python, :func:`derive` plays the role
of that init code.  Single-precision literals of the Fortran source (default
REAL constants such as ``2.**(1./6.)``, ``0.4``, ``2.2``, ``0.98`` and
``pi = 3.1415926536``) are evaluated in float32 and widened, as the compiled
reference does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import MAX_TYPES, MfaParams


def f32(x: float) -> float:
    """Value of a default-REAL (single precision) literal widened to double."""
    return float(np.float32(x))


# init_params.f90:502 -- 2.**(1./6.) evaluated in single precision
C_2_16 = float(np.float32(2.0) ** (np.float32(1.0) / np.float32(6.0)))
C_2_2 = f32(2.2)          # init_params.f90:516
PI_F32 = f32(3.1415926536)  # mfa_common.f90:332
SKIN_REF = f32(0.4)       # init_params.f90:800
BIN_SKIN = f32(0.4)       # make_binning_boxes.f90:43
FENE_CLAMP = f32(0.98)    # intra_molec.f90:44


@dataclass
class Spec:
    """Raw inputs of one system (what mfa_input/system_input/control_simulation.h hold)."""

    n_part: int
    boundary: Sequence[float]
    n_type: int = 1
    n_mon: int = 0
    n_chain: int = 0
    n_mon_d: int = 0
    n_chain_d: int = 0
    symmetry: int = 1
    thermostat: int = _abi.THERMO_DPD
    dpd_weight: int = 0
    wall: int = 0
    charged: int = 0
    bending: int = 0
    force_switch_on: int = 0
    pin_heads: int = 0
    quirks: int = _abi.Q_EWALD_REAL_IN_LJ | _abi.Q_WALL_ENERGY_AW
    noise: int = _abi.NOISE_GAUSS
    eps: Optional[np.ndarray] = None         # n_type x n_type, as read (before x4)
    sigma_ii: Optional[Sequence[float]] = None
    brush_heads: bool = False                # SYSTEM 0,1,3: type 1 = grafted heads
    wall93_zero_last_type: bool = False      # WALL 2 without PARTICLE_4: range_2(:,n_type)=0
    skin: float = SKIN_REF
    dt: float = 0.005
    temp: float = 1.0
    friction: float = 4.5
    k_chain_in: float = 30.0
    r_chain: float = 1.5
    k_ring: float = 0.0
    k_bend: float = 0.0
    alpha_eq: float = 0.0
    a_w: float = 1.0
    sigma_w: float = 1.0
    z_head: float = 1.0
    wall_cut: float = 0.0
    va: Sequence[float] = (0.0, 0.0, 0.0)
    r_2_min_time: float = 40.0
    s_time: int = 1
    alpha_c: float = 0.0
    n_kmax: int = 0
    ewald_rc: float = 0.0
    seed: int = 12345
    n_bin: Optional[Sequence[int]] = None        # None: int(L/(rc_max + 0.4))
    n_bin_init: Optional[Sequence[int]] = None   # values delta_bin is computed from
    extra: dict = field(default_factory=dict)


def derive(spec: Spec) -> MfaParams:
    """Build ``mfa_params`` from raw inputs (init_params.f90:395-845 and friends)."""
    n = spec.n_type
    if not 1 <= n <= MAX_TYPES:
        raise ValueError("n_type out of range")
    eps = np.ones((n, n)) if spec.eps is None else np.asarray(spec.eps, dtype=np.float64)
    sig_ii = np.ones(n) if spec.sigma_ii is None else np.asarray(spec.sigma_ii, dtype=np.float64)
    p = MfaParams()
    p.n_part = spec.n_part
    p.n_type = n
    p.n_mon, p.n_chain = spec.n_mon, spec.n_chain
    p.n_mon_d, p.n_chain_d = spec.n_mon_d, spec.n_chain_d
    p.symmetry, p.thermostat, p.dpd_weight = spec.symmetry, spec.thermostat, spec.dpd_weight
    p.wall, p.charged, p.bending = spec.wall, spec.charged, spec.bending
    p.force_switch_on, p.pin_heads, p.quirks, p.noise = (
        spec.force_switch_on, spec.pin_heads, spec.quirks, spec.noise)
    for d in range(3):
        p.boundary[d] = float(spec.boundary[d])
    # init_params.f90:408-413 additive mixing, :467-472 sigma_2 and epsilon x 4
    sigma = np.empty((n, n))
    for i in range(n):
        for j in range(n):
            sigma[i, j] = (sig_ii[i] + sig_ii[j]) / 2.0
        sigma[i, i] = sig_ii[i]
    rng2 = np.empty((n, n))
    for i in range(n):
        for j in range(n):
            p.sigma_2[i * MAX_TYPES + j] = sigma[i, j] * sigma[i, j]
            p.epsil[i * MAX_TYPES + j] = 4.0 * eps[i, j]
            x = C_2_16 * sigma[i, j]
            rng2[i, j] = x * x                               # :502
    if spec.brush_heads:
        x = C_2_2 * sigma[0, n - 1]
        rng2[0, n - 1] = x * x                               # :516-517
        x = C_2_2 * sigma[n - 1, 0]
        rng2[n - 1, 0] = x * x
    if spec.wall93_zero_last_type:
        rng2[:, n - 1] = 0.0                                 # :604-606
        rng2[n - 1, :] = 0.0
    if spec.brush_heads:
        rng2[0, 0] = 0.0                                     # :703-707
    for i in range(n):
        for j in range(n):
            r2 = rng2[i, j]
            p.range_2[i * MAX_TYPES + j] = r2
            if r2 > 0.0:
                rd = sigma[j, i] * sigma[j, i] / r2
                rd = (rd * rd) * rd                           # :717
                p.e_shift[i * MAX_TYPES + j] = rd * (rd - 1.0)
                p.inv_range_2[i * MAX_TYPES + j] = 1.0 / r2   # :789
    r_cut_max = math.sqrt(float(rng2.max()))                  # :766
    p.skin = spec.skin
    p.skin_2 = (r_cut_max + spec.skin) ** 2 - r_cut_max ** 2  # :807-808
    p.dt, p.temp, p.friction = spec.dt, spec.temp, spec.friction
    p.sig = math.sqrt(2.0 * spec.temp * spec.friction / spec.dt)   # :845
    p.r_chain_2 = spec.r_chain * spec.r_chain                       # :396-398
    p.inv_r_chain_2 = 1.0 / p.r_chain_2
    p.k_chain = spec.k_chain_in * p.r_chain_2
    p.k_ring = spec.k_ring
    p.fene_clamp = FENE_CLAMP
    p.k_bend, p.alpha_eq = spec.k_bend, spec.alpha_eq
    for t in range(n):                                              # :582-585
        p.sigma_wall[t] = (spec.sigma_w + sig_ii[t]) / 2.0
        p.a_wall[t] = spec.a_w
    p.a_w = spec.a_w
    p.z_space_wall = float(spec.boundary[2])
    p.z_head = spec.z_head
    p.wall_cut = spec.wall_cut
    for d in range(3):
        p.va_spring_twall[d] = spec.va[d]
    # make_binning_boxes.f90:14-46
    for d in range(3):
        if spec.n_bin is None:
            p.n_bin[d] = int(spec.boundary[d] / (r_cut_max + BIN_SKIN))
        else:
            p.n_bin[d] = int(spec.n_bin[d])
        nb0 = p.n_bin[d] if spec.n_bin_init is None else int(spec.n_bin_init[d])
        p.delta_bin[d] = 1 if nb0 >= 3 else (0 if nb0 == 2 else -1)
    # init_force_switch_on.f90:13-22
    p.r_2_min_init = (float(sig_ii.max()) / f32(0.9)) ** 2
    p.r_2_min_time = spec.r_2_min_time
    p.s_time = spec.s_time
    # init_config.f90:228-231 and ewald_k.f90
    p.pi = PI_F32
    p.inv_sqrt_pi = 1.0 / PI_F32
    p.alpha_c = spec.alpha_c
    p.sqrt_alpha = math.sqrt(spec.alpha_c) if spec.alpha_c > 0 else 0.0
    p.n_kmax = spec.n_kmax
    p.ewald_rc_2 = spec.ewald_rc * spec.ewald_rc
    p.seed = spec.seed
    return p


def list_cutoff(p: MfaParams) -> float:
    """Largest Verlet-list radius sqrt(max range_2 + skin_2)."""
    r2 = max(p.range_2[k] for k in range(MAX_TYPES * MAX_TYPES)) + p.skin_2
    if p.charged and not (p.quirks & _abi.Q_EWALD_REAL_IN_LJ):
        r2 = max(r2, (math.sqrt(p.ewald_rc_2) + p.skin) ** 2)
    return math.sqrt(r2)
