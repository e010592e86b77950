"""The physical parameters mfa_adjoint differentiates with respect to, and how
each one scales the derived constants of ``mfa_params``.

A gradient entry is dJ/d(parameter) at the parameter's base value.  Scaling a
parameter by f changes the derived constants the way init_params.f90 derives
them from the raw inputs: epsilon enters ``epsil`` (4 epsilon, :467-472); sigma
enters ``sigma_2``, the cutoff ``range_2`` and its inverse (:467-472, :502,
:789); k_FENE and R0 enter ``k_chain`` = k R0^2 and ``inv_r_chain_2``
(:396-398); the DPD friction enters ``friction`` and the noise amplitude
``sig`` = sqrt(2 kT gamma / dt) (:845); the wall strength enters ``a_wall`` and
``a_w`` (:582-585).  Central differences of a trajectory observable over these
copies are the check of the adjoint.
"""
from __future__ import annotations

import math

from ._abi import MAX_TYPES

NAMES = ("eps_lj", "sigma", "k_fene", "r0", "gamma_dpd", "eps_wall")


def _active(p):
    return [k for k in range(MAX_TYPES * MAX_TYPES) if p.range_2[k] > 0.0]


def perturbed(params, name, f):
    """A copy of the derived parameters with one physical parameter scaled by f."""
    p = params.copy()
    act = _active(p)
    if name == "eps_lj":
        for k in act:
            p.epsil[k] *= f
    elif name == "sigma":
        for k in act:
            p.sigma_2[k] *= f * f
            p.range_2[k] *= f * f
            p.inv_range_2[k] /= f * f
    elif name == "k_fene":
        p.k_chain *= f
    elif name == "r0":
        p.r_chain_2 *= f * f
        p.inv_r_chain_2 /= f * f
        p.k_chain *= f * f
    elif name == "gamma_dpd":
        p.friction *= f
        p.sig *= math.sqrt(f)
    elif name == "eps_wall":
        for t in range(MAX_TYPES):
            p.a_wall[t] *= f
        p.a_w *= f
    else:
        raise KeyError(name)
    return p


def base_values(p):
    """The base value of every parameter in NAMES (what f = 1 stands for)."""
    act = _active(p)
    return {"eps_lj": max(p.epsil[k] for k in act) / 4.0, "sigma": max(math.sqrt(p.sigma_2[k]) for k in act),
            "k_fene": p.k_chain * p.inv_r_chain_2, "r0": math.sqrt(p.r_chain_2), "gamma_dpd": p.friction,
            "eps_wall": max(p.a_wall[t] for t in range(MAX_TYPES))}
