"""The oracle pinned to numbers the reference itself produced.

The reference ships the restart file (conf_new) and the energy logs (fort.60,
fort.41) of one of its own runs: SYSTEM 4 of control_simulation.h, one chain of 102
beads in a periodic 70 x 90 x 90 box, WCA (SOLVENT 1) and FENE (k = 30,
R0 = 1.5), written at step 10000.  tests/golden/make_reference_system4.py
copied them here.  fort.60 prints V/N, (V + KE)/N and KE/N at that step
(verlet_velocities.f90:223) with five significant digits, V = v_fluid_fluid +
v_intra_molec (:187; no walls in a bulk box, bending and the external field are
not part of it); fort.41 prints v_fluid_fluid and v_intra_molec themselves
with five decimals (observation.f90:304-307).  The potential energy does not
depend on the Langevin noise of the run, so the oracle evaluated on conf_new's
positions must reproduce each printed term and V/N, and conf_new's
velocities the printed KE/N.

conf_new keeps 7 decimals of each coordinate; the tolerance is half a unit of
the last printed digit plus the largest change those rounded digits can make
to the term (sum of |dV/dx| over all coordinates times 5e-8, with the oracle's
force of that term alone).  The CUDA path is then compared with the oracle on the same
configuration (FP64 to 1e-12; mixed to 1e-3: the chain of the shipped run has
beads as close as 0.3 sigma, where the 1e-5 relative FP32 position difference
is amplified twelvefold by r^-12) and with fort.60 directly.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from mfa_b200 import _abi
from mfa_b200.checkpoint import read_conf
from mfa_b200.params import Spec, derive

GOLDEN = os.path.join(ROOT, "tests", "golden")
FIX = json.load(open(os.path.join(GOLDEN, "reference_system4.json")))
ROW = FIX["fort60"][str(FIX["conf_step"])]
TERMS = FIX["fort41"][str(FIX["conf_step"])]
N = FIX["n_part"]


def reference_params(thermostat=_abi.THERMO_NONE):
    """The derived constants of the shipped run (init_params.f90:395-845 for
    SYSTEM 4, SOLVENT 1, PARTICLE_4 with inter4 = 1: every pair WCA;
    make_binning_boxes.f90:49-54: 3 cells along y and z).  The thermostat is
    off by default: the energies checked here do not depend on it."""
    spec = Spec(n_part=N, boundary=FIX["box"], n_type=4, n_mon=FIX["n_mon"], n_chain=FIX["n_chain"],
                symmetry=1, thermostat=thermostat, eps=np.array(FIX["eps"]), sigma_ii=FIX["sigma"],
                dt=FIX["dt"], temp=FIX["temp"], friction=FIX["friction"][0],
                k_chain_in=FIX["k_chain"], r_chain=FIX["r_chain"], n_bin=FIX["n_bin"])
    return derive(spec)


def reference_state():
    return read_conf(os.path.join(GOLDEN, "reference_conf_new"), N, dt=FIX["dt"])


def oracle_energies():
    from oracle import Oracle
    st = reference_state()
    p = reference_params()
    o = Oracle(p, st["r0"], st["v"], st["a_type"], np.ones(N))
    o.init_forces()
    s = o.scalars()
    f = o.state()["force"]
    return s, f, st


def rounding_bound(force):
    """Largest change of V/N that 7-decimal rounding of the positions can make."""
    return float(np.abs(force).sum()) * 5e-8 / N


def term_forces():
    """The oracle's force of fluid_fluid alone and of intra_molec alone."""
    from oracle import Oracle
    st = reference_state()
    o = Oracle(reference_params(), st["r0"], st["v"], st["a_type"], np.ones(N))
    o.binning()
    out = {}
    for name, call in (("v_fluid_fluid", o.fluid_fluid), ("v_intra_molec", o.intra_molec)):
        o.zero_forces()
        call()
        out[name] = o.state()["force"]
    return out


def test_read_conf_parses_the_reference_restart_file():
    st = reference_state()
    assert (st["n_mon"], st["n_chain"], st["n_mon_d"], st["n_chain_d"]) == (102, 1, 11, 0)
    assert st["n_cell_w"] == (70, 90) and st["n_order"] == 2
    assert (st["a_type"] == 1).all()
    assert st["r0"][0].tolist() == [0.2, 45.0, 45.0]            # first record, i3,3f13.7
    assert st["r0"][1].tolist() == [0.7876744, 45.0, 43.615078]
    assert (st["r0"][:, 1] == 45.0).all()                        # RUN_2D: y held at Ly/2
    assert np.isfinite(st["v"]).all() and np.isfinite(st["a"]).all()
    assert "walls" in st and st["walls"]["pbc_twall"].tolist() == [0, 0, 0]


def test_oracle_potential_energy_matches_the_reference_log():
    s, f, _ = oracle_energies()
    v_per_n = (s["v_fluid_fluid"] + s["v_intra_molec"]) / N
    tol = 0.05 + rounding_bound(f)
    assert tol < 0.2
    assert abs(v_per_n - ROW["v_per_n"]) <= tol, (v_per_n, ROW["text"])
    # both terms matter: neither alone is near the logged value
    assert abs(s["v_fluid_fluid"] / N - ROW["v_per_n"]) > 50
    assert abs(s["v_intra_molec"] / N - ROW["v_per_n"]) > 50
    # the O(N^2) check of util.f90:283-322 agrees with the list energy
    from oracle import Oracle
    st = reference_state()
    o = Oracle(reference_params(), st["r0"], st["v"], st["a_type"], np.ones(N))
    o.init_forces()
    assert abs(o.check_fluid_fluid() - s["v_fluid_fluid"]) <= 1e-12 * abs(s["v_fluid_fluid"])


def test_oracle_energy_terms_match_the_reference_observation_log():
    """Each term on its own, to its 5 printed decimals plus the rounding of
    conf_new's positions (about 3e-6 of the LJ term)."""
    s, _, _ = oracle_energies()
    forces = term_forces()
    for k in ("v_fluid_fluid", "v_intra_molec"):
        tol = 5e-6 + float(np.abs(forces[k]).sum()) * 5e-8
        assert tol < 1e-5 * abs(TERMS[k])
        assert abs(s[k] - TERMS[k]) <= tol, (k, s[k], TERMS["text"], tol)
    assert TERMS["v_fluid_wall"] == 0.0


def test_kinetic_energy_of_the_restart_velocities_matches_the_reference_log():
    st = reference_state()
    ke_per_n = 0.5 * float((st["v"] ** 2).sum()) / N          # mass 1 for every type
    assert abs(ke_per_n - ROW["t_per_n"]) <= 0.05 + 1e-6, (ke_per_n, ROW["text"])
    s, f, _ = oracle_energies()
    e_per_n = (s["v_fluid_fluid"] + s["v_intra_molec"]) / N + ke_per_n
    assert abs(e_per_n - ROW["e_per_n"]) <= 0.1 + rounding_bound(f), (e_per_n, ROW["text"])


def test_fene_clamp_is_exercised_by_the_reference_configuration():
    """Several bonds of the shipped configuration sit beyond the 0.98 R0^2
    clamp (intra_molec.f90:44), so the pin covers the clamped branch too."""
    st = reference_state()
    r = st["r0"]
    L = np.array(FIX["box"])
    d = r[:-1] - r[1:]
    d -= L * np.trunc(2.0 * d / L)
    x = (d * d).sum(1) / FIX["r_chain"] ** 2
    assert (x > float(np.float32(0.98))).sum() >= 1


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [_abi.FP64, _abi.MIXED])
def test_gpu_energies_on_the_reference_configuration(prec):
    from mfa_b200.api import System
    s_o, f_o, st = oracle_energies()
    g = System(reference_params(), st["r0"], st["v"], st["a_type"], np.ones(N), precision=prec)
    g.init_forces()
    s = g.scalars()
    f = g.download(_abi.F)["force"]
    g.close()
    tol = 1e-12 if prec == _abi.FP64 else 1e-3
    for k in ("v_fluid_fluid", "v_intra_molec"):
        assert abs(s[k] - s_o[k]) <= tol * abs(s_o[k]), (k, s[k], s_o[k])
    assert float(np.abs(f - f_o).max()) <= tol * float(np.abs(f_o).max())
    v_per_n = (s["v_fluid_fluid"] + s["v_intra_molec"]) / N
    if prec == _abi.FP64:
        assert abs(v_per_n - ROW["v_per_n"]) <= 0.05 + rounding_bound(f_o), (v_per_n, ROW["text"])
        forces = term_forces()
        for k in ("v_fluid_fluid", "v_intra_molec"):
            assert abs(s[k] - TERMS[k]) <= 5e-6 + float(np.abs(forces[k]).sum()) * 5e-8, (k, s[k])
