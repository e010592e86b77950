"""Observables on the device (mfa_observe, mfa_histogram_z) against the numpy
restatement in oracle/observables.py, and that restatement against closed
forms."""
import numpy as np
import pytest

import observables as ob
from mfa_b200 import _abi
from mfa_b200._abi import FP64


def test_refold_and_rg_of_a_straight_chain_across_the_box():
    """A straight chain of 8 beads (spacing 1) wrapped into a box of 5: the
    refold restores it, and its Rg^2 along the chain is (N^2 - 1)/12."""
    n = 8
    r = np.array([[0.5 + k, 2.0, 2.0] for k in range(n)])
    r[:, 0] %= 5.0
    s = ob.refold(r, [5.0, 5.0, 5.0], n, 1, 0, 0, symmetry=0)
    np.testing.assert_allclose(s[:, 0], 0.5 + np.arange(n))
    rg = ob.radii_of_gyration(s, n, 1, 0, 0)
    np.testing.assert_allclose(rg[0], [(n * n - 1) / 12.0, 0.0, 0.0], atol=1e-14)
    assert np.isnan(rg[1]).all()          # no melt chains: the reference's 0/0
    # SYMMETRY 1 leaves the brush range folded (observation.f90:176-192)
    assert (ob.refold(r, [5.0, 5.0, 5.0], n, 1, 0, 0, symmetry=1) == r).all()


def test_melt_runs_follow_global_ids():
    """mod(i_part - 1, n_mon_d) uses the global id: with 3 brush beads and
    melt chains of 2, bead 3 (0-based) is refolded against the last brush
    bead and bead 4 starts a run."""
    r = np.zeros((7, 3))
    r[:, 0] = [1.0, 1.5, 2.0, 9.5, 9.0, 0.5, 3.0]
    s = ob.refold(r, [10.0, 10.0, 10.0], 3, 1, 2, 2, symmetry=1)
    np.testing.assert_allclose(s[:, 0], [1.0, 1.5, 2.0, -0.5, 9.0, 10.5, 3.0])


def test_z_histogram_bins():
    """int(z / z_step) + 1, clamped (functions.f90:168-172)."""
    r = np.zeros((5, 3))
    r[:, 2] = [0.1, 1.9, 2.0, 59.99, 60.0]
    h = ob.z_histogram(r, [10.0, 10.0, 60.0], 30, 5, 1, 0, 0)
    expect = np.zeros(30)
    expect[0], expect[1], expect[29] = 2, 1, 2
    np.testing.assert_array_equal(h[0], expect)
    assert h[1].sum() == 0


def _oracle_obs(cfg_params, st, mass):
    p = cfg_params
    s = ob.refold(st["r0"], p.boundary, p.n_mon, p.n_chain, p.n_mon_d, p.n_chain_d, p.symmetry)
    return ob.radii_of_gyration(s, p.n_mon, p.n_chain, p.n_mon_d, p.n_chain_d), ob.momentum(st["v"], mass)


@pytest.mark.gpu
def test_observe_brush(brush_small_cfg):
    from mfa_b200.api import System
    cfg = brush_small_cfg
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g.init_forces()
    g.step(50)
    o = g.observe()
    rg, mom = _oracle_obs(cfg.params, g.download(_abi.R0 | _abi.V), cfg.mass)
    np.testing.assert_allclose(o["r_g2_brush"], rg[0], rtol=1e-12)
    np.testing.assert_allclose(o["r_g2_melt"], rg[1], atol=1e-300)      # single-bead solvent: 0
    scale = float(np.abs(cfg.mass[:, None] * g.download(_abi.V)["v"]).sum())
    assert np.abs(o["momentum"] - mom).max() < 1e-12 * scale
    g.close()


@pytest.mark.gpu
def test_observe_melt_chains_in_both_ranges(melt_cfg):
    """Chains in the brush range (not refolded in SYMMETRY 1) and in the melt
    range (refolded): the initial state of the melt split in two."""
    from mfa_b200.api import System
    cfg = melt_cfg
    p = cfg.params.copy()
    half = p.n_chain // 2
    p.n_chain_d, p.n_mon_d, p.n_chain = p.n_chain - half, p.n_mon, half
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    o = g.observe()
    rg, mom = _oracle_obs(p, {"r0": cfg.r0, "v": cfg.v}, cfg.mass)
    np.testing.assert_allclose(o["r_g2_brush"], rg[0], rtol=1e-12)
    np.testing.assert_allclose(o["r_g2_melt"], rg[1], rtol=1e-12)
    assert rg[1].max() < 5.0 < rg[0].max()           # refolded melt chains are compact
    np.testing.assert_allclose(o["momentum"], mom, atol=1e-9)
    g.close()


@pytest.mark.gpu
def test_histogram_z_accumulates_exactly(brush_small_cfg):
    from mfa_b200.api import System
    cfg = brush_small_cfg
    p = cfg.params
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g.init_forces()
    h1, n1 = g.histogram_z(40, reset=True)
    r_a = g.download(_abi.R0)["r0"]
    g.step(30)
    h2, n2 = g.histogram_z(40)
    r_b = g.download(_abi.R0)["r0"]
    args = (p.boundary, 40, p.n_mon, p.n_chain, p.n_mon_d, p.n_chain_d)
    assert n1 == 1 and n2 == 2
    np.testing.assert_array_equal(h1, ob.z_histogram(r_a, *args))
    np.testing.assert_array_equal(h2, ob.z_histogram(r_a, *args) + ob.z_histogram(r_b, *args))
    z, dens = g.density_profiles(h2, n2)
    assert dens.shape == (2, 40) and z[0] == pytest.approx(p.boundary[2] / 80)
    h3, n3 = g.histogram_z(40, reset=True)
    assert n3 == 1 and (h3 == ob.z_histogram(r_b, *args)).all()
    g.close()


def test_end_to_end_of_straight_chains_closed_form():
    """Three straight chains of 4 beads along x (spacing 1): top, bottom and a
    melt chain; every end-to-end vector is (3, 0, 0)."""
    s = np.zeros((12, 3))
    for c in range(3):
        s[4 * c:4 * c + 4, 0] = np.arange(4.0)
    r_ee, r_ee2 = ob.end_to_end(s, 4, 2, 1)
    np.testing.assert_allclose(r_ee, [[3, 0, 0]] * 3)
    np.testing.assert_allclose(r_ee2, [[9, 0, 0]] * 3)
    # n_chain = 1: the brush groups divide by n_chain // 2 = 0 (the reference's 0/0)
    with np.errstate(invalid="ignore", divide="ignore"):
        r1, _ = ob.end_to_end(s[:4], 4, 1, 0)
    assert np.isnan(r1[0]).all() and np.isinf(r1[1][0])
    f = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0]])
    np.testing.assert_allclose(ob.head_forces(f, 3), [[-1, -2, -3], [-11, -13, -15]])


@pytest.mark.gpu
def test_observe_ends_brush_against_restatement_and_oracle_head_forces(brush_small_cfg):
    """End-to-end vectors of the brush (refolded chains) against the numpy
    restatement, and the head forces of the last step against the oracle's
    force on the heads at the same positions (every force term, before the
    pin of verlet_velocities.f90:113-145 zeroes it)."""
    from mfa_b200.api import System
    from oracle import Oracle
    cfg = brush_small_cfg
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g.init_forces(full=True)
    for _ in range(5):
        g.md_step()
    e = g.observe_ends()
    st = g.download(_abi.R0 | _abi.V | _abi.A | _abi.MIC)
    s = ob.refold(st["r0"], p.boundary, p.n_mon, p.n_chain, p.n_mon_d, p.n_chain_d, p.symmetry)
    r_ee, r_ee2 = ob.end_to_end(s, p.n_mon, p.n_chain, 0)
    np.testing.assert_allclose(e["r_ee"][:2], r_ee[:2], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(e["r_ee2"][:2], r_ee2[:2], rtol=1e-12)
    assert np.isnan(e["r_ee"][2]).all()              # solvent: single-bead "chains"
    o = Oracle(p, st["r0"], st["v"], cfg.a_type, cfg.mass, a=st["a"], mic=st["mic"])
    o.binning()
    o.zero_forces()
    o.fluid_fluid()
    o.fluid_wall(p.wall)
    o.intra_molec()
    o.bending(2)
    f = o.state()["force"][0:p.n_chain * p.n_mon:p.n_mon]
    ref = ob.head_forces(f, p.n_chain)
    assert np.abs(ref).max() > 0.0
    np.testing.assert_allclose(e["head_force"], ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())
    g.close()


@pytest.mark.gpu
def test_observe_ends_melt_chains(melt_cfg):
    from mfa_b200.api import System
    cfg = melt_cfg
    p = cfg.params.copy()
    half = p.n_chain // 2
    p.n_chain_d, p.n_mon_d, p.n_chain = p.n_chain - half, p.n_mon, half
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    e = g.observe_ends()
    s = ob.refold(cfg.r0, p.boundary, p.n_mon, p.n_chain, p.n_mon_d, p.n_chain_d, p.symmetry)
    r_ee, r_ee2 = ob.end_to_end(s, p.n_mon, p.n_chain, p.n_chain_d)
    np.testing.assert_allclose(e["r_ee"], r_ee, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(e["r_ee2"], r_ee2, rtol=1e-12)
    assert (e["head_force"] == 0.0).all()            # no pinned heads in a melt
    g.close()
