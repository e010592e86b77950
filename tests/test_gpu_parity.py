"""Parity of the CUDA path (through the C ABI) with the oracle.

Tolerances (max-norm relative error unless stated):
  FP64 path   forces 1e-12; trajectories over 100 steps 1e-10 (thermostat off
              and DPD with Philox noise); neighbour lists and cells bit-exact.
  MIXED path  forces 1e-4 (FP32 pair/bond math); positions after 100 steps
              2e-3 sigma absolute, energies 1e-4 (see the trajectory test).
"""
import math

import numpy as np
import pytest

from conftest import relerr
from mfa_b200 import _abi, configs
from mfa_b200._abi import FP64, MIXED, MfaError
from mfa_b200.api import System
from oracle import Oracle, pair_multiset_full, pair_multiset_half, pair_multiset_rows

pytestmark = pytest.mark.gpu

CFGS = ["melt_cfg", "brush_small_cfg", "charged_small_cfg", "charged_ref_cfg", "charged_slab_cfg"]


def pair(cfg, prec, params=None, list_cap=512):
    p = cfg.params if params is None else params
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, list_cap=list_cap)
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)
    return o, g


@pytest.mark.parametrize("name", CFGS)
def test_binning_bit_exact(name, request):
    cfg = request.getfixturevalue(name)
    o, g = pair(cfg, MIXED)
    o.binning()
    g.binning()
    cell_o, _, ff = o.lists()
    cell_g, cnt, nbr = g.debug_lists(512)
    assert (cell_o == cell_g).all()
    # both are half lists: every unordered pair once (the row that holds it
    # differs: the reference's shorter row, the lower cell slot here)
    ref = pair_multiset_half(ff)
    got = pair_multiset_rows(cnt, nbr)
    assert ref.shape == got.shape and (ref == got).all()
    g.close()


@pytest.mark.parametrize("name", ["melt_cfg", "charged_small_cfg"])
def test_my_binning_bit_exact(name, request):
    cfg = request.getfixturevalue(name)
    o, g = pair(cfg, FP64)
    o.my_binning()
    g.my_binning()
    cell_o, _, ff = o.lists()
    cell_g, cnt, nbr = g.debug_lists(512)
    assert (cell_o == cell_g).all()
    ref = pair_multiset_full(ff[:, 0], ff[:, 1:])
    got = pair_multiset_full(cnt, nbr)
    assert ref.shape == got.shape and (ref == got).all()
    g.close()


def test_binning_duplicate_cell_visits():
    """n_bin = 2 with delta_bin = 1 (make_binning_boxes.f90:14-37): pairs in
    the other cell are listed twice, as in the reference."""
    cfg = configs.melt(seed=5, n_chain=10, n_mon=8, density=0.5)
    p = cfg.params.copy()
    p.n_bin[:] = [2, 2, 2]
    p.delta_bin[:] = [1, 1, 1]
    o, g = pair(cfg, FP64, params=p)
    o.binning()
    g.binning()
    half = pair_multiset_half(o.lists()[2])
    cnt, nbr = g.debug_lists(512)[1:]
    got = pair_multiset_rows(cnt, nbr)
    assert half.shape == got.shape and (half == got).all()
    assert len({tuple(x) for x in half}) < half.shape[0]   # duplicates present
    g.close()


@pytest.mark.parametrize("name", CFGS)
@pytest.mark.parametrize("prec,tol", [(FP64, 1e-12), (MIXED, 1e-4)])
def test_initial_forces_and_energies(name, prec, tol, request):
    cfg = request.getfixturevalue(name)
    o, g = pair(cfg, prec)
    o.init_forces()
    g.init_forces()
    assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < tol
    so, sg = o.scalars(), g.scalars()
    for k in ("v_fluid_fluid", "v_fluid_wall", "v_intra_molec", "v_coul"):
        assert sg[k] == pytest.approx(so[k], rel=tol * 10, abs=tol * 10 * cfg.n), k
    g.close()


def run_both(o, g, nsteps):
    fo, fg = [], []
    for _ in range(nsteps):
        o.md_step()
        fg.append(g.md_step())
        fo.append(o.scalars()["f_skin"])
    return fo, fg


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg", "charged_small_cfg", "charged_slab_cfg"])
@pytest.mark.parametrize("thermo", [_abi.THERMO_NONE, _abi.THERMO_DPD])
def test_fp64_trajectory_100_steps(name, thermo, request):
    cfg = request.getfixturevalue(name)
    p = cfg.params.copy()
    p.thermostat = thermo
    o, g = pair(cfg, FP64, params=p)
    o.init_forces()
    g.init_forces()
    run_both(o, g, 100)
    so, sg = o.state(), g.download()
    assert relerr(sg["r0"], so["r0"]) < 1e-10
    assert relerr(sg["v"], so["v"]) < 1e-10
    assert (sg["mic"] == so["mic"]).all()
    eo, eg = o.scalars(), g.scalars()
    assert eg["e_total"] == pytest.approx(eo["e_total"], rel=1e-10)
    assert eg["n_rebuilds"] == eo["n_rebuilds"]
    g.close()


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg", "charged_small_cfg", "charged_slab_cfg"])
def test_mixed_trajectory_100_steps(name, request):
    cfg = request.getfixturevalue(name)
    o, g = pair(cfg, MIXED)
    o.init_forces()
    g.init_forces()
    run_both(o, g, 100)
    so, sg = o.state(), g.download()
    # FP32 force errors (~1e-5 relative) are amplified by the chaotic dynamics
    # of a freshly generated (hot) configuration; after 100 steps the positions
    # stay within 2e-3 sigma of the FP64 trajectory and the energy within 1e-4.
    assert np.abs(sg["r0"] - so["r0"]).max() < 2e-3
    assert g.scalars()["e_total"] == pytest.approx(o.scalars()["e_total"], rel=1e-4)
    g.close()


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg", "charged_small_cfg", "charged_slab_cfg"])
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_fast_path_equals_subroutine_path(name, prec, request):
    """mfa_step (fused kernels, captured graphs, device-side rebuild decision)
    computes the same physics as the per-subroutine path.  The two paths run
    different instantiations of the pair kernel (wall fused or not), and the
    pair kernel's reductions add into the force array in no fixed order, so
    after 57 steps they agree to rounding (FP64: 1e-12 sigma; MIXED: 1e-4
    sigma, FP32 differences amplified by the dynamics) rather than bit for bit."""
    cfg = request.getfixturevalue(name)
    g1 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)
    g2 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)
    g1.init_forces()
    g2.init_forces()
    for _ in range(57):
        g1.md_step()
    g2.step(57)
    e1, e2 = g1.scalars(), g2.scalars()       # raises on a device-side error
    s1, s2 = g1.download(), g2.download()
    dr = float(np.abs(s1["r0"] - s2["r0"]).max())
    dv = float(np.abs(s1["v"] - s2["v"]).max())
    tol = 1e-12 if prec == FP64 else 1e-4
    assert dr < tol and dv < 100 * tol, (dr, dv)
    assert (s1["mic"] == s2["mic"]).all()
    # energies are reduced over different block shapes when the wall is fused
    # into the pair kernel, so they agree to rounding rather than bit for bit
    assert e1["e_total"] == pytest.approx(e2["e_total"], rel=1e-11 if prec == FP64 else 1e-5)
    assert e1["i_time"] == e2["i_time"] == 57
    assert e1["n_rebuilds"] == e2["n_rebuilds"]
    g1.close()
    g2.close()


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg"])
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_runs_are_reproducible(name, prec, request):
    """Two runs of the fast path see the same noise (Philox keyed by step and
    pair) and the same lists; only the order in which the pair kernel's
    reductions add into the force array differs, so after 123 steps they agree
    to rounding amplified by the dynamics (FP64 1e-11 sigma, MIXED 1e-3 sigma)."""
    cfg = request.getfixturevalue(name)
    out = []
    for _ in range(2):
        g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)
        g.init_forces()
        g.step(123)
        s = g.scalars()
        out.append((g.download(), s))
        g.close()
    tol = 1e-11 if prec == FP64 else 1e-3
    assert float(np.abs(out[0][0]["r0"] - out[1][0]["r0"]).max()) < tol
    assert float(np.abs(out[0][0]["v"] - out[1][0]["v"]).max()) < 100 * tol
    assert out[0][1]["n_rebuilds"] == out[1][1]["n_rebuilds"]


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg", "charged_small_cfg"])
def test_regridding_keeps_the_forces(name, request):
    """mfa_set_cells (the autotuner's knob) changes cells and skin, not physics."""
    from mfa_b200.tune import cells_for
    cfg = request.getfixturevalue(name)
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=FP64)
    g.init_forces()
    f0 = g.download(_abi.F)["force"]
    for skin in (0.15, 0.55):
        g.set_cells(cells_for(g.params, skin), skin)
        assert g.check_skin() == 1
        g.init_forces()
        assert relerr(g.download(_abi.F)["force"], f0) < 1e-12
    g.close()


@pytest.mark.parametrize("name", ["charged_small_cfg", "charged_ref_cfg", "charged_slab_cfg"])
def test_ewald_kspace(name, request):
    cfg = request.getfixturevalue(name)
    o, g = pair(cfg, FP64)
    o.ewald_k(0)
    g.ewald_k(0)
    ko, kg = o.kvecs(), g.kvecs()
    assert ko.shape == kg.shape and (ko == kg).all()     # same vectors, bit for bit
    o.binning()
    g.binning()
    for x in (o, g):
        x.zero_forces()
        x.fluid_fluid()
    o.zero_forces()
    g.zero_forces()
    o.ewald_k(1)
    g.ewald_k(1)
    assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < 1e-10
    assert g.scalars()["v_coul"] == pytest.approx(o.scalars()["v_coul"], rel=1e-11)
    g.close()


def test_ewald_kspace_wide_slab():
    """A slab channel at n_kmax = 10: the z spacing of the slab k-set is a third
    of 2 pi / Lz, so |n_z| reaches 36 and the half-space holds more than 4096
    vectors (tables sized by the largest |n|, vectors in several block rows)."""
    cfg = configs.charged_slab(seed=16, n_kmax=10)
    o, g = pair(cfg, FP64)
    o.ewald_k(0)
    g.ewald_k(0)
    ko, kg = o.kvecs(), g.kvecs()
    assert ko.shape == kg.shape and (ko == kg).all()
    dkz = 2.0 * math.pi / (3.0 * cfg.params.boundary[2])
    assert ko.shape[0] > 4096 and np.abs(ko[:, 2]).max() / dkz > 16.5
    for x in (o, g):
        x.binning()
        x.zero_forces()
        x.fluid_fluid()      # v_coul: real space and self term (fluid_fluid.f90:17)
        x.zero_forces()
        x.ewald_k(1)
    assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < 1e-10
    assert g.scalars()["v_coul"] == pytest.approx(o.scalars()["v_coul"], rel=1e-11)
    g.close()


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-12), (MIXED, 1e-6)])
def test_dipolar_correction(charged_slab_cfg, prec, tol):
    """dipolar_correction (SYMMETRY 0): the slab correction's force and energy
    equal the oracle's; the fast path's force pass includes it."""
    cfg = charged_slab_cfg
    o, g = pair(cfg, prec)
    o.ewald_k(0)
    g.ewald_k(0)
    for x in (o, g):
        x.zero_forces()
    u0o, u0g = o.scalars()["v_coul"], g.scalars()["v_coul"]
    o.dipolar_correction()
    g.dipolar_correction()
    fo, fg = o.state()["force"], g.download(_abi.F)["force"]
    assert np.abs(fo[:, 2]).max() > 0.0
    assert relerr(fg, fo) < tol
    du_o = o.scalars()["v_coul"] - u0o
    du_g = g.scalars()["v_coul"] - u0g
    assert du_g == pytest.approx(du_o, rel=1e-10)
    g.close()


def test_dipolar_correction_needs_the_kspace_setup(charged_slab_cfg):
    cfg = charged_slab_cfg
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=FP64)
    with pytest.raises(MfaError):
        g.dipolar_correction()
    g.close()


def test_walls_hard_and_half_hard(brush_small_cfg):
    cfg = brush_small_cfg
    for it in (3, 4):
        p = cfg.params.copy()
        p.wall = it
        r0 = cfg.r0.copy()
        v = cfg.v.copy()
        r0[:20, 2] = np.linspace(0.001, 0.009, 20)
        v[:20, 2] = -1.0
        r0[20:40, 2] = p.z_space_wall - 0.005
        v[20:40, 2] = 1.0
        o = Oracle(p, r0, v, cfg.a_type, cfg.mass, list_cap=512)
        g = System(p, r0, v, cfg.a_type, cfg.mass, precision=FP64)
        for x in (o, g):
            x.zero_forces()
            x.fluid_wall(it)
        assert relerr(g.download()["v"], o.state()["v"]) == 0.0
        assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < 1e-12
        g.close()


def test_error_particle_outside_grid(brush_small_cfg):
    cfg = brush_small_cfg
    r0 = cfg.r0.copy()
    r0[5, 2] = -3.0     # inside the bottom wall: mod(int(z/r_bin), n) < 0 (binning.f90:29)
    g = System(cfg.params, r0, cfg.v, cfg.a_type, cfg.mass, precision=MIXED)
    with pytest.raises(MfaError) as e:
        g.binning()
    assert e.value.status == _abi.ERR_CELL_RANGE
    g.close()


def test_error_nonfinite_position(melt_cfg):
    cfg = melt_cfg
    r0 = cfg.r0.copy()
    r0[7, 0] = np.nan
    g = System(cfg.params, r0, cfg.v, cfg.a_type, cfg.mass, precision=MIXED)
    with pytest.raises(MfaError) as e:
        g.binning()
    assert e.value.status == _abi.ERR_NONFINITE
    g.close()


def test_neighbour_capacity_grows():
    """A clustered configuration overflows the list capacity estimated from the
    mean density; mfa_binning grows it and the list still matches."""
    cfg = configs.melt(seed=6, n_chain=40, n_mon=20, density=0.85)
    p = cfg.params.copy()
    L = 3.0 * p.boundary[0]
    p.boundary[:] = [L, L, L]
    for d in range(3):
        p.n_bin[d] = int(L / (math.sqrt(p.range_2[0]) + 0.4))
    # squeeze the beads into a corner at ~4x the density the capacity is sized for
    cfg = configs.Config(cfg.name, cfg.spec, p, cfg.r0 * 0.6, cfg.v, cfg.a_type, cfg.mass)
    o, g = pair(cfg, FP64, params=p)
    o.binning()
    g.binning()
    half = pair_multiset_half(o.lists()[2])
    cnt, nbr = g.debug_lists(512)[1:]
    got = pair_multiset_rows(cnt, nbr)
    assert half.shape == got.shape and (half == got).all()
    g.close()


def test_energy_log_and_dpd_temperature(melt_cfg):
    """Thermostat-on physics is checked statistically: the DPD thermostat holds
    kT = 1 (the reference draws its noise in traversal order, so trajectories
    cannot be compared)."""
    cfg = melt_cfg
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=MIXED)
    g.init_forces()
    # the generated melt starts hot (beads at 0.8 sigma); DPD with the WCA range
    # as cutoff relaxes it with a time constant of ~1800 steps
    g.step(14000)
    g.set_energy_log(10, 1000)
    g.step(4000)
    log = g.energy_log()
    assert log.shape[0] == 400
    assert (np.diff(log[:, 0]) == 10).all()
    T = 2.0 * log[:, 3] / (3.0 * cfg.n)
    assert T.mean() == pytest.approx(1.0, abs=0.05)
    g.close()


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg"])
def test_energy_log_of_the_fast_path(name, request):
    """Within a multi-step mfa_step run the kernels reduce energies only for the
    steps the energy log records and for the last step; those entries equal the
    energies the per-step path reports at the same steps (FP64, to rounding of
    the differently fused reductions)."""
    cfg = request.getfixturevalue(name)
    g1 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g2 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g1.init_forces()
    g2.init_forces()
    want = []
    for k in range(1, 48):
        g1.md_step()
        if k % 10 == 0:
            s = g1.scalars()
            want.append((k, s["e_total"], s["t_fluid"]))
    g2.set_energy_log(10, 100)
    g2.step(47)
    log = g2.energy_log()
    assert [int(x) for x in log[:, 0]] == [w[0] for w in want]
    for row, (k, e_tot, t_kin) in zip(log, want):
        assert row[1] == pytest.approx(e_tot, rel=1e-11)
        assert row[3] == pytest.approx(t_kin, rel=1e-11)
    s1, s2 = g1.scalars(), g2.scalars()
    assert s2["i_time"] == 47 and s1["e_total"] == pytest.approx(s2["e_total"], rel=1e-11)
    g1.close()
    g2.close()


def test_fetch_energy_log_while_stepping(melt_cfg):
    """mfa_fetch_energy_log copies each call's entries behind the call without
    waiting: after the next synchronising call the host buffer holds exactly
    what mfa_read_energy_log returns; out-of-range and missing logs are
    rejected."""
    import torch
    cfg = melt_cfg
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=MIXED)
    g.init_forces()
    with pytest.raises(MfaError):
        g.fetch_energy_log(np.zeros((1, 4)), 0, 1)          # no log yet
    g.set_energy_log(1, 64)
    out = torch.zeros((40, 4), dtype=torch.float64, pin_memory=True).numpy()
    done = 0
    for ln in (10, 10, 7, 10, 3):
        g.step(ln)
        g.fetch_energy_log(out[done:], done, ln)
        done += ln
    g.sync()
    log = g.energy_log()
    assert log.shape == (40, 4)
    assert np.array_equal(out, log)
    assert [int(x) for x in out[:, 0]] == list(range(1, 41))
    with pytest.raises(MfaError):
        g.fetch_energy_log(np.zeros((8, 4)), 60, 8)         # past the capacity
    g.close()


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg", "charged_small_cfg", "charged_slab_cfg"])
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_fused_forces_equal_the_subroutines(name, prec, request):
    """mfa_forces (pair pass with walls and bonds fused, then Ewald k-space and
    the slab correction) = fluid_fluid; fluid_wall; intra_molec; bending(2);
    ewald_k(1); dipolar_correction (SYMMETRY 0)."""
    cfg = request.getfixturevalue(name)
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)
    p = g.params
    if p.charged:
        g.ewald_k(0)
    g.binning()
    g.zero_forces()
    g.fluid_fluid()
    if p.symmetry == 0 and p.wall in (2, 3, 4):
        g.fluid_wall(p.wall)
    g.intra_molec()
    g.bending(2)
    if p.charged:
        g.ewald_k(1)
        g.dipolar_correction()          # nothing for SYMMETRY 1
    f1, s1 = g.download(_abi.F)["force"], g.scalars()
    g.zero_forces()
    g.forces()
    f2, s2 = g.download(_abi.F)["force"], g.scalars()
    assert relerr(f2, f1) < (1e-13 if prec == FP64 else 1e-6)
    for k in ("v_fluid_fluid", "v_fluid_wall", "v_intra_molec", "v_bend", "v_coul", "virial"):
        assert s2[k] == pytest.approx(s1[k], rel=1e-12 if prec == FP64 else 1e-6, abs=1e-9), k
    assert s2["fene_clamped"] == 2 * s1["fene_clamped"]   # counted by both passes since init
    g.close()


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg", "charged_small_cfg"])
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_tiled_and_untiled_pair_kernels_agree(name, prec, request):
    """The pair kernel reads neighbour records from its shared-memory tile (one
    block per cell row) or through the caches (blocks of consecutive particles,
    or a fixed grid of 1 or 8 CTAs per SM taking chunks from the work queue,
    where one CTA per SM makes every warp take many chunks), with each chunk's
    list whole or cut into 2 to 64 pieces (static or queued); the forces agree
    to the rounding of the reductions' order, and so do 40 steps of the fast
    path (repeated launches reuse the queue's ticket counter)."""
    cfg = request.getfixturevalue(name)
    out = []
    for k, block, tiled, queue, split in ((2, 128, True, 0, 1), (4, 64, True, 0, 1), (2, 64, False, 0, 1),
                                          (4, 256, False, 0, 1), (2, 128, False, 1, 1), (2, 128, False, 8, 1),
                                          (2, 128, False, 0, 4), (4, 64, False, 0, 64), (2, 256, False, 3, 8)):
        g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)
        g.set_pair_shape(k, block, tiled)
        g.set_pair_queue(queue)
        g.set_pair_split(split)
        if cfg.params.charged:
            g.ewald_k(0)
        g.binning()
        g.zero_forces()
        g.forces()
        f = g.download(_abi.F)["force"]
        g.init_forces()
        g.step(40)
        g.scalars()
        out.append((f, g.download(_abi.R0)["r0"]))
        g.close()
    for f, r in out[1:]:
        assert relerr(f, out[0][0]) < (1e-13 if prec == FP64 else 1e-5)
        assert float(np.abs(r - out[0][1]).max()) < (1e-12 if prec == FP64 else 1e-4)


# how the captured steps hold the rebuild: one cooperative kernel (default),
# conditional graph nodes, or six kernels that return at once when no rebuild
# is due -- (MFA_REBUILD_COOP, MFA_GRAPH_CONDITIONAL)
REBUILD_MODES = {"coop": ("1", "1"), "cond": ("0", "1"), "kernels": ("0", "0")}


def set_rebuild_mode(monkeypatch, mode):
    coop, cond = REBUILD_MODES[mode]
    monkeypatch.setenv("MFA_REBUILD_COOP", coop)
    monkeypatch.setenv("MFA_GRAPH_CONDITIONAL", cond)


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg"])
@pytest.mark.parametrize("mode", ["coop", "cond", "kernels"])
def test_whole_run_graphs(name, mode, request, monkeypatch):
    """A step count repeated from the previous call replays one captured graph
    for the whole run (first step's rebuild included, single steps too; four
    counts kept, the least recently used replaced).  Runs of changing length, whole-run graphs
    and their replacement all follow the per-step path (FP64, to rounding of
    the differently fused reductions), with the energies of each run's last
    step, the step counter and the rebuild count, whichever way the captured
    steps hold the rebuild."""
    set_rebuild_mode(monkeypatch, mode)
    cfg = request.getfixturevalue(name)
    g1 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g2 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g1.init_forces()
    g2.init_forces()
    runs = [10, 10, 10, 10, 7, 7, 3, 3, 2, 2, 1, 1, 1, 4, 4, 5, 5, 10, 10, 6, 7, 7]
    for n in runs:
        for _ in range(n):
            g1.md_step()
        g2.step(n)
        s1, s2 = g1.scalars(), g2.scalars()
        assert s1["i_time"] == s2["i_time"]
        assert s2["e_total"] == pytest.approx(s1["e_total"], rel=1e-11)
        assert s2["t_fluid"] == pytest.approx(s1["t_fluid"], rel=1e-11)
    assert s1["n_rebuilds"] == s2["n_rebuilds"] and s2["n_rebuilds"] > 1
    a, b = g1.download(), g2.download()
    # 125 steps: the pair kernel's reductions add in no fixed order, and the
    # dynamics amplify that rounding (as in the reproducibility test)
    assert float(np.abs(a["r0"] - b["r0"]).max()) < 1e-10
    assert float(np.abs(a["v"] - b["v"]).max()) < 1e-8
    assert (a["mic"] == b["mic"]).all()
    g1.close()
    g2.close()


@pytest.mark.parametrize("name", ["brush_small_cfg", "melt_cfg"])
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_rebuild_coop_conditional_or_early_exit(name, prec, monkeypatch, request):
    """The captured steps hold the rebuild in one cooperative kernel (six stages
    with grid barriers between them, a return after one flag read when none is
    due), in conditional graph nodes, or as six kernels launched every step
    that return at once when none is due.  Same physics, same rebuild count,
    no error flag; the launch counts differ by the kernels of every step: one
    cooperative launch, six early-exit launches, or six only when due."""
    cfg = request.getfixturevalue(name)
    out = {}
    for mode in ("coop", "cond", "kernels"):
        set_rebuild_mode(monkeypatch, mode)
        g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=prec)
        g.init_forces()
        s0 = g.scalars()
        g.step(64)
        s1 = g.scalars()
        assert s1["error_bits"] == 0
        out[mode] = (g.download(_abi.R0)["r0"], s1["n_rebuilds"] - s0["n_rebuilds"],
                     s1["kernel_launches"] - s0["kernel_launches"])
        g.close()
    (rc, nrc, lc), (r1, nr1, l1), (r0, nr0, l0) = out["coop"], out["cond"], out["kernels"]
    assert nr1 == nr0 == nrc and nr1 > 0
    tol = 1e-12 if prec == FP64 else 1e-4
    assert float(np.abs(r1 - r0).max()) < tol
    assert float(np.abs(rc - r0).max()) < tol
    # 63 captured steps, each launching the rebuild chain only when due
    assert l0 - l1 == 6 * (63 - (nr1 - 1)) or l0 - l1 == 6 * (63 - nr1)
    # one cooperative launch in place of six early-exit ones, every step
    assert l0 - lc == 5 * 64


@pytest.mark.parametrize("name", ["melt_cfg", "brush_small_cfg"])
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_pair_forces_is_fluid_fluid_plus_fluid_wall(name, prec, request):
    """mfa_pair_forces (one pass, 9-3 walls fused) = fluid_fluid; fluid_wall."""
    cfg = request.getfixturevalue(name)
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)
    p = g.params
    g.binning()
    g.zero_forces()
    g.fluid_fluid()
    if p.symmetry == 0 and p.wall in (2, 3, 4):
        g.fluid_wall(p.wall)
    f1, s1 = g.download(_abi.F)["force"], g.scalars()
    g.zero_forces()
    g.pair_forces()
    f2, s2 = g.download(_abi.F)["force"], g.scalars()
    assert relerr(f2, f1) < (1e-13 if prec == FP64 else 1e-6)
    for k in ("v_fluid_fluid", "v_fluid_wall", "virial"):
        assert s2[k] == pytest.approx(s1[k], rel=1e-12 if prec == FP64 else 1e-6, abs=1e-9), k
    g.close()
