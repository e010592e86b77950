"""Parity at the sizes the throughput runs use, and the paths the smaller
parity tests leave out.

  * the brush with explicit solvent at full size (32 x 32 chains of 64 beads,
    174,080 beads; the throughput workload, same seed): cells bit-exact and
    the listed pairs bit-exact as multisets; FP64 forces with bending to 1e-12
    and every energy term (v_bend included) to 1e-11; ten FP64 steps without
    thermostat to 1e-10;
  * the charged system at full size (200 chains of 50 + 5000 counterions,
    15,000 beads, |n| <= 10): the k-vector set, FP64 forces to 1e-11 and
    v_coul to 1e-11 after ewald_k(1), mixed forces to 1e-4;
  * my_binning's full list feeding fluid_fluid with DPD (and Ewald real space
    in the charged case), FP64: forces to 1e-12 and 100-step trajectories to
    1e-10 -- the owner-only update of the full list (fluid_fluid.f90:119-126,
    dpd_forces.f90:68-94, ewald_real.f90:30-33, the halved LJ energy of
    fluid_fluid.f90:236);
  * the force switch-on of fluid_fluid.f90:42-49,95-97 (r^2 clamped below a
    minimum that shrinks with time), FP64 forces to 1e-12 and 100 steps to
    1e-10, mixed forces to 1e-4.
"""
import numpy as np
import pytest

from conftest import relerr
from mfa_b200 import _abi, configs
from mfa_b200._abi import FP64, MIXED
from mfa_b200.api import System
from oracle import Oracle, pair_multiset_half, pair_multiset_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def brush_full():
    return configs.brush(seed=2024)


@pytest.fixture(scope="module")
def charged_full():
    return configs.charged(seed=2024)


def test_full_brush_lists_bit_exact(brush_full):
    cfg = brush_full
    assert cfg.n == 174080
    o = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, list_cap=256)
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=MIXED)
    o.binning()
    g.binning()
    cell_o, _, ff = o.lists()
    cell_g, cnt, nbr = g.debug_lists(256)
    g.close()
    assert (cell_o == cell_g).all()
    ref = pair_multiset_half(ff)
    got = pair_multiset_rows(cnt, nbr)
    assert ref.shape[0] > 800_000                 # skin 0.3: about 4.8 listed pairs per bead
    assert ref.shape == got.shape and (ref == got).all()


def test_full_brush_fp64_forces_energies_and_ten_steps(brush_full):
    cfg = brush_full
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, list_cap=256)
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    for s in (o, g):
        s.init_forces()
        s.bending(2)
    assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < 1e-12
    so, sg = o.scalars(), g.scalars()
    assert so["v_bend"] > 0.0
    for k in ("v_fluid_fluid", "v_fluid_wall", "v_intra_molec", "v_bend"):
        assert sg[k] == pytest.approx(so[k], rel=1e-11), k
    for _ in range(10):
        o.md_step()
        g.md_step()
    so, sg = o.state(), g.download()
    assert relerr(sg["r0"], so["r0"]) < 1e-10
    assert relerr(sg["v"], so["v"]) < 1e-10
    eo, eg = o.scalars(), g.scalars()
    for k in ("e_total", "v_bend"):
        assert eg[k] == pytest.approx(eo[k], rel=1e-10), k
    g.close()


def test_full_charged_kvectors_forces_and_coulomb_energy(charged_full):
    cfg = charged_full
    assert cfg.n == 15000
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, list_cap=512)
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=FP64)
    gm = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=MIXED)
    for s in (o, g, gm):
        s.init_forces()
        s.ewald_k(1)
    ko, kg = o.kvecs(), g.kvecs()
    assert ko.shape == kg.shape and ko.shape[0] == 2084
    assert (ko == kg).all()                               # same vectors, bit for bit
    fo = o.state()["force"]
    assert relerr(g.download(_abi.F)["force"], fo) < 1e-11
    assert relerr(gm.download(_abi.F)["force"], fo) < 1e-4
    so, sg = o.scalars(), g.scalars()
    assert sg["v_coul"] == pytest.approx(so["v_coul"], rel=1e-11)
    for k in ("v_fluid_fluid", "v_intra_molec"):
        assert sg[k] == pytest.approx(so[k], rel=1e-11), k
    g.close()
    gm.close()


@pytest.mark.parametrize("name", ["melt_cfg", "charged_small_cfg"])
def test_my_binning_full_list_fp64_dpd_forces_and_100_steps(name, request):
    cfg = request.getfixturevalue(name)
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_DPD
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, list_cap=512, bin_type=1)
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=FP64, bin_type=1)
    o.init_forces()
    g.init_forces()
    assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < 1e-12
    so, sg = o.scalars(), g.scalars()
    for k in ("v_fluid_fluid", "v_intra_molec", "v_coul"):
        assert sg[k] == pytest.approx(so[k], rel=1e-11, abs=1e-11 * cfg.n), k
    for _ in range(100):
        o.md_step()
        g.md_step()
    so, sg = o.state(), g.download()
    assert relerr(sg["r0"], so["r0"]) < 1e-10
    assert relerr(sg["v"], so["v"]) < 1e-10
    eo, eg = o.scalars(), g.scalars()
    assert eg["e_total"] == pytest.approx(eo["e_total"], rel=1e-10)
    assert eg["n_rebuilds"] == eo["n_rebuilds"] and eo["n_rebuilds"] > 1
    assert g.bin_type == 1
    g.close()


def switch_on_params(cfg):
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    p.force_switch_on = 1
    p.r_2_min_time = 40.0          # init_force_switch_on.f90:18-19 (fresh configurations)
    p.s_time = 1
    return p


def test_force_switch_on_clamps_pairs_fp64_and_mixed(melt_cfg):
    cfg = melt_cfg
    p = switch_on_params(cfg)
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    g = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    gm = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=MIXED)
    for s in (o, g, gm):
        s.init_forces()
    fo = o.state()["force"]
    assert relerr(g.download(_abi.F)["force"], fo) < 1e-12
    assert relerr(gm.download(_abi.F)["force"], fo) < 1e-4
    # the clamp is active: the forces differ from the unclamped ones
    o2 = Oracle(cfg.params.copy(), cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o2.init_forces()
    assert relerr(fo, o2.state()["force"]) > 1e-2
    for _ in range(100):
        o.md_step()
        g.md_step()
    so, sg = o.state(), g.download()
    assert relerr(sg["r0"], so["r0"]) < 1e-10
    assert relerr(sg["v"], so["v"]) < 1e-10
    assert g.scalars()["e_total"] == pytest.approx(o.scalars()["e_total"], rel=1e-10)
    g.close()
    gm.close()


@pytest.mark.parametrize("rule", [0, 1])
def test_lists_bit_exact_with_particles_on_the_box_edge(melt_cfg, rule):
    """verlet_positions.f90:243-248 keeps coordinates in [0, L], so a coordinate
    can equal L exactly; binning.f90:27-29 then puts the particle in cell 0.
    Particles moved onto x = L, y = L and x = 0 keep bit-exact lists (the
    list builder's stencil images follow the cell the particle was binned in).
    my_binning (rule 1) rejects a coordinate of L as outside its grid, as its
    int(x / r_bin) indexing would overrun the reference's arrays."""
    cfg = melt_cfg
    r0 = cfg.r0.copy()
    L = [cfg.params.boundary[d] for d in range(3)]
    r0[0:200:7, 0] = L[0]
    r0[1:200:7, 1] = L[1]
    r0[2:200:7, 0] = 0.0
    o = Oracle(cfg.params, r0, cfg.v, cfg.a_type, cfg.mass, list_cap=512)
    g = System(cfg.params, r0, cfg.v, cfg.a_type, cfg.mass, precision=MIXED)
    if rule == 1:
        with pytest.raises(_abi.MfaError):
            g.my_binning()
        g.close()
        return
    o.binning()
    g.binning()
    cell_o, _, ff = o.lists()
    cell_g, cnt, nbr = g.debug_lists(512)
    g.close()
    assert (cell_o == cell_g).all()
    assert (cell_o[0:200:7] % cfg.params.n_bin[0] == 0).all()
    ref = pair_multiset_half(ff)
    got = pair_multiset_rows(cnt, nbr)
    assert ref.shape == got.shape and (ref == got).all()
