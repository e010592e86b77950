"""The oracle against closed-form known answers (tests/golden/known_answers.json),
the reference's own O(N^2) energy check (util.f90:283-322), force/energy
consistency by central differences, the two binning routines against each
other, and the host-side parameter derivation against the oracle's own."""
import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT, relerr
from mfa_b200 import _abi
from mfa_b200.params import Spec, derive, C_2_16, PI_F32
from oracle import Oracle, derive_params, pair_multiset_half, pair_multiset_full

GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "known_answers.json")))


def two_body(r, *, eps=1.0, k_chain=0.0, chain=False, box=10.0):
    n = 2
    e = np.array([[eps]])
    spec = Spec(n_part=n, boundary=(box, box, box), n_type=1, n_mon=2 if chain else 0,
                n_chain=1 if chain else 0, thermostat=_abi.THERMO_NONE, eps=e, k_chain_in=k_chain,
                r_chain=1.5, skin=0.3)
    p = derive(spec)
    r0 = np.array([[5.0, 5.0, 5.0], [5.0 + r, 5.0, 5.0]])
    return Oracle(p, r0, np.zeros((n, 3)), np.ones(n, dtype=np.int32), np.ones(n))


@pytest.mark.parametrize("case", GOLD["lj"])
def test_lj_pair_known_answer(case):
    o = two_body(case["r"])
    o.init_forces()
    s = o.scalars()
    f = o.state()["force"]
    assert s["v_fluid_fluid"] == pytest.approx(case["energy"], rel=1e-12, abs=1e-12)
    assert f[1, 0] == pytest.approx(case["force"], rel=1e-12)
    assert f[0, 0] == pytest.approx(-case["force"], rel=1e-12)


@pytest.mark.parametrize("case", GOLD["fene"])
def test_fene_bond_known_answer(case):
    o = two_body(case["r"], eps=0.0, k_chain=30.0, chain=True)
    o.init_forces()
    s = o.scalars()
    f = o.state()["force"]
    assert s["v_intra_molec"] == pytest.approx(case["energy"], rel=1e-12)
    assert f[1, 0] == pytest.approx(case["force"], rel=1e-12)


@pytest.mark.parametrize("case", GOLD["bend"])
def test_bending_angle_known_answer(case):
    th = case["theta"]
    spec = Spec(n_part=3, boundary=(20.0, 20.0, 20.0), n_type=1, n_mon=3, n_chain=1,
                thermostat=_abi.THERMO_NONE, eps=np.zeros((1, 1)), k_chain_in=0.0, bending=1,
                k_bend=case["k"], alpha_eq=0.0)
    p = derive(spec)
    r0 = np.array([[5.0, 5.0, 5.0], [6.0, 5.0, 5.0], [6.0 + math.cos(th), 5.0 + math.sin(th), 5.0]])
    o = Oracle(p, r0, np.zeros((3, 3)), np.ones(3, dtype=np.int32), np.ones(3))
    o.zero_forces()
    o.bending(2)
    assert o.scalars()["v_bend"] == pytest.approx(case["energy"], rel=1e-10)
    f = o.state()["force"]
    assert np.abs(f.sum(0)).max() < 1e-12          # internal force sums to zero


@pytest.mark.parametrize("case", GOLD["wall"])
def test_wall_93_known_answer(case):
    spec = Spec(n_part=1, boundary=(10.0, 10.0, case["L"]), n_type=1, symmetry=0, wall=2,
                thermostat=_abi.THERMO_NONE, a_w=1.0, sigma_w=1.0)
    p = derive(spec)
    r0 = np.array([[5.0, 5.0, case["z"]]])
    o = Oracle(p, r0, np.zeros((1, 3)), np.ones(1, dtype=np.int32), np.ones(1))
    o.zero_forces()
    o.fluid_wall(2)
    assert o.scalars()["v_fluid_wall"] == pytest.approx(case["energy"], rel=1e-12)
    assert o.state()["force"][0, 2] == pytest.approx(case["force_z"], rel=1e-12)


def rocksalt(n_side=8, a=1.0, alpha=1.2, n_kmax=12, rc=3.9):
    n = n_side ** 3
    idx = np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    r0 = (idx + 0.5) * a
    q = np.where(idx.sum(1) % 2 == 0, 1.0, -1.0)
    L = n_side * a
    spec = Spec(n_part=n, boundary=(L, L, L), n_type=1, thermostat=_abi.THERMO_NONE,
                eps=np.zeros((1, 1)), charged=1, alpha_c=alpha * alpha, n_kmax=n_kmax, ewald_rc=rc,
                quirks=0, skin=0.1)
    p = derive(spec)
    p.inv_sqrt_pi = 1.0 / math.sqrt(p.pi)
    p.n_bin[:] = [2, 2, 2]
    p.delta_bin[:] = [0, 0, 0]
    return p, r0, q


def test_ewald_rocksalt_madelung_constant():
    """Corrected-mode Ewald energy of a rock-salt lattice is -M/a per ion pair
    (pi is the reference's single-precision value, so 1e-6 relative)."""
    p, r0, q = rocksalt()
    n = r0.shape[0]
    o = Oracle(p, r0, np.zeros((n, 3)), np.ones(n, dtype=np.int32), np.ones(n), q=q, list_cap=512)
    o.ewald_k(0)
    o.binning()
    o.zero_forces()
    o.fluid_fluid()
    o.ewald_k(1)
    e_pair = o.scalars()["v_coul"] / (n / 2)
    assert e_pair == pytest.approx(-GOLD["madelung_nacl"], rel=2e-6)
    # every ion sits at a centre of symmetry: zero force
    assert np.abs(o.state()["force"]).max() < 1e-6


def test_ewald_reference_quirk_inv_sqrt_pi():
    """With the reference's inv_sqrt_pi = 1/pi (init_config.f90:230) the real-space
    force is no longer the gradient of its energy; the oracle reproduces that."""
    p, r0, q = rocksalt(n_side=4)
    r0 = r0 + np.random.default_rng(0).normal(scale=0.05, size=r0.shape)
    n = r0.shape[0]
    forces = {}
    for mode, inv in (("corrected", 1.0 / math.sqrt(p.pi)), ("reference", 1.0 / p.pi)):
        pp = p.copy()
        pp.inv_sqrt_pi = inv
        o = Oracle(pp, r0, np.zeros((n, 3)), np.ones(n, dtype=np.int32), np.ones(n), q=q, list_cap=512)
        o.binning()
        o.zero_forces()
        o.fluid_fluid()
        forces[mode] = o.state()["force"]
    assert relerr(forces["reference"], forces["corrected"]) > 1e-2


def energy_total(o, with_bend=True, with_wall=False):
    o.zero_forces()
    o.fluid_fluid()
    e = o.scalars()["v_fluid_fluid"]
    if with_wall:
        o.fluid_wall(2)
        e += o.scalars()["v_fluid_wall"]
    o.intra_molec()
    e += o.scalars()["v_intra_molec"]
    if with_bend and o.params.bending:
        o.bending(2)
        e += o.scalars()["v_bend"]
    return e, o.state()["force"]


def test_forces_are_minus_energy_gradient(brush_small_cfg):
    """Central differences of the total potential (LJ + wall + FENE + bending)
    against the summed forces, thermostat off, on the small brush."""
    cfg = brush_small_cfg
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    p.wall_cut = 0.0
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, list_cap=512)
    o.binning()
    _, f = energy_total(o, with_wall=True)
    rng = np.random.default_rng(1)
    h = 1e-6
    for i in rng.choice(cfg.n, 12, replace=False):
        for d in range(3):
            r = cfg.r0.copy()
            r[i, d] += h
            o.set_state(r0=r)
            ep, _ = energy_total(o, with_wall=True)
            r[i, d] -= 2 * h
            o.set_state(r0=r)
            em, _ = energy_total(o, with_wall=True)
            g = -(ep - em) / (2 * h)
            assert g == pytest.approx(f[i, d], rel=2e-5, abs=2e-4), (i, d)


def test_dipolar_correction_formula(charged_slab_cfg):
    """dipolar_correction.f90:17-39 against the slab correction it states
    (Yeh and Berkowitz): M_z = sum q (z - Lz/2), F_z = -4 pi q M_z / V and
    U = 2 pi M_z^2 / V, with V = Lx Ly Lz (1 + 2) the slab volume of
    ewald_k.f90:92 and pi the widened single-precision literal."""
    cfg = charged_slab_cfg
    o = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q)
    o.ewald_k(0)
    o.zero_forces()
    u0 = o.scalars()["v_coul"]
    o.dipolar_correction()
    f = o.state()["force"]
    L = np.asarray(cfg.params.boundary[:3], dtype=np.float64)
    inv_v = 1.0 / (L[0] * L[1] * L[2] * 3.0)
    m = float(np.sum(cfg.q * (cfg.r0[:, 2] - L[2] / 2.0)))
    assert abs(m) > 1e-3
    assert (f[:, :2] == 0.0).all()
    np.testing.assert_allclose(f[:, 2], -4.0 * PI_F32 * cfg.q * m * inv_v, rtol=1e-12, atol=1e-15)
    assert o.scalars()["v_coul"] - u0 == pytest.approx(2.0 * PI_F32 * m * m * inv_v, rel=1e-9)


def slab_coulomb_energy(o):
    """LJ + Ewald (real, k-space) + slab correction: energy and forces."""
    o.zero_forces()
    o.fluid_fluid()
    o.ewald_k(1)
    o.dipolar_correction()
    s = o.scalars()
    return s["v_fluid_fluid"] + s["v_coul"], o.state()["force"]


def test_slab_coulomb_forces_are_minus_energy_gradient(charged_slab_cfg):
    """Central differences of LJ + Ewald + dipolar energy against the summed
    forces on the charged channel (thermostat off): the slab k-set, the
    k-space forces and the dipolar term belong to one energy."""
    cfg = charged_slab_cfg
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, list_cap=512)
    o.ewald_k(0)
    o.binning()
    _, f = slab_coulomb_energy(o)
    rng = np.random.default_rng(2)
    h = 1e-6
    for i in rng.choice(cfg.n, 10, replace=False):
        for d in range(3):
            r = cfg.r0.copy()
            r[i, d] += h
            o.set_state(r0=r)
            ep, _ = slab_coulomb_energy(o)
            r[i, d] -= 2 * h
            o.set_state(r0=r)
            em, _ = slab_coulomb_energy(o)
            g = -(ep - em) / (2 * h)
            assert g == pytest.approx(f[i, d], rel=2e-5, abs=2e-4), (i, d)


def test_list_energy_equals_all_pairs_energy(melt_cfg):
    """util.f90:283-322: the O(N^2) energy equals the Verlet-list energy."""
    cfg = melt_cfg
    o = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o.init_forces()
    assert o.scalars()["v_fluid_fluid"] == pytest.approx(o.check_fluid_fluid(), rel=1e-12)
    for _ in range(30):
        o.md_step()
    o.zero_forces()
    o.fluid_fluid()
    assert o.scalars()["v_fluid_fluid"] == pytest.approx(o.check_fluid_fluid(), rel=1e-12)


def test_momentum_conserved_with_dpd(melt_cfg):
    """DPD forces are pairwise antisymmetric (Philox noise keyed by the pair), so
    the total force vanishes (bulk, no walls)."""
    cfg = melt_cfg
    o = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o.init_forces()
    for _ in range(5):
        o.md_step()
    f = o.state()["force"]
    assert np.abs(f.sum(0)).max() < 1e-8 * np.abs(f).max() * cfg.n


def test_binning_and_my_binning_list_the_same_pairs(melt_cfg):
    cfg = melt_cfg
    o1 = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o2 = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o1.binning()
    o2.my_binning()
    _, _, ff1 = o1.lists()
    _, _, ff2 = o2.lists()
    half = pair_multiset_half(ff1)
    full = pair_multiset_full(ff2[:, 0], ff2[:, 1:])
    assert half.shape == full.shape and (half == full).all()


def test_binning_small_grid_visits_cells_twice():
    """make_binning_boxes.f90:14-37 takes delta_bin from the pre-binning n_bin;
    with n_bin = 2 and delta_bin = 1 the other cell is scanned twice and pairs
    in it appear twice in the list (the reference's behaviour)."""
    spec = Spec(n_part=2, boundary=(3.2, 3.2, 3.2), n_type=1, thermostat=_abi.THERMO_NONE, skin=0.3,
                n_bin=(2, 2, 2), n_bin_init=(3, 3, 3))
    p = derive(spec)
    assert list(p.delta_bin) == [1, 1, 1]
    r0 = np.array([[0.5, 0.5, 0.5], [2.4, 0.5, 0.5]])   # other x cell, 1.3 apart via the image
    o = Oracle(p, r0, np.zeros((2, 3)), np.ones(2, dtype=np.int32), np.ones(2))
    o.binning()
    _, _, ff = o.lists()
    assert ff[0, 0] + ff[1, 0] == 2


def test_energy_conserved_without_thermostat(melt_cfg):
    cfg = melt_cfg
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    o = Oracle(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o.init_forces()
    # let the fresh configuration's overlaps relax first
    for _ in range(200):
        o.md_step()
    e0 = o.scalars()["e_total"]
    for _ in range(300):
        o.md_step()
    e1 = o.scalars()["e_total"]
    assert abs(e1 - e0) / cfg.n < 5e-3


def test_host_derivation_matches_oracle_derivation():
    eps = np.ones((4, 4))
    eps[0, 0] = 0.0
    kw = dict(n_type=4, eps=eps, sigma_ii=[1.0, 1.0, 1.0, 1.0], k_chain_in=30.0, r_chain=1.5, dt=0.005,
              temp=1.0, friction=4.5, k_bend=2.0, alpha_eq=0.0, a_w=1.0, sigma_w=1.0,
              boundary=(58.42, 58.42, 60.0), skin=0.3)
    po = derive_params(**kw, brush_heads=True, wall93=True)
    ph = derive(Spec(n_part=10, boundary=kw["boundary"], n_type=4, eps=eps, brush_heads=True,
                     wall93_zero_last_type=True, skin=0.3, friction=4.5, k_bend=2.0))
    for name in ("range_2", "epsil", "sigma_2", "e_shift", "inv_range_2"):
        a = np.array(getattr(po, name)[:])
        b = np.array(getattr(ph, name)[:])
        assert (a == b).all(), name
    for name in ("skin_2", "sig", "k_chain", "inv_r_chain_2", "fene_clamp", "pi", "inv_sqrt_pi"):
        assert getattr(po, name) == getattr(ph, name), name
    assert list(po.n_bin) == list(ph.n_bin)
    assert list(po.sigma_wall[:4]) == list(ph.sigma_wall[:4])


def test_single_precision_literals():
    # init_params.f90:502, mfa_common.f90:332, intra_molec.f90:44
    assert C_2_16 == 1.1224620342254639
    assert PI_F32 == 3.1415927410125732
    p = derive(Spec(n_part=1, boundary=(5.0, 5.0, 5.0)))
    assert p.fene_clamp == 0.9800000190734863
    assert p.range_2[0] == C_2_16 * C_2_16


@pytest.mark.parametrize("r", [0.85, 1.0, 1.115])
def test_force_switch_on_known_answer(r):
    """fluid_fluid.f90:42-49,95-97 with init_force_switch_on.f90:15-22: inside
    the cutoff, r^2 is replaced by max(r^2, r_2_min), r_2_min = (1 - t/t_on) *
    (sigma_max / 0.9)^2 at time t = (s_time + i_time - 1) dt; the force keeps
    the direction and length of the true separation (force_loc = r_dummy *
    delta_r)."""
    o = two_body(r)
    p = o.params.copy()
    p.force_switch_on = 1
    p.r_2_min_time = 40.0
    p.s_time = 1
    o = Oracle(p, np.array([[5.0, 5.0, 5.0], [5.0 + r, 5.0, 5.0]]), np.zeros((2, 3)),
               np.ones(2, dtype=np.int32), np.ones(2))
    o.init_forces()
    t = (p.s_time + o.scalars()["i_time"] - 1) * p.dt
    r2_min = (1.0 - t / p.r_2_min_time) * (1.0 / float(np.float32(0.9))) ** 2
    r2 = max(r * r, r2_min)
    rc2 = C_2_16 ** 2
    rd = (1.0 / rc2) ** 3
    s6 = (1.0 / r2) ** 3
    energy = 4.0 * ((s6 * s6 - s6) - rd * (rd - 1.0))
    force = 4.0 * (12.0 * s6 * s6 - 6.0 * s6) / r2 * r      # on particle 2, along +x
    s = o.scalars()
    f = o.state()["force"]
    assert s["v_fluid_fluid"] == pytest.approx(energy, rel=1e-12)
    assert f[1, 0] == pytest.approx(force, rel=1e-12)
    assert f[0, 0] == pytest.approx(-force, rel=1e-12)
    if r * r < r2_min:
        assert force < 4.0 * (12.0 / r ** 13 - 6.0 / r ** 7)   # softer than the true force
