"""Optional force terms behind the reference's cpp switches: external_force.f90
(EXT_FORCE 1), orientation.f90 (ORIENTATION, modes 1 and 2) and the DPD-VV
re-evaluation of the dissipative force, new_dpd_fd.f90 (DPD_VV).

CPU tests pin the oracle's restatement: closed forms of the external force and
of the orientation energy, central differences of the mode-1 energy, and a
numpy restatement of new_dpd_fd over the oracle's own Verlet list.  GPU tests
compare the CUDA path with the oracle.  Tolerances: FP64 path 1e-12 relative
on forces and the orientation energy, 1e-10 on 50-step DPD-VV trajectories;
MIXED path 1e-6 on the external and orientation forces (FP32 force records),
2e-3 sigma absolute on positions after 50 steps.
"""
import math

import numpy as np
import pytest

from conftest import relerr
from mfa_b200 import _abi, configs
from mfa_b200._abi import FP64, MIXED, MfaError
from oracle import Oracle


def _bent_first_bonds(cfg, seed, theta=(0.3, 1.2)):
    """Positions with every grafted chain's second bead placed at a polar angle
    in `theta` from its head's ghost-bond direction (orientation.f90:34-39)."""
    p = cfg.params
    rng = np.random.default_rng(seed)
    r0 = cfg.r0.copy()
    Lz = p.boundary[2]
    heads = np.arange(p.n_chain) * p.n_mon
    s = np.where(r0[heads, 2] > Lz / 2.0, -1.0, 1.0)
    th = rng.uniform(*theta, size=p.n_chain)
    ph = rng.uniform(0.0, 2 * math.pi, size=p.n_chain)
    d = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), s * np.cos(th)], axis=1)
    r0[heads + 1] = r0[heads] + 0.97 * d
    return r0, th


def _oracle(cfg, params=None, r0=None):
    p = cfg.params if params is None else params
    return Oracle(p, cfg.r0 if r0 is None else r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, list_cap=512)


# ---------------------------------------------------------------- oracle (CPU)

def test_oracle_external_force_closed_form(brush_small_cfg):
    cfg = brush_small_cfg
    o = _oracle(cfg)
    o.zero_forces()
    k = 0.37
    o.external_force(1, k)
    f = o.state()["force"]
    L = cfg.params.boundary
    assert (f[:, 0] == 0.0).all()
    assert np.array_equal(f[:, 1], -(k * (cfg.r0[:, 1] - L[1] / 2.0)))
    assert np.array_equal(f[:, 2], -(k * (cfg.r0[:, 2] - L[2] / 2.0)))
    o.zero_forces()
    o.external_force(0, k)   # only case(1) acts
    assert (o.state()["force"] == 0.0).all()


@pytest.mark.parametrize("alpha_or", [0.0, 0.5])
def test_oracle_orientation_mode1_energy_closed_form(brush_small_cfg, alpha_or):
    cfg = brush_small_cfg
    r0, th = _bent_first_bonds(cfg, seed=3)
    o = _oracle(cfg, r0=r0)
    o.zero_forces()
    k = 2.0
    v_or = o.orientation(1, k, alpha_or)
    assert v_or == pytest.approx(float(np.sum(0.5 * k * (th - alpha_or) ** 2)), rel=1e-12)
    f = o.state()["force"]
    heads = np.arange(cfg.params.n_chain) * cfg.params.n_mon
    # forces only on the head and the second bead, equal and opposite
    assert np.allclose(f[heads], -f[heads + 1], rtol=0, atol=1e-15)
    others = np.setdiff1d(np.arange(cfg.params.n_part), np.concatenate([heads, heads + 1]))
    assert (f[others] == 0.0).all()
    # |F| = k (theta - alpha) / |bond|, perpendicular to the bond
    b = r0[heads + 1] - r0[heads]
    mag = np.linalg.norm(f[heads + 1], axis=1)
    assert np.allclose(mag, k * np.abs(th - alpha_or) / 0.97, rtol=1e-10)
    assert np.abs(np.sum(f[heads + 1] * b, axis=1)).max() < 1e-12


def test_oracle_orientation_mode1_force_is_minus_gradient(brush_small_cfg):
    cfg = brush_small_cfg
    r0, _ = _bent_first_bonds(cfg, seed=4)
    o = _oracle(cfg, r0=r0)
    k, alpha = 2.0, 0.4
    o.zero_forces()
    o.orientation(1, k, alpha)
    f = o.state()["force"]
    h = 5 * cfg.params.n_mon + 1   # second bead of chain 5
    eps = 1e-6
    for d in range(3):
        vals = []
        for sgn in (1.0, -1.0):
            r = r0.copy()
            r[h, d] += sgn * eps
            o.set_state(r0=r)
            o.zero_forces()
            vals.append(o.orientation(1, k, alpha))
        assert -(vals[0] - vals[1]) / (2 * eps) == pytest.approx(f[h, d], rel=1e-6, abs=1e-8)


def test_oracle_orientation_mode2_energy_closed_form(melt_cfg):
    cfg = melt_cfg
    p = cfg.params
    o = _oracle(cfg)
    o.zero_forces()
    k, alpha = 1.5, 0.3
    v_or = o.orientation(2, k, alpha)
    L = np.asarray(p.boundary)

    def mi(d):
        return d - L * np.trunc(2.0 * d / L)

    heads = np.arange(p.n_chain) * p.n_mon
    last = heads + p.n_mon - 1
    ex = np.array([1.0, 0.0, 0.0])
    b1 = mi(cfg.r0[heads + 1] - cfg.r0[heads])
    b2 = mi(cfg.r0[last] - cfg.r0[last - 1])
    t1 = np.arccos(b1 @ ex / np.linalg.norm(b1, axis=1))
    t2 = np.arccos(b2 @ ex / np.linalg.norm(b2, axis=1))
    want = float(np.sum(0.5 * k * (t1 - alpha) ** 2 + 0.5 * k * (t2 - alpha) ** 2))
    assert v_or == pytest.approx(want, rel=1e-10)
    for mode in (0, 3):
        o.zero_forces()
        assert o.orientation(mode, k, alpha) == 0.0
        assert (o.state()["force"] == 0.0).all()


def _fd_numpy(r0, v, a_type, ff, params):
    """new_dpd_fd.f90:27-84 restated with numpy over an ff_list (1-based rows)."""
    n = r0.shape[0]
    cnt = ff[:, 0]
    ii = np.repeat(np.arange(n), cnt)
    mask = np.arange(ff.shape[1] - 1)[None, :] < cnt[:, None]
    jj = ff[:, 1:][mask] - 1
    keep = (a_type[ii] != 1) & (a_type[jj] != 1)
    ii, jj = ii[keep], jj[keep]
    L = np.asarray(params.boundary)
    d = r0[ii] - r0[jj]
    d[:, :2] = d[:, :2] - L[:2] * np.trunc(2.0 * d[:, :2] / L[:2])
    r2 = (d[:, 0] ** 2 + d[:, 1] ** 2) + d[:, 2] ** 2
    rr = np.array(params.range_2).reshape(_abi.MAX_TYPES, _abi.MAX_TYPES)[a_type[ii] - 1, a_type[jj] - 1]
    inside = r2 < rr
    ii, jj, d, r2, rr = ii[inside], jj[inside], d[inside], r2[inside], rr[inside]
    wd = (1.0 - np.sqrt(r2 / rr)) ** 2 if params.dpd_weight == 0 else np.ones_like(r2)
    rv = d / np.sqrt(r2)[:, None]
    rd = np.sum((v[ii] - v[jj]) * rv, axis=1)
    fv = (-params.friction * wd * rd)[:, None] * rv
    fd = np.zeros((n, 3))
    np.add.at(fd, ii, fv)
    np.add.at(fd, jj, -fv)
    return fd, int(inside.sum())


def _dpd_vv_step_until_fd(o):
    """One md_main iteration of a DPD_VV build up to (not including) new_dpd_fd."""
    p = o.params
    o.verlet_positions()
    if o.check_skin() == 1:
        o.binning()
    o.zero_forces()
    o.fluid_fluid()
    if p.symmetry == 0 and p.wall in (2, 3, 4):
        o.fluid_wall(p.wall)
    o.intra_molec()
    if p.bending:
        o.bending(2)
    o.verlet_velocities()


def test_oracle_new_dpd_fd_against_numpy(brush_small_cfg):
    cfg = brush_small_cfg
    o = _oracle(cfg)
    o.init_forces()
    o.set_dpd_vv(True)
    fd_prev = np.zeros((cfg.params.n_part, 3))
    for step in range(3):
        _dpd_vv_step_until_fd(o)
        s1 = o.state()
        _, _, ff = o.lists()
        fd, npairs = _fd_numpy(s1["r0"], s1["v"], cfg.a_type, ff, cfg.params)
        assert npairs > 1000
        o.new_dpd_fd()
        s2 = o.state()
        want_f = (s1["force"] - fd_prev) + fd
        assert relerr(s2["force"], want_f) < 1e-12
        want_v = s1["v"] + 0.5 * cfg.params.dt * s2["force"] / cfg.mass[:, None]
        assert relerr(s2["v"], want_v) < 1e-14
        assert relerr(s2["a"], s2["force"] / cfg.mass[:, None]) < 1e-15
        # the pair force conserves momentum; heads feel none of it
        assert np.abs(fd.sum(axis=0)).max() < 1e-10 * np.abs(fd).max()
        assert (fd[cfg.a_type == 1] == 0.0).all()
        sc = o.scalars()
        ke = 0.5 * float(np.sum(cfg.mass[:, None] * s2["v"] ** 2))
        assert sc["t_fluid"] == pytest.approx(ke, rel=1e-12)
        assert sc["e_total"] == pytest.approx(sc["v_total"] + sc["t_fluid"], rel=1e-14)
        fd_prev = fd


def test_oracle_dpd_vv_melt_has_no_pairs(melt_cfg):
    """Every melt bead is type 1, which new_dpd_fd.f90:31,38 skips as a head:
    the call only swaps the (zero) dissipative force and adds a half kick."""
    cfg = melt_cfg
    o = _oracle(cfg)
    o.init_forces()
    o.set_dpd_vv(True)
    _dpd_vv_step_until_fd(o)
    s1 = o.state()
    o.new_dpd_fd()
    s2 = o.state()
    assert np.array_equal(s2["force"], s1["force"])
    assert np.array_equal(s2["v"], s1["v"] + 0.5 * cfg.params.dt * s1["force"] * (1.0 / cfg.mass[:, None]))


def test_oracle_verlet_velocities_under_dpd_vv_keeps_heads_free(brush_small_cfg):
    """verlet_velocities.f90:79-230 (head rules) is compiled out under DPD_VV."""
    cfg = brush_small_cfg
    o = _oracle(cfg)
    o.init_forces()
    o.set_dpd_vv(True)
    _dpd_vv_step_until_fd(o)
    s = o.state()
    heads = np.arange(cfg.params.n_chain) * cfg.params.n_mon
    assert np.abs(s["force"][heads]).max() > 0.0
    assert np.array_equal(s["a"][heads], s["force"][heads] * (1.0 / cfg.mass[heads, None]))


# ---------------------------------------------------------------- GPU parity

def _system(cfg, prec, params=None, r0=None):
    from mfa_b200.api import System
    p = cfg.params if params is None else params
    return System(p, cfg.r0 if r0 is None else r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(FP64, 1e-15), (MIXED, 1e-6)])
def test_gpu_external_force(brush_small_cfg, prec, tol):
    cfg = brush_small_cfg
    o, g = _oracle(cfg), _system(cfg, prec)
    for s in (o, g):
        s.zero_forces()
        s.external_force(1, 0.37)
    assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < tol
    # it adds to the force already there
    g.init_forces()
    f0 = g.download(_abi.F)["force"]
    g.external_force(1, 0.37)
    df = g.download(_abi.F)["force"] - f0
    assert relerr(df, o.state()["force"]) < (1e-12 if prec == FP64 else 1e-4)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(FP64, 1e-12), (MIXED, 1e-6)])
@pytest.mark.parametrize("mode", [1, 2])
def test_gpu_orientation(brush_small_cfg, prec, tol, mode):
    cfg = brush_small_cfg
    r0, _ = _bent_first_bonds(cfg, seed=7)
    o, g = _oracle(cfg, r0=r0), _system(cfg, prec, r0=r0)
    for s in (o, g):
        s.zero_forces()
    vo = o.orientation(mode, 2.0, 0.25)
    vg = g.orientation(mode, 2.0, 0.25, energy=True)
    assert vg == pytest.approx(vo, rel=1e-12)
    assert relerr(g.download(_abi.F)["force"], o.state()["force"]) < tol
    # added to the force already there, and v_or of a mode that does nothing is 0
    vg0 = g.orientation(3, 2.0, 0.25, energy=True)
    assert vg0 == 0.0
    g.close()


@pytest.mark.gpu
def test_gpu_orientation_rejects_one_bead_chains(melt_cfg):
    cfg = melt_cfg
    p = cfg.params.copy()
    p.n_mon, p.n_chain = 1, p.n_part
    g = _system(cfg, FP64, params=p)
    with pytest.raises(MfaError) as e:
        g.orientation(1, 1.0, 0.0)
    assert e.value.status == _abi.ERR_ARGS
    g.close()


@pytest.mark.gpu
def test_gpu_dpd_vv_trajectory_fp64(brush_small_cfg):
    cfg = brush_small_cfg
    o, g = _oracle(cfg), _system(cfg, FP64)
    o.init_forces()
    g.init_forces()
    o.set_dpd_vv(True)
    g.set_dpd_vv(True)
    for _ in range(50):
        o.md_step()
        g.md_step()
    so, sg = o.state(), g.download()
    assert relerr(sg["r0"], so["r0"]) < 1e-10
    assert relerr(sg["v"], so["v"]) < 1e-10
    assert relerr(sg["force"], so["force"]) < 1e-9
    eo, eg = o.scalars(), g.scalars()
    assert eg["t_fluid"] == pytest.approx(eo["t_fluid"], rel=1e-10)
    assert eg["e_total"] == pytest.approx(eo["e_total"], rel=1e-10)
    g.close()


@pytest.mark.gpu
def test_gpu_dpd_vv_trajectory_mixed(brush_small_cfg):
    cfg = brush_small_cfg
    o, g = _oracle(cfg), _system(cfg, MIXED)
    o.init_forces()
    g.init_forces()
    o.set_dpd_vv(True)
    g.set_dpd_vv(True)
    for _ in range(50):
        o.md_step()
        g.md_step()
    so, sg = o.state(), g.download()
    assert np.abs(sg["r0"] - so["r0"]).max() < 2e-3
    assert g.scalars()["t_fluid"] == pytest.approx(o.scalars()["t_fluid"], rel=1e-3)
    g.close()


@pytest.mark.gpu
def test_gpu_dpd_vv_call_rules(brush_small_cfg):
    cfg = brush_small_cfg
    g = _system(cfg, FP64)
    g.init_forces()
    with pytest.raises(MfaError) as e:
        g.new_dpd_fd()              # the switch is off
    assert e.value.status == _abi.ERR_STATE
    g.set_dpd_vv(True)
    with pytest.raises(MfaError) as e:
        g.step(10)                  # the fused step has no new_dpd_fd pass
    assert e.value.status == _abi.ERR_UNSUPPORTED
    g.set_dpd_vv(False)
    g.step(10)
    assert g.scalars()["i_time"] == 10
    g.close()


def test_oracle_new_dpd_fd_full_list_applies_each_pair_twice(brush_small_cfg):
    """new_dpd_fd.f90:33-84 adds each listed entry's force to both beads; with
    my_binning's full list (every pair in both rows) a pair's dissipative force
    is applied twice -- the reference's arithmetic, kept as it is."""
    cfg = brush_small_cfg
    fds = []
    for rebuild in ("binning", "my_binning"):
        o = _oracle(cfg)
        o.init_forces()
        getattr(o, rebuild)()
        o.set_dpd_vv(True)
        s1 = o.state()
        o.new_dpd_fd()
        fds.append(o.state()["force"] - s1["force"])
    half, full = fds
    assert np.abs(half).max() > 0.0
    assert relerr(full, 2.0 * half) < 1e-12
