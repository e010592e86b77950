"""Trajectory sensitivities (mfa_adjoint): the hand-written discrete adjoint of
the velocity-Verlet loop against central finite differences with common
random numbers (the DPD noise is keyed by step and pair, so the perturbed runs
see the same noise), in FP64; the mixed-precision adjoint against the FP64 one.
The adjoint is also wrapped here -- in the test harness only -- as a
torch.autograd.Function, the way a Python optimiser would call it."""

import numpy as np
import pytest

from mfa_b200 import _abi, configs
from mfa_b200._abi import FP64, MIXED
from mfa_b200.api import System
from mfa_b200.sensitivity import NAMES, base_values, perturbed

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_brush():
    """4 x 4 chains of 16 beads, implicit solvent, 9-3 walls, DPD; relaxed a little."""
    cfg = configs.brush(seed=21, nx=4, ny=4, n_mon=16, graft=0.3, z_wall=24.0, solvent=False, k_bend=0.0)
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g.init_forces()
    g.step(400)
    st = g.download()
    g.close()
    return cfg, st


def run(cfg, st, params, prec, fn):
    """A run from the stored state (r, v, a held fixed: the gradient is that of
    the trajectory that starts from this state)."""
    g = System(params, st["r0"], st["v"], cfg.a_type, cfg.mass, a=st["a"], mic=st["mic"], precision=prec)
    g.binning()
    out = fn(g)
    g.close()
    return out


def test_adjoint_matches_central_differences(small_brush):
    cfg, st = small_brush
    nsteps, every, h = 40, 10, 1e-4
    J, grad = run(cfg, st, cfg.params, FP64, lambda g: g.adjoint(nsteps, every))
    J0 = run(cfg, st, cfg.params, FP64, lambda g: g.trajectory_observable(nsteps))
    assert J == pytest.approx(J0, rel=1e-12)
    base = base_values(cfg.params)
    for name in NAMES:
        jp = run(cfg, st, perturbed(cfg.params, name, 1 + h), FP64, lambda g: g.trajectory_observable(nsteps))
        jm = run(cfg, st, perturbed(cfg.params, name, 1 - h), FP64, lambda g: g.trajectory_observable(nsteps))
        fd = (jp - jm) / (2 * h * base[name])
        assert grad[name] == pytest.approx(fd, rel=1e-3, abs=1e-6 * abs(J) / base[name]), (name, grad[name], fd)


@pytest.fixture(scope="module")
def small_brush_bent():
    """The same brush with the harmonic bending term k_b = 2 (bending.f90)."""
    cfg = configs.brush(seed=22, nx=4, ny=4, n_mon=16, graft=0.3, z_wall=24.0, solvent=False, k_bend=2.0)
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=FP64)
    g.init_forces(full=True)
    g.step(400)
    st = g.download()
    g.close()
    return cfg, st


def test_adjoint_with_bending_matches_central_differences(small_brush_bent):
    """The bending term's vector-Jacobian product enters every gradient through
    the state adjoint; a wrong one shows in all six."""
    cfg, st = small_brush_bent
    assert cfg.params.bending == 1
    nsteps, every, h = 40, 10, 1e-4
    J, grad = run(cfg, st, cfg.params, FP64, lambda g: g.adjoint(nsteps, every))
    J0 = run(cfg, st, cfg.params, FP64, lambda g: g.trajectory_observable(nsteps))
    assert J == pytest.approx(J0, rel=1e-12)
    base = base_values(cfg.params)
    for name in NAMES:
        jp = run(cfg, st, perturbed(cfg.params, name, 1 + h), FP64, lambda g: g.trajectory_observable(nsteps))
        jm = run(cfg, st, perturbed(cfg.params, name, 1 - h), FP64, lambda g: g.trajectory_observable(nsteps))
        fd = (jp - jm) / (2 * h * base[name])
        assert grad[name] == pytest.approx(fd, rel=1e-3, abs=1e-6 * abs(J) / base[name]), (name, grad[name], fd)
    _, g32 = run(cfg, st, cfg.params, MIXED, lambda g: g.adjoint(nsteps, every))
    scale = max(abs(v) for v in grad.values())
    for name in NAMES:
        assert abs(g32[name] - grad[name]) < 1e-2 * max(abs(grad[name]), 1e-3 * scale), (name, g32[name], grad[name])


def test_adjoint_checkpoint_interval_does_not_change_the_gradient(small_brush):
    cfg, st = small_brush
    _, g1 = run(cfg, st, cfg.params, FP64, lambda g: g.adjoint(30, 30))
    _, g2 = run(cfg, st, cfg.params, FP64, lambda g: g.adjoint(30, 7))
    for name in NAMES:
        assert g2[name] == pytest.approx(g1[name], rel=1e-9, abs=1e-12)


def test_repeated_adjoint_calls_reuse_the_cached_sequences(small_brush):
    """A second mfa_adjoint call of the same length and checkpoint interval on
    the same context reuses the cached workspace and captured sequences; it
    equals the first call of a fresh context brought to the same state and
    step (the DPD noise is keyed by the step) by the forward run, and so does
    a third call after a new cell grid dropped the context's graphs and the
    cache with them."""
    cfg, st = small_brush

    def fresh():
        g = System(cfg.params, st["r0"], st["v"], cfg.a_type, cfg.mass, a=st["a"], mic=st["mic"], precision=FP64)
        g.binning()
        return g

    g = fresh()
    g.adjoint(40, 10)                      # allocates its workspace, captures its sequences
    for k in range(2):
        J2, grad2 = g.adjoint(40, 10)      # steps 40k+40 .. 40k+80
        f = fresh()
        f.trajectory_observable(40 * (k + 1))
        J1, grad1 = f.adjoint(40, 10)
        f.close()
        assert J2 == pytest.approx(J1, rel=1e-9), k
        for name in NAMES:
            assert grad2[name] == pytest.approx(grad1[name], rel=1e-7, abs=1e-12), (k, name)
        g.set_cells(list(g.params.n_bin), g.params.skin)
    g.close()


def test_mixed_adjoint_close_to_fp64(small_brush):
    cfg, st = small_brush
    _, g64 = run(cfg, st, cfg.params, FP64, lambda g: g.adjoint(40, 10))
    _, g32 = run(cfg, st, cfg.params, MIXED, lambda g: g.adjoint(40, 10))
    scale = max(abs(v) for v in g64.values())
    for name in NAMES:
        assert abs(g32[name] - g64[name]) < 1e-2 * max(abs(g64[name]), 1e-3 * scale), (name, g32[name], g64[name])


def test_torch_autograd_wrapper(small_brush):
    torch = pytest.importorskip("torch")
    cfg, st = small_brush
    base = base_values(cfg.params)

    class Observable(torch.autograd.Function):
        """J(theta) of a 20-step run; backward returns the adjoint's gradient."""

        @staticmethod
        def forward(ctx, theta):
            p = cfg.params
            for name, val in zip(NAMES, theta.tolist()):
                p = perturbed(p, name, val / base[name])
            J, grad = run(cfg, st, p, FP64, lambda g: g.adjoint(20, 5))
            ctx.save_for_backward(torch.tensor([grad[n] for n in NAMES], dtype=torch.float64))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad

    theta = torch.tensor([base[n] for n in NAMES], dtype=torch.float64, requires_grad=True)
    J = Observable.apply(theta)
    J.backward()
    # central differences of the wrapped function on two parameters
    for i in (0, 4):
        e = torch.zeros(6, dtype=torch.float64)
        e[i] = 1e-4 * theta[i].item()
        with torch.no_grad():
            fd = (Observable.apply(theta + e) - Observable.apply(theta - e)) / (2 * e[i])
        assert theta.grad[i].item() == pytest.approx(fd.item(), rel=1e-3, abs=1e-8)


def charged_start(cfg, steps=300):
    """A charged configuration relaxed on the GPU (FP64), Ewald tables set up."""
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=FP64)
    g.init_forces(full=True)
    g.step(steps)
    st = g.download()
    g.close()
    return st


def run_q(cfg, st, params, prec, fn):
    g = System(params, st["r0"], st["v"], cfg.a_type, cfg.mass, q=cfg.q, a=st["a"], mic=st["mic"],
               precision=prec)
    g.ewald_k(0)
    g.binning()
    out = fn(g)
    g.close()
    return out


def fd_check(cfg, st, nsteps=40, every=10, h=1e-4, mixed=False):
    J, grad = run_q(cfg, st, cfg.params, FP64, lambda g: g.adjoint(nsteps, every))
    J0 = run_q(cfg, st, cfg.params, FP64, lambda g: g.trajectory_observable(nsteps))
    assert J == pytest.approx(J0, rel=1e-12)
    base = base_values(cfg.params)
    for name in NAMES:
        jp = run_q(cfg, st, perturbed(cfg.params, name, 1 + h), FP64, lambda g: g.trajectory_observable(nsteps))
        jm = run_q(cfg, st, perturbed(cfg.params, name, 1 - h), FP64, lambda g: g.trajectory_observable(nsteps))
        fd = (jp - jm) / (2 * h * base[name])
        assert grad[name] == pytest.approx(fd, rel=1e-3, abs=1e-6 * abs(J) / base[name]), (name, grad[name], fd)
    if mixed:
        _, g32 = run_q(cfg, st, cfg.params, MIXED, lambda g: g.adjoint(nsteps, every))
        scale = max(abs(v) for v in grad.values())
        for name in NAMES:
            assert abs(g32[name] - grad[name]) < 2e-2 * max(abs(grad[name]), 1e-3 * scale), (name, g32[name])
    return grad


def test_adjoint_charged_bulk_langevin_matches_central_differences():
    """Ewald real space with its own cutoff, the k-space sum (|n| <= 6) and the
    Langevin thermostat (friction and noise amplitude through gamma): their
    vector-Jacobian products enter every gradient through the state adjoint,
    and the Langevin one also the gamma gradient directly."""
    cfg = configs.charged(seed=41, n_chain=16, n_mon=10, density=0.5, n_kmax=6, rc_real=3.0)
    assert cfg.params.thermostat == _abi.THERMO_LGV and cfg.params.charged
    grad = fd_check(cfg, charged_start(cfg), mixed=True)
    assert abs(grad["gamma_dpd"]) > 0.0


def test_adjoint_charged_reference_mode_dpd_matches_central_differences():
    """The reference's form of the Ewald real space (inside the LJ range, its
    1/pi constant) with the DPD thermostat."""
    cfg = configs.charged(seed=42, n_chain=16, n_mon=10, density=0.5, n_kmax=6, reference_mode=True,
                          thermostat=_abi.THERMO_DPD, friction=4.5)
    fd_check(cfg, charged_start(cfg))


def test_adjoint_charged_slab_matches_central_differences():
    """The charged channel: 9-3 walls, the slab k-set and the dipolar
    correction (dipolar_correction.f90) with the Langevin thermostat."""
    cfg = configs.charged_slab(seed=43, n_chain=12, n_mon=10, z_wall=8.0, n_kmax=4)
    assert cfg.params.symmetry == 0
    grad = fd_check(cfg, charged_start(cfg))
    assert abs(grad["eps_wall"]) > 0.0
