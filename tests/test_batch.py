"""Many systems in one launch (mfa_batch_*): a batch of uneven brushes steps
each system exactly as that system stepping alone does (same noise, same
lists, same rebuilds), to the rounding of the force reductions' order."""
import numpy as np
import pytest

from mfa_b200 import _abi, configs
from mfa_b200._abi import FP64, MIXED, MfaError
from mfa_b200.api import Batch, System


def test_uneven_brushes_generator():
    cs = configs.uneven_brushes(seed=5, n_sys=12)
    assert len(cs) == 12
    sizes = {c.n for c in cs}
    assert len(sizes) > 3                                      # uneven
    for c in cs:
        p = c.params
        assert p.n_chain * p.n_mon == c.n and p.n_mon in (16, 32, 64, 128)
        assert p.z_space_wall == pytest.approx(2.2 * p.n_mon)
        g = p.n_chain / (p.boundary[0] * p.boundary[1])
        assert 0.05 <= g <= 0.5
        # overlap-free start: nearest distinct beads >= 0.8 sigma
        from scipy.spatial import cKDTree
        L = np.array(p.boundary[:]) * [1, 1, 10]
        d = cKDTree(np.mod(c.r0, L), boxsize=L).query(np.mod(c.r0, L), 2)[0][:, 1]
        assert d.min() > 0.8
    assert len({c.params.seed for c in cs}) == 12              # seeded per system


def _systems(cfgs, prec):
    out = []
    for c in cfgs:
        g = System(c.params, c.r0, c.v, c.a_type, c.mass, precision=prec)
        g.init_forces()
        out.append(g)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("persist", ["1", "0"])
def test_batch_equals_systems_stepped_alone(prec, persist, monkeypatch):
    """Grouped launches per stage in captured graphs (default), or one
    persistent cooperative launch per run (MFA_BATCH_PERSIST=1)."""
    monkeypatch.setenv("MFA_BATCH_PERSIST", persist)
    cfgs = configs.uneven_brushes(seed=7, n_sys=4, grids=(4, 7), lengths=(16, 32))
    alone = _systems(cfgs, prec)
    grouped = _systems(cfgs, prec)
    for g in alone:
        g.step(47)
    b = Batch(grouped)
    b.step(47)
    sb = b.scalars()
    for g1, g2, s2 in zip(alone, grouped, sb):
        s1 = g1.scalars()
        assert s2["error_bits"] == 0 and s2["i_time"] == s1["i_time"] == 47
        assert s2["n_rebuilds"] == s1["n_rebuilds"]
        r1, r2 = g1.download(_abi.R0)["r0"], g2.download(_abi.R0)["r0"]
        tol = 1e-11 if prec == FP64 else 1e-4
        assert float(np.abs(r1 - r2).max()) < tol
        assert s2["e_total"] == pytest.approx(s1["e_total"], rel=1e-10 if prec == FP64 else 1e-5)
    if persist == "1":
        assert b.launches() == 1                  # the whole 47-step run
    else:
        # one launch per stage for all four systems: two per step plus the rebuilds
        assert b.launches() < 2 * 47 + 6 * 47
    # further runs: the energies reduced are those of each run's last step
    for n in (10, 10, 3):
        for g in alone:
            g.step(n)
        b.step(n)
        for g1, s2 in zip(alone, b.scalars()):
            s1 = g1.scalars()
            assert s2["i_time"] == s1["i_time"]
            assert s2["e_total"] == pytest.approx(s1["e_total"], rel=1e-9 if prec == FP64 else 1e-4)
    b.close()
    for g in alone + grouped:
        g.close()


@pytest.mark.gpu
def test_batch_rejects_mixed_physics(melt_cfg, brush_small_cfg):
    a = System(melt_cfg.params, melt_cfg.r0, melt_cfg.v, melt_cfg.a_type, melt_cfg.mass, precision=MIXED)
    c = brush_small_cfg
    b = System(c.params, c.r0, c.v, c.a_type, c.mass, precision=MIXED)
    with pytest.raises(MfaError) as e:
        Batch([a, b])
    assert e.value.status == _abi.ERR_UNSUPPORTED
    a.close()
    b.close()
