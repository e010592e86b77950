"""Thermostat-on parity: statistics, not trajectories.

The reference draws its DPD noise from one sequential ziggurat stream in the
order the neighbour list is walked (dpd_forces.f90:19), which no parallel
evaluation can reproduce; the CUDA path draws it from Philox keyed by (step,
pair).  So with the thermostat on, the two are compared as ensembles: the
oracle run with the reference's sequential ziggurat noise (rng_mode 1) and the
CUDA fast path (mixed precision, captured graphs), both from the same melt
(the 100 x 32 bead-spring melt at density 0.85, DPD gamma = 4.5, kT = 1,
dt = 0.005; the fresh random-walk chains overlap and start hot, so the state
is first relaxed for 20,000 steps on the GPU, then each run takes 1000 steps
to decorrelate and 20,000 sampled steps):
  * temperature 2 KE / (3 N) every 10 steps, block averages (4 blocks of
    5000 steps; the temperature relaxes in about 1800 steps under this
    thermostat, whose range is the WCA cutoff):
    the two means agree within 4 combined standard errors, and each is kT = 1
    within 3.5 % (the scheme's own bias at dt = 0.005 is about +2 %);
  * the radial distribution function g(r) on 0.7 <= r < 2.5 (36 bins) from 100
    snapshots: block errors from 4 blocks, every bin within 5 combined errors
    and chi^2 per bin below 3.5.  With 4 blocks a side each bin's combined
    error has about 6 degrees of freedom, so z is close to Student's t(6):
    E[z^2] = 1.5, and the mean over ~30 bins (correlated within a snapshot)
    spreads by 0.6 or more; 3.5 is over three such spreads above 1.5 (values
    seen: 0.7 to 2.8 over repeated runs, the GPU trajectory differing from run
    to run with the order of its force reductions);
  * the radius of gyration (observation.f90:248-258) of each of the 100
    chains, averaged over the 100 snapshots: the chain-by-chain differences
    average to zero within 4 standard errors (paired test; both runs start
    from the same chains).
"""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from mfa_b200 import _abi, configs
from mfa_b200.api import System
from oracle import Oracle

pytestmark = pytest.mark.gpu

EQUIL, STEPS, EVERY, SNAP = 1000, 20000, 10, 200
R_LO, R_HI, NBIN = 0.7, 2.5, 36


def gofr(r, L):
    tree = cKDTree(np.mod(r, L), boxsize=L)
    d = tree.query_pairs(R_HI, output_type="ndarray")
    dr = r[d[:, 0]] - r[d[:, 1]]
    dr -= L * np.round(dr / L)
    dist = np.sqrt((dr * dr).sum(1))
    h, edges = np.histogram(dist, bins=NBIN, range=(R_LO, R_HI))
    n = r.shape[0]
    shell = 4.0 / 3.0 * np.pi * (edges[1:] ** 3 - edges[:-1] ** 3)
    return h / (0.5 * n * (n / np.prod(L)) * shell)


def chain_rg2(r_unf, n_chain, n_mon):
    c = r_unf.reshape(n_chain, n_mon, 3)
    cm = c.mean(axis=1, keepdims=True)
    return ((c - cm) ** 2).sum(axis=2).mean(axis=1)


def sample(run_steps, state, n, L, p):
    T, G, RG = [], [], []
    for k in range(STEPS // EVERY):
        run_steps(EVERY)
        st = state()
        T.append(st["t"])
        if ((k + 1) * EVERY) % SNAP == 0:
            G.append(gofr(st["r0"], L))
            RG.append(chain_rg2(st["r0"] + st["mic"] * L, p.n_chain, p.n_mon))
    return np.array(T), np.array(G), np.array(RG)


def blocks(x, nb):
    m = x[: (len(x) // nb) * nb].reshape(nb, -1, *x.shape[1:]).mean(axis=1)
    return m.mean(axis=0), m.std(axis=0, ddof=1) / np.sqrt(nb)


def test_temperature_rdf_and_rg_agree_with_the_reference_noise_within_statistical_error():
    cfg = configs.melt(seed=31)
    p = cfg.params
    n = cfg.n
    L = np.array([p.boundary[d] for d in range(3)])
    g0 = System(p, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=_abi.FP64)
    g0.init_forces()
    g0.step(20000)
    st = g0.download()
    g0.close()
    o = Oracle(p, st["r0"], st["v"], cfg.a_type, cfg.mass, a=st["a"], mic=st["mic"], rng_mode=1)
    o.init_forces()
    g = System(p, st["r0"], st["v"], cfg.a_type, cfg.mass, a=st["a"], mic=st["mic"], precision=_abi.MIXED)
    g.init_forces()

    def o_run(k):
        for _ in range(k):
            o.md_step()

    def o_state():
        s = o.state()
        return {"r0": s["r0"], "mic": s["mic"], "t": 2.0 * o.scalars()["t_fluid"] / (3.0 * n)}

    def g_state():
        s = g.download(_abi.R0 | _abi.MIC)
        return {"r0": s["r0"], "mic": s["mic"], "t": 2.0 * g.scalars()["t_fluid"] / (3.0 * n)}

    o_run(EQUIL)
    g.step(EQUIL)
    To, Go, RGo = sample(o_run, o_state, n, L, p)
    Tg, Gg, RGg = sample(g.step, g_state, n, L, p)
    assert g.scalars()["error_bits"] == 0
    g.close()

    # blocks of 5000 steps, several times the temperature's relaxation time
    # under this weak thermostat (about 1800 steps), so that they are independent
    mo, eo = blocks(To, 4)
    mg, eg = blocks(Tg, 4)
    assert abs(mo - mg) < 4.0 * np.hypot(eo, eg), (mo, eo, mg, eg)
    # velocity Verlet with the DPD forces of the half-step velocity runs about
    # 2 % hot at dt = 0.005 (1.021 measured), in the reference's scheme and here alike
    assert abs(mo - 1.0) < 0.035 and abs(mg - 1.0) < 0.035

    go, sgo = blocks(Go, 4)
    gg, sgg = blocks(Gg, 4)
    ok = (go > 0.05) | (gg > 0.05)
    z = (go - gg)[ok] / np.maximum(np.hypot(sgo, sgg)[ok], 1e-3)
    assert np.abs(z).max() < 5.0, z
    assert (z ** 2).mean() < 3.5, (z ** 2).mean()
    assert go.max() > 1.5 and gg.max() > 1.5        # the first shell is resolved

    d = RGo.mean(axis=0) - RGg.mean(axis=0)          # per chain
    sem = d.std(ddof=1) / np.sqrt(d.size)
    assert abs(d.mean()) < 4.0 * sem + 1e-12, (d.mean(), sem)
