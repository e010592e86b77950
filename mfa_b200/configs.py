"""Seeded initial configurations for the benchmark systems.

These stand in for the reference's generators (gen_chain.f90, gen_brush.f90,
gen_droplet.f90), which draw from the R250 stream and cannot be replayed.  All
placements use random sequential addition with the same rule the workloads
state: a bead is rejected if it comes closer than ``r_min`` (0.8 sigma) to any
bead already placed (minimum image in the periodic directions).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np
from scipy.spatial import cKDTree

from . import _abi
from .params import Spec, derive


@dataclass
class Config:
    """A generated system: raw spec, derived params and particle arrays (reference layouts)."""

    name: str
    spec: Spec
    params: _abi.MfaParams
    r0: np.ndarray       # (n, 3) float64
    v: np.ndarray        # (n, 3)
    a_type: np.ndarray   # (n,) int32, 1-based
    mass: np.ndarray     # (n,)
    q: Optional[np.ndarray] = None

    @property
    def n(self) -> int:
        return self.r0.shape[0]


class _Grid:
    """Overlap rejection against all beads placed so far (k-d tree, periodic
    wrap in the periodic directions)."""

    def __init__(self, box, periodic, r_min):
        self.box = np.asarray(box, dtype=np.float64)
        self.periodic = np.asarray(periodic, dtype=bool)
        self.r_min = float(r_min)
        # a non-periodic axis gets a wrap length far beyond the box, so no image is near
        self.wrap = np.where(self.periodic, self.box, self.box + 10.0 * r_min)
        self.pos = np.zeros((0, 3))
        self.alive = np.zeros(0, dtype=bool)
        self._tree = None
        self._tree_ids = None

    def _current(self):
        if self._tree is None:
            ids = np.nonzero(self.alive)[0]
            self._tree_ids = ids
            self._tree = cKDTree(np.mod(self.pos[ids], self.wrap), boxsize=self.wrap) if ids.size else None
        return self._tree

    def conflicts(self, x):
        """bool per point: closer than r_min to a placed bead."""
        tree = self._current()
        if tree is None:
            return np.zeros(x.shape[0], dtype=bool)
        d, _ = tree.query(np.mod(x, self.wrap), k=1, distance_upper_bound=self.r_min)
        return d < self.r_min

    def try_add(self, x):
        """Add the candidates that keep r >= r_min to everything (incl. each other,
        earlier candidates winning).  Returns each candidate's index, -1 if rejected."""
        x = np.mod(np.asarray(x, dtype=np.float64), self.wrap)
        out = -np.ones(x.shape[0], dtype=np.int64)
        tree = self._current()
        if tree is not None:
            d, _ = tree.query(x, k=1, distance_upper_bound=self.r_min)
            ok = ~(d < self.r_min)
        else:
            ok = np.ones(x.shape[0], dtype=bool)
        cand = np.nonzero(ok)[0]
        if cand.size == 0:
            return out
        if cand.size > 1:
            pairs = cKDTree(x[cand], boxsize=self.wrap).query_pairs(self.r_min, output_type="ndarray")
            if pairs.size:
                drop = np.zeros(cand.size, dtype=bool)
                drop[np.maximum(pairs[:, 0], pairs[:, 1])] = True
                cand = cand[~drop]
        base = self.pos.shape[0]
        out[cand] = base + np.arange(cand.size)
        self.pos = np.concatenate([self.pos, x[cand]], axis=0)
        self.alive = np.concatenate([self.alive, np.ones(cand.size, dtype=bool)])
        self._tree = None
        return out

    def remove(self, idx):
        """Withdraw beads idx."""
        self.alive[np.asarray(idx, dtype=np.int64)] = False
        self._tree = None


def _place_free(rng, grid, count, lo, hi, batch=40000):
    """count uniformly random beads in [lo, hi) that pass the overlap rule."""
    pts, ids = [], []
    got = 0
    stall = 0
    while got < count:
        m = min(batch, 4 * (count - got) + 16)
        cand = lo + rng.random((m, 3)) * (hi - lo)
        idx = grid.try_add(cand)
        acc = idx >= 0
        need = count - got
        sel = np.nonzero(acc)[0]
        if sel.size > need:
            grid.remove(idx[sel[need:]])
            sel = sel[:need]
        pts.append(cand[sel])
        ids.append(idx[sel])
        got += sel.size
        stall = stall + 1 if sel.size == 0 else 0
        if stall > 100:
            raise RuntimeError("random insertion stalled")
    return np.concatenate(pts, axis=0), np.concatenate(ids)


def _random_dirs(rng, m, bias=None):
    v = rng.normal(size=(m, 3))
    if bias is not None:
        v = v / np.linalg.norm(v, axis=1, keepdims=True) + np.asarray(bias)[None, :]
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _grow_chains(rng, grid, heads, head_ids, n_mon, bond, box, periodic, zlim=None,
                 tries=24, patience=8, max_rounds=100000, bias=None):
    """Grow all chains one bead per round from their (already placed) heads.

    Each round every unfinished chain draws `tries` candidate steps and keeps the
    first one that passes the overlap rule.  A chain that finds none `patience`
    rounds in a row gives back its last beads (never the head; more each time it
    gets stuck again) and regrows them.  `bias` (a vector added to the unit step
    before normalising) makes grafted chains grow away from the wall, as the
    reference's gen_brush.f90:57-66 does with its fixed z step."""
    n_chain = heads.shape[0]
    chains = np.zeros((n_chain, n_mon, 3))
    gid = -np.ones((n_chain, n_mon), dtype=np.int64)
    chains[:, 0] = heads
    gid[:, 0] = head_ids
    length = np.ones(n_chain, dtype=np.int64)
    fails = np.zeros(n_chain, dtype=np.int64)
    backs = np.zeros(n_chain, dtype=np.int64)
    for _ in range(max_rounds):
        todo = np.nonzero(length < n_mon)[0]
        if todo.size == 0:
            return chains
        prev = chains[todo, length[todo] - 1]
        cand = prev[:, None, :] + bond * _random_dirs(rng, todo.size * tries, bias).reshape(todo.size, tries, 3)
        ok = np.ones(cand.shape[:2], dtype=bool)
        if zlim is not None:
            # brush chains stay between the walls
            ok &= (cand[..., 2] >= zlim[0]) & (cand[..., 2] <= zlim[1])
        for d in range(3):
            if periodic[d]:
                cand[..., d] %= box[d]
        ok &= ~grid.conflicts(cand.reshape(-1, 3)).reshape(ok.shape)
        has = ok.any(axis=1)
        first = np.argmax(ok, axis=1)
        pick = cand[np.arange(todo.size), first]
        idx = -np.ones(todo.size, dtype=np.int64)
        if has.any():
            sub = np.nonzero(has)[0]
            idx[sub] = grid.try_add(pick[sub])
        acc = idx >= 0
        ch = todo[acc]
        chains[ch, length[ch]] = pick[acc]
        gid[ch, length[ch]] = idx[acc]
        length[ch] += 1
        fails[ch] = 0
        backs[ch[length[ch] == n_mon]] = 0
        rej = todo[~has]
        fails[rej] += 1
        back = rej[(fails[rej] > patience) & (length[rej] > 1)]
        for k in back:
            # give back more beads each time the same chain gets stuck again
            nb = int(min(length[k] - 1, 2 + backs[k]))
            grid.remove(gid[k, length[k] - nb:length[k]])
            gid[k, length[k] - nb:length[k]] = -1
            length[k] -= nb
            fails[k] = 0
            backs[k] += 1
    raise RuntimeError("chain growth did not finish")


def _maxwell(rng, mass, temp):
    v = rng.normal(size=(mass.size, 3)) * np.sqrt(temp / mass)[:, None]
    p = (v * mass[:, None]).sum(0) / mass.sum()
    return v - p[None, :]


def melt(seed: int = 12345, n_chain: int = 100, n_mon: int = 32, density: float = 0.85,
         skin: float = 0.3, thermostat: int = _abi.THERMO_DPD, friction: float = 4.5,
         noise: int = _abi.NOISE_GAUSS) -> Config:
    """Bead-spring melt: n_chain x n_mon beads, cubic periodic box, WCA + FENE + DPD.

    Chains are stored in the grafted/bulk-chain segment (ids 1..n_mon*n_chain),
    which the reference bonds with k_chain (intra_molec.f90:16-96)."""
    rng = np.random.default_rng(seed)
    n = n_chain * n_mon
    L = (n / density) ** (1.0 / 3.0)
    box = np.array([L, L, L])
    periodic = np.array([True, True, True])
    grid = _Grid(box, periodic, 0.8)
    heads, hid = _place_free(rng, grid, n_chain, np.zeros(3), box)
    chains = _grow_chains(rng, grid, heads, hid, n_mon, 0.97, box, periodic)
    r0 = chains.reshape(-1, 3).copy()
    mass = np.ones(n)
    spec = Spec(n_part=n, boundary=box, n_type=1, n_mon=n_mon, n_chain=n_chain, symmetry=1,
                thermostat=thermostat, friction=friction, skin=skin, dt=0.005, temp=1.0,
                k_chain_in=30.0, r_chain=1.5, noise=noise, seed=seed)
    return Config("melt", spec, derive(spec), r0, _maxwell(rng, mass, 1.0),
                  np.ones(n, dtype=np.int32), mass)


def brush(seed: int = 12345, nx: int = 32, ny: int = 32, n_mon: int = 64, graft: float = 0.3,
          z_wall: float = 60.0, density: float = 0.85, solvent: bool = True, skin: float = 0.3,
          k_bend: float = 2.0, wall_cut: float = 2.5, friction: float = 4.5,
          thermostat: int = _abi.THERMO_DPD, z_head: float = 1.0, batch: int = 40000) -> Config:
    """Polymer brush between 9-3 walls, optionally with explicit solvent.

    Types: 1 = grafted head (pinned), 2 = brush monomer, 3 = solvent,
    4 = wall type (cutoffs to it zeroed, as the reference does for WALL 2).
    Heads sit on a square lattice at z = z_head (all on the bottom wall)."""
    rng = np.random.default_rng(seed)
    a = math.sqrt(1.0 / graft)
    Lx, Ly = nx * a, ny * a
    box = np.array([Lx, Ly, z_wall])
    periodic = np.array([True, True, False])
    grid = _Grid(box, periodic, 0.8)
    gx, gy = np.meshgrid((np.arange(nx) + 0.5) * a, (np.arange(ny) + 0.5) * a, indexing="ij")
    heads = np.stack([gx.ravel(), gy.ravel(), np.full(nx * ny, z_head)], axis=1)
    hid = grid.try_add(heads)
    assert (hid >= 0).all()
    chains = _grow_chains(rng, grid, heads, hid, n_mon, 0.97, box, periodic, zlim=(0.9, z_wall - 0.9),
                          bias=(0.0, 0.0, 0.7))
    n_brush = nx * ny * n_mon
    parts = [chains.reshape(-1, 3)]
    n_solv = 0
    if solvent:
        target = int(round(density * Lx * Ly * z_wall)) - n_brush
        placed = []
        got = 0
        lo = np.array([0.0, 0.0, 0.9])
        hi = np.array([Lx, Ly, z_wall - 0.9])
        stall = 0
        while got < target:
            m = min(batch, 4 * (target - got) + 64)
            cand = lo + rng.random((m, 3)) * (hi - lo)
            acc = grid.try_add(cand) >= 0
            take = cand[acc][: target - got]
            placed.append(take)
            got += take.shape[0]
            stall = stall + 1 if take.shape[0] == 0 else 0
            if stall > 50:
                raise RuntimeError("solvent insertion stalled")
        parts.append(np.concatenate(placed, axis=0))
        n_solv = got
    r0 = np.concatenate(parts, axis=0)
    n = r0.shape[0]
    a_type = np.full(n, 3, dtype=np.int32)
    a_type[:n_brush] = 2
    a_type[0:n_brush:n_mon] = 1
    mass = np.ones(n)
    v = _maxwell(rng, mass, 1.0)
    v[0:n_brush:n_mon] = 0.0
    n_type = 4
    eps = np.ones((n_type, n_type))
    eps[0, 0] = 0.0
    spec = Spec(n_part=n, boundary=box, n_type=n_type, n_mon=n_mon, n_chain=nx * ny,
                n_mon_d=1, n_chain_d=n_solv, symmetry=0, thermostat=thermostat, friction=friction,
                wall=2, bending=1 if k_bend else 0, pin_heads=1, eps=eps, brush_heads=True,
                wall93_zero_last_type=True, skin=skin, dt=0.005, temp=1.0, k_chain_in=30.0,
                r_chain=1.5, k_bend=k_bend, alpha_eq=0.0, a_w=1.0, sigma_w=1.0, z_head=z_head,
                wall_cut=wall_cut, seed=seed)
    return Config("brush" if solvent else "brush_implicit", spec, derive(spec), r0, v, a_type, mass)


def charged(seed: int = 12345, n_chain: int = 200, n_mon: int = 50, density: float = 0.5,
            alpha: float = 0.8, rc_real: float = 3.5, n_kmax: int = 10, skin: float = 0.3,
            reference_mode: bool = False, friction: float = 0.5,
            thermostat: int = _abi.THERMO_LGV) -> Config:
    """Polyelectrolyte chains (charge -1 on every second bead) plus monovalent
    counterions in a cubic periodic box, Ewald sums (alpha_c = alpha^2).

    Types: 1 = neutral bead, 2 = charged bead (-1), 3 = counterion (+1).
    reference_mode=True evaluates Ewald real space only inside the LJ range and
    uses 1/pi for 1/sqrt(pi), as the reference does (fluid_fluid.f90:94,166;
    init_config.f90:230)."""
    rng = np.random.default_rng(seed)
    n_poly = n_chain * n_mon
    n_ci = n_poly // 2
    n = n_poly + n_ci
    L = (n / density) ** (1.0 / 3.0)
    box = np.array([L, L, L])
    periodic = np.array([True, True, True])
    grid = _Grid(box, periodic, 0.8)
    heads, hid = _place_free(rng, grid, n_chain, np.zeros(3), box)
    chains = _grow_chains(rng, grid, heads, hid, n_mon, 0.97, box, periodic)
    ci, _ = _place_free(rng, grid, n_ci, np.zeros(3), box)
    r0 = np.concatenate([chains.reshape(-1, 3), ci], axis=0)
    a_type = np.ones(n, dtype=np.int32)
    a_type[1:n_poly:2] = 2
    a_type[n_poly:] = 3
    charge = {1: 0.0, 2: -1.0, 3: 1.0}
    q = np.array([charge[t] for t in a_type])
    mass = np.ones(n)
    quirks = _abi.Q_WALL_ENERGY_AW | (_abi.Q_EWALD_REAL_IN_LJ if reference_mode else 0)
    spec = Spec(n_part=n, boundary=box, n_type=3, n_mon=n_mon, n_chain=n_chain, symmetry=1,
                thermostat=thermostat, friction=friction, charged=1, skin=skin, dt=0.005, temp=1.0,
                k_chain_in=30.0, r_chain=1.5, alpha_c=alpha * alpha, n_kmax=n_kmax,
                ewald_rc=rc_real, quirks=quirks, seed=seed)
    p = derive(spec)
    if not reference_mode:
        p.inv_sqrt_pi = 1.0 / math.sqrt(p.pi)
        # cells large enough for the real-space cutoff
        for d in range(3):
            p.n_bin[d] = max(1, int(L / (rc_real + skin)))
            p.delta_bin[d] = 1 if p.n_bin[d] >= 3 else (0 if p.n_bin[d] == 2 else -1)
    return Config("charged", spec, p, r0, _maxwell(rng, mass, 1.0), a_type, mass, q)


def charged_slab(seed: int = 12345, n_chain: int = 20, n_mon: int = 20, density: float = 0.5,
                 z_wall: float = 12.0, alpha: float = 0.8, rc_real: float = 3.0, n_kmax: int = 4,
                 skin: float = 0.3, friction: float = 0.5, thermostat: int = _abi.THERMO_LGV) -> Config:
    """Polyelectrolyte chains (charge -1 on every second bead) and monovalent
    counterions between two 9-3 walls at z = 0 and z = z_wall: the charged
    channel (SYMMETRY 0, WALL 2) whose Ewald sum takes the slab k-set
    (ewald_k.f90:41-46, an empty gap of twice the channel width in z) and the
    dipolar correction of dipolar_correction.f90.

    Types: 1 = neutral bead, 2 = charged bead (-1), 3 = counterion (+1)."""
    rng = np.random.default_rng(seed)
    n_poly = n_chain * n_mon
    n_ci = n_poly // 2
    n = n_poly + n_ci
    lxy = math.sqrt(n / (density * z_wall))
    box = np.array([lxy, lxy, z_wall])
    periodic = np.array([True, True, False])
    grid = _Grid(box, periodic, 0.8)
    lo, hi = np.array([0.0, 0.0, 0.9]), np.array([lxy, lxy, z_wall - 0.9])
    heads, hid = _place_free(rng, grid, n_chain, lo, hi)
    chains = _grow_chains(rng, grid, heads, hid, n_mon, 0.97, box, periodic, zlim=(0.9, z_wall - 0.9))
    ci, _ = _place_free(rng, grid, n_ci, lo, hi)
    r0 = np.concatenate([chains.reshape(-1, 3), ci], axis=0)
    a_type = np.ones(n, dtype=np.int32)
    a_type[1:n_poly:2] = 2
    a_type[n_poly:] = 3
    charge = {1: 0.0, 2: -1.0, 3: 1.0}
    q = np.array([charge[t] for t in a_type])
    mass = np.ones(n)
    spec = Spec(n_part=n, boundary=box, n_type=3, n_mon=n_mon, n_chain=n_chain, symmetry=0, wall=2,
                thermostat=thermostat, friction=friction, charged=1, skin=skin, dt=0.005, temp=1.0,
                k_chain_in=30.0, r_chain=1.5, alpha_c=alpha * alpha, n_kmax=n_kmax, ewald_rc=rc_real,
                wall_cut=2.5, quirks=_abi.Q_WALL_ENERGY_AW, seed=seed)
    p = derive(spec)
    p.inv_sqrt_pi = 1.0 / math.sqrt(p.pi)
    for d in range(3):
        p.n_bin[d] = max(1, int(box[d] / (rc_real + skin)))
        p.delta_bin[d] = 1 if p.n_bin[d] >= 3 else (0 if p.n_bin[d] == 2 else -1)
    return Config("charged_slab", spec, p, r0, _maxwell(rng, mass, 1.0), a_type, mass, q)


def brush_stretched(seed: int = 12345, nx: int = 16, ny: int = 16, n_mon: int = 64, graft: float = 0.3,
                    z_wall: Optional[float] = None, friction: float = 4.5, skin: float = 0.3,
                    z_head: float = 1.0, jitter: float = 0.15) -> Config:
    """Implicit-solvent brush between 9-3 walls, chains started fully stretched.

    Heads sit on a square lattice at z = z_head (grafting density `graft`);
    bead k of a chain sits at height z_head + 0.97 k above its head with an
    independent lateral jitter of at most `jitter` per bead.  With lattice
    spacing 1/sqrt(graft) >= 1.41 sigma (graft <= 0.5) beads of different
    chains stay more than 0.8 sigma apart and bonds stay below 1.1 sigma, so
    the start is overlap-free by construction at every grafting density (a
    random-walk growth stalls in dense brushes).  The wall gap defaults to
    2.2 x the chain length.  Types: 1 = pinned head, 2 = monomer; WCA
    everywhere, FENE (k = 30, R0 = 1.5), no bending, DPD gamma = friction."""
    rng = np.random.default_rng(seed)
    if z_wall is None:
        z_wall = 2.2 * n_mon
    a = math.sqrt(1.0 / graft)
    Lx, Ly = nx * a, ny * a
    gx, gy = np.meshgrid((np.arange(nx) + 0.5) * a, (np.arange(ny) + 0.5) * a, indexing="ij")
    heads = np.stack([gx.ravel(), gy.ravel()], axis=1)
    n_chain = nx * ny
    k = np.arange(n_mon)
    r0 = np.empty((n_chain, n_mon, 3))
    r0[:, :, 0] = heads[:, None, 0]
    r0[:, :, 1] = heads[:, None, 1]
    r0[:, :, 2] = z_head + 0.97 * k[None, :]
    jit = rng.uniform(-jitter, jitter, size=(n_chain, n_mon, 2))
    jit[:, 0, :] = 0.0
    r0[:, :, :2] += jit
    r0[:, :, 0] %= Lx
    r0[:, :, 1] %= Ly
    r0 = r0.reshape(-1, 3)
    n = r0.shape[0]
    a_type = np.full(n, 2, dtype=np.int32)
    a_type[0:n:n_mon] = 1
    mass = np.ones(n)
    v = _maxwell(rng, mass, 1.0)
    v[0:n:n_mon] = 0.0
    eps = np.ones((3, 3))
    eps[0, 0] = 0.0
    spec = Spec(n_part=n, boundary=np.array([Lx, Ly, z_wall]), n_type=3, n_mon=n_mon, n_chain=n_chain,
                symmetry=0, thermostat=_abi.THERMO_DPD, friction=friction, wall=2, bending=0, pin_heads=1,
                eps=eps, brush_heads=True, wall93_zero_last_type=True, skin=skin, dt=0.005, temp=1.0,
                k_chain_in=30.0, r_chain=1.5, k_bend=0.0, alpha_eq=0.0, a_w=1.0, sigma_w=1.0, z_head=z_head,
                wall_cut=2.5, seed=seed)
    return Config("brush_stretched", spec, derive(spec), r0, v, a_type, mass)


def uneven_brushes(seed: int = 2024, n_sys: int = 64, grids=(8, 24), lengths=(16, 32, 64, 128),
                   graft=(0.05, 0.5)):
    """Independent implicit-solvent brushes of uneven size for one batched run:
    per system a grafting density ~ U(graft), a chain length drawn from
    `lengths`, a square lateral grid of n x n chains with n ~ U{grids}, walls
    2.2 x the chain length apart, DPD noise seeded per system (seed + 1 + s).
    Returns the list of Configs (brush_stretched)."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_sys):
        g = float(rng.uniform(*graft))
        nm = int(rng.choice(lengths))
        nx = int(rng.integers(grids[0], grids[1] + 1))
        out.append(brush_stretched(seed=seed + 1 + s, nx=nx, ny=nx, n_mon=nm, graft=g))
    return out
