"""TEST INFRASTRUCTURE: numpy restatement of the reference's per-observation
quantities, the checker of mfa_observe / mfa_histogram_z.  Nothing in the
product imports it.

- refold: observation.f90:173-232 -- each chain bead is moved by one box
  length when it lies more than half a box from the (already moved) bead
  before it; brush chains (ids 1..part_init_d) only in SYMMETRY 0, melt or
  droplet chains (part_init_d+1..part_init_e) always; one move per bead and
  axis, as the reference does (``cycle`` after the first).
- radii of gyration: observation.f90:238-266 -- r_g2(1,:) over the n_chain
  brush chains of n_mon beads (centre of mass times inv_n_mon = 1/n_mon,
  init_obser.f90:121), r_g2(2,:) over chains n_chain+1..n_chain+n_chain_d
  taken as beads (i_chain-1)*n_mon_d+1..i_chain*n_mon_d, the reference's
  indexing (exact only when n_mon_d = n_mon or no brush precedes them);
  0/0 gives NaN when there are no such chains, as in the reference.
- total momentum: observation.f90:279-283, sum over all particles of m v.
- end-to-end vectors: functions.f90:626-667 (r_end_to_end_2v mode 2) -- chain
  c (0-based, brush then melt) runs from bead c*n_mon to c*n_mon + n_mon - 1
  of the unfolded coordinates (n_mon for the melt chains too, the
  reference's indexing); groups top brushes (c < n_chain // 2), bottom
  brushes, melt; sums divided by n_chain // 2 (both brush groups) and
  n_chain_d.
- head forces: observation.f90:326-328 -- minus the summed force on the
  heads of chains c < n_chain // 2 (upper wall) and of the others.
- z histogram: functions.f90:157-185 (histo mode 2) -- bin int(z / z_step) + 1
  clamped to 1..hist_dim, z_step = Lz / hist_dim, counted for the brush beads
  (column 0) and the melt/droplet beads (column 1).
"""
import numpy as np


def refold(r0, boundary, n_mon, n_chain, n_mon_d, n_chain_d, symmetry):
    """Bead by bead in id order, as the two loops of observation.f90:178-207
    run: bead i (0-based) moves unless i is a multiple of the chain length
    (global id, so a melt whose first id is not a multiple of n_mon_d starts
    its first run against the last brush bead, as in the reference)."""
    s = np.array(r0, dtype=np.float64, copy=True)
    L = np.asarray(boundary[:3], dtype=np.float64)
    half = L / 2.0                                    # init_config.f90:22
    pd = n_mon * n_chain
    pe = pd + n_mon_d * n_chain_d

    def move(i):
        for d in range(3):
            if s[i, d] - s[i - 1, d] > half[d]:
                s[i, d] -= L[d]
            elif s[i - 1, d] - s[i, d] > half[d]:
                s[i, d] += L[d]

    if symmetry == 0 and n_mon > 0:
        for i in range(pd):
            if i % n_mon != 0:
                move(i)
    if n_mon_d > 0:
        for i in range(pd, pe):
            if i % n_mon_d != 0:
                move(i)
    return s


def radii_of_gyration(spabs, n_mon, n_chain, n_mon_d, n_chain_d):
    rg = np.zeros((2, 3))
    inv_n_mon = 1.0 / n_mon if n_mon else 0.0
    for c in range(n_chain):
        seg = spabs[c * n_mon:(c + 1) * n_mon]
        cm = seg.sum(axis=0) * inv_n_mon
        rg[0] += ((seg - cm) ** 2).sum(axis=0) * inv_n_mon
    with np.errstate(invalid="ignore", divide="ignore"):
        rg[0] = rg[0] * (1.0 / n_chain if n_chain else np.nan)
        for c in range(n_chain, n_chain + n_chain_d):
            seg = spabs[c * n_mon_d:(c + 1) * n_mon_d]
            cm = seg.sum(axis=0) / float(n_mon_d)
            rg[1] += ((seg - cm) ** 2).sum(axis=0) / float(n_mon_d)
        rg[1] = rg[1] / float(n_chain_d)
    return rg


def momentum(v, mass):
    return (np.asarray(mass)[:, None] * np.asarray(v)).sum(axis=0)


def z_histogram(r0, boundary, hist_dim, n_mon, n_chain, n_mon_d, n_chain_d):
    z_step = float(boundary[2]) / float(hist_dim)
    inv = 1.0 / z_step
    pd = n_mon * n_chain
    pe = pd + n_mon_d * n_chain_d
    out = np.zeros((2, hist_dim))
    for col, (a, b) in enumerate(((0, pd), (pd, pe))):
        idx = np.trunc(np.asarray(r0)[a:b, 2] * inv).astype(np.int64) + 1
        idx = np.clip(idx, 1, hist_dim)
        np.add.at(out[col], idx - 1, 1.0)
    return out


def end_to_end(spabs, n_mon, n_chain, n_chain_d):
    """(r_ee, r_ee2), 3 groups x xyz each, as r_end_to_end_2v(2) forms them."""
    r_ee = np.zeros((3, 3))
    r_ee2 = np.zeros((3, 3))
    half = n_chain // 2
    for c in range(n_chain + n_chain_d):
        g = 0 if c < half else (1 if c < n_chain else 2)
        v = spabs[c * n_mon + n_mon - 1] - spabs[c * n_mon]
        r_ee[g] += v
        r_ee2[g] += v * v
    with np.errstate(invalid="ignore", divide="ignore"):
        for g, cnt in ((0, half), (1, half), (2, n_chain_d)):
            r_ee[g] = r_ee[g] / float(cnt)
            r_ee2[g] = r_ee2[g] / float(cnt)
    return r_ee, r_ee2


def head_forces(force_on_heads, n_chain):
    """Minus the summed head force of the upper-wall and lower-wall chains."""
    f = np.asarray(force_on_heads, dtype=np.float64).reshape(n_chain, 3)
    half = n_chain // 2
    return np.stack([-f[:half].sum(axis=0), -f[half:].sum(axis=0)])
