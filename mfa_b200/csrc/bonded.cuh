// Bonded force on one bead: FENE (intra_molec.f90) and bending (bending.f90,
// mode 2), evaluated by the thread that owns the bead.
//
// A bead's force comes from its two bonds and the three angles centred on it
// and on its two chain neighbours, so the thread reads the positions of beads
// i-2 .. i+2 of its chain (ids are contiguous per chain) and recomputes those
// terms; no other thread writes the bead's force, so nothing is atomic.  Each
// bond's energy is counted by its first bead, each angle's by its centre.
// Bond vectors are formed in FP64 from the FP64 positions; the force math runs
// in R (float in MIXED, double in FP64).
#pragma once
#include "mfa_internal.cuh"

struct BondParams {
    const double *rx, *ry, *rz;
    int n_chain, n_mon, n_chain_d, n_mon_d, part_init_d;
    int symmetry, do_fene, do_bend;
    double L[3], invL[3];
    double k_chain, k_ring, inv_r_chain_2, fene_clamp, k_bend, alpha_eq;
};

inline BondParams bond_params(const mfa_ctx* c, int do_fene, int do_bend) {
    const mfa_params& p = c->p;
    BondParams b;
    b.rx = c->rx; b.ry = c->ry; b.rz = c->rz;
    b.n_chain = p.n_chain; b.n_mon = p.n_mon; b.n_chain_d = p.n_chain_d; b.n_mon_d = p.n_mon_d;
    b.part_init_d = p.n_mon * p.n_chain;
    b.symmetry = p.symmetry;
    b.do_fene = do_fene;
    b.do_bend = do_bend && p.bending;
    for (int d = 0; d < 3; ++d) { b.L[d] = p.boundary[d]; b.invL[d] = c->inv_boundary[d]; }
    b.k_chain = p.k_chain; b.k_ring = p.k_ring; b.inv_r_chain_2 = p.inv_r_chain_2;
    b.fene_clamp = p.fene_clamp; b.k_bend = p.k_bend; b.alpha_eq = p.alpha_eq;
    return b;
}

namespace bonded {

// bending.f90:88-93: theta = acos(cos) (0 when cos >= 1).  In FP64 the
// reference's acos is used as is; in FP32 acos loses its accuracy as theta -> 0
// (a 6e-8 error in cos becomes 3.5e-4 rad), so the same angle is taken as
// atan2(|p x n|, p . n), which keeps full relative accuracy there.
__device__ __forceinline__ float angle_of(float c, float px, float py, float pz, float nx, float ny, float nz,
                                          float dot) {
    if (c >= 1.0f) return 0.0f;
    const float cx = py * nz - pz * ny, cy = pz * nx - px * nz, cz = px * ny - py * nx;
    return atan2f(sqrtf(cx * cx + cy * cy + cz * cz), dot);
}
__device__ __forceinline__ double angle_of(double c, double, double, double, double, double, double, double) {
    return c >= 1.0 ? 0.0 : acos(c);
}
__device__ __forceinline__ float log1m_(float x) { return logf(1.0f - x); }
__device__ __forceinline__ double log1m_(double x) { return log(1.0 - x); }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }

// image of r(k) - r(k+1) as intra_molec.f90:21-59 forms it (no z image in channels)
__device__ __forceinline__ double fene_image(double d, double L, double iL) {
    return d - L * (double)(int)(2.0 * d * iL);
}

// Angle centred on bead c with bond vectors p = r(c) - r(c-1), n = r(c+1) - r(c)
// (bending.f90:43-117): force on the previous bead (fp) and on the next bead
// (fn); the centre gets -(fp + fn).  Returns the energy 1/2 k (theta - alpha)^2.
template <typename R>
__device__ __forceinline__ double angle_forces(const BondParams& b, const R p[3], const R n[3], R fp[3], R fn[3]) {
    const R tiny = (R)1.0000000116860974e-07;   // 0.0000001 single-precision literal
    const R dot = n[0] * p[0] + n[1] * p[1] + n[2] * p[2];
    const R p2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    const R n2 = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    const R cosa = dot / sqrt_(p2 * n2);
    R dn[3], dp[3];
    for (int d = 0; d < 3; ++d) {
        dn[d] = p[d] * n2 - n[d] * dot;
        dp[d] = -n[d] * p2 + p[d] * dot;
    }
    const R dn2 = dn[0] * dn[0] + dn[1] * dn[1] + dn[2] * dn[2];
    const R dp2 = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
    if (dn2 < tiny) { dn[0] = dn[1] = dn[2] = 0; }
    else { const R s = (R)1 / sqrt_(dn2 * n2); dn[0] *= s; dn[1] *= s; dn[2] *= s; }
    if (dp2 < tiny) { dp[0] = dp[1] = dp[2] = 0; }
    else { const R s = (R)1 / sqrt_(dp2 * p2); dp[0] *= s; dp[1] *= s; dp[2] *= s; }
    const R da = cosa >= (R)1 ? (R)0 : angle_of(cosa, p[0], p[1], p[2], n[0], n[1], n[2], dot) - (R)b.alpha_eq;
    const R fm = (R)b.k_bend * da;
    for (int d = 0; d < 3; ++d) { fp[d] = fm * dp[d]; fn[d] = fm * dn[d]; }
    return (double)((R)0.5 * fm * da);
}

}  // namespace bonded

// Bonded force on bead i (adds to f); e_fene collects the bond potentials
// -1/2 ln(1 - x) of the bond starting at i (to be multiplied by k_chain,
// intra_molec.f90:96,270), e_bend the energy of the angle centred on i.
// The chain window i-2 .. i+2 is walked once, bond by bond, so that only two
// positions and two bond vectors are live at a time.
template <typename R, typename E>
__device__ __forceinline__ void bonded_on_bead(const BondParams& b, int i, R f[3], E& e_fene, E& e_bend,
                                               int& clamped) {
    using namespace bonded;
    int base, nm;
    R kf;
    bool bend;
    if (i < b.n_chain * b.n_mon) {
        base = (i / b.n_mon) * b.n_mon; nm = b.n_mon; kf = (R)b.k_chain; bend = b.do_bend != 0;
    } else if (b.n_mon_d >= 2 && i >= b.part_init_d && i < b.part_init_d + b.n_chain_d * b.n_mon_d) {
        base = b.part_init_d + ((i - b.part_init_d) / b.n_mon_d) * b.n_mon_d; nm = b.n_mon_d;
        kf = (R)b.k_ring; bend = false;
    } else {
        return;
    }
    const int pos = i - base;
    const int q0 = pos - 2 < 0 ? 0 : pos - 2;
    const int q1 = pos + 2 > nm - 1 ? nm - 1 : pos + 2;
    double px = b.rx[base + q0], py = b.ry[base + q0], pz = b.rz[base + q0];
    R w0 = 0, w1 = 0, w2 = 0;      // bending vector of the previous bond
    // bond j = (q-1, q), q = q0+1 .. q1
    for (int q = q0 + 1; q <= q1; ++q) {
        const double x = b.rx[base + q], y = b.ry[base + q], z = b.rz[base + q];
        const double d0 = px - x, d1 = py - y, d2 = pz - z;    // r(j) - r(j+1), j = q-1
        const int j = q - 1;
        if (b.do_fene && (j == pos - 1 || j == pos)) {
            // intra_molec.f90:21-59
            const R dx = (R)fene_image(d0, b.L[0], b.invL[0]);
            const R dy = (R)fene_image(d1, b.L[1], b.invL[1]);
            const R dz = (R)(b.symmetry == 1 ? fene_image(d2, b.L[2], b.invL[2]) : d2);
            const R irc2 = (R)b.inv_r_chain_2, clampv = (R)b.fene_clamp;
            const R r2 = dx * dx + dy * dy + dz * dz;
            R xx = r2 * irc2;
            const bool at_clamp = xx >= clampv;
            if (at_clamp) xx = clampv;
            const R fs = kf / ((R)1 - xx) * irc2;
            // bead j gets -fs d, bead j+1 gets +fs d
            const R sg = (j == pos) ? (R)-1 : (R)1;
            f[0] += sg * fs * dx;
            f[1] += sg * fs * dy;
            f[2] += sg * fs * dz;
            if (j == pos) {
                e_fene += (E)(-0.5 * (double)log1m_(xx));
                clamped += at_clamp ? 1 : 0;
            }
        }
        if (bend) {
            // bending.f90:34-57: r(j+1) - r(j), periodic in x, y and z
            const R v0 = (R)(-d0 + b.L[0] * (double)(int)(2.0 * d0 * b.invL[0]));
            const R v1 = (R)(-d1 + b.L[1] * (double)(int)(2.0 * d1 * b.invL[1]));
            const R v2 = (R)(-d2 + b.L[2] * (double)(int)(2.0 * d2 * b.invL[2]));
            // the angle centred on c = j with bonds (c-1, c) and (c, c+1)
            const int c = j;
            if (q > q0 + 1 && c >= 1 && c <= nm - 2 && c >= pos - 1 && c <= pos + 1) {
                const R pv[3] = {w0, w1, w2}, nv[3] = {v0, v1, v2};
                R fp[3], fn[3];
                const double e = angle_forces<R>(b, pv, nv, fp, fn);
                if (c == pos + 1) {          // this bead is the angle's previous bead
                    f[0] += fp[0]; f[1] += fp[1]; f[2] += fp[2];
                } else if (c == pos) {       // this bead is the centre
                    f[0] -= fp[0] + fn[0]; f[1] -= fp[1] + fn[1]; f[2] -= fp[2] + fn[2];
                    e_bend += (E)e;
                } else {                     // this bead is the angle's next bead
                    f[0] += fn[0]; f[1] += fn[1]; f[2] += fn[2];
                }
            }
            w0 = v0; w1 = v1; w2 = v2;
        }
        px = x; py = y; pz = z;
    }
}
