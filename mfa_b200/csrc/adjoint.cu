// Adjoint of the time-step loop: gradients of a trajectory observable with
// respect to the force-field parameters, by reverse-mode differentiation of
// the discrete velocity-Verlet map that mfa_step runs.
//
// Forward step n -> n+1 (verlet_positions, forces, verlet_velocities):
//   r' = r + dt v + dt^2/2 a          u = v + dt/2 a         (half-step velocity)
//   F' = F(r', u; theta, noise of step n+1)                  (DPD uses u)
//   a' = F'/m                          v' = u + dt/2 a'       (pinned heads: v' = a' = 0)
// Observable J = 1/S sum_{s=1..S} O(r_s), O = <z> (all beads, z unfolded) + <R_ee^2> (chains).
// Backward step n+1 -> n, with rho, nu, alpha the adjoints of r, v, a:
//   lam_F = (alpha' + dt/2 nu') / m,  lam_u = nu'            (heads: 0)
//   lam_r = rho' + (dF/dr')^T lam_F,  lam_u += (dF/du)^T lam_F,  g += (dF/dtheta)^T lam_F
//   rho = lam_r + 1/S dO/dr (s >= 1),  nu = dt lam_r + lam_u,  alpha = dt^2/2 lam_r + dt/2 lam_u
// The vector-Jacobian products are written out by hand for every force term
// of the path: WCA/LJ and DPD pairs (half list, Newton's third law), FENE bonds
// (with the clamp of intra_molec.f90:44), the bending angles of bending.f90
// (forward-mode derivative of the angle force) and the 9-3 walls.  The forward
// states are recomputed segment by segment from checkpoints every K steps, with
// the DPD noise replayed: Philox is keyed by (step, pair), so the recomputed
// forces are those of the first pass.
//
// theta = (eps_LJ, sigma, k_FENE, R0, gamma_DPD, eps_wall), defined as:
//   eps_LJ    all pair epsilons scale with it (epsil = 4 eps e_ij)
//   sigma     all pair sigmas scale with it (sigma_2, range_2 = (2^(1/6) sigma)^2,
//             hence the DPD range); the wall's sigma_wall is not changed
//   k_FENE    k_chain = k R0^2;      R0: r_chain_2 = R0^2 (and k_chain = k R0^2)
//   gamma     friction, and sig = sqrt(2 kT gamma / dt)
//   eps_wall  a_wall of every particle type (and a_w)
#include "mfa_internal.cuh"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

namespace {

enum { G_EPS = 0, G_SIG = 1, G_K = 2, G_R0 = 3, G_GAM = 4, G_WALL = 5, G_N = 6 };

struct AdjArgs {
    const void* pos_s;            // sorted records of r' (w: id << 8 | type)
    const void* vel_s;            // sorted records of u
    const int32_t* __restrict__ nbr;
    const int32_t* __restrict__ ccount;   // entries per 32-slot chunk
    const double* tabs;           // list radius, range_2, epsil, sigma_2, e_shift, inv_range_2
    const double *fx, *fy, *fz;   // lam_F (particle order)
    double *rx, *ry, *rz;         // lam_r accumulators
    double *ux, *uy, *uz;         // lam_u accumulators
    double* g;                    // G_N parameter gradient sums
    const double* mass;           // particle order (Langevin)
    int n, maxnb, half, symmetry, dpd, dpd_weight, noise, wall;
    int lgv;                      // Langevin thermostat (lgv_forces.f90)
    int split;                    // pieces per chunk list (a warp each)
    int charged, real_in_lj;      // Ewald real space: inside the LJ range, or to its own cutoff
    double L[3], invL[3];
    double sig, gam, eps_lj, sigma_lj;
    double sqrt_alpha, alpha_c, inv_sqrt_pi, ewald_rc_2;
    long long step;
    const int64_t* step_ptr;      // the step of the recomputed forward pass (device), or null: step
    PhiloxKeys key;
    uint32_t seed0, seed1;
    double a_wall[T8], sigma_wall[T8], z_space_wall, wall_cut;
};

template <typename R> struct V4;
template <> struct V4<float> { typedef float4 T; };
template <> struct V4<double> { typedef double4 T; };

__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsq(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float mi(float d, float L, float iL) { return fmaf(-L, truncf(2.0f * d * iL), d); }
__device__ __forceinline__ double mi(double d, double L, double iL) { return d - L * (double)(int)(2.0 * d * iL); }

// the DPD variate of a pair, exactly as the pair kernel draws it
__device__ __forceinline__ float dpd_noise(uint32_t x0, uint32_t x1, int shape, float) {
    if (shape == MFA_NOISE_UNIFORM) {
        const float u = (float)(x0 >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f;
        return 1.7320508075688772f * (2.0f * u - 1.0f);
    }
    const float u1 = fmaf((float)x0, 2.3283064365386963e-10f, 1.16415321826934814e-10f);
    const float u2 = fmaf((float)x1, 2.3283064365386963e-10f, 1.16415321826934814e-10f);
    const float s = -2.0f * __logf(u1);
    const float r = s > 0.0f ? s * rsqrtf(s) : 0.0f;
    return -r * __cosf(fmaf(6.283185307179586f, u2, -3.14159265358979f));
}
__device__ __forceinline__ double dpd_noise(uint32_t x0, uint32_t x1, int shape, double) {
    if (shape == MFA_NOISE_UNIFORM) {
        const float u = (float)(x0 >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f;
        return (double)(1.7320508075688772f * (2.0f * u - 1.0f));
    }
    const double u1 = ((double)x0 + 0.5) * 2.3283064365386963e-10;
    const double u2 = ((double)x1 + 0.5) * 2.3283064365386963e-10;
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

__device__ __forceinline__ void warp_add_g(double* g, double (&gl)[G_N]) {
#pragma unroll
    for (int q = 0; q < G_N; ++q) {
        double x = gl[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(&g[q], x);
    }
}

// Pair and wall VJP: a warp per piece of a 32-slot chunk's list (the list cut
// into `split` runs of equal length), its lanes over the piece's entries
// (owner and partner both updated through atomics); the warp of a chunk's
// first piece then goes over the chunk's slots for the walls and Langevin.
template <typename R>
__global__ void k_adj_pair(AdjArgs a) {
    typedef typename V4<R>::T R4;
    __shared__ double s_rc2[T8 * T8], s_eps[T8 * T8], s_sig2[T8 * T8], s_irc2[T8 * T8];
    for (int k = threadIdx.x; k < T8 * T8; k += blockDim.x) {
        s_rc2[k] = a.tabs[1 * T8 * T8 + k];
        s_eps[k] = a.tabs[2 * T8 * T8 + k];
        s_sig2[k] = a.tabs[3 * T8 * T8 + k];
        s_irc2[k] = a.tabs[5 * T8 * T8 + k];
    }
    __syncthreads();
    double gl[G_N] = {0, 0, 0, 0, 0, 0};
    const int lane = threadIdx.x & 31;
    const int piece = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int ch = piece / a.split, part = piece - ch * a.split;
    const long long step = a.step_ptr ? *a.step_ptr : a.step;
    const R4* ps = (const R4*)a.pos_s;
    const R4* vs = (const R4*)a.vel_s;
    const R Lx = (R)a.L[0], Ly = (R)a.L[1], Lz = (R)a.L[2];
    const R iLx = (R)a.invL[0], iLy = (R)a.invL[1], iLz = (R)a.invL[2];
    const R sg = (R)a.sig, gm = (R)a.gam;
    if (ch * 32 < a.n) {
        const int cnt = a.ccount[ch];
        const int eb = (int)(((long long)cnt * part) / a.split);
        const int ee = (int)(((long long)cnt * (part + 1)) / a.split);
        const int32_t* crow = a.nbr + (size_t)ch * 32 * a.maxnb;
        for (int e = eb + lane; e < ee; e += 32) {
            const int ent = crow[e];
            const int t = ch * 32 + (ent & 31), s = (int)((unsigned)ent >> 5);
            const R4 pi = ps[t], pj = ps[s];
            const int wi = wbits(pi.w), ii = wi >> 8, ti = wi & 0xff;
            R dx = mi(pi.x - pj.x, Lx, iLx), dy = mi(pi.y - pj.y, Ly, iLy), dz = pi.z - pj.z;
            if (a.symmetry == 1) dz = mi(dz, Lz, iLz);
            const R r2 = dx * dx + dy * dy + dz * dz;
            const int wj = wbits(pj.w), jj = wj >> 8, ij = (ti - 1) * T8 + (wj & 0xff) - 1;
            const bool in_lj = r2 < (R)s_rc2[ij];
            // Ewald real space (ewald_real.f90:15-33): inside the LJ range in the
            // reference's form (fluid_fluid.f90:94,166), else to its own cutoff
            const bool in_q = a.charged && (a.real_in_lj ? in_lj : r2 < (R)a.ewald_rc_2);
            if (!in_lj && !in_q) continue;
            // the pair force G acts on i (+G) and, with the half list, on j (-G):
            // dl = lam_F_i - lam_F_j (half list) or lam_F_i (full list: j has its own row)
            R dlx = (R)a.fx[ii], dly = (R)a.fy[ii], dlz = (R)a.fz[ii];
            if (a.half) { dlx -= (R)a.fx[jj]; dly -= (R)a.fy[jj]; dlz -= (R)a.fz[jj]; }
            const R ddl = dx * dlx + dy * dly + dz * dlz;
            R gx = 0, gy = 0, gz = 0;
            if (in_q) {
                // G = h(r) d, h = qq (2 s c exp(-a r^2) / r^2 + erfc(s r) / r^3), s = sqrt(a),
                // c the code's 1/sqrt(pi) constant; (dG/dd)^T dl = h dl + (h'(r) / r) (d . dl) d,
                // with d erfc(s r)/dr = -(2/sqrt(pi)) s exp(-a r^2) (the function's own derivative)
                const R4 ui = vs[t], uj = vs[s];
                const R qq = ui.w * uj.w;
                const R ir = rsq(r2), r = r2 * ir, ir2 = ir * ir, ir3 = ir2 * ir;
                const R SQA = (R)a.sqrt_alpha, ALC = (R)a.alpha_c, ISP = (R)a.inv_sqrt_pi;
                const R ex = exp(-ALC * r2), ec = erfc(SQA * r);
                const R h = qq * ((R)2 * SQA * ISP * ex * ir2 + ec * ir3);
                const R dh = qq * ((R)2 * SQA * ISP * ex * ((R)-2 * ALC * ir - (R)2 * ir3) -
                                   (R)1.1283791670955126 * SQA * ex * ir3 - (R)3 * ec * ir3 * ir);
                const R c = dh * ir * ddl;
                gx += h * dlx + c * dx;
                gy += h * dly + c * dy;
                gz += h * dlz + c * dz;
            }
            if (in_lj) {
            // LJ: G = fs(r2) d, fs = eps (12 r12 - 6 r6) / r2
            const R eps = (R)s_eps[ij], ir2 = (R)1 / r2;
            const R r61 = (R)s_sig2[ij] * ir2, r6 = r61 * r61 * r61, r12 = r6 * r6;
            const R fs = eps * ((R)12 * r12 - (R)6 * r6) * ir2;
            const R dfs = eps * ((R)-84 * r12 + (R)24 * r6) * ir2 * ir2;   // d fs / d r2
            gx += fs * dlx + (R)2 * dfs * ddl * dx;
            gy += fs * dly + (R)2 * dfs * ddl * dy;
            gz += fs * dlz + (R)2 * dfs * ddl * dz;
            gl[G_EPS] += (double)(fs * ddl) / a.eps_lj;
            gl[G_SIG] += (double)(eps * ((R)144 * r12 - (R)36 * r6) * ir2 * ddl) / a.sigma_lj;
            if (a.dpd) {
                // DPD: G = P rhat, P = sig w_r g - gamma w_d (du . rhat), w_d = w_r^2
                const R4 ui = vs[t], uj = vs[s];
                const R dux = ui.x - uj.x, duy = ui.y - uj.y, duz = ui.z - uj.z;
                const R ir = rsq(r2), r = r2 * ir;
                const R hx = dx * ir, hy = dy * ir, hz = dz * ir;
                const R sdu = dux * hx + duy * hy + duz * hz;
                const R hdl = hx * dlx + hy * dly + hz * dlz;
                const uint32_t lo = (uint32_t)min(ii, jj), hi = (uint32_t)max(ii, jj);
                const uint4 ph = philox4x32_10(make_uint4(lo, hi, (uint32_t)step, TAG_DPD), a.key);
                const R gn = dpd_noise(ph.x, ph.y, a.noise, R(0));
                const R irc = sqrt((R)s_irc2[ij]);
                R wr, wd, dwr, dwd;                  // weights and d/dr
                if (a.dpd_weight == 1) { wr = 1; wd = 1; dwr = 0; dwd = 0; }
                else { wr = (R)1 - r * irc; wd = wr * wr; dwr = -irc; dwd = (R)2 * wr * dwr; }
                const R P = sg * wr * gn - gm * wd * sdu;
                const R dP = sg * dwr * gn - gm * dwd * sdu;          // dP/dr at fixed du . rhat
                // (dG/dd)^T dl = hdl [dP rhat - gamma w_d (du - sdu rhat) / r] + P/r (dl - hdl rhat)
                const R c1 = hdl * dP, c2 = -hdl * gm * wd * ir, c3 = P * ir;
                gx += c1 * hx + c2 * (dux - sdu * hx) + c3 * (dlx - hdl * hx);
                gy += c1 * hy + c2 * (duy - sdu * hy) + c3 * (dly - hdl * hy);
                gz += c1 * hz + c2 * (duz - sdu * hz) + c3 * (dlz - hdl * hz);
                // (dG/d du)^T dl = -gamma w_d hdl rhat, on u_i (+) and u_j (-)
                const R cu = -gm * wd * hdl;
                atomicAdd(&a.ux[ii], (double)(cu * hx));
                atomicAdd(&a.uy[ii], (double)(cu * hy));
                atomicAdd(&a.uz[ii], (double)(cu * hz));
                atomicAdd(&a.ux[jj], -(double)(cu * hx));
                atomicAdd(&a.uy[jj], -(double)(cu * hy));
                atomicAdd(&a.uz[jj], -(double)(cu * hz));
                // gamma (friction and the noise amplitude sqrt(2 kT gamma / dt))
                gl[G_GAM] += (double)((sg * (R)0.5 / gm * wr * gn - wd * sdu) * hdl);
                // sigma through the DPD range: d w_r / d sigma = (r / rc) / sigma
                if (a.dpd_weight != 1) {
                    const R dws = r * irc / (R)a.sigma_lj;
                    gl[G_SIG] += (double)((sg * dws * gn - gm * (R)2 * wr * dws * sdu) * hdl);
                }
            }
            }
            // G depends on d = r_i - r_j: both positions, whichever side it acts on
            atomicAdd(&a.rx[ii], (double)gx);
            atomicAdd(&a.ry[ii], (double)gy);
            atomicAdd(&a.rz[ii], (double)gz);
            atomicAdd(&a.rx[jj], -(double)gx);
            atomicAdd(&a.ry[jj], -(double)gy);
            atomicAdd(&a.rz[jj], -(double)gz);
        }
        const int t = ch * 32 + lane;
        if (part == 0 && a.wall == 2 && t < a.n) {
            // 9-3 walls (fluid_wall.f90:96-121): F_z += f(z) - f(Z - z), f = A phi(z)
            const R4 pi = ps[t];
            const int wi = wbits(pi.w), ii = wi >> 8, ti = wi & 0xff;
            const R lfz = (R)a.fz[ii];
            const R sw = (R)a.sigma_wall[ti - 1], aw = (R)a.a_wall[ti - 1], cut = (R)a.wall_cut;
            const R sw3 = sw * sw * sw, sw9 = sw3 * sw3 * sw3;
            const R zb = pi.z, zt = (R)a.z_space_wall - pi.z;
            R dfz = 0, phi = 0;
            if (cut <= 0 || zb < cut) {
                const R iz = (R)1 / zb, iz2 = iz * iz, iz4 = iz2 * iz2, iz5 = iz4 * iz, iz10 = iz5 * iz5;
                phi += (R)9 * sw9 * iz10 - (R)3 * sw3 * iz4;
                dfz += aw * ((R)-90 * sw9 * iz10 * iz + (R)12 * sw3 * iz5);
            }
            if (cut <= 0 || zt < cut) {
                const R iz = (R)1 / zt, iz2 = iz * iz, iz4 = iz2 * iz2, iz5 = iz4 * iz, iz10 = iz5 * iz5;
                phi -= (R)9 * sw9 * iz10 - (R)3 * sw3 * iz4;
                dfz += aw * ((R)-90 * sw9 * iz10 * iz + (R)12 * sw3 * iz5);   // d/dz of -f(Z - z)
            }
            atomicAdd(&a.rz[ii], (double)(dfz * lfz));
            if (aw != (R)0) gl[G_WALL] += (double)(phi * lfz);
        }
        if (part == 0 && a.lgv && t < a.n) {
            // Langevin (lgv_forces.f90:22-41): F += sig g sqrt(m) - gamma m u, the
            // variates replayed (same Philox key as the pair kernel's)
            const R4 pi = ps[t];
            const int ii = wbits(pi.w) >> 8;
            const R4 ui = vs[t];
            const double m = a.mass[ii];
            const double lx = a.fx[ii], ly = a.fy[ii], lz = a.fz[ii];
            R g3[3];
            lgv_noise3<R>((uint32_t)ii, (uint32_t)step, a.noise, a.seed0, a.seed1, g3);
            const double cu = -a.gam * m;
            atomicAdd(&a.ux[ii], cu * lx);
            atomicAdd(&a.uy[ii], cu * ly);
            atomicAdd(&a.uz[ii], cu * lz);
            // d/d gamma: the friction and the amplitude sqrt(2 kT gamma / dt)
            const double gdl = (double)g3[0] * lx + (double)g3[1] * ly + (double)g3[2] * lz;
            const double udl = (double)ui.x * lx + (double)ui.y * ly + (double)ui.z * lz;
            gl[G_GAM] += 0.5 * a.sig / a.gam * sqrt(m) * gdl - m * udl;
        }
    }
    warp_add_g(a.g, gl);
}

struct AdjBondArgs {
    const double *px, *py, *pz;   // r' (particle order)
    const double *fx, *fy, *fz;   // lam_F
    double *rx, *ry, *rz;         // lam_r accumulators
    double* g;
    int n_chain, n_mon, n_chain_d, n_mon_d, part_init_d, symmetry;
    double L[3], invL[3];
    double k_fene, r0, inv_r_chain_2, fene_clamp;
};

// FENE VJP, thread per bond (i, i+1): G = -fs d on i, +fs d on i+1, d = r_i - r_{i+1},
// fs = k / (1 - x), x = min(r^2 / R0^2, clamp)
template <typename R>
__global__ void k_adj_fene(AdjBondArgs a) {
    double gl[G_N] = {0, 0, 0, 0, 0, 0};
    const int nb1 = a.n_chain * (a.n_mon - 1);
    const int nb2 = a.n_mon_d >= 2 ? a.n_chain_d * (a.n_mon_d - 1) : 0;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb1 + nb2) {
        int i;
        if (b < nb1) i = (b / (a.n_mon - 1)) * a.n_mon + b % (a.n_mon - 1);
        else i = a.part_init_d + ((b - nb1) / (a.n_mon_d - 1)) * a.n_mon_d + (b - nb1) % (a.n_mon_d - 1);
        const int j = i + 1;
        const R dx = (R)mi(a.px[i] - a.px[j], a.L[0], a.invL[0]);
        const R dy = (R)mi(a.py[i] - a.py[j], a.L[1], a.invL[1]);
        const double dz64 = a.pz[i] - a.pz[j];
        const R dz = (R)(a.symmetry == 1 ? mi(dz64, a.L[2], a.invL[2]) : dz64);
        const R irc2 = (R)a.inv_r_chain_2;
        R x = (dx * dx + dy * dy + dz * dz) * irc2;
        const bool clamped = x >= (R)a.fene_clamp;
        if (clamped) x = (R)a.fene_clamp;
        const R k = (R)a.k_fene;
        const R fs = k / ((R)1 - x);
        const R fsx = clamped ? (R)0 : k / (((R)1 - x) * ((R)1 - x));       // d fs / d x
        // coefficient of fs d: dl = lam_F_{i+1} - lam_F_i
        const R dlx = (R)(a.fx[j] - a.fx[i]), dly = (R)(a.fy[j] - a.fy[i]), dlz = (R)(a.fz[j] - a.fz[i]);
        const R ddl = dx * dlx + dy * dly + dz * dlz;
        const R c = (R)2 * irc2 * fsx * ddl;
        const R gx = fs * dlx + c * dx, gy = fs * dly + c * dy, gz = fs * dlz + c * dz;
        atomicAdd(&a.rx[i], (double)gx); atomicAdd(&a.ry[i], (double)gy); atomicAdd(&a.rz[i], (double)gz);
        atomicAdd(&a.rx[j], -(double)gx); atomicAdd(&a.ry[j], -(double)gy); atomicAdd(&a.rz[j], -(double)gz);
        gl[G_K] += (double)(fs * ddl) / a.k_fene;
        if (!clamped) gl[G_R0] += (double)(fsx * ((R)-2 * x / (R)a.r0) * ddl);
    }
    warp_add_g(a.g, gl);
}

// Bending VJP (bending.f90 mode 2, the angle formula of bonded.cuh), thread
// per angle centred on bead c of a grafted chain.  The bending force is
// conservative, so its Jacobian is symmetric and (dF/dr)^T lam_F is the
// derivative of the force along the displacement lam_F: the angle's force is
// evaluated once more in forward mode (value, derivative) with the bond
// vectors' tangents taken from lam_F.  The branches that zero a direction or
// the angle have zero derivative, as the forward force is constant there.
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double r = sqrt(a.v);
    return {r, a.d / (2.0 * r)};
}
__device__ __forceinline__ Dual dacos(Dual a) { return {acos(a.v), -a.d / sqrt(1.0 - a.v * a.v)}; }

struct AdjBendArgs {
    const double *px, *py, *pz;   // r' (particle order)
    const double *fx, *fy, *fz;   // lam_F
    double *rx, *ry, *rz;         // lam_r accumulators
    int n_chain, n_mon;
    double L[3], invL[3];
    double k_bend, alpha_eq;
};

__global__ void k_adj_bend(AdjBendArgs a) {
    const int na = a.n_mon - 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (na < 1 || t >= a.n_chain * na) return;
    const int c = (t / na) * a.n_mon + t % na + 1;   // centre bead; c-1, c+1 on the same chain
    const int id[3] = {c - 1, c, c + 1};
    const double* P[3] = {a.px, a.py, a.pz};
    const double* F[3] = {a.fx, a.fy, a.fz};
    // bond vectors r(j+1) - r(j), imaged on every axis (bending.f90:34-57), as bonded.cuh forms them
    Dual p[3], n[3];
    for (int d = 0; d < 3; ++d) {
        const double d0 = P[d][id[0]] - P[d][id[1]], d1 = P[d][id[1]] - P[d][id[2]];
        p[d] = {-d0 + a.L[d] * (double)(int)(2.0 * d0 * a.invL[d]), F[d][id[1]] - F[d][id[0]]};
        n[d] = {-d1 + a.L[d] * (double)(int)(2.0 * d1 * a.invL[d]), F[d][id[2]] - F[d][id[1]]};
    }
    const double tiny = 1.0000000116860974e-07;   // the forward's single-precision literal
    const Dual dot = (n[0] * p[0] + n[1] * p[1]) + n[2] * p[2];
    const Dual p2 = (p[0] * p[0] + p[1] * p[1]) + p[2] * p[2];
    const Dual n2 = (n[0] * n[0] + n[1] * n[1]) + n[2] * n[2];
    const Dual cosa = dot / dsqrt(p2 * n2);
    Dual dn[3], dp[3];
    for (int d = 0; d < 3; ++d) {
        dn[d] = p[d] * n2 - n[d] * dot;
        dp[d] = -n[d] * p2 + p[d] * dot;
    }
    const Dual dn2 = (dn[0] * dn[0] + dn[1] * dn[1]) + dn[2] * dn[2];
    const Dual dp2 = (dp[0] * dp[0] + dp[1] * dp[1]) + dp[2] * dp[2];
    const Dual zero = {0.0, 0.0};
    if (dn2.v < tiny) { dn[0] = dn[1] = dn[2] = zero; }
    else { const Dual s = Dual{1.0, 0.0} / dsqrt(dn2 * n2); for (int d = 0; d < 3; ++d) dn[d] = dn[d] * s; }
    if (dp2.v < tiny) { dp[0] = dp[1] = dp[2] = zero; }
    else { const Dual s = Dual{1.0, 0.0} / dsqrt(dp2 * p2); for (int d = 0; d < 3; ++d) dp[d] = dp[d] * s; }
    const Dual da = cosa.v >= 1.0 ? zero : dacos(cosa) - Dual{a.alpha_eq, 0.0};
    const Dual fm = Dual{a.k_bend, 0.0} * da;
    double* R[3] = {a.rx, a.ry, a.rz};
    for (int d = 0; d < 3; ++d) {
        // forward: previous bead += fp, next bead += fn, centre -= fp + fn
        const double gp = (fm * dp[d]).d, gn = (fm * dn[d]).d;
        atomicAdd(&R[d][id[0]], gp);
        atomicAdd(&R[d][id[2]], gn);
        atomicAdd(&R[d][id[1]], -(gp + gn));
    }
}

// lam_F = (alpha' + dt/2 nu') / m, lam_u = nu', lam_r = rho' (pinned heads: 0)
__global__ void k_adj_prep(int n, const double* __restrict__ rho, const double* __restrict__ nu,
                           const double* __restrict__ alpha, const double* __restrict__ inv_mass, double hdt,
                           int pin_heads, int n_head_span, int n_mon, double* lamF, double* lamU, double* lamR) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool head = pin_heads && i < n_head_span && (i % n_mon) == 0;
    for (int d = 0; d < 3; ++d) {
        const size_t k = (size_t)d * n + i;
        lamF[k] = head ? 0.0 : (alpha[k] + hdt * nu[k]) * inv_mass[i];
        lamU[k] = head ? 0.0 : nu[k];
        lamR[k] = rho[k];
    }
}

// rho = lam_r + w dO/dr(r), nu = dt lam_r + lam_u, alpha = dt^2/2 lam_r + dt/2 lam_u
// dO/dr: <z> over all beads (1/n on z), <R_ee^2> over the chains (ends)
__global__ void k_adj_combine(int n, const double* __restrict__ lamR, const double* __restrict__ lamU, double dt,
                              double w_obs, const double* __restrict__ r, const int32_t* __restrict__ mic,
                              double Lx, double Ly, double Lz, int n_chain, int n_mon, int pin_heads,
                              double* rho, double* nu, double* alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool head = pin_heads && i < n_chain * n_mon && (i % n_mon) == 0;
    double o[3] = {0.0, 0.0, 0.0};
    if (w_obs != 0.0) {
        o[2] = w_obs / (double)n;
        if (n_chain > 0 && n_mon > 1 && i < n_chain * n_mon) {
            const int p = i % n_mon;
            if (p == 0 || p == n_mon - 1) {
                const int f = i - p, e = f + n_mon - 1;
                const double L[3] = {Lx, Ly, Lz};
                const double s = (p == 0 ? -2.0 : 2.0) * w_obs / (double)n_chain;
                for (int d = 0; d < 3; ++d) {
                    const double R = (r[(size_t)d * n + e] + L[d] * mic[(size_t)d * n + e]) -
                                     (r[(size_t)d * n + f] + L[d] * mic[(size_t)d * n + f]);
                    o[d] += s * R;
                }
            }
        }
    }
    for (int d = 0; d < 3; ++d) {
        const size_t k = (size_t)d * n + i;
        const double lr = lamR[k], lu = lamU[k];
        rho[k] = lr + o[d];
        nu[k] = head ? 0.0 : dt * lr + lu;
        alpha[k] = head ? 0.0 : 0.5 * dt * dt * lr + 0.5 * dt * lu;
    }
}

// O(r) = <z> + <R_ee^2> of the current state, added (times w) to out[0]
__global__ void k_observable(int n, const double* __restrict__ rx, const double* __restrict__ ry,
                             const double* __restrict__ rz, const int32_t* __restrict__ mx,
                             const int32_t* __restrict__ my, const int32_t* __restrict__ mz, double Lx, double Ly,
                             double Lz, int n_chain, int n_mon, double w, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    // z unfolded by the image counter (continuous across the periodic wrap of
    // a bulk box; in channels z is never wrapped and the counter stays 0)
    if (i < n) v += (rz[i] + Lz * mz[i]) / (double)n;
    if (i < n_chain && n_mon > 1) {
        const int f = i * n_mon, e = f + n_mon - 1;
        const double X = (rx[e] + Lx * mx[e]) - (rx[f] + Lx * mx[f]);
        const double Y = (ry[e] + Ly * my[e]) - (ry[f] + Ly * my[f]);
        const double Z = (rz[e] + Lz * mz[e]) - (rz[f] + Lz * mz[f]);
        v += (X * X + Y * Y + Z * Z) / (double)n_chain;
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out, w * v);
}

constexpr int T = 256;

struct Work {
    int n, S, K, nseg;
    double* ck;          // checkpoints: nseg x (r, v, a) 9n doubles
    int32_t* ckm;        // checkpoints: nseg x mic 3n
    int64_t* ckstep;     // dstep per checkpoint (device, nseg)
    double* seg_r;       // (K + 1) x 3n: r after the position half of each step; slot K: the checkpoint's r
    double* seg_u;       // K x 3n (u)
    int32_t* seg_m;      // (K + 1) x 3n (mic; slot K: the checkpoint's)
    int64_t* seg_step;   // K: dstep as the forces of each recomputed step saw it
    double *rho, *nu, *alpha, *lamF, *lamU, *lamR;   // 3n each
    double* dg;          // G_N + 1 (J)
};

// One launch for the copies of a state (the time step's sequences would
// otherwise hold a copy node per array): up to three FP64 blocks of n3
// values, one int32 block of n3 and one step number; null pointers are
// skipped.
struct StateCopy {
    double* d[3];
    const double* s[3];
    int32_t* dm;
    const int32_t* sm;
    int64_t* dstep;
    const int64_t* sstep;
    size_t n3;
};

__global__ void k_copy_state(StateCopy a) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n3; i += stride) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (a.d[k]) a.d[k][i] = a.s[k][i];
        if (a.dm) a.dm[i] = a.sm[i];
    }
    if (a.dstep && blockIdx.x == 0 && threadIdx.x == 0) *a.dstep = *a.sstep;
}

int copy_state(mfa_ctx* c, double* d0, const double* s0, double* d1, const double* s1, double* d2,
               const double* s2, int32_t* dm, const int32_t* sm, int64_t* dstep, const int64_t* sstep) {
    StateCopy a;
    a.d[0] = d0; a.s[0] = s0; a.d[1] = d1; a.s[1] = s1; a.d[2] = d2; a.s[2] = s2;
    a.dm = dm; a.sm = sm; a.dstep = dstep; a.sstep = sstep;
    a.n3 = (size_t)3 * c->n;
    const int nb = (int)((a.n3 + T - 1) / T);
    k_copy_state<<<nb, T, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    return MFA_OK;
}

// The backward step's state in one pass: r', u and mic of a segment slot back
// in the context, the skin check against the list's snapshot
// (check_skin.f90:8-21, with the integrator's rounding) and the cell-sorted
// records the pair kernels read (a rebuild, when the check trips, rewrites
// them after this).
struct RestoreArgs {
    const double *sr, *su;
    const int32_t* sm;
    double *rx, *vx;
    int32_t* mx;
    const double *ox, *oy, *oz;
    const int32_t* slot;
    const int32_t* type;
    const double* q;
    void* pos_s;
    void* vel_s;
    int32_t* flags;
    double L[3], skin_lim;
    int n;
};

template <typename R4>
__global__ void k_adj_restore(RestoreArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const size_t n = (size_t)a.n;
    double r[3], u[3];
    int m[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        r[d] = a.sr[d * n + i];
        u[d] = a.su[d * n + i];
        m[d] = a.sm[d * n + i];
        a.rx[d * n + i] = r[d];
        a.vx[d * n + i] = u[d];
        a.mx[d * n + i] = m[d];
    }
    // the snapshot holds r0_old + mic_old * L
    const double o[3] = {a.ox[i], a.oy[i], a.oz[i]};
    double dd[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) dd[d] = __dsub_rn(__dsub_rn(o[d], r[d]), __dmul_rn((double)m[d], a.L[d]));
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dd[0], dd[0]), __dmul_rn(dd[1], dd[1])), __dmul_rn(dd[2], dd[2]));
    if (r2 > a.skin_lim) a.flags[F_SKIN] = 1;
    const int s = a.slot[i];
    R4 p;
    p.x = r[0]; p.y = r[1]; p.z = r[2];
    packw(p, i, a.type[i]);
    ((R4*)a.pos_s)[s] = p;
    R4 v;
    v.x = u[0]; v.y = u[1]; v.z = u[2]; v.w = a.q ? a.q[i] : 0.0;
    ((R4*)a.vel_s)[s] = v;
}

int launch_adj_restore(mfa_ctx* c, const double* sr, const double* su, const int32_t* sm) {
    RestoreArgs a;
    a.sr = sr; a.su = su; a.sm = sm;
    a.rx = c->rx; a.vx = c->vx; a.mx = c->mx;
    a.ox = c->ox; a.oy = c->oy; a.oz = c->oz;
    a.slot = c->slot; a.type = c->type; a.q = c->p.charged ? c->q : nullptr;
    a.pos_s = c->pos_s; a.vel_s = c->vel_s; a.flags = c->dflags;
    for (int d = 0; d < 3; ++d) a.L[d] = c->p.boundary[d];
    a.skin_lim = (c->p.skin / 2.0) * (c->p.skin / 2.0);
    a.n = c->n;
    const int nb = (c->n + T - 1) / T;
    if (c->prec == MFA_MIXED) k_adj_restore<float4><<<nb, T, 0, c->st>>>(a);
    else k_adj_restore<double4><<<nb, T, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    return MFA_OK;
}

// The step whose energies the forward steps reduce: dstep[1] = dstep[0] + span
// (the last step of a run of span steps; the energies of the other steps are
// not wanted there), or -1 (span < 0: every step, as the subroutine entry
// points expect).
__global__ void k_energy_want(int64_t* dstep, long long span) {
    dstep[1] = span < 0 ? -1 : dstep[0] + span;
}

int adj_forward_step(mfa_ctx* c, double* sr, double* su, int32_t* sm, double w, double* dJ,
                     int64_t* sstep = nullptr) {
    const int n = c->n;
    TRY_(launch_vv_positions(c, 1, 1));
    if (sr) TRY_(copy_state(c, sr, c->rx, su, c->vx, nullptr, nullptr, sm, c->mx, sstep, c->dstep));
    else if (sstep) MFA_CUDA_TRY(cudaMemcpyAsync(sstep, c->dstep, 8, cudaMemcpyDeviceToDevice, c->st));
    TRY_(c->coop_rebuild ? launch_rebuild_coop(c, c->bin_type) : launch_rebuild(c, c->bin_type, 1));
    TRY_(launch_pair(c, c->p.symmetry == 0));
    if (c->p.charged) {
        TRY_(launch_ewald(c));      // md_main.f90:128-131
        TRY_(launch_dipolar(c));    // SYMMETRY 0 only
    }
    TRY_(launch_vv_velocities(c, 1));
    if (dJ) {
        const mfa_params& p = c->p;
        k_observable<<<(n + T - 1) / T, T, 0, c->st>>>(n, c->rx, c->ry, c->rz, c->mx, c->my, c->mz,
                                                         p.boundary[0], p.boundary[1], p.boundary[2], p.n_chain,
                                                         p.n_mon, w, dJ);
        MFA_CUDA_TRY(cudaGetLastError());
    }
    return MFA_OK;
}

int checkpoint_save(mfa_ctx* c, Work& w, int k) {
    const size_t n3 = (size_t)3 * c->n;
    double* ck = w.ck + k * 3 * n3;
    return copy_state(c, ck, c->rx, ck + n3, c->vx, ck + 2 * n3, c->ax, w.ckm + k * n3, c->mx, w.ckstep + k,
                      c->dstep);
}

// The state of checkpoint k back in the context, and its r and mic in the
// staging slot K of the segment buffers (the observable at the segment's
// first state).  The lists are left as they are: the first position half
// checks the skin against the last rebuild's positions and rebuilds when due.
int checkpoint_restore(mfa_ctx* c, Work& w, int k) {
    const size_t n3 = (size_t)3 * c->n;
    const double* ck = w.ck + k * 3 * n3;
    TRY_(copy_state(c, c->rx, ck, c->vx, ck + n3, c->ax, ck + 2 * n3, c->mx, w.ckm + k * n3, c->dstep,
                    w.ckstep + k));
    return copy_state(c, w.seg_r + (size_t)w.K * n3, ck, nullptr, nullptr, nullptr, nullptr, w.seg_m + (size_t)w.K * n3,
                      w.ckm + k * n3, nullptr, nullptr);
}

AdjArgs pair_adj_args(mfa_ctx* c, Work& w, const int64_t* step_ptr) {
    const mfa_params& p = c->p;
    const int n = c->n;
    AdjArgs a;
    a.pos_s = c->pos_s; a.vel_s = c->vel_s; a.nbr = c->nbr; a.ccount = c->ccount; a.tabs = c->tabs;
    a.maxnb = c->maxnb;
    a.fx = w.lamF; a.fy = w.lamF + n; a.fz = w.lamF + 2 * n;
    a.rx = w.lamR; a.ry = w.lamR + n; a.rz = w.lamR + 2 * n;
    a.ux = w.lamU; a.uy = w.lamU + n; a.uz = w.lamU + 2 * n;
    a.g = w.dg;
    a.n = n;
    a.half = c->bin_type == 0;
    a.symmetry = p.symmetry;
    a.dpd = p.thermostat == MFA_THERMO_DPD;
    a.lgv = p.thermostat == MFA_THERMO_LGV;
    a.mass = c->mass;
    a.charged = p.charged;
    a.real_in_lj = (p.quirks & MFA_Q_EWALD_REAL_IN_LJ) != 0;
    a.sqrt_alpha = p.sqrt_alpha; a.alpha_c = p.alpha_c; a.inv_sqrt_pi = p.inv_sqrt_pi;
    a.ewald_rc_2 = p.ewald_rc_2;
    a.seed0 = (uint32_t)p.seed;
    a.seed1 = (uint32_t)(p.seed >> 32);
    a.dpd_weight = p.dpd_weight;
    a.noise = p.noise;
    a.wall = (p.symmetry == 0 && p.wall == 2) ? 2 : 0;
    for (int d = 0; d < 3; ++d) { a.L[d] = p.boundary[d]; a.invL[d] = c->inv_boundary[d]; }
    a.sig = p.sig; a.gam = p.friction;
    // the physical eps and sigma the pair tables scale with: the largest pair's
    double emax = 0.0, smax = 0.0;
    for (int k = 0; k < T8 * T8; ++k)
        if (p.range_2[k] > 0.0) { emax = fmax(emax, p.epsil[k] / 4.0); smax = fmax(smax, sqrt(p.sigma_2[k])); }
    a.eps_lj = emax > 0.0 ? emax : 1.0;
    a.sigma_lj = smax > 0.0 ? smax : 1.0;
    a.step = 0;
    a.step_ptr = step_ptr;
    // pieces per chunk: double while the warps fit 16 per SM (a small
    // system's few chunks would leave most SMs idle), at most 8
    const long long nchunk = (n + 31) / 32;
    a.split = 1;
    while (a.split < 8 && nchunk * a.split * 2 <= 16LL * c->n_sm) a.split *= 2;
    a.key = philox_round_keys((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    for (int k = 0; k < T8; ++k) { a.a_wall[k] = p.a_wall[k]; a.sigma_wall[k] = p.sigma_wall[k]; }
    a.z_space_wall = p.z_space_wall;
    a.wall_cut = p.wall_cut;
    return a;
}

}  // namespace

extern "C" {

int mfa_trajectory_observable(mfa_ctx* c, int32_t nsteps, double* J) {
    if (!c || nsteps < 1 || !J) return MFA_ERR_ARGS;
    if (!c->lists_valid) TRY_(mfa_binning(c));
    double* dJ = nullptr;
    if (cudaMalloc((void**)&dJ, 8) != cudaSuccess) return MFA_ERR_NOMEM;
    int rc = MFA_OK;
    if (cudaMemsetAsync(dJ, 0, 8, c->st) != cudaSuccess) rc = MFA_ERR_CUDA;
    // energies for the run's last step only
    k_energy_want<<<1, 1, 0, c->st>>>(c->dstep, nsteps);
    for (int s = 0; s < nsteps && rc == MFA_OK; ++s) rc = adj_forward_step(c, nullptr, nullptr, nullptr, 1.0 / nsteps, dJ);
    k_energy_want<<<1, 1, 0, c->st>>>(c->dstep, -1);
    if (rc == MFA_OK && (cudaMemcpyAsync(J, dJ, 8, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
                         cudaStreamSynchronize(c->st) != cudaSuccess))
        rc = MFA_ERR_CUDA;
    cudaFree(dJ);
    if (rc == MFA_OK) c->i_time += nsteps;
    if (rc != MFA_OK) return rc;
    return mfa_sync(c);
}

}  // extern "C"

// mfa_adjoint's device workspace and its four captured sequences, kept on the
// context for the next call with the same length and checkpoint interval: a
// repeated call (optimisation loops call it with the same S and K) then
// allocates and captures nothing.  Dropped when the context's graphs are (list
// capacity, cells, launch shapes, energy log), when what the sequences point
// to moves, after a failed call, and at mfa_finalize.
struct AdjCache {
    int S, K;
    unsigned long long gen;
    const void* key[4];
    size_t sizes[10];
    void* bufs[10];
    cudaGraphExec_t gx[4];
    bool captured;
};

void adj_cache_free(mfa_ctx* c) {
    AdjCache* ac = (AdjCache*)c->adj_cache;
    if (!ac) return;
    cudaStreamSynchronize(c->st);
    for (cudaGraphExec_t g : ac->gx) if (g) cudaGraphExecDestroy(g);
    for (void* b : ac->bufs) if (b) cudaFree(b);
    delete ac;
    c->adj_cache = nullptr;
}

extern "C" {

int mfa_adjoint(mfa_ctx* c, int32_t nsteps, int32_t every, double* out) {
    if (!c || nsteps < 1 || every < 1 || !out) return MFA_ERR_ARGS;
    const mfa_params& p = c->p;
    // the force terms differentiated here: pair (LJ/WCA, DPD, Ewald real
    // space), Langevin, FENE, bending, 9-3 walls, Ewald k-space and the slab
    // correction
    if (p.force_switch_on || c->dpd_vv || (p.symmetry == 0 && (p.wall == 3 || p.wall == 4)) ||
        (p.n_chain_d > 0 && p.n_mon_d >= 2))
        return MFA_ERR_UNSUPPORTED;
    if (p.charged && c->nk == 0) return MFA_ERR_STATE;   // ewald_k(0) first
    if (!c->lists_valid) TRY_(mfa_binning(c));
    const int n = c->n;
    const size_t n3 = (size_t)3 * n;
    Work w;
    w.n = n; w.S = nsteps; w.K = every < nsteps ? every : nsteps;
    w.nseg = (nsteps + w.K - 1) / w.K;
    size_t sizes[10] = {(size_t)w.nseg * 3 * n3 * 8, (size_t)w.nseg * n3 * 4, (size_t)(w.K + 1) * n3 * 8,
                        (size_t)w.K * n3 * 8, (size_t)(w.K + 1) * n3 * 4, 6 * n3 * 8, (G_N + 1) * 8,
                        p.charged ? ewald_adj_bytes(c) : 0, (size_t)w.nseg * 8, (size_t)w.K * 8};
    const void* key[4] = {c->nbr, c->kvec, c->elog, (const void*)(intptr_t)(c->bin_type + 1)};
    AdjCache* ac = (AdjCache*)c->adj_cache;
    if (ac && (ac->S != nsteps || ac->K != w.K || ac->gen != c->graph_gen || memcmp(ac->key, key, sizeof(key)) ||
               memcmp(ac->sizes, sizes, sizeof(sizes))))
        adj_cache_free(c);
    ac = (AdjCache*)c->adj_cache;
    int rc = MFA_OK;
    if (!ac) {
        ac = new AdjCache();
        ac->S = nsteps; ac->K = w.K; ac->gen = c->graph_gen;
        memcpy(ac->key, key, sizeof(key));
        memcpy(ac->sizes, sizes, sizeof(sizes));
        c->adj_cache = ac;
        for (int k = 0; k < 10 && rc == MFA_OK; ++k)
            if (sizes[k] && cudaMalloc(&ac->bufs[k], sizes[k]) != cudaSuccess) rc = MFA_ERR_NOMEM;
        if (rc != MFA_OK) {
            adj_cache_free(c);
            return rc;
        }
    }
    void** bufs = ac->bufs;
    w.ck = (double*)bufs[0]; w.ckm = (int32_t*)bufs[1];
    w.seg_r = (double*)bufs[2]; w.seg_u = (double*)bufs[3]; w.seg_m = (int32_t*)bufs[4];
    w.ckstep = (int64_t*)bufs[8]; w.seg_step = (int64_t*)bufs[9];
    double* adj = (double*)bufs[5];
    w.rho = adj; w.nu = adj + n3; w.alpha = adj + 2 * n3; w.lamF = adj + 3 * n3; w.lamU = adj + 4 * n3;
    w.lamR = adj + 5 * n3;
    w.dg = (double*)bufs[6];
    double* dJ = w.dg + G_N;
    const double dt = p.dt, wobs = 1.0 / nsteps;
    const int nb = (n + T - 1) / T;
    if (p.charged) TRY_(ewald_adjoint_prepare(c));
    // forward steps with the observable (segment of len steps)
    auto fwd = [&](int len) -> int {
        for (int j = 0; j < len; ++j) TRY_(adj_forward_step(c, nullptr, nullptr, nullptr, wobs, dJ));
        return MFA_OK;
    };
    // the segment recomputed from its checkpoint, each step's r', u, mic and step kept
    auto rec = [&](int len) -> int {
        for (int j = 0; j < len; ++j)
            TRY_(adj_forward_step(c, w.seg_r + j * n3, w.seg_u + j * n3, w.seg_m + j * n3, 0.0, nullptr,
                                  w.seg_step + j));
        return MFA_OK;
    };
    // backward through the segment (steps len-1 .. 0); first_seg: the
    // segment's first state is the trajectory's start, which the observable
    // does not count
    auto bwd = [&](int len, bool first_seg) -> int {
        for (int j = len - 1; j >= 0; --j) {
            const double* r1 = w.seg_r + j * n3;
            // state, skin check and sorted records in one pass; then the
            // rebuild when due
            TRY_(launch_adj_restore(c, r1, w.seg_u + j * n3, w.seg_m + j * n3));
            TRY_(c->coop_rebuild ? launch_rebuild_coop(c, c->bin_type) : launch_rebuild(c, c->bin_type, 1));
            k_adj_prep<<<nb, T, 0, c->st>>>(n, w.rho, w.nu, w.alpha, c->inv_mass, 0.5 * dt, p.pin_heads,
                                            p.n_chain * p.n_mon, p.n_mon > 0 ? p.n_mon : 1, w.lamF, w.lamU,
                                            w.lamR);
            AdjArgs aa = pair_adj_args(c, w, w.seg_step + j);
            const int nbw = (int)(((long long)(n + 31) / 32 * aa.split * 32 + T - 1) / T);   // a warp per piece
            if (c->prec == MFA_MIXED) k_adj_pair<float><<<nbw, T, 0, c->st>>>(aa);
            else k_adj_pair<double><<<nbw, T, 0, c->st>>>(aa);
            const int nbonds = p.n_chain * (p.n_mon > 0 ? p.n_mon - 1 : 0) +
                               (p.n_mon_d >= 2 ? p.n_chain_d * (p.n_mon_d - 1) : 0);
            if (nbonds > 0) {
                AdjBondArgs ba;
                ba.px = r1; ba.py = r1 + n; ba.pz = r1 + 2 * n;
                ba.fx = w.lamF; ba.fy = w.lamF + n; ba.fz = w.lamF + 2 * n;
                ba.rx = w.lamR; ba.ry = w.lamR + n; ba.rz = w.lamR + 2 * n;
                ba.g = w.dg;
                ba.n_chain = p.n_chain; ba.n_mon = p.n_mon; ba.n_chain_d = p.n_chain_d; ba.n_mon_d = p.n_mon_d;
                ba.part_init_d = p.n_mon * p.n_chain; ba.symmetry = p.symmetry;
                for (int d = 0; d < 3; ++d) { ba.L[d] = p.boundary[d]; ba.invL[d] = c->inv_boundary[d]; }
                ba.k_fene = p.k_chain * p.inv_r_chain_2;
                ba.r0 = sqrt(p.r_chain_2);
                ba.inv_r_chain_2 = p.inv_r_chain_2;
                ba.fene_clamp = p.fene_clamp;
                const int bb = (nbonds + T - 1) / T;
                if (c->prec == MFA_MIXED) k_adj_fene<float><<<bb, T, 0, c->st>>>(ba);
                else k_adj_fene<double><<<bb, T, 0, c->st>>>(ba);
            }
            if (p.bending && p.n_mon >= 3 && p.n_chain > 0) {
                AdjBendArgs ka;
                ka.px = r1; ka.py = r1 + n; ka.pz = r1 + 2 * n;
                ka.fx = w.lamF; ka.fy = w.lamF + n; ka.fz = w.lamF + 2 * n;
                ka.rx = w.lamR; ka.ry = w.lamR + n; ka.rz = w.lamR + 2 * n;
                ka.n_chain = p.n_chain; ka.n_mon = p.n_mon;
                for (int d = 0; d < 3; ++d) { ka.L[d] = p.boundary[d]; ka.invL[d] = c->inv_boundary[d]; }
                ka.k_bend = p.k_bend; ka.alpha_eq = p.alpha_eq;
                const int nang = p.n_chain * (p.n_mon - 2);
                k_adj_bend<<<(nang + T - 1) / T, T, 0, c->st>>>(ka);
            }
            // Ewald k-space (and the slab correction) at r', c->rx holding r'
            if (p.charged) TRY_(launch_ewald_adjoint(c, w.lamF, w.lamR, bufs[7]));
            // back to the state before this step: the observable at r_s (the
            // previous slot, or the segment's checkpoint in staging slot K)
            const bool at_start = j == 0 && first_seg;
            const double* r0 = j > 0 ? w.seg_r + (j - 1) * n3 : w.seg_r + (size_t)w.K * n3;
            const int32_t* m0 = j > 0 ? w.seg_m + (j - 1) * n3 : w.seg_m + (size_t)w.K * n3;
            k_adj_combine<<<nb, T, 0, c->st>>>(n, w.lamR, w.lamU, dt, at_start ? 0.0 : wobs, r0, m0, p.boundary[0],
                                               p.boundary[1], p.boundary[2], p.n_chain, p.n_mon, p.pin_heads,
                                               w.rho, w.nu, w.alpha);
            MFA_CUDA_TRY(cudaGetLastError());
        }
        return MFA_OK;
    };
    // Full segments replay captured graphs (one per sequence, kept in the
    // cache for the next call); a partial last segment, and any sequence whose
    // capture fails, runs as plain launches.
    cudaGraphExec_t* gx = ac->gx;
    // MFA_DEBUG=1 in the environment reports a sequence that could not be
    // captured (it then runs as plain launches)
    const bool dbg = getenv("MFA_DEBUG") && getenv("MFA_DEBUG")[0] == '1';
    auto capture = [&](int which, auto&& fn) -> void {
        cudaGraph_t gr = nullptr;
        if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return;
        const int r = fn();
        const cudaError_t ee = cudaStreamEndCapture(c->st, &gr);
        if (ee != cudaSuccess || r != MFA_OK || !gr) {
            if (dbg)
                fprintf(stderr, "mfa_adjoint: sequence %d not captured (status %d, %s)\n", which, r,
                        cudaGetErrorString(ee != cudaSuccess ? ee : cudaGetLastError()));
            if (gr) cudaGraphDestroy(gr);
            cudaGetLastError();
            return;
        }
        const cudaError_t ie = cudaGraphInstantiate(&gx[which], gr, 0);
        if (ie != cudaSuccess) {
            if (dbg) fprintf(stderr, "mfa_adjoint: sequence %d not instantiated (%s)\n", which, cudaGetErrorString(ie));
            gx[which] = nullptr;
        }
        cudaGraphDestroy(gr);
        cudaGetLastError();
    };
    auto replay = [&](int which, auto&& fn) -> int {
        if (gx[which]) {
            MFA_CUDA_TRY(cudaGraphLaunch(gx[which], c->st));
            return MFA_OK;
        }
        return fn();
    };
    const bool full_last = nsteps % w.K == 0;
    if (!ac->captured && (w.nseg > 1 || full_last)) {
        capture(0, [&] { return fwd(w.K); });
        capture(1, [&] { return rec(w.K); });
        capture(2, [&] { return bwd(w.K, false); });
        capture(3, [&] { return bwd(w.K, true); });
    }
    ac->captured = true;
    auto run = [&]() -> int {
        TRY_(mfa_sync(c));
        MFA_CUDA_TRY(cudaMemsetAsync(w.dg, 0, (G_N + 1) * 8, c->st));
        MFA_CUDA_TRY(cudaMemsetAsync(adj, 0, 6 * n3 * 8, c->st));
        // the forward and recomputed steps reduce energies for the
        // trajectory's last step only (the adjoint needs none)
        k_energy_want<<<1, 1, 0, c->st>>>(c->dstep, nsteps);
        // forward pass with checkpoints and the observable
        for (int seg = 0; seg < w.nseg; ++seg) {
            const int len = seg * w.K + w.K <= nsteps ? w.K : nsteps - seg * w.K;
            TRY_(checkpoint_save(c, w, seg));
            if (len == w.K) TRY_(replay(0, [&] { return fwd(len); }));
            else TRY_(fwd(len));
        }
        // rho_S = 1/S dO/dr_S (nu_S = alpha_S = 0)
        k_adj_combine<<<nb, T, 0, c->st>>>(n, w.lamR, w.lamU, dt, wobs, c->rx, c->mx, p.boundary[0], p.boundary[1],
                                           p.boundary[2], p.n_chain, p.n_mon, p.pin_heads, w.rho, w.nu, w.alpha);
        MFA_CUDA_TRY(cudaGetLastError());
        // the final state of the trajectory, restored at the end
        std::vector<double> fin_rva(3 * n3);
        std::vector<int32_t> fin_m(n3);
        int64_t fin_step = 0;
        MFA_CUDA_TRY(cudaMemcpyAsync(fin_rva.data(), c->rx, n3 * 8, cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(fin_rva.data() + n3, c->vx, n3 * 8, cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(fin_rva.data() + 2 * n3, c->ax, n3 * 8, cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(fin_m.data(), c->mx, n3 * 4, cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(&fin_step, c->dstep, 8, cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
        // backward, segment by segment
        for (int seg = w.nseg - 1; seg >= 0; --seg) {
            const int len = seg * w.K + w.K <= nsteps ? w.K : nsteps - seg * w.K;
            TRY_(checkpoint_restore(c, w, seg));
            if (len == w.K) {
                TRY_(replay(1, [&] { return rec(len); }));
                TRY_(replay(seg == 0 ? 3 : 2, [&] { return bwd(len, seg == 0); }));
            } else {
                TRY_(rec(len));
                TRY_(bwd(len, seg == 0));
            }
        }
        // leave the context at the end of the trajectory, as mfa_step would
        MFA_CUDA_TRY(cudaMemcpyAsync(c->rx, fin_rva.data(), n3 * 8, cudaMemcpyHostToDevice, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(c->vx, fin_rva.data() + n3, n3 * 8, cudaMemcpyHostToDevice, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(c->ax, fin_rva.data() + 2 * n3, n3 * 8, cudaMemcpyHostToDevice, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(c->mx, fin_m.data(), n3 * 4, cudaMemcpyHostToDevice, c->st));
        MFA_CUDA_TRY(cudaMemcpyAsync(c->dstep, &fin_step, 8, cudaMemcpyHostToDevice, c->st));
        k_energy_want<<<1, 1, 0, c->st>>>(c->dstep, -1);
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
        TRY_(mfa_binning(c));
        double h[G_N + 1];
        MFA_CUDA_TRY(cudaMemcpyAsync(h, w.dg, sizeof(h), cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
        out[0] = h[G_N];
        for (int q = 0; q < G_N; ++q) out[1 + q] = h[q];
        c->i_time += nsteps;
        return mfa_sync(c);
    };
    rc = run();
    cudaStreamSynchronize(c->st);
    // the run may have grown the list or moved what the sequences point to
    // (the closing mfa_binning); a failed run leaves nothing for the next call
    if (rc != MFA_OK) {
        k_energy_want<<<1, 1, 0, c->st>>>(c->dstep, -1);   // every step's energies again
        adj_cache_free(c);
    }
    return rc;
}

}  // extern "C"
