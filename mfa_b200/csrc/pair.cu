// Pair forces: fluid_fluid.f90 with dpd_forces (THERMOSTAT 0), ewald_real
// (charged systems, fused into the same pass) and lgv_forces (THERMOSTAT 1),
// plus optionally the 9-3 walls of fluid_wall.f90 in the per-particle epilogue.
//
// One thread per cell-sorted slot walks its full Verlet list and accumulates
// the force on its own particle only: no atomics, deterministic order, and the
// DPD noise of a pair is drawn from Philox keyed by (step, min(i,j), max(i,j))
// so both sides of a pair see the same random number.  R = float in MIXED mode
// (FP32 force math, FP64 energy/virial accumulators), double in FP64 mode.
#include "mfa_internal.cuh"

namespace {

struct PairArgs {
    const void* pos_s;
    const void* vel_s;
    const int32_t* __restrict__ nbr;
    const int32_t* __restrict__ nnb;
    const double* mass;
    const double* tabs;
    void* force;
    const int64_t* dstep;
    double* partials;
    unsigned* counter;
    double* dscal;
    int n, max_blocks;
    int symmetry, thermostat, dpd_weight, noise, charged, real_in_lj, fsw;
    int wall_type, wall_e_aw;
    int accumulate;
    double coul_energy_factor;
    double L[3], invL[3];
    double sig, friction, dt;
    double r_2_min_init, r_2_min_time;
    long long s_time;
    double sqrt_alpha, alpha_c, inv_sqrt_pi, ewald_rc_2;
    double a_wall[T8], sigma_wall[T8], a_w, z_space_wall, wall_cut;
    uint32_t seed0, seed1;
};

template <typename R> struct Vec4;
template <> struct Vec4<float> { typedef float4 T; };
template <> struct Vec4<double> { typedef double4 T; };

__device__ __forceinline__ float mimg(float d, float L, float iL) { return mimage32(d, L, iL); }
__device__ __forceinline__ double mimg(double d, double L, double iL) {
    return d - L * (double)(int)(2.0 * d * iL);
}
__device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(1.0 / x); }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float erfc_(float x) { return erfcf(x); }
__device__ __forceinline__ double erfc_(double x) { return erfc(x); }
__device__ __forceinline__ float exp_(float x) { return expf(x); }
__device__ __forceinline__ double exp_(double x) { return exp(x); }

// Gaussian (Box-Muller) or uniform variate from two Philox words.
__device__ __forceinline__ float noise1(uint32_t x0, uint32_t x1, int shape, float) {
    if (shape == MFA_NOISE_UNIFORM) {
        const float u = (float)(x0 >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f;
        return 1.7320508075688772f * (2.0f * u - 1.0f);
    }
    const float u1 = fmaf((float)x0, 2.3283064365386963e-10f, 1.16415321826934814e-10f);
    const float u2 = fmaf((float)x1, 2.3283064365386963e-10f, 1.16415321826934814e-10f);
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}
__device__ __forceinline__ double noise1(uint32_t x0, uint32_t x1, int shape, double) {
    if (shape == MFA_NOISE_UNIFORM) {
        const float u = (float)(x0 >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f;
        return (double)(1.7320508075688772f * (2.0f * u - 1.0f));
    }
    const double u1 = ((double)x0 + 0.5) * 2.3283064365386963e-10;
    const double u2 = ((double)x1 + 0.5) * 2.3283064365386963e-10;
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

template <typename R>
__device__ __forceinline__ void lgv_noise3(uint32_t id, uint32_t step, const PairArgs& a, R g[3]) {
    const uint4 w = philox4x32_10(make_uint4(id, 0u, step, TAG_LGV), a.seed0, a.seed1);
    if (a.noise == MFA_NOISE_UNIFORM) {
        g[0] = noise1(w.x, 0u, 1, R(0)); g[1] = noise1(w.y, 0u, 1, R(0)); g[2] = noise1(w.z, 0u, 1, R(0));
        return;
    }
    const double u0 = ((double)w.x + 0.5) * 2.3283064365386963e-10;
    const double u1 = ((double)w.y + 0.5) * 2.3283064365386963e-10;
    const double u2 = ((double)w.z + 0.5) * 2.3283064365386963e-10;
    const double u3 = ((double)w.w + 0.5) * 2.3283064365386963e-10;
    const R r1 = (R)sqrt(-2.0 * log(u0)), r2 = (R)sqrt(-2.0 * log(u2));
    double s1, c1;
    sincospi(2.0 * u1, &s1, &c1);
    g[0] = r1 * (R)c1;
    g[1] = r1 * (R)s1;
    g[2] = r2 * (R)cospi(2.0 * u3);
}

// 9-3 wall (fluid_wall.f90:96-121) on one particle: returns F_z, adds energy.
template <typename R>
__device__ __forceinline__ R wall_force(const PairArgs& a, int t, R z, double& e) {
    R fz = 0;
    const R sw = (R)a.sigma_wall[t - 1], aw = (R)a.a_wall[t - 1];
    const R ae = a.wall_e_aw ? (R)a.a_w : aw;
    const R sw3 = sw * sw * sw, sw9 = sw3 * sw3 * sw3;
    const R faw = aw < 0 ? -aw : aw;
    const R cut = (R)a.wall_cut;
    auto term = [&](R zz, R& f, double& ee) {
        const R iz = (R)1 / zz;
        const R rd = sw * iz, rd3 = rd * rd * rd;
        const R iz2 = iz * iz, iz4 = iz2 * iz2, iz8 = iz4 * iz4;
        ee = (double)(faw * rd3 * rd3 * rd3 - ae * rd3);
        f = (R)9 * faw * sw9 * (iz8 * iz2) - (R)3 * aw * sw3 * iz4;
        if (cut > 0) {
            const R ic = (R)1 / cut, rc = sw * ic, rc3 = rc * rc * rc;
            ee -= (double)(faw * rc3 * rc3 * rc3 - ae * rc3);
        }
    };
    R f;
    double ee;
    if (cut <= 0 || z < cut) { term(z, f, ee); fz += f; e += ee; }
    if (a.wall_type == 2) {
        const R zt = (R)a.z_space_wall - z;
        if (cut <= 0 || zt < cut) { term(zt, f, ee); fz -= f; e += ee; }
    }
    return fz;
}

template <typename R, bool FUSE_WALL>
__global__ void __launch_bounds__(128) k_pair(PairArgs a) {
    typedef typename Vec4<R>::T R4;
    constexpr int NQ = FUSE_WALL ? 4 : 3;
    __shared__ R s_rc2[T8 * T8], s_eps[T8 * T8], s_sig2[T8 * T8], s_esh[T8 * T8], s_irc2[T8 * T8];
    for (int k = threadIdx.x; k < T8 * T8; k += blockDim.x) {
        s_rc2[k] = (R)a.tabs[1 * T8 * T8 + k];
        s_eps[k] = (R)a.tabs[2 * T8 * T8 + k];
        s_sig2[k] = (R)a.tabs[3 * T8 * T8 + k];
        s_esh[k] = (R)a.tabs[4 * T8 * T8 + k];
        s_irc2[k] = (R)a.tabs[5 * T8 * T8 + k];
    }
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
    if (t < a.n) {
        const R4* __restrict__ pos = (const R4*)a.pos_s;
        const R4* __restrict__ vel = (const R4*)a.vel_s;
        const long long step = *a.dstep;
        // fluid_fluid.f90:42-49 force switch-on
        R r2min = 0;
        if (a.fsw) {
            const double r_time = (double)(a.s_time + step - 1) * a.dt;
            r2min = r_time < a.r_2_min_time ? (R)((1.0 - r_time / a.r_2_min_time) * a.r_2_min_init) : (R)0;
        }
        const R4 pi = ldg4(&pos[t]);
        const int wi = wbits(pi.w);
        const int ti = wi & 0xff, ii = wi >> 8;
        const bool need_v = a.thermostat == MFA_THERMO_DPD || a.charged;
        R4 vi;
        if (need_v) vi = ldg4(&vel[t]);
        const R Lx = (R)a.L[0], Ly = (R)a.L[1], Lz = (R)a.L[2];
        const R iLx = (R)a.invL[0], iLy = (R)a.invL[1], iLz = (R)a.invL[2];
        const R sig = (R)a.sig, gam = (R)a.friction;
        R fx = 0, fy = 0, fz = 0;
        double e_lj = 0.0, vir = 0.0, e_c = 0.0;
        const int m = a.nnb[t];
        const int rowi = (ti - 1) * T8;
        for (int k = 0; k < m; ++k) {
            const int s = __ldg(&a.nbr[(size_t)k * a.n + t]);
            const R4 pj = ldg4(&pos[s]);
            R dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            dx = mimg(dx, Lx, iLx);
            dy = mimg(dy, Ly, iLy);
            if (a.symmetry == 1) dz = mimg(dz, Lz, iLz);
            const R r2 = dx * dx + dy * dy + dz * dz;
            const int wj = wbits(pj.w);
            const int ij = rowi + (wj & 0xff) - 1;
            if (r2 < s_rc2[ij]) {
                const R r2c = a.fsw ? (r2 > r2min ? r2 : r2min) : r2;
                const R inv_r2 = (R)1 / r2c;
                const R inv_r = rsqrt_(r2c);
                const R eps = s_eps[ij];
                const R r61 = s_sig2[ij] * inv_r2;
                const R r6 = r61 * r61 * r61;
                const R r12 = r6 * r6;
                e_lj += (double)(eps * ((r12 - r6) - s_esh[ij]));
                const R fs = eps * ((R)12 * r12 - (R)6 * r6) * inv_r2;   // force on i along d
                R fsum = fs;
                vir += (double)(fs * r2);
                if (a.thermostat == MFA_THERMO_DPD) {
                    // dpd_forces.f90:273-348 with Philox noise keyed by the pair
                    const int jj = wj >> 8;
                    const uint32_t lo = (uint32_t)min(ii, jj), hi = (uint32_t)max(ii, jj);
                    const uint4 w = philox4x32_10(make_uint4(lo, hi, (uint32_t)step, TAG_DPD), a.seed0, a.seed1);
                    const R g = noise1(w.x, w.y, a.noise, R(0));
                    R wr, wd;
                    if (a.dpd_weight == 1) { wr = 1; wd = 1; }
                    else { wr = (R)1 - sqrt_(r2c * s_irc2[ij]); wd = wr * wr; }
                    const R4 vj = ldg4(&vel[s]);
                    const R rd = ((vi.x - vj.x) * dx + (vi.y - vj.y) * dy + (vi.z - vj.z) * dz) * inv_r;
                    // F_i += (sig w_r g - gamma w_d (dv . rhat)) rhat, rhat = d * inv_r
                    fsum += (sig * wr * g - gam * wd * rd) * inv_r;
                }
                if (a.charged && a.real_in_lj) {
                    // ewald_real.f90:411-428, inside the LJ range (reference behaviour)
                    const R4 vj = ldg4(&vel[s]);
                    const R qq = vi.w * vj.w;
                    const R r = (R)1 / inv_r;
                    const R ir = inv_r;
                    const R ec = erfc_((R)a.sqrt_alpha * r);
                    e_c += (double)(qq * ec * ir);
                    const R fsc = qq * (R)a.sqrt_alpha * (R)a.inv_sqrt_pi * (R)2 * exp_(-(R)a.alpha_c * r2c) * ir
                                  + qq * ec * ir * ir;
                    fsum += fsc * ir;
                    vir += (double)(fsc * r2 * ir);
                }
                fx += fsum * dx; fy += fsum * dy; fz += fsum * dz;
            }
            if (a.charged && !a.real_in_lj && r2 < (R)a.ewald_rc_2) {
                const R4 vj = ldg4(&vel[s]);
                const R qq = vi.w * vj.w;
                const R ir = rsqrt_(r2);
                const R r = (R)1 / ir;
                const R ec = erfc_((R)a.sqrt_alpha * r);
                e_c += (double)(qq * ec * ir);
                const R fsc = qq * (R)a.sqrt_alpha * (R)a.inv_sqrt_pi * (R)2 * exp_(-(R)a.alpha_c * r2) * ir
                              + qq * ec * ir * ir;
                const R f = fsc * ir;
                fx += f * dx; fy += f * dy; fz += f * dz;
                vir += (double)(fsc * r2 * ir);
            }
        }
        if (a.thermostat == MFA_THERMO_LGV) {
            // lgv_forces.f90:377-393
            R g[3];
            lgv_noise3<R>((uint32_t)ii, (uint32_t)step, a, g);
            const double mi = a.mass[ii];
            const R sm = (R)sqrt(mi), gm = (R)(a.friction * mi);
            if (!need_v) vi = ldg4(&vel[t]);
            fx += sig * g[0] * sm - gm * vi.x;
            fy += sig * g[1] * sm - gm * vi.y;
            fz += sig * g[2] * sm - gm * vi.z;
        }
        if (FUSE_WALL) {
            double ew = 0.0;
            fz += wall_force<R>(a, ti, pi.z, ew);
            acc[NQ - 1] = ew;
        }
        acc[0] = 0.5 * e_lj;   // full list: each pair seen from both sides
        acc[1] = 0.5 * vir;
        acc[2] = a.coul_energy_factor * e_c;
        R4* f4 = (R4*)a.force;
        R4 o;
        if (a.accumulate) {
            o = f4[ii];
            o.x += fx; o.y += fy; o.z += fz;
        } else {
            o.x = fx; o.y = fy; o.z = fz; o.w = 0;
        }
        f4[ii] = o;
    }
    block_sum_commit<NQ>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_VFF);
}

}  // namespace

int launch_pair(mfa_ctx* c, int fuse_wall, int accumulate) {
    if (!c->lists_valid) return MFA_ERR_STATE;
    PairArgs a;
    a.pos_s = c->pos_s; a.vel_s = c->vel_s; a.nbr = c->nbr; a.nnb = c->nnb;
    a.mass = c->mass; a.tabs = c->tabs; a.force = c->force; a.dstep = c->dstep;
    a.partials = c->partials + (size_t)R_PAIR * 4 * c->max_blocks;
    a.counter = c->counters + R_PAIR;
    a.dscal = c->dscal;
    a.n = c->n;
    a.max_blocks = c->max_blocks;
    const mfa_params& p = c->p;
    a.symmetry = p.symmetry; a.thermostat = p.thermostat; a.dpd_weight = p.dpd_weight;
    a.noise = p.noise; a.charged = p.charged;
    a.real_in_lj = (p.quirks & MFA_Q_EWALD_REAL_IN_LJ) != 0;
    a.fsw = p.force_switch_on;
    a.wall_type = p.wall; a.wall_e_aw = (p.quirks & MFA_Q_WALL_ENERGY_AW) != 0;
    a.accumulate = accumulate;
    // ewald_real.f90:416 adds every visit; a full list (my_binning) visits each
    // pair twice, the half list once.
    a.coul_energy_factor = c->bin_type == 1 ? 1.0 : 0.5;
    for (int d = 0; d < 3; ++d) { a.L[d] = p.boundary[d]; a.invL[d] = c->inv_boundary[d]; }
    a.sig = p.sig; a.friction = p.friction; a.dt = p.dt;
    a.r_2_min_init = p.r_2_min_init; a.r_2_min_time = p.r_2_min_time; a.s_time = p.s_time;
    a.sqrt_alpha = p.sqrt_alpha; a.alpha_c = p.alpha_c; a.inv_sqrt_pi = p.inv_sqrt_pi;
    a.ewald_rc_2 = p.ewald_rc_2;
    for (int k = 0; k < T8; ++k) { a.a_wall[k] = p.a_wall[k]; a.sigma_wall[k] = p.sigma_wall[k]; }
    a.a_w = p.a_w; a.z_space_wall = p.z_space_wall; a.wall_cut = p.wall_cut;
    a.seed0 = (uint32_t)p.seed; a.seed1 = (uint32_t)(p.seed >> 32);
    const int T = 128;
    const int nb = (c->n + T - 1) / T;
    if (nb > c->max_blocks) return MFA_ERR_ARGS;
    const bool fw = fuse_wall && p.wall == 2;
    if (c->prec == MFA_MIXED) {
        if (fw) k_pair<float, true><<<nb, T, 0, c->st>>>(a);
        else k_pair<float, false><<<nb, T, 0, c->st>>>(a);
    } else {
        if (fw) k_pair<double, true><<<nb, T, 0, c->st>>>(a);
        else k_pair<double, false><<<nb, T, 0, c->st>>>(a);
    }
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}
