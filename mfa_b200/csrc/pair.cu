// Pair forces: fluid_fluid.f90 with dpd_forces (THERMOSTAT 0), ewald_real
// (charged systems, fused into the same pass) and lgv_forces (THERMOSTAT 1),
// plus optionally the 9-3 walls of fluid_wall.f90 in the per-particle epilogue.
//
// Work unit: a warp takes 32 consecutive cell-sorted slots ("owners") and walks
// their Verlet rows column by column, K entries per lane per round (the K
// position gathers of a lane are in flight together):
//   test   each lane forms d = r_i - r_j (minimum image) and r^2 for its
//          entries; the in-range ones are appended to the warp's queue in shared
//          memory (ballot + popc: no holes), with d, r^2, j and j's id/type;
//   batch  whenever the queue holds 32 pairs, every lane evaluates one of them
//          (LJ/WCA, Philox noise + DPD, Ewald real space): the expensive physics
//          always runs with all 32 lanes busy.
// Newton's third law: with the half list of binning.f90 (pair listed once, in
// the row of its lower slot) the partner j receives -f through a vector
// reduction on the force array (red.global.add.v4.f32 in MIXED), the owner's
// share is summed in shared memory and added once per owner at the end.  With
// the full list of my_binning.f90 only the owner side is updated, as the
// reference does (fluid_fluid.f90:236).  The force array is only ever added
// to; the caller zeroes it (mfa_zero_forces, or the integrator on the fast
// path), so the summation order of a particle's force is not fixed: forces
// agree with a fixed-order sum to rounding, not bit for bit.
//
// DPD noise of a pair is drawn from Philox-4x32-10 keyed by (step, min(i,j),
// max(i,j)) (both sides would see the same number; each pair is evaluated once).
//
// Two launch modes (the autotuner picks):
//   untiled  CTA = blockDim consecutive slots, neighbour records read through
//            L1/L2;
//   tiled    CTA = one cell row (fixed y, z); the neighbouring cell rows, merged
//            into contiguous slot runs, are staged into shared memory with bulk
//            asynchronous copies (cp.async.bulk, completion on an mbarrier,
//            bounded wait) and list entries are translated into tile indices.
//            A row whose neighbourhood does not fit the tile reads global memory.
// R = float in MIXED mode (FP32 force math; each thread's energy and virial
// terms summed in FP32, the grid-wide sums in FP64), double in FP64 mode.
#include "mfa_internal.cuh"

#include <string.h>

namespace {

struct PairArgs {
    const void* pos_s;
    const void* vel_s;
    const int32_t* __restrict__ nbr;
    const int32_t* __restrict__ ccount;       // entries per 32-slot chunk
    const int32_t* __restrict__ cell_start;
    int32_t* flags;
    const double* mass;
    const double* tabs;
    void* force;
    const int64_t* dstep;
    double* partials;
    unsigned* counter;
    double* dscal;
    int n, max_blocks, maxnb;
    unsigned long long* qctr;  // work-queue tickets (untiled launches with a queue), or null
    int qmod;                  // tickets per launch: pieces + warps of the grid
    int split;                 // pieces per chunk (untiled): warps that share one chunk's entries
    int zero_slots;            // energy slots the launch resets: 1 v_coul k-space and slab parts, 2 v_fluid_wall
    int defer_sum;             // energies: block partials only; the integrator launch after it adds them up
    int nb[3], rule, wy, nseg, tile_cap, rowmode;
    int half;                 // 1: half list (partner gets -f), 0: full list
    int symmetry, thermostat, dpd_weight, noise, charged, real_in_lj, fsw;
    int wall_type, wall_e_aw, fuse_wall;
    double lj_energy_factor;  // 1 (half list) or 1/2 (full list: every pair seen twice)
    double L[3], invL[3];
    double sig, friction, dt;
    int elog_every;           // energy log period (0: none): steps whose energies are wanted
    double r_2_min_init, r_2_min_time;
    long long s_time;
    double sqrt_alpha, alpha_c, inv_sqrt_pi, ewald_rc_2;
    double a_wall[T8], sigma_wall[T8], a_w, z_space_wall, wall_cut;
    uint32_t seed0, seed1;
    PhiloxKeys key;           // Philox round keys of (seed0, seed1)
    // the same constants rounded to FP32 once on the host: the FP32 kernels
    // take them straight from the parameter bank instead of holding converted
    // copies in registers
    float fL[3], fiL[3], fsig, fgam, fewrc2, fsqrt_alpha, falpha_c, finv_sqrt_pi;
};

// a run constant in the kernel's precision
template <typename R> __device__ __forceinline__ R pv(double d, float f);
template <> __device__ __forceinline__ float pv<float>(double, float f) { return f; }
template <> __device__ __forceinline__ double pv<double>(double d, float) { return d; }

template <typename R> struct Vec4;
template <> struct Vec4<float> { typedef float4 T; };
template <> struct Vec4<double> { typedef double4 T; };

// d - L*int(2d/L) (fluid_fluid.f90:84-88); truncf rounds toward zero like int()
__device__ __forceinline__ float mimg(float d, float L, float iL) { return fmaf(-L, truncf(2.0f * d * iL), d); }
__device__ __forceinline__ double mimg(double d, double L, double iL) {
    return d - L * (double)(int)(2.0 * d * iL);
}
__device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
__device__ __forceinline__ float rcp_(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double rcp_(double x) { return 1.0 / x; }
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(1.0 / x); }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }

// erfc(x) and exp(-x^2) of the Ewald real-space term (x = sqrt(alpha) r,
// x2 = alpha r^2), the library functions in the kernel's precision
__device__ __forceinline__ void ewald_erfc_exp(float x, float x2, float& ec, float& ex) {
    ec = erfcf(x);
    ex = expf(-x2);
}
__device__ __forceinline__ void ewald_erfc_exp(double x, double x2, double& ec, double& ex) {
    ec = erfc(x);
    ex = exp(-x2);
}

// Gaussian (Box-Muller) or uniform variate from two Philox words.
__device__ __forceinline__ float noise1(uint32_t x0, uint32_t x1, int shape, float) {
    if (shape == MFA_NOISE_UNIFORM) {
        const float u = (float)(x0 >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f;
        return 1.7320508075688772f * (2.0f * u - 1.0f);
    }
    // FP32 (mixed) path: the hardware approximations of log, cos and 1/sqrt;
    // their ~1e-6 relative error is far below the statistical noise they model.
    // cos(2 pi u2) = -cos(2 pi u2 - pi) keeps __cosf inside [-pi, pi].
    const float u1 = fmaf((float)x0, 2.3283064365386963e-10f, 1.16415321826934814e-10f);
    const float u2 = fmaf((float)x1, 2.3283064365386963e-10f, 1.16415321826934814e-10f);
    const float s = -2.0f * __logf(u1);
    const float r = s > 0.0f ? s * rsqrtf(s) : 0.0f;
    return -r * __cosf(fmaf(6.283185307179586f, u2, -3.14159265358979f));
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

// 9-3 wall (fluid_wall.f90:96-121) on one particle: returns F_z, adds energy.
template <typename R, typename E>
__device__ __forceinline__ R wall_force(const PairArgs& a, int t, R z, E& e) {
    R fz = 0;
    const R sw = (R)a.sigma_wall[t - 1], aw = (R)a.a_wall[t - 1];
    const R ae = a.wall_e_aw ? (R)a.a_w : aw;
    const R cut = (R)a.wall_cut;
    R f;
    double ee;
    if (cut <= 0 || z < cut) { wall93_term<R>(z, sw, aw, ae, cut, f, ee); fz += f; e += (E)ee; }
    if (a.wall_type == 2) {
        const R zt = (R)a.z_space_wall - z;
        if (cut <= 0 || zt < cut) { wall93_term<R>(zt, sw, aw, ae, cut, f, ee); fz -= f; e += (E)ee; }
    }
    return fz;
}

// force[i] += (x, y, z) by a reduction in L2 (no return value: RED, not ATOM)
__device__ __forceinline__ void red_add(float4* f, float x, float y, float z) {
    atomicAdd(f, make_float4(x, y, z, 0.0f));
}
__device__ __forceinline__ void red_add(double4* f, double x, double y, double z) {
    double* p = (double*)f;
    atomicAdd(p, x);
    atomicAdd(p + 1, y);
    atomicAdd(p + 2, z);
}

// ---- bulk-copy staging (cp.async.bulk global -> shared, mbarrier completion) ----
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: gives up after `limit` polls; between polls the warp sleeps
// (32 ns doubling to 512 ns), so waiting warps do not take issue slots from
// the CTAs on the same SM that have their data
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit) {
    unsigned ns = 32;
    for (long long it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(ns);
        if (ns < 512) ns <<= 1;
    }
    return false;
}
constexpr long long WAIT_LIMIT = 1LL << 23;   // ~4 s of polls at the longest sleep

// Feature bits of a pair-kernel instantiation.  A specialised instantiation
// compiles only the physics a run uses (fewer registers, more resident warps);
// FT_GENERIC reads every switch at run time and serves all other combinations.
enum {
    FT_DPD = 1,        // DPD thermostat (dpd_forces)
    FT_LGV = 2,        // Langevin thermostat (lgv_forces)
    FT_QLJ = 4,        // Ewald real space inside the LJ range (reference)
    FT_QSEP = 8,       // Ewald real space with its own cutoff
    FT_FSW = 16,       // force switch-on clamp
    FT_WALL = 32,      // 9-3 walls in the epilogue
    FT_GENERIC = 128
};

template <int FT>
__device__ __forceinline__ bool has(const PairArgs& a, int bit) {
    if (FT & FT_GENERIC) {
        switch (bit) {
            case FT_DPD: return a.thermostat == MFA_THERMO_DPD;
            case FT_LGV: return a.thermostat == MFA_THERMO_LGV;
            case FT_QLJ: return a.charged && a.real_in_lj;
            case FT_QSEP: return a.charged && !a.real_in_lj;
            case FT_FSW: return a.fsw != 0;
            case FT_WALL: return a.fuse_wall != 0;
        }
        return false;
    }
    return (FT & bit) != 0;
}

// queue capacity of a warp: up to 31 pairs left over from the previous round
// plus 32 lanes x K tested entries
template <int K> constexpr int qcap() { return 32 * K + 32; }

// per-warp shared memory: queue (d, r^2), queue (j, id/type of j), owner
// positions and velocities, owner id/type, owner force accumulators
template <typename R, int K>
constexpr size_t warp_bytes() {
    return (size_t)qcap<K>() * (sizeof(typename Vec4<R>::T) + sizeof(int2)) + 64 * sizeof(typename Vec4<R>::T) +
           32 * sizeof(int) + 96 * sizeof(R);
}

constexpr int MAXPC = 16;   // staged slot runs (at most 9 neighbouring rows)

// 48 registers in FP32 (40 resident warps per SM: one wave for ~190k
// particles), 128 in FP64, where the doubled operands would otherwise spill
template <typename R, int K, int FT>
__device__ __forceinline__ void pair_body(const PairArgs& a, Blk blk) {
    typedef typename Vec4<R>::T R4;
    constexpr int QC = qcap<K>();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R4* tpos = (R4*)smem_raw;
    R4* tvel = tpos + a.tile_cap;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    unsigned char* wmem = (unsigned char*)(tvel + a.tile_cap) + (size_t)warp * warp_bytes<R, K>();
    R4* qd = (R4*)wmem;                          // QC x (dx, dy, dz, r^2)
    R4* own_v = qd + QC;                         // 32 owner velocities (w = charge)
    R4* own_p = own_v + 32;                      // 32 owner positions
    int2* qw = (int2*)(own_p + 32);              // QC x (owner << 23 | j index, id << 8 | type of j)
    int* own_w = (int*)(qw + QC);                // 32 owner id << 8 | type
    R* facc = (R*)(own_w + 32);                  // 3 x 32 owner force accumulators
    __shared__ R s_rc2[T8 * T8], s_eps[T8 * T8], s_sig2[T8 * T8], s_esh[T8 * T8], s_irc2[T8 * T8];
    __shared__ int pc_start[MAXPC], pc_len[MAXPC], pc_base[MAXPC];
    __shared__ int row_r[MAXPC], row_s[MAXPC], row_l[MAXPC];
    __shared__ int s_npc, s_mode;
    __shared__ __align__(8) uint64_t bar;
    const bool DPD = has<FT>(a, FT_DPD), LGV = has<FT>(a, FT_LGV), QLJ = has<FT>(a, FT_QLJ);
    const bool QSEP = has<FT>(a, FT_QSEP), FSW = has<FT>(a, FT_FSW), WALL = has<FT>(a, FT_WALL);
    const bool need_v = DPD || QLJ || QSEP;
    const int nx = a.nb[0], ny = a.nb[1], nz = a.nb[2];
    if (a.zero_slots && blk.id == 0 && threadIdx.x == 0) {
        // the subroutine entry points' resets (fluid_fluid.f90:17: v_coul),
        // here rather than as copies of their own on the stream
        if (a.zero_slots & 1) { a.dscal[S_VCK] = 0.0; a.dscal[S_VDIP] = 0.0; }
        if (a.zero_slots & 2) a.dscal[S_VFW] = 0.0;
    }
    int p0, p1;
    if (a.rowmode) {
        const int row = blk.id;
        p0 = a.cell_start[nx * row];
        p1 = a.cell_start[nx * row + nx];
        // staging: the neighbouring rows (in the order the list builder scans
        // them), merged into runs of consecutive slots, copied back to back
        if (warp == 0) {
            if (lane < a.nseg) {
                int ky, kz;
                neighbour_row(a.rule, row % ny, row / ny, lane % a.wy, lane / a.wy, ny, nz, ky, kz);
                const int r = ky + ny * kz;
                row_r[lane] = r;
                row_s[lane] = a.cell_start[nx * r];
                row_l[lane] = a.cell_start[nx * r + nx] - row_s[lane];
            }
            __syncwarp();
            if (lane == 0) {
                int npc = 0, total = 0;
                for (int k = 0; k < a.nseg; ++k) {
                    if (k > 0 && row_r[k] == row_r[k - 1] + 1) {
                        pc_len[npc - 1] += row_l[k];
                    } else {
                        pc_start[npc] = row_s[k];
                        pc_len[npc] = row_l[k];
                        ++npc;
                    }
                }
                for (int p = 0; p < npc; ++p) { pc_base[p] = total; total += pc_len[p]; }
                const int mode = total <= a.tile_cap ? 1 : 0;
                s_npc = npc;
                s_mode = mode;
                if (mode) {
                    mbar_init(&bar);
                    mbar_expect_tx(&bar, (uint32_t)total * (uint32_t)sizeof(R4) * (need_v ? 2u : 1u));
                }
            }
            __syncwarp();
            if (s_mode && lane < s_npc && pc_len[lane] > 0) {
                const uint32_t bytes = (uint32_t)pc_len[lane] * (uint32_t)sizeof(R4);
                bulk_g2s(tpos + pc_base[lane], (const R4*)a.pos_s + pc_start[lane], bytes, &bar);
                if (need_v) bulk_g2s(tvel + pc_base[lane], (const R4*)a.vel_s + pc_start[lane], bytes, &bar);
            }
        }
    } else if (a.qctr) {
        p0 = 0;                  // work queue: any chunk of the system
        p1 = a.n;
        if (threadIdx.x == 0) { s_mode = 0; s_npc = 0; }
    } else {
        p0 = 0;                  // static: warp w of the grid takes pieces w, w + warps, ...
        p1 = a.n;
        if (threadIdx.x == 0) { s_mode = 0; s_npc = 0; }
    }
    for (int k = threadIdx.x; k < T8 * T8; k += blockDim.x) {
        s_rc2[k] = (R)a.tabs[1 * T8 * T8 + k];
        s_eps[k] = (R)a.tabs[2 * T8 * T8 + k];
        s_sig2[k] = (R)a.tabs[3 * T8 * T8 + k];
        s_esh[k] = (R)a.tabs[4 * T8 * T8 + k];
        s_irc2[k] = (R)a.tabs[5 * T8 * T8 + k];
    }
    __syncthreads();
    const bool tile = s_mode != 0;
    const int npc = s_npc;
    bool ok = true;
    if (tile && !mbar_wait_bounded(&bar, 0, WAIT_LIMIT)) {
        // the copies did not complete in time: report, wait for them once more
        // (the tile must not be released while they are in flight), skip the work
        set_err(a.flags, MFA_ERR_TIMEOUT);
        mbar_wait_bounded(&bar, 0, WAIT_LIMIT);
        ok = false;
    }
    const bool valid = __syncthreads_and(ok) != 0;   // uniform over the CTA
    const R4* __restrict__ gpos = (const R4*)a.pos_s;
    const R4* __restrict__ gvel = (const R4*)a.vel_s;
    const R4* spos = tile ? tpos : gpos;           // where neighbour records are read
    const R4* svel = tile ? tvel : gvel;
    R4* f4 = (R4*)a.force;
    const long long step = *a.dstep;
    const bool EN = energy_needed(a.dstep, a.elog_every);   // uniform over the grid
    R r2min = 0;
    if (FSW) {
        // fluid_fluid.f90:42-49 force switch-on
        const double r_time = (double)(a.s_time + step - 1) * a.dt;
        r2min = r_time < a.r_2_min_time ? (R)((1.0 - r_time / a.r_2_min_time) * a.r_2_min_init) : (R)0;
    }
#define Lx pv<R>(a.L[0], a.fL[0])
#define Ly pv<R>(a.L[1], a.fL[1])
#define Lz pv<R>(a.L[2], a.fL[2])
#define iLx pv<R>(a.invL[0], a.fiL[0])
#define iLy pv<R>(a.invL[1], a.fiL[1])
#define iLz pv<R>(a.invL[2], a.fiL[2])
#define sig pv<R>(a.sig, a.fsig)
#define gam pv<R>(a.friction, a.fgam)
#define ewrc2 pv<R>(a.ewald_rc_2, a.fewrc2)
#define SQA pv<R>(a.sqrt_alpha, a.fsqrt_alpha)
#define ALC pv<R>(a.alpha_c, a.falpha_c)
#define ISP pv<R>(a.inv_sqrt_pi, a.finv_sqrt_pi)
    const unsigned lt_mask = (1u << lane) - 1u;
    // per-thread energy sums in R (a thread sums a handful of terms), reduced
    // over the grid in FP64
    R e_lj = 0, vir = 0, e_c = 0, e_w = 0;

    // one queued pair: physics, owner share into shared memory, partner share
    // into the force array
    auto evaluate = [&](int q) {
        const R4 d = qd[q];
        const int2 w = qw[q];
        const int ol = w.x >> 23, jx = w.x & 0x7fffff, wj = w.y;
        const int wi = own_w[ol];
        const int ij = ((wi & 0xff) - 1) * T8 + (wj & 0xff) - 1;
        const R r2 = d.w;
        R4 vq, vj;
        if (need_v) { vq = own_v[ol]; vj = svel[jx]; }
        R fsum = 0;
        if (r2 < s_rc2[ij]) {
            const R r2c = FSW ? (r2 > r2min ? r2 : r2min) : r2;
            const R inv_r2 = rcp_(r2c);
            const R eps = s_eps[ij];
            const R r61 = s_sig2[ij] * inv_r2;
            const R r6 = r61 * r61 * r61;
            const R r12 = r6 * r6;
            if (EN) e_lj += eps * ((r12 - r6) - s_esh[ij]);
            const R fs = eps * ((R)12 * r12 - (R)6 * r6) * inv_r2;   // force on i along d
            fsum = fs;
            if (EN) vir += fs * r2;
            if (DPD || QLJ) {
                const R inv_r = rsqrt_(r2c);
                if (DPD) {
                    // dpd_forces.f90:19-94 with Philox noise keyed by the pair
                    const int ii = wi >> 8, jj = wj >> 8;
                    const uint32_t lo = (uint32_t)min(ii, jj), hi = (uint32_t)max(ii, jj);
                    const uint4 ph = philox4x32_10(make_uint4(lo, hi, (uint32_t)step, TAG_DPD), a.key);
                    const R g = noise1(ph.x, ph.y, a.noise, R(0));
                    R wr, wd;
                    if (a.dpd_weight == 1) { wr = 1; wd = 1; }
                    else { wr = (R)1 - sqrt_(r2c * s_irc2[ij]); wd = wr * wr; }
                    const R rd = ((vq.x - vj.x) * d.x + (vq.y - vj.y) * d.y + (vq.z - vj.z) * d.z) * inv_r;
                    // F_i += (sig w_r g - gamma w_d (dv . rhat)) rhat, rhat = d * inv_r
                    fsum += (sig * wr * g - gam * wd * rd) * inv_r;
                }
                if (QLJ) {
                    // ewald_real.f90:15-33, inside the LJ range (reference behaviour)
                    const R qq = vq.w * vj.w;
                    const R r = r2c * inv_r;
                    R ec, ex;
                    ewald_erfc_exp(SQA * r, ALC * r2c, ec, ex);
                    if (EN) e_c += qq * ec * inv_r;
                    const R fsc = qq * SQA * ISP * (R)2 * ex * inv_r + qq * ec * inv_r * inv_r;
                    fsum += fsc * inv_r;
                    if (EN) vir += fsc * r2 * inv_r;
                }
            }
        }
        if (QSEP && r2 < ewrc2) {
            const R qq = vq.w * vj.w;
            const R ir = rsqrt_(r2);
            const R r = r2 * ir;
            R ec, ex;
            ewald_erfc_exp(SQA * r, ALC * r2, ec, ex);
            if (EN) e_c += qq * ec * ir;
            const R fsc = qq * SQA * ISP * (R)2 * ex * ir + qq * ec * ir * ir;
            fsum += fsc * ir;
            if (EN) vir += fsc * r2 * ir;
        }
        const R fx = fsum * d.x, fy = fsum * d.y, fz = fsum * d.z;
        atomicAdd(&facc[ol], fx);
        atomicAdd(&facc[32 + ol], fy);
        atomicAdd(&facc[64 + ol], fz);
        if (a.half) red_add(&f4[wj >> 8], -fx, -fy, -fz);
    };

    // chunks of 32 slots, each with its list as one run of entries (partner
    // slot << 5 | owner lane).  An untiled launch cuts every chunk's run into
    // `split` pieces of equal length (a piece: chunk * split + part), so that a
    // small system with long lists still spreads over every SM; warp w of the
    // grid takes pieces w, w + (warps of the grid), ...  A tiled CTA (one cell
    // row, split 1) takes the chunks overlapping its row and keeps the entries
    // whose owner lies in the row.  The lanes walk a piece's entries together,
    // K per lane per round, whatever row they belong to.
    const long long capc = 32LL * a.maxnb;
    // with the work queue of an untiled launch, pieces are tickets from a
    // 64-bit counter shared by the grid.  Every launch draws exactly
    // npiece + (warps of the grid) tickets (each warp stops at its first ticket
    // past the pieces), so a launch starts at a multiple of that number and
    // ticket % qmod is its piece.
    const bool dyn = a.qctr != nullptr;
    const int S = a.rowmode ? 1 : a.split;
    const int pc_end = ((p1 + 31) >> 5) * S;
    int pc = a.rowmode ? (p0 >> 5) + warp : blk.id * nwarp + warp;
    const int pc_step = a.rowmode ? nwarp : blk.n * nwarp;
    if (dyn) {
        unsigned long long tk = 0;
        if (lane == 0) tk = atomicAdd(a.qctr, 1ull);
        pc = (int)(__shfl_sync(0xffffffffu, tk, 0) % (unsigned long long)a.qmod);
    }
    for (; valid && pc < pc_end; ) {
        const int ch = S == 1 ? pc : pc / S;
        const int t = (ch << 5) + lane;
        const bool act = t >= p0 && t < p1;
        R4 pi;
        if (act) {
            pi = ldg4(&gpos[t]);
            if (need_v || LGV) own_v[lane] = ldg4(&gvel[t]);
        } else {
            pi.x = pi.y = pi.z = 0;
            pi.w = 0;
        }
        const int wi = act ? wbits(pi.w) : 0;
        own_w[lane] = wi;
        own_p[lane] = pi;
        facc[lane] = 0;
        facc[32 + lane] = 0;
        facc[64 + lane] = 0;
        const int cnt = a.ccount[ch];
        const int eb = S == 1 ? 0 : (int)(((long long)cnt * (pc - ch * S)) / S);
        const int ee = S == 1 ? cnt : (int)(((long long)cnt * (pc - ch * S + 1)) / S);
        const int32_t* __restrict__ crow = a.nbr + (size_t)ch * capc;
        int qn = 0;
        __syncwarp();
        for (int e0 = eb; e0 < ee; e0 += 32 * K) {
            int jx[K], ol[K];
            R4 pj[K];
#pragma unroll
            for (int u = 0; u < K; ++u) {
                jx[u] = -1;
                ol[u] = 0;
                const int e = e0 + 32 * u + lane;
                if (e < ee) {
                    const int ent = __ldg(&crow[e]);
                    ol[u] = ent & 31;
                    jx[u] = (int)((unsigned)ent >> 5);
                }
            }
#pragma unroll
            for (int u = 0; u < K; ++u) {
                // owner outside this CTA's row (tiled: a chunk may straddle two
                // rows; untiled, every listed owner is one of the piece's lanes)
                if (tile && jx[u] >= 0 && own_w[ol[u]] == 0) jx[u] = -1;
                if (jx[u] >= 0) {
                    if (tile) {
                        // list entries are slots; find the staged run holding the slot
                        int ix = -1;
                        for (int p = 0; p < npc; ++p) {
                            const unsigned off = (unsigned)(jx[u] - pc_start[p]);
                            if (off < (unsigned)pc_len[p]) { ix = pc_base[p] + (int)off; break; }
                        }
                        if (ix < 0) set_err(a.flags, MFA_ERR_STATE);
                        jx[u] = ix;
                    }
                    if (jx[u] >= 0) pj[u] = spos[jx[u]];
                }
            }
#pragma unroll
            for (int u = 0; u < K; ++u) {
                bool keep = false;
                R dx = 0, dy = 0, dz = 0, r2 = 0;
                int wj = 0;
                if (jx[u] >= 0) {
                    const R4 po = own_p[ol[u]];
                    dx = mimg(po.x - pj[u].x, Lx, iLx);
                    dy = mimg(po.y - pj[u].y, Ly, iLy);
                    dz = po.z - pj[u].z;
                    if (a.symmetry == 1) dz = mimg(dz, Lz, iLz);
                    r2 = dx * dx + dy * dy + dz * dz;
                    wj = wbits(pj[u].w);
                    const int rowo = ((wbits(po.w) & 0xff) - 1) * T8 - 1;   // the owner's type
                    keep = r2 < s_rc2[rowo + (wj & 0xff)] || (QSEP && r2 < ewrc2);
                }
                const unsigned mask = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int pos = qn + __popc(mask & lt_mask);
                    R4 e;
                    e.x = dx; e.y = dy; e.z = dz; e.w = r2;
                    qd[pos] = e;
                    qw[pos] = make_int2((ol[u] << 23) | jx[u], wj);
                }
                qn += __popc(mask);
            }
            __syncwarp();
            while (qn >= 32) {
                evaluate(qn - 32 + lane);
                qn -= 32;
                __syncwarp();
            }
        }
        if (lane < qn) evaluate(lane);
        __syncwarp();
        if (act) {
            // the piece's part of its chunk, recomputed here rather than held
            // through the entry loop
            const int part = S == 1 ? 0 : pc % S;
            R fx = facc[lane], fy = facc[32 + lane], fz = facc[64 + lane];
            const int ti = wi & 0xff, ii = wi >> 8;
            if (LGV && part == 0) {
                // lgv_forces.f90:22-41
                R g[3];
                lgv_noise3<R>((uint32_t)ii, (uint32_t)step, a.noise, a.seed0, a.seed1, g);
                const double mi = a.mass[ii];
                const R sm = (R)sqrt(mi), gm = (R)(a.friction * mi);
                const R4 vi = own_v[lane];
                fx += sig * g[0] * sm - gm * vi.x;
                fy += sig * g[1] * sm - gm * vi.y;
                fz += sig * g[2] * sm - gm * vi.z;
            }
            if (WALL && part == 0) fz += wall_force<R>(a, ti, pi.z, e_w);
            if (part == 0 || fx != (R)0 || fy != (R)0 || fz != (R)0) red_add(&f4[ii], fx, fy, fz);
        }
        __syncwarp();
        if (dyn) {
            unsigned long long tk = 0;
            if (lane == 0) tk = atomicAdd(a.qctr, 1ull);
            pc = (int)(__shfl_sync(0xffffffffu, tk, 0) % (unsigned long long)a.qmod);
        } else {
            pc += pc_step;
        }
    }
    if (!EN) return;   // no energies this step: nothing to reduce
    // with defer_sum the grid-wide sum is left to the next kernel (the time
    // step's integrator, reduce_pair_partials), off this kernel's tail
    if (WALL) {
        double acc[4] = {a.lj_energy_factor * (double)e_lj, a.lj_energy_factor * (double)vir, (double)e_c,
                         (double)e_w};
        if (a.defer_sum) block_partials<4>(acc, a.partials, a.max_blocks, blk);
        else block_sum_commit<4>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_VFF, blk);
    } else {
        double acc[3] = {a.lj_energy_factor * (double)e_lj, a.lj_energy_factor * (double)vir, (double)e_c};
        if (a.defer_sum) block_partials<3>(acc, a.partials, a.max_blocks, blk);
        else block_sum_commit<3>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_VFF, blk);
    }
}
#undef Lx
#undef Ly
#undef Lz
#undef iLx
#undef iLy
#undef iLz
#undef sig
#undef gam
#undef ewrc2
#undef SQA
#undef ALC
#undef ISP

template <typename R, int K, int FT>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 2) k_pair(PairArgs a) {
    pair_body<R, K, FT>(a, plain_blk());
}
// one launch for several contexts (argument records in device memory)
template <typename R, int K, int FT>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 2)
    k_pair_grouped(const PairArgs* __restrict__ as, const int* __restrict__ off, int nsys) {
    const int s = group_of(off, nsys, blockIdx.x);
    pair_body<R, K, FT>(as[s], group_blk(off, s));
}

// the feature sets the time-step fast path and the subroutine entry points
// use, each compiled on its own
constexpr int FT_SETS[] = {0, FT_DPD, FT_DPD | FT_WALL, FT_WALL, FT_LGV, FT_LGV | FT_WALL, FT_LGV | FT_QSEP,
                           FT_LGV | FT_QLJ, FT_DPD | FT_QSEP, FT_DPD | FT_QLJ};
constexpr int N_FT_SETS = sizeof(FT_SETS) / sizeof(int);

// a grouped launch: argument records in device memory, block offsets per context
struct Group {
    const PairArgs* args;
    const int* off;
    int nsys;
};

template <typename R, int K, int F>
void launch_one(const PairArgs& a, const Group* g, int grid, int block, size_t smem, cudaStream_t st) {
    if (g) k_pair_grouped<R, K, F><<<grid, block, smem, st>>>(g->args, g->off, g->nsys);
    else k_pair<R, K, F><<<grid, block, smem, st>>>(a);
}
template <typename R, int K, int F>
int attr_one(size_t smem) {
    if (cudaFuncSetAttribute(k_pair<R, K, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_pair_grouped<R, K, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return MFA_ERR_CUDA;
    return MFA_OK;
}

template <typename R, int K, int I>
struct Dispatch {
    static void run(int ft, const PairArgs& a, const Group* g, int grid, int block, size_t smem, cudaStream_t st) {
        if (ft == FT_SETS[I]) {
            launch_one<R, K, FT_SETS[I]>(a, g, grid, block, smem, st);
            return;
        }
        Dispatch<R, K, I - 1>::run(ft, a, g, grid, block, smem, st);
    }
    static int attr(size_t smem) {
        const int rc = attr_one<R, K, FT_SETS[I]>(smem);
        if (rc != MFA_OK) return rc;
        return Dispatch<R, K, I - 1>::attr(smem);
    }
};
template <typename R, int K>
struct Dispatch<R, K, -1> {
    static void run(int, const PairArgs& a, const Group* g, int grid, int block, size_t smem, cudaStream_t st) {
        launch_one<R, K, FT_GENERIC>(a, g, grid, block, smem, st);
    }
    static int attr(size_t smem) { return attr_one<R, K, FT_GENERIC>(smem); }
};

template <typename R>
size_t smem_bytes(int k, int block, int tile_cap) {
    typedef typename Vec4<R>::T R4;
    const size_t ws = k == 2 ? warp_bytes<R, 2>() : warp_bytes<R, 4>();
    return 2 * (size_t)tile_cap * sizeof(R4) + (size_t)(block / 32) * ws;
}

template <typename R>
int launch_r(int k, int ft, const PairArgs& a, const Group* g, int grid, int block, size_t smem, cudaStream_t st) {
    switch (k) {
        case 2: Dispatch<R, 2, N_FT_SETS - 1>::run(ft, a, g, grid, block, smem, st); break;
        case 4: Dispatch<R, 4, N_FT_SETS - 1>::run(ft, a, g, grid, block, smem, st); break;
        default: return MFA_ERR_ARGS;
    }
    return MFA_OK;
}

template <typename R>
int attr_r(int k, size_t smem) {
    switch (k) {
        case 2: return Dispatch<R, 2, N_FT_SETS - 1>::attr(smem);
        case 4: return Dispatch<R, 4, N_FT_SETS - 1>::attr(smem);
    }
    return MFA_ERR_ARGS;
}

constexpr size_t SMEM_LIMIT = 200 * 1024;   // dynamic shared memory per CTA

}  // namespace

// Largest tile the pair kernel may stage, in records, next to the work space
// of the largest launch shape.
int pair_tile_limit(const mfa_ctx* c) {
    const size_t rec = c->prec == MFA_MIXED ? sizeof(float4) : sizeof(double4);
    const size_t ws = c->prec == MFA_MIXED ? smem_bytes<float>(4, 256, 0) : smem_bytes<double>(4, 256, 0);
    return (int)((SMEM_LIMIT - ws) / (2 * rec));
}

int pair_set_shape(mfa_ctx* c, int k, int block, int tile_cap) {
    if (k != 2 && k != 4) return MFA_ERR_ARGS;
    if (block < 32 || block > 256 || block % 32) return MFA_ERR_ARGS;
    if (tile_cap < 0) tile_cap = 0;
    if (tile_cap > pair_tile_limit(c)) tile_cap = pair_tile_limit(c);
    // every instantiation admits the largest dynamic shared memory any shape
    // uses (the attribute is per function, shared by all contexts and batches)
    static bool admitted[2][5];
    bool& done = admitted[c->prec == MFA_MIXED ? 0 : 1][k];
    if (!done) {
        const int rc = c->prec == MFA_MIXED ? attr_r<float>(k, SMEM_LIMIT) : attr_r<double>(k, SMEM_LIMIT);
        if (rc != MFA_OK) return rc;
        done = true;
    }
    c->pair_tpp = k;
    c->pair_block = block;
    c->tile_cap = tile_cap;
    return MFA_OK;
}

// The pair kernel's argument record, grid, dynamic shared memory and feature set
// for a context.
int pair_stage_args(mfa_ctx* c, int fuse_wall, void* out, int* grid_out, size_t* smem_out, int* ft_out) {
    if (!c->lists_valid) return MFA_ERR_STATE;
    PairArgs a;
    a.pos_s = c->pos_s; a.vel_s = c->vel_s; a.nbr = c->nbr; a.ccount = c->ccount; a.maxnb = c->maxnb;
    a.cell_start = c->cell_start; a.flags = c->dflags;
    a.mass = c->mass; a.tabs = c->tabs; a.force = c->force; a.dstep = c->dstep;
    a.partials = c->partials + (size_t)R_PAIR * 4 * c->max_blocks;
    a.counter = c->counters + R_PAIR;
    a.dscal = c->dscal;
    a.n = c->n;
    a.max_blocks = c->max_blocks;
    const mfa_params& p = c->p;
    for (int d = 0; d < 3; ++d) a.nb[d] = c->nb[d];
    a.rule = c->bin_type;
    a.wy = c->bin_type == 0 ? p.delta_bin[1] + 2 : 3;
    a.nseg = a.wy * (c->bin_type == 0 ? p.delta_bin[2] + 2 : 3);
    // untiled: capacity 0, blocks of consecutive slots read neighbours through the caches
    a.rowmode = c->pair_tiled;
    const int cap = c->pair_tiled ? c->tile_cap : 0;
    a.tile_cap = cap;
    // binning.f90 builds a half list (Newton 3); my_binning.f90 a full list
    a.half = c->bin_type == 0;
    a.lj_energy_factor = c->bin_type == 0 ? 1.0 : 0.5;
    a.symmetry = p.symmetry; a.thermostat = p.thermostat; a.dpd_weight = p.dpd_weight;
    a.noise = p.noise; a.charged = p.charged;
    a.real_in_lj = (p.quirks & MFA_Q_EWALD_REAL_IN_LJ) != 0;
    a.fsw = p.force_switch_on;
    a.wall_type = p.wall; a.wall_e_aw = (p.quirks & MFA_Q_WALL_ENERGY_AW) != 0;
    a.fuse_wall = fuse_wall && p.wall == 2;
    for (int d = 0; d < 3; ++d) { a.L[d] = p.boundary[d]; a.invL[d] = c->inv_boundary[d]; }
    a.sig = p.sig; a.friction = p.friction; a.dt = p.dt;
    a.elog_every = c->elog ? c->elog_every : 0;
    a.r_2_min_init = p.r_2_min_init; a.r_2_min_time = p.r_2_min_time; a.s_time = p.s_time;
    a.sqrt_alpha = p.sqrt_alpha; a.alpha_c = p.alpha_c; a.inv_sqrt_pi = p.inv_sqrt_pi;
    a.ewald_rc_2 = p.ewald_rc_2;
    for (int d = 0; d < 3; ++d) { a.fL[d] = (float)a.L[d]; a.fiL[d] = (float)a.invL[d]; }
    a.fsig = (float)a.sig; a.fgam = (float)a.friction; a.fewrc2 = (float)a.ewald_rc_2;
    a.fsqrt_alpha = (float)a.sqrt_alpha; a.falpha_c = (float)a.alpha_c; a.finv_sqrt_pi = (float)a.inv_sqrt_pi;
    for (int k = 0; k < T8; ++k) { a.a_wall[k] = p.a_wall[k]; a.sigma_wall[k] = p.sigma_wall[k]; }
    a.a_w = p.a_w; a.z_space_wall = p.z_space_wall; a.wall_cut = p.wall_cut;
    a.seed0 = (uint32_t)p.seed; a.seed1 = (uint32_t)(p.seed >> 32);
    a.key = philox_round_keys(a.seed0, a.seed1);
    // untiled: one warp per piece (a chunk's entries cut into `split` pieces),
    // at most max_blocks CTAs (the warps then take several pieces each)
    a.split = c->pair_tiled ? 1 : c->pair_split;
    a.zero_slots = 0;
    a.defer_sum = 0;
    const long long npiece = (long long)((c->n + 31) / 32) * a.split;
    const int nwarp = c->pair_block / 32;
    int grid = c->pair_tiled ? c->nb[1] * c->nb[2] : (int)((npiece + nwarp - 1) / nwarp);
    if (!c->pair_tiled && grid > c->max_blocks) grid = c->max_blocks;
    a.qctr = nullptr;
    a.qmod = 0;
    if (!c->pair_tiled && c->pair_queue > 0 && c->pair_qctr) {
        // a fixed grid of pair_queue CTAs per SM (at most the static grid)
        // fetching pieces from the queue
        const int g2 = c->pair_queue * c->n_sm;
        if (g2 < grid) grid = g2;
        a.qctr = c->pair_qctr;
        a.qmod = (int)npiece + grid * nwarp;
    }
    if (grid > c->max_blocks) return MFA_ERR_ARGS;
    const size_t smem = c->prec == MFA_MIXED ? smem_bytes<float>(c->pair_tpp, c->pair_block, cap)
                                             : smem_bytes<double>(c->pair_tpp, c->pair_block, cap);
    int ft = 0;
    if (p.thermostat == MFA_THERMO_DPD) ft |= FT_DPD;
    if (p.thermostat == MFA_THERMO_LGV) ft |= FT_LGV;
    if (p.charged) ft |= a.real_in_lj ? FT_QLJ : FT_QSEP;
    if (p.force_switch_on) ft |= FT_FSW;
    if (a.fuse_wall) ft |= FT_WALL;
    memcpy(out, &a, sizeof(a));
    *grid_out = grid;
    *smem_out = smem;
    *ft_out = ft;
    return MFA_OK;
}

size_t pair_args_bytes() { return sizeof(PairArgs); }

int launch_pair_grouped(int prec, int k, int block, int ft, const void* dargs, const int* doff, int nsys, int grid,
                        size_t smem, cudaStream_t st) {
    Group g{(const PairArgs*)dargs, doff, nsys};
    PairArgs dummy;
    const int rc = prec == MFA_MIXED ? launch_r<float>(k, ft, dummy, &g, grid, block, smem, st)
                                     : launch_r<double>(k, ft, dummy, &g, grid, block, smem, st);
    if (rc != MFA_OK) return rc;
    MFA_CUDA_TRY(cudaGetLastError());
    return MFA_OK;
}

int launch_pair(mfa_ctx* c, int fuse_wall, int zero_slots, int defer_sum) {
    PairArgs a;
    int grid, ft;
    size_t smem;
    TRY_(pair_stage_args(c, fuse_wall, &a, &grid, &smem, &ft));
    a.zero_slots = zero_slots;
    a.defer_sum = defer_sum;
    // the integrator launch that follows adds up the block partials
    c->pair_sum_nblk = defer_sum ? grid : 0;
    c->pair_sum_nq = (ft & FT_WALL) ? 4 : 3;
    const int rc = c->prec == MFA_MIXED ? launch_r<float>(c->pair_tpp, ft, a, nullptr, grid, c->pair_block, smem, c->st)
                                        : launch_r<double>(c->pair_tpp, ft, a, nullptr, grid, c->pair_block, smem, c->st);
    if (rc != MFA_OK) return rc;
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}
