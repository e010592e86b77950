// Internal declarations of the B200 implementation of mfa's per-step loop.
// Device data layout (all resident in HBM for the life of a context):
//   FP64 SoA state in particle order: r (x,y,z), v, a, mic_count, r0_old, mic_old
//   force:   one 4-wide record per particle (float4 in MIXED, double4 in FP64)
//   pos_s:   cell-sorted copy of positions, w = (id << 8 | type)   (float4 / double4)
//   vel_s:   cell-sorted copy of velocities, w = charge             (float4 / double4)
//   ids:     slot -> particle, slot: particle -> slot (counting sort by cell)
//   nbr:     Verlet list in slot space (half list for binning, full for
//            my_binning): per chunk of 32 consecutive slots one run of entries
//            (partner slot << 5 | owner lane), ccount[chunk] long
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/mfa_gpu.h"

#define T8 MFA_MAX_TYPES

// scalar slots in ctx->dscal (device FP64)
enum {
    S_VFF = 0,      // LJ energy
    S_VIR = 1,      // pair virial
    S_VCR = 2,      // Coulomb real-space energy (without self term)
    S_VFW = 3,      // wall energy
    S_VINTRA = 4,   // FENE energy (already multiplied by k)
    S_VBEND = 5,
    S_TKIN = 6,     // 0.5 sum m v^2
    S_VCK = 7,      // Coulomb k-space energy
    S_VTOT = 8,
    S_ETOT = 9,
    S_VCOUL = 10,   // real + self + k
    S_VDIP = 11,    // slab dipolar correction energy (SYMMETRY 0, charged)
    S_TMP0 = 12,    // 12..15: staging for kernels that publish a subset of slots
    S_NSLOT = 16
};

// int flags in ctx->dflags
enum {
    F_ERR = 0,       // error bits (1 << mfa_status)
    F_SKIN = 1,      // rebuild due
    F_MAXNB = 2,     // largest list row at the last rebuild
    F_MAXCELL = 3,   // largest cell at the last rebuild
    F_NEEDNB = 4,    // list capacity that would have been needed
    F_REBUILDS = 5,  // rebuild counter
    F_FENE = 6,      // FENE bonds at the clamp since init
    F_MAXROW = 7,    // largest cell row (fixed y, z) at the last rebuild
    F_MAXTILE = 8,   // largest neighbourhood of a row (records) at the last rebuild
    F_CONDREB = 9,   // rebuilds run inside conditional graph nodes (launch accounting)
    F_NFLAG = 16
};

// reduction counters (last-block-done pattern), one per reducing kernel
// reduction counters (and partial-sum regions)
enum { R_PAIR = 0, R_BOND = 1, R_WALL = 2, R_VV = 3, R_EWALD = 4, R_OBS = 5, R_BIN = 7, R_N = 8 };
// the cooperative rebuild's grid barrier: a generation word, a root count and
// GB_SUB group counts, each on its own 128-byte line
constexpr int GB_SUB = 16;
constexpr int GB_WORDS = (GB_SUB + 2) * 32;
// whole-run graphs kept per context (distinct step counts of mfa_step calls)
constexpr int N_CALL_GRAPHS = 4;

struct mfa_ctx {
    mfa_params p;
    int prec;            // MFA_FP64 / MFA_MIXED
    int dev;
    cudaStream_t st;
    cudaStream_t st_body;               // captures the bodies of conditional graph nodes
    int n;
    // FP64 state
    double *rx, *ry, *rz, *vx, *vy, *vz, *ax, *ay, *az;
    double *ox, *oy, *oz;               // r0_old + mic_old * L (the skin check's snapshot)
    int32_t *mx, *my, *mz;
    int32_t* type;
    double *mass, *inv_mass, *q;
    // every particle has the same mass (then the integrator takes it from its
    // arguments instead of streaming two arrays): its value and inverse
    int uniform_mass;
    double umass, uinv_mass;
    void* force;                        // float4 / double4 [n]
    void* pos_s;                        // float4 / double4 [n]
    void* vel_s;                        // float4 / double4 [n]
    double4* pos64;                     // FP64 sorted positions for the list builder (scratch)
    float4* pos32;                      // FP32 copy of pos64 (the builder's prefilter)
    int32_t *ids, *slot;
    // cells
    int nb[3], ncell;
    double rbin[3], inv_rbin[3], inv_boundary[3];
    int32_t *cell_count, *cell_start, *cell_cursor, *cell_of, *row_count;
    // pair kernel launch shape (threads per particle, block size) and the
    // shared-memory capacity of its staged tile, in records
    int pair_tpp, pair_block, tile_cap, pair_tiled;
    // pair tables on the device: range_2+skin_2, range_2, epsil, sigma_2, e_shift, inv_range_2
    double* tabs;                       // 6 x T8*T8
    // Verlet list
    int maxnb;                          // list capacity per slot (a chunk holds 32 x maxnb)
    int32_t *nbr, *nnb;
    int32_t* ccount;                    // entries per 32-slot chunk (after nnb)
    // reductions / flags
    double* partials;                   // R_N regions x max_blocks x 4 quantities
    int max_blocks;
    unsigned* counters;                 // R_N
    double* dscal;                      // S_NSLOT, followed by the flags in the same allocation
    int32_t* dflags;                    // F_NFLAG (= dscal + S_NSLOT: one copy reads both)
    int64_t* dstep;                     // [0] device copy of i_time; [1] the step whose energies
                                        // are wanted (-1: every step)
    // Ewald
    int nk;
    double4* kvec;                      // (kx, ky, kz, inv_k2*exp(-k2/(4 alpha_c)))
    double2* rho;                       // nk
    double2* rho_part;                  // nblk_rho x nk
    int nblk_rho;
    void* kruns;                        // runs of the k-vectors (int4: n_x, n_y, n_z, first k), nrun + 1
    int nrun;
    int ew_rho_rows, ew_force_warps;    // launch shapes of the k-space passes (ewald_setup; rows 0: k_rho_partial)
    int* qidx;                          // ids of the charged particles (k-space sums skip the rest)
    int nq;
    int kmax[3];
    double inv_V, v_coul_self;
    // host-side bookkeeping
    int64_t i_time;
    int bin_type;                       // 0 after binning, 1 after my_binning
    int lists_valid;
    int n_rebuilds_host;
    // fast path: captured graphs (0: one fused body step, 1: GRAPH_BODY fused
    // body steps, 2..: whole runs of call_n[k - 2] steps) and the number of
    // kernels in each
    cudaGraphExec_t gexec[2 + N_CALL_GRAPHS];
    cudaGraph_t graph[2 + N_CALL_GRAPHS];
    int graph_kernels[2 + N_CALL_GRAPHS];
    int call_n[N_CALL_GRAPHS];
    long long call_used[N_CALL_GRAPHS];   // last use, for replacement
    long long call_clock;
    int last_call_n;                      // steps of the previous mfa_step call
    const void* graph_key[4];           // what the captured arguments depend on
    unsigned long long graph_gen;       // advanced whenever the captured graphs are dropped
    void* adj_cache;                    // mfa_adjoint's workspace and captured sequences (adjoint.cu)
    int cond_rebuild;                   // rebuilds in conditional graph nodes (1) or early-exit kernels (0)
    int coop_rebuild;                   // captured steps rebuild in one cooperative kernel (1) or as above (0)
    int pair_sum_nblk, pair_sum_nq;     // block partials of the last pair launch left to the next integrator launch
    int coop_grid;                      // its grid (co-resident CTAs)
    unsigned* grid_bar;                 // its barrier words (GB_WORDS, zeroed)
    unsigned long long* coop_stage_ns;  // its stage times under MFA_DEBUG=1, else null
    // kernel launch accounting
    long long launches;
    long long cap_count;
    int capturing;
    // energy log
    double* elog;
    int elog_every, elog_cap;
    int32_t* elog_n;
    // device staging for uploads/downloads (3 x n doubles): the host's r0(3,n)
    // layout is copied as it is and (de)interleaved on the device
    double* d_stage;
    double* h_scal;                     // pinned copy of dscal and dflags (mfa_get_scalars)
    // pair-kernel work queue: CTAs per SM (0: one CTA per block of slots) and
    // its 64-bit ticket counter; n_sm = multiprocessors of the device;
    // pair_split = pieces each 32-slot chunk's list is cut into (untiled)
    int pair_queue, n_sm, pair_split;
    unsigned long long* pair_qctr;
    // observables (observe.cu), allocated at their first use: unfolded
    // coordinates (3 n) and 16 result slots; the z histogram and its count
    double* obs_buf;
    // the force on each grafted head before the pin zeroes it
    // (verlet_velocities.f90:18, f_on_heads), 3 x n_chain chain-major; null
    // unless the heads are pinned
    double* f_heads;
    double* hist;
    int hist_dim, hist_obs;
    // optional terms (terms.cu): DPD_VV switch and its two 3 x n FP64
    // dissipative-force buffers (previous, current), and a small result buffer
    int dpd_vv;
    double* fd;
    double* term_buf;
};

#define TRY_(x)                          \
    do {                                 \
        int s__ = (x);                   \
        if (s__ != MFA_OK) return s__;   \
    } while (0)

// stages of the integrator kernels
enum { VV_POSITIONS = 0, VV_VELOCITIES = 1, VV_FUSED = 2 };

// ---------- launchers (each file) ----------
// integrate.cu
// energy_span > 0: the first position half of a run of that many steps
int launch_vv_positions(mfa_ctx* c, int fused_skin, int zero_force, long long energy_span = 0);
int launch_check_skin(mfa_ctx* c);
// energy_reset: the last velocity half of a run of steps
int launch_vv_velocities(mfa_ctx* c, int fuse_bonds, int energy_reset = 0);
// the one-thread kernel that opens a conditional rebuild node after a position half
int launch_open_rebuild(mfa_ctx* c, cudaGraphConditionalHandle h);
int launch_vv_fused(mfa_ctx* c, cudaGraphConditionalHandle rebuild_cond, int fuse_bonds);
// argument record of an integrator stage (for grouped launches) and the launch
size_t vv_args_bytes();
int vv_stage_args(mfa_ctx* c, int stage, int fused_skin, int zero_force, int fuse_bonds,
                  cudaGraphConditionalHandle rebuild_cond, void* out, int* nblocks);
// energy_span / energy_reset: the first position half / last velocity half of
// a run of steps (as launch_vv_positions / launch_vv_velocities)
int launch_vv_grouped(int prec, int stage, const void* dargs, const int* doff, int nsys, int nblocks,
                      cudaStream_t st, long long energy_span = 0, int energy_reset = 0);
// binning.cu
int launch_rebuild(mfa_ctx* c, int rule, int conditional);
int launch_rebuild_on(mfa_ctx* c, int rule, int conditional, cudaStream_t st, int in_cond_body);
// the six rebuild stages as grouped launches
constexpr int N_BIN_STAGES = 6;
size_t bin_args_bytes();
int bin_stage_args(mfa_ctx* c, int rule, int conditional, int in_cond_body, void* out, int nblocks[N_BIN_STAGES]);
int launch_bin_grouped(int prec, int stage, const void* dargs, const int* doff, int nsys, int nblocks,
                       cudaStream_t st, int* node_count);
int launch_refresh_sorted(mfa_ctx* c);
int launch_rebuild_coop(mfa_ctx* c, int rule);
void adj_cache_free(mfa_ctx* c);
int rebuild_coop_setup(mfa_ctx* c);
void rebuild_coop_report(mfa_ctx* c);
// pair.cu
// adds to force; zero_slots: energy slots the kernel resets (1: S_VCK and
// S_VDIP, 2: S_VFW), for the subroutine entry points
// defer_sum: the energies' grid-wide sum is left to the integrator launch
// that follows (launch_vv_fused / launch_vv_velocities), off the pair kernel's tail
int launch_pair(mfa_ctx* c, int fuse_wall, int zero_slots = 0, int defer_sum = 0);
size_t pair_args_bytes();
int pair_stage_args(mfa_ctx* c, int fuse_wall, void* out, int* grid_out, size_t* smem_out, int* ft_out);
int launch_pair_grouped(int prec, int k, int block, int ft, const void* dargs, const int* doff, int nsys, int grid,
                        size_t smem, cudaStream_t st);
int pair_set_shape(mfa_ctx* c, int tpp, int block, int tile_cap);
int pair_set_queue(mfa_ctx* c, int ctas_per_sm);
int pair_tile_limit(const mfa_ctx* c);
// bonds.cu
int launch_bonds(mfa_ctx* c, int do_fene, int do_bend);
int bonds_setup(mfa_ctx* c);
// wall.cu
int launch_wall(mfa_ctx* c, int inter_type);
// ewald.cu
int ewald_setup(mfa_ctx* c);
int launch_ewald(mfa_ctx* c);
// dipolar_correction.f90 (charged SYMMETRY 0; nothing otherwise)
int launch_dipolar(mfa_ctx* c);
// adjoint of the k-space force and of the slab correction: out += (dF/dr)^T lam
// (lam, out: 3 x n, particle order); scratch of ewald_adj_bytes(c) bytes
size_t ewald_adj_bytes(const mfa_ctx* c);
int ewald_adjoint_prepare(mfa_ctx* c);
int launch_ewald_adjoint(mfa_ctx* c, const double* lam, double* out, void* scratch);
// terms.cu: the velocity half of verlet_velocities under DPD_VV
int launch_dpd_vv_kick(mfa_ctx* c);

// every kernel launch is recorded (graph captures count towards their graph)
inline void note_launch(mfa_ctx* c, int k) {
    if (c->capturing) c->cap_count += k;
    else c->launches += k;
}

#define MFA_CUDA_TRY(x)                                   \
    do {                                                  \
        cudaError_t e__ = (x);                            \
        if (e__ != cudaSuccess) return MFA_ERR_CUDA;      \
    } while (0)

// ---------- device helpers ----------
__device__ __forceinline__ double mimage64(double d, double L, double invL) {
    // d - L*int(2d/L) with int() truncating toward zero (fluid_fluid.f90:84-88);
    // explicit round-to-nearest ops so that no multiply-add is fused.
    double t = __dmul_rn(__dmul_rn(2.0, d), invL);
    return __dsub_rn(d, __dmul_rn(L, (double)(int)t));
}
__device__ __forceinline__ float mimage32(float d, float L, float invL) {
    float t = 2.0f * d * invL;
    return d - L * (float)(int)t;
}

__device__ __forceinline__ void set_err(int32_t* flags, int status) {
    atomicOr(&flags[F_ERR], 1 << status);
}

// Whether the kernels of the current step accumulate energies: always for the
// subroutine entry points (dstep[1] = -1), else for the last step of an
// mfa_step run (dstep[1]) and the steps the energy log records.
__device__ __forceinline__ bool energy_needed(const int64_t* dstep, int elog_every) {
    const long long st = dstep[0], want = dstep[1];
    return want < 0 || st == want || (elog_every > 0 && st % elog_every == 0);
}

// Philox-4x32-10 (Salmon et al., SC'11), counter (c0..c3), key (k0, k1).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        uint4 o;
        o.x = hi1 ^ c.y ^ k0;
        o.y = lo1;
        o.z = hi0 ^ c.w ^ k1;
        o.w = lo0;
        c = o;
        k0 += W0;
        k1 += W1;
    }
    return c;
}
// The same generator with the key schedule (k0 + r W0, k1 + r W1), r = 0..9,
// precomputed on the host and passed in the kernel parameters, so that the
// round keys are constant-bank operands instead of per-round additions.
struct PhiloxKeys {
    uint32_t k[20];
};
inline PhiloxKeys philox_round_keys(uint32_t k0, uint32_t k1) {
    PhiloxKeys r;
    for (int i = 0; i < 10; ++i) {
        r.k[2 * i] = k0 + (uint32_t)i * 0x9E3779B9u;
        r.k[2 * i + 1] = k1 + (uint32_t)i * 0xBB67AE85u;
    }
    return r;
}
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, const PhiloxKeys& key) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)M0 * c.x, p1 = (uint64_t)M1 * c.z;
        uint4 o;
        o.x = (uint32_t)(p1 >> 32) ^ c.y ^ key.k[2 * r];
        o.y = (uint32_t)p1;
        o.z = (uint32_t)(p0 >> 32) ^ c.w ^ key.k[2 * r + 1];
        o.w = (uint32_t)p0;
        c = o;
    }
    return c;
}
#define TAG_DPD 0x44504400u
#define TAG_LGV 0x4C475600u

// The three Langevin variates of particle `id` at `step` (lgv_forces.f90:25-27:
// three rnor() per particle): one Philox-4x32-10 block keyed by (id, step),
// Box-Muller on its four words (FP64 log/sincos), or the uniform alternative
// sqrt(3)(2u - 1).  Shared by the pair kernel and its adjoint, which replays it.
template <typename R>
__device__ __forceinline__ void lgv_noise3(uint32_t id, uint32_t step, int noise, uint32_t seed0, uint32_t seed1,
                                           R g[3]) {
    const uint4 w = philox4x32_10(make_uint4(id, 0u, step, TAG_LGV), seed0, seed1);
    if (noise == MFA_NOISE_UNIFORM) {
        const uint32_t x[3] = {w.x, w.y, w.z};
        for (int d = 0; d < 3; ++d) {
            const float u = (float)(x[d] >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f;
            g[d] = (R)(1.7320508075688772f * (2.0f * u - 1.0f));
        }
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

// Position of a block in the launch it belongs to.  A plain launch uses
// blockIdx/gridDim; a grouped launch (one kernel stage for several contexts,
// see group_of) gives each block its index within its own context's share.
struct Blk {
    int id, n;
};
__device__ __forceinline__ Blk plain_blk() { return Blk{(int)blockIdx.x, (int)gridDim.x}; }

// Grouped launch: off[0..nsys] are prefix sums of the contexts' block counts;
// returns the context of block b.
__device__ __forceinline__ int group_of(const int* __restrict__ off, int nsys, int b) {
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&off[mid]) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ Blk group_blk(const int* __restrict__ off, int s) {
    const int o = __ldg(&off[s]);
    return Blk{(int)blockIdx.x - o, __ldg(&off[s + 1]) - o};
}

// Block-wide FP64 sums of NQ values: the block's partials into
// partials[q * max_blocks + blk.id].  Requires blockDim.x a multiple of 32,
// <= 1024.
template <int NQ>
__device__ __forceinline__ void block_partials(double (&v)[NQ], double* partials, int max_blocks, Blk blk) {
    __shared__ double sm[NQ][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sm[q][wid] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double x = lane < nw ? sm[q][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) partials[q * max_blocks + blk.id] = x;
        }
    }
}

// The sums of the nblk partials of each of NQ quantities, added in a fixed
// order (deterministic) by the whole block and stored in out[0..NQ).  Every
// thread of the block calls it.
template <int NQ>
__device__ __forceinline__ void reduce_partials(const double* partials, int max_blocks, int nblk, double* out) {
    __shared__ double sm[NQ][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // every thread sums a fixed stripe of blocks; the loads of U blocks x NQ
    // quantities are issued before any of them is used, so the block waits for
    // ~n/(U blockDim) L2 round trips, not n/blockDim
    double xs[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) xs[q] = 0.0;
    constexpr int U = NQ <= 2 ? 8 : 4;
    for (int b0 = threadIdx.x; b0 < nblk; b0 += U * blockDim.x) {
        double v[U][NQ];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int b = b0 + u * blockDim.x;
#pragma unroll
            for (int q = 0; q < NQ; ++q) v[u][q] = b < nblk ? __ldcg(&partials[q * max_blocks + b]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < NQ; ++q) xs[q] += v[u][q];
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double x = xs[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        __syncthreads();
        if (lane == 0) sm[q][wid] = x;
        __syncthreads();
        if (wid == 0) {
            double y = lane < nw ? sm[q][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) y += __shfl_down_sync(0xffffffffu, y, o);
            if (lane == 0) out[q] = y;
        }
    }
}

// Block-wide FP64 sums of NQ values, committed deterministically: each block
// writes its partials, the last block to finish adds them in block order and
// stores the result in out[0..NQ) (true in that block).
template <int NQ>
__device__ __forceinline__ bool block_sum_commit(double (&v)[NQ], double* partials, int max_blocks,
                                                 unsigned* counter, double* out, Blk blk = plain_blk()) {
    __shared__ bool am_last;
    block_partials<NQ>(v, partials, max_blocks, blk);
    __threadfence();
    if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == (unsigned)blk.n - 1);
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    reduce_partials<NQ>(partials, max_blocks, blk.n, out);
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// Arrival of a block that has no sums to commit: true in the last block to
// arrive (which resets the counter); the writes of every block before its
// arrival are visible to that block.
__device__ __forceinline__ bool block_arrive_last(unsigned* counter, Blk blk) {
    __shared__ bool arrive_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) arrive_last = (atomicAdd(counter, 1u) == (unsigned)blk.n - 1);
    __syncthreads();
    if (!arrive_last) return false;
    __threadfence();
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// One 9-3 wall term (fluid_wall.f90:96-101) at inverse distance 1/zz:
// energy |A| (s/z)^9 - A_e (s/z)^3 and the force along the wall normal
// 9|A| s^9 / z^10 - 3 A s^3 / z^4; with cut > 0 the energy is shifted to zero at
// z = cut.  Shared by the stand-alone wall pass and the pair-kernel epilogue so
// that both round identically.
template <typename R>
__device__ __forceinline__ void wall93_term(R zz, R sw, R aw, R ae, R cut, R& f, double& e) {
    const R faw = aw < (R)0 ? -aw : aw;
    const R iz = (R)1 / zz;
    const R rd = sw * iz;
    const R rd2 = rd * rd, rd4 = rd2 * rd2, rd8 = rd4 * rd4;
    const R sw2 = sw * sw, sw4 = sw2 * sw2, sw8 = sw4 * sw4;
    const R iz2 = iz * iz, iz4 = iz2 * iz2, iz8 = iz4 * iz4;
    e = (double)(faw * (rd8 * rd) - ae * (rd2 * rd));
    f = (R)9 * faw * (sw8 * sw) * (iz8 * iz2) - (R)3 * aw * (sw2 * sw) * iz4;
    if (cut > (R)0) {
        const R rc = sw / cut, rc3 = rc * rc * rc;
        e -= (double)(faw * rc3 * rc3 * rc3 - ae * rc3);
    }
}

// Row (ky, kz) of neighbour-row index (iy, iz) around the row (cy, cz):
// binning.f90:73-76 for rule 0 (j = c-1 .. c+delta_bin, mod n), my_binning.f90:74-80
// for rule 1 (c-1 .. c+1 with a single wrap).  The pair kernel stages the rows
// in this order and the list builder encodes entries with the same index.
__host__ __device__ __forceinline__ int wrap_near(int k, int n) {
    // k in [-n, 2n): the periodic index without a division (the stencil offsets
    // are -1..+1, so (c - 1 + i + n) % n of binning.f90 never needs more)
    return k < 0 ? k + n : (k >= n ? k - n : k);
}
__host__ __device__ __forceinline__ void neighbour_row(int rule, int cy, int cz, int iy, int iz, int ny, int nz,
                                                       int& ky, int& kz) {
    if (rule == 0) {
        ky = wrap_near(cy - 1 + iy, ny);
        kz = wrap_near(cz - 1 + iz, nz);
    } else {
        ky = cy + iy - 1;
        if (ky < 0) ky = ny - 1;
        if (ky == ny) ky = 0;
        kz = cz + iz - 1;
        if (kz < 0) kz = nz - 1;
        if (kz == nz) kz = 0;
    }
}

// read-only-path loads of 4-wide records
__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ldg4(const double4* p) {
    const double2* q = (const double2*)p;
    const double2 a = __ldg(q), b = __ldg(q + 1);
    double4 r;
    r.x = a.x; r.y = a.y; r.z = b.x; r.w = b.y;
    return r;
}

// The w lane of the sorted position record carries (particle id << 8 | type)
// as raw bits; no arithmetic is ever done on it.
__device__ __forceinline__ void packw(float4& p, int id, int t) { p.w = __int_as_float((id << 8) | t); }
__device__ __forceinline__ void packw(double4& p, int id, int t) {
    p.w = __longlong_as_double((long long)((id << 8) | t));
}
__device__ __forceinline__ int wbits(float w) { return __float_as_int(w); }
__device__ __forceinline__ int wbits(double w) { return (int)__double_as_longlong(w); }
