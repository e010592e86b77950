// Ewald k-space (ewald_k.f90), FP64 throughout.
//
// mode 0 (host): the half-space set of k-vectors with |k| <= k_c, enumerated
//   exactly as ewald_k.f90:47-124 does (same FP64 expressions, same int()
//   truncations, so the same vectors are kept at the boundary of the sphere).
// mode 1 (device), over "runs": the k-vectors are enumerated x fastest
// (ewald_k.f90:104-124), so those with the same (n_y, n_z) form runs of
// consecutive n_x, and along a run exp(i k.r) advances by one complex product
// with exp(i dk_x x).  Per particle, exp(i n dk_d r_d) for n = 0..kmax_d per
// axis comes from one sincos and a complex power recurrence (tables in shared
// memory, laid out so the 32 lanes of a warp read 32 particles' entries).
//   k_rho_runs     - structure factors rho(k) = sum_i q_i exp(i k.r_i): a
//                    lane holds RG particles, a warp walks runs, and per k
//                    the warp sums its lanes' q exp(i k.r) with a fixed
//                    shuffle tree (deterministic); partials per block row.
//   k_rho_reduce   - a warp per k sums the block partials (each lane a fixed
//                    stride of blocks, then a fixed shuffle tree: deterministic)
//                    and the energy 4 pi / V sum_k inv_k2 exp(-k2/4a) |rho|^2.
//   k_force_runs   - a lane per particle, the warps of a block over runs (the
//                    k data of a run read by the whole warp at once), then the
//                    warps' partial forces summed in a fixed order:
//                    F_i = -8 pi q_i / V sum_k k inv_k2 exp(..) (cos Im - sin Re).
// Per (particle, k) both passes take one complex product (the run step) and
// three to five FP64 multiply-adds.
// Both k-space passes visit the charged particles only (a list made once by
// ewald_k(0)): the others contribute nothing to rho and feel no k-space force.
// Slab correction (dipolar_correction.f90, SYMMETRY 0):
//   k_dipole_moment - M_z = sum_i q_i (z_i - Lz/2), a deterministic grid
//                     reduction, and the energy 2 pi M_z^2 / V;
//   k_dipole_force  - F_z,i -= 4 pi q_i M_z / V.
#include "mfa_internal.cuh"

#include <math.h>
#include <vector>

namespace {

constexpr int KM = 64;        // largest |n| per axis held in the tables
constexpr int RHO_T = 512;    // threads per block in k_rho_partial
constexpr int KPT = 8;        // k per thread: a block row covers KPT * RHO_T vectors
constexpr int NK_MAX = 1 << 16;   // k-vectors of one context
constexpr int CH = 32;        // particles per table batch
constexpr int FT = 64;        // threads per block in k_ewald_adj

struct EwArgs {
    const double *rx, *ry, *rz, *q;
    const int* qidx;          // the charged particles
    int nq;
    const double4* kvec;      // kx, ky, kz, inv_k2 * exp(-k2 fac_alpha)
    const int4* kn;           // nx, ny, nz
    double2* rho_part;
    double2* rho;
    double2* rhow;            // rho(k) * inv_k2 exp(-k2/4a) (the force pass's weight per k)
    void* force;
    double* partials;
    unsigned* counter;
    double* dscal;
    int max_blocks;
    int n, nk, nblk, per_blk;
    int kmax[3];
    int ts;                   // table stride: largest kmax + 1
    double dk[3];
    double pi, inv_V;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// tables t[d*ts + n] = exp(i n dk_d r_d), n = 0..kmax_d (ts = largest kmax + 1)
__device__ __forceinline__ void build_tables(double2* t, const EwArgs& a, double x, double y, double z) {
    const double r[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double s, c;
        sincos(a.dk[d] * r[d], &s, &c);
        const double2 e1 = make_double2(c, s);
        double2 e = make_double2(1.0, 0.0);
        t[d * a.ts] = e;
        for (int n = 1; n <= a.kmax[d]; ++n) {
            e = cmul(e, e1);
            t[d * a.ts + n] = e;
        }
    }
}

__device__ __forceinline__ double2 phase_from(const double2* t, int ts, int4 kn) {
    double2 ex = t[abs(kn.x)];
    if (kn.x < 0) ex.y = -ex.y;
    double2 ey = t[ts + abs(kn.y)];
    if (kn.y < 0) ey.y = -ey.y;
    const double2 ez = t[2 * ts + kn.z];
    return cmul(cmul(ex, ey), ez);
}

// Structure factors with a thread per k (the layout of the adjoint's
// k_sig_partial, which runs beside it): blockIdx.x: a range of particles;
// blockIdx.y: a row of KPT * RHO_T k-vectors.  Dynamic shared memory: CH
// tables of 3 * ts phases, then CH charges.
__global__ void __launch_bounds__(RHO_T) k_rho_partial(EwArgs a) {
    extern __shared__ double2 rtab[];
    double* sq = (double*)(rtab + CH * 3 * a.ts);
    const int p0 = blockIdx.x * a.per_blk, p1 = min(a.nq, p0 + a.per_blk);
    const int kb = blockIdx.y * KPT * RHO_T;
    double2 acc[KPT];
    int4 kn[KPT];
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        acc[j] = make_double2(0.0, 0.0);
        const int k = kb + threadIdx.x + j * RHO_T;
        kn[j] = k < a.nk ? a.kn[k] : make_int4(0, 0, 0, 0);
    }
    for (int b0 = p0; b0 < p1; b0 += CH) {
        const int nb = min(CH, p1 - b0);
        __syncthreads();
        if (threadIdx.x < nb) {
            const int i = a.qidx[b0 + threadIdx.x];
            build_tables(rtab + threadIdx.x * 3 * a.ts, a, a.rx[i], a.ry[i], a.rz[i]);
            sq[threadIdx.x] = a.q[i];
        }
        __syncthreads();
        for (int pp = 0; pp < nb; ++pp) {
            const double qi = sq[pp];
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                const double2 e = phase_from(rtab + pp * 3 * a.ts, a.ts, kn[j]);
                acc[j].x += qi * e.x;
                acc[j].y += qi * e.y;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        const int k = kb + threadIdx.x + j * RHO_T;
        if (k < a.nk) a.rho_part[(size_t)blockIdx.x * a.nk + k] = acc[j];
    }
}

// the partials of one k summed by a warp: lane l takes blocks l, l+32, ...,
// then a fixed shuffle tree (the same order every call)
__device__ __forceinline__ double2 warp_sum_partials(const double2* part, int nblk, int nk, int k, int lane) {
    double2 s = make_double2(0.0, 0.0);
    for (int b = lane; b < nblk; b += 32) {
        const double2 v = part[(size_t)b * nk + k];
        s.x += v.x;
        s.y += v.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_down_sync(0xffffffffu, s.x, o);
        s.y += __shfl_down_sync(0xffffffffu, s.y, o);
    }
    return s;
}

// warps over k with a grid stride (the grid is capped at the context's
// partial-sum slots); each warp's energy terms summed in its lane 0
__global__ void k_rho_reduce(EwArgs a) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double acc[1] = {0.0};
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < a.nk; k += nw) {
        const double2 s = warp_sum_partials(a.rho_part, a.nblk, a.nk, k, lane);
        if (lane == 0) {
            a.rho[k] = s;
            const double w = a.kvec[k].w;
            a.rhow[k] = make_double2(s.x * w, s.y * w);
            acc[0] += a.kvec[k].w * (s.x * s.x + s.y * s.y);   // ewald_k.f90:155-156
        }
    }
    if (block_sum_commit<1>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_TMP0 + 2) && threadIdx.x == 0)
        a.dscal[S_VCK] = ((a.dscal[S_TMP0 + 2] * 4.0) * a.pi) * a.inv_V;   // :159
}

// The run kernels take their warps per block from blockDim and k_rho_runs its
// run sets from gridDim.y; ewald_setup chooses both from the occupancy
// calculator so that the whole grid is resident at once (a second wave would
// double the time: every block walks all of its runs).
constexpr int RP = 32;        // particles per block (a lane each) in k_force_runs
constexpr int RWMAX = 16;     // most warps per block in k_force_runs
constexpr int RHW = 8;        // warps per block in k_rho_runs
constexpr int RG = 4;         // particles per lane in k_rho_runs
constexpr int RSEG = 8;       // longest run (longer ones are cut, for balance between warps)

// run r: (n_x of its first vector, n_y, n_z, index of its first vector); the
// entry nrun holds nk in .w, so a run's length is runs[r+1].w - runs[r].w
struct RunArgs {
    const int4* runs;
    int nrun;
};

// the per-axis tables of np particles (slots b0 ..), one (particle, axis) per
// thread: t[(d * ts + n) * np + p] = exp(i n dk_d r_d)
__device__ __forceinline__ void run_tables(double2* t, const EwArgs& a, int b0, int np) {
    for (int w = threadIdx.x; w < 3 * np; w += blockDim.x) {
        const int p = w % np, d = w / np;
        const int slot = b0 + p;
        double r = 0.0;
        if (slot < a.nq) {
            const int i = a.qidx[slot];
            r = d == 0 ? a.rx[i] : (d == 1 ? a.ry[i] : a.rz[i]);
        }
        double s, c;
        sincos(a.dk[d] * r, &s, &c);
        const double2 e1 = make_double2(c, s);
        double2 e = make_double2(1.0, 0.0);
        t[(d * a.ts) * np + p] = e;
        for (int n = 1; n <= a.kmax[d]; ++n) {
            e = cmul(e, e1);
            t[(d * a.ts + n) * np + p] = e;
        }
    }
}

// exp(i n dk_d r_d) for a signed n (conjugate for n < 0)
__device__ __forceinline__ double2 tab_at(const double2* t, int ts, int np, int d, int n, int p) {
    double2 e = t[(d * ts + abs(n)) * np + p];
    if (n < 0) e.y = -e.y;
    return e;
}

// Dynamic shared memory: RG * 32 particles' tables, then their charges.
// blockIdx.x: particles [blockIdx.x * 32 RG, +32 RG); blockIdx.y: runs
// blockIdx.y * RHW + warp, + RHW * gridDim.y, ...
__global__ void __launch_bounds__(RHW * 32) k_rho_runs(EwArgs a, RunArgs ra) {
    constexpr int NP = 32 * RG;
    extern __shared__ double2 rt[];
    double* sq = (double*)(rt + 3 * a.ts * NP);
    const int b0 = blockIdx.x * NP;
    run_tables(rt, a, b0, NP);
    for (int p = threadIdx.x; p < NP; p += blockDim.x)
        sq[p] = b0 + p < a.nq ? a.q[a.qidx[b0 + p]] : 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double qg[RG];
    double2 ex1[RG];
#pragma unroll
    for (int g = 0; g < RG; ++g) {
        qg[g] = sq[lane + 32 * g];
        ex1[g] = tab_at(rt, a.ts, NP, 0, 1, lane + 32 * g);
    }
    double2* part = a.rho_part + (size_t)blockIdx.x * a.nk;
    for (int r = blockIdx.y * RHW + warp; r < ra.nrun; r += RHW * gridDim.y) {
        const int4 run = __ldg(&ra.runs[r]);
        const int k1 = __ldg(&ra.runs[r + 1].w);
        double2 e[RG];
#pragma unroll
        for (int g = 0; g < RG; ++g) {
            const int p = lane + 32 * g;
            const double2 ezy = cmul(tab_at(rt, a.ts, NP, 2, run.z, p), tab_at(rt, a.ts, NP, 1, run.y, p));
            e[g] = cmul(ezy, tab_at(rt, a.ts, NP, 0, run.x, p));
        }
        for (int k = run.w; k < k1; ++k) {
            double vx = 0.0, vy = 0.0;
#pragma unroll
            for (int g = 0; g < RG; ++g) {
                vx += qg[g] * e[g].x;
                vy += qg[g] * e[g].y;
                e[g] = cmul(e[g], ex1[g]);
            }
            for (int o = 16; o > 0; o >>= 1) {
                vx += __shfl_down_sync(0xffffffffu, vx, o);
                vy += __shfl_down_sync(0xffffffffu, vy, o);
            }
            if (lane == 0) part[k] = make_double2(vx, vy);
        }
    }
}

// Dynamic shared memory: RP particles' tables, then (warps) x RP x 3 partial forces.
template <typename R4>
__global__ void __launch_bounds__(RWMAX * 32) k_force_runs(EwArgs a, RunArgs ra) {
    extern __shared__ double2 ft2[];
    double* red = (double*)(ft2 + 3 * a.ts * RP);
    const int b0 = blockIdx.x * RP;
    run_tables(ft2, a, b0, RP);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, RW = blockDim.x >> 5;
    const double2 ex1 = tab_at(ft2, a.ts, RP, 0, 1, lane);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int r = warp; r < ra.nrun; r += RW) {
        const int4 run = __ldg(&ra.runs[r]);
        const int k1 = __ldg(&ra.runs[r + 1].w);
        const double2 ezy = cmul(tab_at(ft2, a.ts, RP, 2, run.z, lane), tab_at(ft2, a.ts, RP, 1, run.y, lane));
        double2 e = cmul(ezy, tab_at(ft2, a.ts, RP, 0, run.x, lane));
        // along a run k_y and k_z are fixed and k_x = n_x dk_x (the product the
        // k-set is built with); one 16-byte load per k: rho(k) A_k
        double ssum = 0.0;
        for (int k = run.w; k < k1; ++k) {
            const double2 rw = __ldg(&a.rhow[k]);
            const double sc = e.x * rw.y - e.y * rw.x;   // (cos Im - sin Re) inv_k2 exp()
            fx += ((double)(run.x + (k - run.w)) * a.dk[0]) * sc;
            ssum += sc;
            e = cmul(e, ex1);
        }
        fy += ((double)run.y * a.dk[1]) * ssum;
        fz += ((double)run.z * a.dk[2]) * ssum;
    }
    red[(warp * RP + lane) * 3 + 0] = fx;
    red[(warp * RP + lane) * 3 + 1] = fy;
    red[(warp * RP + lane) * 3 + 2] = fz;
    __syncthreads();
    if (warp != 0) return;
    const int slot = b0 + lane;
    if (slot >= a.nq) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int w = 0; w < RW; ++w) {
        sx += red[(w * RP + lane) * 3 + 0];
        sy += red[(w * RP + lane) * 3 + 1];
        sz += red[(w * RP + lane) * 3 + 2];
    }
    const int i = a.qidx[slot];
    const double pre = ((-8.0 * a.pi) * a.q[i]) * a.inv_V;   // ewald_k.f90:194
    R4* f4 = (R4*)a.force;
    R4 o = f4[i];
    o.x += pre * sx;
    o.y += pre * sy;
    o.z += pre * sz;
    f4[i] = o;
}

int table_stride(const mfa_ctx* c) {
    int m = c->kmax[0];
    if (c->kmax[1] > m) m = c->kmax[1];
    if (c->kmax[2] > m) m = c->kmax[2];
    return m + 1;
}
size_t rho_smem(const mfa_ctx* c) { return (size_t)CH * (3 * table_stride(c) * sizeof(double2) + sizeof(double)); }
// blocks of 8 warps over the k-vectors, at most one per partial-sum slot
int reduce_grid(const mfa_ctx* c) {
    int g = (c->nk + 7) / 8;
    if (g > c->max_blocks) g = c->max_blocks;
    return g < 1 ? 1 : g;
}
size_t adj_smem(const mfa_ctx* c) { return (size_t)FT * 3 * table_stride(c) * sizeof(double2); }
size_t rho_runs_smem(const mfa_ctx* c) {
    return (size_t)32 * RG * (3 * table_stride(c) * sizeof(double2) + sizeof(double));
}
size_t force_runs_smem(const mfa_ctx* c, int warps) {
    return (size_t)RP * 3 * table_stride(c) * sizeof(double2) + (size_t)warps * RP * 3 * sizeof(double);
}
RunArgs run_args(const mfa_ctx* c) { return RunArgs{(const int4*)c->kruns, c->nrun}; }

EwArgs make_args(mfa_ctx* c) {
    EwArgs a;
    a.rx = c->rx; a.ry = c->ry; a.rz = c->rz; a.q = c->q;
    a.kvec = c->kvec; a.kn = (const int4*)(c->kvec + c->nk);
    a.rho_part = c->rho_part; a.rho = c->rho; a.rhow = c->rho + c->nk; a.force = c->force;
    a.qidx = c->qidx; a.nq = c->nq;
    a.partials = c->partials + (size_t)R_EWALD * 4 * c->max_blocks;
    a.counter = c->counters + R_EWALD;
    a.dscal = c->dscal;
    a.max_blocks = c->max_blocks;
    a.n = c->n; a.nk = c->nk; a.nblk = c->nblk_rho;
    a.per_blk = (c->nq + c->nblk_rho - 1) / c->nblk_rho;
    const mfa_params& p = c->p;
    for (int d = 0; d < 3; ++d) a.kmax[d] = c->kmax[d];
    a.ts = table_stride(c);
    a.pi = p.pi;
    a.inv_V = c->inv_V;
    // the k components are n * delta_k (ewald_k.f90:117); the tables use delta_k
    if (p.symmetry == 1) {
        for (int d = 0; d < 3; ++d) a.dk[d] = (2.0 * p.pi) * c->inv_boundary[d];
    } else {
        a.dk[0] = (2.0 * p.pi) * c->inv_boundary[0];
        a.dk[1] = (2.0 * p.pi) * c->inv_boundary[1];
        a.dk[2] = (2.0 * p.pi) / (p.boundary[2] + 2.0 * p.boundary[2]);
    }
    return a;
}

}  // namespace

int ewald_setup(mfa_ctx* c) {
    const mfa_params& p = c->p;
    if (!p.charged) return MFA_OK;
    double dk[3], z_slab;
    if (p.symmetry == 1) {
        for (int d = 0; d < 3; ++d) dk[d] = (2.0 * p.pi) * c->inv_boundary[d];
        z_slab = 0.0;
    } else {
        z_slab = 2.0;
        dk[0] = (2.0 * p.pi) * c->inv_boundary[0];
        dk[1] = (2.0 * p.pi) * c->inv_boundary[1];
        dk[2] = (2.0 * p.pi) / (p.boundary[2] + z_slab * p.boundary[2]);
    }
    volatile double kc_v = ((dk[0] + dk[1]) * (double)p.n_kmax) / 2.0;
    const double k_c = kc_v;
    const int nkx = (int)(k_c / dk[0]), nky = (int)(k_c / dk[1]), nkz = (int)(k_c / dk[2]);
    if (nkx > KM || nky > KM || nkz > KM) return MFA_ERR_UNSUPPORTED;
    const double kc2 = k_c * k_c;
    const double fac_alpha = 1.0 / (4.0 * p.alpha_c);
    std::vector<double4> kv;
    std::vector<int4> kn;
    for (int z = 0; z <= nkz; ++z)
        for (int y = -nky; y <= nky; ++y)
            for (int x = -nkx; x <= nkx; ++x) {
                volatile double a0 = (double)x * dk[0], a1 = (double)y * dk[1], a2 = (double)z * dk[2];
                volatile double s01 = a0 * a0 + a1 * a1;
                volatile double rk_2 = s01 + a2 * a2;
                if (rk_2 > kc2) continue;
                if (z == 0 && y == 0 && x == 0) continue;
                if (z == 0 && x + y < 0) continue;
                if (z == 0 && -x == y && y > 0) continue;
                const double k2 = rk_2;
                volatile double inv = 1.0 / k2;
                kv.push_back(make_double4(a0, a1, a2, inv * exp(-k2 * fac_alpha)));
                kn.push_back(make_int4(x, y, z, 0));
            }
    if (kv.size() > (size_t)NK_MAX) return MFA_ERR_UNSUPPORTED;
    c->nk = (int)kv.size();
    c->kmax[0] = nkx; c->kmax[1] = nky; c->kmax[2] = nkz;
    c->inv_V = (c->inv_boundary[0] * c->inv_boundary[1]) / (p.boundary[2] * (1.0 + z_slab));
    if (c->kvec) cudaFree(c->kvec);
    if (c->rho) cudaFree(c->rho);
    if (c->rho_part) cudaFree(c->rho_part);
    c->kvec = nullptr; c->rho = nullptr; c->rho_part = nullptr;
    // kvec block: nk double4 followed by nk int4
    MFA_CUDA_TRY(cudaMalloc(&c->kvec, (size_t)c->nk * (sizeof(double4) + sizeof(int4))));
    // on the context's (non-blocking) stream, so that the kernels see the table
    MFA_CUDA_TRY(cudaMemcpyAsync(c->kvec, kv.data(), kv.size() * sizeof(double4), cudaMemcpyHostToDevice, c->st));
    MFA_CUDA_TRY(cudaMemcpyAsync(c->kvec + c->nk, kn.data(), kn.size() * sizeof(int4), cudaMemcpyHostToDevice, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    // the charged particles, in id order
    {
        std::vector<double> qh(c->n);
        MFA_CUDA_TRY(cudaMemcpyAsync(qh.data(), c->q, (size_t)c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
        std::vector<int> idx;
        for (int i = 0; i < c->n; ++i)
            if (qh[i] != 0.0) idx.push_back(i);
        if (c->qidx) cudaFree(c->qidx);
        c->qidx = nullptr;
        c->nq = (int)idx.size();
        MFA_CUDA_TRY(cudaMalloc(&c->qidx, (idx.size() + 1) * sizeof(int)));
        if (!idx.empty())
            MFA_CUDA_TRY(cudaMemcpyAsync(c->qidx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    // runs of consecutive n_x at fixed (n_y, n_z), at most RSEG long; entry nrun closes the last
    {
        std::vector<int4> runs;
        for (int k = 0; k < c->nk; ++k) {
            const bool cont = k > 0 && kn[k].y == kn[k - 1].y && kn[k].z == kn[k - 1].z &&
                              kn[k].x == kn[k - 1].x + 1 && k - runs.back().w < RSEG;
            if (!cont) runs.push_back(make_int4(kn[k].x, kn[k].y, kn[k].z, k));
        }
        c->nrun = (int)runs.size();
        runs.push_back(make_int4(0, 0, 0, c->nk));
        if (c->kruns) cudaFree(c->kruns);
        c->kruns = nullptr;
        MFA_CUDA_TRY(cudaMalloc(&c->kruns, runs.size() * sizeof(int4)));
        MFA_CUDA_TRY(cudaMemcpyAsync(c->kruns, runs.data(), runs.size() * sizeof(int4), cudaMemcpyHostToDevice, c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    // block partials of rho: one per 32 RG charged particles
    int nblk = (c->nq + 32 * RG - 1) / (32 * RG);
    if (nblk < 1) nblk = 1;
    c->nblk_rho = nblk;
    MFA_CUDA_TRY(cudaMalloc(&c->rho, (size_t)2 * c->nk * sizeof(double2)));   // rho, then rho * A_k
    MFA_CUDA_TRY(cudaMalloc(&c->rho_part, (size_t)nblk * c->nk * sizeof(double2)));
    // the attribute is per function and shared by every context: admit the
    // largest tables any context can have (a launch passes its own size)
    const int rsm = CH * (3 * (KM + 1) * (int)sizeof(double2) + (int)sizeof(double));
    MFA_CUDA_TRY(cudaFuncSetAttribute(k_rho_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm));
    // (k_rho_runs: as far as the device's shared memory per block goes; a
    // context whose tables need more uses k_rho_partial)
    int optin = 0;
    MFA_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    int rrs = 32 * RG * (3 * (KM + 1) * (int)sizeof(double2) + (int)sizeof(double));
    if (rrs > optin) rrs = optin;
    const int frs = RP * 3 * (KM + 1) * (int)sizeof(double2) + RWMAX * RP * 3 * (int)sizeof(double);
    MFA_CUDA_TRY(cudaFuncSetAttribute(k_rho_runs, cudaFuncAttributeMaxDynamicSharedMemorySize, rrs));
    MFA_CUDA_TRY(cudaFuncSetAttribute(k_force_runs<float4>, cudaFuncAttributeMaxDynamicSharedMemorySize, frs));
    MFA_CUDA_TRY(cudaFuncSetAttribute(k_force_runs<double4>, cudaFuncAttributeMaxDynamicSharedMemorySize, frs));
    // launch shapes that keep each grid resident at once: the structure-factor
    // pass adds run sets (block rows) while they fit, the force pass takes the
    // most warps per block that still fit every block
    {
        int occ = 0;
        if (rho_runs_smem(c) <= (size_t)rrs) {
            MFA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rho_runs, RHW * 32, rho_runs_smem(c)));
            const int cap = (occ > 0 ? occ : 1) * c->n_sm;
            const int ry = cap / nblk;
            c->ew_rho_rows = ry < 1 ? 1 : (ry > 16 ? 16 : ry);
        } else {
            c->ew_rho_rows = 0;   // k_rho_partial
        }
        const int fb = (c->nq + RP - 1) / RP;
        const void* ff = c->prec == MFA_MIXED ? (const void*)k_force_runs<float4> : (const void*)k_force_runs<double4>;
        c->ew_force_warps = 4;
        for (int w = RWMAX; w > 4; --w) {
            MFA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ff, w * 32, force_runs_smem(c, w)));
            if ((long long)occ * c->n_sm >= fb) {
                c->ew_force_warps = w;
                break;
            }
        }
    }
    return MFA_OK;
}

int launch_ewald(mfa_ctx* c) {
    if (!c->p.charged) return MFA_OK;
    if (c->nk == 0) return MFA_ERR_STATE;
    EwArgs a = make_args(c);
    const RunArgs ra = run_args(c);
    if (c->ew_rho_rows > 0) {
        k_rho_runs<<<dim3(c->nblk_rho, c->ew_rho_rows), RHW * 32, rho_runs_smem(c), c->st>>>(a, ra);
    } else {
        const dim3 rgrid(c->nblk_rho, (c->nk + KPT * RHO_T - 1) / (KPT * RHO_T));
        k_rho_partial<<<rgrid, RHO_T, rho_smem(c), c->st>>>(a);
    }
    k_rho_reduce<<<reduce_grid(c), 256, 0, c->st>>>(a);
    const int fgrid = (c->nq + RP - 1) / RP;
    const int fw = c->ew_force_warps;
    if (fgrid > 0) {
        if (c->prec == MFA_MIXED) k_force_runs<float4><<<fgrid, fw * 32, force_runs_smem(c, fw), c->st>>>(a, ra);
        else k_force_runs<double4><<<fgrid, fw * 32, force_runs_smem(c, fw), c->st>>>(a, ra);
    }
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 3);
    return MFA_OK;
}

namespace {

// dipolar_correction.f90:20-24 (lz_half = boundary(3)/2, init_config.f90:246);
// the moment is kept in the last staging slot for the force pass, the energy
// (:32) in S_VDIP
constexpr int S_DIPM = S_TMP0 + 3;

__global__ void k_dipole_moment(EwArgs a, double lz_half) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {0.0};
    if (i < a.n) acc[0] = a.q[i] * (a.rz[i] - lz_half);
    if (block_sum_commit<1>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_DIPM) && threadIdx.x == 0) {
        const double m = a.dscal[S_DIPM];
        a.dscal[S_VDIP] = (((2.0 * a.pi) * m) * m) * a.inv_V;
    }
}

// dipolar_correction.f90:26-30
template <typename R4>
__global__ void k_dipole_force(EwArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double qi = a.q[i];
    if (qi == 0.0) return;
    const double m = a.dscal[S_DIPM];
    R4* f4 = (R4*)a.force;
    f4[i].z -= (((4.0 * a.pi) * qi) * m) * a.inv_V;
}

}  // namespace

int launch_dipolar(mfa_ctx* c) {
    if (!c->p.charged || c->p.symmetry != 0) return MFA_OK;
    if (c->nk == 0) return MFA_ERR_STATE;   // V is the slab volume ewald_k(0) sets
    EwArgs a = make_args(c);
    const int T = 256, nb = (c->n + T - 1) / T;
    if (nb > c->max_blocks) return MFA_ERR_ARGS;
    k_dipole_moment<<<nb, T, 0, c->st>>>(a, c->p.boundary[2] / 2.0);
    if (c->prec == MFA_MIXED) k_dipole_force<float4><<<nb, T, 0, c->st>>>(a);
    else k_dipole_force<double4><<<nb, T, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 2);
    return MFA_OK;
}

namespace {

// Adjoint of the k-space force.  F = -grad U_k, so its Jacobian is symmetric
// and (dF/dr)^T lam = (dF/dr) lam, the change of the force when every particle
// j moves along lam_j.  With theta_j = k.r_j, rho_k = sum_j q_j exp(i theta_j)
// and sigma_k = sum_j q_j (k.lam_j) exp(i theta_j):
//   dF_i = pre_i sum_k k A_k [cos theta_i Re sigma_k + sin theta_i Im sigma_k
//                              - (k.lam_i)(cos theta_i Re rho_k + sin theta_i Im rho_k)],
// pre_i = -8 pi q_i / V, A_k = inv_k2 exp(-k2 / 4 alpha) (the force of
// ewald_k.f90:168-197 differentiated).  sigma_k is summed like rho_k (block
// partials, then a block-ordered reduction).
__global__ void __launch_bounds__(RHO_T) k_sig_partial(EwArgs a, const double* __restrict__ lam) {
    extern __shared__ double2 rtab[];
    double* sq = (double*)(rtab + CH * 3 * a.ts);
    double* sl = sq + CH;                      // CH x 3 adjoint vectors
    const int p0 = blockIdx.x * a.per_blk, p1 = min(a.nq, p0 + a.per_blk);
    const int kb = blockIdx.y * KPT * RHO_T;
    double2 acc[KPT];
    int4 kn[KPT];
    double3 kv[KPT];
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        acc[j] = make_double2(0.0, 0.0);
        const int k = kb + threadIdx.x + j * RHO_T;
        kn[j] = k < a.nk ? a.kn[k] : make_int4(0, 0, 0, 0);
        const double4 v = k < a.nk ? a.kvec[k] : make_double4(0.0, 0.0, 0.0, 0.0);
        kv[j] = make_double3(v.x, v.y, v.z);
    }
    for (int b0 = p0; b0 < p1; b0 += CH) {
        const int nb = min(CH, p1 - b0);
        __syncthreads();
        if (threadIdx.x < nb) {
            const int i = a.qidx[b0 + threadIdx.x];
            build_tables(rtab + threadIdx.x * 3 * a.ts, a, a.rx[i], a.ry[i], a.rz[i]);
            sq[threadIdx.x] = a.q[i];
            sl[3 * threadIdx.x] = lam[i];
            sl[3 * threadIdx.x + 1] = lam[a.n + i];
            sl[3 * threadIdx.x + 2] = lam[2 * a.n + i];
        }
        __syncthreads();
        for (int pp = 0; pp < nb; ++pp) {
            const double qi = sq[pp], l0 = sl[3 * pp], l1 = sl[3 * pp + 1], l2 = sl[3 * pp + 2];
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                const double w = qi * (kv[j].x * l0 + kv[j].y * l1 + kv[j].z * l2);
                const double2 e = phase_from(rtab + pp * 3 * a.ts, a.ts, kn[j]);
                acc[j].x += w * e.x;
                acc[j].y += w * e.y;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        const int k = kb + threadIdx.x + j * RHO_T;
        if (k < a.nk) a.rho_part[(size_t)blockIdx.x * a.nk + k] = acc[j];
    }
}

__global__ void k_sig_reduce(EwArgs a, double2* sig) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < a.nk; k += nw) {
        const double2 s = warp_sum_partials(a.rho_part, a.nblk, a.nk, k, lane);
        if (lane == 0) sig[k] = s;
    }
}

__global__ void __launch_bounds__(FT) k_ewald_adj(EwArgs a, const double2* __restrict__ sig,
                                                  const double* __restrict__ lam, double* out) {
    extern __shared__ double2 ftab[];
    double2* t = ftab + threadIdx.x * 3 * a.ts;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double qi = a.q[i];
    if (qi == 0.0) return;
    build_tables(t, a, a.rx[i], a.ry[i], a.rz[i]);
    const double l0 = lam[i], l1 = lam[a.n + i], l2 = lam[2 * a.n + i];
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int k = 0; k < a.nk; ++k) {
        const double2 e = phase_from(t, a.ts, __ldg(&a.kn[k]));
        const double2 r = __ldg(&a.rho[k]);
        const double2 sg = __ldg(&sig[k]);
        const double4 kv = ldg4(&a.kvec[k]);
        const double kl = kv.x * l0 + kv.y * l1 + kv.z * l2;
        const double sc = ((e.x * sg.x + e.y * sg.y) - kl * (e.x * r.x + e.y * r.y)) * kv.w;
        gx += kv.x * sc;
        gy += kv.y * sc;
        gz += kv.z * sc;
    }
    const double pre = ((-8.0 * a.pi) * qi) * a.inv_V;
    out[i] += pre * gx;
    out[a.n + i] += pre * gy;
    out[2 * a.n + i] += pre * gz;
}

// Adjoint of the slab correction F_z,i = -4 pi q_i M_z / V, M_z = sum_j q_j
// (z_j - Lz/2): J_{iz,jz} = -4 pi q_i q_j / V (symmetric), so the product is
// -4 pi q_i / V sum_j q_j lam_z,j.
__global__ void k_dipole_adj_sum(EwArgs a, const double* __restrict__ lam, double* sum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = i < a.n ? a.q[i] * lam[2 * a.n + i] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(sum, v);
}

__global__ void k_dipole_adj(EwArgs a, const double* __restrict__ sum, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    out[2 * a.n + i] += (((-4.0 * a.pi) * a.q[i]) * *sum) * a.inv_V;
}

}  // namespace

// the adjoint kernels' shared-memory limits, set once before any launch or capture
int ewald_adjoint_prepare(mfa_ctx* c) {
    (void)c;
    const int fsm = FT * 3 * (KM + 1) * (int)sizeof(double2);
    const int rsm = CH * (3 * (KM + 1) * (int)sizeof(double2) + (int)sizeof(double));
    MFA_CUDA_TRY(cudaFuncSetAttribute(k_sig_partial, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      rsm + CH * 3 * (int)sizeof(double)));
    MFA_CUDA_TRY(cudaFuncSetAttribute(k_ewald_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
    return MFA_OK;
}

size_t ewald_adj_bytes(const mfa_ctx* c) { return (size_t)(c->nk > 0 ? c->nk : 1) * sizeof(double2) + 64; }

int launch_ewald_adjoint(mfa_ctx* c, const double* lam, double* out, void* scratch) {
    if (!c->p.charged) return MFA_OK;
    if (c->nk == 0) return MFA_ERR_STATE;
    EwArgs a = make_args(c);
    double2* sig = (double2*)scratch;
    double* dsum = (double*)((char*)scratch + (size_t)c->nk * sizeof(double2));

    const dim3 rgrid(c->nblk_rho, (c->nk + KPT * RHO_T - 1) / (KPT * RHO_T));
    // rho_k at the current positions, then sigma_k, then the product
    k_rho_partial<<<rgrid, RHO_T, rho_smem(c), c->st>>>(a);
    k_rho_reduce<<<reduce_grid(c), 256, 0, c->st>>>(a);
    const size_t ssm = rho_smem(c) + (size_t)CH * 3 * sizeof(double);
    k_sig_partial<<<rgrid, RHO_T, ssm, c->st>>>(a, lam);
    k_sig_reduce<<<reduce_grid(c), 256, 0, c->st>>>(a, sig);
    k_ewald_adj<<<(c->n + FT - 1) / FT, FT, adj_smem(c), c->st>>>(a, sig, lam, out);
    if (c->p.symmetry == 0) {
        const int T = 256, nb = (c->n + T - 1) / T;
        MFA_CUDA_TRY(cudaMemsetAsync(dsum, 0, sizeof(double), c->st));
        k_dipole_adj_sum<<<nb, T, 0, c->st>>>(a, lam, dsum);
        k_dipole_adj<<<nb, T, 0, c->st>>>(a, dsum, out);
    }
    MFA_CUDA_TRY(cudaGetLastError());
    return MFA_OK;
}

int mfa_ewald_download_kvecs(mfa_ctx* c, double* out3, int max_k) {
    if (!c->kvec) return 0;
    std::vector<double4> kv(c->nk);
    if (cudaMemcpy(kv.data(), c->kvec, kv.size() * sizeof(double4), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    const int m = c->nk < max_k ? c->nk : max_k;
    for (int k = 0; k < m; ++k) { out3[3 * k] = kv[k].x; out3[3 * k + 1] = kv[k].y; out3[3 * k + 2] = kv[k].z; }
    return c->nk;
}
