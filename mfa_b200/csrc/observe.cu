// Per-observation quantities of observation.f90 and functions.f90 (histo),
// computed on the device so that an observation step reads back a few numbers
// instead of the whole state (md_main.f90:159-165).
//
//   k_obs_copy          unfolded coordinates start as the positions;
//   k_obs_refold_brush  thread per brush chain (SYMMETRY 0): each bead moves
//                       by one box length when it lies more than half a box
//                       from the (already moved) bead before it
//                       (observation.f90:178-191);
//   k_obs_refold_melt   thread per run of the melt/droplet ids between
//                       multiples of n_mon_d (global ids, as the reference's
//                       mod(i_part-1, n_mon_d) test, observation.f90:193-207);
//   k_obs_rg            thread per chain: centre of mass and per-axis mean
//                       square distance from it, grid-reduced in block order
//                       (observation.f90:238-266);
//   k_obs_momentum      sum of m v over all particles (:279-283);
//   k_obs_histo         z bins of the brush and melt beads, int(z / z_step) + 1
//                       clamped to 1..hist_dim (functions.f90:157-185), counted
//                       with FP64 atomics (exact for integers below 2^53);
//   k_obs_ends          one block: end-to-end vectors of the chains
//                       (functions.f90:626-667) summed per group (top brushes,
//                       bottom brushes, melt) and the force on the grafted
//                       heads of the last step summed per wall
//                       (observation.f90:326-328), each thread over a fixed
//                       stride of chains, then a fixed reduction tree.
#include "mfa_internal.cuh"

namespace {

struct ObsArgs {
    const double *rx, *ry, *rz, *vx, *vy, *vz, *mass;
    double *sx, *sy, *sz;            // unfolded coordinates
    double* out;                     // 9: r_g2 brush, r_g2 melt, momentum
    double* partials;
    unsigned* counter;
    int max_blocks;
    int n, n_mon, n_chain, n_mon_d, n_chain_d, symmetry;
    double L[3], half[3];
};

__global__ void k_obs_copy(ObsArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    a.sx[i] = a.rx[i];
    a.sy[i] = a.ry[i];
    a.sz[i] = a.rz[i];
}

__device__ __forceinline__ void move(const ObsArgs& a, int i) {
    double* s[3] = {a.sx, a.sy, a.sz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double cur = s[d][i], prev = s[d][i - 1];
        if (cur - prev > a.half[d]) s[d][i] = cur - a.L[d];
        else if (prev - cur > a.half[d]) s[d][i] = cur + a.L[d];
    }
}

__global__ void k_obs_refold_brush(ObsArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n_chain) return;
    const int b = c * a.n_mon;
    for (int j = 1; j < a.n_mon; ++j) move(a, b + j);
}

__global__ void k_obs_refold_melt(ObsArgs a, int first_run, int n_runs) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_runs) return;
    const int pd = a.n_mon * a.n_chain, pe = pd + a.n_mon_d * a.n_chain_d;
    const long long r0 = (long long)(first_run + r) * a.n_mon_d;
    const int s = (int)(r0 > pd ? r0 : pd);
    const int e = (int)(r0 + a.n_mon_d < pe ? r0 + a.n_mon_d : pe);
    for (int i = s; i < e; ++i)
        if (i % a.n_mon_d != 0) move(a, i);
}

// group 0: brush chains c = 0..n_chain-1 at c*n_mon (centre of mass times
// 1/n_mon); group 1: chains n_chain..n_chain+n_chain_d-1 at c*n_mon_d, the
// reference's indexing (divided by n_mon_d)
__global__ void k_obs_rg(ObsArgs a, int group) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int count = group == 0 ? a.n_chain : a.n_chain_d;
    const int len = group == 0 ? a.n_mon : a.n_mon_d;
    double acc[3] = {0.0, 0.0, 0.0};
    if (k < count) {
        const int b = group == 0 ? k * len : (a.n_chain + k) * len;
        const double* s[3] = {a.sx, a.sy, a.sz};
        const double inv = 1.0 / (double)len;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double cm = 0.0;
            for (int j = 0; j < len; ++j) cm += s[d][b + j];
            cm = group == 0 ? cm * inv : cm / (double)len;
            double v = 0.0;
            for (int j = 0; j < len; ++j) {
                const double x = s[d][b + j] - cm;
                v += x * x;
            }
            acc[d] = group == 0 ? v * inv : v / (double)len;
        }
    }
    if (block_sum_commit<3>(acc, a.partials, a.max_blocks, a.counter, a.out + 3 * group) && threadIdx.x == 0) {
        for (int d = 0; d < 3; ++d)
            a.out[3 * group + d] = group == 0 ? a.out[3 * group + d] * (1.0 / (double)count)
                                              : a.out[3 * group + d] / (double)count;
    }
}

__global__ void k_obs_momentum(ObsArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[3] = {0.0, 0.0, 0.0};
    if (i < a.n) {
        const double m = a.mass[i];
        acc[0] = m * a.vx[i];
        acc[1] = m * a.vy[i];
        acc[2] = m * a.vz[i];
    }
    block_sum_commit<3>(acc, a.partials, a.max_blocks, a.counter, a.out + 6);
}

__global__ void k_obs_histo(const double* rz, int pd, int pe, double inv_z_step, int hist_dim, double* hist) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pe) return;
    int z = (int)(rz[i] * inv_z_step) + 1;
    if (z < 1) z = 1;
    if (z > hist_dim) z = hist_dim;
    atomicAdd(&hist[(i < pd ? 0 : hist_dim) + z - 1], 1.0);
}

// 24 sums: r_ee (3 groups x xyz), r_ee^2 (3 x xyz), head force (2 walls x xyz).
// Chains 1..n_chain/2 are the top brushes, n_chain/2+1..n_chain the bottom
// ones, n_chain+1..n_chain+nmelt the melt, every chain taken as n_mon beads
// from (c-1) n_mon + 1 (the reference's indexing); the group sums are divided
// by n_chain/2 (integer division, both brush groups) and n_chain_d, and the
// head forces negated, as the reference writes them.  nmelt = 0 leaves the
// melt group NaN.
constexpr int NE = 24;
__global__ void __launch_bounds__(1024) k_obs_ends(ObsArgs a, const double* __restrict__ f_heads, int nmelt) {
    __shared__ double sm[NE][32];
    double acc[NE];
#pragma unroll
    for (int q = 0; q < NE; ++q) acc[q] = 0.0;
    const int nct = a.n_chain + nmelt, half = a.n_chain / 2;
    for (int c = threadIdx.x; c < nct; c += blockDim.x) {
        const int g = c < half ? 0 : (c < a.n_chain ? 1 : 2);
        const int f = c * a.n_mon, e = f + a.n_mon - 1;
        const double v[3] = {a.sx[e] - a.sx[f], a.sy[e] - a.sy[f], a.sz[e] - a.sz[f]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            acc[3 * g + d] += v[d];
            acc[9 + 3 * g + d] += v[d] * v[d];
        }
    }
    if (f_heads)
        for (int c = threadIdx.x; c < a.n_chain; c += blockDim.x) {
            const int w = c < half ? 0 : 1;
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[18 + 3 * w + d] += f_heads[3 * (size_t)c + d];
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NE; ++q) {
        double x = acc[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sm[q][wid] = x;
    }
    __syncthreads();
    if (wid == 0) {
        for (int q = 0; q < NE; ++q) {
            double x = lane < nw ? sm[q][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) {
                const int grp = q < 18 ? (q % 9) / 3 : -1;
                if (grp == 0 || grp == 1) x = x / (double)half;
                else if (grp == 2) x = nmelt > 0 ? x / (double)a.n_chain_d : __longlong_as_double(0x7ff8000000000000LL);
                else x = -x;
                a.out[9 + q] = x;
            }
        }
    }
}

constexpr int T = 256;

ObsArgs make_args(mfa_ctx* c) {
    const mfa_params& p = c->p;
    ObsArgs a;
    a.rx = c->rx; a.ry = c->ry; a.rz = c->rz;
    a.vx = c->vx; a.vy = c->vy; a.vz = c->vz;
    a.mass = c->mass;
    a.sx = c->obs_buf; a.sy = c->obs_buf + c->n; a.sz = c->obs_buf + 2 * (size_t)c->n;
    a.out = c->obs_buf + 3 * (size_t)c->n;
    a.max_blocks = c->max_blocks;
    a.n = c->n;
    a.n_mon = p.n_mon; a.n_chain = p.n_chain; a.n_mon_d = p.n_mon_d; a.n_chain_d = p.n_chain_d;
    a.symmetry = p.symmetry;
    for (int d = 0; d < 3; ++d) { a.L[d] = p.boundary[d]; a.half[d] = p.boundary[d] / 2.0; }
    return a;
}

int blocks(long long m) { return (int)((m + T - 1) / T); }

}  // namespace

extern "C" {

int mfa_observe(mfa_ctx* c, mfa_observables* o) {
    if (!c || !o) return MFA_ERR_ARGS;
    const mfa_params& p = c->p;
    // the melt indexing of observation.f90:256-259 must stay inside the particles
    if ((long long)(p.n_chain + p.n_chain_d) * p.n_mon_d > c->n) return MFA_ERR_UNSUPPORTED;
    if (blocks(c->n) > c->max_blocks) return MFA_ERR_ARGS;
    if (!c->obs_buf) MFA_CUDA_TRY(cudaMalloc((void**)&c->obs_buf, (3 * (size_t)c->n + 40) * sizeof(double)));
    ObsArgs a = make_args(c);
    int launches = 0;
    k_obs_copy<<<blocks(c->n), T, 0, c->st>>>(a);
    ++launches;
    if (p.symmetry == 0 && p.n_chain > 0 && p.n_mon > 1) {
        k_obs_refold_brush<<<blocks(p.n_chain), T, 0, c->st>>>(a);
        ++launches;
    }
    if (p.n_chain_d > 0 && p.n_mon_d > 1) {
        const int pd = p.n_mon * p.n_chain, pe = pd + p.n_mon_d * p.n_chain_d;
        const int first = pd / p.n_mon_d, last = (pe - 1) / p.n_mon_d;
        k_obs_refold_melt<<<blocks(last - first + 1), T, 0, c->st>>>(a, first, last - first + 1);
        ++launches;
    }
    // reductions in the observables' own partial-sum region
    a.partials = c->partials + (size_t)R_OBS * 4 * c->max_blocks;
    a.counter = c->counters + R_OBS;
    for (int g = 0; g < 2; ++g) {
        const int count = g == 0 ? p.n_chain : p.n_chain_d;
        if (count > 0 && (g == 0 ? p.n_mon : p.n_mon_d) > 0) {
            k_obs_rg<<<blocks(count), T, 0, c->st>>>(a, g);
            ++launches;
        }
    }
    k_obs_momentum<<<blocks(c->n), T, 0, c->st>>>(a);
    ++launches;
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, launches);
    double h[9];
    MFA_CUDA_TRY(cudaMemcpyAsync(h, a.out, sizeof(h), cudaMemcpyDeviceToHost, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    const double nan = __builtin_nan("");
    for (int d = 0; d < 3; ++d) {
        // no chains: 0/0 in the reference
        o->r_g2_brush[d] = p.n_chain > 0 && p.n_mon > 0 ? h[d] : nan;
        o->r_g2_melt[d] = p.n_chain_d > 0 && p.n_mon_d > 0 ? h[3 + d] : nan;
        o->momentum[d] = h[6 + d];
    }
    return MFA_OK;
}

int mfa_observe_ends(mfa_ctx* c, double* r_ee9, double* r_ee2_9, double* f_heads6) {
    if (!c) return MFA_ERR_ARGS;
    const mfa_params& p = c->p;
    // every chain, melt ones included, is read as n_mon beads (the reference's
    // indexing); melt "chains" of single beads (explicit solvent), or an
    // indexing that would run past the particles, leave the melt group NaN
    if (p.n_mon < 1 || (long long)p.n_chain * p.n_mon > c->n) return MFA_ERR_UNSUPPORTED;
    const int nmelt = (p.n_mon_d > 1 && (long long)(p.n_chain + p.n_chain_d) * p.n_mon <= c->n) ? p.n_chain_d : 0;
    if (!c->obs_buf) MFA_CUDA_TRY(cudaMalloc((void**)&c->obs_buf, (3 * (size_t)c->n + 40) * sizeof(double)));
    ObsArgs a = make_args(c);
    int launches = 1;
    // the chains refolded bead by bead, as for the radii of gyration
    k_obs_copy<<<blocks(c->n), T, 0, c->st>>>(a);
    if (p.symmetry == 0 && p.n_chain > 0 && p.n_mon > 1) {
        k_obs_refold_brush<<<blocks(p.n_chain), T, 0, c->st>>>(a);
        ++launches;
    }
    if (p.n_chain_d > 0 && p.n_mon_d > 1) {
        const int pd = p.n_mon * p.n_chain, pe = pd + p.n_mon_d * p.n_chain_d;
        const int first = pd / p.n_mon_d, last = (pe - 1) / p.n_mon_d;
        k_obs_refold_melt<<<blocks(last - first + 1), T, 0, c->st>>>(a, first, last - first + 1);
        ++launches;
    }
    k_obs_ends<<<1, 1024, 0, c->st>>>(a, c->f_heads, nmelt);
    ++launches;
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, launches);
    double h[NE];
    MFA_CUDA_TRY(cudaMemcpyAsync(h, a.out + 9, sizeof(h), cudaMemcpyDeviceToHost, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    for (int k = 0; k < 9; ++k) {
        if (r_ee9) r_ee9[k] = h[k];
        if (r_ee2_9) r_ee2_9[k] = h[9 + k];
    }
    for (int k = 0; k < 6; ++k)
        if (f_heads6) f_heads6[k] = c->f_heads ? h[18 + k] : 0.0;
    return MFA_OK;
}

int mfa_histogram_z(mfa_ctx* c, int32_t hist_dim, int32_t reset, double* counts, int32_t* n_obs) {
    if (!c || hist_dim < 1) return MFA_ERR_ARGS;
    const mfa_params& p = c->p;
    if (hist_dim != c->hist_dim) {
        if (c->hist) cudaFree(c->hist);
        c->hist = nullptr;
        c->hist_dim = 0;
        MFA_CUDA_TRY(cudaMalloc((void**)&c->hist, 2 * (size_t)hist_dim * sizeof(double)));
        c->hist_dim = hist_dim;
        reset = 1;
    }
    if (reset) {
        MFA_CUDA_TRY(cudaMemsetAsync(c->hist, 0, 2 * (size_t)hist_dim * sizeof(double), c->st));
        c->hist_obs = 0;
    }
    const int pd = p.n_mon * p.n_chain, pe = pd + p.n_mon_d * p.n_chain_d;
    if (pe > c->n) return MFA_ERR_ARGS;
    // functions.f90:124-125 (z_step) and :161 (r_scaled = z * inv_z_step)
    const double z_step = p.boundary[2] / (double)hist_dim;
    if (pe > 0) {
        k_obs_histo<<<blocks(pe), T, 0, c->st>>>(c->rz, pd, pe, 1.0 / z_step, hist_dim, c->hist);
        MFA_CUDA_TRY(cudaGetLastError());
        note_launch(c, 1);
    }
    c->hist_obs += 1;
    if (n_obs) *n_obs = c->hist_obs;
    if (counts) {
        MFA_CUDA_TRY(cudaMemcpyAsync(counts, c->hist, 2 * (size_t)hist_dim * sizeof(double), cudaMemcpyDeviceToHost,
                                     c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    return MFA_OK;
}

}  // extern "C"
