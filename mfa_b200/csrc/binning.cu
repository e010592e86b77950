// Cell binning and Verlet-list construction (binning.f90 / my_binning.f90).
//
// Integer work, HBM/L2 bound: a counting sort of the particles by cell
// (histogram with atomics, one-block exclusive scan, scatter, a per-cell sort by
// particle id so that the order is deterministic), a gather of the sorted
// position/velocity records, and a thread-per-particle scan of the neighbouring
// cells that keeps j with r^2 < range_2(ti,tj) + skin_2.  The distance test is
// the reference's FP64 expression evaluated without contraction, so the pair
// set equals the reference's bit for bit.  The list is stored full (both
// directions) in slot space, column-major: nbr[k*n + t].
#include "mfa_internal.cuh"

namespace {

struct BinArgs {
    const double *rx, *ry, *rz, *vx, *vy, *vz;
    double *ox, *oy, *oz;
    const int32_t *mx, *my, *mz;
    int32_t *omx, *omy, *omz;
    const int32_t* type;
    const double* q;
    int32_t *cell_count, *cell_start, *cell_cursor, *cell_of;
    int32_t *ids, *slot;
    void* pos_s;
    void* vel_s;
    double4* pos64;
    int32_t *nbr, *nnb;
    int32_t* flags;
    unsigned* counter;
    int n, ncell, maxnb;
    int nb[3], dl[3];
    double L[3], invL[3], rbin[3], inv_rbin[3];
    int symmetry;
    int conditional;
    int rule;            // 0: binning.f90, 1: my_binning.f90
};

__device__ __forceinline__ bool skip(const BinArgs& a) {
    return a.conditional && (*(volatile int32_t*)&a.flags[F_SKIN]) == 0;
}

__device__ __forceinline__ int cell_coord(const BinArgs& a, double x, int d, bool& bad) {
    int ic;
    if (a.rule == 0) {
        ic = ((int)__dmul_rn(x, a.inv_rbin[d])) % a.nb[d];   // binning.f90:27-29
        if (ic < 0) { bad = true; ic = 0; }
    } else {
        ic = (int)__ddiv_rn(x, a.rbin[d]);                   // my_binning.f90:28-30
        if (ic < 0 || ic >= a.nb[d]) { bad = true; ic = ic < 0 ? 0 : a.nb[d] - 1; }
    }
    return ic;
}

__global__ void k_cell_assign(BinArgs a) {
    if (skip(a)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double x = a.rx[i], y = a.ry[i], z = a.rz[i];
    bool bad = false;
    const int cx = cell_coord(a, x, 0, bad), cy = cell_coord(a, y, 1, bad), cz = cell_coord(a, z, 2, bad);
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) set_err(a.flags, MFA_ERR_NONFINITE);
    else if (bad) set_err(a.flags, MFA_ERR_CELL_RANGE);
    const int c = cx + a.nb[0] * (cy + a.nb[1] * cz);
    a.cell_of[i] = c;
    atomicAdd(&a.cell_count[c], 1);
    // binning.f90:126-127 snapshot
    a.ox[i] = x; a.oy[i] = y; a.oz[i] = z;
    a.omx[i] = a.mx[i]; a.omy[i] = a.my[i]; a.omz[i] = a.mz[i];
}

// One block: exclusive scan of cell_count into cell_start[0..ncell] and
// cell_cursor, largest occupancy, and cell_count cleared for the next rebuild.
__global__ void k_scan_cells(BinArgs a) {
    if (skip(a)) return;
    __shared__ int wsum[32];
    __shared__ int wmax[32];
    const int T = blockDim.x, tid = threadIdx.x;
    const int chunk = (a.ncell + T - 1) / T;
    const int b0 = tid * chunk, b1 = min(a.ncell, b0 + chunk);
    int local = 0, lmax = 0;
    for (int c = b0; c < b1; ++c) { int k = a.cell_count[c]; local += k; lmax = max(lmax, k); }
    // inclusive warp scan
    const int lane = tid & 31, wid = tid >> 5;
    int x = local;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    int m = lmax;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if (lane == 31) wsum[wid] = x;
    if (lane == 0) wmax[wid] = m;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (T >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, s, o); if (lane >= o) s += y; }
        wsum[lane] = s;
        int mm = lane < (T >> 5) ? wmax[lane] : 0;
        for (int o = 16; o > 0; o >>= 1) mm = max(mm, __shfl_down_sync(0xffffffffu, mm, o));
        if (lane == 0) a.flags[F_MAXCELL] = mm;
    }
    __syncthreads();
    int run = (x - local) + (wid > 0 ? wsum[wid - 1] : 0);
    for (int c = b0; c < b1; ++c) {
        const int k = a.cell_count[c];
        a.cell_start[c] = run;
        a.cell_cursor[c] = run;
        a.cell_count[c] = 0;
        run += k;
    }
    if (tid == T - 1) a.cell_start[a.ncell] = run;
}

__global__ void k_cell_scatter(BinArgs a) {
    if (skip(a)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int p = atomicAdd(&a.cell_cursor[a.cell_of[i]], 1);
    a.ids[p] = i;
}

// insertion sort of each cell's ids (cells hold a few to a few tens of particles)
__global__ void k_cell_sort(BinArgs a) {
    if (skip(a)) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncell) return;
    const int b = a.cell_start[c], e = a.cell_start[c + 1];
    for (int k = b + 1; k < e; ++k) {
        const int v = a.ids[k];
        int j = k - 1;
        while (j >= b && a.ids[j] > v) { a.ids[j + 1] = a.ids[j]; --j; }
        a.ids[j + 1] = v;
    }
}

template <typename R4>
__global__ void k_gather_sorted(BinArgs a, int with_pos64) {
    if (skip(a)) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int i = a.ids[t];
    a.slot[i] = t;
    const int ty = a.type[i];
    const double x = a.rx[i], y = a.ry[i], z = a.rz[i];
    R4 p;
    p.x = x; p.y = y; p.z = z;
    packw(p, i, ty);
    ((R4*)a.pos_s)[t] = p;
    R4 v;
    v.x = a.vx[i]; v.y = a.vy[i]; v.z = a.vz[i]; v.w = a.q ? a.q[i] : 0.0;
    ((R4*)a.vel_s)[t] = v;
    if (with_pos64) {
        double4 d;
        d.x = x; d.y = y; d.z = z;
        packw(d, i, ty);
        a.pos64[t] = d;
    }
}

__global__ void k_build_nbr(BinArgs a, const double* __restrict__ cut2 /*T8*T8*/) {
    if (skip(a)) return;
    __shared__ double sc[T8 * T8];
    for (int k = threadIdx.x; k < T8 * T8; k += blockDim.x) sc[k] = cut2[k];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < a.n) {
        const double4 pi = a.pos64[t];
        const int wi = wbits(pi.w);
        const int ti = wi & 0xff, ii = wi >> 8;
        const int c = a.cell_of[ii];
        const int cx = c % a.nb[0], cy = (c / a.nb[0]) % a.nb[1], cz = c / (a.nb[0] * a.nb[1]);
        int cnt = 0;
        const int nx = a.nb[0], ny = a.nb[1], nz = a.nb[2];
        const int ncells = a.rule == 0 ? (a.dl[0] + 2) * (a.dl[1] + 2) * (a.dl[2] + 2) : 27;
        for (int k = 0; k < ncells; ++k) {
            int kx, ky, kz;
            if (a.rule == 0) {
                // binning.f90:71-76: j = i-1 .. i+delta_bin, k = mod(j+n, n)
                const int wx = a.dl[0] + 2, wy = a.dl[1] + 2;
                const int jx = cx - 1 + k % wx, jy = cy - 1 + (k / wx) % wy, jz = cz - 1 + k / (wx * wy);
                kx = (jx + nx) % nx; ky = (jy + ny) % ny; kz = (jz + nz) % nz;
            } else {
                // my_binning.f90:70-80
                kx = cx + k % 3 - 1; if (kx < 0) kx = nx - 1; if (kx == nx) kx = 0;
                ky = cy + (k / 3) % 3 - 1; if (ky < 0) ky = ny - 1; if (ky == ny) ky = 0;
                kz = cz + k / 9 - 1; if (kz < 0) kz = nz - 1; if (kz == nz) kz = 0;
            }
            const int c2 = kx + nx * (ky + ny * kz);
            const int s0 = a.cell_start[c2], s1 = a.cell_start[c2 + 1];
            for (int s = s0; s < s1; ++s) {
                if (s == t) continue;
                const double4 pj = a.pos64[s];
                const int tj = wbits(pj.w) & 0xff;
                double d0 = __dsub_rn(pi.x, pj.x), d1 = __dsub_rn(pi.y, pj.y), d2 = __dsub_rn(pi.z, pj.z);
                d0 = mimage64(d0, a.L[0], a.invL[0]);
                d1 = mimage64(d1, a.L[1], a.invL[1]);
                if (a.symmetry == 1) d2 = mimage64(d2, a.L[2], a.invL[2]);
                const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
                if (r2 < sc[(ti - 1) * T8 + (tj - 1)]) {
                    if (cnt < a.maxnb) a.nbr[(size_t)cnt * a.n + t] = s;
                    ++cnt;
                }
            }
        }
        a.nnb[t] = min(cnt, a.maxnb);
        atomicMax(&a.flags[F_MAXNB], cnt);
        if (cnt > a.maxnb) {
            set_err(a.flags, MFA_ERR_NEIGH_OVERFLOW);
            atomicMax(&a.flags[F_NEEDNB], cnt);
        }
    }
    // the last block to finish closes the rebuild: f_skin = 0 (binning.f90:125)
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(a.counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (last && threadIdx.x == 0) {
        *a.counter = 0u;
        a.flags[F_SKIN] = 0;
        a.flags[F_REBUILDS] += 1;
    }
}

BinArgs make_args(mfa_ctx* c, int rule, int conditional) {
    BinArgs a;
    a.rx = c->rx; a.ry = c->ry; a.rz = c->rz; a.vx = c->vx; a.vy = c->vy; a.vz = c->vz;
    a.ox = c->ox; a.oy = c->oy; a.oz = c->oz;
    a.mx = c->mx; a.my = c->my; a.mz = c->mz;
    a.omx = c->omx; a.omy = c->omy; a.omz = c->omz;
    a.type = c->type; a.q = c->p.charged ? c->q : nullptr;
    a.cell_count = c->cell_count; a.cell_start = c->cell_start; a.cell_cursor = c->cell_cursor;
    a.cell_of = c->cell_of; a.ids = c->ids; a.slot = c->slot;
    a.pos_s = c->pos_s; a.vel_s = c->vel_s; a.pos64 = c->pos64;
    a.nbr = c->nbr; a.nnb = c->nnb; a.flags = c->dflags;
    a.counter = c->counters + R_N - 1;
    a.n = c->n; a.ncell = c->ncell; a.maxnb = c->maxnb;
    for (int d = 0; d < 3; ++d) {
        a.nb[d] = c->nb[d]; a.dl[d] = c->p.delta_bin[d];
        a.L[d] = c->p.boundary[d]; a.invL[d] = c->inv_boundary[d];
        a.rbin[d] = c->rbin[d]; a.inv_rbin[d] = c->inv_rbin[d];
    }
    a.symmetry = c->p.symmetry;
    a.conditional = conditional;
    a.rule = rule;
    return a;
}

}  // namespace

int launch_rebuild(mfa_ctx* c, int rule, int conditional) {
    if (rule == 0)
        for (int d = 0; d < 3; ++d)
            if (c->p.delta_bin[d] < -1 || c->p.delta_bin[d] > 1) return MFA_ERR_ARGS;
    BinArgs a = make_args(c, rule, conditional);
    const int T = 256;
    const int nbp = (c->n + T - 1) / T;
    k_cell_assign<<<nbp, T, 0, c->st>>>(a);
    k_scan_cells<<<1, 1024, 0, c->st>>>(a);
    k_cell_scatter<<<nbp, T, 0, c->st>>>(a);
    k_cell_sort<<<(c->ncell + 127) / 128, 128, 0, c->st>>>(a);
    if (c->prec == MFA_MIXED) k_gather_sorted<float4><<<nbp, T, 0, c->st>>>(a, 1);
    else k_gather_sorted<double4><<<nbp, T, 0, c->st>>>(a, 1);
    k_build_nbr<<<(c->n + 127) / 128, 128, 0, c->st>>>(a, c->tabs);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 6);
    return MFA_OK;
}

int launch_refresh_sorted(mfa_ctx* c) {
    BinArgs a = make_args(c, 0, 0);
    const int T = 256;
    const int nbp = (c->n + T - 1) / T;
    if (c->prec == MFA_MIXED) k_gather_sorted<float4><<<nbp, T, 0, c->st>>>(a, 0);
    else k_gather_sorted<double4><<<nbp, T, 0, c->st>>>(a, 0);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}
