// Cell binning and Verlet-list construction (binning.f90 / my_binning.f90).
//
// Integer work, HBM/L2 bound.  A counting sort of the particles by cell:
//   k_cell_assign   cell per particle (the reference's FP64 formula), cell and
//                   row histograms with atomics, r0_old/mic_old snapshot;
//   k_scan_rows     multi-block: each block gets its row offset from the row
//                   histogram, then one warp per row scans that row's cells;
//   k_cell_scatter  slot per particle (atomic cursor per cell);
//   k_cell_sort     per-cell sort by particle id, so the order is deterministic
//                   (the cooperative rebuild of the time-step graphs skips it
//                   and writes the records as it scatters);
//   k_gather_sorted the cell-sorted position/velocity records.
// A "row" is the run of cells at fixed (y, z); cells are numbered x-fastest, so
// a row is a contiguous range of slots.
//   k_build_nbr     thread per slot: scans the neighbouring cells and keeps j with
//                   r^2 < range_2(ti,tj) + skin_2, the reference's FP64
//                   expression evaluated without contraction (bit-exact pair set);
//                   a warp (32 consecutive slots) writes its entries as one run.
// binning.f90 keeps each pair once (i < j, binning.f90:81-104); here the pair is
// kept in the row of its lower slot (the pair kernel applies Newton's third
// law), so the set of unordered pairs -- with the reference's repeats when a
// cell is scanned twice -- is the reference's.  my_binning.f90 keeps both
// directions (a full list).  Layout: the entries of the 32 slots of chunk c are
// one run at nbr[c * 32 * maxnb ..] (ccount[c] of them, in no fixed order); an
// entry is (partner slot << 5 | lane of the owning slot in the chunk).
#include "mfa_internal.cuh"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

namespace {

struct BinArgs {
    const double *rx, *ry, *rz, *vx, *vy, *vz;
    double *ox, *oy, *oz;
    const int32_t *mx, *my, *mz;
    const int32_t* type;
    const double* q;
    int32_t *cell_count, *cell_start, *cell_cursor, *cell_of, *row_count;
    int32_t *ids, *slot;
    void* pos_s;
    void* vel_s;
    double4* pos64;
    float4* pos32;             // FP32 copy of pos64 for the list builder's prefilter
    int32_t *nbr, *nnb;
    int32_t* ccount;           // entries per 32-slot chunk
    int32_t* flags;
    unsigned* counter;
    int n, ncell, nrow, maxnb;
    int nb[3], dl[3];
    double L[3], invL[3], rbin[3], inv_rbin[3];
    int symmetry;
    int conditional;
    int rule;            // 0: binning.f90, 1: my_binning.f90
    int prefilter;       // FP32 prefilter of list candidates (n_bin >= 3 on every axis)
    int dense;           // crowded cells (prefilter grids only): a warp per cell sorts, 4 warps per chunk build
    float prefilter_margin;
    int in_cond_body;    // launched from a conditional graph node: count the rebuild there
    int with_pos64;      // the gather also writes the list builder's FP64/FP32 copies
    const double* cut2;  // list criterion range_2 + skin_2 (T8 x T8)
    int vnb[N_BIN_STAGES];   // cooperative rebuild: blocks of each stage at COOP_T threads
    unsigned* bar;           // cooperative rebuild: grid barrier words
    unsigned long long* stage_ns;   // cooperative rebuild: CTA 0's stage times (MFA_DEBUG=1), or null
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

// coordinate x moved by -L when binning.f90:27-29 wraps it into cell 0
// (int(x / r_bin) = n_bin, i.e. x at the upper edge of the box)
__device__ __forceinline__ double cell_image(const BinArgs& a, double x, int d) {
    if (a.rule != 0) return x;
    return (int)__dmul_rn(x, a.inv_rbin[d]) >= a.nb[d] ? __dsub_rn(x, a.L[d]) : x;
}

__device__ __forceinline__ void cell_assign_body(const BinArgs& a, Blk blk) {
    if (skip(a)) return;
    const int i = blk.id * blockDim.x + threadIdx.x;
    if (i == 0) {
        a.flags[F_MAXCELL] = 0;
        a.flags[F_MAXROW] = 0;
        a.flags[F_MAXTILE] = 0;
        a.flags[F_MAXNB] = 0;
    }
    if (i >= a.n) return;
    const double x = a.rx[i], y = a.ry[i], z = a.rz[i];
    bool bad = false;
    const int cx = cell_coord(a, x, 0, bad), cy = cell_coord(a, y, 1, bad), cz = cell_coord(a, z, 2, bad);
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) set_err(a.flags, MFA_ERR_NONFINITE);
    else if (bad) set_err(a.flags, MFA_ERR_CELL_RANGE);
    const int r = cy + a.nb[1] * cz;
    const int c = cx + a.nb[0] * r;
    a.cell_of[i] = c;
    atomicAdd(&a.cell_count[c], 1);
    atomicAdd(&a.row_count[r], 1);
    // binning.f90:126-127 snapshot, kept unwrapped: r0_old + mic_old * L,
    // rounded as the first operation of check_skin.f90:14-16 rounds it (the
    // skin check then reads 24 bytes per particle instead of 36)
    a.ox[i] = __dadd_rn(x, __dmul_rn((double)a.mx[i], a.L[0]));
    a.oy[i] = __dadd_rn(y, __dmul_rn((double)a.my[i], a.L[1]));
    a.oz[i] = __dadd_rn(z, __dmul_rn((double)a.mz[i], a.L[2]));
}

// Exclusive scan of the cell histogram into cell_start[0..ncell] (and the
// scatter cursors).  Block b owns rows [b*W, b*W + W), one warp per row; its
// starting offset is the sum of the row histogram below its first row.
__device__ __forceinline__ void scan_rows_body(const BinArgs& a, Blk blk) {
    if (skip(a)) return;
    __shared__ int wpart[32];
    __shared__ int rpre[33];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, W = blockDim.x >> 5;
    const int r0 = blk.id * W;
    // offset of this block: sum of row_count[0 .. r0)
    int s = 0;
    for (int r = threadIdx.x; r < r0; r += blockDim.x) s += a.row_count[r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) wpart[wid] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int base = 0;
        for (int w = 0; w < W; ++w) base += wpart[w];
        rpre[0] = base;
        for (int w = 0; w < W; ++w) rpre[w + 1] = rpre[w] + (r0 + w < a.nrow ? a.row_count[r0 + w] : 0);
    }
    __syncthreads();
    const int r = r0 + wid;
    if (r >= a.nrow) return;
    const int nx = a.nb[0];
    int carry = rpre[wid];
    int cmax = 0;
    for (int x0 = 0; x0 < nx; x0 += 32) {
        const int x = x0 + lane;
        const int k = x < nx ? a.cell_count[nx * r + x] : 0;
        cmax = max(cmax, k);
        int incl = k;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (x < nx) {
            const int st = carry + incl - k;
            a.cell_start[nx * r + x] = st;
            a.cell_cursor[nx * r + x] = st;
            a.cell_count[nx * r + x] = 0;
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    for (int o = 16; o > 0; o >>= 1) cmax = max(cmax, __shfl_down_sync(0xffffffffu, cmax, o));
    // records of this row's neighbourhood (the pair kernel's tile)
    const int wy = a.rule == 0 ? a.dl[1] + 2 : 3, wz = a.rule == 0 ? a.dl[2] + 2 : 3;
    int tile = 0;
    if (lane < wy * wz) {
        int ky, kz;
        neighbour_row(a.rule, r % a.nb[1], r / a.nb[1], lane % wy, lane / wy, a.nb[1], a.nb[2], ky, kz);
        tile = a.row_count[ky + a.nb[1] * kz];
    }
    for (int o = 16; o > 0; o >>= 1) tile += __shfl_down_sync(0xffffffffu, tile, o);
    if (lane == 0) {
        atomicMax(&a.flags[F_MAXCELL], cmax);
        atomicMax(&a.flags[F_MAXROW], rpre[wid + 1] - rpre[wid]);
        atomicMax(&a.flags[F_MAXTILE], tile);
        if (r == a.nrow - 1) a.cell_start[a.ncell] = carry;
    }
}

__device__ __forceinline__ void cell_scatter_body(const BinArgs& a, Blk blk) {
    if (skip(a)) return;
    const int i = blk.id * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int p = atomicAdd(&a.cell_cursor[a.cell_of[i]], 1);
    a.ids[p] = i;
}

// each cell's ids in ascending order; the row histogram is cleared here for
// the next rebuild.  Thread per cell: insertion sort (cells of a few to a few
// tens of particles).  Crowded cells (dense): a warp per cell, each lane ranks
// up to 4 ids against all of the cell's ids (ids are distinct) and writes them
// to their places -- O(k) steps for the warp instead of O(k^2) for one thread;
// a cell of more than 128 falls back to lane 0's insertion sort.
__device__ __forceinline__ void insertion_sort_ids(int32_t* ids, int b, int e) {
    for (int k = b + 1; k < e; ++k) {
        const int v = ids[k];
        int j = k - 1;
        while (j >= b && ids[j] > v) { ids[j + 1] = ids[j]; --j; }
        ids[j + 1] = v;
    }
}

__device__ __forceinline__ void cell_sort_body(const BinArgs& a, Blk blk) {
    if (skip(a)) return;
    const int t = blk.id * blockDim.x + threadIdx.x;
    if (t < a.nrow) a.row_count[t] = 0;
    if (!a.dense) {
        if (t >= a.ncell) return;
        insertion_sort_ids(a.ids, a.cell_start[t], a.cell_start[t + 1]);
        return;
    }
    const int c = t >> 5, lane = t & 31;      // c is the same for the whole warp
    if (c >= a.ncell) return;
    const int b = a.cell_start[c], k = a.cell_start[c + 1] - b;
    if (k > 128) {
        if (lane == 0) insertion_sort_ids(a.ids, b, b + k);
        return;
    }
    int v[4], rk[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        v[m] = lane + 32 * m < k ? a.ids[b + lane + 32 * m] : 0x7fffffff;
        rk[m] = 0;
    }
    for (int j = 0; j < k; ++j) {
        const int w = a.ids[b + j];
#pragma unroll
        for (int m = 0; m < 4; ++m) rk[m] += w < v[m] ? 1 : 0;
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m < 4; ++m)
        if (lane + 32 * m < k) a.ids[b + rk[m]] = v[m];
}

// the records of slot t, which holds particle i
template <typename R4>
__device__ __forceinline__ void write_slot(const BinArgs& a, int t, int i) {
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
    if (a.with_pos64) {
        double4 d;
        d.x = x; d.y = y; d.z = z;
        packw(d, i, ty);
        a.pos64[t] = d;
        // the list builder's FP32 copy holds the image of the particle that
        // lies in its cell: a coordinate equal to L (the wrap of
        // verlet_positions.f90:243-248 keeps x <= L) is binned into cell 0 by
        // binning.f90:27-29 and stored as x - L here.  z keeps its raw value
        // in channels (no z image there).
        float4 f;
        f.x = (float)(cell_image(a, x, 0)); f.y = (float)(cell_image(a, y, 1));
        f.z = (float)(a.symmetry == 1 ? cell_image(a, z, 2) : z);
        packw(f, i, ty);
        a.pos32[t] = f;
    }
}

template <typename R4>
__device__ __forceinline__ void gather_sorted_body(const BinArgs& a, Blk blk) {
    if (skip(a)) return;
    const int t = blk.id * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    write_slot<R4>(a, t, a.ids[t]);
}

// The cooperative rebuild's scatter: each particle takes a slot of its cell
// from the cell's cursor (order of arrival within a cell) and writes the
// slot's records at once, in place of the plain launches' scatter, per-cell
// id sort and gather (three stages and two grid barriers fewer).  The order
// within a cell changes neither the listed pairs nor the forces beyond the
// summation order, which the pair kernel's vector reductions leave unfixed
// anyway.  The row histogram is cleared here for the next rebuild (the scan
// was its last reader).
template <typename R4>
__device__ __forceinline__ void scatter_gather_body(const BinArgs& a, Blk blk) {
    if (skip(a)) return;
    const int i = blk.id * blockDim.x + threadIdx.x;
    for (int r = i; r < a.nrow; r += blk.n * blockDim.x) a.row_count[r] = 0;
    if (i >= a.n) return;
    const int t = atomicAdd(&a.cell_cursor[a.cell_of[i]], 1);
    a.ids[t] = i;
    write_slot<R4>(a, t, i);
}

// The x neighbours of cell column cx, as runs of consecutive cells [x0, x1)
// (a run breaks where the periodic wrap does, and repeats stay repeats: with
// nx = 2 the reference visits the other cell twice).
__device__ __forceinline__ int x_runs(const BinArgs& a, int cx, int nx, int wx, int* x0, int* x1) {
    int nr = 0;
    for (int ix = 0; ix < wx; ++ix) {
        int kx;
        if (a.rule == 0) {
            kx = wrap_near(cx - 1 + ix, nx);     // binning.f90:71-76: mod(cx - 1 + ix, nx)
        } else {
            kx = cx + ix - 1;                    // my_binning.f90:70-72
            if (kx < 0) kx = nx - 1;
            if (kx == nx) kx = 0;
        }
        if (nr > 0 && kx == x1[nr - 1]) {
            x1[nr - 1] = kx + 1;
        } else {
            x0[nr] = kx;
            x1[nr] = kx + 1;
            ++nr;
        }
    }
    return nr;
}

// Thread per slot: the neighbouring cells are visited as runs of consecutive
// slots (one or two per neighbouring row).  On grids with at least 3 cells on
// every axis (the prefilter path) a candidate is first tested in FP32 with the
// periodic image of its run applied to the owner's position once per run (a
// pair within the list radius lies in a neighbouring cell, so the cell
// stencil's image is its minimum image), against the owner type's largest
// list radius plus a margin far above FP32 rounding: about a dozen
// instructions per candidate.  Only those that pass get the reference's FP64
// test with the pair's own radius, so the kept set is exactly the FP64
// criterion's.  Smaller grids (where the reference may scan a cell twice and a
// pair's nearest image can be ambiguous in FP32) test every candidate in FP64.
__device__ __forceinline__ void build_nbr_body(const BinArgs& a, Blk blk) {
    if (skip(a)) return;
    __shared__ double sc[T8 * T8];
    __shared__ float scmax[T8];
    // the list of a 32-slot chunk is one run of entries (partner slot << 5 |
    // owner lane), appended through a shared cursor.  A chunk is one warp, or
    // with crowded cells (dense) four warps that split the owners' nine
    // neighbouring rows (3, 2, 2 and 2 of them), their counts summed in
    // shared memory.
    __shared__ int wcur[32];
    __shared__ int ccnt[8 * 32];
    const int R = a.dense ? 4 : 1;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int cib = wib / R, part = wib - cib * R;
    const int chunk = blk.id * ((blockDim.x >> 5) / R) + cib;
    const int t = (chunk << 5) + lane;
    const long long capc = 32LL * a.maxnb;
    int32_t* crow = a.nbr + (size_t)chunk * capc;
    for (int k = threadIdx.x; k < T8 * T8; k += blockDim.x) sc[k] = a.cut2[k];
    if (threadIdx.x < T8) {
        double m = 0.0;
        for (int k = 0; k < T8; ++k) m = fmax(m, a.cut2[threadIdx.x * T8 + k]);
        scmax[threadIdx.x] = (float)m + a.prefilter_margin;
    }
    if (part == 0) {
        if (lane == 0) wcur[cib] = 0;
        if (R > 1) ccnt[cib * 32 + lane] = 0;
    }
    __syncthreads();
    int cnt = 0;
    if (t < a.n) {
        const double4 pi = a.pos64[t];
        const int wi = wbits(pi.w);
        const int ti = wi & 0xff;
        const int nx = a.nb[0], ny = a.nb[1], nz = a.nb[2];
        // the owner's cell from its position, as cell_assign computes it
        bool bad = false;
        const int cx = cell_coord(a, pi.x, 0, bad), cy = cell_coord(a, pi.y, 1, bad),
                  cz = cell_coord(a, pi.z, 2, bad);
        const int trow = (ti - 1) * T8 - 1;
        // the reference's FP64 test of candidate slot s (binning.f90:89-104)
        auto exact = [&](int s) {
            const double4 pj = a.pos64[s];
            const int tj = wbits(pj.w) & 0xff;
            double d0 = __dsub_rn(pi.x, pj.x), d1 = __dsub_rn(pi.y, pj.y), d2 = __dsub_rn(pi.z, pj.z);
            d0 = mimage64(d0, a.L[0], a.invL[0]);
            d1 = mimage64(d1, a.L[1], a.invL[1]);
            if (a.symmetry == 1) d2 = mimage64(d2, a.L[2], a.invL[2]);
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
            if (r2 < sc[trow + tj]) {
                const int q = atomicAdd(&wcur[cib], 1);
                if (q < capc) crow[q] = (s << 5) | lane;
                ++cnt;
            }
        };
        if (a.prefilter) {
            // 3 x 3 x 3 stencil, nx, ny, nz >= 3: x runs [cx-1, cx+2) split where
            // the periodic wrap breaks them, each with the owner's image shift
            const float4 pf = a.pos32[t];
            const float cut = scmax[ti - 1];
            const float Lx = (float)a.L[0], Ly = (float)a.L[1], Lz = (float)a.L[2];
            const int xa0 = cx == 0 ? nx - 1 : (cx == nx - 1 ? nx - 2 : cx - 1);
            const int xa1 = cx == 0 ? nx : (cx == nx - 1 ? nx : cx + 2);
            const float sxa = cx == 0 ? Lx : 0.0f;
            const bool two = cx == 0 || cx == nx - 1;
            const int xb1 = cx == 0 ? 2 : 1;
            const float sxb = cx == 0 ? 0.0f : -Lx;
            for (int iz = 0; iz < 3; ++iz)
            for (int iy = 0; iy < 3; ++iy) {
                const int rr = 3 * iz + iy;
                if (R > 1 && part != (rr < 3 ? 0 : (rr - 1) >> 1)) continue;
                int ky, kz;
                neighbour_row(a.rule, cy, cz, iy, iz, ny, nz, ky, kz);
                const int uy = cy - 1 + iy, uz = cz - 1 + iz;
                const float oy = pf.y + (uy < 0 ? Ly : (uy >= ny ? -Ly : 0.0f));
                const float oz = a.symmetry == 1 ? pf.z + (uz < 0 ? Lz : (uz >= nz ? -Lz : 0.0f)) : pf.z;
                const int rb = nx * (ky + ny * kz);
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    if (r == 1 && !two) break;
                    int s0 = a.cell_start[rb + (r == 0 ? xa0 : 0)];
                    const int s1 = a.cell_start[rb + (r == 0 ? xa1 : xb1)];
                    const float ox = pf.x + (r == 0 ? sxa : sxb);
                    // half list: only partners at higher slots (the lower slot owns the pair)
                    if (a.rule == 0 && s0 <= t) s0 = t + 1;
                    for (int s = s0; s < s1; ++s) {
                        const float4 q = a.pos32[s];
                        const float dx = ox - q.x, dy = oy - q.y, dz = oz - q.z;
                        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        if (r2 < cut && s != t) exact(s);
                    }
                }
            }
        } else if (part == 0) {
            const int wx = a.rule == 0 ? a.dl[0] + 2 : 3;
            const int wy = a.rule == 0 ? a.dl[1] + 2 : 3;
            const int wz = a.rule == 0 ? a.dl[2] + 2 : 3;
            int x0[3], x1[3];
            const int nr = x_runs(a, cx, nx, wx, x0, x1);
            for (int iz = 0; iz < wz; ++iz)
            for (int iy = 0; iy < wy; ++iy) {
                int ky, kz;
                neighbour_row(a.rule, cy, cz, iy, iz, ny, nz, ky, kz);
                const int rb = nx * (ky + ny * kz);
                for (int r = 0; r < nr; ++r) {
                    int s0 = a.cell_start[rb + x0[r]];
                    const int s1 = a.cell_start[rb + x1[r]];
                    if (a.rule == 0 && s0 <= t) s0 = t + 1;
                    for (int s = s0; s < s1; ++s)
                        if (s != t) exact(s);
                }
            }
        }
        if (R > 1) atomicAdd(&ccnt[cib * 32 + lane], cnt);
    }
    __syncthreads();
    if (part == 0) {
        int mine = 0;
        if (t < a.n) {
            mine = R > 1 ? ccnt[cib * 32 + lane] : cnt;
            a.nnb[t] = mine;
        }
        // the longest row: one atomic per warp (a per-thread atomic on this one
        // address would serialise every thread of the grid at one L2 slice)
        const int mx = __reduce_max_sync(0xffffffffu, mine);
        if (lane == 0 && mx > 0) atomicMax(&a.flags[F_MAXNB], mx);
        if (lane == 0 && chunk * 32 < a.n) {
            const int total = wcur[cib];
            a.ccount[chunk] = (int)(total < capc ? total : capc);
            if (total > capc) {
                set_err(a.flags, MFA_ERR_NEIGH_OVERFLOW);
                atomicMax(&a.flags[F_NEEDNB], (total + 31) / 32);
            }
        }
    }
    // the last block to finish closes the rebuild: f_skin = 0 (binning.f90:125)
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(a.counter, 1u) == (unsigned)blk.n - 1);
    __syncthreads();
    if (last && threadIdx.x == 0) {
        *a.counter = 0u;
        a.flags[F_SKIN] = 0;
        a.flags[F_REBUILDS] += 1;
        if (a.in_cond_body) a.flags[F_CONDREB] += 1;
    }
}

// plain launches (one context) and the grouped launch (one stage for several
// contexts, argument records in device memory)
__global__ void k_cell_assign(BinArgs a) { cell_assign_body(a, plain_blk()); }
__global__ void k_scan_rows(BinArgs a) { scan_rows_body(a, plain_blk()); }
__global__ void k_cell_scatter(BinArgs a) { cell_scatter_body(a, plain_blk()); }
__global__ void k_cell_sort(BinArgs a) { cell_sort_body(a, plain_blk()); }
template <typename R4> __global__ void k_gather_sorted(BinArgs a) { gather_sorted_body<R4>(a, plain_blk()); }
__global__ void k_build_nbr(BinArgs a) { build_nbr_body(a, plain_blk()); }

// node_count (grouped rebuilds in a conditional graph node): counts the times
// the node ran, for the launch accounting of a batch
template <typename R4>
__global__ void k_bin_grouped(const BinArgs* __restrict__ as, const int* __restrict__ off, int nsys, int stage,
                              int* node_count) {
    if (node_count && stage == 0 && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(node_count, 1);
    const int s = group_of(off, nsys, blockIdx.x);
    const Blk blk = group_blk(off, s);
    switch (stage) {
        case 0: cell_assign_body(as[s], blk); break;
        case 1: scan_rows_body(as[s], blk); break;
        case 2: cell_scatter_body(as[s], blk); break;
        case 3: cell_sort_body(as[s], blk); break;
        case 4: gather_sorted_body<R4>(as[s], blk); break;
        default: build_nbr_body(as[s], blk); break;
    }
}

// One cooperative launch for the whole rebuild, used by the captured time-step
// graphs: cell assign, row scan, the scatter that writes the slots' records
// (scatter_gather_body) and the list build, each a grid-stride loop over the
// blocks it would have as a launch of its own, with a grid-wide barrier
// between stages.
// When no rebuild is due every CTA returns after one flag read -- a launch of
// one to three microseconds in place of a conditional graph node, whose
// evaluation held the device idle for about seven.  The grid is co-resident
// (cooperative launch), so the barrier's waits end; each is bounded all the
// same (2 s), after which the CTA reports MFA_ERR_TIMEOUT and returns.
constexpr int COOP_T = 256;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Two-level arrival: CTA b counts into group b % GB_SUB, the last of a group
// into the root, the last group resets the root and advances the generation
// (bar[0]); the CTAs of the other groups poll the generation with a growing
// pause.  Spreading the arrivals over GB_SUB + 1 lines keeps any one line's
// atomics to a few dozen.  Every CTA's writes before the barrier are visible
// to every CTA after it (fences on both sides, as a cooperative group's grid
// sync does).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int32_t* flags) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x;
        const unsigned grp = blockIdx.x % GB_SUB;
        const unsigned ngrp = nb < (unsigned)GB_SUB ? nb : (unsigned)GB_SUB;
        const unsigned in_grp = (nb - grp + GB_SUB - 1) / GB_SUB;
        unsigned* gen = bar;
        unsigned* root = bar + 32;
        unsigned* sub = bar + 64 + 32 * grp;
        const unsigned g = ld_acquire(gen);
        int ok = 1;
        __threadfence();
        bool released = false;
        if (atomicAdd(sub, 1u) == in_grp - 1) {
            *sub = 0u;
            __threadfence();   // the reset lands before the release that lets the group count again
            if (atomicAdd(root, 1u) == ngrp - 1) {
                *root = 0u;
                __threadfence();
                atomicAdd(gen, 1u);
                released = true;
            }
        }
        if (!released) {
            const unsigned long long t0 = global_ns();
            unsigned pause = 32;
            while (ld_acquire(gen) == g) {
                if (global_ns() - t0 > 2000000000ull) {
                    set_err(flags, MFA_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(pause);
                if (pause < 512) pause *= 2;
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// The stages of a cooperative rebuild on a co-resident grid: cell assign,
// row scan, scatter with the records, list build, with a grid barrier between
// stages.  False when a barrier wait timed out.  With MFA_DEBUG=1 (stage_ns
// set), CTA 0 sums the time from each stage's start to the barrier after it
// (the stage's critical path; the last stage: its own part).
template <typename R4>
__device__ __forceinline__ bool rebuild_stages(const BinArgs& a) {
    __shared__ unsigned long long t_prev;   // thread 0 of CTA 0 only (no register held across stages)
    if (a.stage_ns && blockIdx.x == 0 && threadIdx.x == 0) t_prev = global_ns();
    constexpr int NST = 4;
#pragma unroll
    for (int k = 0; k < NST; ++k) {
        const int st = k < 3 ? k : 5;
        const int nv = a.vnb[st];
        for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
            const Blk blk{vb, nv};
            switch (st) {
                case 0: cell_assign_body(a, blk); break;
                case 1: scan_rows_body(a, blk); break;
                case 2: scatter_gather_body<R4>(a, blk); break;
                default: build_nbr_body(a, blk); break;
            }
            __syncthreads();
        }
        if (k + 1 < NST && !grid_barrier(a.bar, a.flags)) return false;
        if (a.stage_ns && blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long t = global_ns();
            atomicAdd(&a.stage_ns[st], t - t_prev);
            t_prev = t;
        }
    }
    if (a.stage_ns && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.stage_ns[N_BIN_STAGES], 1ull);
    return true;
}

// 48 registers: five 256-thread CTAs per SM, 740 on 148 SMs, so every stage of
// a 189k-particle system takes one round (a few bytes of the list builder's
// registers spill)
template <typename R4>
__global__ void __launch_bounds__(COOP_T, 5) k_rebuild_coop(BinArgs a) {
    // the flag is set before this launch and cleared only by the last stage,
    // after every CTA has passed the barriers: all CTAs read the same value
    if (*(volatile const int32_t*)&a.flags[F_SKIN] == 0) return;
    rebuild_stages<R4>(a);
}

// block size of each rebuild stage (assign, row scan, scatter, sort, gather, build)
constexpr int BIN_T[N_BIN_STAGES] = {256, 256, 256, 128, 256, 128};

// crowded cells (8 or more particles on average, on a grid of at least 3
// cells per axis): the sort and the list build take more threads per cell
int bin_dense(const mfa_ctx* c) {
    return c->nb[0] >= 3 && c->nb[1] >= 3 && c->nb[2] >= 3 && (long long)c->n >= 8LL * c->ncell;
}

// blocks of T threads of each rebuild stage (T a multiple of 128)
int bin_stage_blocks(const mfa_ctx* c, int stage, int T) {
    const int nrow = c->nb[1] * c->nb[2];
    const bool dense = bin_dense(c) != 0;
    switch (stage) {
        case 1: return (nrow + T / 32 - 1) / (T / 32);
        case 3: return dense ? (int)(((long long)c->ncell * 32 + T - 1) / T) : (c->ncell + T - 1) / T;
        case 5: {
            const int nchunk = (c->n + 31) / 32, per = dense ? T / 128 : T / 32;
            return (nchunk + per - 1) / per;
        }
        default: return (c->n + T - 1) / T;
    }
}

BinArgs make_args(mfa_ctx* c, int rule, int conditional) {
    BinArgs a;
    a.rx = c->rx; a.ry = c->ry; a.rz = c->rz; a.vx = c->vx; a.vy = c->vy; a.vz = c->vz;
    a.ox = c->ox; a.oy = c->oy; a.oz = c->oz;
    a.mx = c->mx; a.my = c->my; a.mz = c->mz;
    a.type = c->type; a.q = c->p.charged ? c->q : nullptr;
    a.cell_count = c->cell_count; a.cell_start = c->cell_start; a.cell_cursor = c->cell_cursor;
    a.cell_of = c->cell_of; a.row_count = c->row_count; a.ids = c->ids; a.slot = c->slot;
    a.pos_s = c->pos_s; a.vel_s = c->vel_s; a.pos64 = c->pos64; a.pos32 = c->pos32;
    a.nbr = c->nbr; a.nnb = c->nnb; a.ccount = c->ccount; a.flags = c->dflags;
    a.counter = c->counters + R_BIN;
    a.n = c->n; a.ncell = c->ncell; a.nrow = c->nb[1] * c->nb[2]; a.maxnb = c->maxnb;
    for (int d = 0; d < 3; ++d) {
        a.nb[d] = c->nb[d]; a.dl[d] = c->p.delta_bin[d];
        a.L[d] = c->p.boundary[d]; a.invL[d] = c->inv_boundary[d];
        a.rbin[d] = c->rbin[d]; a.inv_rbin[d] = c->inv_rbin[d];
    }
    a.symmetry = c->p.symmetry;
    a.conditional = conditional;
    a.rule = rule;
    // FP32 candidate test: |r2_fp32 - r2| stays below ~1e-5 (L + 1) r_list for
    // positions in [0, L); the margin is orders of magnitude above that
    double lmax = 0.0, c2max = 0.0;
    for (int d = 0; d < 3; ++d) lmax = fmax(lmax, c->p.boundary[d]);
    for (int k = 0; k < T8 * T8; ++k) c2max = fmax(c2max, c->p.range_2[k] + c->p.skin_2);
    a.prefilter = c->nb[0] >= 3 && c->nb[1] >= 3 && c->nb[2] >= 3;
    a.dense = bin_dense(c);
    a.prefilter_margin = (float)(0.01 + 1e-4 * (lmax + 1.0) * sqrt(c2max));
    return a;
}

}  // namespace

size_t bin_args_bytes() { return sizeof(BinArgs); }

int bin_stage_args(mfa_ctx* c, int rule, int conditional, int in_cond_body, void* out, int nblocks[N_BIN_STAGES]) {
    if (rule == 0)
        for (int d = 0; d < 3; ++d)
            if (c->p.delta_bin[d] < -1 || c->p.delta_bin[d] > 1) return MFA_ERR_ARGS;
    BinArgs a = make_args(c, rule, conditional);
    for (int s = 0; s < N_BIN_STAGES; ++s) a.vnb[s] = 0;
    a.bar = nullptr;
    a.stage_ns = nullptr;
    a.in_cond_body = in_cond_body;
    a.with_pos64 = 1;
    a.cut2 = c->tabs;
    for (int s = 0; s < N_BIN_STAGES; ++s) nblocks[s] = bin_stage_blocks(c, s, BIN_T[s]);
    memcpy(out, &a, sizeof(a));
    return MFA_OK;
}

int launch_bin_grouped(int prec, int stage, const void* dargs, const int* doff, int nsys, int nblocks,
                       cudaStream_t st, int* node_count) {
    if (prec == MFA_MIXED)
        k_bin_grouped<float4><<<nblocks, BIN_T[stage], 0, st>>>((const BinArgs*)dargs, doff, nsys, stage, node_count);
    else
        k_bin_grouped<double4><<<nblocks, BIN_T[stage], 0, st>>>((const BinArgs*)dargs, doff, nsys, stage,
                                                                  node_count);
    MFA_CUDA_TRY(cudaGetLastError());
    return MFA_OK;
}

int launch_rebuild(mfa_ctx* c, int rule, int conditional) {
    return launch_rebuild_on(c, rule, conditional, c->st, 0);
}

int launch_rebuild_on(mfa_ctx* c, int rule, int conditional, cudaStream_t st, int in_cond_body) {
    BinArgs a;
    int nb[N_BIN_STAGES];
    TRY_(bin_stage_args(c, rule, conditional, in_cond_body, &a, nb));
    k_cell_assign<<<nb[0], BIN_T[0], 0, st>>>(a);
    k_scan_rows<<<nb[1], BIN_T[1], 0, st>>>(a);
    k_cell_scatter<<<nb[2], BIN_T[2], 0, st>>>(a);
    k_cell_sort<<<nb[3], BIN_T[3], 0, st>>>(a);
    if (c->prec == MFA_MIXED) k_gather_sorted<float4><<<nb[4], BIN_T[4], 0, st>>>(a);
    else k_gather_sorted<double4><<<nb[4], BIN_T[4], 0, st>>>(a);
    k_build_nbr<<<nb[5], BIN_T[5], 0, st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    if (!in_cond_body) note_launch(c, N_BIN_STAGES);
    return MFA_OK;
}

int launch_rebuild_coop(mfa_ctx* c, int rule) {
    BinArgs a;
    int nb[N_BIN_STAGES];
    TRY_(bin_stage_args(c, rule, 0, 0, &a, nb));
    for (int s = 0; s < N_BIN_STAGES; ++s) a.vnb[s] = bin_stage_blocks(c, s, COOP_T);
    a.bar = c->grid_bar;
    a.stage_ns = c->coop_stage_ns;
    const void* fn = c->prec == MFA_MIXED ? (const void*)k_rebuild_coop<float4> : (const void*)k_rebuild_coop<double4>;
    if (c->coop_grid < 1) return MFA_ERR_STATE;
    int vmax = 1;
    for (int s = 0; s < N_BIN_STAGES; ++s) vmax = a.vnb[s] > vmax ? a.vnb[s] : vmax;
    const int grid = c->coop_grid < vmax ? c->coop_grid : vmax;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(COOP_T);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    void* argv[] = {&a};
    MFA_CUDA_TRY(cudaLaunchKernelExC(&cfg, fn, argv));
    note_launch(c, 1);
    return MFA_OK;
}

// the cooperative rebuild's grid: the CTAs that fit the device at once
int rebuild_coop_setup(mfa_ctx* c) {
    const void* fn = c->prec == MFA_MIXED ? (const void*)k_rebuild_coop<float4> : (const void*)k_rebuild_coop<double4>;
    if (!c->grid_bar) {
        MFA_CUDA_TRY(cudaMalloc((void**)&c->grid_bar, GB_WORDS * sizeof(unsigned)));
        MFA_CUDA_TRY(cudaMemsetAsync(c->grid_bar, 0, GB_WORDS * sizeof(unsigned), c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    const char* dbg = getenv("MFA_DEBUG");
    if (dbg && dbg[0] == '1' && !c->coop_stage_ns) {
        MFA_CUDA_TRY(cudaMalloc((void**)&c->coop_stage_ns, 8 * sizeof(unsigned long long)));
        MFA_CUDA_TRY(cudaMemsetAsync(c->coop_stage_ns, 0, 8 * sizeof(unsigned long long), c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    int per_sm = 0;
    MFA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, COOP_T, 0));
    c->coop_grid = per_sm * c->n_sm;
    return per_sm >= 1 ? MFA_OK : MFA_ERR_UNSUPPORTED;
}

// MFA_DEBUG=1: the cooperative rebuild's stage times to stderr (at mfa_finalize)
void rebuild_coop_report(mfa_ctx* c) {
    if (!c->coop_stage_ns) return;
    unsigned long long h[8] = {0};
    if (cudaMemcpy(h, c->coop_stage_ns, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess || h[N_BIN_STAGES] == 0)
        return;
    const double k = 1e-3 / (double)h[N_BIN_STAGES];
    fprintf(stderr,
            "mfa: cooperative rebuild, %llu rebuilds, mean us per stage (CTA 0, to the barrier after it): "
            "assign %.1f scan %.1f scatter with records %.1f build %.1f\n",
            h[N_BIN_STAGES], h[0] * k, h[1] * k, h[2] * k, h[5] * k);
}

int launch_refresh_sorted(mfa_ctx* c) {
    BinArgs a = make_args(c, 0, 0);
    a.in_cond_body = 0;
    a.with_pos64 = 0;
    a.cut2 = c->tabs;
    const int nbp = (c->n + BIN_T[4] - 1) / BIN_T[4];
    if (c->prec == MFA_MIXED) k_gather_sorted<float4><<<nbp, BIN_T[4], 0, c->st>>>(a);
    else k_gather_sorted<double4><<<nbp, BIN_T[4], 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}
