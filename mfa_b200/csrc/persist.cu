// One persistent launch for a whole run of steps of a batch (mfa_batch_step).
//
// This file is the translation unit of the time-step kernels: it includes the
// pair kernel (pair.cu), the integrator (integrate.cu) and the rebuild
// (binning.cu), so that their per-block bodies -- which take the block's
// position in its own context as an argument (Blk) -- can run as stages of one
// cooperative kernel.  A run of n steps of all systems is then ONE launch:
//
//   positions (first half step) | rebuild of the systems due |
//   n-1 x [ pair forces | velocities + positions (bonds, skin check) | rebuild ] |
//   pair forces | velocities
//
// with a grid-wide barrier between stages ("|").  Each stage is a grid-stride
// loop over the blocks the stage would have as a grouped launch (every
// system's share, found by binary search over block offsets), so the bodies
// are the single-context ones.  The rebuild stages run only when some
// system's skin check tripped (every CTA reads all systems' flags after the
// barrier that follows the integrator; a flag is cleared only after every CTA
// has passed five more barriers, so all CTAs decide alike), and inside them
// the systems not due return at once.  The grid is co-resident (cooperative
// launch sized by the occupancy calculator); every barrier wait is bounded
// (grid_barrier: 2 s, then MFA_ERR_TIMEOUT in the batch's status word and the
// CTA returns).
#include "pair.cu"
#include "integrate.cu"
#include "binning.cu"

namespace {

constexpr int PT = 256;   // threads per CTA of the persistent kernel

struct PersistArgs {
    const PairArgs* pair;          // per system (built for PT-thread blocks, untiled, no queue)
    const VVArgs* vvpos;
    const VVArgs* vvfused;
    const VVArgs* vvvel;
    const BinArgs* bin_first;      // the first step's rebuild (conditional on the skin flag)
    const BinArgs* bin_body;
    const int* off_pair;           // nsys + 1 block offsets per stage
    const int* off_vv;
    const int* off_bin;            // N_BIN_STAGES consecutive tables
    int nsys, nsteps;
    long long energy_span;
    unsigned* bar;                 // grid barrier words (GB_WORDS, zeroed)
    int32_t* status;               // the batch's error word (barrier timeouts)
};

__device__ __forceinline__ Blk vgroup(const int* __restrict__ off, int nsys, int vb, int& s) {
    s = group_of(off, nsys, vb);
    return Blk{vb - __ldg(&off[s]), __ldg(&off[s + 1]) - __ldg(&off[s])};
}

// the stages are separate functions (not inlined), so that each gets the
// register allocation of its own body instead of the union of all three
template <typename R, int K, int FT>
__device__ __noinline__ void stage_pair(const PersistArgs& p) {
    const int nv = p.off_pair[p.nsys];
    for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
        int s;
        const Blk blk = vgroup(p.off_pair, p.nsys, vb, s);
        pair_body<R, K, FT>(p.pair[s], blk);
        __syncthreads();
    }
}

template <typename R4>
__device__ __noinline__ void stage_vv(const PersistArgs& p, const VVArgs* tab, int stage, int energy_reset) {
    const int nv = p.off_vv[p.nsys];
    for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
        int s;
        const Blk blk = vgroup(p.off_vv, p.nsys, vb, s);
        if (stage == VV_POSITIONS) vv_positions_body<R4>(tab[s], blk, p.energy_span);
        else if (stage == VV_VELOCITIES) vv_velocities_body<R4>(tab[s], blk, energy_reset);
        else vv_fused_body<R4, false>(tab[s], blk);
        __syncthreads();
    }
}

// the rebuild of the systems whose skin check tripped; false: a barrier timed out
template <typename R4>
__device__ __noinline__ bool stage_rebuild(const PersistArgs& p, const BinArgs* tab) {
    int due = 0;
    for (int i = threadIdx.x; i < p.nsys; i += blockDim.x) due |= *(volatile const int32_t*)&tab[i].flags[F_SKIN];
    if (!__syncthreads_or(due)) return true;
    for (int st = 0; st < N_BIN_STAGES; ++st) {
        const int* off = p.off_bin + st * (p.nsys + 1);
        const int nv = off[p.nsys];
        for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
            int s;
            const Blk blk = vgroup(off, p.nsys, vb, s);
            switch (st) {
                case 0: cell_assign_body(tab[s], blk); break;
                case 1: scan_rows_body(tab[s], blk); break;
                case 2: cell_scatter_body(tab[s], blk); break;
                case 3: cell_sort_body(tab[s], blk); break;
                case 4: gather_sorted_body<R4>(tab[s], blk); break;
                default: build_nbr_body(tab[s], blk); break;
            }
            __syncthreads();
        }
        if (!grid_barrier(p.bar, p.status)) return false;
    }
    return true;
}

// FP32: 64 registers, four CTAs of 256 threads per SM (the integrator's bonded
// window would spill at 48); FP64: 128 registers, two CTAs (the FP64 pair body)
template <typename R4, typename R, int K, int FT>
__global__ void __launch_bounds__(PT, sizeof(R) == 4 ? 4 : 2) k_batch_run(PersistArgs p) {
    stage_vv<R4>(p, p.vvpos, VV_POSITIONS, 0);
    if (!grid_barrier(p.bar, p.status)) return;
    if (!stage_rebuild<R4>(p, p.bin_first)) return;
    for (int step = 1; step < p.nsteps; ++step) {
        stage_pair<R, K, FT>(p);
        if (!grid_barrier(p.bar, p.status)) return;
        stage_vv<R4>(p, p.vvfused, VV_FUSED, 0);
        if (!grid_barrier(p.bar, p.status)) return;
        if (!stage_rebuild<R4>(p, p.bin_body)) return;
    }
    stage_pair<R, K, FT>(p);
    if (!grid_barrier(p.bar, p.status)) return;
    stage_vv<R4>(p, p.vvvel, VV_VELOCITIES, 1);
}

// the feature sets a batch can have (no Ewald: charged systems are not batched)
constexpr int PERSIST_FT[] = {0, FT_DPD, FT_DPD | FT_WALL, FT_WALL, FT_LGV, FT_LGV | FT_WALL};
constexpr int N_PERSIST_FT = sizeof(PERSIST_FT) / sizeof(int);

template <typename R4, typename R, int I>
struct PersistDispatch {
    static const void* fn(int ft) {
        if (ft == PERSIST_FT[I]) return (const void*)k_batch_run<R4, R, 2, PERSIST_FT[I]>;
        return PersistDispatch<R4, R, I - 1>::fn(ft);
    }
};
template <typename R4, typename R>
struct PersistDispatch<R4, R, -1> {
    static const void* fn(int) { return nullptr; }
};

}  // namespace

// The persistent kernel of a batch's precision and feature set (its pair stage
// tests two list entries per lane at a time), or null when there is none.
const void* persist_kernel(int prec, int ft) {
    return prec == MFA_MIXED ? PersistDispatch<float4, float, N_PERSIST_FT - 1>::fn(ft)
                             : PersistDispatch<double4, double, N_PERSIST_FT - 1>::fn(ft);
}

size_t persist_args_bytes() { return sizeof(PersistArgs); }

// dynamic shared memory of the pair stage for PT-thread CTAs
size_t persist_smem(int prec) {
    return prec == MFA_MIXED ? smem_bytes<float>(2, PT, 0) : smem_bytes<double>(2, PT, 0);
}

int persist_threads() { return PT; }

// block counts of the rebuild stages for PT-thread CTAs (the stage bodies take
// their geometry from blockDim)
void persist_bin_blocks(const mfa_ctx* c, int nb[N_BIN_STAGES]) {
    for (int s = 0; s < N_BIN_STAGES; ++s) nb[s] = bin_stage_blocks(c, s, PT);
}

// Writes the argument record of the persistent kernel (device table pointers,
// sizes) into `out` (persist_args_bytes() bytes).
void persist_args(const void* pair, const void* vvpos, const void* vvfused, const void* vvvel, const void* bin_first,
                  const void* bin_body, const int* off_pair, const int* off_vv, const int* off_bin, int nsys,
                  int nsteps, long long energy_span, unsigned* bar, int32_t* status, void* out) {
    PersistArgs p;
    p.pair = (const PairArgs*)pair;
    p.vvpos = (const VVArgs*)vvpos;
    p.vvfused = (const VVArgs*)vvfused;
    p.vvvel = (const VVArgs*)vvvel;
    p.bin_first = (const BinArgs*)bin_first;
    p.bin_body = (const BinArgs*)bin_body;
    p.off_pair = off_pair;
    p.off_vv = off_vv;
    p.off_bin = off_bin;
    p.nsys = nsys;
    p.nsteps = nsteps;
    p.energy_span = energy_span;
    p.bar = bar;
    p.status = status;
    memcpy(out, &p, sizeof(p));
}
