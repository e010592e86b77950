// mfa_bin_cells_noalloc: the cell binning of binning.f90 (the counting sort
// that mfa_binning performs first) for callers that must not allocate device
// memory.  Some host programs own every byte of the GPU through their own
// pools, or call this at a point where an allocation -- with the device-wide
// synchronisation cudaMalloc/cudaFree may imply -- is not acceptable.  Such a
// caller passes its own input and output buffers; the only scratch the sort
// needs (a counter and a cursor per cell) lives in the fixed array below.
//
// g_noalloc_cells is a file-scope device array: every GPU that loads this
// library holds its MFA_NOALLOC_MAX_CELLS x 2 int32 (1 MiB) until the process
// exits, and all calls share it.  Calls whose work overlaps on the GPU (from
// several host threads or streams at once) race on it and must be serialised
// by the caller.  The counters are cleared at the start of every call, so
// the contents a previous call left behind do not matter.
//
// Host code cannot use the symbol itself as a device address, so every call
// looks the array's device address up with cudaGetSymbolAddress, with the
// caller's device current.  The lookup allocates nothing; doing it on every
// call (rather than caching it per device) keeps the address right after a
// cudaDeviceReset has re-created the context and reloaded this module.  The
// first call on a device loads the module there, so it should be made before
// any stream capture begins.
#include "mfa_internal.cuh"

#define MFA_NOALLOC_MAX_CELLS (1 << 17)

static __device__ __align__(256) int32_t g_noalloc_cells[2 * MFA_NOALLOC_MAX_CELLS + 32];

namespace {

struct NaArgs {
    const double* r0;      // device, xyz interleaved per particle
    int32_t* cell_of;      // device, n
    int32_t* cell_start;   // device, ncell + 1
    int32_t* ids;          // device, n
    int32_t* count;        // scratch, ncell
    int32_t* cursor;       // scratch, ncell
    int32_t* err;          // scratch, 1
    int n, ncell, rule;
    int nb[3];
    double rbin[3], inv_rbin[3];
};

__global__ void k_na_clear(NaArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) *a.err = 0;
    if (c < a.ncell) a.count[c] = 0;
}

// cell index of binning.f90:27-29 (rule 0) or my_binning.f90:28-30 (rule 1)
__global__ void k_na_count(NaArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int cc[3];
    bool bad = false, nonfinite = false;
    for (int d = 0; d < 3; ++d) {
        const double x = a.r0[3 * (size_t)i + d];
        if (!isfinite(x)) nonfinite = true;
        int ic;
        if (a.rule == 0) {
            ic = ((int)__dmul_rn(x, a.inv_rbin[d])) % a.nb[d];
            if (ic < 0) { bad = true; ic = 0; }
        } else {
            ic = (int)__ddiv_rn(x, a.rbin[d]);
            if (ic < 0 || ic >= a.nb[d]) { bad = true; ic = ic < 0 ? 0 : a.nb[d] - 1; }
        }
        cc[d] = ic;
    }
    if (nonfinite) atomicOr(a.err, 1 << MFA_ERR_NONFINITE);
    else if (bad) atomicOr(a.err, 1 << MFA_ERR_CELL_RANGE);
    const int c = cc[0] + a.nb[0] * (cc[1] + a.nb[1] * cc[2]);
    a.cell_of[i] = c;
    atomicAdd(&a.count[c], 1);
}

// one block: exclusive scan of the counters into cell_start and the cursors
__global__ void k_na_scan(NaArgs a) {
    __shared__ int wsum[32];
    const int T = blockDim.x, tid = threadIdx.x;
    const int chunk = (a.ncell + T - 1) / T;
    const int b0 = tid * chunk, b1 = min(a.ncell, b0 + chunk);
    int local = 0;
    for (int c = b0; c < b1; ++c) local += a.count[c];
    const int lane = tid & 31, wid = tid >> 5;
    int x = local;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (T >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    int run = (x - local) + (wid > 0 ? wsum[wid - 1] : 0);
    for (int c = b0; c < b1; ++c) {
        a.cell_start[c] = run;
        a.cursor[c] = run;
        run += a.count[c];
    }
    if (tid == T - 1) a.cell_start[a.ncell] = run;
}

__global__ void k_na_scatter(NaArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    a.ids[atomicAdd(&a.cursor[a.cell_of[i]], 1)] = i;
}

// particles of a cell in increasing id order (the order mfa_binning uses)
__global__ void k_na_sort(NaArgs a) {
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

// device address of the fixed scratch on the current device
int scratch_for_current_device(int32_t** out) {
    void* p = nullptr;
    MFA_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_cells));
    if (!p) return MFA_ERR_CUDA;
    *out = (int32_t*)p;
    return MFA_OK;
}

}  // namespace

extern "C" int mfa_bin_cells_noalloc(const double* r0, int32_t n, const double* boundary,
                                     const int32_t* n_bin, int32_t rule, int32_t* cell_of,
                                     int32_t* cell_start, int32_t* sorted_ids, void* stream) {
    if (n < 0 || !boundary || !n_bin || (rule != 0 && rule != 1)) return MFA_ERR_ARGS;
    if (n > 0 && (!r0 || !cell_of || !sorted_ids)) return MFA_ERR_ARGS;
    if (!cell_start) return MFA_ERR_ARGS;
    long long ncell = 1;
    NaArgs a;
    for (int d = 0; d < 3; ++d) {
        if (n_bin[d] < 1 || !(boundary[d] > 0.0)) return MFA_ERR_ARGS;
        // each factor and each partial product stays within the capacity, so
        // the product cannot overflow whatever the three values are
        if (n_bin[d] > MFA_NOALLOC_MAX_CELLS) return MFA_ERR_CAPACITY;
        ncell *= n_bin[d];
        if (ncell > MFA_NOALLOC_MAX_CELLS) return MFA_ERR_CAPACITY;
        a.nb[d] = n_bin[d];
        a.rbin[d] = boundary[d] / (double)n_bin[d];   // make_binning_boxes.f90:57-64
        a.inv_rbin[d] = 1.0 / a.rbin[d];
    }
    if (ncell > MFA_NOALLOC_MAX_CELLS) return MFA_ERR_CAPACITY;
    int32_t* scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != MFA_OK) return rc;
    a.r0 = r0; a.cell_of = cell_of; a.cell_start = cell_start; a.ids = sorted_ids;
    a.count = scratch;
    a.cursor = scratch + MFA_NOALLOC_MAX_CELLS;
    a.err = scratch + 2 * MFA_NOALLOC_MAX_CELLS;
    a.n = n; a.ncell = (int)ncell; a.rule = rule;
    cudaStream_t st = (cudaStream_t)stream;
    const int T = 256;
    k_na_clear<<<(int)((ncell + T - 1) / T), T, 0, st>>>(a);
    if (n > 0) k_na_count<<<(n + T - 1) / T, T, 0, st>>>(a);
    k_na_scan<<<1, 1024, 0, st>>>(a);
    if (n > 0) k_na_scatter<<<(n + T - 1) / T, T, 0, st>>>(a);
    k_na_sort<<<(int)((ncell + 127) / 128), 128, 0, st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    int32_t err = 0;
    MFA_CUDA_TRY(cudaMemcpyAsync(&err, a.err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MFA_CUDA_TRY(cudaStreamSynchronize(st));
    for (int s = 1; s < 31; ++s)
        if (err & (1 << s)) return s;
    return MFA_OK;
}
