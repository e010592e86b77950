// C ABI entry points (include/mfa_gpu.h): context lifetime, the per-step
// subroutines of md_main.f90:68-147, the captured-graph fast path, host mirrors.
#include "mfa_internal.cuh"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

int mfa_ewald_download_kvecs(mfa_ctx* c, double* out3, int max_k);

namespace {

template <typename T>
int dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (cudaMalloc((void**)p, count * sizeof(T)) != cudaSuccess) return MFA_ERR_NOMEM;
    return MFA_OK;
}

#define TRY(x)                          \
    do {                                \
        int s__ = (x);                  \
        if (s__ != MFA_OK) return s__;  \
    } while (0)

size_t esz(const mfa_ctx* c) { return c->prec == MFA_MIXED ? sizeof(float) : sizeof(double); }

// Host -> device copy ordered on the context's stream.  The stream is created
// non-blocking, so a copy or memset on the legacy default stream would not be
// ordered before the context's kernels (cudaMemcpy may return before its DMA
// lands); every upload and reset goes through the context's stream instead.
int h2d(mfa_ctx* c, void* dst, const void* src, size_t bytes) {
    MFA_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));   // the host buffer may be temporary
    return MFA_OK;
}
int dzero(mfa_ctx* c, void* dst, size_t bytes) {
    MFA_CUDA_TRY(cudaMemsetAsync(dst, 0, bytes, c->st));
    return MFA_OK;
}

int first_error(int bits) {
    for (int s = 1; s < 31; ++s)
        if (bits & (1 << s)) return s;
    return MFA_OK;
}

int check_params(const mfa_params* p, int precision) {
    if (!p) return MFA_ERR_ARGS;
    if (precision != MFA_FP64 && precision != MFA_MIXED) return MFA_ERR_ARGS;
    if (p->n_part <= 0 || p->n_part >= (1 << 23)) return MFA_ERR_ARGS;
    if (p->n_type < 1 || p->n_type > MFA_MAX_TYPES) return MFA_ERR_ARGS;
    for (int d = 0; d < 3; ++d) {
        if (!(p->boundary[d] > 0.0) || p->n_bin[d] < 1) return MFA_ERR_ARGS;
        if (p->delta_bin[d] < -1 || p->delta_bin[d] > 1) return MFA_ERR_ARGS;
    }
    if (p->n_mon < 0 || p->n_chain < 0 || p->n_mon_d < 0 || p->n_chain_d < 0) return MFA_ERR_ARGS;
    if ((long long)p->n_mon * p->n_chain + (long long)p->n_mon_d * p->n_chain_d > p->n_part) return MFA_ERR_ARGS;
    if (p->symmetry != 0 && p->symmetry != 1) return MFA_ERR_ARGS;
    if (p->thermostat < 0 || p->thermostat > 2) return MFA_ERR_ARGS;
    if (p->dpd_weight != 0 && p->dpd_weight != 1) return MFA_ERR_UNSUPPORTED;
    if (p->wall != 0 && p->wall != 2 && p->wall != 3 && p->wall != 4) return MFA_ERR_ARGS;
    if (!(p->dt > 0.0)) return MFA_ERR_ARGS;
    return MFA_OK;
}

void invalidate_graph(mfa_ctx* c) {
    for (int k = 0; k < 2 + N_CALL_GRAPHS; ++k) {
        if (c->gexec[k]) cudaGraphExecDestroy(c->gexec[k]);
        if (c->graph[k]) cudaGraphDestroy(c->graph[k]);
        c->gexec[k] = nullptr;
        c->graph[k] = nullptr;
        c->graph_kernels[k] = 0;
    }
    for (int k = 0; k < N_CALL_GRAPHS; ++k) c->call_n[k] = 0;
    c->graph_gen += 1;   // mfa_adjoint's cached sequences are stale too
}

// r0(3,n) <-> three contiguous arrays (x[0..n), y[n..2n), z[2n..3n))
__global__ void k_interleave3(const double* __restrict__ soa, double* __restrict__ aos, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    aos[3 * (size_t)i] = soa[i];
    aos[3 * (size_t)i + 1] = soa[(size_t)n + i];
    aos[3 * (size_t)i + 2] = soa[2 * (size_t)n + i];
}
__global__ void k_deinterleave3(const double* __restrict__ aos, double* __restrict__ soa, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    soa[i] = aos[3 * (size_t)i];
    soa[(size_t)n + i] = aos[3 * (size_t)i + 1];
    soa[2 * (size_t)n + i] = aos[3 * (size_t)i + 2];
}

void free_all(mfa_ctx* c) {
    invalidate_graph(c);
    adj_cache_free(c);
    void* ptrs[] = {c->rx, c->mx, c->type, c->mass, c->force, c->pos_s, c->vel_s, c->pos64, c->pos32,
                    c->ids, c->cell_count, c->nbr, c->nnb, c->partials, c->counters, c->dscal,
                    c->dstep, c->kvec, c->rho, c->rho_part, c->qidx, c->elog, c->elog_n, c->tabs,
                    c->obs_buf, c->hist, c->fd, c->term_buf, c->d_stage, c->f_heads, c->pair_qctr,
                    c->grid_bar, c->coop_stage_ns, c->kruns};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->h_scal) cudaFreeHost(c->h_scal);
    if (c->st) cudaStreamDestroy(c->st);
    if (c->st_body) cudaStreamDestroy(c->st_body);
}

int alloc_list(mfa_ctx* c, int maxnb) {
    if (c->nbr) cudaFree(c->nbr);
    c->nbr = nullptr;
    c->maxnb = maxnb;
    return dalloc(&c->nbr, (size_t)maxnb * 32 * ((c->n + 31) / 32));
}

int read_flags(mfa_ctx* c, int32_t* f) {
    MFA_CUDA_TRY(cudaMemcpyAsync(f, c->dflags, F_NFLAG * sizeof(int32_t), cudaMemcpyDeviceToHost, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    return MFA_OK;
}

// rebuild through the ABI (unconditional) with capacity growth on overflow
int rebuild_abi(mfa_ctx* c, int rule) {
    for (int attempt = 0; attempt < 3; ++attempt) {
        c->bin_type = rule;
        TRY(launch_rebuild(c, rule, 0));
        c->lists_valid = 1;
        int32_t f[F_NFLAG];
        TRY(read_flags(c, f));
        const int bits = f[F_ERR];
        if (bits & (1 << MFA_ERR_NEIGH_OVERFLOW)) {
            const int need = f[F_NEEDNB];
            int grow = ((need + need / 4 + 32) + 31) / 32 * 32;
            TRY(alloc_list(c, grow));
            invalidate_graph(c);
            int32_t zero[2] = {0, 0};
            const int32_t clear = bits & ~(1 << MFA_ERR_NEIGH_OVERFLOW);
            TRY(h2d(c, c->dflags + F_ERR, &clear, sizeof(int32_t)));
            TRY(h2d(c, c->dflags + F_NEEDNB, zero, sizeof(int32_t)));
            continue;
        }
        // size the pair kernel's shared-memory tile for the largest row seen
        // (with headroom); rows that outgrow it later are read from global memory
        const long long want = f[F_MAXTILE];
        if (want > c->tile_cap && c->tile_cap < pair_tile_limit(c)) {
            long long cap = want + want / 8 + 32;
            if (cap > pair_tile_limit(c)) cap = pair_tile_limit(c);
            TRY(pair_set_shape(c, c->pair_tpp, c->pair_block, (int)cap));
            // only tiled launches size their shared memory by the tile
            if (c->pair_tiled) invalidate_graph(c);
        }
        return first_error(bits);
    }
    return MFA_ERR_NEIGH_OVERFLOW;
}

// The non-bonded forces of a step (md_main.f90:93-97, 129) in the fewest
// passes: the pair kernel with the 9-3 walls (WALL 2) in its per-particle
// epilogue, then hard walls (WALL 3/4) and Ewald k-space if used.  The chains'
// FENE and bending forces (md_main.f90:106-111) are added bead by bead by the
// integrator kernel that consumes the force (launch_vv_* with fuse_bonds).
// defer_sum: the pair energies' grid sum is left to the integrator launch of
// the same step (the time-step fast path, where one always follows)
int forces_fused(mfa_ctx* c, int defer_sum = 0) {
    // fluid_wall is called for SYMMETRY 0 only (md_main.f90:97)
    TRY(launch_pair(c, c->p.symmetry == 0, 0, defer_sum));
    if (c->p.symmetry == 0 && (c->p.wall == 3 || c->p.wall == 4)) TRY(launch_wall(c, c->p.wall));
    if (c->p.charged) {
        TRY(launch_ewald(c));
        TRY(launch_dipolar(c));   // SYMMETRY 0 only (md_main.f90:128-131)
    }
    return MFA_OK;
}

constexpr int GRAPH_BODY = 10;

// The rebuild of a captured step as a conditional graph node: the kernel
// captured before it (the integrator's last block in a body step, a one-thread
// kernel after the first position half of a run) sets the node's condition
// from the skin check, and the six rebuild kernels run only when it tripped
// (no launches otherwise).  opener 0: the fused integrator; 1: positions only.
int capture_conditional_rebuild(mfa_ctx* c, int opener) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    MFA_CUDA_TRY(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return MFA_ERR_STATE;
    cudaGraphConditionalHandle h;
    MFA_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    if (opener == 0) TRY(launch_vv_fused(c, h, 1));
    else TRY(launch_open_rebuild(c, h));
    MFA_CUDA_TRY(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    MFA_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    MFA_CUDA_TRY(cudaStreamBeginCaptureToGraph(c->st_body, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
    const int rc = launch_rebuild_on(c, c->bin_type, 0, c->st_body, 1);
    cudaGraph_t out;
    const cudaError_t e = cudaStreamEndCapture(c->st_body, &out);
    if (rc != MFA_OK) return rc;
    MFA_CUDA_TRY(e);
    MFA_CUDA_TRY(cudaStreamUpdateCaptureDependencies(c->st, &node, 1, cudaStreamSetCaptureDependencies));
    return MFA_OK;
}

// A body step of a run of steps: forces of step n, then velocities of n fused
// with positions of n+1, then the rebuild of n+1 if due.
int launch_body_step(mfa_ctx* c) {
    TRY(forces_fused(c, 1));
    if (c->coop_rebuild) {
        TRY(launch_vv_fused(c, 0, 1));
        return launch_rebuild_coop(c, c->bin_type);
    }
    if (c->capturing && c->cond_rebuild) return capture_conditional_rebuild(c, 0);
    TRY(launch_vv_fused(c, 0, 1));
    return launch_rebuild(c, c->bin_type, 1);
}

// The first step of a run of nsteps steps: positions (+ skin check, force
// reset; the run's last step is the one whose energies are reduced), then the
// rebuild if due.  A run of one step is one time step as the reference orders
// it (md_main.f90:73-147): positions, rebuild if due, forces, velocities.
int launch_head_step(mfa_ctx* c, int nsteps) {
    TRY(launch_vv_positions(c, 1, 1, nsteps));
    if (c->coop_rebuild) return launch_rebuild_coop(c, c->bin_type);
    if (c->capturing && c->cond_rebuild) return capture_conditional_rebuild(c, 1);
    return launch_rebuild(c, c->bin_type, 1);
}

// The last step of a run: forces and the velocity half (energies reduced, and
// every step's energies wanted again afterwards).
int launch_tail_step(mfa_ctx* c) {
    TRY(forces_fused(c, 1));
    return launch_vv_velocities(c, 1, 1);
}

// kind 0: one body step; 1: GRAPH_BODY body steps; 2 + k: a whole run of
// call_n[k] steps (head, body steps, tail)
int capture(mfa_ctx* c, int kind) {
    cudaGraph_t g;
    MFA_CUDA_TRY(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    c->capturing = 1;
    c->cap_count = 0;
    int rc = MFA_OK;
    if (kind >= 2) {
        const int n = c->call_n[kind - 2];
        rc = launch_head_step(c, n);
        for (int s = 1; s < n && rc == MFA_OK; ++s) rc = launch_body_step(c);
        if (rc == MFA_OK) rc = launch_tail_step(c);
    } else {
        for (int s = 0; s < (kind == 0 ? 1 : GRAPH_BODY) && rc == MFA_OK; ++s) rc = launch_body_step(c);
    }
    c->capturing = 0;
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (rc != MFA_OK) return rc;
    MFA_CUDA_TRY(e);
    MFA_CUDA_TRY(cudaGraphInstantiate(&c->gexec[kind], g, 0));
    c->graph[kind] = g;
    c->graph_kernels[kind] = (int)c->cap_count;
    return MFA_OK;
}

// the captured graphs are dropped when what their arguments point to changed
void check_graph_key(mfa_ctx* c) {
    const void* key[4] = {c->nbr, c->elog, c->kvec, (const void*)(intptr_t)(c->bin_type + 1)};
    if (memcmp(key, c->graph_key, sizeof(key)) != 0) {
        invalidate_graph(c);
        memcpy(c->graph_key, key, sizeof(key));
    }
}

int replay(mfa_ctx* c, int kind) {
    check_graph_key(c);
    if (!c->gexec[kind]) {
        int rc = capture(c, kind);
        if (rc != MFA_OK && c->coop_rebuild) {
            // a runtime or device without captured cooperative launches: the
            // rebuild in conditional graph nodes
            cudaGetLastError();
            c->coop_rebuild = 0;
            int keep[N_CALL_GRAPHS];
            memcpy(keep, c->call_n, sizeof(keep));
            invalidate_graph(c);
            memcpy(c->call_n, keep, sizeof(keep));
            rc = capture(c, kind);
        }
        if (rc != MFA_OK && c->cond_rebuild) {
            // a runtime without conditional graph nodes: rebuild kernels that
            // return at once when no rebuild is due
            cudaGetLastError();
            c->cond_rebuild = 0;
            int keep[N_CALL_GRAPHS];
            memcpy(keep, c->call_n, sizeof(keep));
            invalidate_graph(c);
            memcpy(c->call_n, keep, sizeof(keep));
            rc = capture(c, kind);
        }
        TRY(rc);
    }
    MFA_CUDA_TRY(cudaGraphLaunch(c->gexec[kind], c->st));
    c->launches += c->graph_kernels[kind];
    return MFA_OK;
}

// Runs of up to CALL_GRAPH_MAX steps replay one graph for the whole run (its
// first step's rebuild in a conditional node too), captured once per step
// count and kept for the N_CALL_GRAPHS counts used last.
constexpr int CALL_GRAPH_MAX = 32;

int call_graph_slot(const mfa_ctx* c, int nsteps) {
    for (int k = 0; k < N_CALL_GRAPHS; ++k)
        if (c->call_n[k] == nsteps) return k;
    return -1;
}

int replay_call(mfa_ctx* c, int nsteps) {
    check_graph_key(c);
    int k = call_graph_slot(c, nsteps);
    if (k < 0) {
        k = 0;
        for (int j = 1; j < N_CALL_GRAPHS; ++j)
            if (c->call_used[j] < c->call_used[k]) k = j;
        if (c->gexec[2 + k]) cudaGraphExecDestroy(c->gexec[2 + k]);
        if (c->graph[2 + k]) cudaGraphDestroy(c->graph[2 + k]);
        c->gexec[2 + k] = nullptr;
        c->graph[2 + k] = nullptr;
        c->graph_kernels[2 + k] = 0;
        c->call_n[k] = nsteps;
    }
    c->call_used[k] = ++c->call_clock;
    return replay(c, 2 + k);
}

}  // namespace

extern "C" {

int mfa_abi_version(void) { return MFA_ABI_VERSION; }

int mfa_abi_sizes(int32_t* params_bytes, int32_t* scalars_bytes) {
    if (params_bytes) *params_bytes = (int32_t)sizeof(mfa_params);
    if (scalars_bytes) *scalars_bytes = (int32_t)sizeof(mfa_scalars);
    return MFA_OK;
}

const char* mfa_status_string(int s) {
    switch (s) {
        case MFA_OK: return "ok";
        case MFA_ERR_ARGS: return "invalid argument or parameter combination";
        case MFA_ERR_CUDA: return "CUDA runtime error";
        case MFA_ERR_CELL_RANGE: return "particle outside the binning grid";
        case MFA_ERR_NEIGH_OVERFLOW: return "neighbour list capacity exceeded";
        case MFA_ERR_NONFINITE: return "non-finite position or force";
        case MFA_ERR_TIMEOUT: return "bounded device wait timed out";
        case MFA_ERR_NOMEM: return "device allocation failed";
        case MFA_ERR_STATE: return "call order violated";
        case MFA_ERR_UNSUPPORTED: return "unsupported parameter set";
        case MFA_ERR_CAPACITY: return "request larger than a fixed-size buffer";
        default: return "unknown status";
    }
}

int mfa_init(const mfa_params* p, int precision, int device, const double* r0, const double* v,
             const double* a, const int32_t* a_type, const double* mass, const double* q,
             const int32_t* mic_count, mfa_ctx** out) {
    if (!out) return MFA_ERR_ARGS;
    *out = nullptr;
    TRY(check_params(p, precision));
    if (!r0 || !a_type || !mass) return MFA_ERR_ARGS;
    if (p->charged && !q) return MFA_ERR_ARGS;
    const int n = p->n_part;
    for (int i = 0; i < n; ++i) {
        if (a_type[i] < 1 || a_type[i] > p->n_type) return MFA_ERR_ARGS;
        if (!(mass[i] > 0.0)) return MFA_ERR_ARGS;
    }
    if (device >= 0) MFA_CUDA_TRY(cudaSetDevice(device));
    mfa_ctx* c = (mfa_ctx*)calloc(1, sizeof(mfa_ctx));
    if (!c) return MFA_ERR_NOMEM;
    c->p = *p;
    c->prec = precision;
    MFA_CUDA_TRY(cudaGetDevice(&c->dev));
    c->n = n;
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) { free(c); return MFA_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c->st_body, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(c->st);
        free(c);
        return MFA_ERR_CUDA;
    }
    // MFA_GRAPH_CONDITIONAL=0: the captured steps launch the rebuild kernels
    // every step and they return at once when no rebuild is due, instead of
    // holding them in conditional graph nodes (for tools that replay graph
    // nodes one at a time, such as kernel profilers)
    {
        const char* e = getenv("MFA_GRAPH_CONDITIONAL");
        c->cond_rebuild = (e && e[0] == '0') ? 0 : 1;
        // MFA_REBUILD_COOP=0: no cooperative rebuild kernel (the rebuild as
        // above); on by default where the device runs cooperative launches
        const char* k = getenv("MFA_REBUILD_COOP");
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->dev);
        c->coop_rebuild = (k && k[0] == '0') ? 0 : (coop ? 1 : 0);
        c->coop_grid = 0;
    }
    int rc = MFA_OK;
#define A(x) do { if (rc == MFA_OK) rc = (x); } while (0)
    // FP64 state: r, v, a, r0_old + mic_old * L (12 arrays)
    double* d12 = nullptr;
    A(dalloc(&d12, (size_t)12 * n));
    int32_t* i7 = nullptr;
    A(dalloc(&i7, (size_t)3 * n));
    if (rc == MFA_OK) {
        c->rx = d12; c->ry = d12 + n; c->rz = d12 + 2 * n;
        c->vx = d12 + 3 * n; c->vy = d12 + 4 * n; c->vz = d12 + 5 * n;
        c->ax = d12 + 6 * n; c->ay = d12 + 7 * n; c->az = d12 + 8 * n;
        c->ox = d12 + 9 * n; c->oy = d12 + 10 * n; c->oz = d12 + 11 * n;
        c->mx = i7; c->my = i7 + n; c->mz = i7 + 2 * n;
    }
    A(dalloc(&c->type, n));
    double* d3 = nullptr;
    A(dalloc(&d3, (size_t)3 * n));
    if (rc == MFA_OK) { c->mass = d3; c->inv_mass = d3 + n; c->q = d3 + 2 * n; }
    A(dalloc((unsigned char**)&c->force, (size_t)4 * n * esz(c)));
    A(dalloc((unsigned char**)&c->pos_s, (size_t)4 * n * esz(c)));
    A(dalloc((unsigned char**)&c->vel_s, (size_t)4 * n * esz(c)));
    A(dalloc(&c->pos64, n));
    A(dalloc(&c->pos32, n));
    int32_t* i2 = nullptr;
    A(dalloc(&i2, (size_t)2 * n));
    if (rc == MFA_OK) { c->ids = i2; c->slot = i2 + n; }
    // cells (make_binning_boxes.f90:57-64)
    c->ncell = 1;
    for (int d = 0; d < 3; ++d) {
        c->nb[d] = p->n_bin[d];
        c->ncell *= p->n_bin[d];
        c->rbin[d] = p->boundary[d] / (double)p->n_bin[d];
        c->inv_rbin[d] = 1.0 / c->rbin[d];
        c->inv_boundary[d] = 1.0 / p->boundary[d];   // init_config.f90:20
    }
    const int nrow = p->n_bin[1] * p->n_bin[2];
    int32_t* cells = nullptr;
    A(dalloc(&cells, (size_t)3 * c->ncell + 2 + n + nrow));
    if (rc == MFA_OK) {
        c->cell_count = cells;
        c->cell_start = cells + c->ncell;
        c->cell_cursor = cells + 2 * c->ncell + 1;
        c->cell_of = cells + 3 * c->ncell + 2;
        c->row_count = cells + 3 * c->ncell + 2 + n;
    }
    // Verlet list capacity: twice the expected count at the mean density
    double rc2max = 0.0;
    for (int k = 0; k < T8 * T8; ++k) rc2max = fmax(rc2max, p->range_2[k]);
    double rlist2 = rc2max + p->skin_2;
    if (p->charged && !(p->quirks & MFA_Q_EWALD_REAL_IN_LJ)) {
        const double re = sqrt(p->ewald_rc_2) + p->skin;
        rlist2 = fmax(rlist2, re * re);
    }
    const double vol = p->boundary[0] * p->boundary[1] * p->boundary[2];
    const double expect = 4.18879020478639 * pow(rlist2, 1.5) * (double)n / vol;
    int maxnb = ((int)(2.0 * expect) + 32 + 31) / 32 * 32;
    if (maxnb > n) maxnb = ((n + 31) / 32) * 32;
    if (rc == MFA_OK) rc = alloc_list(c, maxnb);
    A(dalloc(&c->nnb, (size_t)n + (n + 31) / 32));
    if (rc == MFA_OK) c->ccount = c->nnb + n;
    if (rc == MFA_OK && cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, c->dev) != cudaSuccess)
        rc = MFA_ERR_CUDA;
    if (rc == MFA_OK && c->coop_rebuild && rebuild_coop_setup(c) != MFA_OK) {
        cudaGetLastError();
        c->coop_rebuild = 0;
    }
    // partial-sum slots: enough for the largest grid of any reducing kernel
    // (particles / 32, cell rows, chains; 16 CTAs per SM for the pair kernel
    // of a small system whose chunks are cut into pieces)
    c->max_blocks = (n + 31) / 32 + 64;
    if (nrow + 64 > c->max_blocks) c->max_blocks = nrow + 64;
    if (p->n_chain + p->n_chain_d + 64 > c->max_blocks) c->max_blocks = p->n_chain + p->n_chain_d + 64;
    if (16 * c->n_sm > c->max_blocks) c->max_blocks = 16 * c->n_sm;
    A(dalloc(&c->partials, (size_t)R_N * 4 * c->max_blocks));
    A(dalloc(&c->counters, R_N));
    A(dalloc(&c->pair_qctr, 1));
    if (rc == MFA_OK && dzero(c, c->pair_qctr, sizeof(unsigned long long)) != MFA_OK) rc = MFA_ERR_CUDA;
    // pieces per chunk of the pair kernel's list: double while the warps
    // still fit the device twice over (32 per SM) and a piece keeps at least
    // two rounds of 64 entries (a half list: 32 owners x expect / 2 entries)
    {
        const long long nchunk = (n + 31) / 32;
        const double per_chunk = 16.0 * expect;
        c->pair_split = 1;
        while (c->pair_split < 16 && nchunk * c->pair_split * 2 <= 32LL * c->n_sm &&
               per_chunk / (2.0 * c->pair_split) >= 128.0)
            c->pair_split *= 2;
    }
    static_assert(F_NFLAG % 2 == 0, "the flags fill whole doubles after the energies");
    A(dalloc(&c->dscal, S_NSLOT + F_NFLAG / 2));
    if (rc == MFA_OK) c->dflags = (int32_t*)(c->dscal + S_NSLOT);
    A(dalloc(&c->dstep, 2));
    A(dalloc(&c->tabs, 6 * T8 * T8));
    if (p->pin_heads && p->n_chain > 0 && p->n_mon > 0) {
        A(dalloc(&c->f_heads, (size_t)3 * p->n_chain));
        if (rc == MFA_OK && dzero(c, c->f_heads, (size_t)3 * p->n_chain * sizeof(double)) != MFA_OK)
            rc = MFA_ERR_CUDA;
    }
    A(dalloc(&c->d_stage, (size_t)9 * n));   // three 3 x n slots: r0, v, a move together
    if (rc == MFA_OK && cudaMallocHost((void**)&c->h_scal, (S_NSLOT + F_NFLAG / 2) * sizeof(double)) != cudaSuccess)
        rc = MFA_ERR_NOMEM;
    if (rc != MFA_OK) { free_all(c); free(c); return rc; }
    // host-side staging
    std::vector<double> soa((size_t)12 * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            soa[(size_t)d * n + i] = r0[3 * i + d];
            soa[(size_t)(3 + d) * n + i] = v ? v[3 * i + d] : 0.0;
            soa[(size_t)(6 + d) * n + i] = a ? a[3 * i + d] : 0.0;
            // the skin snapshot holds r0_old + mic_old * L (check_skin.f90:14-16)
            const double m = mic_count ? (double)mic_count[3 * i + d] : 0.0;
            soa[(size_t)(9 + d) * n + i] = r0[3 * i + d] + m * p->boundary[d];
        }
    std::vector<int32_t> mic((size_t)3 * n, 0);
    if (mic_count)
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) mic[(size_t)d * n + i] = mic_count[3 * i + d];
    std::vector<double> m3((size_t)3 * n, 0.0);
    double vself = 0.0;
    for (int i = 0; i < n; ++i) {
        m3[i] = mass[i];
        m3[n + i] = 1.0 / mass[i];
        m3[2 * n + i] = q ? q[i] : 0.0;
        if (q) vself = vself - q[i] * q[i];
    }
    c->uniform_mass = 1;
    for (int i = 1; i < n; ++i)
        if (mass[i] != mass[0]) { c->uniform_mass = 0; break; }
    c->umass = n > 0 ? mass[0] : 1.0;
    c->uinv_mass = 1.0 / c->umass;
    c->v_coul_self = p->charged ? vself * p->sqrt_alpha / sqrt(p->pi) : 0.0;   // init_config.f90:235-239
    std::vector<double> tabs((size_t)6 * T8 * T8);
    // list criterion: range_2 + skin_2 (binning.f90:104); with the real-space
    // Ewald cutoff decoupled from the LJ range, out to rc_ewald + skin as well
    double ew_list2 = 0.0;
    if (p->charged && !(p->quirks & MFA_Q_EWALD_REAL_IN_LJ)) {
        const double re = sqrt(p->ewald_rc_2) + p->skin;
        ew_list2 = re * re;
    }
    for (int k = 0; k < T8 * T8; ++k) {
        tabs[k] = p->range_2[k] + p->skin_2;
        if (ew_list2 > tabs[k]) tabs[k] = ew_list2;
        tabs[T8 * T8 + k] = p->range_2[k];
        tabs[2 * T8 * T8 + k] = p->epsil[k];
        tabs[3 * T8 * T8 + k] = p->sigma_2[k];
        tabs[4 * T8 * T8 + k] = p->e_shift[k];
        tabs[5 * T8 * T8 + k] = p->inv_range_2[k];
    }
    rc = MFA_OK;
    A(dzero(c, c->force, (size_t)4 * n * esz(c)));
    A(dzero(c, c->cell_count, ((size_t)3 * c->ncell + 2 + n + nrow) * 4));
    A(dzero(c, c->nnb, ((size_t)n + (n + 31) / 32) * 4));
    A(dzero(c, c->counters, R_N * sizeof(unsigned)));
    A(dzero(c, c->dscal, S_NSLOT * 8));
    A(dzero(c, c->dflags, F_NFLAG * 4));
    A(dzero(c, c->dstep, 16));
    A(h2d(c, d12, soa.data(), soa.size() * 8));
    A(h2d(c, i7, mic.data(), mic.size() * 4));
    A(h2d(c, c->type, a_type, (size_t)n * 4));
    A(h2d(c, d3, m3.data(), m3.size() * 8));
    A(h2d(c, c->tabs, tabs.data(), tabs.size() * 8));
    if (rc == MFA_OK) rc = bonds_setup(c);
    // the step whose energies are wanted: -1 (all bytes set), every step
    if (rc == MFA_OK && cudaMemsetAsync(c->dstep + 1, 0xFF, 8, c->st) != cudaSuccess) rc = MFA_ERR_CUDA;
    if (rc == MFA_OK) {
        // pair kernel: 2 list entries per lane and round, 128-thread blocks
        // of consecutive slots; the tile (used when tiling is switched on) is
        // sized for 1.2x the mean neighbourhood of a row and grown at a rebuild
        const long long cap = 9LL * (6LL * n / (5LL * nrow) + 8);
        c->pair_tiled = 0;
        rc = pair_set_shape(c, 2, 128, (int)(cap < pair_tile_limit(c) ? cap : pair_tile_limit(c)));
    }
    if (rc != MFA_OK) { free_all(c); free(c); return rc; }
#undef A
    *out = c;
    return MFA_OK;
}

int mfa_finalize(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    cudaStreamSynchronize(c->st);
    rebuild_coop_report(c);
    free_all(c);
    free(c);
    return MFA_OK;
}

int mfa_set_step(mfa_ctx* c, int64_t i_time) {
    if (!c) return MFA_ERR_ARGS;
    c->i_time = i_time;
    MFA_CUDA_TRY(cudaMemcpyAsync(c->dstep, &c->i_time, 8, cudaMemcpyHostToDevice, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    return MFA_OK;
}

int mfa_verlet_positions(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    c->i_time += 1;
    return launch_vv_positions(c, 0, 0);
}

int mfa_check_skin(mfa_ctx* c, int32_t* f_skin) {
    if (!c || !f_skin) return MFA_ERR_ARGS;
    TRY(launch_check_skin(c));
    int32_t f[F_NFLAG];
    TRY(read_flags(c, f));
    *f_skin = f[F_SKIN];
    return first_error(f[F_ERR]);
}

int mfa_binning(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    return rebuild_abi(c, 0);
}

int mfa_my_binning(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    return rebuild_abi(c, 1);
}

int mfa_zero_forces(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaMemsetAsync(c->force, 0, (size_t)4 * c->n * esz(c), c->st));
    return MFA_OK;
}

int mfa_fluid_fluid(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    // fluid_fluid.f90:17 resets v_coul (the kernel does); the k-space part is
    // added by ewald_k, the slab correction by dipolar_correction
    return launch_pair(c, 0, 1);
}

int mfa_pair_forces(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    // v_coul reset as in fluid_fluid, and v_fluid_wall where no wall is fused
    const bool wall_fused = c->p.symmetry == 0 && (c->p.wall == 2 || c->p.wall == 3 || c->p.wall == 4);
    TRY(launch_pair(c, c->p.symmetry == 0, wall_fused ? 1 : 3));
    if (c->p.symmetry == 0 && (c->p.wall == 3 || c->p.wall == 4)) TRY(launch_wall(c, c->p.wall));
    return MFA_OK;
}

int mfa_forces(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    if (c->p.charged && c->nk == 0) return MFA_ERR_STATE;
    if (c->p.symmetry != 0 || (c->p.wall != 2 && c->p.wall != 3 && c->p.wall != 4))
        MFA_CUDA_TRY(cudaMemsetAsync(c->dscal + S_VFW, 0, 8, c->st));
    TRY(forces_fused(c));
    const bool chains = c->p.n_chain > 0 || (c->p.n_chain_d > 0 && c->p.n_mon_d >= 2);
    if (chains) TRY(launch_bonds(c, 1, 1));
    return MFA_OK;
}

int mfa_fluid_wall(mfa_ctx* c, int32_t inter_type) {
    if (!c) return MFA_ERR_ARGS;
    return launch_wall(c, inter_type);
}

int mfa_intra_molec(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    return launch_bonds(c, 1, 0);
}

int mfa_bending(mfa_ctx* c, int32_t mode) {
    if (!c) return MFA_ERR_ARGS;
    if (mode == 0 || mode == 1) return MFA_OK;   // bending.f90:12-20: report / no-op
    if (mode != 2) return MFA_ERR_ARGS;
    if (!c->p.bending) return MFA_OK;
    return launch_bonds(c, 0, 1);
}

int mfa_ewald_k(mfa_ctx* c, int32_t mode) {
    if (!c) return MFA_ERR_ARGS;
    if (!c->p.charged) return MFA_OK;
    if (mode == 0) {
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
        return ewald_setup(c);
    }
    if (mode != 1) return MFA_ERR_ARGS;
    return launch_ewald(c);
}

int mfa_dipolar_correction(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    return launch_dipolar(c);
}

int mfa_verlet_velocities(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    if (c->dpd_vv) return launch_dpd_vv_kick(c);
    return launch_vv_velocities(c, 0);
}

int mfa_step(mfa_ctx* c, int32_t nsteps) {
    if (!c || nsteps < 0) return MFA_ERR_ARGS;
    if (nsteps == 0) return MFA_OK;
    if (c->dpd_vv) return MFA_ERR_UNSUPPORTED;   // the fused step has no new_dpd_fd pass
    if (c->p.charged && c->nk == 0) return MFA_ERR_STATE;
    if (!c->lists_valid) TRY(rebuild_abi(c, c->bin_type));
    // energies are reduced for the last step only (and for the steps the
    // energy log records).  A step count seen in the previous call (or
    // captured before) replays one graph for the whole run; a new count runs
    // the first and last step as plain launches around the body graphs, so
    // that calls of ever-changing length capture nothing new.
    const bool whole = nsteps <= CALL_GRAPH_MAX &&
                       (nsteps == c->last_call_n || call_graph_slot(c, nsteps) >= 0);
    c->last_call_n = nsteps;
    if (whole) {
        TRY(replay_call(c, nsteps));
        c->i_time += nsteps;
        return MFA_OK;
    }
    // first step: positions (+ skin check, force reset), rebuild if due
    TRY(launch_head_step(c, nsteps));
    int body = nsteps - 1;
    while (body >= GRAPH_BODY) {
        TRY(replay(c, 1));
        body -= GRAPH_BODY;
    }
    while (body > 0) {
        TRY(replay(c, 0));
        --body;
    }
    // last step: forces and the velocity half
    TRY(launch_tail_step(c));
    c->i_time += nsteps;
    return MFA_OK;
}

int mfa_set_energy_log(mfa_ctx* c, int32_t every, int32_t capacity) {
    if (!c || every < 0 || capacity < 0) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    if (c->elog) cudaFree(c->elog);
    if (c->elog_n) cudaFree(c->elog_n);
    c->elog = nullptr;
    c->elog_n = nullptr;
    c->elog_every = 0;
    c->elog_cap = 0;
    invalidate_graph(c);
    if (every == 0 || capacity == 0) return MFA_OK;
    TRY(dalloc(&c->elog, (size_t)4 * capacity));
    TRY(dalloc(&c->elog_n, 1));
    TRY(dzero(c, c->elog_n, 4));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    c->elog_every = every;
    c->elog_cap = capacity;
    return MFA_OK;
}

int mfa_read_energy_log(mfa_ctx* c, double* out, int32_t max_entries, int32_t* n_out) {
    if (!c || !n_out) return MFA_ERR_ARGS;
    *n_out = 0;
    if (!c->elog) return MFA_OK;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    int32_t k = 0;
    MFA_CUDA_TRY(cudaMemcpy(&k, c->elog_n, 4, cudaMemcpyDeviceToHost));
    const int m = k < max_entries ? k : max_entries;
    if (out && m > 0) MFA_CUDA_TRY(cudaMemcpy(out, c->elog, (size_t)m * 4 * 8, cudaMemcpyDeviceToHost));
    *n_out = m;
    return MFA_OK;
}

int mfa_fetch_energy_log(mfa_ctx* c, double* out, int32_t first, int32_t count) {
    if (!c || first < 0 || count < 0 || (count > 0 && !out)) return MFA_ERR_ARGS;
    if (!c->elog) return MFA_ERR_STATE;
    if ((long long)first + count > c->elog_cap) return MFA_ERR_ARGS;
    if (count == 0) return MFA_OK;
    // ordered after every step already enqueued on the context stream; the
    // caller synchronises (mfa_sync, mfa_download, ...) before reading `out`
    MFA_CUDA_TRY(cudaMemcpyAsync(out, c->elog + (size_t)4 * first, (size_t)count * 4 * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->st));
    return MFA_OK;
}

int mfa_get_scalars(mfa_ctx* c, mfa_scalars* o) {
    if (!c || !o) return MFA_ERR_ARGS;
    // energies and flags are one device allocation: one copy into pinned memory
    MFA_CUDA_TRY(cudaMemcpyAsync(c->h_scal, c->dscal, (S_NSLOT + F_NFLAG / 2) * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    const double* s = c->h_scal;
    const int32_t* f = (const int32_t*)(c->h_scal + S_NSLOT);
    memset(o, 0, sizeof(*o));
    o->v_fluid_fluid = s[S_VFF];
    o->v_fluid_wall = s[S_VFW];
    o->v_intra_molec = s[S_VINTRA];
    o->v_bend = s[S_VBEND];
    o->v_coul = c->p.charged ? ((s[S_VCR] + c->v_coul_self) + s[S_VCK]) + s[S_VDIP] : 0.0;
    o->t_fluid = s[S_TKIN];
    o->v_total = s[S_VTOT];
    o->e_total = s[S_ETOT];
    o->virial = s[S_VIR];
    o->i_time = c->i_time;
    o->f_skin = f[F_SKIN];
    o->n_rebuilds = f[F_REBUILDS];
    o->max_neigh = f[F_MAXNB];
    o->max_cell = f[F_MAXCELL];
    o->fene_clamped = f[F_FENE];
    o->error_bits = f[F_ERR];
    // kernels of rebuilds that ran inside conditional graph nodes are counted on the device
    o->kernel_launches = c->launches + 6LL * f[F_CONDREB];
    return first_error(f[F_ERR]);
}

int mfa_set_cells(mfa_ctx* c, const int32_t* n_bin, double skin) {
    if (!c || !n_bin || !(skin >= 0.0)) return MFA_ERR_ARGS;
    mfa_params p = c->p;
    // skin_2 as init_params.f90:807-808 derives it
    double rc2max = 0.0;
    for (int k = 0; k < T8 * T8; ++k) rc2max = fmax(rc2max, p.range_2[k]);
    const double rcm = sqrt(rc2max);
    p.skin = skin;
    p.skin_2 = (rcm + skin) * (rcm + skin) - rcm * rcm;
    double rlist2 = rc2max + p.skin_2;
    if (p.charged && !(p.quirks & MFA_Q_EWALD_REAL_IN_LJ)) {
        const double re = sqrt(p.ewald_rc_2) + skin;
        rlist2 = fmax(rlist2, re * re);
    }
    const double rlist = sqrt(rlist2);
    long long ncell = 1;
    for (int d = 0; d < 3; ++d) {
        if (n_bin[d] < 1) return MFA_ERR_ARGS;
        // every pair within the list radius must lie in neighbouring cells
        if (n_bin[d] >= 3 && p.boundary[d] / n_bin[d] < rlist) return MFA_ERR_ARGS;
        ncell *= n_bin[d];
    }
    if (ncell > (1LL << 26)) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    const int n = c->n;
    const int nrow = n_bin[1] * n_bin[2];
    int32_t* cells = nullptr;
    TRY(dalloc(&cells, (size_t)3 * ncell + 2 + n + nrow));
    TRY(dzero(c, cells, ((size_t)3 * ncell + 2 + n + nrow) * 4));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    if (nrow + 64 > c->max_blocks) {
        double* part = nullptr;
        TRY(dalloc(&part, (size_t)R_N * 4 * (nrow + 64)));
        cudaFree(c->partials);
        c->partials = part;
        c->max_blocks = nrow + 64;
    }
    cudaFree(c->cell_count);
    c->cell_count = cells;
    c->cell_start = cells + ncell;
    c->cell_cursor = cells + 2 * ncell + 1;
    c->cell_of = cells + 3 * ncell + 2;
    c->row_count = cells + 3 * ncell + 2 + n;
    c->ncell = (int)ncell;
    for (int d = 0; d < 3; ++d) {
        p.n_bin[d] = n_bin[d];
        p.delta_bin[d] = n_bin[d] >= 3 ? 1 : (n_bin[d] == 2 ? 0 : -1);
        c->nb[d] = n_bin[d];
        c->rbin[d] = p.boundary[d] / (double)n_bin[d];
        c->inv_rbin[d] = 1.0 / c->rbin[d];
    }
    c->p = p;
    // list criterion table and capacity for the new radius
    double tab0[T8 * T8];
    for (int k = 0; k < T8 * T8; ++k) tab0[k] = fmax(p.range_2[k] + p.skin_2, rlist2 > rc2max + p.skin_2 ? rlist2 : 0.0);
    TRY(h2d(c, c->tabs, tab0, sizeof(tab0)));
    const double vol = p.boundary[0] * p.boundary[1] * p.boundary[2];
    int maxnb = ((int)(2.0 * 4.18879020478639 * rlist2 * rlist * n / vol) + 32 + 31) / 32 * 32;
    if (maxnb > n) maxnb = ((n + 31) / 32) * 32;
    if (maxnb > c->maxnb) TRY(alloc_list(c, maxnb));
    const long long cap = 9LL * (6LL * n / (5LL * nrow) + 8);
    TRY(pair_set_shape(c, c->pair_tpp, c->pair_block, (int)(cap < pair_tile_limit(c) ? cap : pair_tile_limit(c))));
    // the next step rebuilds the cells and the list: mfa_step does so itself,
    // and check_skin reports the rebuild as due to a subroutine-level driver
    c->lists_valid = 0;
    const int32_t one = 1;
    TRY(h2d(c, c->dflags + F_SKIN, &one, sizeof(one)));
    invalidate_graph(c);
    return MFA_OK;
}

int mfa_set_pair_shape(mfa_ctx* c, int32_t k, int32_t block, int32_t tiled) {
    if (!c || (tiled != 0 && tiled != 1)) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    c->pair_tiled = tiled;
    TRY(pair_set_shape(c, k, block, c->tile_cap));
    TRY(dzero(c, c->pair_qctr, sizeof(unsigned long long)));   // the queue's grid may change
    invalidate_graph(c);
    return MFA_OK;
}

int mfa_set_pair_split(mfa_ctx* c, int32_t pieces) {
    if (!c || pieces < 1 || pieces > 64) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    c->pair_split = pieces;
    // the queue's ticket count per launch follows the number of pieces
    TRY(dzero(c, c->pair_qctr, sizeof(unsigned long long)));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    invalidate_graph(c);
    return MFA_OK;
}

int mfa_get_pair_split(mfa_ctx* c, int32_t* pieces) {
    if (!c || !pieces) return MFA_ERR_ARGS;
    *pieces = c->pair_split;
    return MFA_OK;
}

int mfa_set_pair_queue(mfa_ctx* c, int32_t ctas_per_sm) {
    if (!c || ctas_per_sm < 0 || ctas_per_sm > 64) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    c->pair_queue = ctas_per_sm;
    // a new grid changes the tickets a launch draws: restart the counter
    TRY(dzero(c, c->pair_qctr, sizeof(unsigned long long)));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    invalidate_graph(c);
    return MFA_OK;
}

int mfa_stream(mfa_ctx* c, void** s) {
    if (!c || !s) return MFA_ERR_ARGS;
    *s = (void*)c->st;
    return MFA_OK;
}

int mfa_sync(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    int32_t f[F_NFLAG];
    TRY(read_flags(c, f));
    MFA_CUDA_TRY(cudaGetLastError());
    return first_error(f[F_ERR]);
}

int mfa_download(mfa_ctx* c, uint32_t mask, double* r0, double* v, double* a, double* force, int32_t* mic) {
    if (!c) return MFA_ERR_ARGS;
    const int n = c->n;
    // x, y, z of one quantity are contiguous on the device: each quantity is
    // interleaved into the r0(3,n) layout in a stage slot of its own, then the
    // copies run back to back (one DMA stream from pinned memory), one
    // synchronisation
    double* dst3[3] = {(mask & MFA_R0) ? r0 : nullptr, (mask & MFA_V) ? v : nullptr, (mask & MFA_A) ? a : nullptr};
    const double* src3[3] = {c->rx, c->vx, c->ax};
    for (int k = 0; k < 3; ++k)
        if (dst3[k]) k_interleave3<<<(n + 255) / 256, 256, 0, c->st>>>(src3[k], c->d_stage + (size_t)3 * n * k, n);
    MFA_CUDA_TRY(cudaGetLastError());
    for (int k = 0; k < 3; ++k)
        if (dst3[k])
            MFA_CUDA_TRY(cudaMemcpyAsync(dst3[k], c->d_stage + (size_t)3 * n * k, (size_t)3 * n * 8,
                                         cudaMemcpyDeviceToHost, c->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    if ((mask & MFA_F) && force) {
        if (c->prec == MFA_MIXED) {
            std::vector<float> f4((size_t)4 * n);
            MFA_CUDA_TRY(cudaMemcpy(f4.data(), c->force, f4.size() * 4, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; ++i)
                for (int d = 0; d < 3; ++d) force[3 * i + d] = f4[4 * i + d];
        } else {
            std::vector<double> f4((size_t)4 * n);
            MFA_CUDA_TRY(cudaMemcpy(f4.data(), c->force, f4.size() * 8, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; ++i)
                for (int d = 0; d < 3; ++d) force[3 * i + d] = f4[4 * i + d];
        }
    }
    if ((mask & MFA_MIC) && mic) {
        std::vector<int32_t> m((size_t)3 * n);
        MFA_CUDA_TRY(cudaMemcpy(m.data(), c->mx, m.size() * 4, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) mic[3 * i + d] = m[(size_t)d * n + i];
    }
    return MFA_OK;
}

int mfa_upload(mfa_ctx* c, uint32_t mask, const double* r0, const double* v, const double* a,
               const double* force, const int32_t* mic) {
    if (!c) return MFA_ERR_ARGS;
    const int n = c->n;
    // the r0(3,n) layout copied as it is into a stage slot per quantity (the
    // copies back to back), then de-interleaved on the device; the copies and
    // kernels are stream-ordered, and the call returns once they are done (the
    // caller may reuse its buffers)
    const double* src3[3] = {(mask & MFA_R0) ? r0 : nullptr, (mask & MFA_V) ? v : nullptr, (mask & MFA_A) ? a : nullptr};
    double* dst3[3] = {c->rx, c->vx, c->ax};
    for (int k = 0; k < 3; ++k)
        if (src3[k])
            MFA_CUDA_TRY(cudaMemcpyAsync(c->d_stage + (size_t)3 * n * k, src3[k], (size_t)3 * n * 8,
                                         cudaMemcpyHostToDevice, c->st));
    for (int k = 0; k < 3; ++k)
        if (src3[k]) k_deinterleave3<<<(n + 255) / 256, 256, 0, c->st>>>(c->d_stage + (size_t)3 * n * k, dst3[k], n);
    MFA_CUDA_TRY(cudaGetLastError());
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    if ((mask & MFA_F) && force) {
        if (c->prec == MFA_MIXED) {
            std::vector<float> f4((size_t)4 * n, 0.0f);
            for (int i = 0; i < n; ++i)
                for (int d = 0; d < 3; ++d) f4[4 * i + d] = (float)force[3 * i + d];
            TRY(h2d(c, c->force, f4.data(), f4.size() * 4));
        } else {
            std::vector<double> f4((size_t)4 * n, 0.0);
            for (int i = 0; i < n; ++i)
                for (int d = 0; d < 3; ++d) f4[4 * i + d] = force[3 * i + d];
            TRY(h2d(c, c->force, f4.data(), f4.size() * 8));
        }
    }
    if ((mask & MFA_MIC) && mic) {
        std::vector<int32_t> m((size_t)3 * n);
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) m[(size_t)d * n + i] = mic[3 * i + d];
        TRY(h2d(c, c->mx, m.data(), m.size() * 4));
    }
    if (c->lists_valid && (mask & (MFA_R0 | MFA_V))) TRY(launch_refresh_sorted(c));
    return MFA_OK;
}

int mfa_debug_lists(mfa_ctx* c, int32_t* cell_of, int32_t* nbr_count, int32_t* nbr, int32_t max_per) {
    if (!c) return MFA_ERR_ARGS;
    if (!c->lists_valid) return MFA_ERR_STATE;
    const int n = c->n;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    const int nchunk = (n + 31) / 32;
    const size_t capc = (size_t)32 * c->maxnb;
    std::vector<int32_t> co(n), ids(n), cnt(n), ccnt(nchunk), lst(capc * nchunk), cs(c->ncell + 1);
    MFA_CUDA_TRY(cudaMemcpy(co.data(), c->cell_of, (size_t)n * 4, cudaMemcpyDeviceToHost));
    MFA_CUDA_TRY(cudaMemcpy(ids.data(), c->ids, (size_t)n * 4, cudaMemcpyDeviceToHost));
    MFA_CUDA_TRY(cudaMemcpy(cnt.data(), c->nnb, (size_t)n * 4, cudaMemcpyDeviceToHost));
    MFA_CUDA_TRY(cudaMemcpy(ccnt.data(), c->ccount, (size_t)nchunk * 4, cudaMemcpyDeviceToHost));
    MFA_CUDA_TRY(cudaMemcpy(lst.data(), c->nbr, lst.size() * 4, cudaMemcpyDeviceToHost));
    MFA_CUDA_TRY(cudaMemcpy(cs.data(), c->cell_start, cs.size() * 4, cudaMemcpyDeviceToHost));
    if (cell_of) memcpy(cell_of, co.data(), (size_t)n * 4);
    std::vector<int> fill(n, 0);
    for (int t = 0; t < n; ++t)
        if (nbr_count) nbr_count[ids[t]] = cnt[t];
    if (nbr)
        for (int ch = 0; ch < nchunk; ++ch)
            for (int k = 0; k < ccnt[ch]; ++k) {
                const int e = lst[ch * capc + k];
                const int t = ch * 32 + (e & 31), s = (int)((unsigned)e >> 5);   // owner slot, partner slot
                if (t >= n) continue;
                const int i = ids[t];
                if (fill[t] < max_per) nbr[(size_t)i * max_per + fill[t]] = (s >= 0 && s < n) ? ids[s] + 1 : 0;
                ++fill[t];
            }
    return MFA_OK;
}

int mfa_debug_kvecs(mfa_ctx* c, int32_t* nk, double* kvecs3, int32_t max_k) {
    if (!c || !nk) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    const int r = mfa_ewald_download_kvecs(c, kvecs3, max_k);
    if (r < 0) return MFA_ERR_CUDA;
    *nk = r;
    return MFA_OK;
}

}  // extern "C"
