// Many independent systems advanced together (mfa_batch_*).
//
// Each system keeps its own context (its own buffers, cell grid, lists, energy
// slots and error flags), exactly as mfa_init made it.  The argument records of
// the systems sit in device memory, and a table of block offsets per kernel
// stage maps each block of a stage to its system and to its block index there
// (group_of).  By default every kernel stage of a step is one grouped launch
// for all systems, captured as CUDA graphs, with the rebuild in a conditional
// node that any system whose skin check tripped opens; inside it every block
// returns at once unless its own system is due.  With MFA_BATCH_PERSIST=1 a
// run of steps of all systems is instead ONE persistent cooperative launch
// (persist.cu: every stage of every step as a grid-stride loop over those
// blocks, grid barriers between stages).  Measured on 64 uneven brushes
// (949k beads, B200): 0.574 ms per step persistent against 0.397 ms grouped --
// the persistent kernel runs its pair stage at four CTAs per SM instead of
// five, reads the argument records from device memory inside function calls
// that spill, and pays seven grid barriers per step -- so the grouped launches
// stay the default.
#include "mfa_internal.cuh"

#include <stdlib.h>
#include <string.h>
#include <vector>

struct mfa_batch {
    int nsys;
    std::vector<mfa_ctx*> ctx;
    int prec, dev;
    cudaStream_t st, st_body;
    int k, block, ft;             // pair kernel shape and feature set (the same for all systems)
    int fuse_wall;
    size_t pair_smem;             // largest dynamic shared memory over the systems
    // device tables: argument records and block offsets of every stage
    unsigned char* dargs;
    size_t dargs_cap;
    int* doff;
    size_t doff_cap;
    std::vector<unsigned char> hargs;
    std::vector<int> hoff;
    size_t o_pair, o_vvpos, o_vvvel, o_bin_first, o_bin_body, o_vvfused;   // byte offsets in dargs
    size_t f_pair, f_vv, f_bin;   // int offsets in doff (f_bin: 6 consecutive tables)
    int nb_pair, nb_vv, nb_bin[N_BIN_STAGES];   // total blocks of each stage
    size_t sz_pair, sz_vv, sz_bin;
    int n_fused_slots, next_fused_slot;
    std::vector<cudaGraphConditionalHandle> fused_handles;
    bool tables_ok;
    std::vector<const void*> key;  // what the tables depend on
    cudaGraphExec_t gexec[2];
    cudaGraph_t graph[2];
    int graph_kernels[2];
    long long launches;
    long long cap_count;
    int capturing;
    int* dnodes;                  // conditional rebuild nodes that opened (device counter)
    // the persistent launch: kernel (null: grouped launches), grid, dynamic
    // shared memory, barrier words, block offsets of its rebuild stages
    const void* persist_fn;
    int persist_grid;
    size_t persist_smem;
    unsigned* grid_bar;
    size_t f_binp;
};

// persist.cu
const void* persist_kernel(int prec, int ft);
size_t persist_args_bytes();
size_t persist_smem(int prec);
int persist_threads();
void persist_bin_blocks(const mfa_ctx* c, int nb[N_BIN_STAGES]);
void persist_args(const void* pair, const void* vvpos, const void* vvfused, const void* vvvel, const void* bin_first,
                  const void* bin_body, const int* off_pair, const int* off_vv, const int* off_bin, int nsys,
                  int nsteps, long long energy_span, unsigned* bar, int32_t* status, void* out);

namespace {

constexpr int BODY = 10;   // body steps per captured graph of kind 0 (kind 1: one)

int upload(mfa_batch* b) {
    if (b->hargs.size() > b->dargs_cap) {
        if (b->dargs) cudaFree(b->dargs);
        b->dargs = nullptr;
        if (cudaMalloc((void**)&b->dargs, b->hargs.size()) != cudaSuccess) return MFA_ERR_NOMEM;
        b->dargs_cap = b->hargs.size();
    }
    if (b->hoff.size() * sizeof(int) > b->doff_cap) {
        if (b->doff) cudaFree(b->doff);
        b->doff = nullptr;
        if (cudaMalloc((void**)&b->doff, b->hoff.size() * sizeof(int)) != cudaSuccess) return MFA_ERR_NOMEM;
        b->doff_cap = b->hoff.size() * sizeof(int);
    }
    MFA_CUDA_TRY(cudaMemcpyAsync(b->dargs, b->hargs.data(), b->hargs.size(), cudaMemcpyHostToDevice, b->st));
    MFA_CUDA_TRY(cudaMemcpyAsync(b->doff, b->hoff.data(), b->hoff.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 b->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(b->st));
    return MFA_OK;
}

void invalidate(mfa_batch* b) {
    for (int k = 0; k < 2; ++k) {
        if (b->gexec[k]) cudaGraphExecDestroy(b->gexec[k]);
        if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
        b->gexec[k] = nullptr;
        b->graph[k] = nullptr;
        b->graph_kernels[k] = 0;
    }
    b->tables_ok = false;
}

std::vector<const void*> current_key(const mfa_batch* b) {
    std::vector<const void*> k;
    for (mfa_ctx* c : b->ctx) {
        k.push_back(c->nbr);
        k.push_back(c->cell_count);
        k.push_back(c->partials);
        k.push_back(c->elog);
        k.push_back((const void*)(intptr_t)(c->maxnb * 4 + c->bin_type));
        k.push_back((const void*)(intptr_t)c->tile_cap);
        k.push_back((const void*)(intptr_t)(c->pair_tiled * 1000 + c->pair_tpp * 100 + c->pair_block / 32));
        k.push_back((const void*)(intptr_t)c->pair_split);
    }
    return k;
}

// Builds the argument records and block-offset tables of every stage (the
// integrator records of the captured body steps get their conditional node
// handles when those are created during capture).
int build_tables(mfa_batch* b) {
    const int n = b->nsys;
    b->sz_pair = pair_args_bytes();
    b->sz_vv = vv_args_bytes();
    b->sz_bin = bin_args_bytes();
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    b->o_pair = 0;
    b->o_vvpos = b->o_pair + al(n * b->sz_pair);
    b->o_vvvel = b->o_vvpos + al(n * b->sz_vv);
    b->o_bin_first = b->o_vvvel + al(n * b->sz_vv);
    b->o_bin_body = b->o_bin_first + al(n * b->sz_bin);
    b->o_vvfused = b->o_bin_body + al(n * b->sz_bin);
    b->n_fused_slots = BODY + 1;
    b->hargs.assign(b->o_vvfused + (size_t)b->n_fused_slots * al(n * b->sz_vv), 0);
    b->f_pair = 0;
    b->f_vv = n + 1;
    b->f_bin = 2 * (n + 1);
    b->f_binp = (2 + N_BIN_STAGES) * (size_t)(n + 1);
    b->hoff.assign((2 + 2 * N_BIN_STAGES) * (size_t)(n + 1), 0);
    // one pair-kernel shape for all systems (the batch's), set before the
    // records are made; whole chunk lists (the systems together fill the GPU);
    // the persistent kernel's pair stage is untiled without a work queue
    for (mfa_ctx* c : b->ctx) {
        if (b->persist_fn) {
            c->pair_tiled = 0;
            c->pair_queue = 0;
        }
        TRY_(pair_set_shape(c, b->k, b->block, c->tile_cap));
        c->pair_split = 1;
    }
    int nbp_total[N_BIN_STAGES] = {0, 0, 0, 0, 0, 0};
    b->pair_smem = 0;
    b->nb_pair = b->nb_vv = 0;
    for (int s = 0; s < N_BIN_STAGES; ++s) b->nb_bin[s] = 0;
    for (int i = 0; i < n; ++i) {
        mfa_ctx* c = b->ctx[i];
        int grid, ft, nb;
        size_t smem;
        TRY_(pair_stage_args(c, b->fuse_wall, &b->hargs[b->o_pair + i * b->sz_pair], &grid, &smem, &ft));
        if (ft != b->ft) return MFA_ERR_UNSUPPORTED;
        b->hoff[b->f_pair + i] = b->nb_pair;
        b->nb_pair += grid;
        if (smem > b->pair_smem) b->pair_smem = smem;
        TRY_(vv_stage_args(c, VV_POSITIONS, 1, 1, 1, 0, &b->hargs[b->o_vvpos + i * b->sz_vv], &nb));
        TRY_(vv_stage_args(c, VV_VELOCITIES, 0, 0, 1, 0, &b->hargs[b->o_vvvel + i * b->sz_vv], &nb));
        for (int f = 0; f < b->n_fused_slots; ++f)
            TRY_(vv_stage_args(c, VV_FUSED, 1, 1, 1, 0, &b->hargs[b->o_vvfused + f * al(n * b->sz_vv) + i * b->sz_vv],
                               &nb));
        b->hoff[b->f_vv + i] = b->nb_vv;
        b->nb_vv += nb;
        int nbs[N_BIN_STAGES];
        TRY_(bin_stage_args(c, c->bin_type, 1, 0, &b->hargs[b->o_bin_first + i * b->sz_bin], nbs));
        TRY_(bin_stage_args(c, c->bin_type, 1, 1, &b->hargs[b->o_bin_body + i * b->sz_bin], nbs));
        for (int s = 0; s < N_BIN_STAGES; ++s) {
            b->hoff[b->f_bin + s * (n + 1) + i] = b->nb_bin[s];
            b->nb_bin[s] += nbs[s];
        }
        // the persistent kernel's rebuild stages run with its own CTA size
        int nbp[N_BIN_STAGES];
        persist_bin_blocks(c, nbp);
        for (int s = 0; s < N_BIN_STAGES; ++s) {
            b->hoff[b->f_binp + s * (n + 1) + i] = nbp_total[s];
            nbp_total[s] += nbp[s];
        }
    }
    b->hoff[b->f_pair + n] = b->nb_pair;
    b->hoff[b->f_vv + n] = b->nb_vv;
    for (int s = 0; s < N_BIN_STAGES; ++s) b->hoff[b->f_bin + s * (n + 1) + n] = b->nb_bin[s];
    for (int s = 0; s < N_BIN_STAGES; ++s) b->hoff[b->f_binp + s * (n + 1) + n] = nbp_total[s];
    b->next_fused_slot = 0;
    TRY_(upload(b));
    b->tables_ok = true;
    return MFA_OK;
}

void note(mfa_batch* b, int k) {
    if (b->capturing) b->cap_count += k;
    else b->launches += k;
}

const void* vvfused_slot(mfa_batch* b, int slot) {
    const size_t stride = (b->nsys * b->sz_vv + 255) / 256 * 256;
    return b->dargs + b->o_vvfused + slot * stride;
}

int stage_pair(mfa_batch* b) {
    TRY_(launch_pair_grouped(b->prec, b->k, b->block, b->ft, b->dargs + b->o_pair, b->doff + b->f_pair, b->nsys,
                             b->nb_pair, b->pair_smem, b->st));
    note(b, 1);
    return MFA_OK;
}

int stage_rebuild(mfa_batch* b, size_t o_args, cudaStream_t st, bool in_node) {
    for (int s = 0; s < N_BIN_STAGES; ++s)
        TRY_(launch_bin_grouped(b->prec, s, b->dargs + o_args, b->doff + b->f_bin + s * (b->nsys + 1), b->nsys,
                                b->nb_bin[s], st, in_node ? b->dnodes : nullptr));
    if (!in_node) note(b, N_BIN_STAGES);
    return MFA_OK;
}

// forces of step n, integrator (velocities of n, positions of n+1; opens the
// rebuild node if any system needs one), the rebuild of n+1 in that node
int capture_body_step(mfa_batch* b) {
    TRY_(stage_pair(b));
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    MFA_CUDA_TRY(cudaStreamGetCaptureInfo(b->st, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return MFA_ERR_STATE;
    cudaGraphConditionalHandle h;
    MFA_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    if (b->next_fused_slot >= b->n_fused_slots) return MFA_ERR_STATE;
    const int slot = b->next_fused_slot++;
    b->fused_handles[slot] = h;
    TRY_(launch_vv_grouped(b->prec, VV_FUSED, vvfused_slot(b, slot), b->doff + b->f_vv, b->nsys, b->nb_vv, b->st));
    note(b, 1);
    MFA_CUDA_TRY(cudaStreamGetCaptureInfo(b->st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    MFA_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    MFA_CUDA_TRY(cudaStreamBeginCaptureToGraph(b->st_body, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
    const int rc = stage_rebuild(b, b->o_bin_body, b->st_body, true);
    cudaGraph_t out;
    const cudaError_t e = cudaStreamEndCapture(b->st_body, &out);
    if (rc != MFA_OK) return rc;
    MFA_CUDA_TRY(e);
    MFA_CUDA_TRY(cudaStreamUpdateCaptureDependencies(b->st, &node, 1, cudaStreamSetCaptureDependencies));
    return MFA_OK;
}

int capture(mfa_batch* b, int kind) {
    const int first_slot = b->next_fused_slot;
    cudaGraph_t g;
    MFA_CUDA_TRY(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    b->capturing = 1;
    b->cap_count = 0;
    int rc = MFA_OK;
    for (int s = 0; s < (kind == 0 ? BODY : 1) && rc == MFA_OK; ++s) rc = capture_body_step(b);
    b->capturing = 0;
    cudaError_t e = cudaStreamEndCapture(b->st, &g);
    if (rc != MFA_OK) return rc;
    MFA_CUDA_TRY(e);
    // the integrator records of this graph now carry their node handles
    for (int slot = first_slot; slot < b->next_fused_slot; ++slot) {
        const size_t stride = (b->nsys * b->sz_vv + 255) / 256 * 256;
        for (int i = 0; i < b->nsys; ++i) {
            unsigned char* rec = &b->hargs[b->o_vvfused + slot * stride + i * b->sz_vv];
            int nb;
            TRY_(vv_stage_args(b->ctx[i], VV_FUSED, 1, 1, 1, b->fused_handles[slot], rec, &nb));
        }
    }
    TRY_(upload(b));
    MFA_CUDA_TRY(cudaGraphInstantiate(&b->gexec[kind], g, 0));
    b->graph[kind] = g;
    b->graph_kernels[kind] = (int)b->cap_count;
    return MFA_OK;
}

// A whole run of nsteps steps of every system as one cooperative launch.
int run_persistent(mfa_batch* b, int nsteps) {
    if (b->persist_grid == 0) {
        int per_sm = 0, n_sm = 0;
        MFA_CUDA_TRY(cudaFuncSetAttribute(b->persist_fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)b->persist_smem));
        MFA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->persist_fn, persist_threads(),
                                                                   b->persist_smem));
        MFA_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, b->dev));
        if (per_sm < 1) return MFA_ERR_UNSUPPORTED;
        b->persist_grid = per_sm * n_sm;
    }
    std::vector<unsigned char> rec(persist_args_bytes());
    persist_args(b->dargs + b->o_pair, b->dargs + b->o_vvpos, vvfused_slot(b, 0), b->dargs + b->o_vvvel,
                 b->dargs + b->o_bin_first, b->dargs + b->o_bin_body, b->doff + b->f_pair, b->doff + b->f_vv,
                 b->doff + b->f_binp, b->nsys, nsteps, nsteps, b->grid_bar, b->ctx[0]->dflags, rec.data());
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)b->persist_grid);
    cfg.blockDim = dim3((unsigned)persist_threads());
    cfg.dynamicSmemBytes = b->persist_smem;
    cfg.stream = b->st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    void* argv[] = {rec.data()};
    MFA_CUDA_TRY(cudaLaunchKernelExC(&cfg, b->persist_fn, argv));
    note(b, 1);
    return MFA_OK;
}

int replay(mfa_batch* b, int kind) {
    if (!b->gexec[kind]) TRY_(capture(b, kind));
    MFA_CUDA_TRY(cudaGraphLaunch(b->gexec[kind], b->st));
    b->launches += b->graph_kernels[kind];
    return MFA_OK;
}

}  // namespace

extern "C" {

int mfa_batch_create(mfa_ctx* const* ctxs, int32_t n, mfa_batch** out) {
    if (!ctxs || n < 1 || !out) return MFA_ERR_ARGS;
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        mfa_ctx* c = ctxs[i];
        if (!c) return MFA_ERR_ARGS;
        if (c->dev != ctxs[0]->dev || c->prec != ctxs[0]->prec) return MFA_ERR_UNSUPPORTED;
        // Ewald k-space and the hard walls of WALL 3/4 are not batched
        if (c->p.charged || c->p.wall == 3 || c->p.wall == 4 || c->dpd_vv) return MFA_ERR_UNSUPPORTED;
        if (c->p.symmetry != ctxs[0]->p.symmetry || c->p.thermostat != ctxs[0]->p.thermostat ||
            c->p.force_switch_on != ctxs[0]->p.force_switch_on || c->p.wall != ctxs[0]->p.wall)
            return MFA_ERR_UNSUPPORTED;
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == c) return MFA_ERR_ARGS;
    }
    MFA_CUDA_TRY(cudaSetDevice(ctxs[0]->dev));
    mfa_batch* b = new mfa_batch();
    b->nsys = n;
    b->ctx.assign(ctxs, ctxs + n);
    b->prec = ctxs[0]->prec;
    b->dev = ctxs[0]->dev;
    b->k = ctxs[0]->pair_tpp;
    b->block = ctxs[0]->pair_block;
    b->fuse_wall = ctxs[0]->p.symmetry == 0;
    b->ft = -1;
    b->fused_handles.assign(BODY + 1, 0);
    b->persist_fn = nullptr;
    b->persist_grid = 0;
    b->persist_smem = 0;
    b->grid_bar = nullptr;
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->st_body, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void**)&b->dnodes, sizeof(int)) != cudaSuccess) {
        mfa_batch_destroy(b);
        return MFA_ERR_CUDA;
    }
    if (cudaMemsetAsync(b->dnodes, 0, sizeof(int), b->st) != cudaSuccess ||
        cudaStreamSynchronize(b->st) != cudaSuccess) {
        mfa_batch_destroy(b);
        return MFA_ERR_CUDA;
    }
    // the feature set of the first system is the batch's
    {
        std::vector<unsigned char> tmp(pair_args_bytes());
        int grid, ft;
        size_t smem;
        for (mfa_ctx* c : b->ctx) {
            cudaStreamSynchronize(c->st);
            if (!c->lists_valid) {
                const int rc = mfa_binning(c);
                if (rc != MFA_OK) { mfa_batch_destroy(b); return rc; }
            }
            const int rc = pair_stage_args(c, b->fuse_wall, tmp.data(), &grid, &smem, &ft);
            if (rc != MFA_OK) { mfa_batch_destroy(b); return rc; }
            if (b->ft < 0) b->ft = ft;
            else if (ft != b->ft) { mfa_batch_destroy(b); return MFA_ERR_UNSUPPORTED; }
        }
    }
    // the persistent launch with MFA_BATCH_PERSIST=1, where the device has
    // cooperative launches and the feature set a persistent kernel
    {
        const char* e = getenv("MFA_BATCH_PERSIST");
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->dev);
        const void* fn = persist_kernel(b->prec, b->ft);
        if (e && e[0] == '1' && coop && fn &&
            cudaMalloc((void**)&b->grid_bar, GB_WORDS * sizeof(unsigned)) == cudaSuccess &&
            cudaMemsetAsync(b->grid_bar, 0, GB_WORDS * sizeof(unsigned), b->st) == cudaSuccess &&
            cudaStreamSynchronize(b->st) == cudaSuccess) {
            b->persist_fn = fn;
            b->persist_smem = persist_smem(b->prec);
            b->k = 2;
            b->block = persist_threads();
        }
        cudaGetLastError();
    }
    *out = b;
    return MFA_OK;
}

int mfa_batch_destroy(mfa_batch* b) {
    if (!b) return MFA_ERR_ARGS;
    if (b->st) cudaStreamSynchronize(b->st);
    invalidate(b);
    if (b->dargs) cudaFree(b->dargs);
    if (b->doff) cudaFree(b->doff);
    if (b->dnodes) cudaFree(b->dnodes);
    if (b->grid_bar) cudaFree(b->grid_bar);
    if (b->st) cudaStreamDestroy(b->st);
    if (b->st_body) cudaStreamDestroy(b->st_body);
    delete b;
    return MFA_OK;
}

int mfa_batch_step(mfa_batch* b, int32_t nsteps) {
    if (!b || nsteps < 0) return MFA_ERR_ARGS;
    if (nsteps == 0) return MFA_OK;
    // work the contexts queued on their own streams comes first
    for (mfa_ctx* c : b->ctx) {
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
        if (!c->lists_valid) TRY_(mfa_binning(c));
    }
    const std::vector<const void*> key = current_key(b);
    if (!b->tables_ok || key != b->key) {
        invalidate(b);
        TRY_(build_tables(b));
        b->key = current_key(b);
    }
    if (b->persist_fn) {
        TRY_(run_persistent(b, nsteps));
        for (mfa_ctx* c : b->ctx) c->i_time += nsteps;
        return MFA_OK;
    }
    // first step: positions (+ skin check, force reset; every system reduces
    // its energies on the last step of the run only, and on the steps its
    // energy log records), rebuild of the systems due
    TRY_(launch_vv_grouped(b->prec, VV_POSITIONS, b->dargs + b->o_vvpos, b->doff + b->f_vv, b->nsys, b->nb_vv,
                           b->st, nsteps));
    note(b, 1);
    TRY_(stage_rebuild(b, b->o_bin_first, b->st, false));
    int body = nsteps - 1;
    while (body >= BODY) {
        TRY_(replay(b, 0));
        body -= BODY;
    }
    while (body > 0) {
        TRY_(replay(b, 1));
        --body;
    }
    // last step: forces (chains' bonds in the integrator) and the velocity half
    TRY_(stage_pair(b));
    TRY_(launch_vv_grouped(b->prec, VV_VELOCITIES, b->dargs + b->o_vvvel, b->doff + b->f_vv, b->nsys, b->nb_vv,
                           b->st, 0, 1));
    note(b, 1);
    for (mfa_ctx* c : b->ctx) c->i_time += nsteps;
    return MFA_OK;
}

int mfa_batch_sync(mfa_batch* b) {
    if (!b) return MFA_ERR_ARGS;
    MFA_CUDA_TRY(cudaStreamSynchronize(b->st));
    MFA_CUDA_TRY(cudaGetLastError());
    return MFA_OK;
}

int mfa_batch_stream(mfa_batch* b, void** stream) {
    if (!b || !stream) return MFA_ERR_ARGS;
    *stream = (void*)b->st;
    return MFA_OK;
}

int mfa_batch_launches(mfa_batch* b, int64_t* launches) {
    if (!b || !launches) return MFA_ERR_ARGS;
    int opened = 0;
    MFA_CUDA_TRY(cudaMemcpyAsync(&opened, b->dnodes, sizeof(int), cudaMemcpyDeviceToHost, b->st));
    MFA_CUDA_TRY(cudaStreamSynchronize(b->st));
    *launches = b->launches + (int64_t)N_BIN_STAGES * opened;
    return MFA_OK;
}

}  // extern "C"
