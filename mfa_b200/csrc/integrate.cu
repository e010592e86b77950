// Velocity-Verlet integration (verlet_positions.f90, verlet_velocities.f90) and
// the skin check (check_skin.f90).  FP64 state, streamed once per call:
// thread per particle, SoA arrays, coalesced.  The FP64 arithmetic uses explicit
// round-to-nearest intrinsics so that no multiply-add is contracted and the
// update rounds exactly like the Fortran statement order.
#include "mfa_internal.cuh"
#include "bonded.cuh"

#include <string.h>

namespace {

struct VVArgs {
    double *rx, *ry, *rz, *vx, *vy, *vz, *ax, *ay, *az;
    const double *ox, *oy, *oz;
    int32_t *mx, *my, *mz;
    const int32_t* slot;
    const int32_t* type;
    const double* q;
    const double *mass, *inv_mass;
    int uniform_mass;             // every particle has mass umass (no per-particle loads)
    double umass, uinv_mass;
    void* pos_s;
    void* vel_s;
    void* force;
    int32_t* flags;
    int64_t* dstep;
    double* partials;
    unsigned* counter;
    double* dscal;
    double* elog;
    int32_t* elog_n;
    int elog_every, elog_cap;
    int max_blocks;
    int n;
    int symmetry;
    int write_sorted;
    int pin_heads, n_chain, n_mon;
    double* f_heads;              // force on each head before the pin (3 x n_chain), or null
    double L[3];
    double dt, skin_lim;
    double va[3];
    // conditional graph node that holds the next rebuild (0: none): the last
    // block opens it when the skin check tripped
    cudaGraphConditionalHandle rebuild_cond;
    // time-step fast path: the chains' FENE and bending forces are computed
    // here, bead by bead, and added to the force before a = F/m
    int fuse_bonds;
    BondParams bond;
    int fused_skin, zero_force;   // position half: skin check, force reset
    // a run of steps on the fast path: its first position half sets the step
    // whose energies are wanted to its last step (energy_span steps on), and
    // its last velocity half resets it to -1 (every step) afterwards (grouped
    // launches pass both as kernel parameters instead)
    long long energy_span;
    int energy_reset;
    // the energies of the pair launch before this one, left as block partials
    // (pair_nblk blocks, pair_nq quantities; 0: none): block 0 adds them up
    // into the pair's energy slots before it arrives at the grid reduction
    const double* pair_partials;
    int pair_nblk, pair_nq, pair_max_blocks;
};

// the pair kernel's deferred grid sum (see VVArgs), by block 0, uniform over
// the block; before the block's own arrival, so the last block sees it
__device__ __forceinline__ void reduce_pair_partials(const VVArgs& a, Blk blk, bool en) {
    if (!en || a.pair_nblk <= 0 || blk.id != 0) return;
    if (a.pair_nq == 4) reduce_partials<4>(a.pair_partials, a.pair_max_blocks, a.pair_nblk, a.dscal + S_VFF);
    else reduce_partials<3>(a.pair_partials, a.pair_max_blocks, a.pair_nblk, a.dscal + S_VFF);
}

// r += dt v + (0.5 dt^2) a ; v += (0.5 dt) a   (verlet_positions.f90:153,169)
__device__ __forceinline__ void drift_kick(double& r, double& v, double a, double dt, double hdt2, double hdt) {
    r = __dadd_rn(__dadd_rn(r, __dmul_rn(dt, v)), __dmul_rn(hdt2, a));
    v = __dadd_rn(v, __dmul_rn(hdt, a));
}

// verlet_positions.f90:237-251
__device__ __forceinline__ void wrap(double& r, int32_t& m, double L) {
    if (r > L) { r = __dsub_rn(r, L); m += 1; }
    else if (r < 0.0) { r = __dadd_rn(r, L); m -= 1; }
}

template <typename R4>
__device__ __forceinline__ void store_sorted(const VVArgs& a, int i, double x, double y, double z,
                                             double vx, double vy, double vz) {
    const int s = a.slot[i];
    R4* ps = (R4*)a.pos_s;
    R4* vs = (R4*)a.vel_s;
    R4 pw;
    pw.x = x; pw.y = y; pw.z = z;
    packw(pw, i, a.type[i]);
    ps[s] = pw;
    R4 vw;
    vw.x = vx; vw.y = vy; vw.z = vz; vw.w = a.q ? a.q[i] : 0.0;
    vs[s] = vw;
}

// check_skin.f90:8-21 on one particle; the snapshot (ox, oy, oz) holds
// r0_old + mic_old * L, the first sum of the reference's expression, rounded
// when the list was built
__device__ __forceinline__ bool skin_tripped(const VVArgs& a, int i, double x, double y, double z,
                                             int mx, int my, int mz) {
    double d0 = __dsub_rn(__dsub_rn(a.ox[i], x), __dmul_rn((double)mx, a.L[0]));
    double d1 = __dsub_rn(__dsub_rn(a.oy[i], y), __dmul_rn((double)my, a.L[1]));
    double d2 = __dsub_rn(__dsub_rn(a.oz[i], z), __dmul_rn((double)mz, a.L[2]));
    double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
    return r2 > a.skin_lim;
}

template <typename R4>
__device__ __forceinline__ void position_half(const VVArgs& a, int i, double x, double y, double z,
                                              double vx, double vy, double vz, double ax, double ay, double az,
                                              bool fused_skin) {
    const double dt = a.dt, hdt2 = 0.5 * (dt * dt), hdt = 0.5 * dt;
    drift_kick(x, vx, ax, dt, hdt2, hdt);
    drift_kick(y, vy, ay, dt, hdt2, hdt);
    drift_kick(z, vz, az, dt, hdt2, hdt);
    int32_t mx = a.mx[i], my = a.my[i], mz = a.mz[i];
    wrap(x, mx, a.L[0]);
    wrap(y, my, a.L[1]);
    if (a.symmetry == 1) wrap(z, mz, a.L[2]);
    a.rx[i] = x; a.ry[i] = y; a.rz[i] = z;
    a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
    a.mx[i] = mx; a.my[i] = my; a.mz[i] = mz;
    if (fused_skin && skin_tripped(a, i, x, y, z, mx, my, mz)) a.flags[F_SKIN] = 1;
    if (a.write_sorted) store_sorted<R4>(a, i, x, y, z, vx, vy, vz);
}

// zero_force: the fast path resets the force array here (md_main.f90:88), so
// that the force kernels of the step only ever add to it
template <typename R4>
__device__ __forceinline__ void vv_positions_body(const VVArgs& a, Blk blk, long long energy_span) {
    const int i = blk.id * blockDim.x + threadIdx.x;
    if (i == 0) {
        const long long st = a.dstep[0];
        if (energy_span > 0) a.dstep[1] = st + energy_span;
        a.dstep[0] = st + 1;
    }
    if (i >= a.n) return;
    position_half<R4>(a, i, a.rx[i], a.ry[i], a.rz[i], a.vx[i], a.vy[i], a.vz[i],
                      a.ax[i], a.ay[i], a.az[i], a.fused_skin != 0);
    if (a.zero_force) {
        R4 z4; z4.x = 0; z4.y = 0; z4.z = 0; z4.w = 0;
        ((R4*)a.force)[i] = z4;
    }
}

__global__ void k_check_skin(VVArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    if (skin_tripped(a, i, a.rx[i], a.ry[i], a.rz[i], a.mx[i], a.my[i], a.mz[i])) a.flags[F_SKIN] = 1;
}

// velocity half of verlet_velocities.f90:174-185 and the head rules :269-282,
// with fb the bonded force of bead i (intra_molec + bending(2),
// md_main.f90:106-111) when fuse_bonds.  Returns the kinetic contribution
// m v^2 of particle i.
template <typename R4>
__device__ __forceinline__ double velocity_half(const VVArgs& a, int i, double& vx, double& vy, double& vz,
                                                double& ax, double& ay, double& az,
                                                const decltype(R4::x) fb[3], bool store_force) {
    R4* f = (R4*)a.force;
    R4 fi = f[i];
    if (a.fuse_bonds) {
        fi.x += fb[0];
        fi.y += fb[1];
        fi.z += fb[2];
        if (store_force) f[i] = fi;
    }
    const double im = a.uniform_mass ? a.uinv_mass : a.inv_mass[i];
    const double hdt = 0.5 * a.dt;
    ax = __dmul_rn((double)fi.x, im);
    ay = __dmul_rn((double)fi.y, im);
    az = __dmul_rn((double)fi.z, im);
    vx = __dadd_rn(vx, __dmul_rn(hdt, ax));
    vy = __dadd_rn(vy, __dmul_rn(hdt, ay));
    vz = __dadd_rn(vz, __dmul_rn(hdt, az));
    if (a.pin_heads && i < a.n_chain * a.n_mon && (i % a.n_mon) == 0) {
        if (a.f_heads) {
            // f_on_heads(:,:) = force(:,1:part_init_d:n_mon) (verlet_velocities.f90:18)
            double* fh = a.f_heads + 3 * (size_t)(i / a.n_mon);
            fh[0] = (double)fi.x;
            fh[1] = (double)fi.y;
            fh[2] = (double)fi.z;
        }
        const double sg = (i / a.n_mon < a.n_chain / 2) ? 1.0 : -1.0;
        vx = sg * a.va[0];
        vy = sg * a.va[1];
        vz = 0.0;
        ax = ay = az = 0.0;
        R4 z4; z4.x = 0; z4.y = 0; z4.z = 0; z4.w = 0;
        f[i] = z4;
    }
    const double m = a.uniform_mass ? a.umass : a.mass[i];
    return __dmul_rn(m, __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz)));
}

__device__ __forceinline__ void finish_energies(const VVArgs& a) {
    // verlet_velocities.f90:155-198 (v_wall_wall = 0, t_wall = 0); the block
    // sums arrive in S_TMP0.. (kinetic, and FENE, bending when fused)
    double* s = a.dscal;
    s[S_TKIN] = 0.5 * s[S_TMP0];
    if (a.fuse_bonds) {
        s[S_VINTRA] = s[S_TMP0 + 1];
        s[S_VBEND] = s[S_TMP0 + 2];
    }
    s[S_VTOT] = (s[S_VFW] + s[S_VFF]) + s[S_VINTRA];
    s[S_ETOT] = s[S_VTOT] + s[S_TKIN];
    if (a.elog && a.elog_every > 0) {
        const long long st = *a.dstep;
        if (st % a.elog_every == 0) {
            const int k = *a.elog_n;
            if (k < a.elog_cap) {
                a.elog[4 * k + 0] = (double)st;
                a.elog[4 * k + 1] = s[S_ETOT];
                a.elog[4 * k + 2] = s[S_VTOT];
                a.elog[4 * k + 3] = s[S_TKIN];
                *a.elog_n = k + 1;
            }
        }
    }
}

// the FENE bonds at the clamp counted by the warp, and -- in the steps whose
// energies are wanted (en) -- the block sums of m v^2, FENE (times k_chain,
// intra_molec.f90:96,270) and bending energy; true in the last block
__device__ __forceinline__ bool vv_commit(const VVArgs& a, double ke, const double eb[2], int clamped, Blk blk,
                                          bool en) {
    for (int o = 16; o > 0; o >>= 1) clamped += __shfl_down_sync(0xffffffffu, clamped, o);
    if ((threadIdx.x & 31) == 0 && clamped) atomicAdd(&a.flags[F_FENE], clamped);
    if (!en) return block_arrive_last(a.counter, blk);
    double acc[3] = {ke, a.bond.k_chain * eb[0], eb[1]};
    return block_sum_commit<3>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_TMP0, blk);
}

template <typename R4>
__device__ __forceinline__ void vv_velocities_body(const VVArgs& a, Blk blk, int energy_reset) {
    const int i = blk.id * blockDim.x + threadIdx.x;
    reduce_pair_partials(a, blk, energy_needed(a.dstep, a.elog ? a.elog_every : 0));
    double ke = 0.0, eb[2] = {0.0, 0.0};
    int clamped = 0;
    // the bonded force first: its chain-window loads are in flight before the
    // force record is read (fewer registers live across them)
    decltype(R4::x) fb[3] = {0, 0, 0};
    if (i < a.n && a.fuse_bonds) bonded_on_bead(a.bond, i, fb, eb[0], eb[1], clamped);
    if (i < a.n) {
        double vx = a.vx[i], vy = a.vy[i], vz = a.vz[i], ax, ay, az;
        ke = velocity_half<R4>(a, i, vx, vy, vz, ax, ay, az, fb, true);
        a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
        a.ax[i] = ax; a.ay[i] = ay; a.az[i] = az;
    }
    const bool en = energy_needed(a.dstep, a.elog ? a.elog_every : 0);
    if (vv_commit(a, ke, eb, clamped, blk, en)) {
        if (threadIdx.x == 0) {
            if (en) finish_energies(a);
            if (energy_reset) a.dstep[1] = -1;   // every block has read it
        }
    }
}

// verlet_velocities of step n followed by verlet_positions of step n+1 in one
// pass over the state (the skin check of n+1 fused in); the force array is
// reset for the force kernels of step n+1 (md_main.f90:88).
// COND: the kernel may open the rebuild's conditional graph node (a kernel
// that can does not run under profilers that replay graph nodes one by one,
// so the launches without a node use the variant that cannot)
template <typename R4, bool COND>
__device__ __forceinline__ void vv_fused_body(const VVArgs& a, Blk blk) {
    const int i = blk.id * blockDim.x + threadIdx.x;
    reduce_pair_partials(a, blk, energy_needed(a.dstep, a.elog ? a.elog_every : 0));
    double ke = 0.0, eb[2] = {0.0, 0.0};
    int clamped = 0;
    decltype(R4::x) fb[3] = {0, 0, 0};
    if (i < a.n && a.fuse_bonds) bonded_on_bead(a.bond, i, fb, eb[0], eb[1], clamped);
    if (i < a.n) {
        double vx = a.vx[i], vy = a.vy[i], vz = a.vz[i], ax, ay, az;
        ke = velocity_half<R4>(a, i, vx, vy, vz, ax, ay, az, fb, false);
        R4 z4; z4.x = 0; z4.y = 0; z4.z = 0; z4.w = 0;
        ((R4*)a.force)[i] = z4;
        // a = F/m is used at once by the position half; the stored copy of a
        // is written by the velocity half that closes a run of steps
        position_half<R4>(a, i, a.rx[i], a.ry[i], a.rz[i], vx, vy, vz, ax, ay, az, true);
    }
    // every block reads the step before the last block advances it
    const bool en = energy_needed(a.dstep, a.elog ? a.elog_every : 0);
    if (vv_commit(a, ke, eb, clamped, blk, en)) {
        if (threadIdx.x == 0) {
            if (en) finish_energies(a);
            *a.dstep += 1;  // the next step has begun
            // every block's skin verdict is visible here (each fenced before
            // taking its turn on the counter).  Only a rebuild that is due
            // opens the node (the condition starts at 0 every graph launch),
            // so that several contexts may share one node.
            if (COND && a.rebuild_cond && *(volatile int32_t*)&a.flags[F_SKIN] != 0)
                cudaGraphSetConditional(a.rebuild_cond, 1u);
        }
    }
}

// plain launches (one context) and grouped launches (the same stage for
// several contexts, argument records in device memory)
template <typename R4>
__global__ void k_vv_positions(VVArgs a) { vv_positions_body<R4>(a, plain_blk(), a.energy_span); }
// 64 registers in MIXED: four 256-thread blocks per SM (the bonded window of
// the chain beads would otherwise take ~80; at 48 registers it spills, and the
// spills cost more than the extra wave: measured 58.3 vs 60.9 us per step);
// FP64 keeps 85 (three blocks), where 64 would spill the doubled operands
#define VV_BOUNDS __launch_bounds__(256, sizeof(R4) == 16 ? 4 : 3)
template <typename R4>
__global__ void VV_BOUNDS k_vv_velocities(VVArgs a) { vv_velocities_body<R4>(a, plain_blk(), a.energy_reset); }
template <typename R4>
__global__ void VV_BOUNDS k_vv_fused(VVArgs a) { vv_fused_body<R4, false>(a, plain_blk()); }
template <typename R4>
__global__ void VV_BOUNDS k_vv_fused_cond(VVArgs a) { vv_fused_body<R4, true>(a, plain_blk()); }
template <typename R4>
__global__ void VV_BOUNDS
    k_vv_grouped(const VVArgs* __restrict__ as, const int* __restrict__ off, int nsys, int stage,
                 long long energy_span, int energy_reset) {
    const int s = group_of(off, nsys, blockIdx.x);
    const Blk blk = group_blk(off, s);
    if (stage == VV_POSITIONS) vv_positions_body<R4>(as[s], blk, energy_span);
    else if (stage == VV_VELOCITIES) vv_velocities_body<R4>(as[s], blk, energy_reset);
    else vv_fused_body<R4, true>(as[s], blk);
}

VVArgs make_args(mfa_ctx* c) {
    VVArgs a;
    a.rx = c->rx; a.ry = c->ry; a.rz = c->rz;
    a.vx = c->vx; a.vy = c->vy; a.vz = c->vz;
    a.ax = c->ax; a.ay = c->ay; a.az = c->az;
    a.ox = c->ox; a.oy = c->oy; a.oz = c->oz;
    a.mx = c->mx; a.my = c->my; a.mz = c->mz;
    a.slot = c->slot; a.type = c->type; a.q = c->p.charged ? c->q : nullptr;
    a.mass = c->mass; a.inv_mass = c->inv_mass;
    a.uniform_mass = c->uniform_mass; a.umass = c->umass; a.uinv_mass = c->uinv_mass;
    a.pos_s = c->pos_s; a.vel_s = c->vel_s; a.force = c->force;
    a.flags = c->dflags; a.dstep = c->dstep;
    a.partials = c->partials + (size_t)R_VV * 4 * c->max_blocks;
    a.counter = c->counters + R_VV;
    a.dscal = c->dscal;
    a.elog = c->elog; a.elog_n = c->elog_n; a.elog_every = c->elog_every; a.elog_cap = c->elog_cap;
    a.max_blocks = c->max_blocks;
    a.n = c->n;
    a.symmetry = c->p.symmetry;
    a.write_sorted = c->lists_valid;
    a.pin_heads = c->p.pin_heads; a.n_chain = c->p.n_chain; a.n_mon = c->p.n_mon;
    a.f_heads = c->f_heads;
    for (int d = 0; d < 3; ++d) { a.L[d] = c->p.boundary[d]; a.va[d] = c->p.va_spring_twall[d]; }
    a.dt = c->p.dt;
    a.skin_lim = (c->p.skin / 2.0) * (c->p.skin / 2.0);
    a.rebuild_cond = 0;
    a.fuse_bonds = 0;
    a.bond = bond_params(c, 0, 0);
    a.fused_skin = 0;
    a.zero_force = 0;
    a.energy_span = 0;
    a.energy_reset = 0;
    a.pair_partials = c->partials + (size_t)R_PAIR * 4 * c->max_blocks;
    a.pair_nblk = 0;
    a.pair_nq = 3;
    a.pair_max_blocks = c->max_blocks;
    return a;
}

// the pair launch just before left its energy sum to this launch
void take_pair_sum(mfa_ctx* c, VVArgs& a) {
    a.pair_nblk = c->pair_sum_nblk;
    a.pair_nq = c->pair_sum_nq;
    c->pair_sum_nblk = 0;
}

constexpr int TPB = 256;

void set_bonds(const mfa_ctx* c, VVArgs& a, int fuse_bonds) {
    const bool chains = c->p.n_chain > 0 || (c->p.n_chain_d > 0 && c->p.n_mon_d >= 2);
    a.fuse_bonds = fuse_bonds && chains;
    a.bond = bond_params(c, a.fuse_bonds, a.fuse_bonds);
}

}  // namespace

int vv_stage_args(mfa_ctx* c, int stage, int fused_skin, int zero_force, int fuse_bonds,
                  cudaGraphConditionalHandle rebuild_cond, void* out, int* nblocks) {
    VVArgs a = make_args(c);
    a.fused_skin = fused_skin;
    a.zero_force = zero_force;
    a.rebuild_cond = rebuild_cond;
    set_bonds(c, a, fuse_bonds);
    const int nb = (c->n + TPB - 1) / TPB;
    if (stage != VV_POSITIONS && nb > c->max_blocks) return MFA_ERR_ARGS;
    memcpy(out, &a, sizeof(a));
    *nblocks = nb;
    return MFA_OK;
}

size_t vv_args_bytes() { return sizeof(VVArgs); }

int launch_vv_grouped(int prec, int stage, const void* dargs, const int* doff, int nsys, int nblocks,
                      cudaStream_t st, long long energy_span, int energy_reset) {
    const VVArgs* as = (const VVArgs*)dargs;
    if (prec == MFA_MIXED)
        k_vv_grouped<float4><<<nblocks, TPB, 0, st>>>(as, doff, nsys, stage, energy_span, energy_reset);
    else k_vv_grouped<double4><<<nblocks, TPB, 0, st>>>(as, doff, nsys, stage, energy_span, energy_reset);
    MFA_CUDA_TRY(cudaGetLastError());
    return MFA_OK;
}

// Opens the conditional node that holds the rebuild when the skin check of the
// position half before it tripped (the first step of a captured run).
__global__ void k_open_rebuild(const int32_t* flags, cudaGraphConditionalHandle h) {
    if (*(volatile const int32_t*)&flags[F_SKIN] != 0) cudaGraphSetConditional(h, 1u);
}

int launch_open_rebuild(mfa_ctx* c, cudaGraphConditionalHandle h) {
    k_open_rebuild<<<1, 1, 0, c->st>>>(c->dflags, h);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}

int launch_vv_positions(mfa_ctx* c, int fused_skin, int zero_force, long long energy_span) {
    VVArgs a;
    int nb;
    TRY_(vv_stage_args(c, VV_POSITIONS, fused_skin, zero_force, 0, 0, &a, &nb));
    a.energy_span = energy_span;
    if (c->prec == MFA_MIXED) k_vv_positions<float4><<<nb, TPB, 0, c->st>>>(a);
    else k_vv_positions<double4><<<nb, TPB, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}

int launch_check_skin(mfa_ctx* c) {
    VVArgs a = make_args(c);
    const int nb = (c->n + TPB - 1) / TPB;
    k_check_skin<<<nb, TPB, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}

// an integrator kernel on the context's stream
int launch_vv_kernel(mfa_ctx* c, void (*kernel)(VVArgs), int nb, const VVArgs& a) {
    kernel<<<nb, TPB, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}

int launch_vv_velocities(mfa_ctx* c, int fuse_bonds, int energy_reset) {
    VVArgs a;
    int nb;
    TRY_(vv_stage_args(c, VV_VELOCITIES, 0, 0, fuse_bonds, 0, &a, &nb));
    a.energy_reset = energy_reset;
    take_pair_sum(c, a);
    return launch_vv_kernel(c, c->prec == MFA_MIXED ? k_vv_velocities<float4> : k_vv_velocities<double4>, nb, a);
}

int launch_vv_fused(mfa_ctx* c, cudaGraphConditionalHandle rebuild_cond, int fuse_bonds) {
    VVArgs a;
    int nb;
    TRY_(vv_stage_args(c, VV_FUSED, 1, 1, fuse_bonds, rebuild_cond, &a, &nb));
    take_pair_sum(c, a);
    void (*k)(VVArgs);
    if (rebuild_cond) k = c->prec == MFA_MIXED ? k_vv_fused_cond<float4> : k_vv_fused_cond<double4>;
    else k = c->prec == MFA_MIXED ? k_vv_fused<float4> : k_vv_fused<double4>;
    return launch_vv_kernel(c, k, nb, a);
}
