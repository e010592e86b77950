// Optional force terms that the reference compiles in behind cpp switches:
//   external_force.f90 (EXT_FORCE 1): an elastic pull of every bead to the
//       axis y = Ly/2, z = Lz/2 (md_main.f90:122-124);
//   orientation.f90 (ORIENTATION): an angle term on the first bond of every
//       grafted chain, mode 1 (SYMMETRY 0, md_main.f90:119) and mode 2 (the
//       first and last bond against the x axis, as compiled with CHAIN_BC 2);
//   new_dpd_fd.f90 (DPD_VV): the dissipative force re-evaluated with the
//       velocities after verlet_velocities, then a half kick with the
//       corrected force and the step's energies (md_main.f90:149-155).
// All three are thread-per-item passes over the resident FP64 state.  The file
// is compiled with -fmad=false, so that every FP64 operation rounds on its own
// in the order of the Fortran statements and the FP64 path reproduces the
// serial FP64 evaluation to rounding.
#include "mfa_internal.cuh"

namespace {

constexpr int TPB = 256;
constexpr int R_TERMS = 6;   // reduction counter / partials region of this file

// device scratch of this file (ctx->term_buf): [0] v_or of the last
// orientation call, [1] the kinetic sum of the last new_dpd_fd
int term_buf(mfa_ctx* c) {
    if (!c->term_buf) MFA_CUDA_TRY(cudaMalloc((void**)&c->term_buf, 8 * sizeof(double)));
    return MFA_OK;
}

// ---------------- external_force.f90:14-17 ----------------

template <typename R4>
__global__ void k_external_force(R4* __restrict__ f, const double* __restrict__ ry, const double* __restrict__ rz,
                                 int n, double k, double hy, double hz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    using R = decltype(R4::x);
    R4 fi = f[i];
    fi.y = (R)((double)fi.y - k * (ry[i] - hy));
    fi.z = (R)((double)fi.z - k * (rz[i] - hz));
    f[i] = fi;
}

// ---------------- orientation.f90 ----------------

struct OrientArgs {
    void* force;
    const double *rx, *ry, *rz;
    double L[3], invL[3];
    int n_chain, n_mon, mode, max_blocks;
    double k_or, alpha_or;
    double* partials;
    unsigned* counter;
    double* out;   // v_or
};

// cos of the angle between rp and rn, and the unit direction of the force on
// the far end of rn (dn) and, when want_dp, of rp (dp), zeroed below `small`
// (orientation.f90:50-75, :132-151); returns the angle change acos - alpha_or
__device__ double angle_dirs(const double rp[3], const double rn[3], double small, bool want_dp, double alpha_or,
                             double dn[3], double dp[3]) {
    double dot = 0.0, rp2 = 0.0, rn2 = 0.0;
    for (int j = 0; j < 3; ++j) {
        dot = dot + rn[j] * rp[j];
        rp2 = rp2 + rp[j] * rp[j];
        rn2 = rn2 + rn[j] * rn[j];
    }
    const double cosa = dot / sqrt(rp2 * rn2);
    double dn2 = 0.0, dp2 = 0.0;
    for (int j = 0; j < 3; ++j) {
        dn[j] = rp[j] * rn2 - rn[j] * dot;
        dp[j] = want_dp ? -rn[j] * rp2 + rp[j] * dot : 0.0;
    }
    for (int j = 0; j < 3; ++j) {
        dp2 = dp2 + dp[j] * dp[j];
        dn2 = dn2 + dn[j] * dn[j];
    }
    if (dn2 < small) {
        for (int j = 0; j < 3; ++j) dn[j] = dn[j] * 0.0;
    } else {
        const double den = sqrt(dn2 * rn2);
        for (int j = 0; j < 3; ++j) dn[j] = dn[j] / den;
    }
    if (want_dp) {
        if (dp2 < small) {
            for (int j = 0; j < 3; ++j) dp[j] = dp[j] * 0.0;
        } else {
            const double den = sqrt(dp2 * rp2);
            for (int j = 0; j < 3; ++j) dp[j] = dp[j] / den;
        }
    }
    return acos(cosa) - alpha_or;
}

// force(:, i) += sgn * v(:) on one 4-wide record
template <typename R4>
__device__ __forceinline__ void add_to(R4* f, int i, const double v[3], double sgn) {
    using R = decltype(R4::x);
    R4 fi = f[i];
    fi.x = (R)((double)fi.x + sgn * v[0]);
    fi.y = (R)((double)fi.y + sgn * v[1]);
    fi.z = (R)((double)fi.z + sgn * v[2]);
    f[i] = fi;
}

// one thread per chain: a chain's beads are written by its thread only
template <typename R4>
__global__ void k_orientation(OrientArgs a) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    double vor = 0.0;
    if (l < a.n_chain) {
        R4* f = (R4*)a.force;
        const int h = l * a.n_mon;
        if (a.mode == 1) {
            // :34-48: ghost bond from the head one unit away from the mid-plane
            const double hx = a.rx[h], hy = a.ry[h], hz = a.rz[h];
            const double gz = hz > a.L[2] / 2.0 ? hz + 1.0 : hz - 1.0;
            double rp[3] = {hx - hx, hy - hy, hz - gz};
            double rn[3] = {a.rx[h + 1] - hx, a.ry[h + 1] - hy, a.rz[h + 1] - hz};
            for (int j = 0; j < 2; ++j) {
                rn[j] = mimage64(rn[j], a.L[j], a.invL[j]);
                rp[j] = mimage64(rp[j], a.L[j], a.invL[j]);
            }
            double dn[3], dp[3];
            // 0.0001 is a default-REAL literal (orientation.f90:67)
            const double da = angle_dirs(rp, rn, (double)0.0001f, false, a.alpha_or, dn, dp);
            const double fm = a.k_or * da;
            vor = 0.5 * fm * da;
            double fv[3];
            for (int j = 0; j < 3; ++j) fv[j] = fm * dn[j];
            add_to(f, h, fv, -1.0);
            add_to(f, h + 1, fv, 1.0);
        } else {
            // :89-175 with CHAIN_BC 2: the far ends held along x
            const int last = h + a.n_mon - 1;
            for (int b = 1; b <= 2; ++b) {
                double rp[3], rn[3];
                if (b == 1) {
                    rp[0] = 1.0; rp[1] = 0.0; rp[2] = 0.0;
                    rn[0] = a.rx[h + 1] - a.rx[h];
                    rn[1] = a.ry[h + 1] - a.ry[h];
                    rn[2] = a.rz[h + 1] - a.rz[h];
                } else {
                    rp[0] = a.rx[last] - a.rx[last - 1];
                    rp[1] = a.ry[last] - a.ry[last - 1];
                    rp[2] = a.rz[last] - a.rz[last - 1];
                    rn[0] = 1.0; rn[1] = 0.0; rn[2] = 0.0;
                }
                for (int j = 0; j < 3; ++j) {
                    rn[j] = mimage64(rn[j], a.L[j], a.invL[j]);
                    rp[j] = mimage64(rp[j], a.L[j], a.invL[j]);
                }
                double dn[3], dp[3];
                const double da = angle_dirs(rp, rn, (double)0.000001f, true, a.alpha_or, dn, dp);
                const double fm = a.k_or * da;
                vor = vor + 0.5 * fm * da;
                double fb[3], fb3[3];
                for (int j = 0; j < 3; ++j) { fb[j] = fm * dp[j]; fb3[j] = fm * dn[j]; }
                // :155-172 in statement order: far end, middle bead (- fb - fb3), near end
                const int i0 = b == 1 ? last : last - 1, i1 = b == 1 ? h : last, i2 = b == 1 ? h + 1 : h;
                add_to(f, i0, fb, 1.0);
                {
                    using R = decltype(R4::x);
                    R4 fi = f[i1];
                    fi.x = (R)(((double)fi.x - fb[0]) - fb3[0]);
                    fi.y = (R)(((double)fi.y - fb[1]) - fb3[1]);
                    fi.z = (R)(((double)fi.z - fb[2]) - fb3[2]);
                    f[i1] = fi;
                }
                add_to(f, i2, fb3, 1.0);
            }
        }
    }
    double acc[1] = {vor};
    block_sum_commit<1>(acc, a.partials, a.max_blocks, a.counter, a.out);
}

// ---------------- new_dpd_fd.f90 ----------------

// :27-84 over the Verlet list (one warp per 32-slot chunk, lanes over its
// entries): Fd of every listed pair inside range_2, heads excluded, x and y
// minimum-imaged only; added to fdn (zero on entry) with atomics
struct DpdFdArgs {
    const int32_t* __restrict__ nbr;
    const int32_t* __restrict__ ccount;
    const int32_t* __restrict__ ids;
    const int32_t* __restrict__ type;
    const double *rx, *ry, *rz, *vx, *vy, *vz;
    const double* __restrict__ range_2;   // T8 x T8
    double* fdn;                          // 3 x n
    int n, maxnb, dpd_weight;
    double L[2], invL[2];
    double friction;
};

__global__ void k_dpd_fd(DpdFdArgs a) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int ch = gt >> 5, lane = gt & 31;
    if (ch * 32 >= a.n) return;
    const int cnt = a.ccount[ch];
    const int32_t* crow = a.nbr + (size_t)ch * 32 * a.maxnb;
    for (int e = lane; e < cnt; e += 32) {
        const int ent = crow[e];
        const int t = ch * 32 + (ent & 31), s = (int)((unsigned)ent >> 5);
        if (t >= a.n || s >= a.n) continue;
        const int i = a.ids[t], j = a.ids[s];
        const int ti = a.type[i], tj = a.type[j];
        if (ti == 1 || tj == 1) continue;
        double dr[3] = {a.rx[i] - a.rx[j], a.ry[i] - a.ry[j], a.rz[i] - a.rz[j]};
        dr[0] = mimage64(dr[0], a.L[0], a.invL[0]);
        dr[1] = mimage64(dr[1], a.L[1], a.invL[1]);
        const double r2 = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
        const double rr = __ldg(&a.range_2[(ti - 1) * T8 + (tj - 1)]);
        if (!(r2 < rr)) continue;
        double wd = 1.0;
        if (a.dpd_weight == 0) {
            const double u = 1.0 - sqrt(r2 / rr);
            wd = u * u;
        }
        const double rs = sqrt(r2);
        const double rv[3] = {dr[0] / rs, dr[1] / rs, dr[2] / rs};
        const double dv[3] = {a.vx[i] - a.vx[j], a.vy[i] - a.vy[j], a.vz[i] - a.vz[j]};
        const double rd = (dv[0] * rv[0] + dv[1] * rv[1]) + dv[2] * rv[2];
        const double g = -1.0 * a.friction * wd * rd;
        for (int d = 0; d < 3; ++d) {
            const double fv = g * rv[d];
            atomicAdd(&a.fdn[(size_t)d * a.n + i], fv);
            atomicAdd(&a.fdn[(size_t)d * a.n + j], -fv);
        }
    }
}

struct VVTermArgs {
    void* force;
    double *vx, *vy, *vz, *ax, *ay, *az;
    const double *mass, *inv_mass;
    double* fdp;   // 3 x n: Fd of the previous new_dpd_fd (taken out, then replaced)
    double* fdn;   // 3 x n: Fd of this call (reset to zero for the next)
    double* partials;
    unsigned* counter;
    double* tbuf;
    double* dscal;
    int n, max_blocks;
    double dt;
};

// :17 and :88 (force - Fd_old + Fd_new), :92-104 (half kick with the corrected
// force, a = F/m), :124-160 (kinetic and total energies, t_wall = 0, v_wall_wall = 0)
template <typename R4>
__global__ void k_dpd_vv_finish(VVTermArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0;
    if (i < a.n) {
        using R = decltype(R4::x);
        R4* f = (R4*)a.force;
        R4 fi = f[i];
        const size_t n = a.n;
        fi.x = (R)(((double)fi.x - a.fdp[i]) + a.fdn[i]);
        fi.y = (R)(((double)fi.y - a.fdp[n + i]) + a.fdn[n + i]);
        fi.z = (R)(((double)fi.z - a.fdp[2 * n + i]) + a.fdn[2 * n + i]);
        f[i] = fi;
        for (int d = 0; d < 3; ++d) {
            a.fdp[d * n + i] = a.fdn[d * n + i];
            a.fdn[d * n + i] = 0.0;
        }
        const double fx = (double)fi.x, fy = (double)fi.y, fz = (double)fi.z;
        const double im = a.inv_mass[i], hdt = 0.5 * a.dt;
        const double vx = a.vx[i] + hdt * fx * im;
        const double vy = a.vy[i] + hdt * fy * im;
        const double vz = a.vz[i] + hdt * fz * im;
        a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
        a.ax[i] = fx * im; a.ay[i] = fy * im; a.az[i] = fz * im;
        const double m = a.mass[i];
        ke = (m * (vx * vx) + m * (vy * vy)) + m * (vz * vz);
    }
    double acc[1] = {ke};
    if (block_sum_commit<1>(acc, a.partials, a.max_blocks, a.counter, a.tbuf + 1) && threadIdx.x == 0) {
        double* s = a.dscal;
        s[S_TKIN] = a.tbuf[1] / 2.0;
        s[S_VTOT] = (s[S_VFW] + s[S_VFF]) + s[S_VINTRA];
        s[S_ETOT] = s[S_VTOT] + s[S_TKIN];
    }
}

// verlet_velocities.f90:23-35 alone (DPD_VV compiles out :79-230: head
// rules and energies): a = F/m, v += (dt/2) a
template <typename R4>
__global__ void k_dpd_vv_kick(VVTermArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const R4 fi = ((const R4*)a.force)[i];
    const double im = a.inv_mass[i], hdt = 0.5 * a.dt;
    const double ax = (double)fi.x * im, ay = (double)fi.y * im, az = (double)fi.z * im;
    a.ax[i] = ax; a.ay[i] = ay; a.az[i] = az;
    a.vx[i] = a.vx[i] + hdt * ax;
    a.vy[i] = a.vy[i] + hdt * ay;
    a.vz[i] = a.vz[i] + hdt * az;
}

VVTermArgs vv_term_args(mfa_ctx* c) {
    VVTermArgs a;
    a.force = c->force;
    a.vx = c->vx; a.vy = c->vy; a.vz = c->vz;
    a.ax = c->ax; a.ay = c->ay; a.az = c->az;
    a.mass = c->mass; a.inv_mass = c->inv_mass;
    a.fdp = c->fd; a.fdn = c->fd ? c->fd + (size_t)3 * c->n : nullptr;
    a.partials = c->partials + (size_t)R_TERMS * 4 * c->max_blocks;
    a.counter = c->counters + R_TERMS;
    a.tbuf = c->term_buf;
    a.dscal = c->dscal;
    a.n = c->n;
    a.max_blocks = c->max_blocks;
    a.dt = c->p.dt;
    return a;
}

}  // namespace

// DPD_VV velocity half (called by mfa_verlet_velocities when the switch is on)
int launch_dpd_vv_kick(mfa_ctx* c) {
    const VVTermArgs a = vv_term_args(c);
    const int nb = (c->n + TPB - 1) / TPB;
    if (c->prec == MFA_MIXED) k_dpd_vv_kick<float4><<<nb, TPB, 0, c->st>>>(a);
    else k_dpd_vv_kick<double4><<<nb, TPB, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}

extern "C" {

int mfa_external_force(mfa_ctx* c, int32_t mode, double k_elastic) {
    if (!c) return MFA_ERR_ARGS;
    if (mode != 1) return MFA_OK;   // external_force.f90:10: only case(1) acts
    const int nb = (c->n + TPB - 1) / TPB;
    const double hy = c->p.boundary[1] / 2.0, hz = c->p.boundary[2] / 2.0;
    if (c->prec == MFA_MIXED)
        k_external_force<<<nb, TPB, 0, c->st>>>((float4*)c->force, c->ry, c->rz, c->n, k_elastic, hy, hz);
    else
        k_external_force<<<nb, TPB, 0, c->st>>>((double4*)c->force, c->ry, c->rz, c->n, k_elastic, hy, hz);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}

int mfa_orientation(mfa_ctx* c, int32_t mode, double k_or, double alpha_or, double* v_or) {
    if (!c) return MFA_ERR_ARGS;
    if (v_or) *v_or = 0.0;
    if (mode != 1 && mode != 2) return MFA_OK;   // modes 0 (report) and 3 do nothing here
    if (c->p.n_chain == 0) return MFA_OK;
    if (c->p.n_mon < 2) return MFA_ERR_ARGS;
    TRY_(term_buf(c));
    OrientArgs a;
    a.force = c->force;
    a.rx = c->rx; a.ry = c->ry; a.rz = c->rz;
    for (int d = 0; d < 3; ++d) {
        a.L[d] = c->p.boundary[d];
        a.invL[d] = c->inv_boundary[d];
    }
    a.n_chain = c->p.n_chain;
    a.n_mon = c->p.n_mon;
    a.mode = mode;
    a.k_or = k_or;
    a.alpha_or = alpha_or;
    a.partials = c->partials + (size_t)R_TERMS * 4 * c->max_blocks;
    a.counter = c->counters + R_TERMS;
    a.max_blocks = c->max_blocks;
    a.out = c->term_buf;
    const int nb = (c->p.n_chain + TPB - 1) / TPB;
    if (c->prec == MFA_MIXED) k_orientation<float4><<<nb, TPB, 0, c->st>>>(a);
    else k_orientation<double4><<<nb, TPB, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    if (v_or) {
        MFA_CUDA_TRY(cudaMemcpyAsync(v_or, c->term_buf, sizeof(double), cudaMemcpyDeviceToHost, c->st));
        MFA_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    return MFA_OK;
}

int mfa_set_dpd_vv(mfa_ctx* c, int32_t on) {
    if (!c) return MFA_ERR_ARGS;
    if (on && !c->fd) {
        // force_d(:,:) = 0 at start (init_params.f90:839); two 3 x n FP64 buffers
        MFA_CUDA_TRY(cudaMalloc((void**)&c->fd, (size_t)6 * c->n * sizeof(double)));
        MFA_CUDA_TRY(cudaMemsetAsync(c->fd, 0, (size_t)6 * c->n * sizeof(double), c->st));
    }
    TRY_(term_buf(c));
    c->dpd_vv = on != 0;
    return MFA_OK;
}

int mfa_new_dpd_fd(mfa_ctx* c) {
    if (!c) return MFA_ERR_ARGS;
    if (!c->dpd_vv || !c->fd || !c->lists_valid) return MFA_ERR_STATE;
    DpdFdArgs d;
    d.nbr = c->nbr; d.ccount = c->ccount; d.ids = c->ids; d.type = c->type;
    d.rx = c->rx; d.ry = c->ry; d.rz = c->rz;
    d.vx = c->vx; d.vy = c->vy; d.vz = c->vz;
    d.range_2 = c->tabs + T8 * T8;
    d.fdn = c->fd + (size_t)3 * c->n;
    d.n = c->n;
    d.maxnb = c->maxnb;
    d.dpd_weight = c->p.dpd_weight;
    for (int k = 0; k < 2; ++k) {
        d.L[k] = c->p.boundary[k];
        d.invL[k] = c->inv_boundary[k];
    }
    d.friction = c->p.friction;
    const int nchunk = (c->n + 31) / 32;
    const int nb1 = (nchunk * 32 + TPB - 1) / TPB;
    k_dpd_fd<<<nb1, TPB, 0, c->st>>>(d);
    MFA_CUDA_TRY(cudaGetLastError());
    const VVTermArgs a = vv_term_args(c);
    const int nb2 = (c->n + TPB - 1) / TPB;
    if (c->prec == MFA_MIXED) k_dpd_vv_finish<float4><<<nb2, TPB, 0, c->st>>>(a);
    else k_dpd_vv_finish<double4><<<nb2, TPB, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 2);
    return MFA_OK;
}

}  // extern "C"
