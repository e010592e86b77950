// Implicit walls (fluid_wall.f90) as a stand-alone per-particle pass:
//   inter_type 2: 9-3 walls at z = 0 and z = z_space_wall (:77-125)
//   inter_type 3: 9-3 bottom wall, hard (reflecting) top wall (:127-163)
//   inter_type 4: hard walls at both ends (:165-180)
// The time-step fast path folds inter_type 2 into the pair kernel instead.
#include "mfa_internal.cuh"

namespace {

struct WallArgs {
    const double* rz;
    double* vz;
    const int32_t* type;
    void* force;
    double* partials;
    unsigned* counter;
    double* dscal;
    int max_blocks, n, inter_type, e_aw;
    double a_wall[T8], sigma_wall[T8], a_w, z_space_wall, z_head, wall_cut;
};

template <typename R>
__device__ __forceinline__ void term93(const WallArgs& a, int t, R zz, R& f, double& e) {
    const R aw = (R)a.a_wall[t - 1];
    wall93_term<R>(zz, (R)a.sigma_wall[t - 1], aw, a.e_aw ? (R)a.a_w : aw, (R)a.wall_cut, f, e);
}

template <typename R, typename R4>
__global__ void k_wall(WallArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {0.0};
    if (i < a.n) {
        const R z = (R)a.rz[i];
        if (a.inter_type == 2 || a.inter_type == 3) {
            const int t = a.type[i];
            R fz = 0, f;
            double e;
            if (a.wall_cut <= 0 || z < (R)a.wall_cut) { term93<R>(a, t, z, f, e); fz += f; acc[0] += e; }
            if (a.inter_type == 2) {
                const R zt = (R)a.z_space_wall - z;
                if (a.wall_cut <= 0 || zt < (R)a.wall_cut) { term93<R>(a, t, zt, f, e); fz -= f; acc[0] += e; }
            } else if ((double)z > (a.z_space_wall - a.z_head) && a.vz[i] > 0.0) {
                a.vz[i] = -a.vz[i];
            }
            R4* f4 = (R4*)a.force;
            R4 o = f4[i];
            o.z += fz;
            f4[i] = o;
        } else if (a.inter_type == 4) {
            const double eps01 = (double)0.01f;   // single-precision literal
            const double zz = a.rz[i];
            if (zz < eps01 && a.vz[i] < 0.0) a.vz[i] = -a.vz[i];
            if (zz > (a.z_space_wall - eps01) && a.vz[i] > 0.0) a.vz[i] = -a.vz[i];
        }
    }
    block_sum_commit<1>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_VFW);
}

}  // namespace

int launch_wall(mfa_ctx* c, int inter_type) {
    if (inter_type != 2 && inter_type != 3 && inter_type != 4) return MFA_ERR_ARGS;
    const mfa_params& p = c->p;
    WallArgs a;
    a.rz = c->rz; a.vz = c->vz; a.type = c->type; a.force = c->force;
    a.partials = c->partials + (size_t)R_WALL * 4 * c->max_blocks;
    a.counter = c->counters + R_WALL;
    a.dscal = c->dscal;
    a.max_blocks = c->max_blocks; a.n = c->n; a.inter_type = inter_type;
    a.e_aw = (p.quirks & MFA_Q_WALL_ENERGY_AW) != 0;
    for (int k = 0; k < T8; ++k) { a.a_wall[k] = p.a_wall[k]; a.sigma_wall[k] = p.sigma_wall[k]; }
    a.a_w = p.a_w; a.z_space_wall = p.z_space_wall; a.z_head = p.z_head; a.wall_cut = p.wall_cut;
    const int T = 256, nb = (c->n + T - 1) / T;
    if (nb > c->max_blocks) return MFA_ERR_ARGS;
    if (c->prec == MFA_MIXED) k_wall<float, float4><<<nb, T, 0, c->st>>>(a);
    else k_wall<double, double4><<<nb, T, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}
