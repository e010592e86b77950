// Bonded forces: FENE (intra_molec.f90) and bending (bending.f90, mode 2).
//
// One chain per warp.  Lanes stride over the chain's beads (ids are contiguous
// per chain, so the FP64 position reads are coalesced); the per-bond FENE
// forces, the bond vectors and the per-angle forces go to the warp's slice of
// shared memory, and each lane then sums the terms that touch its own beads, so
// there are no atomics and the force on a bead is summed in a fixed order.
// Bond vectors are formed in FP64 from the FP64 positions; the force math runs
// in R (float in MIXED, double in FP64).
#include "mfa_internal.cuh"

namespace {

struct BondArgs {
    const double *rx, *ry, *rz;
    void* force;
    int32_t* flags;
    double* partials;
    unsigned* counter;
    double* dscal;
    int max_blocks;
    int n_chain, n_mon, n_chain_d, n_mon_d, part_init_d;
    int symmetry;
    int do_fene, do_bend;
    double L[3], invL[3];
    double k_chain, k_ring, inv_r_chain_2, fene_clamp, k_bend, alpha_eq;
    int nm_max;
};

template <typename R> struct V4;
template <> struct V4<float> { typedef float4 T; };
template <> struct V4<double> { typedef double4 T; };

// bending.f90:88-93: theta = acos(cos) (0 when cos >= 1).  In FP64 the
// reference's acos is used as is; in FP32 acos loses its accuracy as theta -> 0
// (a 6e-8 error in cos becomes 3.5e-4 rad), so the same angle is taken as
// atan2(|p x n|, p . n), which keeps full relative accuracy there.
__device__ __forceinline__ float angle_of(float c, float px, float py, float pz, float nx, float ny, float nz,
                                          float dot) {
    if (c >= 1.0f) return 0.0f;
    const float cx = py * nz - pz * ny, cy = pz * nx - px * nz, cz = px * ny - py * nx;
    return atan2f(sqrtf(cx * cx + cy * cy + cz * cz), dot);
}
__device__ __forceinline__ double angle_of(double c, double, double, double, double, double, double, double) {
    return c >= 1.0 ? 0.0 : acos(c);
}
__device__ __forceinline__ float log1m_(float x) { return logf(1.0f - x); }
__device__ __forceinline__ double log1m_(double x) { return log(1.0 - x); }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }

template <typename R>
__global__ void k_bonds(BondArgs a) {
    typedef typename V4<R>::T R4;
    extern __shared__ unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nmx = a.nm_max;
    R* sm = (R*)smem_raw + (size_t)wib * nmx * 12;
    R* s_fene = sm;              // 3 per bond: force on the bond's second bead
    R* s_bv = sm + 3 * nmx;      // 3 per bond: bending bond vector (3D PBC)
    R* s_fp = sm + 6 * nmx;      // 3 per centre: force on the previous bead
    R* s_fn = sm + 9 * nmx;      // 3 per centre: force on the next bead
    const int chain = blockIdx.x * (blockDim.x >> 5) + wib;
    double e_fene = 0.0, e_fene_d = 0.0, e_bend = 0.0;
    int clamped = 0;
    const int nchains = a.n_chain + (a.n_mon_d >= 2 ? a.n_chain_d : 0);
    if (chain < nchains) {
        int base, nm;
        R kf;
        bool bend, melt;
        if (chain < a.n_chain) {
            base = chain * a.n_mon; nm = a.n_mon; kf = (R)a.k_chain; bend = a.do_bend; melt = false;
        } else {
            base = a.part_init_d + (chain - a.n_chain) * a.n_mon_d; nm = a.n_mon_d; kf = (R)a.k_ring;
            bend = false; melt = true;
        }
        const R irc2 = (R)a.inv_r_chain_2, clampv = (R)a.fene_clamp;
        // phase 1: bonds b = (b, b+1)
        for (int b = lane; b < nm - 1; b += 32) {
            const int i = base + b;
            const double d0 = a.rx[i] - a.rx[i + 1];
            const double d1 = a.ry[i] - a.ry[i + 1];
            const double d2 = a.rz[i] - a.rz[i + 1];
            if (a.do_fene) {
                // intra_molec.f90:225-263: delta = r(i) - r(i+1)
                const R dx = (R)(d0 - a.L[0] * (double)(int)(2.0 * d0 * a.invL[0]));
                const R dy = (R)(d1 - a.L[1] * (double)(int)(2.0 * d1 * a.invL[1]));
                const R dz = (R)(a.symmetry == 1 ? d2 - a.L[2] * (double)(int)(2.0 * d2 * a.invL[2]) : d2);
                const R r2 = dx * dx + dy * dy + dz * dz;
                R x = r2 * irc2;
                if (x >= clampv) { x = clampv; ++clamped; }
                const double pot = -0.5 * (double)log1m_(x);
                if (melt) e_fene_d += pot; else e_fene += pot;
                const R fs = kf / ((R)1 - x) * irc2;
                s_fene[3 * b + 0] = fs * dx;   // force_loc: bead b gets -, bead b+1 gets +
                s_fene[3 * b + 1] = fs * dy;
                s_fene[3 * b + 2] = fs * dz;
            }
            if (bend) {
                // bending.f90:34-57: r_next = r(b+1) - r(b), periodic in x, y and z
                s_bv[3 * b + 0] = (R)(-d0 + a.L[0] * (double)(int)(2.0 * d0 * a.invL[0]));
                s_bv[3 * b + 1] = (R)(-d1 + a.L[1] * (double)(int)(2.0 * d1 * a.invL[1]));
                s_bv[3 * b + 2] = (R)(-d2 + a.L[2] * (double)(int)(2.0 * d2 * a.invL[2]));
            }
        }
        __syncwarp();
        // phase 2: angles centred on bead c = 1 .. nm-2 (bending.f90:43-117)
        if (bend) {
            const R tiny = (R)1.0000000116860974e-07;   // 0.0000001 single-precision literal
            for (int c = 1 + lane; c < nm - 1; c += 32) {
                const R px = s_bv[3 * (c - 1) + 0], py = s_bv[3 * (c - 1) + 1], pz = s_bv[3 * (c - 1) + 2];
                const R nx = s_bv[3 * c + 0], ny = s_bv[3 * c + 1], nz = s_bv[3 * c + 2];
                const R dot = nx * px + ny * py + nz * pz;
                const R p2 = px * px + py * py + pz * pz;
                const R n2 = nx * nx + ny * ny + nz * nz;
                const R cosa = dot / sqrt_(p2 * n2);
                R dnx = px * n2 - nx * dot, dny = py * n2 - ny * dot, dnz = pz * n2 - nz * dot;
                R dpx = -nx * p2 + px * dot, dpy = -ny * p2 + py * dot, dpz = -nz * p2 + pz * dot;
                const R dn2 = dnx * dnx + dny * dny + dnz * dnz;
                const R dp2 = dpx * dpx + dpy * dpy + dpz * dpz;
                if (dn2 < tiny) { dnx = dny = dnz = 0; }
                else { const R s = (R)1 / sqrt_(dn2 * n2); dnx *= s; dny *= s; dnz *= s; }
                if (dp2 < tiny) { dpx = dpy = dpz = 0; }
                else { const R s = (R)1 / sqrt_(dp2 * p2); dpx *= s; dpy *= s; dpz *= s; }
                const R da = cosa >= (R)1 ? (R)0 : angle_of(cosa, px, py, pz, nx, ny, nz, dot) - (R)a.alpha_eq;
                const R fm = (R)a.k_bend * da;
                e_bend += (double)((R)0.5 * fm * da);
                s_fp[3 * c + 0] = fm * dpx; s_fp[3 * c + 1] = fm * dpy; s_fp[3 * c + 2] = fm * dpz;
                s_fn[3 * c + 0] = fm * dnx; s_fn[3 * c + 1] = fm * dny; s_fn[3 * c + 2] = fm * dnz;
            }
        }
        __syncwarp();
        // phase 3: every term that touches bead b
        R4* f4 = (R4*)a.force;
        for (int b = lane; b < nm; b += 32) {
            // FENE and bending are added to the force in two steps, so that the
            // fused pass rounds exactly like intra_molec followed by bending(2)
            R gx = 0, gy = 0, gz = 0, hx = 0, hy = 0, hz = 0;
            if (a.do_fene) {
                if (b < nm - 1) { gx -= s_fene[3 * b]; gy -= s_fene[3 * b + 1]; gz -= s_fene[3 * b + 2]; }
                if (b > 0) { gx += s_fene[3 * (b - 1)]; gy += s_fene[3 * (b - 1) + 1]; gz += s_fene[3 * (b - 1) + 2]; }
            }
            if (bend) {
                if (b + 1 <= nm - 2) { hx += s_fp[3 * (b + 1)]; hy += s_fp[3 * (b + 1) + 1]; hz += s_fp[3 * (b + 1) + 2]; }
                if (b >= 1 && b <= nm - 2) {
                    hx -= s_fp[3 * b] + s_fn[3 * b];
                    hy -= s_fp[3 * b + 1] + s_fn[3 * b + 1];
                    hz -= s_fp[3 * b + 2] + s_fn[3 * b + 2];
                }
                if (b - 1 >= 1) { hx += s_fn[3 * (b - 1)]; hy += s_fn[3 * (b - 1) + 1]; hz += s_fn[3 * (b - 1) + 2]; }
            }
            R4 o = f4[base + b];
            if (a.do_fene) { o.x += gx; o.y += gy; o.z += gz; }
            if (bend) { o.x += hx; o.y += hy; o.z += hz; }
            f4[base + b] = o;
        }
    }
    // intra_molec.f90:300 / :272: energies multiplied by k_chain
    for (int o = 16; o > 0; o >>= 1) clamped += __shfl_down_sync(0xffffffffu, clamped, o);
    if (lane == 0 && clamped) atomicAdd(&a.flags[F_FENE], clamped);
    double acc[2] = {a.k_chain * (e_fene + e_fene_d), e_bend};
    if (block_sum_commit<2>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_TMP0) && threadIdx.x == 0) {
        // publish only what this pass computed (intra_molec and bending are separate calls)
        if (a.do_fene) a.dscal[S_VINTRA] = a.dscal[S_TMP0];
        if (a.do_bend) a.dscal[S_VBEND] = a.dscal[S_TMP0 + 1];
    }
}

}  // namespace

int bonds_setup(mfa_ctx* c) {
    const int nm = c->p.n_mon > c->p.n_mon_d ? c->p.n_mon : c->p.n_mon_d;
    const size_t esz = c->prec == MFA_MIXED ? 4 : 8;
    const size_t per_warp = (size_t)(nm > 1 ? nm : 2) * 12 * esz;
    // dynamic shared memory per block stays under 40 KB (the kernel also holds
    // a little static shared memory for its reductions)
    int wpb = (int)((40 * 1024) / per_warp);
    if (wpb > 8) wpb = 8;
    if (wpb < 1) {
        if (per_warp > 200 * 1024) return MFA_ERR_UNSUPPORTED;
        wpb = 1;
    }
    c->bond_warps_per_block = wpb;
    c->bond_smem = per_warp * wpb;
    if (c->prec == MFA_MIXED)
        MFA_CUDA_TRY(cudaFuncSetAttribute(k_bonds<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->bond_smem));
    else
        MFA_CUDA_TRY(cudaFuncSetAttribute(k_bonds<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->bond_smem));
    return MFA_OK;
}

int launch_bonds(mfa_ctx* c, int do_fene, int do_bend) {
    const mfa_params& p = c->p;
    BondArgs a;
    a.rx = c->rx; a.ry = c->ry; a.rz = c->rz;
    a.force = c->force; a.flags = c->dflags;
    a.partials = c->partials + (size_t)R_BOND * 4 * c->max_blocks;
    a.counter = c->counters + R_BOND;
    a.dscal = c->dscal;
    a.max_blocks = c->max_blocks;
    a.n_chain = p.n_chain; a.n_mon = p.n_mon; a.n_chain_d = p.n_chain_d; a.n_mon_d = p.n_mon_d;
    a.part_init_d = p.n_mon * p.n_chain;
    a.symmetry = p.symmetry;
    a.do_fene = do_fene; a.do_bend = do_bend && p.bending;
    for (int d = 0; d < 3; ++d) { a.L[d] = p.boundary[d]; a.invL[d] = c->inv_boundary[d]; }
    a.k_chain = p.k_chain; a.k_ring = p.k_ring; a.inv_r_chain_2 = p.inv_r_chain_2;
    a.fene_clamp = p.fene_clamp; a.k_bend = p.k_bend; a.alpha_eq = p.alpha_eq;
    a.nm_max = p.n_mon > p.n_mon_d ? p.n_mon : p.n_mon_d;
    if (a.nm_max < 2) a.nm_max = 2;
    const int nchains = p.n_chain + (p.n_mon_d >= 2 ? p.n_chain_d : 0);
    const int wpb = c->bond_warps_per_block;
    int nb = (nchains + wpb - 1) / wpb;
    if (nb < 1) nb = 1;
    if (nb > c->max_blocks) return MFA_ERR_ARGS;
    if (c->prec == MFA_MIXED) k_bonds<float><<<nb, 32 * wpb, c->bond_smem, c->st>>>(a);
    else k_bonds<double><<<nb, 32 * wpb, c->bond_smem, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}
