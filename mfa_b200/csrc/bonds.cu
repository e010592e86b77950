// Bonded forces: FENE (intra_molec.f90) and bending (bending.f90, mode 2).
//
// Thread per chain bead (bonded.cuh): the bead's two bonds and the three angles
// that move it, recomputed by each bead that needs them, so that every bead's
// force is summed by one thread in a fixed order, without atomics.  The time-step
// fast path folds the same computation into the fused integrator (k_vv_fused in
// integrate.cu), which adds it to the force record before a = F/m.
#include "mfa_internal.cuh"

#include <type_traits>

#include "bonded.cuh"

namespace {

struct BondArgs {
    BondParams b;
    void* force;
    int32_t* flags;
    double* partials;
    unsigned* counter;
    double* dscal;
    int max_blocks;
    int n1, n2;          // beads of grafted/bulk chains, beads of melt chains
};

// thread per chain bead: the bead's FENE and bending forces, added to force
template <typename R>
__global__ void k_bonds(BondArgs a) {
    typedef typename std::conditional<sizeof(R) == 4, float4, double4>::type R4;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double e_fene = 0.0, e_bend = 0.0;
    int clamped = 0;
    if (t < a.n1 + a.n2) {
        const int i = t < a.n1 ? t : a.b.part_init_d + (t - a.n1);
        R f[3] = {0, 0, 0};
        bonded_on_bead<R>(a.b, i, f, e_fene, e_bend, clamped);
        R4* f4 = (R4*)a.force;
        R4 o = f4[i];
        o.x += f[0]; o.y += f[1]; o.z += f[2];
        f4[i] = o;
    }
    for (int o = 16; o > 0; o >>= 1) clamped += __shfl_down_sync(0xffffffffu, clamped, o);
    if ((threadIdx.x & 31) == 0 && clamped) atomicAdd(&a.flags[F_FENE], clamped);
    // intra_molec.f90:96 / :270: energies multiplied by k_chain
    double acc[2] = {a.b.k_chain * e_fene, e_bend};
    if (block_sum_commit<2>(acc, a.partials, a.max_blocks, a.counter, a.dscal + S_TMP0) && threadIdx.x == 0) {
        // publish only what this pass computed (intra_molec and bending are separate calls)
        if (a.b.do_fene) a.dscal[S_VINTRA] = a.dscal[S_TMP0];
        if (a.b.do_bend) a.dscal[S_VBEND] = a.dscal[S_TMP0 + 1];
    }
}

}  // namespace

int bonds_setup(mfa_ctx* c) {
    (void)c;
    return MFA_OK;
}

int launch_bonds(mfa_ctx* c, int do_fene, int do_bend) {
    const mfa_params& p = c->p;
    BondArgs a;
    a.b = bond_params(c, do_fene, do_bend);
    a.force = c->force; a.flags = c->dflags;
    a.partials = c->partials + (size_t)R_BOND * 4 * c->max_blocks;
    a.counter = c->counters + R_BOND;
    a.dscal = c->dscal;
    a.max_blocks = c->max_blocks;
    a.n1 = p.n_chain * p.n_mon;
    a.n2 = p.n_mon_d >= 2 ? p.n_chain_d * p.n_mon_d : 0;
    const int T = 256;
    int nb = (a.n1 + a.n2 + T - 1) / T;
    if (nb < 1) nb = 1;
    if (nb > c->max_blocks) return MFA_ERR_ARGS;
    if (c->prec == MFA_MIXED) k_bonds<float><<<nb, T, 0, c->st>>>(a);
    else k_bonds<double><<<nb, T, 0, c->st>>>(a);
    MFA_CUDA_TRY(cudaGetLastError());
    note_launch(c, 1);
    return MFA_OK;
}
