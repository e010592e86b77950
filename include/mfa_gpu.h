/*
 * mfa_gpu.h -- C ABI of the B200 (sm_100a) implementation of mfa's per-timestep
 * force and integration loop.
 *
 * The reference program (feindas/mfa) drives one MD/DPD time step from
 * md_main.f90:68-157 by calling argument-less Fortran subroutines that read and
 * write the global module `commons` (mfa_common.f90).  Every entry point below
 * replaces one of those subroutines; a Fortran shim with the same subroutine
 * name calls it through iso_c_binding.  After mfa_init the GPU owns all
 * particle state; host arrays are mirrors that are valid after mfa_download.
 *
 * Conventions at this boundary (they follow the Fortran layouts):
 *   - positions/velocities/accelerations/forces are double[3*n_part], xyz
 *     contiguous per particle (Fortran r0(3,n_part), column-major);
 *   - mic_count is int32[3*n_part] (Fortran mic_count(3,n_part));
 *   - a_type is int32[n_part] with values 1..n_type (Fortran a_type);
 *   - particle ids in lists are 1-based (Fortran ff_list / bin_fluid);
 *   - pair tables are indexed [(ti-1)*MFA_MAX_TYPES + (tj-1)].
 * Every function returns an mfa_status code (0 = ok).  Calls are asynchronous on
 * the context's CUDA stream; mfa_check_skin, mfa_get_scalars, mfa_download and
 * mfa_sync synchronise and report device-side errors.
 */
#ifndef MFA_GPU_H
#define MFA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MFA_MAX_TYPES 8
#define MFA_ABI_VERSION 1

typedef enum mfa_status {
    MFA_OK = 0,
    MFA_ERR_ARGS = 1,            /* bad argument or parameter combination        */
    MFA_ERR_CUDA = 2,            /* a CUDA runtime call failed                   */
    MFA_ERR_CELL_RANGE = 3,      /* particle outside the binning grid (z<0 ...)  */
    MFA_ERR_NEIGH_OVERFLOW = 4,  /* neighbour list capacity exceeded             */
    MFA_ERR_NONFINITE = 5,       /* NaN/Inf in positions or forces               */
    MFA_ERR_TIMEOUT = 6,         /* a bounded device wait gave up                */
    MFA_ERR_NOMEM = 7,           /* device allocation failed                     */
    MFA_ERR_STATE = 8,           /* call order violated (e.g. forces before lists) */
    MFA_ERR_UNSUPPORTED = 9,     /* feature not built for this parameter set     */
    MFA_ERR_CAPACITY = 10        /* request larger than a fixed-size buffer      */
} mfa_status;

typedef enum mfa_precision {
    MFA_FP64 = 0,   /* every quantity in FP64 (plain FP64 GPU path)                   */
    MFA_MIXED = 1   /* FP32 pair/bond forces; FP64 positions, VV, reductions, Ewald-k */
} mfa_precision;

/* Reference quirk switches (mfa_params.quirks).  Set = reproduce the reference. */
#define MFA_Q_EWALD_REAL_IN_LJ  0x1  /* fluid_fluid.f90:94,166: Ewald real only inside range_2 */
#define MFA_Q_WALL_ENERGY_AW    0x2  /* fluid_wall.f90:98,116: energy uses a_w, force a_wall(t) */

/* Thermostat selector (control_simulation.h:45 THERMOSTAT) */
#define MFA_THERMO_DPD  0
#define MFA_THERMO_LGV  1
#define MFA_THERMO_NONE 2

/* Noise shape for DPD / Langevin random forces */
#define MFA_NOISE_GAUSS   0   /* Box-Muller on Philox-4x32-10 (stands in for rnor())   */
#define MFA_NOISE_UNIFORM 1   /* sqrt(3)*(2u-1), the alternative of dpd_forces.f90:24 */

/*
 * Run parameters.  These are the *derived* constants the reference computes in
 * init_params.f90 / init_config.f90 / make_binning_boxes.f90 (epsilon already
 * multiplied by 4, k_chain already multiplied by R0^2, range_2 with the
 * single-precision 2.**(1./6.) literal, ...).  A Fortran shim fills this struct
 * from the `commons` module variables of the same names.
 */
typedef struct mfa_params {
    /* sizes and topology */
    int32_t n_part;          /* particles (= n_mon_tot; explicit wall atoms unsupported) */
    int32_t n_type;          /* 1..MFA_MAX_TYPES                                        */
    int32_t n_mon, n_chain;  /* grafted/bulk chains, ids 1..n_mon*n_chain               */
    int32_t n_mon_d, n_chain_d; /* melt/droplet chains, ids part_init_d+1..            */
    /* control_simulation.h switches as runtime fields */
    int32_t symmetry;        /* 0 channel (PBC x,y), 1 bulk (PBC x,y,z)                 */
    int32_t thermostat;      /* MFA_THERMO_*                                            */
    int32_t dpd_weight;      /* 0: w_r = 1-r/rc, w_d = w_r^2; 1: w_r = w_d = 1          */
    int32_t wall;            /* 0 none, 2: 9-3 both walls, 3: 9-3 bottom + hard top,
                                4: hard walls (fluid_wall.f90 inter_type)                */
    int32_t charged;         /* Ewald real + k-space (SYSTEM 2,3)                       */
    int32_t bending;         /* bending(2) over the grafted/bulk chains                 */
    int32_t force_switch_on; /* FORCE_SWITCH_ON clamp r^2 = max(r^2, r_2_min)           */
    int32_t pin_heads;       /* brush heads pinned (verlet_velocities.f90:113-145)      */
    int32_t quirks;          /* MFA_Q_* bits                                            */
    int32_t noise;           /* MFA_NOISE_*                                             */
    /* geometry and cell grid */
    double  boundary[3];
    int32_t n_bin[3];        /* cells per axis (make_binning_boxes.f90:44-46)         */
    int32_t delta_bin[3];    /* upper neighbour-cell offset (make_binning_boxes.f90:14-37) */
    int32_t pad0;
    /* pair tables [(ti-1)*MFA_MAX_TYPES + (tj-1)] */
    double  range_2[MFA_MAX_TYPES * MFA_MAX_TYPES];
    double  epsil[MFA_MAX_TYPES * MFA_MAX_TYPES];      /* already x4              */
    double  sigma_2[MFA_MAX_TYPES * MFA_MAX_TYPES];
    double  e_shift[MFA_MAX_TYPES * MFA_MAX_TYPES];
    double  inv_range_2[MFA_MAX_TYPES * MFA_MAX_TYPES];
    double  skin, skin_2;    /* check_skin.f90:18, init_params.f90:807-808              */
    /* integrator and thermostat */
    double  dt, temp, friction, sig;  /* sig = sqrt(2 T friction / dt) (init_params.f90:845) */
    /* bonds */
    double  k_chain;         /* FENE k * R0^2 (init_params.f90:398), grafted chains     */
    double  k_ring;          /* FENE constant used for melt/droplet chains (intra_molec.f90:133) */
    double  r_chain_2, inv_r_chain_2;
    double  fene_clamp;      /* 0.98 (single-precision literal, intra_molec.f90:44)    */
    double  k_bend, alpha_eq;
    /* walls */
    double  a_wall[MFA_MAX_TYPES], sigma_wall[MFA_MAX_TYPES];
    double  a_w, z_space_wall, z_head;
    double  wall_cut;        /* 0: no cutoff (reference); >0: truncate+shift at z = wall_cut */
    double  va_spring_twall[3];
    /* force switch-on (fluid_fluid.f90:42-49, init_force_switch_on.f90:15-22) */
    double  r_2_min_init, r_2_min_time;
    int64_t s_time;
    /* Ewald (init_config.f90:217-246, ewald_k.f90) */
    double  alpha_c;         /* the code's alpha_c (= alpha^2)                          */
    double  sqrt_alpha;
    double  inv_sqrt_pi;     /* 1/pi in the reference (init_config.f90:230)             */
    double  pi;              /* value of pi used in the k-space sums                    */
    double  ewald_rc_2;      /* real-space cutoff^2 when MFA_Q_EWALD_REAL_IN_LJ is off  */
    int32_t n_kmax;
    int32_t pad1;
    /* counter-based noise */
    uint64_t seed;
} mfa_params;

/* Scalars after a step (the `commons` variables of the same name). */
typedef struct mfa_scalars {
    double  v_fluid_fluid;   /* LJ energy, pairs counted once                    */
    double  v_fluid_wall;
    double  v_intra_molec;   /* FENE, brush + melt                               */
    double  v_bend;
    double  v_coul;          /* real + k-space + self                            */
    double  t_fluid;         /* 0.5 * sum m v^2 over n_part                      */
    double  v_total;         /* v_fluid_wall + v_fluid_fluid + v_intra_molec     */
    double  e_total;         /* v_total + t_fluid                                */
    double  virial;          /* sum over pairs of r_ij . F_ij (LJ + DPD + Coulomb real) */
    int64_t i_time;          /* step counter of the context                      */
    int32_t f_skin;
    int32_t n_rebuilds;      /* neighbour-list rebuilds since mfa_init           */
    int32_t max_neigh;       /* largest list row seen at the last rebuild        */
    int32_t max_cell;        /* largest cell occupancy at the last rebuild       */
    int32_t fene_clamped;    /* bonds that hit the 0.98 clamp since mfa_init     */
    int32_t error_bits;      /* device error word                                */
    int64_t kernel_launches; /* kernels this context launched since mfa_init
                                (each kernel of a replayed graph counted)       */
} mfa_scalars;

typedef struct mfa_ctx mfa_ctx;

/* Download / upload masks */
#define MFA_R0   0x01
#define MFA_V    0x02
#define MFA_A    0x04
#define MFA_F    0x08
#define MFA_MIC  0x10

/* ---------------- lifetime ---------------- */

/* Replaces the allocation in init_system.f90:228-299 plus the state upload that
 * follows init_config (md_main.f90:51-53).  q may be NULL unless p->charged;
 * mic_count may be NULL (zeros).  device < 0 keeps the current device. */
int mfa_init(const mfa_params* p, int precision, int device,
             const double* r0, const double* v, const double* a,
             const int32_t* a_type, const double* mass, const double* q,
             const int32_t* mic_count, mfa_ctx** out);
int mfa_finalize(mfa_ctx* ctx);
int mfa_abi_version(void);
/* sizeof(mfa_params) and sizeof(mfa_scalars) as compiled into the library, so a
 * binding (Fortran iso_c_binding, ctypes) can check its struct mirrors. */
int mfa_abi_sizes(int32_t* params_bytes, int32_t* scalars_bytes);
const char* mfa_status_string(int status);

/* Sets the step counter i_time (md_main.f90:68); r_time = (s_time+i_time-1)*dt. */
int mfa_set_step(mfa_ctx* ctx, int64_t i_time);

/* ---------------- the per-step subroutines ---------------- */

/* verlet_positions.f90:146-171,237-251: r += dt v + dt^2/2 a; v += dt/2 a; wrap.
 * Also advances i_time by one (the loop counter of md_main.f90:68). */
int mfa_verlet_positions(mfa_ctx* ctx);
/* check_skin.f90:4-24.  Synchronises; *f_skin = 1 if a rebuild is due. */
int mfa_check_skin(mfa_ctx* ctx, int32_t* f_skin);
/* binning.f90:2-131 (BIN_TYPE 0).  Cell binning + Verlet list, f_skin = 0,
 * snapshot r0_old/mic_old.  The list is held as a full (both-direction) list;
 * as a set of unordered pairs it equals the reference's half list. */
int mfa_binning(mfa_ctx* ctx);
/* my_binning.f90:5-140 (BIN_TYPE 1).  Same cells and pairs; the full list is
 * what my_binning builds. */
int mfa_my_binning(mfa_ctx* ctx);
/* force(:,:) = 0 (md_main.f90:88). */
int mfa_zero_forces(mfa_ctx* ctx);
/* fluid_fluid.f90:1-254 with dpd_forces (THERMOSTAT 0), lgv_forces
 * (THERMOSTAT 1) and ewald_real (charged) fused in.  Adds to force. */
int mfa_fluid_fluid(mfa_ctx* ctx);
/* md_main.f90:93-97 in one pass: fluid_fluid (with the thermostat and Ewald
 * real space, as mfa_fluid_fluid) and, for SYMMETRY 0, fluid_wall(wall): the
 * 9-3 walls of WALL 2 (fluid_wall.f90:77-125) in the same kernel, WALL 3/4 as
 * mfa_fluid_wall.  Adds to force.  The pair kernel the time-step loop of
 * mfa_step runs. */
int mfa_pair_forces(mfa_ctx* ctx);
/* Every force of a step, md_main.f90:93-131: mfa_pair_forces, ewald_k(1),
 * dipolar_correction (charged SYMMETRY 0) and the chains' intra_molec +
 * bending(2) (one pass, thread per bead).  Adds to force (after
 * mfa_zero_forces it replaces the seven subroutine calls). */
int mfa_forces(mfa_ctx* ctx);
/* fluid_wall.f90:2-204, inter_type 2, 3 or 4.  Adds to force (2,3), reflects v (3,4). */
int mfa_fluid_wall(mfa_ctx* ctx, int32_t inter_type);
/* intra_molec.f90:1-539: FENE bonds of grafted and melt chains.  Adds to force. */
int mfa_intra_molec(mfa_ctx* ctx);
/* bending.f90:2-149 (mode 0: no-op, mode 2: angle forces).  Adds to force. */
int mfa_bending(mfa_ctx* ctx, int32_t mode);
/* ewald_k.f90:1-211 (mode 0: build k-vectors, mode 1: k-space energy + force).
 * Mode 0 returns MFA_ERR_UNSUPPORTED beyond 64 multiples of delta_k on an axis
 * or 65,536 vectors. */
int mfa_ewald_k(mfa_ctx* ctx, int32_t mode);
/* dipolar_correction.f90:17-39, called after ewald_k(1) for SYMMETRY 0
 * (md_main.f90:128-131): the slab correction of Yeh and Berkowitz,
 * M_z = sum q (z - Lz/2), F_z -= 4 pi q M_z / V, v_coul += 2 pi M_z^2 / V, with
 * V the slab volume of ewald_k(0).  Adds to force; nothing for uncharged or
 * SYMMETRY 1 systems; MFA_ERR_STATE before mfa_ewald_k(ctx, 0). */
int mfa_dipolar_correction(mfa_ctx* ctx);
/* verlet_velocities.f90:1-246: a = F/m, v += dt/2 a, heads pinned, energies.
 * With DPD_VV switched on (mfa_set_dpd_vv) only a = F/m and the kick
 * (:23-35); the head rules and energies are compiled out there (:79-230). */
int mfa_verlet_velocities(mfa_ctx* ctx);

/* ---------------- optional terms behind cpp switches ---------------- */

/* external_force.f90:1-20 (EXT_FORCE 1, md_main.f90:122-124): mode 1 adds
 * -k_elastic (y - Ly/2) and -k_elastic (z - Lz/2) to every bead's force; other
 * modes do nothing.  k_elastic is the commons variable read by init_params.f90:216. */
int mfa_external_force(mfa_ctx* ctx, int32_t mode, double k_elastic);
/* orientation.f90:3-185 (ORIENTATION, md_main.f90:114-121).  mode 1: angle
 * term between a ghost bond at each grafted chain's head (one unit further
 * from the mid-plane) and the chain's first bond, forces on the head and the
 * second bead (x, y minimum-imaged); mode 2: the first and last bond against
 * the x axis, as compiled with CHAIN_BC 2; modes 0 and 3 do nothing (mode 0's
 * k_or = k_bend, alpha_or = 0 are the caller's arguments).  Adds to force.
 * v_or may be NULL; otherwise the call synchronises and stores the
 * orientation energy (v_or of the commons, not part of v_total).
 * MFA_ERR_ARGS for chains of fewer than 2 beads. */
int mfa_orientation(mfa_ctx* ctx, int32_t mode, double k_or, double alpha_or, double* v_or);
/* The DPD_VV switch (control_simulation.h:51) as a runtime setting: on, it
 * allocates force_d (zero, init_params.f90:839), makes mfa_verlet_velocities
 * the kick alone and enables mfa_new_dpd_fd.  mfa_step, batches and the
 * adjoint refuse a context with the switch on (MFA_ERR_UNSUPPORTED). */
int mfa_set_dpd_vv(mfa_ctx* ctx, int32_t on);
/* new_dpd_fd.f90:1-215 (md_main.f90:149-155): the dissipative force over the
 * Verlet list with the current velocities (heads excluded, x and y
 * minimum-imaged, no force switch-on); force += Fd_new - Fd_previous; then
 * v += dt/2 F/m, a = F/m, t_fluid, v_total, e_total.  MFA_ERR_STATE unless
 * DPD_VV is on and the lists are built. */
int mfa_new_dpd_fd(mfa_ctx* ctx);

/* ---------------- fast path ---------------- */

/* Runs nsteps complete time steps (md_main.f90:69-147) on the device: fused
 * kernels, rebuild decided on the device, steps replayed as captured CUDA
 * graphs.  No host synchronisation inside.  The rebuild of a captured step
 * sits in a conditional graph node that the integrator opens when the skin
 * check trips; with the environment variable MFA_GRAPH_CONDITIONAL=0 at
 * mfa_init the rebuild kernels are launched every step instead and return at
 * once when no rebuild is due (for profilers that replay graph nodes one by
 * one, which do not handle conditional nodes).  A call of at most 32 steps
 * whose count equals the previous call's (or one of the four counts captured
 * last) replays a single graph for the whole call; the first call with a new
 * count captures nothing new.  Energies (mfa_get_scalars) are those of the
 * call's last step; the steps in between reduce none, except the steps the
 * energy log records. */
int mfa_step(mfa_ctx* ctx, int32_t nsteps);
/* Records e_total/v_total/t_fluid every `every` steps of mfa_step into a device
 * log of `capacity` entries (0 disables).  Read back with mfa_read_energy_log. */
int mfa_set_energy_log(mfa_ctx* ctx, int32_t every, int32_t capacity);
int mfa_read_energy_log(mfa_ctx* ctx, double* out3, int32_t max_entries, int32_t* n_out);
/* No counterpart in the reference (its fort.60 is written by the time-step
 * loop itself).  Enqueues, without waiting, the copy of log entries
 * [first, first + count) (4 doubles each: step, e_total, v_total, t_fluid)
 * into `out` on the context's stream, after every step enqueued before it, so
 * a driver can collect each call's energies while the next call runs.  `out`
 * should be pinned host memory; it is valid after the next synchronising call
 * (mfa_sync, mfa_get_scalars, mfa_download).  With `every` = 1 the entry of
 * the k-th step logged since mfa_set_energy_log is entry k - 1.
 * MFA_ERR_STATE without a log, MFA_ERR_ARGS beyond its capacity. */
int mfa_fetch_energy_log(mfa_ctx* ctx, double* out, int32_t first, int32_t count);

/* Launch shape of the pair kernel: how many list entries a thread tests per
 * round before its warp evaluates the in-range pairs 32 at a time (2 or 4),
 * threads per block (32..256, multiple of 32), and whether each block (one
 * cell row) stages its neighbourhood in shared memory (tiled = 1) or blocks
 * of consecutive particles read neighbours through the cache hierarchy
 * (tiled = 0).  The forces do not depend on it beyond rounding; it is what the
 * autotuner (mfa_b200.tune) chooses. */
int mfa_set_pair_shape(mfa_ctx* ctx, int32_t entries_per_round, int32_t block, int32_t tiled);
/* No counterpart in the reference.  Untiled launches of the pair kernel with a
 * work queue: a fixed grid of ctas_per_sm CTAs per multiprocessor whose warps
 * take 32-particle chunks from a shared counter until none is left, so that
 * warps that finish early take more work; 0 (the default) gives every block
 * of consecutive particles its own CTA.  The forces do not depend on it beyond
 * rounding; the autotuner chooses it.  Launches of one context must not
 * overlap on the GPU (they share the counter), which a context's own stream
 * guarantees. */
int mfa_set_pair_queue(mfa_ctx* ctx, int32_t ctas_per_sm);
/* No counterpart in the reference.  Untiled launches of the pair kernel cut
 * the list of every 32-particle chunk into `pieces` runs of equal length (1 to
 * 64), each taken by its own warp, so that a small system with long lists
 * (few chunks, many entries each) still occupies every multiprocessor; the
 * owners' forces of the pieces are summed by atomic adds.  The default is set
 * at mfa_init from the expected neighbour count and the device's
 * multiprocessor count; tiled launches use 1.  The forces do not depend on it
 * beyond rounding; the autotuner chooses it. */
int mfa_set_pair_split(mfa_ctx* ctx, int32_t pieces);
/* The current pieces per chunk (mfa_set_pair_split). */
int mfa_get_pair_split(mfa_ctx* ctx, int32_t* pieces);

/* Re-grids the cell list (n_bin cells per axis) and sets the Verlet skin
 * (skin_2 derived as init_params.f90:807-808 does).  Cells must be at least as
 * wide as the list radius wherever n_bin >= 3, or MFA_ERR_ARGS is returned.
 * The lists are rebuilt at the next step (mfa_check_skin reports 1).  The
 * forces do not depend on either choice; the autotuner uses it. */
int mfa_set_cells(mfa_ctx* ctx, const int32_t* n_bin, double skin);

/* ---------------- observables on the device ---------------- */

/* One observation of the current state (observation.f90:173-283), computed
 * on the device; only these nine numbers come back (md_main.f90:159-165 reads
 * the whole state for them).  Chains are unfolded bead by bead as the
 * reference does (a bead moves by one box length when it lies more than half
 * a box from the bead before it; brush chains in SYMMETRY 0 only, melt or
 * droplet chains always).  r_g2_brush = r_g2(1,:), the per-axis mean square
 * radius of gyration of the n_chain chains of n_mon beads; r_g2_melt =
 * r_g2(2,:) over chains n_chain+1..n_chain+n_chain_d taken as ids
 * (i_chain-1)*n_mon_d+1..i_chain*n_mon_d (the reference's indexing; NaN when
 * there are none, its 0/0); momentum = sum m v (:279-283).  Synchronises.
 * MFA_ERR_UNSUPPORTED when that melt indexing would run past the particles. */
typedef struct mfa_observables {
    double r_g2_brush[3];
    double r_g2_melt[3];
    double momentum[3];
} mfa_observables;
int mfa_observe(mfa_ctx* ctx, mfa_observables* out);
/* r_end_to_end_2v(2) of functions.f90:626-667 and the head forces of
 * observation.f90:326-328, from the chains unfolded as for mfa_observe:
 * r_ee9 = the mean end-to-end vector of the top brushes (chains
 * 1..n_chain/2), the bottom brushes (n_chain/2+1..n_chain) and the melt
 * (n_chain+1..n_chain+n_chain_d), x y z each; r_ee2_9 = the means of its
 * squared components; every chain is read as n_mon beads from
 * (i_chain-1)*n_mon+1, and the brush sums are divided by n_chain/2 in integer
 * arithmetic, both as the reference does.  f_heads6 = minus the summed force
 * on the grafted heads of the upper-wall chains (1..n_chain/2) and of the
 * lower-wall chains, xyz each, as the last velocity half saw it before the pin
 * (f_on_heads of verlet_velocities.f90:18; zeros when the heads are not
 * pinned).  Any pointer may be NULL.  Synchronises.  The melt group is NaN
 * when its chains are single beads (explicit solvent) or its indexing would
 * run past the particles. */
int mfa_observe_ends(mfa_ctx* ctx, double* r_ee9, double* r_ee2_9, double* f_heads6);
/* histo(2) of functions.f90:157-185: adds the current z positions of the brush
 * beads (ids 1..n_mon*n_chain) and the melt/droplet beads (the next
 * n_mon_d*n_chain_d) to device-resident histograms of hist_dim bins
 * (bin int(z / (Lz / hist_dim)) + 1, clamped), restarting them when reset is
 * set or hist_dim changes.  counts (2 x hist_dim: brush, then melt) and n_obs
 * (observations accumulated), when not NULL, receive the totals (then the
 * call synchronises).  The normalisation of histo(1) -- counts * hist_dim /
 * (Lz * n_obs * Lx * Ly) -- is the caller's. */
int mfa_histogram_z(mfa_ctx* ctx, int32_t hist_dim, int32_t reset, double* counts, int32_t* n_obs);

/* ---------------- host mirrors ---------------- */

int mfa_get_scalars(mfa_ctx* ctx, mfa_scalars* out);
int mfa_download(mfa_ctx* ctx, uint32_t mask, double* r0, double* v, double* a,
                 double* force, int32_t* mic_count);
int mfa_upload(mfa_ctx* ctx, uint32_t mask, const double* r0, const double* v,
               const double* a, const double* force, const int32_t* mic_count);
int mfa_sync(mfa_ctx* ctx);
/* The CUDA stream (cudaStream_t) all of the context's work is ordered on, for
 * callers that time it with events or order their own copies after it. */
int mfa_stream(mfa_ctx* ctx, void** cuda_stream);

/* Parity hooks: cell index per particle (0-based ix + nbx*(iy + nby*iz)) and the
 * Verlet list, rows in particle order, 1-based ids, row i = nbr[i*max_per ..
 * i*max_per + nbr_count[i]).  After mfa_binning a half list (every pair once,
 * in the row of the particle with the lower cell-sorted slot); after
 * mfa_my_binning a full list (both directions), as the reference builds them. */
int mfa_debug_lists(mfa_ctx* ctx, int32_t* cell_of, int32_t* nbr_count,
                    int32_t* nbr, int32_t max_per);
/* Number of k-vectors and their components (after mfa_ewald_k(ctx, 0)). */
int mfa_debug_kvecs(mfa_ctx* ctx, int32_t* nk, double* kvecs3, int32_t max_k);

/* ---------------- many systems in one launch ---------------- */

/* No counterpart in the reference, which runs one system per process (the
 * md_main.f90:68-184 loop).  Groups n contexts made by mfa_init -- independent
 * systems of any size and box, same device, precision and physics switches
 * (thermostat, SYMMETRY, WALL; no Ewald, no WALL 3/4) -- so that
 * mfa_batch_step advances all of them: each kernel stage of the time step is
 * ONE launch for the whole batch (a table maps every block to its system),
 * steps are captured CUDA graphs, and a system's lists are rebuilt when its
 * own skin check trips.  Every context keeps its state, energies and error
 * flags; read them with mfa_get_scalars / mfa_download after mfa_batch_sync.
 * The contexts must outlive the batch; their pair-kernel shape becomes the
 * first context's. */
typedef struct mfa_batch mfa_batch;
int mfa_batch_create(mfa_ctx* const* ctxs, int32_t n, mfa_batch** out);
/* nsteps time steps of every system of the batch (asynchronous, one stream). */
int mfa_batch_step(mfa_batch* batch, int32_t nsteps);
int mfa_batch_sync(mfa_batch* batch);
/* The batch's CUDA stream (cudaStream_t), for event timing. */
int mfa_batch_stream(mfa_batch* batch, void** cuda_stream);
/* Kernels the batch has launched so far (grouped launches; a rebuild node
 * that opened counts its six kernels once, however many systems rebuilt). */
int mfa_batch_launches(mfa_batch* batch, int64_t* launches);
/* Releases the batch (not its contexts). */
int mfa_batch_destroy(mfa_batch* batch);

/* ---------------- trajectory sensitivities ---------------- */

/* No counterpart in the reference.  The observable of a run of nsteps time
 * steps from the current state, J = 1/S sum_{s=1..S} [<z>(s) + <R_ee^2>(s)]
 * (<z>: mean height of all beads, unfolded through mic_count in a bulk box;
 * <R_ee^2>: mean squared end-to-end distance of the grafted/bulk chains,
 * unwrapped through mic_count), advancing the state by nsteps along the
 * subroutine-level step (verlet_positions, binning when due, fluid_fluid +
 * fluid_wall, intra_molec, bending, ewald_k(1) + dipolar_correction,
 * verlet_velocities). */
int mfa_trajectory_observable(mfa_ctx* ctx, int32_t nsteps, double* J);
/* The same run, differentiated: out[0] = J, out[1..6] = dJ/d(eps_LJ, sigma,
 * k_FENE, R0, gamma_DPD, eps_wall) by the discrete adjoint of the
 * velocity-Verlet map (hand-written vector-Jacobian products of the pair,
 * DPD, FENE, bending and 9-3 wall forces), recomputing the forward states from
 * checkpoints every `every` steps with the DPD noise replayed.  Parameters:
 * eps_LJ and sigma scale every pair's epsil and sigma (range_2 with it);
 * k_FENE and R0 enter as k_chain = k R0^2 and r_chain_2 = R0^2; gamma_DPD as
 * friction and sig = sqrt(2 kT gamma / dt); eps_wall as every type's a_wall.
 * The run starts from the context's state (r, v and a = F/m as they are) and
 * that state is held fixed: the gradient is that of the trajectory from it.
 * Every force term of the step is differentiated: LJ/WCA, DPD or Langevin
 * (gamma_DPD is then the Langevin friction, with its noise amplitude), Ewald
 * real space (either form), k-space and the slab correction (charged systems
 * need ewald_k(0) first, else MFA_ERR_STATE), FENE, bending and the 9-3 walls;
 * the Ewald parameters and k_bend are not among the parameters.  Systems with
 * the force switch-on, WALL 3/4, melt chains or DPD_VV return
 * MFA_ERR_UNSUPPORTED.  The state advances by nsteps.  The call's device
 * workspace (checkpoints, one segment's states, adjoint vectors) and its
 * captured sequences stay with the context for the next call of the same
 * nsteps and every (freed by mfa_finalize, or rebuilt when the context's
 * cells, list capacity, launch shapes or energy log change). */
int mfa_adjoint(mfa_ctx* ctx, int32_t nsteps, int32_t every, double* out7);

/* ---------------- binning without device allocation ---------------- */

/* No counterpart in the reference.  The cell binning that mfa_binning starts
 * with (binning.f90:25-50 for rule 0, my_binning.f90:26-44 for rule 1), for
 * callers that must not allocate device memory -- host programs that already
 * own all of the GPU's memory through their own pools, or that call at a point
 * where the device-wide synchronisation an allocation may imply is not
 * acceptable.  Nothing is allocated: the caller passes device buffers
 *   r0         n particles, xyz interleaved (Fortran r0(3,n)), read only
 *   cell_of    n, the cell of each particle (0-based, ix + nbx*(iy + nby*iz))
 *   cell_start n_bin[0]*n_bin[1]*n_bin[2] + 1, first slot of each cell
 *   sorted_ids n, particle ids (0-based) grouped by cell, ascending in a cell
 * and the per-cell counters live in a fixed device array inside the library of
 * at most 131072 cells (1 MiB, held by every GPU that loads the library until
 * the process exits); larger grids return MFA_ERR_CAPACITY.  All calls share
 * that array: calls whose work overlaps on the GPU race and must be serialised
 * by the caller.  boundary and n_bin are host arrays of 3; stream is a
 * cudaStream_t (NULL for the default stream).  Every call looks the array's
 * device address up on the current device (so it stays right after a
 * cudaDeviceReset); the first call on a device also loads the library's device
 * code there, so make it before any stream capture.  Any n_bin[d] or partial
 * product above the capacity returns MFA_ERR_CAPACITY.  Every call synchronises
 * `stream` before returning and reports particles outside
 * the grid (MFA_ERR_CELL_RANGE) or non-finite (MFA_ERR_NONFINITE). */
int mfa_bin_cells_noalloc(const double* r0, int32_t n, const double* boundary,
                          const int32_t* n_bin, int32_t rule, int32_t* cell_of,
                          int32_t* cell_start, int32_t* sorted_ids, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MFA_GPU_H */
