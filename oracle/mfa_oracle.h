/*
 * mfa_oracle.h -- TEST INFRASTRUCTURE.  A CPU, FP64, single-threaded
 * restatement of mfa's per-timestep force and integration loop, used only by
 * the tests, the smoke check and the CPU-baseline leg of the benchmark as the
 * checker.  It is never linked into, loaded by, or called from the product
 * library.
 *
 * Parity status: UNPINNED by reference data.  The reference (Fortran) cannot be
 * compiled in this image (no Fortran compiler) and ships no golden vectors for
 * this path; the oracle is pinned by the reference's own known-answer check
 * (util.f90:283-322, the O(N^2) energy that must equal the list energy), by
 * energy/force consistency checks and by hand-derived fixtures.
 */
#ifndef MFA_ORACLE_H
#define MFA_ORACLE_H

#include <stdint.h>
#include "../include/mfa_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

/* rng_mode: 0 = Philox-4x32-10 keyed by (step, min(i,j), max(i,j)) exactly as
 * the GPU draws it; 1 = one sequential stream in traversal order (the shape of
 * the reference's rnor(), used only for CPU timing). */
int  orc_create(const mfa_params* p, const double* r0, const double* v,
                const double* a, const int32_t* a_type, const double* mass,
                const double* q, const int32_t* mic, int bin_cap, int list_cap,
                int rng_mode, orc_state** out);
void orc_destroy(orc_state* s);
void orc_set_step(orc_state* s, int64_t i_time);
int64_t orc_get_step(const orc_state* s);

void orc_verlet_positions(orc_state* s);
int  orc_check_skin(orc_state* s);
int  orc_binning(orc_state* s);        /* returns 0 or an MFA_ERR_* code */
int  orc_my_binning(orc_state* s);
void orc_zero_forces(orc_state* s);
void orc_fluid_fluid(orc_state* s);
void orc_fluid_wall(orc_state* s, int inter_type);
void orc_intra_molec(orc_state* s);
void orc_bending(orc_state* s, int mode);
int  orc_ewald_k(orc_state* s, int mode);
void orc_dipolar_correction(orc_state* s);
void orc_verlet_velocities(orc_state* s);
/* optional terms: external_force.f90 (EXT_FORCE), orientation.f90
 * (ORIENTATION; returns v_or), and DPD_VV (new_dpd_fd.f90; orc_md_step calls
 * it after verlet_velocities once switched on) */
void orc_external_force(orc_state* s, int mode, double k_elastic);
double orc_orientation(orc_state* s, int mode, double k_or, double alpha_or);
void orc_set_dpd_vv(orc_state* s, int on);
void orc_new_dpd_fd(orc_state* s);
/* one md_main.f90:68-147 iteration in the reference's call order */
int  orc_md_step(orc_state* s);

/* O(N^2) LJ energy over all pairs (util.f90:283-322 check_fluid_fluid). */
double orc_check_fluid_fluid(orc_state* s);

void orc_get_state(const orc_state* s, double* r0, double* v, double* a,
                   double* force, int32_t* mic);
void orc_set_state(orc_state* s, const double* r0, const double* v,
                   const double* a, const double* force, const int32_t* mic);
void orc_get_scalars(const orc_state* s, mfa_scalars* out);
/* cell_of: 0-based linear cell per particle; bin_fluid/ff_list in the Fortran
 * layouts bin_fluid(0:nx-1,0:ny-1,0:nz-1,0:bin_cap), ff_list(0:list_cap,n). */
void orc_get_lists(const orc_state* s, int32_t* cell_of, int32_t* bin_fluid,
                   int32_t* ff_list);
int  orc_get_kvecs(const orc_state* s, double* kvecs3, int max_k);

/* Derived constants of init_params.f90/init_config.f90/make_binning_boxes.f90,
 * restated independently of the product's host code (for cross-checking it). */
typedef struct orc_inputs {
    int32_t n_type;
    double  eps[MFA_MAX_TYPES * MFA_MAX_TYPES];   /* as read from mfa_input */
    double  sigma_ii[MFA_MAX_TYPES];
    double  k_chain_in, r_chain, dt, temp, friction, k_bend, alpha_eq;
    double  a_w, sigma_w, boundary[3], skin;
    int32_t brush_heads;   /* SYSTEM 0,1,3: range_2(1,1)=0, range_2(1,n)=(2.2 s)^2 */
    int32_t wall93;        /* WALL 2: range_2(:,n_type) = 0 */
    int32_t binning_rule;  /* 0: int(L/(rc_max+0.4)); 1: keep n_bin_in */
    int32_t n_bin_in[3];
    int32_t n_bin_init[3]; /* the init_system.f90:273-275 values used for delta_bin */
} orc_inputs;
void orc_derive_params(const orc_inputs* in, mfa_params* out);

#ifdef __cplusplus
}
#endif
#endif
