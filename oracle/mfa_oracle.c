/*
 * mfa_oracle.c -- TEST INFRASTRUCTURE (see mfa_oracle.h).
 *
 * CPU, FP64, single-threaded restatement of the reference's per-step routines,
 * written to follow the Fortran statement by statement (same operation order,
 * same single-precision literals, same list ownership rule) so that its output
 * is what the reference would print.  Each routine cites the Fortran it
 * follows.  Build: oracle/Makefile (gcc -O2 -ffp-contract=off, no FMA).
 *
 * Parity: UNPINNED by reference data (no Fortran compiler here; the reference
 * ships no golden vectors for this path).
 */
#include "mfa_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define T8 MFA_MAX_TYPES
#define IDX(ti, tj) (((ti) - 1) * T8 + ((tj) - 1))

struct orc_state {
    mfa_params p;
    int n;
    double *r0, *v, *a, *force, *r0_old;
    int32_t *mic, *mic_old, *a_type;
    double *mass, *inv_mass, *q;
    double inv_boundary[3];
    int64_t i_time;
    int f_skin;
    /* binning (binning.f90 / my_binning.f90) */
    int nb[3], ncell;
    double r_bin[3], inv_r_bin[3];
    int bin_cap, list_cap;
    int32_t *bin_fluid;   /* cell + ncell*k, k = 0..bin_cap              */
    int32_t *ff_list;     /* k + (list_cap+1)*i, k = 0..list_cap          */
    int32_t *cell_of;
    int32_t *binpnt, *bin; /* my_binning linked cells                     */
    int bin_type;
    int n_neigh_fl_max, n_rebuilds, max_cell, max_neigh;
    /* scalars (commons) */
    double v_fluid_fluid, v_fluid_wall, v_intra_molec, v_bend, v_coul;
    double v_coul_self, t_fluid, v_total, e_total, virial;
    int fene_clamped;
    /* DPD_VV (new_dpd_fd.f90): the dissipative force of the last re-evaluation */
    int dpd_vv;
    double* force_d;
    /* Ewald k-space (ewald_k.f90 saved variables) */
    int nk;
    double *k_vecs, *k_vecs_2, *inv_k_vecs_2, *re_rho_k, *im_rho_k, *cphase;
    double fac_alpha, inv_V;
    /* noise */
    int rng_mode;
    uint32_t shr3;
    double zk_wn[128], zk_fn[128];
    uint32_t zk_kn[128];
};

/* ------------------------------------------------------------------ */
/* Counter-based noise: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw,     */
/* SC'11 "Parallel random numbers: as easy as 1, 2, 3").               */
/* ------------------------------------------------------------------ */
static void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * ctr[0];
        uint64_t p1 = (uint64_t)M1 * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
        k0 += W0; k1 += W1;
    }
}

#define TAG_DPD 0x44504400u
#define TAG_LGV 0x4C475600u

static double u01_open(uint32_t x) { return ((double)x + 0.5) * 2.3283064365386963e-10; }

/* the uniform variate built so that float arithmetic reproduces it exactly */
static float u24(uint32_t x) { return (float)(x >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f; }

static double noise_from(uint32_t x0, uint32_t x1, int shape) {
    if (shape == MFA_NOISE_UNIFORM) {
        float u = u24(x0);
        return (double)(1.7320508075688772f * (2.0f * u - 1.0f));
    }
    double u1 = u01_open(x0), u2 = u01_open(x1);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* ---- Marsaglia & Tsang (2000) ziggurat, for rng_mode 1 (timing shape only) ---- */
static uint32_t shr3(orc_state* s) {
    uint32_t j = s->shr3;
    s->shr3 ^= s->shr3 << 13; s->shr3 ^= s->shr3 >> 17; s->shr3 ^= s->shr3 << 5;
    return j + s->shr3;
}
static double uni(orc_state* s) { return 0.5 + (double)(int32_t)shr3(s) * 2.328306e-10; }
static void zig_setup(orc_state* s, uint32_t seed) {
    const double m1 = 2147483648.0;
    double dn = 3.442619855899, tn = dn, vn = 9.91256303526217e-3;
    double q = vn / exp(-0.5 * dn * dn);
    s->shr3 = seed ? seed : 123456789u;
    s->zk_kn[0] = (uint32_t)((dn / q) * m1);
    s->zk_kn[1] = 0;
    s->zk_wn[0] = q / m1;
    s->zk_wn[127] = dn / m1;
    s->zk_fn[0] = 1.0;
    s->zk_fn[127] = exp(-0.5 * dn * dn);
    for (int i = 126; i >= 1; --i) {
        dn = sqrt(-2.0 * log(vn / dn + exp(-0.5 * dn * dn)));
        s->zk_kn[i + 1] = (uint32_t)((dn / tn) * m1);
        tn = dn;
        s->zk_fn[i] = exp(-0.5 * dn * dn);
        s->zk_wn[i] = dn / m1;
    }
}
static double rnor_seq(orc_state* s) {
    int32_t hz = (int32_t)shr3(s);
    uint32_t iz = (uint32_t)hz & 127u;
    if ((uint32_t)abs(hz) < s->zk_kn[iz]) return hz * s->zk_wn[iz];
    const double r = 3.442620;
    for (;;) {
        double x = hz * s->zk_wn[iz];
        if (iz == 0) {
            double y;
            do { x = -log(uni(s)) * 0.2904764; y = -log(uni(s)); } while (y + y < x * x);
            return hz > 0 ? r + x : -r - x;
        }
        if (s->zk_fn[iz] + uni(s) * (s->zk_fn[iz - 1] - s->zk_fn[iz]) < exp(-0.5 * x * x)) return x;
        hz = (int32_t)shr3(s);
        iz = (uint32_t)hz & 127u;
        if ((uint32_t)abs(hz) < s->zk_kn[iz]) return hz * s->zk_wn[iz];
    }
}

static double pair_noise(orc_state* s, int i, int j) {
    if (s->rng_mode == 1) return rnor_seq(s);
    uint32_t c[4];
    c[0] = (uint32_t)(i < j ? i : j);
    c[1] = (uint32_t)(i < j ? j : i);
    c[2] = (uint32_t)s->i_time;
    c[3] = TAG_DPD;
    philox4x32_10(c, (uint32_t)s->p.seed, (uint32_t)(s->p.seed >> 32));
    return noise_from(c[0], c[1], s->p.noise);
}

static void particle_noise3(orc_state* s, int i, double g[3]) {
    if (s->rng_mode == 1) { g[0] = rnor_seq(s); g[1] = rnor_seq(s); g[2] = rnor_seq(s); return; }
    uint32_t c[4] = {(uint32_t)i, 0u, (uint32_t)s->i_time, TAG_LGV};
    philox4x32_10(c, (uint32_t)s->p.seed, (uint32_t)(s->p.seed >> 32));
    if (s->p.noise == MFA_NOISE_UNIFORM) {
        g[0] = noise_from(c[0], 0, 1); g[1] = noise_from(c[1], 0, 1); g[2] = noise_from(c[2], 0, 1);
        return;
    }
    double r1 = sqrt(-2.0 * log(u01_open(c[0])));
    double r2 = sqrt(-2.0 * log(u01_open(c[2])));
    g[0] = r1 * cos(6.283185307179586 * u01_open(c[1]));
    g[1] = r1 * sin(6.283185307179586 * u01_open(c[1]));
    g[2] = r2 * cos(6.283185307179586 * u01_open(c[3]));
}

/* ------------------------------------------------------------------ */
/* lifetime                                                            */
/* ------------------------------------------------------------------ */
static void* xcalloc(size_t n, size_t sz) { void* p = calloc(n ? n : 1, sz); return p; }

static void setup_cells(orc_state* s) {
    /* make_binning_boxes.f90:57-64 */
    for (int d = 0; d < 3; ++d) {
        s->nb[d] = s->p.n_bin[d];
        s->r_bin[d] = s->p.boundary[d] / (double)s->nb[d];
        s->inv_r_bin[d] = 1.0 / s->r_bin[d];
    }
    s->ncell = s->nb[0] * s->nb[1] * s->nb[2];
}

int orc_create(const mfa_params* p, const double* r0, const double* v,
               const double* a, const int32_t* a_type, const double* mass,
               const double* q, const int32_t* mic, int bin_cap, int list_cap,
               int rng_mode, orc_state** out) {
    if (!p || !out || p->n_part <= 0) return MFA_ERR_ARGS;
    orc_state* s = (orc_state*)xcalloc(1, sizeof(orc_state));
    s->p = *p;
    int n = s->n = p->n_part;
    s->r0 = xcalloc(3 * n, 8); s->v = xcalloc(3 * n, 8); s->a = xcalloc(3 * n, 8);
    s->force = xcalloc(3 * n, 8); s->r0_old = xcalloc(3 * n, 8);
    s->mic = xcalloc(3 * n, 4); s->mic_old = xcalloc(3 * n, 4);
    s->a_type = xcalloc(n, 4); s->mass = xcalloc(n, 8); s->inv_mass = xcalloc(n, 8);
    s->q = xcalloc(n, 8); s->cell_of = xcalloc(n, 4);
    memcpy(s->r0, r0, 24 * (size_t)n);
    if (v) memcpy(s->v, v, 24 * (size_t)n);
    if (a) memcpy(s->a, a, 24 * (size_t)n);
    if (mic) memcpy(s->mic, mic, 12 * (size_t)n);
    memcpy(s->a_type, a_type, 4 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        s->mass[i] = mass[i];
        s->inv_mass[i] = 1.0 / mass[i];
        s->q[i] = q ? q[i] : 0.0;
    }
    for (int d = 0; d < 3; ++d) s->inv_boundary[d] = 1.0 / p->boundary[d]; /* init_config.f90:20 */
    setup_cells(s);
    s->bin_cap = bin_cap > 0 ? bin_cap : 300;    /* n_bin_fl, mfa_common.f90:76 */
    s->list_cap = list_cap > 0 ? list_cap : 256; /* n_neigh_fl, mfa_common.f90:78 */
    s->bin_fluid = xcalloc((size_t)s->ncell * (s->bin_cap + 1), 4);
    s->ff_list = xcalloc((size_t)n * (s->list_cap + 1), 4);
    s->binpnt = xcalloc(s->ncell + 1, 4);
    s->bin = xcalloc(n, 4);
    s->rng_mode = rng_mode;
    zig_setup(s, (uint32_t)p->seed);
    /* init_config.f90:235-239 self energy (uses sqrt(pi) with the single-precision pi) */
    if (p->charged) {
        double vs = 0.0;
        for (int i = 0; i < n; ++i) vs = vs - s->q[i] * s->q[i];
        s->v_coul_self = vs * p->sqrt_alpha / sqrt(p->pi);
    }
    *out = s;
    return MFA_OK;
}

void orc_destroy(orc_state* s) {
    if (!s) return;
    free(s->r0); free(s->v); free(s->a); free(s->force); free(s->r0_old);
    free(s->mic); free(s->mic_old); free(s->a_type); free(s->mass); free(s->inv_mass);
    free(s->q); free(s->cell_of); free(s->bin_fluid); free(s->ff_list);
    free(s->binpnt); free(s->bin); free(s->force_d);
    free(s->k_vecs); free(s->k_vecs_2); free(s->inv_k_vecs_2);
    free(s->re_rho_k); free(s->im_rho_k); free(s->cphase);
    free(s);
}

void orc_set_step(orc_state* s, int64_t t) { s->i_time = t; }
int64_t orc_get_step(const orc_state* s) { return s->i_time; }

/* minimum image of binning.f90:89-93 / fluid_fluid.f90:84-88: d - L*int(2d/L) */
static inline double mimage(double d, double L, double invL) {
    return d - L * (double)(int32_t)(2.0 * d * invL);
}

/* ------------------------------------------------------------------ */
/* verlet_positions.f90:146-171 (update) and :237-251 (wrap)           */
/* ------------------------------------------------------------------ */
void orc_verlet_positions(orc_state* s) {
    const double dt = s->p.dt, dt_2 = dt * dt;
    s->i_time += 1; /* md_main.f90:68 loop counter */
    for (int i = 0; i < s->n; ++i) {
        for (int d = 0; d < 3; ++d) {
            double* r = &s->r0[3 * i + d];
            *r = (*r + dt * s->v[3 * i + d]) + (0.5 * dt_2) * s->a[3 * i + d];
            s->v[3 * i + d] = s->v[3 * i + d] + (0.5 * dt) * s->a[3 * i + d];
        }
    }
    int nd = s->p.symmetry == 1 ? 3 : 2;
    for (int i = 0; i < s->n; ++i) {
        for (int d = 0; d < nd; ++d) {
            double* r = &s->r0[3 * i + d];
            if (*r > s->p.boundary[d]) {
                *r = *r - s->p.boundary[d];
                s->mic[3 * i + d] += 1;
            } else if (*r < 0.0) {
                *r = *r + s->p.boundary[d];
                s->mic[3 * i + d] -= 1;
            }
        }
    }
}

/* check_skin.f90:8-21 */
int orc_check_skin(orc_state* s) {
    const double lim = (s->p.skin / 2.0) * (s->p.skin / 2.0);
    for (int i = 0; i < s->n; ++i) {
        double dr[3];
        for (int d = 0; d < 3; ++d)
            dr[d] = ((s->r0_old[3 * i + d] + s->mic_old[3 * i + d] * s->p.boundary[d]) - s->r0[3 * i + d])
                    - s->mic[3 * i + d] * s->p.boundary[d];
        double r_dummy = 0.0;
        for (int d = 0; d < 3; ++d) r_dummy = r_dummy + dr[d] * dr[d];
        if (r_dummy > lim) s->f_skin = 1;
    }
    return s->f_skin;
}

/* List criterion of binning.f90:104: range_2(ti,tj) + skin_2.  With the
 * real-space Ewald cutoff decoupled from the LJ range (the corrected mode; the
 * reference always evaluates it inside range_2), pairs out to rc_ewald + skin
 * are listed as well. */
static double list_cut2(const mfa_params* p, int ti, int tj) {
    double c2 = p->range_2[IDX(ti, tj)] + p->skin_2;
    if (p->charged && !(p->quirks & MFA_Q_EWALD_REAL_IN_LJ)) {
        const double re = sqrt(p->ewald_rc_2) + p->skin;
        if (re * re > c2) c2 = re * re;
    }
    return c2;
}

static void snapshot_old(orc_state* s) {
    s->f_skin = 0;
    memcpy(s->r0_old, s->r0, 24 * (size_t)s->n);
    memcpy(s->mic_old, s->mic, 12 * (size_t)s->n);
    s->n_rebuilds += 1;
}

/* ------------------------------------------------------------------ */
/* binning.f90:2-131 (BIN_TYPE 0)                                       */
/* ------------------------------------------------------------------ */
int orc_binning(orc_state* s) {
    const int nx = s->nb[0], ny = s->nb[1], nz = s->nb[2], nc = s->ncell;
    const int cap = s->bin_cap, lcap = s->list_cap;
    int err = 0;
    s->bin_type = 0;
    memset(s->bin_fluid, 0, sizeof(int32_t) * (size_t)nc * (cap + 1));
    for (int i = 0; i < s->n; ++i) {
        /* binning.f90:27-29: mod(int(r*inv_r_bin), n_bin) */
        int ix = (int32_t)(s->r0[3 * i + 0] * s->inv_r_bin[0]) % nx;
        int iy = (int32_t)(s->r0[3 * i + 1] * s->inv_r_bin[1]) % ny;
        int iz = (int32_t)(s->r0[3 * i + 2] * s->inv_r_bin[2]) % nz;
        if (ix < 0 || iy < 0 || iz < 0) { err = MFA_ERR_CELL_RANGE; s->cell_of[i] = -1; continue; }
        int c = ix + nx * (iy + ny * iz);
        s->cell_of[i] = c;
        int cnt = ++s->bin_fluid[c];
        if (cnt > cap) { err = MFA_ERR_CELL_RANGE; continue; }
        s->bin_fluid[c + nc * cnt] = i + 1;
    }
    s->max_cell = 0;
    for (int c = 0; c < nc; ++c) if (s->bin_fluid[c] > s->max_cell) s->max_cell = s->bin_fluid[c];
    if (s->max_cell > cap) return MFA_ERR_CELL_RANGE;
    for (int i = 0; i < s->n; ++i) {
        int* row = &s->ff_list[(size_t)(lcap + 1) * i];
        if (row[0] > s->n_neigh_fl_max) s->n_neigh_fl_max = row[0];
        row[0] = 0;
    }
    const int* dl = s->p.delta_bin;
    for (int bz = 0; bz < nz; ++bz)
    for (int by = 0; by < ny; ++by)
    for (int bx = 0; bx < nx; ++bx) {
        int c = bx + nx * (by + ny * bz);
        int n1 = s->bin_fluid[c];
        for (int k1 = 1; k1 <= n1; ++k1) {
            int ip = s->bin_fluid[c + nc * k1];           /* 1-based */
            int ti = s->a_type[ip - 1];
            for (int jx = bx - 1; jx <= bx + dl[0]; ++jx) {
                int kx = (jx + nx) % nx;
                for (int jy = by - 1; jy <= by + dl[1]; ++jy) {
                    int ky = (jy + ny) % ny;
                    for (int jz = bz - 1; jz <= bz + dl[2]; ++jz) {
                        int kz = (jz + nz) % nz;
                        int c2 = kx + nx * (ky + ny * kz);
                        int n2 = s->bin_fluid[c2];
                        for (int k2 = 1; k2 <= n2; ++k2) {
                            int jp = s->bin_fluid[c2 + nc * k2];
                            if (ip < jp) {
                                int tj = s->a_type[jp - 1];
                                const double* ri = &s->r0[3 * (ip - 1)];
                                const double* rj = &s->r0[3 * (jp - 1)];
                                double d0 = ri[0] - rj[0], d1 = ri[1] - rj[1], d2 = ri[2] - rj[2];
                                d0 = d0 - s->p.boundary[0] * (double)(int32_t)(2.0 * d0 * s->inv_boundary[0]);
                                d1 = d1 - s->p.boundary[1] * (double)(int32_t)(2.0 * d1 * s->inv_boundary[1]);
                                if (s->p.symmetry == 1)
                                    d2 = d2 - s->p.boundary[2] * (double)(int32_t)(2.0 * d2 * s->inv_boundary[2]);
                                double r_2 = 0.0;
                                r_2 = r_2 + d0 * d0;
                                r_2 = r_2 + d1 * d1;
                                r_2 = r_2 + d2 * d2;
                                if (r_2 < list_cut2(&s->p, ti, tj)) {
                                    /* binning.f90:106-112: append to the shorter row */
                                    int* rowi = &s->ff_list[(size_t)(lcap + 1) * (ip - 1)];
                                    int* rowj = &s->ff_list[(size_t)(lcap + 1) * (jp - 1)];
                                    if (rowi[0] <= rowj[0]) {
                                        if (rowi[0] >= lcap) { err = MFA_ERR_NEIGH_OVERFLOW; continue; }
                                        rowi[0] += 1; rowi[rowi[0]] = jp;
                                    } else {
                                        if (rowj[0] >= lcap) { err = MFA_ERR_NEIGH_OVERFLOW; continue; }
                                        rowj[0] += 1; rowj[rowj[0]] = ip;
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
    }
    s->max_neigh = 0;
    for (int i = 0; i < s->n; ++i) {
        int c = s->ff_list[(size_t)(lcap + 1) * i];
        if (c > s->max_neigh) s->max_neigh = c;
    }
    snapshot_old(s);
    return err;
}

/* ------------------------------------------------------------------ */
/* my_binning.f90:22-131 (BIN_TYPE 1): linked cells, full list          */
/* ------------------------------------------------------------------ */
int orc_my_binning(orc_state* s) {
    const int nx = s->nb[0], ny = s->nb[1], nz = s->nb[2], nc = s->ncell;
    const int lcap = s->list_cap;
    int err = 0;
    s->bin_type = 1;
    for (int i = 0; i < s->n; ++i) s->ff_list[(size_t)(lcap + 1) * i] = 0;
    memset(s->binpnt, 0, sizeof(int32_t) * (size_t)(nc + 1));
    memset(s->bin, 0, sizeof(int32_t) * (size_t)s->n);
    for (int i = 0; i < s->n; ++i) {
        int ix = (int32_t)(s->r0[3 * i + 0] / s->r_bin[0]);
        int iy = (int32_t)(s->r0[3 * i + 1] / s->r_bin[1]);
        int iz = (int32_t)(s->r0[3 * i + 2] / s->r_bin[2]);
        if (ix < 0 || iy < 0 || iz < 0 || ix >= nx || iy >= ny || iz >= nz) {
            err = MFA_ERR_CELL_RANGE; s->cell_of[i] = -1; continue;
        }
        int ib = iz * nx * ny + iy * nx + ix;
        s->cell_of[i] = ib;
        s->bin[i] = s->binpnt[ib];
        s->binpnt[ib] = i + 1;
    }
    if (err) return err;
    for (int i = 0; i < s->n; ++i) {
        int ti = s->a_type[i];
        int ixx = (int32_t)(s->r0[3 * i + 0] / s->r_bin[0]);
        int iyy = (int32_t)(s->r0[3 * i + 1] / s->r_bin[1]);
        int izz = (int32_t)(s->r0[3 * i + 2] / s->r_bin[2]);
        int* row = &s->ff_list[(size_t)(lcap + 1) * i];
        for (int k = 0; k <= 26; ++k) {
            int ix = ixx + k % 3 - 1; if (ix < 0) ix = nx - 1; if (ix == nx) ix = 0;
            int iy = iyy + (k / 3) % 3 - 1; if (iy < 0) iy = ny - 1; if (iy == ny) iy = 0;
            int iz = izz + k / 9 - 1; if (iz < 0) iz = nz - 1; if (iz == nz) iz = 0;
            int ib = iz * nx * ny + iy * nx + ix;
            int jp = s->binpnt[ib];
            while (jp != 0) {
                int tj = s->a_type[jp - 1];
                double dr[3];
                for (int d = 0; d < 3; ++d) dr[d] = s->r0[3 * i + d] - s->r0[3 * (jp - 1) + d];
                int nd = s->p.symmetry == 1 ? 3 : 2;
                for (int d = 0; d < nd; ++d)
                    dr[d] = dr[d] - s->p.boundary[d] * (double)(int32_t)(2.0 * dr[d] * s->inv_boundary[d]);
                double dr_2 = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
                if (dr_2 < list_cut2(&s->p, ti, tj) && (i + 1) != jp) {
                    if (row[0] >= lcap) err = MFA_ERR_NEIGH_OVERFLOW;
                    else { row[0] += 1; row[row[0]] = jp; }
                }
                jp = s->bin[jp - 1];
            }
        }
    }
    s->max_neigh = 0;
    for (int i = 0; i < s->n; ++i) {
        int c = s->ff_list[(size_t)(lcap + 1) * i];
        if (c > s->max_neigh) s->max_neigh = c;
    }
    snapshot_old(s);
    return err;
}

void orc_zero_forces(orc_state* s) { memset(s->force, 0, 24 * (size_t)s->n); }

/* ------------------------------------------------------------------ */
/* fluid_fluid.f90:1-254 with dpd_forces.f90:1-98 (THERMOSTAT 0),     */
/* lgv_forces.f90:1-44 (THERMOSTAT 1), ewald_real.f90:1-41         */
/* ------------------------------------------------------------------ */
void orc_fluid_fluid(orc_state* s) {
    const mfa_params* p = &s->p;
    const int lcap = s->list_cap;
    const int bt = s->bin_type;
    const double r_time = (double)(p->s_time + s->i_time - 1) * p->dt; /* md_main.f90:69 */
    double r_2_min = 0.0;
    if (p->force_switch_on) { /* fluid_fluid.f90:42-49 */
        if (r_time < p->r_2_min_time) r_2_min = (1.0 - r_time / p->r_2_min_time) * p->r_2_min_init;
        else r_2_min = 0.0;
    }
    double v_ff = 0.0, v_coul = 0.0, vir = 0.0;
    const int real_in_lj = (p->quirks & MFA_Q_EWALD_REAL_IN_LJ) != 0;
    for (int i = 0; i < s->n; ++i) {
        const int ti = s->a_type[i];
        const int* row = &s->ff_list[(size_t)(lcap + 1) * i];
        const int nn = row[0];
        double f_ipart[3] = {0.0, 0.0, 0.0};
        for (int k = 1; k <= nn; ++k) {
            const int j = row[k] - 1;
            const int tj = s->a_type[j];
            const double r_cut2 = p->range_2[IDX(ti, tj)];
            double dr[3];
            dr[0] = s->r0[3 * i + 0] - s->r0[3 * j + 0];
            dr[1] = s->r0[3 * i + 1] - s->r0[3 * j + 1];
            dr[2] = s->r0[3 * i + 2] - s->r0[3 * j + 2];
            dr[0] = dr[0] - p->boundary[0] * (double)(int32_t)(2.0 * dr[0] * s->inv_boundary[0]);
            dr[1] = dr[1] - p->boundary[1] * (double)(int32_t)(2.0 * dr[1] * s->inv_boundary[1]);
            if (p->symmetry == 1)
                dr[2] = dr[2] - p->boundary[2] * (double)(int32_t)(2.0 * dr[2] * s->inv_boundary[2]);
            double r_2 = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
            const double r_2_raw = r_2;
            if (r_2 < r_cut2) {
                if (p->force_switch_on) r_2 = fmax(r_2, r_2_min);
                const double inv_r_2 = 1.0 / r_2;
                const double inv_sqrt_r_2 = sqrt(1.0 / r_2);
                const double l_eps = p->epsil[IDX(ti, tj)];
                const double r_61 = p->sigma_2[IDX(ti, tj)] * inv_r_2;
                const double r_6 = (r_61 * r_61) * r_61;
                const double r_12 = r_6 * r_6;
                const double pot_loc = (r_12 - r_6) - p->e_shift[IDX(ti, tj)];
                v_ff = v_ff + l_eps * pot_loc;
                const double r_dummy = (l_eps * (-12.0 * r_12 + 6.0 * r_6)) * inv_r_2;
                double fl[3] = {r_dummy * dr[0], r_dummy * dr[1], r_dummy * dr[2]};
                if (bt == 0) {
                    f_ipart[0] = f_ipart[0] - fl[0];
                    f_ipart[1] = f_ipart[1] - fl[1];
                    f_ipart[2] = f_ipart[2] - fl[2];
                }
                s->force[3 * j + 0] += fl[0];
                s->force[3 * j + 1] += fl[1];
                s->force[3 * j + 2] += fl[2];
                vir = vir - r_dummy * r_2_raw;
                if (p->thermostat == MFA_THERMO_DPD) {
                    /* dpd_forces.f90:19-94 */
                    const double g_rand = pair_noise(s, i, j);
                    double w_d, w_r;
                    if (p->dpd_weight == 1) { w_d = 1.0; w_r = 1.0; }
                    else {
                        w_d = 1.0 - sqrt(r_2 * p->inv_range_2[IDX(ti, tj)]);
                        w_r = w_d;
                        w_d = w_d * w_d;
                    }
                    double rv[3] = {dr[0] * inv_sqrt_r_2, dr[1] * inv_sqrt_r_2, dr[2] * inv_sqrt_r_2};
                    double vd[3];
                    for (int d = 0; d < 3; ++d) vd[d] = ((p->sig * w_r) * g_rand) * rv[d];
                    if (bt == 0 || i > j) {
                        for (int d = 0; d < 3; ++d) { s->force[3 * i + d] += vd[d]; s->force[3 * j + d] -= vd[d]; }
                    }
                    double dv[3];
                    for (int d = 0; d < 3; ++d) dv[d] = s->v[3 * i + d] - s->v[3 * j + d];
                    const double rd = (dv[0] * rv[0] + dv[1] * rv[1]) + dv[2] * rv[2];
                    for (int d = 0; d < 3; ++d) vd[d] = (((-1.0 * p->friction) * w_d) * rd) * rv[d];
                    for (int d = 0; d < 3; ++d) s->force[3 * i + d] += vd[d];
                    if (bt == 0) for (int d = 0; d < 3; ++d) s->force[3 * j + d] -= vd[d];
                }
                if (p->charged && real_in_lj) {
                    /* ewald_real.f90:15-33 */
                    const double r = sqrt(r_2);
                    const double inv_r = 1.0 / r;
                    const double qq = s->q[i] * s->q[j];
                    const double ec = erfc(p->sqrt_alpha * r);
                    v_coul = v_coul + (qq * ec) * inv_r;
                    const double f_scal = (((qq * p->sqrt_alpha) * p->inv_sqrt_pi) * 2.0) * exp(-p->alpha_c * r_2) * inv_r
                                          + ((qq * ec) * inv_r) * inv_r;
                    for (int d = 0; d < 3; ++d) {
                        const double fc = (f_scal * dr[d]) * inv_r;
                        s->force[3 * i + d] += fc;
                        if (bt == 0) s->force[3 * j + d] -= fc;
                    }
                    vir = vir + f_scal * r_2_raw * inv_r;
                }
            }
            if (p->charged && !real_in_lj && r_2_raw < p->ewald_rc_2) {
                /* corrected mode: the real-space sum with its own cutoff */
                const double r = sqrt(r_2_raw);
                const double inv_r = 1.0 / r;
                const double qq = s->q[i] * s->q[j];
                const double ec = erfc(p->sqrt_alpha * r);
                v_coul = v_coul + (qq * ec) * inv_r;
                const double f_scal = (((qq * p->sqrt_alpha) * p->inv_sqrt_pi) * 2.0) * exp(-p->alpha_c * r_2_raw) * inv_r
                                      + ((qq * ec) * inv_r) * inv_r;
                for (int d = 0; d < 3; ++d) {
                    const double fc = (f_scal * dr[d]) * inv_r;
                    s->force[3 * i + d] += fc;
                    if (bt == 0) s->force[3 * j + d] -= fc;
                }
                vir = vir + f_scal * r_2_raw * inv_r;
            }
        }
        if (bt == 0) {
            s->force[3 * i + 0] += f_ipart[0];
            s->force[3 * i + 1] += f_ipart[1];
            s->force[3 * i + 2] += f_ipart[2];
        }
        if (p->thermostat == MFA_THERMO_LGV) {
            /* lgv_forces.f90:22-41 */
            double g[3];
            particle_noise3(s, i, g);
            const double sm = sqrt(s->mass[i]);
            for (int d = 0; d < 3; ++d) {
                double vd = (p->sig * g[d]) * sm;
                vd = vd - (p->friction * s->mass[i]) * s->v[3 * i + d];
                s->force[3 * i + d] += vd;
            }
        }
    }
    if (bt == 1) { v_ff = 0.5 * v_ff; vir = 0.5 * vir; } /* fluid_fluid.f90:236 */
    s->v_fluid_fluid = v_ff;
    s->virial = vir;
    if (p->charged) s->v_coul = v_coul + s->v_coul_self; /* fluid_fluid.f90:17,239 */
}

/* integer powers evaluated by one fixed multiplication chain */
static inline double pw3(double x) { return (x * x) * x; }
static inline double pw4(double x) { double x2 = x * x; return x2 * x2; }
static inline double pw9(double x) { double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4; return x8 * x; }
static inline double pw10(double x) { double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4; return x8 * x2; }

/* one 9-3 wall term: energy and the force along +z for inverse distance inv_z */
static void wall93(const mfa_params* p, int t, double inv_z, double* e, double* f) {
    const double sw = p->sigma_wall[t - 1], aw = p->a_wall[t - 1];
    const double rd = sw * inv_z;
    const double a_e = (p->quirks & MFA_Q_WALL_ENERGY_AW) ? p->a_w : aw;
    *e = fabs(aw) * pw9(rd) - a_e * pw3(rd);
    *f = (9.0 * fabs(aw)) * pw9(sw) * pw10(inv_z) - (3.0 * aw) * pw3(sw) * pw4(inv_z);
}

/* fluid_wall.f90:2-204 */
void orc_fluid_wall(orc_state* s, int inter_type) {
    const mfa_params* p = &s->p;
    double vfw = 0.0;
    if (inter_type == 2 || inter_type == 3) {
        for (int i = 0; i < s->n; ++i) {
            const int t = s->a_type[i];
            const double z = s->r0[3 * i + 2];
            double e, f;
            /* bottom wall: fluid_wall.f90:96-101 */
            if (p->wall_cut <= 0.0 || z < p->wall_cut) {
                wall93(p, t, 1.0 / z, &e, &f);
                if (p->wall_cut > 0.0) { double ec, fc; wall93(p, t, 1.0 / p->wall_cut, &ec, &fc); e -= ec; }
                vfw = vfw + e;
                s->force[3 * i + 2] += f;
            }
            if (inter_type == 2) {
                /* top wall: fluid_wall.f90:113-121 */
                const double zt = p->z_space_wall - z;
                if (p->wall_cut <= 0.0 || zt < p->wall_cut) {
                    wall93(p, t, 1.0 / zt, &e, &f);
                    if (p->wall_cut > 0.0) { double ec, fc; wall93(p, t, 1.0 / p->wall_cut, &ec, &fc); e -= ec; }
                    vfw = vfw + e;
                    s->force[3 * i + 2] -= f;
                }
            } else {
                /* fluid_wall.f90:159-161 hard top wall */
                if (z > (p->z_space_wall - p->z_head) && s->v[3 * i + 2] > 0.0) s->v[3 * i + 2] = -s->v[3 * i + 2];
            }
        }
    } else if (inter_type == 4) {
        /* fluid_wall.f90:170-180; 0.01 is a single-precision literal */
        const double eps01 = (double)0.01f;
        for (int i = 0; i < s->n; ++i) {
            const double z = s->r0[3 * i + 2];
            if (z < eps01 && s->v[3 * i + 2] < 0.0) s->v[3 * i + 2] = -s->v[3 * i + 2];
            if (z > (p->z_space_wall - eps01) && s->v[3 * i + 2] > 0.0) s->v[3 * i + 2] = -s->v[3 * i + 2];
        }
    }
    s->v_fluid_wall = vfw;
}

/* FENE term of intra_molec.f90:21-59; returns the pot_loc sum contribution */
static double fene_bond(orc_state* s, int ip, int jp, double k, int pbc_z) {
    const mfa_params* p = &s->p;
    double dr[3];
    for (int d = 0; d < 3; ++d) dr[d] = s->r0[3 * ip + d] - s->r0[3 * jp + d];
    dr[0] = dr[0] - p->boundary[0] * (double)(int32_t)(2.0 * dr[0] * s->inv_boundary[0]);
    dr[1] = dr[1] - p->boundary[1] * (double)(int32_t)(2.0 * dr[1] * s->inv_boundary[1]);
    if (pbc_z) dr[2] = dr[2] - p->boundary[2] * (double)(int32_t)(2.0 * dr[2] * s->inv_boundary[2]);
    double r_2 = 0.0;
    for (int d = 0; d < 3; ++d) r_2 = r_2 + dr[d] * dr[d];
    double x = r_2 * p->inv_r_chain_2;
    if (x >= p->fene_clamp) { s->fene_clamped += 1; x = p->fene_clamp; }
    const double pot_loc = -0.5 * log(1.0 - x);
    const double r_dummy = (k / (1.0 - x)) * p->inv_r_chain_2;
    for (int d = 0; d < 3; ++d) {
        const double fl = r_dummy * dr[d];
        s->force[3 * ip + d] -= fl;
        s->force[3 * jp + d] += fl;
    }
    return pot_loc;
}

/* intra_molec.f90:12-139,269-273,537 (grafted chains with k_chain; melt chains with k_ring) */
void orc_intra_molec(orc_state* s) {
    const mfa_params* p = &s->p;
    s->fene_clamped = 0;
    double v = 0.0;
    for (int c = 0; c < p->n_chain; ++c)
        for (int m = 0; m < p->n_mon - 1; ++m) {
            int ip = c * p->n_mon + m;
            v = v + fene_bond(s, ip, ip + 1, p->k_chain, p->symmetry == 1);
        }
    const double v_brush = p->k_chain * v;
    double vd = 0.0;
    const int part_init_d = p->n_mon * p->n_chain;
    for (int c = 0; c < p->n_chain_d; ++c)
        for (int m = 0; m < p->n_mon_d - 1; ++m) {
            int ip = part_init_d + c * p->n_mon_d + m;
            vd = vd + fene_bond(s, ip, ip + 1, p->k_ring, p->symmetry == 1);
        }
    /* intra_molec.f90:270 multiplies the melt sum by k_chain for SYSTEM != 4 */
    s->v_intra_molec = v_brush + p->k_chain * vd;
}

/* bending.f90:32-127 (mode 2) */
void orc_bending(orc_state* s, int mode) {
    if (mode != 2) return;
    const mfa_params* p = &s->p;
    const double tiny = (double)0.0000001f;
    double v_bend = 0.0;
    for (int l = 0; l < p->n_chain; ++l) {
        const int base = l * p->n_mon;
        double r_next[3], r_prev[3];
        for (int d = 0; d < 3; ++d) {
            r_next[d] = s->r0[3 * (base + 1) + d] - s->r0[3 * base + d];
            r_next[d] = r_next[d] - p->boundary[d] * (double)(int32_t)(2.0 * r_next[d] * s->inv_boundary[d]);
        }
        for (int i = 2; i <= p->n_mon - 1; ++i) {
            double dot_pr = 0.0, r_prev_2 = 0.0, r_next_2 = 0.0, dp2 = 0.0, dn2 = 0.0;
            for (int d = 0; d < 3; ++d) r_prev[d] = r_next[d];
            for (int d = 0; d < 3; ++d) {
                r_next[d] = s->r0[3 * (base + i) + d] - s->r0[3 * (base + i - 1) + d];
                r_next[d] = r_next[d] - p->boundary[d] * (double)(int32_t)(2.0 * r_next[d] * s->inv_boundary[d]);
            }
            for (int d = 0; d < 3; ++d) {
                dot_pr = dot_pr + r_next[d] * r_prev[d];
                r_prev_2 = r_prev_2 + r_prev[d] * r_prev[d];
                r_next_2 = r_next_2 + r_next[d] * r_next[d];
            }
            const double cos_alpha = dot_pr / sqrt(r_prev_2 * r_next_2);
            double dir_next[3], dir_prev[3];
            for (int d = 0; d < 3; ++d) {
                dir_next[d] = r_prev[d] * r_next_2 - r_next[d] * dot_pr;
                dir_prev[d] = -r_next[d] * r_prev_2 + r_prev[d] * dot_pr;
            }
            for (int d = 0; d < 3; ++d) {
                dp2 = dp2 + dir_prev[d] * dir_prev[d];
                dn2 = dn2 + dir_next[d] * dir_next[d];
            }
            if (dn2 < tiny) { for (int d = 0; d < 3; ++d) dir_next[d] = dir_next[d] * 0.0; }
            else { const double nn = sqrt(dn2 * r_next_2); for (int d = 0; d < 3; ++d) dir_next[d] = dir_next[d] / nn; }
            if (dp2 < tiny) { for (int d = 0; d < 3; ++d) dir_prev[d] = dir_prev[d] * 0.0; }
            else { const double nn = sqrt(dp2 * r_prev_2); for (int d = 0; d < 3; ++d) dir_prev[d] = dir_prev[d] / nn; }
            double delta_alpha;
            if (cos_alpha >= 1.0) delta_alpha = 0.0;
            else delta_alpha = acos(cos_alpha) - p->alpha_eq;
            const double F_mod = p->k_bend * delta_alpha;
            v_bend = v_bend + (0.5 * F_mod) * delta_alpha;
            for (int d = 0; d < 3; ++d) {
                const double fp = F_mod * dir_prev[d], fn = F_mod * dir_next[d];
                s->force[3 * (base + i - 2) + d] += fp;
                s->force[3 * (base + i - 1) + d] = (s->force[3 * (base + i - 1) + d] - fp) - fn;
                s->force[3 * (base + i) + d] += fn;
            }
        }
    }
    s->v_bend = v_bend;
}

/* ------------------------------------------------------------------ */
/* ewald_k.f90:1-211                                                    */
/* ------------------------------------------------------------------ */
static int ewald_init(orc_state* s) {
    const mfa_params* p = &s->p;
    double delta_k[3], z_slab;
    const double pi = p->pi;
    if (p->symmetry == 1) {
        for (int d = 0; d < 3; ++d) delta_k[d] = (2.0 * pi) * s->inv_boundary[d];
        z_slab = 0.0;
    } else {
        z_slab = 2.0;
        delta_k[0] = (2.0 * pi) * s->inv_boundary[0];
        delta_k[1] = (2.0 * pi) * s->inv_boundary[1];
        delta_k[2] = (2.0 * pi) / (p->boundary[2] + z_slab * p->boundary[2]);
    }
    const double k_c = ((delta_k[0] + delta_k[1]) * (double)p->n_kmax) / 2.0;
    const int nkx = (int32_t)(k_c / delta_k[0]);
    const int nky = (int32_t)(k_c / delta_k[1]);
    const int nkz = (int32_t)(k_c / delta_k[2]);
    const double kc2 = k_c * k_c;
    int nk = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int idx = 0;
        for (int z = 0; z <= nkz; ++z)
        for (int y = -nky; y <= nky; ++y)
        for (int x = -nkx; x <= nkx; ++x) {
            const double a0 = (double)x * delta_k[0], a1 = (double)y * delta_k[1], a2 = (double)z * delta_k[2];
            const double rk_2 = (a0 * a0 + a1 * a1) + a2 * a2;
            if (rk_2 > kc2) continue;
            if (z == 0 && y == 0 && x == 0) continue;
            if (z == 0 && x + y < 0) continue;
            if (z == 0 && -x == y && y > 0) continue;
            if (pass == 1) {
                s->k_vecs[3 * idx + 0] = a0;
                s->k_vecs[3 * idx + 1] = a1;
                s->k_vecs[3 * idx + 2] = a2;
                s->k_vecs_2[idx] = (a0 * a0 + a1 * a1) + a2 * a2;
                s->inv_k_vecs_2[idx] = 1.0 / s->k_vecs_2[idx];
            }
            ++idx;
        }
        if (pass == 0) {
            nk = idx;
            s->nk = nk;
            free(s->k_vecs); free(s->k_vecs_2); free(s->inv_k_vecs_2);
            free(s->re_rho_k); free(s->im_rho_k); free(s->cphase);
            s->k_vecs = xcalloc(3 * (size_t)nk, 8);
            s->k_vecs_2 = xcalloc(nk, 8);
            s->inv_k_vecs_2 = xcalloc(nk, 8);
            s->re_rho_k = xcalloc(nk, 8);
            s->im_rho_k = xcalloc(nk, 8);
            s->cphase = xcalloc((size_t)nk * s->n, 8);
            if (!s->cphase) return MFA_ERR_NOMEM;
        }
    }
    s->fac_alpha = 1.0 / (4.0 * p->alpha_c);
    s->inv_V = (s->inv_boundary[0] * s->inv_boundary[1]) / (p->boundary[2] * (1.0 + z_slab));
    return MFA_OK;
}

int orc_ewald_k(orc_state* s, int mode) {
    const mfa_params* p = &s->p;
    if (!p->charged) return MFA_OK;
    if (mode == 0) return ewald_init(s);
    if (s->nk == 0) return MFA_ERR_STATE;
    const int nk = s->nk, n = s->n;
    double u = 0.0;
    for (int k = 0; k < nk; ++k) { s->re_rho_k[k] = 0.0; s->im_rho_k[k] = 0.0; }
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < nk; ++k) {
            const double* kv = &s->k_vecs[3 * k];
            const double lphase = (kv[0] * s->r0[3 * i] + kv[1] * s->r0[3 * i + 1]) + kv[2] * s->r0[3 * i + 2];
            s->cphase[(size_t)k * n + i] = lphase;
            s->re_rho_k[k] = s->re_rho_k[k] + s->q[i] * cos(lphase);
            s->im_rho_k[k] = s->im_rho_k[k] + s->q[i] * sin(lphase);
        }
    }
    for (int k = 0; k < nk; ++k)
        u = u + (s->inv_k_vecs_2[k] * exp(-s->k_vecs_2[k] * s->fac_alpha))
                * (s->re_rho_k[k] * s->re_rho_k[k] + s->im_rho_k[k] * s->im_rho_k[k]);
    u = ((u * 4.0) * p->pi) * s->inv_V;
    for (int i = 0; i < n; ++i) {
        double fk[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < nk; ++k) {
            const double ph = s->cphase[(size_t)k * n + i];
            const double sc = cos(ph) * s->im_rho_k[k] - sin(ph) * s->re_rho_k[k];
            for (int d = 0; d < 3; ++d) fk[d] = fk[d] + ((s->k_vecs[3 * k + d] * s->inv_k_vecs_2[k]) * exp(-s->k_vecs_2[k] * s->fac_alpha)) * sc;
        }
        for (int d = 0; d < 3; ++d) s->force[3 * i + d] += (((-8.0 * p->pi) * s->q[i]) * fk[d]) * s->inv_V;
    }
    s->v_coul = s->v_coul + u;
    return MFA_OK;
}

/* dipolar_correction.f90:17-39 (Yeh-Berkowitz slab correction, called after
 * ewald_k(1) for SYMMETRY 0, md_main.f90:128-131): M_z = sum q (z - Lz/2)
 * (lz_half = boundary(3)/2, init_config.f90:246), F_z -= 4 pi q M_z / V,
 * v_coul += 2 pi M_z^2 / V, with V the slab volume of ewald_k.f90:92 and pi
 * the single-precision literal widened (twopi = 2*pi exactly). */
void orc_dipolar_correction(orc_state* s) {
    const mfa_params* p = &s->p;
    if (!p->charged || p->symmetry != 0) return;
    const double lz_half = p->boundary[2] / 2.0;
    double m_z = 0.0;
    for (int i = 0; i < s->n; ++i) m_z = m_z + s->q[i] * (s->r0[3 * i + 2] - lz_half);
    for (int i = 0; i < s->n; ++i)
        s->force[3 * i + 2] = s->force[3 * i + 2] - (((4.0 * p->pi) * s->q[i]) * m_z) * s->inv_V;
    s->v_coul = s->v_coul + (((2.0 * p->pi) * m_z) * m_z) * s->inv_V;
}

/* verlet_velocities.f90:174-185 (kick), :262-294 (heads), :304-347 (energies) */
void orc_verlet_velocities(orc_state* s) {
    const mfa_params* p = &s->p;
    const double hdt = 0.5 * p->dt;
    for (int i = 0; i < s->n; ++i)
        for (int d = 0; d < 3; ++d) {
            s->a[3 * i + d] = s->force[3 * i + d] * s->inv_mass[i];
            s->v[3 * i + d] = s->v[3 * i + d] + hdt * s->a[3 * i + d];
        }
    /* verlet_velocities.f90:79-230 (head rules, kinetic and total energies)
     * are compiled out under DPD_VV; new_dpd_fd computes the energies */
    if (s->dpd_vv) return;
    if (p->pin_heads) {
        for (int c = 0; c < p->n_chain; ++c) {
            const int h = c * p->n_mon;
            const double sgn = (c < p->n_chain / 2) ? 1.0 : -1.0;
            s->v[3 * h + 0] = sgn * p->va_spring_twall[0];
            s->v[3 * h + 1] = sgn * p->va_spring_twall[1];
            s->v[3 * h + 2] = 0.0;
            for (int d = 0; d < 3; ++d) { s->force[3 * h + d] = 0.0; s->a[3 * h + d] = 0.0; }
        }
    }
    double T_inst = 0.0;
    for (int i = 0; i < s->n; ++i) {
        const double* vi = &s->v[3 * i];
        T_inst = T_inst + s->mass[i] * ((vi[0] * vi[0] + vi[1] * vi[1]) + vi[2] * vi[2]);
    }
    s->t_fluid = 0.5 * T_inst;
    s->v_total = (s->v_fluid_wall + s->v_fluid_fluid) + s->v_intra_molec;
    s->e_total = s->v_total + s->t_fluid;
}

/* ------------------------------------------------------------------ */
/* Optional terms behind cpp switches                                  */
/* ------------------------------------------------------------------ */

/* external_force.f90:9-18, mode 1 (EXT_FORCE 1): an elastic pull of every
 * bead towards the axis y = Ly/2, z = Lz/2.  No energy is kept. */
void orc_external_force(orc_state* s, int mode, double k_elastic) {
    if (mode != 1) return;
    const mfa_params* p = &s->p;
    for (int i = 0; i < s->n; ++i) {
        s->force[3 * i + 1] = s->force[3 * i + 1] - k_elastic * (s->r0[3 * i + 1] - p->boundary[1] / 2.0);
        s->force[3 * i + 2] = s->force[3 * i + 2] - k_elastic * (s->r0[3 * i + 2] - p->boundary[2] / 2.0);
    }
}

/* orientation.f90:3-185.  mode 1 (SYMMETRY 0, :24-85): the angle between a
 * ghost bond (head to a point one unit further from the mid-plane, :34-39)
 * and the first bond; forces on the head and the second bead, x and y
 * minimum-imaged (:43-48).  mode 2 (:89-175, as compiled with CHAIN_BC 2):
 * the first and the last bond against the fixed unit vector x, every axis
 * minimum-imaged.  Modes 0 and 3 do nothing.  Returns v_or. */
double orc_orientation(orc_state* s, int mode, double k_or, double alpha_or) {
    const mfa_params* p = &s->p;
    const double* L = p->boundary;
    const double* iL = s->inv_boundary;
    const int nm = p->n_mon;
    const double small1 = (double)0.0001f, small2 = (double)0.000001f;   /* default-REAL literals */
    double v_or = 0.0;
    if (mode != 1 && mode != 2) return 0.0;
    for (int l = 0; l < p->n_chain; ++l) {
        const int h = l * nm;
        if (mode == 1) {
            double g[3], rp[3], rn[3];
            for (int j = 0; j < 3; ++j) g[j] = s->r0[3 * h + j];
            if (s->r0[3 * h + 2] > L[2] / 2.0) g[2] = g[2] + 1.0;
            else g[2] = g[2] - 1.0;
            for (int j = 0; j < 3; ++j) {
                rp[j] = s->r0[3 * h + j] - g[j];
                rn[j] = s->r0[3 * (h + 1) + j] - s->r0[3 * h + j];
            }
            for (int j = 0; j < 2; ++j) {
                rn[j] = mimage(rn[j], L[j], iL[j]);
                rp[j] = mimage(rp[j], L[j], iL[j]);
            }
            double dot = 0.0, rp2 = 0.0, rn2 = 0.0, dn2 = 0.0, dn[3];
            for (int j = 0; j < 3; ++j) {
                dot = dot + rn[j] * rp[j];
                rp2 = rp2 + rp[j] * rp[j];
                rn2 = rn2 + rn[j] * rn[j];
            }
            const double cosa = dot / sqrt(rp2 * rn2);
            for (int j = 0; j < 3; ++j) dn[j] = rp[j] * rn2 - rn[j] * dot;
            for (int j = 0; j < 3; ++j) dn2 = dn2 + dn[j] * dn[j];
            if (dn2 < small1) {
                for (int j = 0; j < 3; ++j) dn[j] = dn[j] * 0.0;
            } else {
                const double den = sqrt(dn2 * rn2);
                for (int j = 0; j < 3; ++j) dn[j] = dn[j] / den;
            }
            const double da = acos(cosa) - alpha_or;
            const double fm = k_or * da;
            v_or = v_or + 0.5 * fm * da;
            for (int j = 0; j < 3; ++j) {
                s->force[3 * h + j] = s->force[3 * h + j] - fm * dn[j];
                s->force[3 * (h + 1) + j] = s->force[3 * (h + 1) + j] + fm * dn[j];
            }
        } else {
            const int last = h + nm - 1;
            for (int b = 1; b <= 2; ++b) {
                double rp[3], rn[3], dn[3], dp[3];
                if (b == 1) {
                    rp[0] = 1.0; rp[1] = 0.0; rp[2] = 0.0;
                    for (int j = 0; j < 3; ++j) rn[j] = s->r0[3 * (h + 1) + j] - s->r0[3 * h + j];
                } else {
                    for (int j = 0; j < 3; ++j) rp[j] = s->r0[3 * last + j] - s->r0[3 * (last - 1) + j];
                    rn[0] = 1.0; rn[1] = 0.0; rn[2] = 0.0;
                }
                for (int j = 0; j < 3; ++j) {
                    rn[j] = mimage(rn[j], L[j], iL[j]);
                    rp[j] = mimage(rp[j], L[j], iL[j]);
                }
                double dot = 0.0, rp2 = 0.0, rn2 = 0.0, dn2 = 0.0, dp2 = 0.0;
                for (int j = 0; j < 3; ++j) {
                    dot = dot + rn[j] * rp[j];
                    rp2 = rp2 + rp[j] * rp[j];
                    rn2 = rn2 + rn[j] * rn[j];
                }
                const double cosa = dot / sqrt(rp2 * rn2);
                for (int j = 0; j < 3; ++j) {
                    dn[j] = rp[j] * rn2 - rn[j] * dot;
                    dp[j] = -rn[j] * rp2 + rp[j] * dot;
                }
                for (int j = 0; j < 3; ++j) {
                    dp2 = dp2 + dp[j] * dp[j];
                    dn2 = dn2 + dn[j] * dn[j];
                }
                if (dn2 < small2) {
                    for (int j = 0; j < 3; ++j) dn[j] = dn[j] * 0.0;
                } else {
                    const double den = sqrt(dn2 * rn2);
                    for (int j = 0; j < 3; ++j) dn[j] = dn[j] / den;
                }
                if (dp2 < small2) {
                    for (int j = 0; j < 3; ++j) dp[j] = dp[j] * 0.0;
                } else {
                    const double den = sqrt(dp2 * rp2);
                    for (int j = 0; j < 3; ++j) dp[j] = dp[j] / den;
                }
                const double da = acos(cosa) - alpha_or;
                const double fm = k_or * da;
                v_or = v_or + 0.5 * fm * da;
                double fb[6];
                for (int j = 0; j < 3; ++j) { fb[j] = fm * dp[j]; fb[3 + j] = fm * dn[j]; }
                const int i0 = b == 1 ? last : last - 1, i1 = b == 1 ? h : last, i2 = b == 1 ? h + 1 : h;
                for (int j = 0; j < 3; ++j) {
                    s->force[3 * i0 + j] = s->force[3 * i0 + j] + fb[j];
                    s->force[3 * i1 + j] = s->force[3 * i1 + j] - fb[j] - fb[3 + j];
                    s->force[3 * i2 + j] = s->force[3 * i2 + j] + fb[3 + j];
                }
            }
        }
    }
    return v_or;
}

/* DPD_VV (control_simulation.h:51): force_d starts at zero (init_params.f90:839) */
void orc_set_dpd_vv(orc_state* s, int on) {
    s->dpd_vv = on != 0;
    if (s->dpd_vv && !s->force_d) s->force_d = (double*)calloc((size_t)3 * s->n, sizeof(double));
}

/* new_dpd_fd.f90:17-112: the dissipative force re-evaluated over ff_list with
 * the velocities after verlet_velocities, heads (type 1) excluded, x and y
 * minimum-imaged only (:40-43), no force switch-on; the previous call's force_d
 * is taken out of the force and the new one added (:17,:88); then a half kick
 * with the corrected force, a = F/m, and the kinetic and total energies
 * (:92-160; t_wall = 0, v_wall_wall = 0). */
void orc_new_dpd_fd(orc_state* s) {
    const mfa_params* p = &s->p;
    const int n = s->n;
    double* fd = s->force_d;
    if (!fd) return;
    for (int k = 0; k < 3 * n; ++k) s->force[k] = s->force[k] - fd[k];
    for (int k = 0; k < 3 * n; ++k) fd[k] = 0.0;
    const int row = s->list_cap + 1;
    for (int i = 0; i < n; ++i) {
        const int ti = s->a_type[i];
        if (ti == 1) continue;
        const int cnt = s->ff_list[(size_t)row * i];
        for (int k = 1; k <= cnt; ++k) {
            const int j = s->ff_list[(size_t)row * i + k] - 1;
            const int tj = s->a_type[j];
            if (tj == 1) continue;
            double dr[3];
            for (int d = 0; d < 3; ++d) dr[d] = s->r0[3 * i + d] - s->r0[3 * j + d];
            for (int d = 0; d < 2; ++d) dr[d] = mimage(dr[d], p->boundary[d], s->inv_boundary[d]);
            double r2 = 0.0;
            for (int d = 0; d < 3; ++d) r2 = r2 + dr[d] * dr[d];
            const double rr = p->range_2[(ti - 1) * MFA_MAX_TYPES + (tj - 1)];
            if (!(r2 < rr)) continue;
            double wd = 1.0;
            if (p->dpd_weight == 0) {
                const double u = 1.0 - sqrt(r2 / rr);
                wd = u * u;
            }
            const double rs = sqrt(r2);
            double rv[3], dv[3];
            for (int d = 0; d < 3; ++d) {
                rv[d] = dr[d] / rs;
                dv[d] = s->v[3 * i + d] - s->v[3 * j + d];
            }
            const double rd = (dv[0] * rv[0] + dv[1] * rv[1]) + dv[2] * rv[2];
            for (int d = 0; d < 3; ++d) {
                const double f = -1.0 * p->friction * wd * rd * rv[d];
                fd[3 * i + d] = fd[3 * i + d] + f;
                fd[3 * j + d] = fd[3 * j + d] - f;
            }
        }
    }
    for (int k = 0; k < 3 * n; ++k) s->force[k] = s->force[k] + fd[k];
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d)
            s->v[3 * i + d] = s->v[3 * i + d] + 0.5 * p->dt * s->force[3 * i + d] * s->inv_mass[i];
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) s->a[3 * i + d] = s->force[3 * i + d] * s->inv_mass[i];
    double t = 0.0;
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < n; ++i) t = t + s->mass[i] * (s->v[3 * i + d] * s->v[3 * i + d]);
    s->t_fluid = t / 2.0;
    s->v_total = (s->v_fluid_wall + s->v_fluid_fluid) + s->v_intra_molec;
    s->e_total = s->v_total + s->t_fluid;
}

/* md_main.f90:68-147 in order */
int orc_md_step(orc_state* s) {
    const mfa_params* p = &s->p;
    int err = 0;
    orc_verlet_positions(s);
    orc_check_skin(s);
    /* md_main.f90:81-85: the rule the program was built with (BIN_TYPE); here
       the rule of the last list build */
    if (s->f_skin == 1) err = s->bin_type == 1 ? orc_my_binning(s) : orc_binning(s);
    if (err) return err;
    orc_zero_forces(s);
    orc_fluid_fluid(s);
    if (p->symmetry == 0 && p->wall != 0) orc_fluid_wall(s, p->wall);
    orc_intra_molec(s);
    if (p->bending) orc_bending(s, 2);
    if (p->charged) err = orc_ewald_k(s, 1);
    if (p->charged && p->symmetry == 0) orc_dipolar_correction(s);
    orc_verlet_velocities(s);
    if (s->dpd_vv) orc_new_dpd_fd(s);   /* md_main.f90:149-155 */
    return err;
}

/* util.f90:283-322: O(N^2) LJ energy with the same cutoffs/shifts */
double orc_check_fluid_fluid(orc_state* s) {
    const mfa_params* p = &s->p;
    double v = 0.0;
    for (int i = 0; i < s->n; ++i)
        for (int j = i + 1; j < s->n; ++j) {
            const int ti = s->a_type[i], tj = s->a_type[j];
            double dr[3];
            for (int d = 0; d < 3; ++d) dr[d] = s->r0[3 * i + d] - s->r0[3 * j + d];
            dr[0] = mimage(dr[0], p->boundary[0], s->inv_boundary[0]);
            dr[1] = mimage(dr[1], p->boundary[1], s->inv_boundary[1]);
            if (p->symmetry == 1) dr[2] = mimage(dr[2], p->boundary[2], s->inv_boundary[2]);
            const double r_2 = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
            if (r_2 < p->range_2[IDX(ti, tj)]) {
                const double r_61 = p->sigma_2[IDX(ti, tj)] / r_2;
                const double r_6 = (r_61 * r_61) * r_61;
                v = v + p->epsil[IDX(ti, tj)] * ((r_6 * r_6 - r_6) - p->e_shift[IDX(ti, tj)]);
            }
        }
    return v;
}

void orc_get_state(const orc_state* s, double* r0, double* v, double* a, double* force, int32_t* mic) {
    size_t n = (size_t)s->n;
    if (r0) memcpy(r0, s->r0, 24 * n);
    if (v) memcpy(v, s->v, 24 * n);
    if (a) memcpy(a, s->a, 24 * n);
    if (force) memcpy(force, s->force, 24 * n);
    if (mic) memcpy(mic, s->mic, 12 * n);
}

void orc_set_state(orc_state* s, const double* r0, const double* v, const double* a,
                   const double* force, const int32_t* mic) {
    size_t n = (size_t)s->n;
    if (r0) memcpy(s->r0, r0, 24 * n);
    if (v) memcpy(s->v, v, 24 * n);
    if (a) memcpy(s->a, a, 24 * n);
    if (force) memcpy(s->force, force, 24 * n);
    if (mic) memcpy(s->mic, mic, 12 * n);
}

void orc_get_scalars(const orc_state* s, mfa_scalars* o) {
    memset(o, 0, sizeof(*o));
    o->v_fluid_fluid = s->v_fluid_fluid;
    o->v_fluid_wall = s->v_fluid_wall;
    o->v_intra_molec = s->v_intra_molec;
    o->v_bend = s->v_bend;
    o->v_coul = s->v_coul;
    o->t_fluid = s->t_fluid;
    o->v_total = s->v_total;
    o->e_total = s->e_total;
    o->virial = s->virial;
    o->i_time = s->i_time;
    o->f_skin = s->f_skin;
    o->n_rebuilds = s->n_rebuilds;
    o->max_neigh = s->max_neigh;
    o->max_cell = s->max_cell;
    o->fene_clamped = s->fene_clamped;
}

void orc_get_lists(const orc_state* s, int32_t* cell_of, int32_t* bin_fluid, int32_t* ff_list) {
    if (cell_of) memcpy(cell_of, s->cell_of, 4 * (size_t)s->n);
    if (bin_fluid) memcpy(bin_fluid, s->bin_fluid, 4 * (size_t)s->ncell * (s->bin_cap + 1));
    if (ff_list) memcpy(ff_list, s->ff_list, 4 * (size_t)s->n * (s->list_cap + 1));
}

int orc_get_kvecs(const orc_state* s, double* kv, int max_k) {
    int n = s->nk < max_k ? s->nk : max_k;
    if (kv) memcpy(kv, s->k_vecs, 24 * (size_t)n);
    return s->nk;
}

/* ------------------------------------------------------------------ */
/* init_params.f90:395-845, make_binning_boxes.f90:14-64,             */
/* init_config.f90:228-239 derived constants                           */
/* ------------------------------------------------------------------ */
void orc_derive_params(const orc_inputs* in, mfa_params* o) {
    const int n = in->n_type;
    const double c16 = (double)powf(2.0f, 1.0f / 6.0f); /* 2.**(1./6.) in single precision */
    const double c22 = (double)2.2f;
    o->n_type = n;
    double sigma[T8][T8] = {{0.0}};
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) sigma[i][j] = (in->sigma_ii[i] + in->sigma_ii[j]) / 2.0;
    for (int i = 0; i < n; ++i) sigma[i][i] = in->sigma_ii[i];
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            o->sigma_2[i * T8 + j] = sigma[i][j] * sigma[i][j];
            o->epsil[i * T8 + j] = 4.0 * in->eps[i * T8 + j];
            o->range_2[i * T8 + j] = (c16 * sigma[i][j]) * (c16 * sigma[i][j]);
        }
    if (in->brush_heads) {
        o->range_2[0 * T8 + (n - 1)] = (c22 * sigma[0][n - 1]) * (c22 * sigma[0][n - 1]);
        o->range_2[(n - 1) * T8 + 0] = (c22 * sigma[n - 1][0]) * (c22 * sigma[n - 1][0]);
    }
    if (in->wall93)
        for (int i = 0; i < n; ++i) { o->range_2[i * T8 + (n - 1)] = 0.0; o->range_2[(n - 1) * T8 + i] = 0.0; }
    if (in->brush_heads) o->range_2[0] = 0.0;
    double rc2max = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const double r2 = o->range_2[i * T8 + j];
            if (r2 > 0.0) {
                const double rd = pw3(sigma[j][i] * sigma[j][i] / r2);
                o->e_shift[i * T8 + j] = rd * (rd - 1.0);
                o->inv_range_2[i * T8 + j] = 1.0 / r2;
            } else {
                o->e_shift[i * T8 + j] = 0.0;
                o->inv_range_2[i * T8 + j] = 0.0;
            }
            if (r2 > rc2max) rc2max = r2;
        }
    const double r_cut_max = sqrt(rc2max);
    o->skin = in->skin;
    o->skin_2 = (r_cut_max + o->skin) * (r_cut_max + o->skin) - r_cut_max * r_cut_max;
    o->dt = in->dt; o->temp = in->temp; o->friction = in->friction;
    o->sig = sqrt(2.0 * in->temp * in->friction / in->dt);
    o->r_chain_2 = in->r_chain * in->r_chain;
    o->inv_r_chain_2 = 1.0 / o->r_chain_2;
    o->k_chain = in->k_chain_in * o->r_chain_2;
    o->fene_clamp = (double)0.98f;
    o->k_bend = in->k_bend; o->alpha_eq = in->alpha_eq;
    for (int i = 0; i < n; ++i) {
        o->sigma_wall[i] = (in->sigma_w + in->sigma_ii[i]) / 2.0;
        o->a_wall[i] = in->a_w;
    }
    o->a_w = in->a_w;
    for (int d = 0; d < 3; ++d) {
        o->boundary[d] = in->boundary[d];
        if (in->binning_rule == 0) o->n_bin[d] = (int32_t)(in->boundary[d] / (r_cut_max + (double)0.4f));
        else o->n_bin[d] = in->n_bin_in[d];
        const int nb0 = in->n_bin_init[d];
        o->delta_bin[d] = nb0 >= 3 ? 1 : (nb0 == 2 ? 0 : -1);
    }
    o->pi = (double)3.1415926536f;
    o->inv_sqrt_pi = 1.0 / o->pi;
}
