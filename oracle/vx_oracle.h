/*
 * vx_oracle.h — CPU oracle for the vortex-element time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C99 (+OpenMP) restatement of the
 * reference solver's step (grechkin-pogrebnyakov/vortex, src/kernel.cu and
 * src/unit_1.cu), used by the parity tests, by __graft_entry__.smoke() and by
 * the CPU-baseline leg of bench.py as the checker.  The product library never
 * links it, and nothing shipped calls it.
 *
 * Two arithmetic modes for the pair sums:
 *   VXO_PREC_FP64 — "plain" form: every quantity in FP64.  This is the
 *                   correctness oracle for the CUDA library.
 *   VXO_PREC_REF  — the reference's own types: FP32 inner loops with FP64
 *                   I/O, used to compare against the reference's CUDA build.
 *
 * Floating-point contract (the CUDA library follows the same one): the file is
 * compiled with -ffp-contract=off, and every fused multiply-add is written out
 * as fma().  With identical inputs this makes the 3-nearest distances, the
 * compaction permutation, the collapse pairing and merge, the advection and
 * the panel matrix bit-identical between the oracle and the library.
 */
#ifndef VX_ORACLE_H_
#define VX_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Panel record: same 120-byte layout as the reference's tPanel
 * (include/definitions.h:82-103). */
typedef struct vxo_panel {
    uint32_t n;
    uint32_t pad_;
    double left[2];
    double right[2];
    double contr[2];
    double birth[2];
    double norm[2];
    double tang[2];
    double length;
    uint32_t n_of_lpanel;
    uint32_t n_of_rpanel;
} vxo_panel;

enum { VXO_PREC_FP64 = 0, VXO_PREC_REF = 1 };
enum { VXO_BIRTH_REF = 0, VXO_BIRTH_FILE = 1, VXO_BIRTH_HALF_PANEL = 2 };

/* Resolved run parameters (the reference keeps them in __constant__ memory,
 * src/unit_1.cu:20-44, filled by init_device_conf_values :1220-1252). */
typedef struct vxo_params {
    double dt, nu, rho;
    double vinf_x, vinf_y;
    double eps;                /* ve_size: core radius */
    double r_col_diff_sign;    /* collapse radius ratios to eps */
    double r_col_same_sign;
    double max_ve_g;
    double x_min, x_max, y_min, y_max;                 /* wake window */
    double prof_x_min, prof_x_max, prof_y_min, prof_y_max; /* profile bbox */
    double rc_x, rc_y;         /* moment reference point */
    double drop_eps;           /* |G| below this is removed (reference DELT) */
    int64_t n_of_points;       /* sub-points per panel in the wall integral */
    int64_t n_col;             /* collapse rounds per pass */
    int32_t birth_mode;        /* VXO_BIRTH_* */
    int32_t prec;              /* VXO_PREC_* */
} vxo_params;

/* ---- panel system (src/unit_1.cu:115-402) ---- */
/* Builds the (P+1)x(P+1) influence matrix with the Kelvin row/column and
 * inverts it by Gauss-Jordan elimination.  Minv is row-major (P+1)^2.
 * Returns 0, or 1 when a pivot falls below 1e-12 (singular system). */
int vxo_panel_matrix(const vxo_panel *pan, int64_t P, double *L_out, double *Minv);

/* ---- birth (src/kernel.cu:779-873) ---- */
void vxo_birth_rhs(const vxo_params *p, const vxo_panel *pan, int64_t P,
                   const double *x, const double *y, const double *g, int64_t nsrc,
                   double *R);
void vxo_birth_gamma(int64_t P, const double *Minv, const double *R, double dg,
                     double *gamma);
void vxo_birth_place(const vxo_params *p, const vxo_panel *pan, int64_t P,
                     const double *gamma, double *x, double *y, double *g);

/* ---- convective velocity + 3-nearest distance (src/kernel.cu:875-983) ----
 * Targets [0,n); the 3-nearest search runs over sources [0,s) (s = n rounded
 * up to 32, the reference's padded launch), the velocity sum over [0,n). */
void vxo_velocity(const vxo_params *p, const double *x, const double *y, const double *g,
                  int64_t n, int64_t s, double *vx, double *vy, double *d);

/* Targets [i0, i1) only, over all n sources (outputs indexed from i0). */
void vxo_velocity_targets(const vxo_params *p, const double *x, const double *y, const double *g,
                          int64_t n, int64_t i0, int64_t i1, double *vx, double *vy, double *d);
void vxo_diffusion_targets(const vxo_params *p, const double *x, const double *y, const double *g,
                           int64_t n, int64_t i0, int64_t i1, const double *d, double *vx, double *vy);

/* ---- diffusive velocities (src/kernel.cu:985-1088, 1300-1346) ---- */
void vxo_diffusion(const vxo_params *p, const double *x, const double *y, const double *g,
                   int64_t n, const double *d, double *vx, double *vy);
void vxo_diffusion_sums(const vxo_params *p, const double *x, const double *y, const double *g,
                        int64_t n, const double *d, double *I1, double *A1);
void vxo_wall_diffusion(const vxo_params *p, const vxo_panel *pan, int64_t P,
                        const double *x, const double *y, int64_t n, const double *d,
                        double *vx, double *vy);

/* ---- convection, absorption, force terms (src/kernel.cu:1090-1157, 1357-1431) ---- */
int  vxo_hitting(const vxo_params *p, const vxo_panel *pan, int64_t P,
                 double x1, double y1, double x2, double y2, int32_t *hitpan);
void vxo_advect(const vxo_params *p, const vxo_panel *pan, int64_t P,
                double *x, double *y, double *g, const double *vx, const double *vy,
                int64_t n, int64_t n_new,
                double *dg_i, double *fx_i, double *fy_i, double *m_i);
void vxo_sums(const vxo_params *p, int64_t n, const double *dg_i, const double *fx_i,
              const double *fy_i, const double *m_i,
              double *dg, double *fx, double *fy, double *m);

/* ---- compaction (src/kernel.cu:1159-1178) ---- */
int64_t vxo_compact(double *x, double *y, double *g, int64_t n, double drop_eps);

/* ---- collapse (src/kernel.cu:1180-1271, src/unit_1.cu:1137-1216) ----
 * pass 1 = opposite signs, pass 2 = same sign. */
void vxo_collapse_col(const vxo_params *p, int pass, const double *x, const double *y,
                      const double *g, int64_t n, int32_t *col);
void vxo_collapse_merge(int pass, double *x, double *y, double *g, int64_t n, int32_t *col);
int64_t vxo_collapse(const vxo_params *p, int pass, double *x, double *y, double *g,
                     int64_t n, int32_t *col_scratch);

/* ---- probe velocity (src/kernel.cu:1434-1475) ---- */
void vxo_probe(const vxo_params *p, const double *x, const double *y, const double *g,
               int64_t n, const double *px, const double *py, int64_t np,
               double *vx, double *vy);

/* ---- one whole step in the reference's order (src/main.c:652-785) ----
 * State arrays have capacity >= round32(n+P)+32.  dg/fx/fy/m are the carried
 * scalars: dg feeds this step's birth and is overwritten with the circulation
 * absorbed in this step; fx/fy/m receive this step's force and moment.
 * Returns the new particle count. */
typedef struct vxo_state {
    int64_t cap;
    int64_t n;
    double *x, *y, *g;
    double *vx, *vy, *d;
    double dg, fx, fy, m;
} vxo_state;

int64_t vxo_step(const vxo_params *p, const vxo_panel *pan, int64_t P,
                 const double *Minv, vxo_state *st);

/* Deterministic far-away filler for never-written slots (the reference
 * uses rand() at 2e5..; any far point with G=0 gives the same results). */
void vxo_fill_tail(double *x, double *y, double *g, int64_t from, int64_t to);

int vxo_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif /* VX_ORACLE_H_ */
