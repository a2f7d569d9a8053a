/*
 * vx_oracle.c — CPU oracle for the vortex-element time step.
 *
 * TEST INFRASTRUCTURE ONLY (see vx_oracle.h).  Each function restates one
 * piece of the reference solver grechkin-pogrebnyakov/vortex and cites the
 * file:line it follows.  Build with -ffp-contract=off: every fused
 * multiply-add below is an explicit fma(), matching the CUDA library.
 */
#define _GNU_SOURCE
#include "vx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TWO_PI 6.283185307179586     /* 2*M_PI, exact doubling */
#define DELT_PIVOT 1e-12             /* reference include/definitions.h:36 */

int vxo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static inline int64_t round32(int64_t v) { return (v + 31) / 32 * 32; }

void vxo_fill_tail(double *x, double *y, double *g, int64_t from, int64_t to) {
    for (int64_t i = from; i < to; ++i) {
        x[i] = 4.0e5 + (double)i;
        y[i] = 4.0e5 + (double)i;
        g[i] = 0.0;
    }
}

/* ------------------------------------------------------------------------ */
/* Panel influence matrix: src/unit_1.cu:256-402 (matr_creation).  The
 * expression trees are kept as in the reference so that, compiled without
 * contraction, the matrix is bit-identical to the reference's host code.   */
static inline double sp2(const double a[2], const double b[2]) {
    return a[0] * b[0] + a[1] * b[1];
}

static void panel_influence(const vxo_panel *pan, int64_t P, double *L) {
    const int64_t S = P + 1;
    for (int64_t i = 0; i < P; ++i) {
        const double *tau = pan[i].tang;
        for (int64_t j = 0; j < P; ++j) {
            if (j == i) { L[i * S + j] = -0.5; continue; }
            double a0[2], a1[2], b0[2], b1[2];
            int next = (j == i + 1) || (j == 0 && i == P - 1);
            if (next) {   /* neighbour on the right: endpoints exchanged (src/unit_1.cu:303-313) */
                a1[0] = pan[i].left[0];  a1[1] = pan[i].left[1];
                a0[0] = pan[i].right[0]; a0[1] = pan[i].right[1];
                b1[0] = pan[j].left[0];  b1[1] = pan[j].left[1];
                b0[0] = pan[j].right[0]; b0[1] = pan[j].right[1];
            } else {
                a0[0] = pan[i].left[0];  a0[1] = pan[i].left[1];
                a1[0] = pan[i].right[0]; a1[1] = pan[i].right[1];
                b0[0] = pan[j].left[0];  b0[1] = pan[j].left[1];
                b1[0] = pan[j].right[0]; b1[1] = pan[j].right[1];
            }
            double dj[2] = {b1[0] - b0[0], b1[1] - b0[1]};
            double di[2] = {a1[0] - a0[0], a1[1] - a0[1]};
            double p1[2] = {a0[0] - b1[0], a0[1] - b1[1]};
            double p2[2] = {a1[0] - b1[0], a1[1] - b1[1]};
            double s1[2] = {a0[0] - b0[0], a0[1] - b0[1]};
            double s2[2] = {a1[0] - b0[0], a1[1] - b0[1]};
            double z1 = p1[0] * p2[1] - p1[1] * p2[0];
            double z2 = s1[0] * s2[1] - s1[1] * s2[0];
            double z3 = s2[0] * p2[1] - s2[1] * p2[0];
            double q11, q21;
            int adj = (j == i - 1) || (j == i + 1) || (j == 0 && i == P - 1) || (i == 0 && j == P - 1);
            if (adj) {    /* shared vertex: the p-terms vanish (src/unit_1.cu:334-341) */
                q11 = 0.0; q21 = 0.0;
            } else {
                q11 = atan(sp2(di, p1) / z1) - atan(sp2(di, p2) / z1);
                q21 = 0.5 * log(sp2(p2, p2) / sp2(p1, p1));
            }
            double q12 = atan(sp2(di, s2) / z2) - atan(sp2(di, s1) / z2);
            double q13 = atan(sp2(dj, p2) / z3) - atan(sp2(dj, s2) / z3);
            double q22 = 0.5 * log(sp2(s1, s1) / sp2(s2, s2));
            double q23 = 0.5 * log(sp2(p2, p2) / sp2(s2, s2));
            double c1[2], c2[2], c3[2];
            for (int k = 0; k < 2; ++k)
                c1[k] = sp2(dj, p1) * di[k] + sp2(di, s1) * dj[k] - sp2(di, dj) * s1[k];
            for (int k = 0; k < 2; ++k) c2[k] = c1[k] + sp2(dj, dj) * di[k];
            for (int k = 0; k < 2; ++k) c3[k] = sp2(di, di) * dj[k];
            double f = 1.0 / (TWO_PI * sqrt(sp2(dj, dj)) * sp2(di, di));
            double v0 = f * (q11 * c1[0] + q12 * c2[0] + q13 * c3[0]
                             + (q21 * c1[1] + q22 * c2[1] + q23 * c3[1]));
            double v1 = f * (q11 * c1[1] + q12 * c2[1] + q13 * c3[1]
                             - (q21 * c1[0] + q22 * c2[0] + q23 * c3[0]));
            L[i * S + j] = v0 * tau[0] + v1 * tau[1];
        }
    }
    for (int64_t i = 0; i < P; ++i) {     /* Kelvin row and column */
        L[P * S + i] = pan[i].length;
        L[i * S + P] = 1.0;
    }
    L[P * S + P] = 0.0;
}

static void swap_rows(double *A, int64_t S, int64_t r1, int64_t r2) {
    if (r1 == r2) return;
    for (int64_t j = 0; j < S; ++j) {
        double t = A[r1 * S + j]; A[r1 * S + j] = A[r2 * S + j]; A[r2 * S + j] = t;
    }
}

/* Gauss-Jordan inverse with the reference's pivoting rule:
 * src/unit_1.cu:115-254 (inverse_matrix).  Row k eliminates column k from
 * every other row after choosing the pivot row for column k+1. */
static int gauss_jordan(double *A, double *Inv, int64_t S) {
    memset(Inv, 0, sizeof(double) * S * S);
    for (int64_t i = 0; i < S; ++i) Inv[i * S + i] = 1.0;
    if (fabs(A[0]) < DELT_PIVOT) {
        double mx = fabs(A[0]);
        int64_t num = 0;
        for (int64_t i = 1; i < S; ++i)
            if (fabs(A[i * S]) > mx) { mx = fabs(A[i * S]); num = i; }
        if (num != 0) { swap_rows(A, S, 0, num); swap_rows(Inv, S, 0, num); }
    }
    for (int64_t k = 0; k < S - 1; ++k) {
        if (fabs(A[k * S + k]) < DELT_PIVOT) return 1;
        double mx = fabs(A[(k + 1) * S + k + 1]);
        int64_t line = k + 1;
        for (int64_t i = k + 1; i < S; ++i)
            if (fabs(A[i * S + k + 1]) > mx) { mx = fabs(A[i * S + k + 1]); line = i; }
        if (mx < DELT_PIVOT) return 1;
        swap_rows(A, S, k + 1, line);
        swap_rows(Inv, S, k + 1, line);
        const double piv = A[k * S + k];
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < S; ++i) {
            if (i == k) continue;
            double c = A[i * S + k] / piv;
            for (int64_t j = 0; j < S; ++j) {
                A[i * S + j] = A[i * S + j] - c * A[k * S + j];
                Inv[i * S + j] = Inv[i * S + j] - c * Inv[k * S + j];
            }
        }
    }
    const int64_t l = S - 1;
    if (fabs(A[l * S + l]) < DELT_PIVOT) return 1;
    for (int64_t i = 0; i < l; ++i) {
        double c = A[i * S + l] / A[l * S + l];
        for (int64_t j = 0; j < S; ++j) Inv[i * S + j] = Inv[i * S + j] - c * Inv[l * S + j];
    }
    for (int64_t i = 0; i < S; ++i)
        for (int64_t j = 0; j < S; ++j) Inv[i * S + j] = Inv[i * S + j] / A[i * S + i];
    return 0;
}

int vxo_panel_matrix(const vxo_panel *pan, int64_t P, double *L_out, double *Minv) {
    const int64_t S = P + 1;
    double *L = (double *)malloc(sizeof(double) * S * S);
    if (!L) return 2;
    panel_influence(pan, P, L);
    if (L_out) memcpy(L_out, L, sizeof(double) * S * S);
    int rc = gauss_jordan(L, Minv, S);
    free(L);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Birth right-hand side: src/kernel.cu:779-847 (Right_part_Kernel).        */
void vxo_birth_rhs(const vxo_params *p, const vxo_panel *pan, int64_t P,
                   const double *x, const double *y, const double *g, int64_t nsrc,
                   double *R) {
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < P; ++i) {
        if (p->prec == VXO_PREC_FP64) {
            const double al0 = pan[i].left[0], al1 = pan[i].left[1];
            const double ar0 = pan[i].right[0], ar1 = pan[i].right[1];
            const double d0 = ar0 - al0, d1 = ar1 - al1;
            const double kd0 = -d1, kd1 = d0;
            double y0 = 0.0, y1 = 0.0;
            for (int64_t j = 0; j < nsrc; ++j) {
                double s00 = al0 - x[j], s01 = al1 - y[j];
                double s10 = ar0 - x[j], s11 = ar1 - y[j];
                double z = d0 * s01 - d1 * s00;
                double alpha = atan((s00 * d0 + s01 * d1) / z) - atan((s10 * d0 + s11 * d1) / z);
                double beta = 0.5 * log((s10 * s10 + s11 * s11) / (s00 * s00 + s01 * s01));
                y0 = fma(g[j], alpha * d0 + beta * kd0, y0);
                y1 = fma(g[j], alpha * d1 + beta * kd1, y1);
            }
            double mnog = 1.0 / (TWO_PI * (d0 * d0 + d1 * d1));
            R[i] = -((mnog * y0 + p->vinf_x) * pan[i].tang[0] + (mnog * y1 + p->vinf_y) * pan[i].tang[1]);
        } else {
            const float al0 = (float)pan[i].left[0], al1 = (float)pan[i].left[1];
            const float ar0 = (float)pan[i].right[0], ar1 = (float)pan[i].right[1];
            const float t0 = (float)pan[i].tang[0], t1 = (float)pan[i].tang[1];
            const float d0 = ar0 - al0, d1 = ar1 - al1;
            const float kd0 = -d1, kd1 = d0;
            float y0 = 0.0f, y1 = 0.0f;
            for (int64_t j = 0; j < nsrc; ++j) {
                float b0 = (float)x[j], b1 = (float)y[j], gj = (float)g[j];
                float s00 = al0 - b0, s01 = al1 - b1, s10 = ar0 - b0, s11 = ar1 - b1;
                float z = d0 * s01 - d1 * s00;
                float alpha = atanf((s00 * d0 + s01 * d1) / z) - atanf((s10 * d0 + s11 * d1) / z);
                float beta = (float)(0.5 * logf((s10 * s10 + s11 * s11) / (s00 * s00 + s01 * s01)));
                y0 = fmaf(gj, alpha * d0 + beta * kd0, y0);
                y1 = fmaf(gj, alpha * d1 + beta * kd1, y1);
            }
            float mnog = (float)(1.0 / (TWO_PI * (d0 * d0 + d1 * d1)));
            R[i] = -(double)((mnog * y0 + (float)p->vinf_x) * t0 + (mnog * y1 + (float)p->vinf_y) * t1);
        }
    }
}

/* Birth strengths: src/kernel.cu:849-873 (birth_Kernel), gamma = M [R; dg]. */
void vxo_birth_gamma(int64_t P, const double *Minv, const double *R, double dg, double *gamma) {
    const int64_t S = P + 1;
    for (int64_t i = 0; i < P; ++i) {
        double acc = 0.0;
        for (int64_t j = 0; j < P; ++j) acc = fma(Minv[i * S + j], R[j], acc);
        gamma[i] = fma(Minv[i * S + P], dg, acc);
    }
}

/* New vortices: src/kernel.cu:862-872 and include/kernel.cuh:109-116. */
void vxo_birth_place(const vxo_params *p, const vxo_panel *pan, int64_t P,
                     const double *gamma, double *x, double *y, double *g) {
    for (int64_t i = 0; i < P; ++i) {
        int64_t in = pan[i].n_of_rpanel;
        double mx = (pan[i].left[0] + pan[i].right[0]) / 2;
        double my = (pan[i].left[1] + pan[i].right[1]) / 2;
        if (p->birth_mode == VXO_BIRTH_FILE) {
            x[i] = pan[i].birth[0]; y[i] = pan[i].birth[1];
        } else if (p->birth_mode == VXO_BIRTH_HALF_PANEL) {
            double h = 0.5 * pan[i].length;
            x[i] = mx + h * pan[i].norm[0]; y[i] = my + h * pan[i].norm[1];
        } else {
            x[i] = mx + 1e-6 * pan[i].norm[0]; y[i] = my + 1e-6 * pan[i].norm[1];
        }
        g[i] = 0.5 * (gamma[i] * pan[i].length + gamma[in] * pan[in].length);
    }
}

/* ------------------------------------------------------------------------ */
/* Convective velocity + mean distance to the 3 nearest: src/kernel.cu:875-983. */
#define NN3_INSERT(d1, d2, d3, r2, MINF, MAXF) do {                           \
        if ((d3) > (r2)) {                                                       \
            (d3) = (r2);                                                         \
            __typeof__(d1) t_ = MINF((d3), (d2)); (d3) = MAXF((d3), (d2)); (d2) = t_; \
            t_ = MINF((d1), (d2)); (d2) = MAXF((d1), (d2)); (d1) = t_;           \
        } } while (0)

void vxo_velocity(const vxo_params *p, const double *x, const double *y, const double *g,
                  int64_t n, int64_t s, double *vx, double *vy, double *d) {
    const double eps2 = p->eps * p->eps;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
        if (p->prec == VXO_PREC_FP64) {
            const double a0 = x[i], a1 = y[i];
            double d1 = 1e5, d2 = 1e5, d3 = 1e5, y0 = 0.0, y1 = 0.0;
            for (int64_t j = 0; j < s; ++j) {
                if (j == i) continue;
                double dx = a0 - x[j], dy = a1 - y[j];
                double r2 = fma(dx, dx, dy * dy);
                NN3_INSERT(d1, d2, d3, r2, fmin, fmax);
                if (j < n) {
                    double m = g[j] / fmax(r2, eps2);
                    y1 = fma(m, dx, y1);
                    y0 = fma(-m, dy, y0);
                }
            }
            d[i] = (sqrt(d1) + sqrt(d2) + sqrt(d3)) / 3;
            vx[i] = y0 / TWO_PI + p->vinf_x;
            vy[i] = y1 / TWO_PI + p->vinf_y;
        } else {
            const float a0 = (float)x[i], a1 = (float)y[i];
            const float e2 = (float)eps2;
            float d1 = 1e5f, d2 = 1e5f, d3 = 1e5f, y0 = 0.0f, y1 = 0.0f;
            for (int64_t j = 0; j < s; ++j) {
                if (j == i) continue;
                float dx = a0 - (float)x[j], dy = a1 - (float)y[j];
                float r2 = fmaf(dx, dx, dy * dy);
                NN3_INSERT(d1, d2, d3, r2, fminf, fmaxf);
                float m = (float)g[j] / fmaxf(r2, e2);
                y1 = fmaf(m, dx, y1);
                y0 = fmaf(-m, dy, y0);
            }
            d[i] = (double)((sqrtf(d1) + sqrtf(d2) + sqrtf(d3)) / 3);
            vx[i] = (double)y0 / TWO_PI + p->vinf_x;
            vy[i] = (double)y1 / TWO_PI + p->vinf_y;
        }
    }
}

/* Vortex-vortex diffusive velocity: src/kernel.cu:985-1029. */
void vxo_diffusion(const vxo_params *p, const double *x, const double *y, const double *g,
                   int64_t n, const double *d, double *vx, double *vy) {
    const double thr = 0.001 * p->eps;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
        if (p->prec == VXO_PREC_FP64) {
            const double a0 = x[i], a1 = y[i], dd = d[i];
            double I2x = 0.0, I2y = 0.0, I1 = 0.0;
            for (int64_t j = 0; j < n; ++j) {
                double dx = a0 - x[j], dy = a1 - y[j];
                double dist = sqrt(fma(dx, dx, dy * dy));
                if (dist > thr) {
                    double m = g[j] / dist;
                    double e = exp(-dist / dd);
                    double me = m * e;
                    I2x = fma(-me, dx, I2x);
                    I2y = fma(-me, dy, I2y);
                    I1 = fma(g[j], e, I1);
                }
            }
            if (fabs(I1) > 1e-5) {
                vx[i] += -p->nu * I2x / (I1 * dd);
                vy[i] += -p->nu * I2y / (I1 * dd);
            }
        } else {
            const float a0 = (float)x[i], a1 = (float)y[i], dd = (float)d[i];
            const float nu = (float)p->nu;
            float I2x = 0.0f, I2y = 0.0f, I1 = 0.0f;
            for (int64_t j = 0; j < n; ++j) {
                float dx = a0 - (float)x[j], dy = a1 - (float)y[j];
                float dist = sqrtf(fmaf(dx, dx, dy * dy));
                if ((double)dist > thr) {
                    float gj = (float)g[j];
                    float m = gj / dist;
                    float e = expf(-dist / dd);
                    I2x = fmaf(-m * dx, e, I2x);
                    I2y = fmaf(-m * dy, e, I2y);
                    I1 = fmaf(gj, e, I1);
                }
            }
            if (fabs(I1) > 1e-5) {
                vx[i] += (double)(-nu * I2x / (I1 * dd));
                vy[i] += (double)(-nu * I2y / (I1 * dd));
            }
        }
    }
}

/* Wall integral over one panel: src/kernel.cu:1300-1322 (FP64 twin I_0_I_3)
 * and 1324-1346 (I_0_I_3f, FP32). */
static void wall_integral(double Ra0, double Ra1, double Rb0, double Rb1, double N0, double N1,
                          double Rj0, double Rj1, double dL, double d, int64_t N,
                          double *R0, double *R30, double *R31) {
    double dR0 = (Rb0 - Ra0) / N, dR1 = (Rb1 - Ra1) / N;
    double delt = dL / N;
    double s0 = 0.0, s30 = 0.0, s31 = 0.0;
    for (int64_t k = 0; k < N; ++k) {
        double Rk0 = (Ra0 + k * dR0 + Ra0 + (k + 1) * dR0) / 2;
        double Rk1 = (Ra1 + k * dR1 + Ra1 + (k + 1) * dR1) / 2;
        double E0 = (Rj0 - Rk0) / d, E1 = (Rj1 - Rk1) / d;
        double e2 = fma(E0, E0, E1 * E1);
        double me = sqrt(e2);
        double ex = exp(-me);
        s0 += (E0 * N0 + E1 * N1) / e2 * (me + 1) * ex * delt;
        s30 += N0 * ex * delt;
        s31 += N1 * ex * delt;
    }
    *R0 = s0; *R30 = s30; *R31 = s31;
}

static void wall_integral_f(float Ra0, float Ra1, float Rb0, float Rb1, float N0, float N1,
                            float Rj0, float Rj1, float dL, float d, int64_t N,
                            float *R0, float *R30, float *R31) {
    float dR0 = (Rb0 - Ra0) / N, dR1 = (Rb1 - Ra1) / N;
    float delt = dL / N;
    float s0 = 0.0f, s30 = 0.0f, s31 = 0.0f;
    for (int64_t k = 0; k < N; ++k) {
        float Rk0 = (Ra0 + k * dR0 + Ra0 + (k + 1) * dR0) / 2;
        float Rk1 = (Ra1 + k * dR1 + Ra1 + (k + 1) * dR1) / 2;
        float E0 = (Rj0 - Rk0) / d, E1 = (Rj1 - Rk1) / d;
        double me = sqrtf(E0 * E0 + E1 * E1);
        float ex = expf((float)(-me));
        s0 = (float)(s0 + (E0 * N0 + E1 * N1) / (E0 * E0 + E1 * E1) * (me + 1) * ex * delt);
        s30 += N0 * ex * delt;
        s31 += N1 * ex * delt;
    }
    *R0 = s0; *R30 = s30; *R31 = s31;
}

/* The vortex-diffusion sums of each target in FP64 (the loop of
 * vxo_diffusion, src/kernel.cu:985-1029): I1 = sum G_j e^(-r/d_i) and its
 * magnitude sum A1 = sum |G_j| e^(-r/d_i).  A1 / |I1| is the cancellation
 * factor of I1, |I1| against 1e-5 the reference's switch of the term. */
void vxo_diffusion_sums(const vxo_params *p, const double *x, const double *y, const double *g,
                        int64_t n, const double *d, double *I1o, double *A1o) {
    const double thr = 0.001 * p->eps;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
        const double a0 = x[i], a1 = y[i], dd = d[i];
        double I1 = 0.0, A1 = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            double dx = a0 - x[j], dy = a1 - y[j];
            double dist = sqrt(fma(dx, dx, dy * dy));
            if (dist > thr) {
                double e = exp(-dist / dd);
                I1 = fma(g[j], e, I1);
                A1 = fma(fabs(g[j]), e, A1);
            }
        }
        I1o[i] = I1;
        A1o[i] = A1;
    }
}

/* Wall diffusive velocity: src/kernel.cu:1031-1088 (diffusion_2_Kernel). */
void vxo_wall_diffusion(const vxo_params *p, const vxo_panel *pan, int64_t P,
                        const double *x, const double *y, int64_t n, const double *d,
                        double *vx, double *vy) {
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
        if (p->prec == VXO_PREC_FP64) {
            const double a0 = x[i], a1 = y[i], dd = d[i];
            double I0 = TWO_PI * dd * dd, I30 = 0.0, I31 = 0.0;
            for (int64_t f = 0; f < P; ++f) {
                const double dL = pan[f].length;
                double dx = a0 - pan[f].birth[0], dy = a1 - pan[f].birth[1];
                double r = sqrt(fma(dx, dx, dy * dy));
                if (r < 5 * dL && r > 0.1 * dL) {
                    double R0, R30, R31;
                    wall_integral(pan[f].left[0], pan[f].left[1], pan[f].right[0], pan[f].right[1],
                                  -pan[f].norm[0], -pan[f].norm[1], a0, a1, dL, dd,
                                  p->n_of_points, &R0, &R30, &R31);
                    I0 += (-dd) * R0;
                    I30 -= R30;
                    I31 -= R31;
                } else if (r <= 0.1 * dL) {
                    double ex = 1 - exp(-dL / (2 * dd));
                    I0 = M_PI * dd * dd;
                    I30 = 2 * pan[f].norm[0] * dd * ex;
                    I31 = 2 * pan[f].norm[1] * dd * ex;
                    break;
                }
            }
            vx[i] += p->nu * I30 / I0;
            vy[i] += p->nu * I31 / I0;
        } else {
            const float a0 = (float)x[i], a1 = (float)y[i], dd = (float)d[i];
            const float nu = (float)p->nu;
            float I0 = (float)(TWO_PI * dd * dd), I30 = 0.0f, I31 = 0.0f;
            for (int64_t f = 0; f < P; ++f) {
                const float dL = (float)pan[f].length;
                float dx = a0 - (float)pan[f].birth[0], dy = a1 - (float)pan[f].birth[1];
                float r = sqrtf(fmaf(dx, dx, dy * dy));
                if (r < 5 * dL && r > 0.1 * dL) {
                    float R0, R30, R31;
                    wall_integral_f((float)pan[f].left[0], (float)pan[f].left[1],
                                    (float)pan[f].right[0], (float)pan[f].right[1],
                                    -(float)pan[f].norm[0], -(float)pan[f].norm[1], a0, a1, dL, dd,
                                    p->n_of_points, &R0, &R30, &R31);
                    I0 += (-dd) * R0;
                    I30 -= R30;
                    I31 -= R31;
                } else if (r <= 0.1 * dL) {
                    float n0 = (float)pan[f].norm[0], n1 = (float)pan[f].norm[1];
                    I0 = (float)(M_PI * dd * dd);
                    I30 = 2 * n0 * dd * (1 - expf(-dL / (2 * dd)));
                    I31 = 2 * n1 * dd * (1 - expf(-dL / (2 * dd)));
                    break;
                }
            }
            vx[i] += (double)(float)(nu * I30 / I0);
            vy[i] += (double)(float)(nu * I31 / I0);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Segment/panel crossing test: src/kernel.cu:1357-1431 (hitting).
 * (x1,y1) is the new position, (x2,y2) the old one. */
int vxo_hitting(const vxo_params *p, const vxo_panel *pan, int64_t P,
                double x1, double y1, double x2, double y2, int32_t *hitpan) {
    const double thr = 1e-12;
    double minDist = 25.0;
    int32_t minN = -1;
    int hit = !(((x1 < p->prof_x_min) && (x2 < p->prof_x_min)) ||
                ((x1 > p->prof_x_max) && (x2 > p->prof_x_max)) ||
                ((y1 < p->prof_y_min) && (y2 < p->prof_y_min)) ||
                ((y1 > p->prof_y_max) && (y2 > p->prof_y_max)));
    if (hit) {
        hit = 0;
        double A = y2 - y1, B = x1 - x2, D = y1 * x2 - x1 * y2;
        for (int64_t i = 0; i < P; ++i) {
            double r0 = A * pan[i].left[0] + B * pan[i].left[1] + D;
            double r1 = A * pan[i].right[0] + B * pan[i].right[1] + D;
            if (fabs(r0) < thr) r0 = 0.0;
            if (fabs(r1) < thr) r1 = 0.0;
            if (r0 * r1 <= 0) {
                double A1 = pan[i].right[1] - pan[i].left[1];
                double B1 = pan[i].left[0] - pan[i].right[0];
                double D1 = pan[i].left[1] * pan[i].right[0] - pan[i].left[0] * pan[i].right[1];
                double r2 = A1 * x1 + B1 * y1 + D1;
                double r3 = A1 * x2 + B1 * y2 + D1;
                if (fabs(r2) < thr) r2 = 0.0;
                if (fabs(r3) < thr) r3 = 0.0;
                if (r2 * r3 <= 0) {
                    hit = 1;
                    double den = A * B1 - B * A1;
                    double X = (B * D1 - D * B1) / den;
                    double Y = (A1 * D - D1 * A) / den;
                    double d2 = (x2 - X) * (x2 - X) + (y2 - Y) * (y2 - Y);
                    if (d2 < minDist) { minDist = d2; minN = (int32_t)i; }
                }
            }
        }
    }
    *hitpan = minN;
    return hit;
}

/* Convection + absorption + per-particle force terms: src/kernel.cu:1090-1143.
 * n_new = number of vortices born this step (they sit at [n-n_new, n)). */
void vxo_advect(const vxo_params *p, const vxo_panel *pan, int64_t P,
                double *x, double *y, double *g, const double *vx, const double *vy,
                int64_t n, int64_t n_new,
                double *dg_i, double *fx_i, double *fy_i, double *m_i) {
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        double dgv = 0.0, fx = 0.0, fy = 0.0, m = 0.0;
        double gi = g[i];
        if (i >= n - n_new) {
            double dx = x[i] - p->rc_x, dy = y[i] - p->rc_y;
            fx = gi * (-y[i]);
            fy = gi * x[i];
            m = gi * fma(dx, dx, dy * dy);
        }
        double xn = fma(vx[i], p->dt, x[i]);
        double yn = fma(vy[i], p->dt, y[i]);
        int32_t hp = -1;
        if (gi != 0 && vxo_hitting(p, pan, P, xn, yn, x[i], y[i], &hp)) {
            if (hp >= 0) {
                double cx = pan[hp].contr[0], cy = pan[hp].contr[1];
                double dx = cx - p->rc_x, dy = cy - p->rc_y;
                fx -= gi * (-cy);
                fy -= gi * cx;
                m -= gi * fma(dx, dx, dy * dy);
            }
            dgv = gi;
            gi = 0.0;
        }
        if (gi != 0 && (xn > p->x_max || xn < p->x_min || yn > p->y_max || yn < p->y_min)) {
            xn = -2.0e5; yn = -2.0e5; gi = 0.0;
        }
        x[i] = xn; y[i] = yn; g[i] = gi;
        dg_i[i] = dgv; fx_i[i] = fx; fy_i[i] = fy; m_i[i] = m;
    }
}

/* Serial sums: src/kernel.cu:1144-1157 (summ_Kernel). */
void vxo_sums(const vxo_params *p, int64_t n, const double *dg_i, const double *fx_i,
              const double *fy_i, const double *m_i,
              double *dg, double *fx, double *fy, double *m) {
    double sdg = 0.0, sfx = 0.0, sfy = 0.0, sm = 0.0;
    for (int64_t k = 0; k < n; ++k) {
        sdg += dg_i[k]; sfx += fx_i[k]; sfy += fy_i[k]; sm += m_i[k];
    }
    *dg = sdg;
    *fx = sfx * (p->rho / p->dt);
    *fy = sfy * (p->rho / p->dt);
    *m = sm * (p->rho / (2 * p->dt));
}

/* Swap-with-last removal of |G| < drop_eps: src/kernel.cu:1159-1178. */
int64_t vxo_compact(double *x, double *y, double *g, int64_t n, double drop_eps) {
    for (int64_t i = 0; i < n; ++i) {
        if (fabs(g[i]) < drop_eps) {
            double r0 = x[i], r1 = y[i];
            g[i] = g[n - 1]; x[i] = x[n - 1]; y[i] = y[n - 1];
            g[n - 1] = 0; x[n - 1] = r0; y[n - 1] = r1;
            n--; i--;
        }
    }
    return n;
}

/* COL[i] = smallest j > i that qualifies: src/kernel.cu:1180-1235. */
void vxo_collapse_col(const vxo_params *p, int pass, const double *x, const double *y,
                      const double *g, int64_t n, int32_t *col) {
    const double eps2 = p->eps * p->eps;
    const double rd2 = p->r_col_diff_sign * p->r_col_diff_sign * eps2;
    const double rs2 = p->r_col_same_sign * p->r_col_same_sign * eps2;
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        const double r0 = x[i], r1 = y[i], gi = g[i];
        int32_t c = -1;
        for (int64_t j = i + 1; j < n; ++j) {
            double dx = r0 - x[j], dy = r1 - y[j];
            double r2 = fma(dx, dx, dy * dy);
            if (pass == 1) {
                if (gi * g[j] < 0 && r2 < rd2) { c = (int32_t)j; break; }
            } else {
                if (gi * g[j] > 0 && r2 < rs2 && fabs(gi + g[j]) < p->max_ve_g) { c = (int32_t)j; break; }
            }
        }
        col[i] = c;
    }
}

/* Serial greedy merge: src/kernel.cu:1237-1271. */
void vxo_collapse_merge(int pass, double *x, double *y, double *g, int64_t n, int32_t *col) {
    for (int64_t i = 0; i < n; ++i) {
        if (col[i] > -1) {
            int64_t j = col[i];
            if (pass == 1) {
                double ai = fabs(g[i]), aj = fabs(g[j]);
                double mn = ai + aj;
                x[i] = (x[i] * ai + x[j] * aj) / fabs(mn);
                y[i] = (y[i] * ai + y[j] * aj) / fabs(mn);
                g[i] = g[i] + g[j];
            } else {
                double ng = g[i] + g[j];
                x[i] = (x[i] * g[i] + x[j] * g[j]) / ng;
                y[i] = (y[i] * g[i] + y[j] * g[j]) / ng;
                g[i] = ng;
            }
            g[j] = 0;
            x[j] = 1e10;
            y[j] = 1e10;
            col[j] = -1;
        }
    }
}

/* One collapse pass, up to n_col rounds: src/unit_1.cu:1137-1216. */
int64_t vxo_collapse(const vxo_params *p, int pass, double *x, double *y, double *g,
                     int64_t n, int32_t *col) {
    for (int64_t cc = 0; cc < p->n_col; ++cc) {
        vxo_collapse_col(p, pass, x, y, g, n, col);
        vxo_collapse_merge(pass, x, y, g, n, col);
        int64_t nt = vxo_compact(x, y, g, n, p->drop_eps);
        if (nt == n) break;
        n = nt;
    }
    return n;
}

/* Probe velocity: src/kernel.cu:1434-1475 (velocity_control_Kernel). */
void vxo_probe(const vxo_params *p, const double *x, const double *y, const double *g,
               int64_t n, const double *px, const double *py, int64_t np,
               double *vx, double *vy) {
    const double eps2 = p->eps * p->eps;
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < np; ++i) {
        if (p->prec == VXO_PREC_FP64) {
            double y0 = 0.0, y1 = 0.0;
            for (int64_t j = 0; j < n; ++j) {
                double dx = px[i] - x[j], dy = py[i] - y[j];
                double m = g[j] / fmax(fma(dx, dx, dy * dy), eps2);
                y1 = fma(m, dx, y1);
                y0 = fma(-m, dy, y0);
            }
            vx[i] = y0 / TWO_PI + p->vinf_x;
            vy[i] = y1 / TWO_PI + p->vinf_y;
        } else {
            const float a0 = (float)px[i], a1 = (float)py[i], e2 = (float)eps2;
            float y0 = 0.0f, y1 = 0.0f;
            for (int64_t j = 0; j < n; ++j) {
                float dx = a0 - (float)x[j], dy = a1 - (float)y[j];
                float m = (float)g[j] / fmaxf(fmaf(dx, dx, dy * dy), e2);
                y1 = fmaf(m, dx, y1);
                y0 = fmaf(-m, dy, y0);
            }
            vx[i] = (double)y0 / TWO_PI + p->vinf_x;
            vy[i] = (double)y1 / TWO_PI + p->vinf_y;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* One time step in the order of src/main.c:676-784: birth, velocity,
 * diffusion (vortex, wall), convection with absorption, sums, compaction,
 * collapse of opposite then same signs. */
int64_t vxo_step(const vxo_params *p, const vxo_panel *pan, int64_t P,
                 const double *Minv, vxo_state *st) {
    int64_t n0 = st->n;
    double *R = (double *)malloc(sizeof(double) * P);
    double *gam = (double *)malloc(sizeof(double) * P);
    vxo_birth_rhs(p, pan, P, st->x, st->y, st->g, n0, R);
    vxo_birth_gamma(P, Minv, R, st->dg, gam);
    vxo_birth_place(p, pan, P, gam, st->x + n0, st->y + n0, st->g + n0);
    free(R); free(gam);
    int64_t n = n0 + P;
    int64_t s = round32(n);
    vxo_velocity(p, st->x, st->y, st->g, n, s, st->vx, st->vy, st->d);
    vxo_diffusion(p, st->x, st->y, st->g, n, st->d, st->vx, st->vy);
    vxo_wall_diffusion(p, pan, P, st->x, st->y, n, st->d, st->vx, st->vy);
    double *tmp = (double *)malloc(sizeof(double) * 4 * (size_t)n);
    int32_t *col = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    vxo_advect(p, pan, P, st->x, st->y, st->g, st->vx, st->vy, n, P,
               tmp, tmp + n, tmp + 2 * n, tmp + 3 * n);
    vxo_sums(p, n, tmp, tmp + n, tmp + 2 * n, tmp + 3 * n, &st->dg, &st->fx, &st->fy, &st->m);
    n = vxo_compact(st->x, st->y, st->g, n, p->drop_eps);
    n = vxo_collapse(p, 1, st->x, st->y, st->g, n, col);
    n = vxo_collapse(p, 2, st->x, st->y, st->g, n, col);
    free(tmp); free(col);
    st->n = n;
    return n;
}

/* Target range [i0, i1) of vxo_velocity / vxo_diffusion over all n sources
 * (the CPU baseline times a sample of targets and extrapolates). */
void vxo_velocity_targets(const vxo_params *p, const double *x, const double *y, const double *g,
                          int64_t n, int64_t i0, int64_t i1, double *vx, double *vy, double *d) {
    const double eps2 = p->eps * p->eps;
    const int64_t s = round32(n);
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = i0; i < i1; ++i) {
        const double a0 = x[i], a1 = y[i];
        double d1 = 1e5, d2 = 1e5, d3 = 1e5, y0 = 0.0, y1 = 0.0;
        for (int64_t j = 0; j < s; ++j) {
            if (j == i) continue;
            double dx = a0 - x[j], dy = a1 - y[j];
            double r2 = fma(dx, dx, dy * dy);
            NN3_INSERT(d1, d2, d3, r2, fmin, fmax);
            if (j < n) {
                double m = g[j] / fmax(r2, eps2);
                y1 = fma(m, dx, y1);
                y0 = fma(-m, dy, y0);
            }
        }
        d[i - i0] = (sqrt(d1) + sqrt(d2) + sqrt(d3)) / 3;
        vx[i - i0] = y0 / TWO_PI + p->vinf_x;
        vy[i - i0] = y1 / TWO_PI + p->vinf_y;
    }
}

void vxo_diffusion_targets(const vxo_params *p, const double *x, const double *y, const double *g,
                           int64_t n, int64_t i0, int64_t i1, const double *d, double *vx, double *vy) {
    const double thr = 0.001 * p->eps;
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = i0; i < i1; ++i) {
        const double a0 = x[i], a1 = y[i], dd = d[i - i0];
        double I2x = 0.0, I2y = 0.0, I1 = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            double dx = a0 - x[j], dy = a1 - y[j];
            double dist = sqrt(fma(dx, dx, dy * dy));
            if (dist > thr) {
                double m = g[j] / dist;
                double e = exp(-dist / dd);
                double me = m * e;
                I2x = fma(-me, dx, I2x);
                I2y = fma(-me, dy, I2y);
                I1 = fma(g[j], e, I1);
            }
        }
        if (fabs(I1) > 1e-5) {
            vx[i - i0] += -p->nu * I2x / (I1 * dd);
            vy[i - i0] += -p->nu * I2y / (I1 * dd);
        }
    }
}
