// vx_birth.cu — panel system (influence matrix + Gauss-Jordan inverse on the
// device) and vortex birth: right-hand side over all particles, strengths
// gamma = M [R; dg], placement of one new vortex per panel.
//
// Reference: matr_creation/inverse_matrix src/unit_1.cu:115-402,
// Right_part_Kernel src/kernel.cu:779-847, birth_Kernel src/kernel.cu:849-873.
#include "vx_internal.cuh"

// ---------------------------------------------------------------------------
// Influence matrix L (P+1)^2: one thread per entry, the expression trees of
// src/unit_1.cu:270-373 (see the oracle's panel_influence).
__device__ __forceinline__ double vx_sp(const double a[2], const double b[2]) {
    return a[0] * b[0] + a[1] * b[1];
}

__global__ void k_panel_influence(const vx_panel *pan, int P, double *L) {
    const long long S = P + 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S * S;
         e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e / S), j = (int)(e % S);
        double val;
        if (i == P) {
            val = (j == P) ? 0.0 : pan[j].length;     // Kelvin row
        } else if (j == P) {
            val = 1.0;
        } else if (i == j) {
            val = -0.5;
        } else {
            double a0[2], a1[2], b0[2], b1[2];
            bool next = (j == i + 1) || (j == 0 && i == P - 1);
            const vx_panel &pi = pan[i], &pj = pan[j];
            if (next) {
                a1[0] = pi.left[0];  a1[1] = pi.left[1];
                a0[0] = pi.right[0]; a0[1] = pi.right[1];
                b1[0] = pj.left[0];  b1[1] = pj.left[1];
                b0[0] = pj.right[0]; b0[1] = pj.right[1];
            } else {
                a0[0] = pi.left[0];  a0[1] = pi.left[1];
                a1[0] = pi.right[0]; a1[1] = pi.right[1];
                b0[0] = pj.left[0];  b0[1] = pj.left[1];
                b1[0] = pj.right[0]; b1[1] = pj.right[1];
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
            double q11 = 0.0, q21 = 0.0;
            bool adj = (j == i - 1) || (j == i + 1) || (j == 0 && i == P - 1) || (i == 0 && j == P - 1);
            if (!adj) {
                q11 = atan(vx_sp(di, p1) / z1) - atan(vx_sp(di, p2) / z1);
                q21 = 0.5 * log(vx_sp(p2, p2) / vx_sp(p1, p1));
            }
            double q12 = atan(vx_sp(di, s2) / z2) - atan(vx_sp(di, s1) / z2);
            double q13 = atan(vx_sp(dj, p2) / z3) - atan(vx_sp(dj, s2) / z3);
            double q22 = 0.5 * log(vx_sp(s1, s1) / vx_sp(s2, s2));
            double q23 = 0.5 * log(vx_sp(p2, p2) / vx_sp(s2, s2));
            double c1[2], c2[2], c3[2];
            for (int k = 0; k < 2; ++k)
                c1[k] = vx_sp(dj, p1) * di[k] + vx_sp(di, s1) * dj[k] - vx_sp(di, dj) * s1[k];
            for (int k = 0; k < 2; ++k) c2[k] = c1[k] + vx_sp(dj, dj) * di[k];
            for (int k = 0; k < 2; ++k) c3[k] = vx_sp(di, di) * dj[k];
            double f = 1.0 / (VX_TWO_PI * sqrt(vx_sp(dj, dj)) * vx_sp(di, di));
            double v0 = f * (q11 * c1[0] + q12 * c2[0] + q13 * c3[0]
                             + (q21 * c1[1] + q22 * c2[1] + q23 * c3[1]));
            double v1 = f * (q11 * c1[1] + q12 * c2[1] + q13 * c3[1]
                             - (q21 * c1[0] + q22 * c2[0] + q23 * c3[0]));
            val = v0 * pi.tang[0] + v1 * pi.tang[1];
        }
        L[e] = val;
    }
}

__global__ void k_identity(double *A, long long S) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S * S;
         e += (long long)gridDim.x * blockDim.x)
        A[e] = (e / S == e % S) ? 1.0 : 0.0;
}

// Block-wide arg-max of |A[i][col]| over i in [lo, S): the first row that
// holds the maximum wins (the reference's strict '>' scan).
__device__ void vx_block_argmax(const double *A, long long S, long long lo, long long col,
                                double *s_val, long long *s_idx, double &best, long long &bidx) {
    double mv = -1.0;
    long long mi = S;
    for (long long i = lo + threadIdx.x; i < S; i += blockDim.x) {
        double a = fabs(A[i * S + col]);
        if (a > mv) { mv = a; mi = i; }
    }
    s_val[threadIdx.x] = mv;
    s_idx[threadIdx.x] = mi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            double a = s_val[threadIdx.x + o];
            long long ai = s_idx[threadIdx.x + o];
            if (a > s_val[threadIdx.x] || (a == s_val[threadIdx.x] && ai < s_idx[threadIdx.x])) {
                s_val[threadIdx.x] = a;
                s_idx[threadIdx.x] = ai;
            }
        }
        __syncthreads();
    }
    best = s_val[0];
    bidx = s_idx[0];
    __syncthreads();
}

__device__ void vx_block_swap_rows(double *A, long long S, long long r1, long long r2) {
    if (r1 == r2) return;
    for (long long j = threadIdx.x; j < S; j += blockDim.x) {
        double t = A[r1 * S + j];
        A[r1 * S + j] = A[r2 * S + j];
        A[r2 * S + j] = t;
    }
}

// Pivot step k of src/unit_1.cu:160-227: singularity checks, choice and swap
// of the pivot row for column k+1, then the multipliers c[i] = A[i][k]/A[k][k].
__global__ void k_gj_pivot(double *A, double *Inv, long long S, long long k, double *c, int *flag) {
    __shared__ double s_val[1024];
    __shared__ long long s_idx[1024];
    if (*flag) return;
    const double DELT = 1e-12;
    double best;
    long long line;
    if (k == 0 && fabs(A[0]) < DELT) {
        vx_block_argmax(A, S, 1, 0, s_val, s_idx, best, line);
        if (best > fabs(A[0])) {
            vx_block_swap_rows(A, S, 0, line);
            vx_block_swap_rows(Inv, S, 0, line);
        }
        __syncthreads();
    }
    if (fabs(A[k * S + k]) < DELT) { if (threadIdx.x == 0) *flag = 1; return; }
    vx_block_argmax(A, S, k + 1, k + 1, s_val, s_idx, best, line);
    if (best < DELT) { if (threadIdx.x == 0) *flag = 1; return; }
    vx_block_swap_rows(A, S, k + 1, line);
    vx_block_swap_rows(Inv, S, k + 1, line);
    __syncthreads();
    const double piv = A[k * S + k];
    for (long long i = threadIdx.x; i < S; i += blockDim.x) c[i] = A[i * S + k] / piv;
}

// Row operations of step k: every row but k loses c[i] times row k.
__global__ void k_gj_elim(double *A, double *Inv, long long S, long long k, const double *c,
                          const int *flag) {
    if (*flag) return;
    const long long W = 2 * S;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S * W;
         e += (long long)gridDim.x * blockDim.x) {
        long long i = e / W, j = e % W;
        if (i == k) continue;
        double ci = c[i];
        if (j < S) A[i * S + j] = A[i * S + j] - ci * A[k * S + j];
        else { j -= S; Inv[i * S + j] = Inv[i * S + j] - ci * Inv[k * S + j]; }
    }
}

__global__ void k_gj_last_pivot(const double *A, long long S, double *c, int *flag) {
    if (*flag) return;
    const long long l = S - 1;
    if (fabs(A[l * S + l]) < 1e-12) { if (threadIdx.x == 0) *flag = 1; return; }
    for (long long i = threadIdx.x; i < l; i += blockDim.x) c[i] = A[i * S + l] / A[l * S + l];
}

__global__ void k_gj_last_elim(double *Inv, long long S, const double *c, const int *flag) {
    if (*flag) return;
    const long long l = S - 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < l * S;
         e += (long long)gridDim.x * blockDim.x) {
        long long i = e / S, j = e % S;
        Inv[i * S + j] = Inv[i * S + j] - c[i] * Inv[l * S + j];
    }
}

__global__ void k_gj_scale(const double *A, double *Inv, long long S, const int *flag) {
    if (*flag) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S * S;
         e += (long long)gridDim.x * blockDim.x) {
        long long i = e / S;
        Inv[e] = Inv[e] / A[i * S + i];
    }
}

// d_work must hold 2 (P+1)^2 + (P+1) doubles.  *d_flag is set when a pivot
// falls below 1e-12 (the reference returns NULL then).
cudaError_t vx_build_matrix(const VxLaunch &L, const vx_panel *d_pan, int P, double *d_minv,
                            double *d_work, int *d_flag, double *d_L_out) {
    const long long S = P + 1;
    double *A = d_work;
    double *c = d_work + S * S;
    const int grid = L.num_sms * 4;
    cudaMemsetAsync(d_flag, 0, sizeof(int), L.stream);
    k_panel_influence<<<grid, 256, 0, L.stream>>>(d_pan, P, A); VX_COUNT(L);
    if (d_L_out) cudaMemcpyAsync(d_L_out, A, sizeof(double) * S * S, cudaMemcpyDeviceToDevice, L.stream);
    k_identity<<<grid, 256, 0, L.stream>>>(d_minv, S); VX_COUNT(L);
    for (long long k = 0; k < S - 1; ++k) {
        k_gj_pivot<<<1, 1024, 0, L.stream>>>(A, d_minv, S, k, c, d_flag); VX_COUNT(L);
        k_gj_elim<<<grid, 256, 0, L.stream>>>(A, d_minv, S, k, c, d_flag); VX_COUNT(L);
    }
    k_gj_last_pivot<<<1, 1024, 0, L.stream>>>(A, S, c, d_flag); VX_COUNT(L);
    k_gj_last_elim<<<grid, 256, 0, L.stream>>>(d_minv, S, c, d_flag); VX_COUNT(L);
    k_gj_scale<<<grid, 256, 0, L.stream>>>(A, d_minv, S, d_flag); VX_COUNT(L);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Step begin: V_inf ramp (src/main.c:654-659) and the pre-birth count.
__global__ void k_step_begin(VxScalars *S) {
    if (S->step < S->incr_steps) {
        S->vinf[0] += S->dvinf[0];
        S->vinf[1] += S->dvinf[1];
    }
    S->n0 = S->n;
}

cudaError_t vx_launch_step_begin(const VxLaunch &L, VxScalars *S) {
    k_step_begin<<<1, 1, 0, L.stream>>>(S); VX_COUNT(L);
    return cudaGetLastError();
}

__global__ void k_step_end(VxScalars *S) { S->step += 1; }

// ---------------------------------------------------------------------------
// Birth right-hand side (src/kernel.cu:779-847), partial sums per source
// chunk.  The difference of the two arctangents is evaluated as one
// atan2 of the same angle: with A = s0.d, B = s1.d and B - A = |d|^2,
//   atan(A/z) - atan(B/z) = atan2(-|d|^2 z, z^2 + A B).
constexpr int RHS_T = 128;

template <typename T>
struct RhsMath;
template <>
struct RhsMath<double> {
    static __device__ __forceinline__ double at2(double y, double x) { return atan2(y, x); }
    static __device__ __forceinline__ double lg(double x) { return log(x); }
};
template <>
struct RhsMath<float> {
    static __device__ __forceinline__ float at2(float y, float x) { return atan2f(y, x); }
    static __device__ __forceinline__ float lg(float x) { return logf(x); }
};

template <typename T>
__global__ void __launch_bounds__(RHS_T) k_rhs_partial(VxView v, const VxScalars *S,
                                                       const vx_panel *pan, int P, int P32,
                                                       double *part, int nchunks) {
    __shared__ T sx[RHS_T], sy[RHS_T], sg[RHS_T];
    const long long n0 = S->n0;
    const long long cs = vx_ceil_div(vx_ceil_div(n0, nchunks), RHS_T) * RHS_T;
    const int tiles = (P + RHS_T - 1) / RHS_T;
    const long long items = (long long)tiles * nchunks;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int pt = (int)(it % tiles);
        const long long sc = it / tiles;
        const int i = pt * RHS_T + threadIdx.x;
        const bool valid = i < P;
        T al0 = 0, al1 = 0, d0 = 1, d1 = 0;
        if (valid) {
            al0 = (T)pan[i].left[0]; al1 = (T)pan[i].left[1];
            d0 = (T)pan[i].right[0] - al0; d1 = (T)pan[i].right[1] - al1;
        }
        const T kd0 = -d1, kd1 = d0;
        const T dd2 = fma(d0, d0, d1 * d1);
        T y0 = 0, y1 = 0;
        const long long j0 = sc * cs, j1 = min(n0, j0 + cs);
        for (long long jt = j0; jt < j1; jt += RHS_T) {
            __syncthreads();
            long long j = jt + threadIdx.x;
            if (j < j1) {
                sx[threadIdx.x] = (T)v.x[j * v.ps];
                sy[threadIdx.x] = (T)v.y[j * v.ps];
                sg[threadIdx.x] = (T)v.g[j * v.ps];
            }
            __syncthreads();
            const int cnt = (int)min((long long)RHS_T, j1 - jt);
            for (int q = 0; q < cnt; ++q) {
                T s00 = al0 - sx[q], s01 = al1 - sy[q];
                T s10 = s00 + d0, s11 = s01 + d1;
                T A = fma(s00, d0, s01 * d1);
                T B = fma(s10, d0, s11 * d1);
                T z = fma(d0, s01, -(d1 * s00));
                T alpha = RhsMath<T>::at2(-dd2 * z, fma(z, z, A * B));
                T r1 = fma(s10, s10, s11 * s11), r0 = fma(s00, s00, s01 * s01);
                T beta = (T)0.5 * RhsMath<T>::lg(r1 / r0);
                y0 = fma(sg[q], fma(alpha, d0, beta * kd0), y0);
                y1 = fma(sg[q], fma(alpha, d1, beta * kd1), y1);
            }
        }
        if (valid) {
            part[(sc * P32 + i) * 2 + 0] = (double)y0;
            part[(sc * P32 + i) * 2 + 1] = (double)y1;
        }
    }
}

__global__ void k_rhs_final(const VxScalars *S, const vx_panel *pan, int P, int P32,
                            const double *part, int nchunks, double *R) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    double y0 = 0.0, y1 = 0.0;
    for (int sc = 0; sc < nchunks; ++sc) {
        y0 += part[((long long)sc * P32 + i) * 2 + 0];
        y1 += part[((long long)sc * P32 + i) * 2 + 1];
    }
    double d0 = pan[i].right[0] - pan[i].left[0], d1 = pan[i].right[1] - pan[i].left[1];
    double mnog = 1.0 / (VX_TWO_PI * (d0 * d0 + d1 * d1));
    R[i] = -((mnog * y0 + S->vinf[0]) * pan[i].tang[0] + (mnog * y1 + S->vinf[1]) * pan[i].tang[1]);
}

// gamma_i = sum_j M_ij R_j + M_iP dg, sequential in j with fma (as the
// oracle), one thread per row; ld is the matrix row stride.
__global__ void k_gamma(const VxScalars *S, const double *M, long long ld, int P, const double *R,
                        double *gamma) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const double *row = M + (long long)i * ld;
    double acc = 0.0;
    for (int j = 0; j < P; ++j) acc = fma(row[j], R[j], acc);
    gamma[i] = fma(row[P], S->dg, acc);
}

// One new vortex per panel at [n0, n0+P) (src/kernel.cu:862-872).
__global__ void k_place(VxParams p, VxView v, VxScalars *S, const vx_panel *pan, int P,
                        const double *gamma) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const long long n0 = S->n0;
    if (i < P) {
        int in = (int)pan[i].n_of_rpanel;
        double mx = (pan[i].left[0] + pan[i].right[0]) / 2;
        double my = (pan[i].left[1] + pan[i].right[1]) / 2;
        double bx, by;
        if (p.birth_mode == VX_BIRTH_FILE) {
            bx = pan[i].birth[0]; by = pan[i].birth[1];
        } else if (p.birth_mode == VX_BIRTH_HALF_PANEL) {
            double h = 0.5 * pan[i].length;
            bx = mx + h * pan[i].norm[0]; by = my + h * pan[i].norm[1];
        } else {
            bx = mx + 1e-6 * pan[i].norm[0]; by = my + 1e-6 * pan[i].norm[1];
        }
        long long k = (n0 + i) * v.ps;
        v.x[k] = bx;
        v.y[k] = by;
        v.g[k] = 0.5 * (gamma[i] * pan[i].length + gamma[in] * pan[in].length);
    }
    if (i == 0) S->n = n0 + P;
}

cudaError_t vx_launch_birth_ld(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                               VxWork &w, const vx_panel *pan, const double *minv, long long ld,
                               int rhs_chunks) {
    const int P = p.P, P32 = (int)vx_round32(P);
    const int tiles = (P + RHS_T - 1) / RHS_T;
    const int grid = (int)min((long long)tiles * rhs_chunks, (long long)L.num_sms * 8);
    if (p.prec == VX_PREC_FP32)
        k_rhs_partial<float><<<grid, RHS_T, 0, L.stream>>>(v, S, pan, P, P32, w.rhs_part, rhs_chunks);
    else
        k_rhs_partial<double><<<grid, RHS_T, 0, L.stream>>>(v, S, pan, P, P32, w.rhs_part, rhs_chunks);
    VX_COUNT(L);
    const int b = (P + 127) / 128;
    k_rhs_final<<<b, 128, 0, L.stream>>>(S, pan, P, P32, w.rhs_part, rhs_chunks, w.R); VX_COUNT(L);
    k_gamma<<<b, 128, 0, L.stream>>>(S, minv, ld, P, w.R, w.gamma); VX_COUNT(L);
    k_place<<<b, 128, 0, L.stream>>>(p, v, S, pan, P, w.gamma); VX_COUNT(L);
    return cudaGetLastError();
}

// Native engine: the inverse is stored unpadded, row stride P+1.
cudaError_t vx_launch_birth(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                            VxWork &w, const vx_panel *pan, const double *minv, int rhs_chunks) {
    return vx_launch_birth_ld(L, p, v, S, w, pan, minv, (long long)p.P + 1, rhs_chunks);
}

cudaError_t vx_launch_step_end(const VxLaunch &L, VxScalars *S) {
    k_step_end<<<1, 1, 0, L.stream>>>(S); VX_COUNT(L);
    return cudaGetLastError();
}
