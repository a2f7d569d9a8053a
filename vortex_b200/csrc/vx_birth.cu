// vx_birth.cu — panel system (influence matrix + Gauss-Jordan inverse on the
// device) and vortex birth: right-hand side over all particles, strengths
// gamma = M [R; dg], placement of one new vortex per panel.
//
// Reference: matr_creation/inverse_matrix src/unit_1.cu:115-402,
// Right_part_Kernel src/kernel.cu:779-847, birth_Kernel src/kernel.cu:849-873.
#include <algorithm>

#include "vx_internal.cuh"

// ---------------------------------------------------------------------------
// Influence matrix L (P+1)^2: one thread per entry, the expression trees of
// src/unit_1.cu:270-373 (see the oracle's panel_influence).
__device__ __forceinline__ double vx_sp(const double a[2], const double b[2]) {
    return a[0] * b[0] + a[1] * b[1];
}

VX_DEVK void k_panel_influence_body(VxBlkB<0, 0> vb, const vx_panel *pan, int P, double *L) {
    const long long S = P + 1;
    for (long long e = vb.x * (long long)blockDim.x + threadIdx.x; e < S * S;
         e += (long long)vb.n * blockDim.x) {
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
__global__ void k_panel_influence(const vx_panel *pan, int P, double *L) {
    VX_PDL_WAIT();
    k_panel_influence_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, pan, P, L);
}

VX_DEVK void k_identity_body(VxBlkB<0, 0> vb, double *A, long long S) {
    for (long long e = vb.x * (long long)blockDim.x + threadIdx.x; e < S * S;
         e += (long long)vb.n * blockDim.x)
        A[e] = (e / S == e % S) ? 1.0 : 0.0;
}
__global__ void k_identity(double *A, long long S) {
    VX_PDL_WAIT();
    k_identity_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, A, S);
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
// The reference chooses the pivot of column k+1 before column k is
// eliminated, so a well-conditioned system can still meet a pivot below
// 1e-12 there.  robust != 0: ordinary partial pivoting instead (the pivot of
// column k chosen among rows k.. after the previous eliminations).
VX_DEVK void k_gj_pivot_body(VxBlkB<0, 0> vb, double *A, double *Inv, long long S, long long k, double *c, int *flag, int robust) {
    __shared__ double s_val[1024];
    __shared__ long long s_idx[1024];
    if (*flag) return;
    const double DELT = 1e-12;
    double best;
    long long line;
    if (robust) {
        vx_block_argmax(A, S, k, k, s_val, s_idx, best, line);
        if (best < DELT) { if (threadIdx.x == 0) *flag = 1; return; }
        vx_block_swap_rows(A, S, k, line);
        vx_block_swap_rows(Inv, S, k, line);
        __syncthreads();
        const double piv = A[k * S + k];
        for (long long i = threadIdx.x; i < S; i += blockDim.x) c[i] = A[i * S + k] / piv;
        return;
    }
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
__global__ void k_gj_pivot(double *A, double *Inv, long long S, long long k, double *c, int *flag, int robust) {
    VX_PDL_WAIT();
    k_gj_pivot_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, A, Inv, S, k, c, flag, robust);
}

// Row operations of step k: every row but k loses c[i] times row k.
VX_DEVK void k_gj_elim_body(VxBlkB<0, 0> vb, double *A, double *Inv, long long S, long long k, const double *c,
                            const int *flag) {
    if (*flag) return;
    const long long W = 2 * S;
    for (long long e = vb.x * (long long)blockDim.x + threadIdx.x; e < S * W;
         e += (long long)vb.n * blockDim.x) {
        long long i = e / W, j = e % W;
        if (i == k) continue;
        double ci = c[i];
        if (j < S) A[i * S + j] = A[i * S + j] - ci * A[k * S + j];
        else { j -= S; Inv[i * S + j] = Inv[i * S + j] - ci * Inv[k * S + j]; }
    }
}
__global__ void k_gj_elim(double *A, double *Inv, long long S, long long k, const double *c,
                          const int *flag) {
    VX_PDL_WAIT();
    k_gj_elim_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, A, Inv, S, k, c, flag);
}

VX_DEVK void k_gj_last_pivot_body(VxBlkB<0, 0> vb, const double *A, long long S, double *c, int *flag) {
    if (*flag) return;
    const long long l = S - 1;
    if (fabs(A[l * S + l]) < 1e-12) { if (threadIdx.x == 0) *flag = 1; return; }
    for (long long i = threadIdx.x; i < l; i += blockDim.x) c[i] = A[i * S + l] / A[l * S + l];
}
__global__ void k_gj_last_pivot(const double *A, long long S, double *c, int *flag) {
    VX_PDL_WAIT();
    k_gj_last_pivot_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, A, S, c, flag);
}

VX_DEVK void k_gj_last_elim_body(VxBlkB<0, 0> vb, double *Inv, long long S, const double *c, const int *flag) {
    if (*flag) return;
    const long long l = S - 1;
    for (long long e = vb.x * (long long)blockDim.x + threadIdx.x; e < l * S;
         e += (long long)vb.n * blockDim.x) {
        long long i = e / S, j = e % S;
        Inv[i * S + j] = Inv[i * S + j] - c[i] * Inv[l * S + j];
    }
}
__global__ void k_gj_last_elim(double *Inv, long long S, const double *c, const int *flag) {
    VX_PDL_WAIT();
    k_gj_last_elim_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, Inv, S, c, flag);
}

VX_DEVK void k_gj_scale_body(VxBlkB<0, 0> vb, const double *A, double *Inv, long long S, const int *flag) {
    if (*flag) return;
    for (long long e = vb.x * (long long)blockDim.x + threadIdx.x; e < S * S;
         e += (long long)vb.n * blockDim.x) {
        long long i = e / S;
        Inv[e] = Inv[e] / A[i * S + i];
    }
}
__global__ void k_gj_scale(const double *A, double *Inv, long long S, const int *flag) {
    VX_PDL_WAIT();
    k_gj_scale_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, A, Inv, S, flag);
}

// d_work must hold 2 (P+1)^2 + (P+1) doubles.  *d_flag is set when a pivot
// falls below 1e-12 (the reference returns NULL then).
cudaError_t vx_build_matrix(const VxLaunch &L, const vx_panel *d_pan, int P, double *d_minv,
                            double *d_work, int *d_flag, double *d_L_out, int robust) {
    const long long S = P + 1;
    double *A = d_work;
    double *c = d_work + S * S;
    const int grid = L.num_sms * 4;
    cudaMemsetAsync(d_flag, 0, sizeof(int), L.stream);
    vx_launch<k_panel_influence, k_panel_influence_body>(L, grid, 256, 0, d_pan, P, A);
    if (d_L_out) cudaMemcpyAsync(d_L_out, A, sizeof(double) * S * S, cudaMemcpyDeviceToDevice, L.stream);
    if (robust == 3)   // blocked LU with partial pivoting (vx_lu.cu)
        return vx_invert_lu(L, A, d_minv, S, reinterpret_cast<int *>(c), d_flag);
    vx_launch<k_identity, k_identity_body>(L, grid, 256, 0, d_minv, S);
    for (long long k = 0; k < S - 1; ++k) {
        vx_launch<k_gj_pivot, k_gj_pivot_body>(L, 1, 1024, 0, A, d_minv, S, k, c, d_flag, robust);
        vx_launch<k_gj_elim, k_gj_elim_body>(L, grid, 256, 0, A, d_minv, S, k, c, d_flag);
    }
    vx_launch<k_gj_last_pivot, k_gj_last_pivot_body>(L, 1, 1024, 0, A, S, c, d_flag);
    vx_launch<k_gj_last_elim, k_gj_last_elim_body>(L, grid, 256, 0, d_minv, S, c, d_flag);
    vx_launch<k_gj_scale, k_gj_scale_body>(L, grid, 256, 0, A, d_minv, S, d_flag);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Step begin: V_inf ramp (src/main.c:654-659) and the pre-birth count.
VX_DEVK void k_step_begin_body(VxBlkB<0, 0> vb, VxScalars *S) {
    if (S->step < S->incr_steps) {
        S->vinf[0] += S->dvinf[0];
        S->vinf[1] += S->dvinf[1];
    }
    S->n0 = S->n;
}
__global__ void k_step_begin(VxScalars *S) {
    VX_PDL_WAIT();
    k_step_begin_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, S);
}

cudaError_t vx_launch_step_begin(const VxLaunch &L, VxScalars *S) {
    vx_launch<k_step_begin, k_step_begin_body>(L, 1, 1, 0, S);
    return cudaGetLastError();
}

VX_DEVK void k_step_end_body(VxBlkB<0, 0> vb, VxScalars *S) {
S->step += 1; }
__global__ void k_step_end(VxScalars *S) {
    VX_PDL_WAIT();
    k_step_end_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, S);
}

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
VX_DEVK void k_rhs_partial_body(VxBlkB<RHS_T, 0> vb, const VxView &v, const VxScalars *S,
                                const vx_panel *pan, int P, int P32,
                                double *part, int sms) {
    const int nchunks = vx_rhs_chunks(S->n0, P, sms);   // from the body's own count
    __shared__ T sx[RHS_T], sy[RHS_T], sg[RHS_T];
    const long long n0 = S->n0;
    const long long cs = vx_ceil_div(vx_ceil_div(n0, nchunks), RHS_T) * RHS_T;
    const int tiles = (P + RHS_T - 1) / RHS_T;
    const long long items = (long long)tiles * nchunks;
    for (long long it = vb.x; it < items; it += vb.n) {
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
template <typename T>
__global__ void __launch_bounds__(RHS_T) k_rhs_partial(VxView v, const VxScalars *S,
                                                       const vx_panel *pan, int P, int P32,
                                                       double *part, int sms) {
    VX_PDL_WAIT();
    k_rhs_partial_body<T>(VxBlkB<RHS_T, 0>{blockIdx.x, gridDim.x}, v, S, pan, P, P32, part, sms);
}

// ---------------------------------------------------------------------------
// Birth right-hand side of the bulk form with a far field.  The sum over
// vortex j of the panel terms (alpha d + beta k_d) / (2 pi |d|^2) is the
// mean velocity induced along the panel; with w(z) = u - i v and
// dz = (tau_x + i tau_y) ds along it,
//   mean (u, v) . tau = Re[ (1 / dz_panel) integral w dz ],
//   integral_{za}^{zb} G / (2 pi i (z - zj)) dz.
// For |zj - c| > 1.5 r_body (c: body centre) the kernel expands about c:
//   1 / (z - zj) = sum_l a_l (z - c)^l,  a_l = -1 / (zj - c)^(l+1),
// and the panel integral of the series is exact:
//   sum_l a_l [(zb - c)^(l+1) - (za - c)^(l+1)] / (l + 1).
// On the panels |z - c| <= r_body, so the terms fall as (2/3)^l (48 terms:
// the remainder below 3 (2/3)^49 = 7e-9 relative).  Far coefficients: FP64,
// fixed-order block partials.  Near vortices (inside 1.5 r_body) keep the
// direct FP32 panel terms, over a list compacted in index order.
constexpr int BF_T = 256;
constexpr int BF_P = VX_BF_P;
static_assert(BF_P % 16 == 0, "16 far-field coefficients per pass");

struct bcplx {
    double r, i;
};

// Source chunks of the far-field pass: two per SM's worth of the body
// (vx_body_sms of its count after birth), at most VX_BF_MAX_BLOCKS.
__device__ __forceinline__ int vx_bf_parts(long long n, int sms) {
    const int q = 2 * vx_body_sms(n, sms);
    return q < VX_BF_MAX_BLOCKS ? q : VX_BF_MAX_BLOCKS;
}

// Block b: sources [b cs, (b+1) cs) of the n0 pre-birth vortices.
__device__ __forceinline__ void bf_chunk(const VxScalars *S, int nb, int b, long long &j0, long long &j1) {
    const long long n0 = S->n0;
    const long long cs = vx_ceil_div(vx_ceil_div(n0, (long long)nb), (long long)BF_T) * BF_T;
    j0 = min((long long)b * cs, n0);
    j1 = min(j0 + cs, n0);
}

__device__ __forceinline__ bool bf_near(const VxParams &p, double x, double y) {
    const double dx = x - p.bc_x, dy = y - p.bc_y;
    return dx * dx + dy * dy <= p.b_rfar2;
}

// Far-field coefficient partials (one per block, fixed order) and the
// number of near sources of each block.  Each thread sums the terms of its
// own sources in registers, 16 coefficients per pass (a_16k .. a_16k+15 in
// pass k, from -G w^(16k+1), w^16 by squarings); then a reduce-scatter over the
// warp (at each halving a lane keeps the half of its values selected by its
// lane bit and adds the partner's copy: lane q ends with value q, i.e.
// coefficient q/2, part q&1) and a fixed-order sum over the block's warps.
// Partition q of nparts: sources [j0, j1) (bf_chunk).
__device__ __forceinline__ void bf_far_part(unsigned q, unsigned nparts, const VxParams &p, const VxView &v,
                                            const VxScalars *S, double *part, int *cnt, long long j0,
                                            long long j1) {
    __shared__ double sacc[BF_T / 32][32];
    __shared__ int snear[BF_T / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int nnear = 0;
    for (int pass = 0; pass < BF_P / 16; ++pass) {
        double acc[32];   // (re, im) of the pass's 16 coefficients
#pragma unroll
        for (int k = 0; k < 32; ++k) acc[k] = 0.0;
        for (long long j = j0 + threadIdx.x; j < j1; j += BF_T) {
            const double x = v.x[j * v.ps], y = v.y[j * v.ps], g = v.g[j * v.ps];
            if (bf_near(p, x, y)) {
                nnear += pass == 0;
                continue;
            }
            const double zr = x - p.bc_x, zi = y - p.bc_y;
            const double q = 1.0 / (zr * zr + zi * zi);
            const double wr = zr * q, wi = -zi * q;   // w = 1 / (zj - c)
            double tr = -g * wr, ti = -g * wi;        // a_0 term: -G w
            if (pass > 0) {                           // times w^(16 pass)
                double pr = wr, pi = wi;
#pragma unroll
                for (int s2 = 0; s2 < 4; ++s2) {
                    const double nr = pr * pr - pi * pi, ni = 2.0 * pr * pi;
                    pr = nr; pi = ni;
                }
                for (int k = 0; k < pass; ++k) {
                    const double nr = tr * pr - ti * pi, ni = tr * pi + ti * pr;
                    tr = nr; ti = ni;
                }
            }
#pragma unroll
            for (int l = 0; l < 16; ++l) {
                acc[2 * l] += tr;
                acc[2 * l + 1] += ti;
                const double nr = tr * wr - ti * wi, ni = tr * wi + ti * wr;
                tr = nr; ti = ni;
            }
        }
#pragma unroll
        for (int half = 16; half > 0; half >>= 1) {
            const bool up = (lane & half) != 0;
#pragma unroll
            for (int i = 0; i < half; ++i) {
                const double send = up ? acc[i] : acc[i + half];
                const double keep = up ? acc[i + half] : acc[i];
                acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, half);
            }
        }
        sacc[wid][lane] = acc[0];
        __syncthreads();
        if (threadIdx.x < 32) {
            double sum = 0.0;
            for (int q = 0; q < BF_T / 32; ++q) sum += sacc[q][threadIdx.x];
            // value q of this pass: coefficient 16 pass + q/2, part q&1
            part[((long long)q * BF_P + 16 * pass + (threadIdx.x >> 1)) * 2 + (threadIdx.x & 1)] = sum;
        }
        __syncthreads();
    }
    for (int o = 16; o > 0; o >>= 1) nnear += __shfl_xor_sync(0xffffffffu, nnear, o);
    if (lane == 0) snear[wid] = nnear;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int q = 0; q < BF_T / 32; ++q) t += snear[q];
        cnt[q] = t;
    }
}
// The sources are split into nparts fixed chunks whatever the grid; each
// block takes chunks blockIdx, blockIdx + grid, ...; an empty chunk has zero
// partials.  The block that finishes last then scans the chunks' near-source
// counts into offsets and adds the coefficient partials in chunk order
// (thread t scans the counts of chunks BF_SCAN_PER t .., then a warp and
// block scan of the thread totals).  The summed coefficients do not depend
// on the launch's grid.
constexpr int BF_SCAN_PER = VX_BF_MAX_BLOCKS / BF_T;
static_assert(BF_SCAN_PER * BF_T == VX_BF_MAX_BLOCKS, "whole chunks per scan thread");
VX_DEVK void k_bf_far_body(VxBlkB<BF_T, 2> vb, const VxParams &p, const VxView &v, VxScalars *S, double *part, int *cnt,
                           int sms, long long *off, double *coef) {
    const int nparts = vx_bf_parts(S->n0 + p.P, sms);
    for (unsigned q = vb.x; q < (unsigned)nparts; q += vb.n) {
        long long j0, j1;
        bf_chunk(S, nparts, q, j0, j1);
        if (j0 >= j1) {
            for (int t = threadIdx.x; t < 2 * BF_P; t += blockDim.x) part[(long long)q * 2 * BF_P + t] = 0.0;
            if (threadIdx.x == 0) cnt[q] = 0;
            continue;
        }
        bf_far_part(q, (unsigned)nparts, p, v, S, part, cnt, j0, j1);
    }
    if (!vx_last_block(&S->sync_ctr, vb.n)) return;
    __shared__ long long wsum[BF_T / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nb = nparts;
    long long c[BF_SCAN_PER], tot = 0;
    for (int q = 0; q < BF_SCAN_PER; ++q) {
        const int b = BF_SCAN_PER * t + q;
        c[q] = b < nb ? __ldcg(&cnt[b]) : 0;
        tot += c[q];
    }
    long long inc = tot;
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    long long run = inc - tot, all = 0;
    for (int q = 0; q < BF_T / 32; ++q) {
        run += q < warp ? wsum[q] : 0;
        all += wsum[q];
    }
    for (int q = 0; q < BF_SCAN_PER; ++q) {
        const int b = BF_SCAN_PER * t + q;
        if (b < nb) off[b] = run;
        run += c[q];
    }
    if (t == 0) {
        off[nb] = all;
        S->bf_nnear = all;
    }
    if (t < 2 * BF_P) {
        double acc = 0.0;
        for (int b = 0; b < nb; ++b) acc += __ldcg(&part[(long long)b * 2 * BF_P + t]);
        coef[t] = acc;
    }
}
__global__ void __launch_bounds__(BF_T) k_bf_far(VxParams p, VxView v, VxScalars *S, double *part, int *cnt,
                                                 int sms, long long *off, double *coef) {
    VX_PDL_WAIT();
    k_bf_far_body(VxBlkB<BF_T, 2>{blockIdx.x, gridDim.x}, p, v, S, part, cnt, sms, off, coef);
}

// Near sources of each block in index order (block-wide ballot scan).
__device__ __forceinline__ void bf_scatter_part(unsigned q, unsigned nparts, const VxParams &p, const VxView &v,
                                                const VxScalars *S, const long long *off, float4 *near) {
    __shared__ int swarp[BF_T / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long j0, j1;
    bf_chunk(S, nparts, q, j0, j1);
    long long base = off[q];
    for (long long jt = j0; jt < j1; jt += BF_T) {
        const long long j = jt + threadIdx.x;
        double x = 0.0, y = 0.0, g = 0.0;
        bool nr = false;
        if (j < j1) {
            x = v.x[j * v.ps]; y = v.y[j * v.ps]; g = v.g[j * v.ps];
            nr = bf_near(p, x, y);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, nr);
        __syncthreads();
        if (lane == 0) swarp[wid] = __popc(bal);
        __syncthreads();
        int before = 0, total = 0;
        for (int q = 0; q < BF_T / 32; ++q) {
            before += q < wid ? swarp[q] : 0;
            total += swarp[q];
        }
        if (nr)
            near[base + before + __popc(bal & ((1u << lane) - 1u))] = make_float4((float)x, (float)y, (float)g, 0.f);
        base += total;
    }
}
VX_DEVK void k_bf_scatter_body(VxBlkB<BF_T, 0> vb, const VxParams &p, const VxView &v, const VxScalars *S,
                               const long long *off, float4 *near, int sms) {
    const int nparts = vx_bf_parts(S->n0 + p.P, sms);
    for (unsigned q = vb.x; q < (unsigned)nparts; q += vb.n) bf_scatter_part(q, (unsigned)nparts, p, v, S, off, near);
}
__global__ void __launch_bounds__(BF_T) k_bf_scatter(VxParams p, VxView v, const VxScalars *S,
                                                     const long long *off, float4 *near, int sms) {
    VX_PDL_WAIT();
    k_bf_scatter_body(VxBlkB<BF_T, 0>{blockIdx.x, gridDim.x}, p, v, S, off, near, sms);
}

// atan2 in FP32 for the bulk form's near panel terms: the octant reduction
// (a = min(|x|,|y|) / max(|x|,|y|) in [0, 1], then pi/2 - r, pi - r and the
// sign of y) and atan(a) = a P(a^2) with P of degree 8, P(0) = 1, fitted here
// to atan on [0, 1] for least relative error (1.2e-7 relative, 9e-8
// absolute in FP32, the accuracy of the library atan2f).  Signed zeros and
// the x < 0 half-plane follow the usual atan2 conventions.
__device__ __forceinline__ float vx_atan2_bulk(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mn = fminf(ax, ay), mx = fmaxf(ax, ay);
    float rc;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rc) : "f"(mx));
    const float a = mx > 0.0f ? mn * rc : 0.0f;
    const float t = a * a;
    float p = 0.002921519335359335f;
    p = fmaf(p, t, -0.01637130416929722f);
    p = fmaf(p, t, 0.04321747645735741f);
    p = fmaf(p, t, -0.07552702724933624f);
    p = fmaf(p, t, 0.10666241496801376f);
    p = fmaf(p, t, -0.1421111822128296f);
    p = fmaf(p, t, 0.19993780553340912f);
    p = fmaf(p, t, -0.33333152532577515f);
    p = fmaf(p, t, 1.0f);
    float r = a * p;
    r = ay > ax ? 1.57079632679489662f - r : r;
    r = x < 0.0f ? 3.14159265358979324f - r : r;
    return copysignf(r, y);
}

__global__ void k_eval_atan2(const float *y, const float *x, float *out, long long n) {
    VX_PDL_WAIT();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = vx_atan2_bulk(y[i], x[i]);
}

// Validation hook: evaluates the bulk form's atan2 on device arrays.
extern "C" vx_status vx_eval_bulk_atan2(const float *y, const float *x, float *out, int64_t n) {
    if (n < 0 || (n > 0 && (!y || !x || !out))) return VX_ERR_ARG;
    if (n == 0) return VX_OK;
    k_eval_atan2<<<(int)std::min<long long>(vx_ceil_div((long long)n, 256LL), 4096LL), 256>>>(y, x, out, n);
    if (cudaDeviceSynchronize() != cudaSuccess) return VX_ERR_CUDA;
    return VX_OK;
}

// beta = ln(r1 / r0) / 2 for the bulk form.  With t = (r1 - r0) / (r1 + r0),
// ln(r1 / r0) / 2 = atanh(t); r1 - r0 = 2 A + |d|^2 comes without
// cancellation from the panel's own terms (num).  For |t| <= 1/4 (every
// source more than about two panel lengths away) the Taylor series of atanh,
// t (1 + t^2/3 + t^4/5 + ... + t^10/11), truncated below t^12/13 = 5e-9
// relative; closer sources take logf of the ratio.
__device__ __forceinline__ float vx_half_log_ratio(float r0, float r1, float num) {
    const float den = r0 + r1;
    float rc;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rc) : "f"(den));
    rc = fmaf(rc, fmaf(-den, rc, 1.0f), rc);   // one Newton step
    const float t = num * rc;
    if (fabsf(t) <= 0.25f) {
        const float t2 = t * t;
        float q = 1.0f / 11.0f;
        q = fmaf(q, t2, 1.0f / 9.0f);
        q = fmaf(q, t2, 1.0f / 7.0f);
        q = fmaf(q, t2, 1.0f / 5.0f);
        q = fmaf(q, t2, 1.0f / 3.0f);
        q = fmaf(q, t2, 1.0f);
        return t * q;
    }
    return 0.5f * logf(r1 / r0);
}

// Direct FP32 panel terms over the near list (chunked like k_rhs_partial).
VX_DEVK void k_rhs_near_body(VxBlkB<RHS_T, 8> vb, const VxScalars *S, const vx_panel *pan, int P, int P32,
                             const float4 *near, double *part, int sms) {
    const int nchunks = vx_rhs_chunks(S->n0, P, sms);   // from the body's own count
    __shared__ float4 sq4[RHS_T];   // (x, y, G, unused)
    const long long nn = S->bf_nnear;
    const long long cs = vx_ceil_div(vx_ceil_div(nn, nchunks), RHS_T) * RHS_T;
    const int tiles = (P + RHS_T - 1) / RHS_T;
    const long long items = (long long)tiles * nchunks;
    for (long long it = vb.x; it < items; it += vb.n) {
        const int pt = (int)(it % tiles);
        const long long sc = it / tiles;
        const int i = pt * RHS_T + threadIdx.x;
        const bool valid = i < P;
        float al0 = 0, al1 = 0, d0 = 1, d1 = 0;
        if (valid) {
            al0 = (float)pan[i].left[0]; al1 = (float)pan[i].left[1];
            d0 = (float)pan[i].right[0] - al0; d1 = (float)pan[i].right[1] - al1;
        }
        const float kd0 = -d1, kd1 = d0;
        const float dd2 = fmaf(d0, d0, d1 * d1);
        float y0 = 0, y1 = 0;
        const long long j0 = sc * cs, j1 = min(nn, j0 + cs);
        for (long long jt = j0; jt < j1; jt += RHS_T) {
            __syncthreads();
            const long long j = jt + threadIdx.x;
            if (j < j1) sq4[threadIdx.x] = near[j];
            __syncthreads();
            const int cnt = (int)min((long long)RHS_T, j1 - jt);
            for (int q = 0; q < cnt; ++q) {
                const float4 src = sq4[q];
                float s00 = al0 - src.x, s01 = al1 - src.y;
                float s10 = s00 + d0, s11 = s01 + d1;
                float A = fmaf(s00, d0, s01 * d1);
                float B = fmaf(s10, d0, s11 * d1);
                float z = fmaf(d0, s01, -(d1 * s00));
                float alpha = vx_atan2_bulk(-dd2 * z, fmaf(z, z, A * B));
                float r1 = fmaf(s10, s10, s11 * s11), r0 = fmaf(s00, s00, s01 * s01);
                float beta = vx_half_log_ratio(r0, r1, fmaf(2.0f, A, dd2));
                y0 = fmaf(src.z, fmaf(alpha, d0, beta * kd0), y0);
                y1 = fmaf(src.z, fmaf(alpha, d1, beta * kd1), y1);
            }
        }
        if (valid) {
            part[(sc * P32 + i) * 2 + 0] = (double)y0;
            part[(sc * P32 + i) * 2 + 1] = (double)y1;
        }
    }
}
__global__ void __launch_bounds__(RHS_T) k_rhs_near(const VxScalars *S, const vx_panel *pan, int P, int P32,
                                                    const float4 *near, double *part, int sms) {
    VX_PDL_WAIT();
    k_rhs_near_body(VxBlkB<RHS_T, 8>{blockIdx.x, gridDim.x}, S, pan, P, P32, near, part, sms);
}

// R_i = -(mean velocity along panel i + V_inf) . tau_i; the far field (if
// coef) adds Re[I_far (tau_x + i tau_y) / (2 pi i dz)] with dz = zb - za.
// WARP: one warp per panel, its lanes summing the chunk partials (bulk form,
// fixed butterfly); otherwise one thread per panel in chunk order.
template <bool WARP>
VX_DEVK void k_rhs_final_body(VxBlkB<0, 0> vb, const VxScalars *S, const vx_panel *pan, int P, int P32,
                              const double *part, int sms, double *R, const VxParams &p, const double *coef) {
    const int nchunks = vx_rhs_chunks(S->n0, P, sms);   // from the body's own count
    const int i = WARP ? (int)((vb.x * blockDim.x + threadIdx.x) >> 5) : vb.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    double y0 = 0.0, y1 = 0.0;
    if (WARP) {
        const int lane = threadIdx.x & 31;
        for (int sc = lane; sc < nchunks; sc += 32) {
            y0 += part[((long long)sc * P32 + i) * 2 + 0];
            y1 += part[((long long)sc * P32 + i) * 2 + 1];
        }
        for (int o = 16; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
        }
        if (lane != 0) return;
    } else {
        for (int sc = 0; sc < nchunks; ++sc) {
            y0 += part[((long long)sc * P32 + i) * 2 + 0];
            y1 += part[((long long)sc * P32 + i) * 2 + 1];
        }
    }
    double d0 = pan[i].right[0] - pan[i].left[0], d1 = pan[i].right[1] - pan[i].left[1];
    double mnog = 1.0 / (VX_TWO_PI * (d0 * d0 + d1 * d1));
    double u = mnog * y0, w = mnog * y1;
    if (coef) {
        const double ar = pan[i].left[0] - p.bc_x, ai = pan[i].left[1] - p.bc_y;
        const double br = pan[i].right[0] - p.bc_x, bi = pan[i].right[1] - p.bc_y;
        double pa_r = ar, pa_i = ai, pb_r = br, pb_i = bi;   // (z - c)^(l+1)
        double Ir = 0.0, Ii = 0.0;
        for (int l = 0; l < BF_P; ++l) {
            const double dr = (pb_r - pa_r) / (double)(l + 1), di = (pb_i - pa_i) / (double)(l + 1);
            const double cr = coef[2 * l], ci = coef[2 * l + 1];
            Ir += cr * dr - ci * di;
            Ii += cr * di + ci * dr;
            double t = pa_r * ar - pa_i * ai; pa_i = pa_r * ai + pa_i * ar; pa_r = t;
            t = pb_r * br - pb_i * bi; pb_i = pb_r * bi + pb_i * br; pb_r = t;
        }
        // mean conjugate velocity W = I / (2 pi i dz): u = Re W, v = -Im W
        const double qr = -VX_TWO_PI * d1, qi = VX_TWO_PI * d0;   // 2 pi i dz
        const double qq = qr * qr + qi * qi;
        const double Wr = (Ir * qr + Ii * qi) / qq, Wi = (Ii * qr - Ir * qi) / qq;
        u += Wr;
        w += -Wi;
    }
    R[i] = -((u + S->vinf[0]) * pan[i].tang[0] + (w + S->vinf[1]) * pan[i].tang[1]);
}
template <bool WARP>
__global__ void k_rhs_final(const VxScalars *S, const vx_panel *pan, int P, int P32,
                            const double *part, int sms, double *R, VxParams p, const double *coef) {
    VX_PDL_WAIT();
    k_rhs_final_body<WARP>(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, S, pan, P, P32, part, sms, R, p, coef);
}

// One new vortex per panel at [n0, n0+P) (src/kernel.cu:862-872), written
// by the block that finishes the gamma solve last (a vortex takes the gamma
// of its panel's right neighbour too, so every gamma must be final).
__device__ void birth_place(const VxParams &p, const VxView &v, VxScalars *S, const vx_panel *pan, int P,
                            const double *gamma) {
    const long long n0 = S->n0;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int in = (int)pan[i].n_of_rpanel;
        const double mx = (pan[i].left[0] + pan[i].right[0]) / 2;
        const double my = (pan[i].left[1] + pan[i].right[1]) / 2;
        double bx, by;
        if (p.birth_mode == VX_BIRTH_FILE) {
            bx = pan[i].birth[0]; by = pan[i].birth[1];
        } else if (p.birth_mode == VX_BIRTH_HALF_PANEL) {
            const double h = 0.5 * pan[i].length;
            bx = mx + h * pan[i].norm[0]; by = my + h * pan[i].norm[1];
        } else {
            bx = mx + 1e-6 * pan[i].norm[0]; by = my + 1e-6 * pan[i].norm[1];
        }
        const long long k = (n0 + i) * v.ps;
        v.x[k] = bx;
        v.y[k] = by;
        v.g[k] = 0.5 * (__ldcg(&gamma[i]) * pan[i].length + __ldcg(&gamma[in]) * pan[in].length);
    }
    if (threadIdx.x == 0) S->n = n0 + P;
}

// gamma_i = sum_j M_ij R_j + M_iP dg, sequential in j with fma (as the
// oracle), one thread per row; ld is the matrix row stride.  Then the
// vortices are placed (birth_place).
VX_DEVK void k_gamma_body(VxBlkB<0, 0> vb, const VxParams &p, const VxView &v, VxScalars *S, const vx_panel *pan, const double *M,
                          long long ld, int P, const double *R, double *gamma) {
    const int i = vb.x * blockDim.x + threadIdx.x;
    if (i < P) {
        const double *row = M + (long long)i * ld;
        double acc = 0.0;
        for (int j = 0; j < P; ++j) acc = fma(row[j], R[j], acc);
        gamma[i] = fma(row[P], S->dg, acc);
    }
    if (vx_last_block(&S->sync_ctr, vb.n)) birth_place(p, v, S, pan, P, gamma);
}
__global__ void k_gamma(VxParams p, VxView v, VxScalars *S, const vx_panel *pan, const double *M, long long ld, int P,
                        const double *R, double *gamma) {
    VX_PDL_WAIT();
    k_gamma_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, p, v, S, pan, M, ld, P, R, gamma);
}

// The same sums from the transposed inverse Mt (Mt[j ld + i] = M[i ld + j]):
// the same order and fma per row, but a warp's 32 rows read 32 consecutive
// doubles per step instead of 32 rows' worth of cache lines.
VX_DEVK void k_gamma_t_body(VxBlkB<0, 0> vb, const VxParams &p, const VxView &v, VxScalars *S, const vx_panel *pan,
                            const double *Mt, long long ld, int P, const double *R, double *gamma) {
    const int i = vb.x * blockDim.x + threadIdx.x;
    if (i < P) {
        double acc = 0.0;
        for (int j = 0; j < P; ++j) acc = fma(Mt[(long long)j * ld + i], R[j], acc);
        gamma[i] = fma(Mt[(long long)P * ld + i], S->dg, acc);
    }
    if (vx_last_block(&S->sync_ctr, vb.n)) birth_place(p, v, S, pan, P, gamma);
}
__global__ void k_gamma_t(VxParams p, VxView v, VxScalars *S, const vx_panel *pan, const double *Mt, long long ld,
                          int P, const double *R, double *gamma) {
    VX_PDL_WAIT();
    k_gamma_t_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, p, v, S, pan, Mt, ld, P, R, gamma);
}

// Bulk form: one warp per row, lanes striding the row (coalesced), FP64
// partial sums combined by a fixed butterfly.
VX_DEVK void k_gamma_w_body(VxBlkB<0, 0> vb, const VxParams &p, const VxView &v, VxScalars *S, const vx_panel *pan,
                            const double *M, long long ld, int P, const double *R, double *gamma) {
    const int lane = threadIdx.x & 31;
    const int i = (vb.x * blockDim.x + threadIdx.x) >> 5;
    if (i < P) {
        const double *row = M + (long long)i * ld;
        double acc = 0.0;
        for (int j = lane; j < P; j += 32) acc = fma(row[j], R[j], acc);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) gamma[i] = fma(row[P], S->dg, acc);
    }
    if (vx_last_block(&S->sync_ctr, vb.n)) birth_place(p, v, S, pan, P, gamma);
}
__global__ void k_gamma_w(VxParams p, VxView v, VxScalars *S, const vx_panel *pan, const double *M, long long ld,
                          int P, const double *R, double *gamma) {
    VX_PDL_WAIT();
    k_gamma_w_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, p, v, S, pan, M, ld, P, R, gamma);
}

VX_DEVK void k_transpose_body(VxBlkB<0, 0> vb, const double *A, double *At, long long nr) {
    __shared__ double t[32][33];
    for (long long by = blockIdx.y; by * 32 < nr; by += gridDim.y)
        for (long long bx = vb.x; bx * 32 < nr; bx += vb.n) {
            for (int r = threadIdx.y; r < 32; r += blockDim.y) {
                const long long i = by * 32 + r, j = bx * 32 + threadIdx.x;
                if (i < nr && j < nr) t[r][threadIdx.x] = A[i * nr + j];
            }
            __syncthreads();
            for (int r = threadIdx.y; r < 32; r += blockDim.y) {
                const long long i = bx * 32 + r, j = by * 32 + threadIdx.x;
                if (i < nr && j < nr) At[i * nr + j] = t[threadIdx.x][r];
            }
            __syncthreads();
        }
}
__global__ void k_transpose(const double *A, double *At, long long nr) {
    VX_PDL_WAIT();
    k_transpose_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, A, At, nr);
}

cudaError_t vx_transpose_square(const VxLaunch &L, const double *A, double *At, long long nr) {
    const long long nb = vx_ceil_div(nr, 32LL);
    const dim3 grid((unsigned)std::min(nb, 64LL), (unsigned)std::min(nb, 64LL)), block(32, 8);
    vx_launch<k_transpose, k_transpose_body>(L, grid, block, 0, A, At, nr);
    return cudaGetLastError();
}

// rhs_chunks: the source chunks the host expects, for the grid only (the
// kernels take the chunk count from the body's own count, vx_rhs_chunks).
static cudaError_t birth_impl(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S, VxWork &w,
                              const vx_panel *pan, const double *minv, long long ld, const double *minv_t,
                              int rhs_chunks) {
    const int P = p.P, P32 = (int)vx_round32(P);
    const int tiles = (P + RHS_T - 1) / RHS_T;
    const int grid = (int)min((long long)tiles * rhs_chunks, (long long)L.num_sms * 16);
    const int sms = vx_full_sms(L);   // the device's SMs: partitions follow the body, not the launch
    const bool far = p.prec == VX_PREC_FP32 && p.birth_far;
    if (far) {
        const int gb = std::min(VX_BF_MAX_BLOCKS, 2 * L.num_sms);
        vx_launch<k_bf_far, k_bf_far_body>(L, gb, BF_T, 0, p, v, S, w.bf_part, w.bf_cnt, sms, w.bf_off, w.bf_coef);
        vx_launch<k_bf_scatter, k_bf_scatter_body>(L, gb, BF_T, 0, p, v, S, w.bf_off, w.bf_near, sms);
        vx_launch<k_rhs_near, k_rhs_near_body>(L, grid, RHS_T, 0, S, pan, P, P32, w.bf_near, w.rhs_part, sms);
    } else if (p.prec == VX_PREC_FP32) {
        vx_launch<k_rhs_partial<float>, k_rhs_partial_body<float>>(L, grid, RHS_T, 0, v, S, pan, P, P32, w.rhs_part, sms);
    } else {
        vx_launch<k_rhs_partial<double>, k_rhs_partial_body<double>>(L, grid, RHS_T, 0, v, S, pan, P, P32, w.rhs_part, sms);
    }

    const int b = (P + 127) / 128;
    if (far)
        vx_launch<k_rhs_final<true>, k_rhs_final_body<true>>(L, (P + 3) / 4, 128, 0, S, pan, P, P32, w.rhs_part, sms, w.R, p, w.bf_coef);
    else
        vx_launch<k_rhs_final<false>, k_rhs_final_body<false>>(L, b, 128, 0, S, pan, P, P32, w.rhs_part, sms, w.R, p, nullptr);

    if (minv_t && p.prec == VX_PREC_FP32)
        vx_launch<k_gamma_w, k_gamma_w_body>(L, (P + 3) / 4, 128, 0, p, v, S, pan, minv, ld, P, w.R, w.gamma);
    else if (minv_t)
        vx_launch<k_gamma_t, k_gamma_t_body>(L, b, 128, 0, p, v, S, pan, minv_t, ld, P, w.R, w.gamma);
    else
        vx_launch<k_gamma, k_gamma_body>(L, b, 128, 0, p, v, S, pan, minv, ld, P, w.R, w.gamma);
    return cudaGetLastError();
}

// Row-major inverse with row stride ld (the reference's padded matrix).
cudaError_t vx_launch_birth_ld(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                               VxWork &w, const vx_panel *pan, const double *minv, long long ld,
                               int rhs_chunks) {
    return birth_impl(L, p, v, S, w, pan, minv, ld, nullptr, rhs_chunks);
}

// Native engine: the inverse and its transpose, unpadded, stride P+1.  The
// plain form solves in the reference's row order from the transpose; the
// bulk form a warp per row.
cudaError_t vx_launch_birth(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                            VxWork &w, const vx_panel *pan, const double *minv, const double *minv_t,
                            int rhs_chunks) {
    return birth_impl(L, p, v, S, w, pan, minv, (long long)p.P + 1, minv_t, rhs_chunks);
}

cudaError_t vx_launch_step_end(const VxLaunch &L, VxScalars *S) {
    vx_launch<k_step_end, k_step_end_body>(L, 1, 1, 0, S);
    return cudaGetLastError();
}
