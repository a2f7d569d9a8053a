// vx_wall.cu — diffusive velocity induced by the wall.
//
// Reference: diffusion_2_Kernel src/kernel.cu:1031-1088 with the panel
// integral I_0_I_3 (FP64 twin src/kernel.cu:1300-1322, FP32 1324-1346).
// A panel contributes only when the particle is within 5 L of the panel's
// birth point, so particles outside the birth-point bounding box grown by
// 5 L_max skip the panel loop: their contribution is exactly +0.  Inside
// that box, when panel lists are given, a particle tests only the panels of
// its wall cell: every panel whose birth point lies within one cell (side
// > 5 L_max) of the cell, in ascending panel order.  A panel left out is
// farther than 5 L from the particle, so it would add nothing; the panels
// kept are visited in the reference's order, so the sums and the first
// r <= 0.1 L override are unchanged bit for bit.  The FP32 (bulk) form
// evaluates the integral with reciprocals and MUFU rsqrt / ex2
// (vx_wall_integral_bulk); the FP64 form follows the reference's expression
// order.
#include "vx_internal.cuh"

template <typename T>
__device__ __forceinline__ T vx_exp(T x);
template <> __device__ __forceinline__ double vx_exp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float vx_exp<float>(float x) { return expf(x); }
template <typename T>
__device__ __forceinline__ T vx_sqrt(T x);
template <> __device__ __forceinline__ double vx_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float vx_sqrt<float>(float x) { return sqrtf(x); }

// n_of_points-point midpoint rule along the panel (same expression order as
// the oracle's wall_integral).
template <typename T>
__device__ void vx_wall_integral(T Ra0, T Ra1, T Rb0, T Rb1, T N0, T N1, T Rj0, T Rj1, T dL, T d,
                                 int N, T &R0, T &R30, T &R31) {
    T dR0 = (Rb0 - Ra0) / (T)N, dR1 = (Rb1 - Ra1) / (T)N;
    T delt = dL / (T)N;
    T s0 = 0, s30 = 0, s31 = 0;
    for (int k = 0; k < N; ++k) {
        T Rk0 = (Ra0 + (T)k * dR0 + Ra0 + (T)(k + 1) * dR0) / 2;
        T Rk1 = (Ra1 + (T)k * dR1 + Ra1 + (T)(k + 1) * dR1) / 2;
        T E0 = (Rj0 - Rk0) / d, E1 = (Rj1 - Rk1) / d;
        T e2 = fma(E0, E0, E1 * E1);
        T me = vx_sqrt<T>(e2);
        T ex = vx_exp<T>(-me);
        s0 += (E0 * N0 + E1 * N1) / e2 * (me + 1) * ex * delt;
        s30 += N0 * ex * delt;
        s31 += N1 * ex * delt;
    }
    R0 = s0; R30 = s30; R31 = s31;
}

// The bulk form's integral (FP32): the same midpoint rule with the
// divisions by d and |E|^2 taken as products with reciprocals, |E| and
// 1/|E| from one rsqrt, and e^-|E| as 2^(-|E| log2 e), all on the MUFU pipe.
__device__ __forceinline__ void vx_wall_integral_bulk(float Ra0, float Ra1, float Rb0, float Rb1, float N0,
                                                      float N1, float Rj0, float Rj1, float dL, float inv_d,
                                                      int N, float &R0, float &R30, float &R31) {
    const float invN = 1.0f / (float)N;
    const float dR0 = (Rb0 - Ra0) * invN, dR1 = (Rb1 - Ra1) * invN;
    const float delt = dL * invN;
    float s0 = 0, s30 = 0, s31 = 0;
    for (int k = 0; k < N; ++k) {
        const float h = (float)k + 0.5f;
        const float E0 = (Rj0 - fmaf(h, dR0, Ra0)) * inv_d, E1 = (Rj1 - fmaf(h, dR1, Ra1)) * inv_d;
        const float e2 = fmaf(E0, E0, E1 * E1);
        float rs, ex;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(rs) : "f"(e2));
        const float me = e2 * rs;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(ex) : "f"(-1.4426950408889634f * me));
        s0 = fmaf(fmaf(E0, N0, E1 * N1) * (rs * rs) * (me + 1.0f), ex, s0);
        s30 = fmaf(N0, ex, s30);
        s31 = fmaf(N1, ex, s31);
    }
    R0 = s0 * delt; R30 = s30 * delt; R31 = s31 * delt;
}

template <typename T>
VX_DEVK void k_wall_body(VxBlkB<128, sizeof(T) == 4 ? 8 : 0> vb, const VxParams &p, const VxView &v, const VxScalars *S, const vx_panel *pan, const int *wstart,
                         const int *widx) {
    const long long n = S->n;
    const T nu = (T)p.nu;
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        const double xd = v.x[i * v.ps], yd = v.y[i * v.ps];
        if (xd < p.wall_x0 || xd > p.wall_x1 || yd < p.wall_y0 || yd > p.wall_y1) continue;
        int q0 = 0, q1 = p.P;
        if (wstart) {
            const int cx = min(max((int)floor((xd - p.wall_x0) / p.wall_h), 0), p.wall_nx - 1);
            const int cy = min(max((int)floor((yd - p.wall_y0) / p.wall_h), 0), p.wall_ny - 1);
            q0 = wstart[cy * p.wall_nx + cx];
            q1 = wstart[cy * p.wall_nx + cx + 1];
        }
        const T a0 = (T)xd, a1 = (T)yd, dd = (T)v.d[i];
        T I0 = (T)VX_TWO_PI * dd * dd, I30 = 0, I31 = 0;
        for (int q = q0; q < q1; ++q) {
            const vx_panel &pf = pan[wstart ? widx[q] : q];
            const T dL = (T)pf.length;
            T dx = a0 - (T)pf.birth[0], dy = a1 - (T)pf.birth[1];
            T r = vx_sqrt<T>(fma(dx, dx, dy * dy));
            if (r < 5 * dL && r > (T)0.1 * dL) {
                T R0, R30, R31;
                if constexpr (sizeof(T) == 4)
                    vx_wall_integral_bulk((T)pf.left[0], (T)pf.left[1], (T)pf.right[0], (T)pf.right[1],
                                          -(T)pf.norm[0], -(T)pf.norm[1], a0, a1, dL, 1.0f / dd, p.n_of_points,
                                          R0, R30, R31);
                else
                    vx_wall_integral<T>((T)pf.left[0], (T)pf.left[1], (T)pf.right[0], (T)pf.right[1],
                                        -(T)pf.norm[0], -(T)pf.norm[1], a0, a1, dL, dd, p.n_of_points,
                                        R0, R30, R31);
                I0 += (-dd) * R0;
                I30 -= R30;
                I31 -= R31;
            } else if (r <= (T)0.1 * dL) {
                T ex = 1 - vx_exp<T>(-dL / (2 * dd));
                I0 = (T)VX_PI * dd * dd;
                I30 = 2 * (T)pf.norm[0] * dd * ex;
                I31 = 2 * (T)pf.norm[1] * dd * ex;
                break;
            }
        }
        v.vx[i * v.vs] += (double)(nu * I30 / I0);
        v.vy[i * v.vs] += (double)(nu * I31 / I0);
    }
}
template <typename T>
__global__ void k_wall(VxParams p, VxView v, const VxScalars *S, const vx_panel *pan, const int *wstart,
                       const int *widx) {
    VX_PDL_WAIT();
    k_wall_body<T>(VxBlkB<128, sizeof(T) == 4 ? 8 : 0>{blockIdx.x, gridDim.x}, p, v, S, pan, wstart, widx);
}

cudaError_t vx_launch_wall(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                           const vx_panel *pan, const int *wstart, const int *widx) {
    if (p.wall_nx <= 0 || p.wall_ny <= 0) wstart = widx = nullptr;
    if (p.prec == VX_PREC_FP32)
        vx_launch<k_wall<float>, k_wall_body<float>>(L, L.num_sms * 8, 128, 0, p, v, S, pan, wstart, widx);
    else
        vx_launch<k_wall<double>, k_wall_body<double>>(L, L.num_sms * 8, 128, 0, p, v, S, pan, wstart, widx);

    return cudaGetLastError();
}
