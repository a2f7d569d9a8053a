// vx_pairs.cu — direct pair sums: convective (Biot-Savart) velocity with the
// mean distance to the 3 nearest particles, vortex-vortex diffusive velocity,
// and the probe velocity.
//
// Reference: shared_Kernel src/kernel.cu:875-983, diffusion_Kernel
// src/kernel.cu:985-1029, velocity_control_Kernel src/kernel.cu:1434-1475.
//
// Work decomposition: a target tile (TPT targets per thread, 256 threads) x a
// source chunk is one work item; persistent CTAs walk the items.  Sources are
// staged through shared memory 256 at a time and read as warp-wide broadcasts.
// Each item writes partial sums; a combine kernel adds the chunks in a fixed
// order, so results are deterministic for a given split.
//
// Precision: FP64 (plain form) computes every pair in double.  FP32 (bulk
// form) computes pairs in float and accumulates each 256-source tile in
// float, adding tile sums into a double accumulator (blocked compensation).
#include "vx_internal.cuh"

constexpr int PT = 256;       // threads per block = sources per shared tile

__host__ __device__ constexpr int pairs_tpt(bool fp32) { return fp32 ? 4 : 2; }

// Source split of the pair kernels: K source chunks; the partial sums of
// target i and chunk sc sit at part[(sc nout + q) tstride + i], tstride =
// cap / (nout K).  K > 0: the caller's split (probe points); K == 0: from the
// body's own count on the device (vx_ksplit of it rounded up to a power of
// two), so a step's sums never depend on the host's running bound.
struct VxSplit {
    long long cap;
    int K, sms, tile, nout;
};
__device__ __forceinline__ void vx_split_of(const VxScalars *S, const VxSplit &sp, int &K, long long &tstride) {
    K = sp.K > 0 ? sp.K : vx_ksplit(vx_pow2_ceil(S->n), sp.tile, sp.sms);
    tstride = sp.cap / ((long long)sp.nout * K);
}


// ---------------------------------------------------------------------------
// Packed FP32 sources for the bulk form: (x, y, G, 0), G masked to 0 beyond n.
VX_DEVK void k_pack32_body(VxBlkB<0, 0> vb, const VxView &v, const VxScalars *S, float4 *src, long long upto) {
    const long long n = S->n;
    const long long s = vx_round32(n);
    for (long long j = vb.x * (long long)blockDim.x + threadIdx.x; j < s;
         j += (long long)vb.n * blockDim.x) {
        if (j >= upto) break;
        src[j] = make_float4((float)v.x[j * v.ps], (float)v.y[j * v.ps],
                             j < n ? (float)v.g[j * v.ps] : 0.0f, 0.0f);
    }
}
__global__ void k_pack32(VxView v, const VxScalars *S, float4 *src, long long upto) {
    VX_PDL_WAIT();
    k_pack32_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, src, upto);
}

template <typename T> struct PairMath;
template <> struct PairMath<double> {
    static __device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
};
template <> struct PairMath<float> {
    static __device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
};

// Sources of one shared tile.
template <typename T>
struct SrcTile {
    T x[PT], y[PT], g[PT];
};

template <typename T>
__device__ __forceinline__ void load_src(SrcTile<T> &t, const VxView &v, const float4 *src32,
                                         long long j, long long jend, long long nvel) {
    if (j < jend) {
        if (src32) {
            float4 q = src32[j];
            t.x[threadIdx.x] = (T)q.x; t.y[threadIdx.x] = (T)q.y; t.g[threadIdx.x] = (T)q.z;
        } else {
            t.x[threadIdx.x] = (T)v.x[j * v.ps];
            t.y[threadIdx.x] = (T)v.y[j * v.ps];
            t.g[threadIdx.x] = j < nvel ? (T)v.g[j * v.ps] : (T)0;
        }
    }
}

// ---------------------------------------------------------------------------
// Biot-Savart (+ 3 nearest when NN3).  Targets: particles (nt < 0 -> n) or
// probe points (tx/ty with stride tstr).  Partials: [sc][5][tstride].
template <typename T, bool NN3>
VX_DEVK void k_bs_partial_body(VxBlkB<PT, 0> vb, const VxParams &p, const VxView &v, const VxScalars *S,
                               const float4 *src32, const double *tx,
                               const double *ty, long long tstr, long long nt_in,
                               double *part, VxSplit sp) {
    int K;
    long long tstride;
    vx_split_of(S, sp, K, tstride);
    constexpr int TPT = pairs_tpt(sizeof(T) == 4);
    constexpr int NOUT = NN3 ? 5 : 2;
    __shared__ SrcTile<T> st;
    const long long n = S->n;
    const long long nt = nt_in < 0 ? n : nt_in;
    const long long srange = NN3 ? vx_round32(n) : n;
    const long long tile = (long long)PT * TPT;
    const long long tiles = vx_ceil_div(nt, tile);
    const long long cs = vx_ceil_div(vx_ceil_div(srange, K), PT) * PT;
    const long long items = tiles * K;
    const T eps2 = (T)p.eps2;
    for (long long it = vb.x; it < items; it += vb.n) {
        const long long tt = it % tiles, sc = it / tiles;
        T ax[TPT], ay[TPT];
        long long ti[TPT];
        double vxa[TPT], vya[TPT];
        T d1[TPT], d2[TPT], d3[TPT];
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
            ti[k] = tt * tile + (long long)k * PT + threadIdx.x;
            long long i = ti[k] < nt ? ti[k] : 0;
            ax[k] = (T)tx[i * tstr];
            ay[k] = (T)ty[i * tstr];
            vxa[k] = 0.0; vya[k] = 0.0;
            d1[k] = d2[k] = d3[k] = (T)1e5;
        }
        const long long j0 = sc * cs, j1 = min(srange, j0 + cs);
        for (long long jt = j0; jt < j1; jt += PT) {
            __syncthreads();
            load_src<T>(st, v, src32, jt + threadIdx.x, j1, n);
            __syncthreads();
            const int cnt = (int)min((long long)PT, j1 - jt);
            T sx[TPT], sy[TPT];
#pragma unroll
            for (int k = 0; k < TPT; ++k) { sx[k] = 0; sy[k] = 0; }
            for (int q = 0; q < cnt; ++q) {
                const T bx = st.x[q], by = st.y[q], bg = st.g[q];
                const long long j = jt + q;
#pragma unroll
                for (int k = 0; k < TPT; ++k) {
                    T dx = ax[k] - bx, dy = ay[k] - by;
                    T r2 = fma(dx, dx, dy * dy);
                    if (NN3) {
                        T r2n = (j == ti[k]) ? (T)INFINITY : r2;
                        vx_nn3_insert<T>(d1[k], d2[k], d3[k], r2n);
                    }
                    T m = bg * PairMath<T>::rcp(fmax(r2, eps2));
                    sy[k] = fma(m, dx, sy[k]);
                    sx[k] = fma(-m, dy, sx[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < TPT; ++k) { vxa[k] += (double)sx[k]; vya[k] += (double)sy[k]; }
        }
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
            if (ti[k] < nt) {
                double *o = part + (long long)sc * NOUT * tstride + ti[k];
                o[0] = vxa[k];
                o[tstride] = vya[k];
                if (NN3) {
                    o[2 * tstride] = (double)d1[k];
                    o[3 * tstride] = (double)d2[k];
                    o[4 * tstride] = (double)d3[k];
                }
            }
        }
    }
}
template <typename T, bool NN3>
__global__ void __launch_bounds__(PT) k_bs_partial(VxParams p, VxView v, const VxScalars *S,
                                                   const float4 *src32, const double *tx,
                                                   const double *ty, long long tstr, long long nt_in,
                                                   double *part, VxSplit sp) {
    VX_PDL_WAIT();
    k_bs_partial_body<T, NN3>(VxBlkB<PT, 0>{blockIdx.x, gridDim.x}, p, v, S, src32, tx, ty, tstr, nt_in, part, sp);
}

// ---------------------------------------------------------------------------
// Bulk-form Biot-Savart + 3 nearest, FP32.  Same decomposition as above, with
// the inner loop cut to the arithmetic: sources come from shared memory as
// one float4 broadcast each, the loop runs unrolled over full tiles, the
// reciprocal is the hardware approximation (rcp.approx, 1 ulp), and the
// self pair is excluded only in the one tile per target that can contain it
// (a uniform branch per tile), so the hot loop has no index compare.
__device__ __forceinline__ float vx_rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

constexpr int BS32_TPT = 4;

template <bool NN3, bool CHECK_SELF>
__device__ __forceinline__ void bs32_tile(const float4 *sm, int cnt, int jbase, const int *ti,
                                          const float *ax, const float *ay, float eps2, float *sx,
                                          float *sy, float *d1, float *d2, float *d3) {
#pragma unroll 4
    for (int q = 0; q < cnt; ++q) {
        const float4 s = sm[q];
#pragma unroll
        for (int k = 0; k < BS32_TPT; ++k) {
            const float dx = ax[k] - s.x, dy = ay[k] - s.y;
            const float r2 = fmaf(dx, dx, dy * dy);
            if (NN3) {
                if (r2 < d3[k] && (!CHECK_SELF || jbase + q != ti[k])) {
                    d3[k] = r2;
                    float t = fminf(d3[k], d2[k]); d3[k] = fmaxf(d3[k], d2[k]); d2[k] = t;
                    t = fminf(d1[k], d2[k]); d2[k] = fmaxf(d1[k], d2[k]); d1[k] = t;
                }
            }
            const float m = s.z * vx_rcp_approx(fmaxf(r2, eps2));
            sy[k] = fmaf(m, dx, sy[k]);
            sx[k] = fmaf(-m, dy, sx[k]);
        }
    }
}

template <bool NN3>
VX_DEVK void k_bs32_partial_body(VxBlkB<PT, 0> vb, const VxParams &p, const VxScalars *S, const float4 *src32,
                                 const double *tx, const double *ty, long long tstr,
                                 long long nt_in, double *part, VxSplit sp) {
    int K;
    long long tstride;
    vx_split_of(S, sp, K, tstride);
    constexpr int NOUT = NN3 ? 5 : 2;
    __shared__ float4 sm[PT];
    const long long n = S->n;
    const long long nt = nt_in < 0 ? n : nt_in;
    const long long srange = NN3 ? vx_round32(n) : n;
    const long long tile = (long long)PT * BS32_TPT;
    const long long tiles = vx_ceil_div(nt, tile);
    const long long cs = vx_ceil_div(vx_ceil_div(srange, K), PT) * PT;
    const long long items = tiles * K;
    const float eps2 = (float)p.eps2;
    for (long long it = vb.x; it < items; it += vb.n) {
        const long long tt = it % tiles, sc = it / tiles;
        const long long tlo = tt * tile, thi = min(nt, tlo + tile);
        float ax[BS32_TPT], ay[BS32_TPT], d1[BS32_TPT], d2[BS32_TPT], d3[BS32_TPT];
        int ti[BS32_TPT];
        double vxa[BS32_TPT], vya[BS32_TPT];
#pragma unroll
        for (int k = 0; k < BS32_TPT; ++k) {
            const long long t = tlo + (long long)k * PT + threadIdx.x;
            ti[k] = (int)t;
            const long long i = t < nt ? t : 0;
            ax[k] = (float)tx[i * tstr];
            ay[k] = (float)ty[i * tstr];
            vxa[k] = 0.0; vya[k] = 0.0;
            d1[k] = d2[k] = d3[k] = 1e5f;
        }
        const long long j0 = sc * cs, j1 = min(srange, j0 + cs);
        for (long long jt = j0; jt < j1; jt += PT) {
            __syncthreads();
            if (jt + threadIdx.x < j1) {
                float4 q = src32[jt + threadIdx.x];
                if (!NN3 && jt + threadIdx.x >= n) q.z = 0.0f;
                sm[threadIdx.x] = q;
            }
            __syncthreads();
            const int cnt = (int)min((long long)PT, j1 - jt);
            float sx[BS32_TPT], sy[BS32_TPT];
#pragma unroll
            for (int k = 0; k < BS32_TPT; ++k) { sx[k] = 0.0f; sy[k] = 0.0f; }
            const bool self = NN3 && jt < thi && jt + cnt > tlo;   // uniform per block
            if (self)
                bs32_tile<NN3, true>(sm, cnt, (int)jt, ti, ax, ay, eps2, sx, sy, d1, d2, d3);
            else
                bs32_tile<NN3, false>(sm, cnt, (int)jt, ti, ax, ay, eps2, sx, sy, d1, d2, d3);
#pragma unroll
            for (int k = 0; k < BS32_TPT; ++k) { vxa[k] += (double)sx[k]; vya[k] += (double)sy[k]; }
        }
#pragma unroll
        for (int k = 0; k < BS32_TPT; ++k) {
            if (ti[k] < nt) {
                double *o = part + (long long)sc * NOUT * tstride + ti[k];
                o[0] = vxa[k];
                o[tstride] = vya[k];
                if (NN3) {
                    o[2 * tstride] = (double)d1[k];
                    o[3 * tstride] = (double)d2[k];
                    o[4 * tstride] = (double)d3[k];
                }
            }
        }
    }
}
template <bool NN3>
__global__ void __launch_bounds__(PT) k_bs32_partial(VxParams p, const VxScalars *S, const float4 *src32,
                                                     const double *tx, const double *ty, long long tstr,
                                                     long long nt_in, double *part, VxSplit sp) {
    VX_PDL_WAIT();
    k_bs32_partial_body<NN3>(VxBlkB<PT, 0>{blockIdx.x, gridDim.x}, p, S, src32, tx, ty, tstr, nt_in, part, sp);
}

// Combine: V = sum/(2 pi) + V_inf, d = mean of the 3 nearest distances.
template <bool FP32>
VX_DEVK void k_bs_combine_body(VxBlkB<0, 0> vb, const VxView &v, const VxScalars *S, const double *part, VxSplit sp) {
    int K;
    long long tstride;
    vx_split_of(S, sp, K, tstride);
    const long long n = S->n;
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        double sx = 0.0, sy = 0.0;
        double d1 = 1e5, d2 = 1e5, d3 = 1e5;
        for (int sc = 0; sc < K; ++sc) {
            const double *o = part + (long long)sc * 5 * tstride + i;
            sx += o[0];
            sy += o[tstride];
            vx_nn3_insert<double>(d1, d2, d3, o[2 * tstride]);
            vx_nn3_insert<double>(d1, d2, d3, o[3 * tstride]);
            vx_nn3_insert<double>(d1, d2, d3, o[4 * tstride]);
        }
        if (FP32)
            v.d[i] = (double)((sqrtf((float)d1) + sqrtf((float)d2) + sqrtf((float)d3)) / 3);
        else
            v.d[i] = (sqrt(d1) + sqrt(d2) + sqrt(d3)) / 3;
        v.vx[i * v.vs] = sx / VX_TWO_PI + S->vinf[0];
        v.vy[i * v.vs] = sy / VX_TWO_PI + S->vinf[1];
    }
}
template <bool FP32>
__global__ void k_bs_combine(VxView v, const VxScalars *S, const double *part, VxSplit sp) {
    VX_PDL_WAIT();
    k_bs_combine_body<FP32>(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, part, sp);
}

VX_DEVK void k_probe_combine_body(VxBlkB<0, 0> vb, const VxScalars *S, const double *part, VxSplit sp,
                                  long long np, double *ovx, double *ovy, long long ostride) {
    int K;
    long long tstride;
    vx_split_of(S, sp, K, tstride);
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < np;
         i += (long long)vb.n * blockDim.x) {
        double sx = 0.0, sy = 0.0;
        for (int sc = 0; sc < K; ++sc) {
            const double *o = part + (long long)sc * 2 * tstride + i;
            sx += o[0];
            sy += o[tstride];
        }
        ovx[i * ostride] = sx / VX_TWO_PI + S->vinf[0];
        ovy[i * ostride] = sy / VX_TWO_PI + S->vinf[1];
    }
}
__global__ void k_probe_combine(const VxScalars *S, const double *part, VxSplit sp,
                                long long np, double *ovx, double *ovy, long long ostride) {
    VX_PDL_WAIT();
    k_probe_combine_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, S, part, sp, np, ovx, ovy, ostride);
}

// ---------------------------------------------------------------------------
// Vortex-vortex diffusion (src/kernel.cu:985-1029).  Partials [sc][3][tstride].
template <typename T>
struct DiffMath;
template <> struct DiffMath<double> {
    // dist = sqrt(r2); 1/dist; exp(-dist/dd)
    static __device__ __forceinline__ void eval(double r2, double ndd, double &dist, double &rd,
                                                double &e) {
        dist = sqrt(r2);
        rd = __drcp_rn(dist);
        e = exp(dist * ndd);
    }
};
template <> struct DiffMath<float> {
    static __device__ __forceinline__ void eval(float r2, float ndd, float &dist, float &rd,
                                                float &e) {
        rd = rsqrtf(r2);
        dist = r2 * rd;
        e = __expf(dist * ndd);
    }
};

template <typename T>
VX_DEVK void k_diff_partial_body(VxBlkB<PT, 0> vb, const VxParams &p, const VxView &v, const VxScalars *S,
                                 const float4 *src32, double *part,
                                 VxSplit sp) {
    int K;
    long long tstride;
    vx_split_of(S, sp, K, tstride);
    constexpr int TPT = pairs_tpt(sizeof(T) == 4);
    __shared__ SrcTile<T> st;
    const long long n = S->n;
    const long long tile = (long long)PT * TPT;
    const long long tiles = vx_ceil_div(n, tile);
    const long long cs = vx_ceil_div(vx_ceil_div(n, K), PT) * PT;
    const long long items = tiles * K;
    const T thr = (T)(0.001 * p.eps);
    const T thr2 = thr * thr;
    for (long long it = vb.x; it < items; it += vb.n) {
        const long long tt = it % tiles, sc = it / tiles;
        T ax[TPT], ay[TPT], ndd[TPT];
        long long ti[TPT];
        double a2x[TPT], a2y[TPT], a1[TPT];
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
            ti[k] = tt * tile + (long long)k * PT + threadIdx.x;
            long long i = ti[k] < n ? ti[k] : 0;
            ax[k] = (T)v.x[i * v.ps];
            ay[k] = (T)v.y[i * v.ps];
            ndd[k] = -(T)1 / (T)v.d[i];
            a2x[k] = a2y[k] = a1[k] = 0.0;
        }
        const long long j0 = sc * cs, j1 = min(n, j0 + cs);
        for (long long jt = j0; jt < j1; jt += PT) {
            __syncthreads();
            load_src<T>(st, v, src32, jt + threadIdx.x, j1, n);
            __syncthreads();
            const int cnt = (int)min((long long)PT, j1 - jt);
            T s2x[TPT], s2y[TPT], s1[TPT];
#pragma unroll
            for (int k = 0; k < TPT; ++k) { s2x[k] = 0; s2y[k] = 0; s1[k] = 0; }
            for (int q = 0; q < cnt; ++q) {
                const T bx = st.x[q], by = st.y[q], bg = st.g[q];
#pragma unroll
                for (int k = 0; k < TPT; ++k) {
                    T dx = ax[k] - bx, dy = ay[k] - by;
                    T r2 = fma(dx, dx, dy * dy);
                    T dist, rd, e;
                    DiffMath<T>::eval(r2, ndd[k], dist, rd, e);
                    bool use = sizeof(T) == 8 ? (dist > thr) : (r2 > thr2);
                    T ge = use ? bg * e : (T)0;
                    T me = use ? ge * rd : (T)0;   // r = 0 would give 0 * inf
                    s2x[k] = fma(-me, dx, s2x[k]);
                    s2y[k] = fma(-me, dy, s2y[k]);
                    s1[k] += ge;
                }
            }
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
                a2x[k] += (double)s2x[k]; a2y[k] += (double)s2y[k]; a1[k] += (double)s1[k];
            }
        }
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
            if (ti[k] < n) {
                double *o = part + (long long)sc * 3 * tstride + ti[k];
                o[0] = a2x[k];
                o[tstride] = a2y[k];
                o[2 * tstride] = a1[k];
            }
        }
    }
}
template <typename T>
__global__ void __launch_bounds__(PT) k_diff_partial(VxParams p, VxView v, const VxScalars *S,
                                                     const float4 *src32, double *part,
                                                     VxSplit sp) {
    VX_PDL_WAIT();
    k_diff_partial_body<T>(VxBlkB<PT, 0>{blockIdx.x, gridDim.x}, p, v, S, src32, part, sp);
}

VX_DEVK void k_diff_combine_body(VxBlkB<0, 0> vb, const VxParams &p, const VxView &v, const VxScalars *S, const double *part,
                                 VxSplit sp) {
    int K;
    long long tstride;
    vx_split_of(S, sp, K, tstride);
    const long long n = S->n;
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        double I2x = 0.0, I2y = 0.0, I1 = 0.0;
        for (int sc = 0; sc < K; ++sc) {
            const double *o = part + (long long)sc * 3 * tstride + i;
            I2x += o[0];
            I2y += o[tstride];
            I1 += o[2 * tstride];
        }
        if (fabs(I1) > 1e-5) {
            const double dd = v.d[i];
            v.vx[i * v.vs] += -p.nu * I2x / (I1 * dd);
            v.vy[i * v.vs] += -p.nu * I2y / (I1 * dd);
        }
    }
}
__global__ void k_diff_combine(VxParams p, VxView v, const VxScalars *S, const double *part,
                               VxSplit sp) {
    VX_PDL_WAIT();
    k_diff_combine_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, p, v, S, part, sp);
}

// ---------------------------------------------------------------------------
static int pair_grid(const VxLaunch &L) { return vx_full_sms(L) * 4; }

static cudaError_t maybe_pack(const VxLaunch &L, const VxParams &p, const VxView &v,
                              VxScalars *S, VxWork &w) {
    if (p.prec != VX_PREC_FP32) return cudaSuccess;
    vx_launch<k_pack32, k_pack32_body>(L, L.num_sms * 4, 256, 0, v, S, w.src32, w.cap);

    return cudaGetLastError();
}

// Source split of a step's pair sums: derived on the device from the body's
// own count (vx_ksplit), tiles of 1024 targets in FP32, 512 in FP64.
static VxSplit step_split(const VxLaunch &L, const VxParams &p, const VxWork &w, int nout) {
    VxSplit sp;
    sp.cap = w.part_cap;
    sp.K = 0;
    sp.sms = vx_full_sms(L);
    sp.tile = p.prec == VX_PREC_FP32 ? 1024 : 512;
    sp.nout = nout;
    return sp;
}

cudaError_t vx_launch_velocity(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                               VxWork &w) {
    const VxSplit sp = step_split(L, p, w, 5);
    if (maybe_pack(L, p, v, S, w) != cudaSuccess) return cudaGetLastError();
    if (p.prec == VX_PREC_FP32) {
        VX_EV(L, 0);
        vx_launch<k_bs32_partial<true>, k_bs32_partial_body<true>>(L, pair_grid(L), PT, 0, p, S, w.src32, v.x, v.y, v.ps, -1, w.part, sp);
        VX_EV(L, 1);

        vx_launch<k_bs_combine<true>, k_bs_combine_body<true>>(L, L.num_sms * 4, 256, 0, v, S, w.part, sp);
    } else {
        VX_EV(L, 0);
        vx_launch<k_bs_partial<double, true>, k_bs_partial_body<double, true>>(L, pair_grid(L), PT, 0, p, v, S, nullptr, v.x, v.y, v.ps, -1, w.part, sp);
        VX_EV(L, 1);

        vx_launch<k_bs_combine<false>, k_bs_combine_body<false>>(L, L.num_sms * 4, 256, 0, v, S, w.part, sp);
    }

    return cudaGetLastError();
}

cudaError_t vx_launch_diffusion(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                                VxWork &w) {
    // bulk form: neighbour lists within diff_cutoff * d_i (vx_cells.cu)
    if (p.prec == VX_PREC_FP32 && p.diff_cutoff > 0.0) return vx_launch_diffusion_cells(L, p, v, S, w);
    const VxSplit sp = step_split(L, p, w, 3);
    VX_EV(L, 2);
    if (p.prec == VX_PREC_FP32) {
        vx_launch<k_diff_partial<float>, k_diff_partial_body<float>>(L, pair_grid(L), PT, 0, p, v, S, w.src32, w.part, sp);
    } else {
        vx_launch<k_diff_partial<double>, k_diff_partial_body<double>>(L, pair_grid(L), PT, 0, p, v, S, nullptr, w.part, sp);
    }
    VX_EV(L, 3);

    vx_launch<k_diff_combine, k_diff_combine_body>(L, L.num_sms * 4, 256, 0, p, v, S, w.part, sp);

    return cudaGetLastError();
}

// Probe points: the caller's split K (chosen from the point count), at
// least one point per partial slot.
cudaError_t vx_launch_probe(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                            VxWork &w, const double *px, const double *py, long long pstride,
                            long long np, double *ovx, double *ovy, long long ostride, int K) {
    if (K < 1 || w.part_cap / (2LL * K) < np) return cudaErrorInvalidValue;
    VxSplit sp;
    sp.cap = w.part_cap;
    sp.K = K;
    sp.sms = vx_full_sms(L);
    sp.tile = p.prec == VX_PREC_FP32 ? 1024 : 512;
    sp.nout = 2;
    if (maybe_pack(L, p, v, S, w) != cudaSuccess) return cudaGetLastError();
    if (p.prec == VX_PREC_FP32)
        vx_launch<k_bs32_partial<false>, k_bs32_partial_body<false>>(L, pair_grid(L), PT, 0, p, S, w.src32, px, py, pstride, np, w.part, sp);
    else
        vx_launch<k_bs_partial<double, false>, k_bs_partial_body<double, false>>(L, pair_grid(L), PT, 0, p, v, S, nullptr, px, py, pstride, np, w.part, sp);

    vx_launch<k_probe_combine, k_probe_combine_body>(L, (int)vx_ceil_div(np, 256), 256, 0, S, w.part, sp, np, ovx, ovy, ostride);

    return cudaGetLastError();
}
