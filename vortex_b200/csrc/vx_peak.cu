// vx_peak.cu — measured vector-pipe peak of the GPU (FP32 or FP64 fused
// multiply-add throughput), the roofline denominator of the pair kernels,
// which run on the SIMT pipes rather than the tensor cores.
#include "vx_internal.cuh"

template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T *out, int iters, T a, T b) {
    T r[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = (T)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = fma(r[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += r[k];
    if (s == (T)12345.678) out[blockIdx.x] = s;   // keeps the chain alive
}

// Packed FP32 pairs (fma.rn.f32x2, PTX ISA 8.6, sm_100+): two FMAs per
// instruction on 64-bit register pairs.
__device__ __forceinline__ unsigned long long vx_fma2(unsigned long long a, unsigned long long b,
                                                      unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

__global__ void __launch_bounds__(256) k_fma2_peak(float *out, int iters, float a, float b) {
    unsigned long long r[8];
    const unsigned long long A = ((unsigned long long)__float_as_uint(a) << 32) | __float_as_uint(a);
    const unsigned long long B = ((unsigned long long)__float_as_uint(b) << 32) | __float_as_uint(b);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        unsigned v = __float_as_uint((float)(threadIdx.x + k));
        r[k] = ((unsigned long long)v << 32) | v;
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = vx_fma2(r[k], A, B);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += __uint_as_float((unsigned)r[k]) + __uint_as_float((unsigned)(r[k] >> 32));
    if (s == 12345.678f) out[blockIdx.x] = s;
}

// Special-function pipe: one rsqrt and one ex2 per unit (the MUFU work of a
// vortex-diffusion pair), eight independent chains per thread.
__global__ void __launch_bounds__(256) k_mufu_peak(float *out, int iters) {
    float r[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = 1.0f + 0.001f * (float)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float q, e;
            asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(q) : "f"(r[k]));
            asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-0.01f * q));
            r[k] = e;
        }
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += r[k];
    if (s == 12345.678f) out[blockIdx.x] = s;
}

// FLOP/s of back-to-back FMAs over the whole GPU (2 flops per FMA), best of
// 5 timed launches after a warm-up.  fp64: 0 = FP32, 1 = FP64, 2 = packed
// FP32 pairs (f32x2), 3 = rsqrt + ex2 units per second (in units of 1e12: the
// special-function ceiling of the diffusion pairs).
extern "C" vx_status vx_measure_peak(int device, int fp64, double *tflops) {
    if (!tflops) return VX_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return VX_ERR_CUDA;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = fp64 ? 4096 : 16384;
    void *out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks) != cudaSuccess) return VX_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(e0);
        if (fp64 == 1) k_fma_peak<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
        else if (fp64 == 2) k_fma2_peak<<<blocks, threads>>>((float *)out, iters, 0.9999f, 1e-4f);
        else if (fp64 == 3) k_mufu_peak<<<blocks, threads>>>((float *)out, iters / 4);
        else k_fma_peak<float><<<blocks, threads>>>((float *)out, iters, 0.9999f, 1e-4f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return VX_ERR_CUDA;
    const double flops = fp64 == 3 ? 8.0 * (double)(iters / 4) * threads * blocks
                                   : (fp64 == 2 ? 4.0 : 2.0) * 8.0 * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return VX_OK;
}
