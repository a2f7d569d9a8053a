// vx_compact.cu — removal of vortices with |G| < drop_eps, reproducing the
// reference's serial swap-with-last permutation exactly, in parallel.
//
// Reference: sort_Kernel src/kernel.cu:1159-1178 (one thread walks i upward
// and swaps every dead element with the current last one).  Closed form of
// its result, with m = number of live elements among [0, n0), scan[p] = live
// elements before p, H = dead elements below m (= live elements at or above m):
//  * live elements below m stay;
//  * the t-th dead position below m (ascending) receives the live element
//    that is t-th from the top among positions >= m;
//  * each tail position e in [m, n0) gets G = 0 and the position of
//      - the hole it was swapped with, when e is the first slot of its run
//        (e = n0-1, or e+1 holds a live element); the hole of the run with
//        k live elements above e is the k-th hole, or m itself once all
//        holes are filled,
//      - otherwise the element that was at e+1.
// Four launches: chunk counts (whose last block scans them), per-chunk
// classification, gather into scratch, scatter back.  Everything outside
// [0, n0) is untouched.
#include "vx_internal.cuh"

__device__ __forceinline__ bool vx_live(const VxView &v, long long p, double eps) {
    return fabs(v.g[p * v.ps]) >= eps;
}

// Live elements per chunk; the block that finishes last then scans the
// chunk counts and finds m, scan[m] and H.
VX_DEVK void k_cmp_count_body(VxBlkB<VX_THREADS, 0> vb, const VxView &v, VxScalars *S, double eps, int *cnt,
                              long long *off, const int *skip) {
    if (skip && *skip) return;
    __shared__ long long sh[VX_THREADS];
    const long long n0 = S->n;
    const long long nch = vx_ceil_div(n0, VX_CHUNK);
    for (long long c = vb.x; c < nch; c += vb.n) {
        int k = 0;
        const long long b = c * VX_CHUNK, e = min(n0, b + VX_CHUNK);
        for (long long p = b + threadIdx.x; p < e; p += blockDim.x) k += vx_live(v, p, eps);
        sh[threadIdx.x] = k;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) cnt[c] = (int)sh[0];
        __syncthreads();
    }
    if (!vx_last_block(&S->sync_ctr, vb.n)) return;
    // exclusive scan of the chunk counts, VX_THREADS at a time
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < nch; base += blockDim.x) {
        const long long c = base + threadIdx.x;
        const long long val = c < nch ? __ldcg(&cnt[c]) : 0;
        sh[threadIdx.x] = val;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {       // inclusive Hillis-Steele
            const long long t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (c < nch) off[c] = carry + sh[threadIdx.x] - val;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += sh[threadIdx.x];
        __syncthreads();
    }
    const long long m = carry;
    // live elements in [0, m)
    long long scan_m = m;
    if (m < n0) {
        const long long cm = m / VX_CHUNK;
        long long k = 0;
        for (long long p = cm * VX_CHUNK + threadIdx.x; p < m; p += blockDim.x) k += vx_live(v, p, eps);
        sh[threadIdx.x] = k;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        scan_m = off[cm] + sh[0];
    }
    if (threadIdx.x == 0) {
        S->c_n0 = n0;
        S->c_m = m;
        S->c_scan_m = scan_m;
        S->c_H = m - scan_m;
    }
}
__global__ void __launch_bounds__(VX_THREADS) k_cmp_count(VxView v, VxScalars *S, double eps, int *cnt,
                                                          long long *off, const int *skip) {
    VX_PDL_WAIT();
    k_cmp_count_body(VxBlkB<VX_THREADS, 0>{blockIdx.x, gridDim.x}, v, S, eps, cnt, off, skip);
}

// Per chunk: local scan, then hole positions, hole sources and tail sources.
// tail_src < 0 encodes "the position of hole -(value+1)".
VX_DEVK void k_cmp_classify_body(VxBlkB<VX_THREADS, 0> vb, const VxView &v, const VxScalars *S, double eps,
                                 const long long *off, int *hole_pos,
                                 int *hole_src, int *tail_src,
                                 const int *skip) {
    if (skip && *skip) return;
    constexpr int PER = VX_CHUNK / VX_THREADS;
    __shared__ int sh[VX_THREADS];
    const long long n0 = S->c_n0, m = S->c_m, H = S->c_H, scan_m = S->c_scan_m;
    if (m == n0) return;
    const long long nch = vx_ceil_div(n0, VX_CHUNK);
    for (long long c = vb.x; c < nch; c += vb.n) {
        const long long b = c * VX_CHUNK + (long long)threadIdx.x * PER;
        bool lv[PER];
        int loc = 0;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            long long p = b + q;
            lv[q] = p < n0 && vx_live(v, p, eps);
            loc += lv[q];
        }
        sh[threadIdx.x] = loc;
        __syncthreads();
        for (int o = 1; o < VX_THREADS; o <<= 1) {
            int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        long long scan = off[c] + sh[threadIdx.x] - loc;   // live before b
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const long long p = b + q;
            if (p >= n0) break;
            if (p < m && !lv[q]) hole_pos[p - scan] = (int)p;
            if (p >= m && lv[q]) hole_src[H - 1 - (scan - scan_m)] = (int)p;
            if (p >= m) {
                const bool next_live = (p + 1 < n0) && vx_live(v, p + 1, eps);
                const long long scan_next = scan + lv[q];
                int src;
                if (p == n0 - 1 || next_live) {
                    const long long grp = m - scan_next;   // live elements in (p, n0)
                    src = grp < H ? -(int)(grp + 1) : (int)m;
                } else {
                    src = (int)(p + 1);
                }
                tail_src[p - m] = src;
            }
            scan += lv[q];
        }
    }
}
__global__ void __launch_bounds__(VX_THREADS) k_cmp_classify(VxView v, const VxScalars *S, double eps,
                                                             const long long *off, int *hole_pos,
                                                             int *hole_src, int *tail_src,
                                                             const int *skip) {
    VX_PDL_WAIT();
    k_cmp_classify_body(VxBlkB<VX_THREADS, 0>{blockIdx.x, gridDim.x}, v, S, eps, off, hole_pos, hole_src, tail_src, skip);
}

VX_DEVK void k_cmp_gather_body(VxBlkB<0, 0> vb, const VxView &v, const VxScalars *S, const int *hole_pos, const int *hole_src,
                               const int *tail_src, double *hx, double *hy, double *hg, double *tx,
                               double *ty, const int *skip) {
    if (skip && *skip) return;
    const long long n0 = S->c_n0, m = S->c_m, H = S->c_H;
    if (m == n0) return;
    const long long T = n0 - m;
    for (long long k = vb.x * (long long)blockDim.x + threadIdx.x; k < H + T;
         k += (long long)vb.n * blockDim.x) {
        if (k < H) {
            const long long s = (long long)hole_src[k] * v.ps;
            hx[k] = v.x[s]; hy[k] = v.y[s]; hg[k] = v.g[s];
        } else {
            const long long e = k - H;
            int s = tail_src[e];
            if (s < 0) s = hole_pos[-s - 1];
            tx[e] = v.x[(long long)s * v.ps];
            ty[e] = v.y[(long long)s * v.ps];
        }
    }
}
__global__ void k_cmp_gather(VxView v, const VxScalars *S, const int *hole_pos, const int *hole_src,
                             const int *tail_src, double *hx, double *hy, double *hg, double *tx,
                             double *ty, const int *skip) {
    VX_PDL_WAIT();
    k_cmp_gather_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, hole_pos, hole_src, tail_src, hx, hy, hg, tx, ty, skip);
}

// count_step: this compaction closes a whole step, which it counts (no
// kernel after it in the step reads the step index).
VX_DEVK void k_cmp_scatter_body(VxBlkB<0, 0> vb, const VxView &v, VxScalars *S, const int *hole_pos, const double *hx,
                                const double *hy, const double *hg, const double *tx, const double *ty,
                                const int *skip, int count_step) {
    if (count_step && vb.x == 0 && threadIdx.x == 0) S->step += 1;
    if (skip && *skip) return;
    const long long n0 = S->c_n0, m = S->c_m, H = S->c_H;
    if (m != n0) {
        const long long T = n0 - m;
        for (long long k = vb.x * (long long)blockDim.x + threadIdx.x; k < H + T;
             k += (long long)vb.n * blockDim.x) {
            if (k < H) {
                const long long d = (long long)hole_pos[k] * v.ps;
                v.x[d] = hx[k]; v.y[d] = hy[k]; v.g[d] = hg[k];
            } else {
                const long long e = k - H;
                const long long d = (m + e) * v.ps;
                v.x[d] = tx[e]; v.y[d] = ty[e]; v.g[d] = 0.0;
            }
        }
    }
    if (vb.x == 0 && threadIdx.x == 0) S->n = m;
}
__global__ void k_cmp_scatter(VxView v, VxScalars *S, const int *hole_pos, const double *hx,
                              const double *hy, const double *hg, const double *tx, const double *ty,
                              const int *skip, int count_step) {
    VX_PDL_WAIT();
    k_cmp_scatter_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, hole_pos, hx, hy, hg, tx, ty, skip, count_step);
}

cudaError_t vx_launch_compact_skip(const VxLaunch &L, const VxParams &p, const VxView &v,
                                   VxScalars *S, VxWork &w, const int *skip, bool count_step) {
    const int grid = L.num_sms * 4;
    vx_launch<k_cmp_count, k_cmp_count_body>(L, grid, VX_THREADS, 0, v, S, p.drop_eps, w.cmp_cnt, w.cmp_off, skip);
    vx_launch<k_cmp_classify, k_cmp_classify_body>(L, grid, VX_THREADS, 0, v, S, p.drop_eps, w.cmp_off, w.hole_pos, w.hole_src, w.tail_src, skip);
    vx_launch<k_cmp_gather, k_cmp_gather_body>(L, grid, VX_THREADS, 0, v, S, w.hole_pos, w.hole_src, w.tail_src, w.hx, w.hy, w.hg, w.tx, w.ty, skip);
    vx_launch<k_cmp_scatter, k_cmp_scatter_body>(L, grid, VX_THREADS, 0, v, S, w.hole_pos, w.hx, w.hy, w.hg, w.tx, w.ty, skip, count_step ? 1 : 0);

    return cudaGetLastError();
}

cudaError_t vx_launch_compact(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                              VxWork &w, bool count_step) {
    return vx_launch_compact_skip(L, p, v, S, w, nullptr, count_step);
}
