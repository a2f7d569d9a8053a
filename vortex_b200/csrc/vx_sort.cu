// vx_sort.cu — the stable bucket order of the particle grids (cells of the
// diffusion grid, leaves of the quadtree): particle indices arranged by
// bucket, each bucket's particles in index order, from per-bucket counts and
// their exclusive scan (which the grids compute anyway), without a radix sort.
// Equal keys keep their input order, so sorting particle indices by cell gives
// a deterministic order inside every cell.
#include <climits>
#include <vector>

#include "vx_internal.cuh"

// Stable order by bucket, for keys whose buckets already have counts and
// starts (an exclusive scan of the counts): every element
// takes a slot of its bucket (its start plus an atomic rank, in no fixed
// order), then each bucket's slots are put back in element-index order, the
// order a stable sort by bucket gives (rank of an element = the number of
// the bucket's elements with a lower index).  A bucket of up to 16 elements
// takes one thread, one of up to 128 a warp, a larger one a block (the warps
// and blocks in one launch after the threads').  The
// counts are used up by the placement and written back by the ordering.
VX_DEVK void k_bk_place_body(VxBlkB<0, 0> vb, const long long *d_n, const unsigned *key, const int *start, int *cnt0,
                             const long long *d_off, unsigned *okey, int *oval) {
    const long long n = *d_n;
    int *cnt = cnt0 + (d_off ? *d_off : 0);
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        const unsigned c = key[i];
        const int pos = start[c] + atomicSub(&cnt[c], 1) - 1;
        okey[pos] = c;
        oval[pos] = (int)i;
    }
}
__global__ void k_bk_place(const long long *d_n, const unsigned *key, const int *start, int *cnt0,
                           const long long *d_off, unsigned *okey, int *oval) {
    VX_PDL_WAIT();
    k_bk_place_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, d_n, key, start, cnt0, d_off, okey, oval);
}

constexpr int BK_S = 16;  // a thread orders buckets of up to BK_S elements
constexpr int BK_E = 4;   // elements per lane: a warp orders buckets of up to 32 * BK_E

// One thread per bucket: writes the count back, orders a bucket of up to
// BK_S elements itself (ranks by counting, in registers) and lists larger
// ones for a warp (mid) or a block (big).
VX_DEVK void k_bk_order_body(VxBlkB<256, 3> vb, VxScalars *S, const long long *d_nb, const int *start, int *cnt0, const long long *d_off,
                             int *oval, int *mid, int *big, VxGather gt) {
    const long long nb = *d_nb;
    int *cnt = cnt0 + (d_off ? *d_off : 0);
    for (long long b = vb.x * (long long)blockDim.x + threadIdx.x; b < nb;
         b += (long long)vb.n * blockDim.x) {
        const int a = start[b], m = start[b + 1] - a;
        cnt[b] = gt.zero_counts ? 0 : m;
        if (m <= 1) {
            if (m == 1 && gt.mode) vx_gather_slot(gt, a, oval[a], (unsigned)b);
            continue;
        }
        if (m > BK_S) {
            if (m > 32 * BK_E) big[atomicAdd(&S->bk_nbig, 1)] = (int)b;
            else mid[atomicAdd(&S->bk_nmid, 1)] = (int)b;
            continue;
        }
        int v[BK_S];
#pragma unroll
        for (int e = 0; e < BK_S; ++e) v[e] = e < m ? oval[a + e] : INT_MAX;
#pragma unroll
        for (int e = 0; e < BK_S; ++e) {
            int r = 0;
#pragma unroll
            for (int k = 0; k < BK_S; ++k) r += v[k] < v[e];
            if (e < m) {
                oval[a + r] = v[e];
                if (gt.mode) vx_gather_slot(gt, a + r, v[e], (unsigned)b);
            }
        }
    }
}
__global__ void k_bk_order(VxScalars *S, const long long *d_nb, const int *start, int *cnt0, const long long *d_off,
                           int *oval, int *mid, int *big, VxGather gt) {
    VX_PDL_WAIT();
    k_bk_order_body(VxBlkB<256, 3>{blockIdx.x, gridDim.x}, S, d_nb, start, cnt0, d_off, oval, mid, big, gt);
}

// The listed buckets, one launch: a block per bucket of more than 32 BK_E
// elements (each element counts the smaller ones, the bucket staged in
// shared memory when it fits), then a warp per bucket of BK_S < m <= 32 BK_E
// elements (lane holds elements lane, lane + 32, ...).
constexpr int BK_T = 512;
constexpr int BK_SH = 4096;   // elements of a bucket held in shared memory; larger ones go through scratch
VX_DEVK void k_bk_order_rest_body(VxBlkB<BK_T, 0> vb, const VxScalars *S, const int *start, const int *mid,
                                  const int *big, int *oval, int *scratch, VxGather gt) {
    __shared__ int sv[BK_SH];
    const int nbig = S->bk_nbig;
    for (int q = vb.x; q < nbig; q += vb.n) {
        const int b = big[q];
        const int a = start[b], m = start[b + 1] - a;
        const bool sh = m <= BK_SH;
        int *src = sh ? sv : scratch + a;
        for (int e = threadIdx.x; e < m; e += BK_T) src[e] = oval[a + e];
        __syncthreads();
        for (int e = threadIdx.x; e < m; e += BK_T) {
            const int v = src[e];
            int r = 0;
            for (int k = 0; k < m; ++k) r += src[k] < v;
            oval[a + r] = v;
            if (gt.mode) vx_gather_slot(gt, a + r, v, (unsigned)b);
        }
        __syncthreads();
    }
    const int nmid = S->bk_nmid;
    const int lane = threadIdx.x & 31;
    const int nw = (vb.n * BK_T) >> 5;
    for (int q = (vb.x * BK_T + threadIdx.x) >> 5; q < nmid; q += nw) {
        const int b = mid[q];
        const int a = start[b], m = start[b + 1] - a;
        int v[BK_E], r[BK_E];
#pragma unroll
        for (int e = 0; e < BK_E; ++e) {
            v[e] = lane + 32 * e < m ? oval[a + lane + 32 * e] : INT_MAX;
            r[e] = 0;
        }
        const int rounds = (m + 31) / 32;
        for (int g = 0; g < rounds; ++g) {
            int u0 = v[0];
#pragma unroll
            for (int e = 1; e < BK_E; ++e) u0 = g == e ? v[e] : u0;   // the round's element of this lane
            for (int k = 0; k < 32; ++k) {
                const int u = __shfl_sync(0xffffffffu, u0, k);
#pragma unroll
                for (int e = 0; e < BK_E; ++e) r[e] += u < v[e];
            }
        }
        __syncwarp();
#pragma unroll
        for (int e = 0; e < BK_E; ++e)
            if (lane + 32 * e < m) {
                oval[a + r[e]] = v[e];
                if (gt.mode) vx_gather_slot(gt, a + r[e], v[e], (unsigned)b);
            }
    }
}
__global__ void __launch_bounds__(BK_T) k_bk_order_rest(const VxScalars *S, const int *start, const int *mid,
                                                        const int *big, int *oval, int *scratch, VxGather gt) {
    VX_PDL_WAIT();
    k_bk_order_rest_body(VxBlkB<BK_T, 0>{blockIdx.x, gridDim.x}, S, start, mid, big, oval, scratch, gt);
}

cudaError_t vx_bucket_order(const VxLaunch &L, VxScalars *S, const long long *d_n, const long long *d_nbuckets,
                            const unsigned *key, const int *start, int *cnt, const long long *d_cnt_off,
                            unsigned *okey, int *oval, int *mid, int *big, int *scratch, const VxGather &gt) {
    vx_launch<k_bk_place, k_bk_place_body>(L, L.num_sms * 4, 256, 0, d_n, key, start, cnt, d_cnt_off, okey, oval);

    vx_launch<k_bk_order, k_bk_order_body>(L, L.num_sms * 4, 256, 0, S, d_nbuckets, start, cnt, d_cnt_off, oval, mid, big, gt);

    vx_launch<k_bk_order_rest, k_bk_order_rest_body>(L, L.num_sms * 4, BK_T, 0, S, start, mid, big, oval, scratch, gt);

    return cudaGetLastError();
}

// Validation hook: the bucket order of n keys (device array, each below nb)
// into `order` (device array of n element indices), with counts and starts
// computed on the host.  Allocates its own scratch; not for the step path.
extern "C" vx_status vx_eval_bucket_order(const unsigned *key, int64_t n, int64_t nb, int *order) {
    if (n < 0 || nb < 1 || n > INT_MAX || (n > 0 && (!key || !order))) return VX_ERR_ARG;
    if (n == 0) return VX_OK;
    std::vector<unsigned> hk((size_t)n);
    if (cudaMemcpy(hk.data(), key, sizeof(unsigned) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return VX_ERR_CUDA;
    std::vector<int> cnt((size_t)nb, 0), start((size_t)nb + 1, 0);
    for (unsigned k : hk) {
        if ((int64_t)k >= nb) return VX_ERR_ARG;
        ++cnt[k];
    }
    for (int64_t b = 0; b < nb; ++b) start[b + 1] = start[b] + cnt[b];
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void *mem[8] = {};
    const size_t sz[8] = {sizeof(VxScalars), 2 * sizeof(long long), sizeof(int) * (nb + 1), sizeof(int) * nb,
                          sizeof(unsigned) * n, sizeof(int) * (n / 16 + 2), sizeof(int) * (n / 128 + 2),
                          sizeof(int) * n};
    vx_status st = VX_OK;
    for (int q = 0; q < 8 && st == VX_OK; ++q)
        if (cudaMalloc(&mem[q], sz[q]) != cudaSuccess) st = VX_ERR_NOMEM;
    if (st == VX_OK) {
        VxScalars *S = (VxScalars *)mem[0];
        long long *dn = (long long *)mem[1];
        const long long hn[2] = {(long long)n, (long long)nb};
        int *dstart = (int *)mem[2], *dcnt = (int *)mem[3];
        bool ok = cudaMemset(S, 0, sizeof(VxScalars)) == cudaSuccess &&
                  cudaMemcpy(dn, hn, sizeof(hn), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(dstart, start.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(dcnt, cnt.data(), sizeof(int) * nb, cudaMemcpyHostToDevice) == cudaSuccess;
        if (ok) {
            VxLaunch L;
            L.stream = 0;
            L.launches = nullptr;
            L.num_sms = sms;
            ok = vx_bucket_order(L, S, dn, dn + 1, key, dstart, dcnt, nullptr, (unsigned *)mem[4], order,
                                 (int *)mem[5], (int *)mem[6], (int *)mem[7]) == cudaSuccess &&
                 cudaDeviceSynchronize() == cudaSuccess;
        }
        std::vector<int> back((size_t)nb);
        if (ok) ok = cudaMemcpy(back.data(), dcnt, sizeof(int) * nb, cudaMemcpyDeviceToHost) == cudaSuccess;
        if (ok && back != cnt) st = VX_ERR_DEVICE;   // the counts must come back as they went in
        if (!ok) st = VX_ERR_CUDA;
    }
    for (void *p : mem) if (p) cudaFree(p);
    return st;
}
