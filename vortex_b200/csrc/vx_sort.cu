// vx_sort.cu — stable LSD radix sort of (32-bit key, int value) pairs with
// the element count read from device memory.
//
// Per 8-bit digit: (1) every tile of VX_RS_TILE elements counts its digits,
// (2) one block per digit scans that digit's tile counts, (3) every tile
// scatters its elements in their original order: the rank of an element
// among equal digits is (elements of earlier tiles) + (earlier rounds of this
// tile) + (earlier warps of this round) + (earlier lanes of this warp), the
// last from a warp match.  Equal keys keep their input order, so sorting
// particle indices by cell gives a deterministic order inside every cell.
#include "vx_internal.cuh"

constexpr int RS_THREADS = 256;
constexpr int RS_ROUNDS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;   // elements per tile
constexpr int RS_WARPS = RS_THREADS / 32;

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const long long *d_n, const unsigned *keys, int shift,
                                                        int *hist, long long tiles_cap) {
    VX_PDL_WAIT();
    __shared__ int cnt[256];
    const long long n = *d_n;
    const long long tiles = vx_ceil_div(n, RS_TILE);
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        cnt[threadIdx.x] = 0;
        __syncthreads();
        for (int r = 0; r < RS_ROUNDS; ++r) {
            const long long e = t * RS_TILE + (long long)r * RS_THREADS + threadIdx.x;
            if (e < n) atomicAdd(&cnt[(keys[e] >> shift) & 255u], 1);
        }
        __syncthreads();
        hist[(long long)threadIdx.x * tiles_cap + t] = cnt[threadIdx.x];   // digit-major
        __syncthreads();
    }
}

// Exclusive scan of each digit's tile counts, one block per digit (digit-
// local offsets in off, digit totals in dtot); the scatter adds the digit's
// prefix over dtot.
constexpr int RS_SCAN_T = 512;
__global__ void __launch_bounds__(RS_SCAN_T) k_rs_scan(const long long *d_n, const int *hist, long long *off,
                                                       long long tiles_cap, long long *dtot) {
    VX_PDL_WAIT();
    __shared__ long long wsum[RS_SCAN_T / 32];
    const long long tiles = vx_ceil_div(*d_n, RS_TILE);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long d = blockIdx.x;
    long long carry = 0;
    for (long long t0 = 0; t0 < tiles; t0 += RS_SCAN_T) {
        const long long t = t0 + threadIdx.x;
        const long long c = t < tiles ? hist[d * tiles_cap + t] : 0;
        long long inc = c;
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) wsum[warp] = inc;
        __syncthreads();
        long long before = 0, total = 0;
        for (int q = 0; q < RS_SCAN_T / 32; ++q) {
            before += q < warp ? wsum[q] : 0;
            total += wsum[q];
        }
        if (t < tiles) off[d * tiles_cap + t] = carry + before + inc - c;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) dtot[d] = carry;
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const long long *d_n, const unsigned *keys,
                                                           const int *vals, unsigned *okeys, int *ovals, int shift,
                                                           const long long *off, long long tiles_cap,
                                                           const long long *dtot) {
    VX_PDL_WAIT();
    static_assert(RS_THREADS == 256, "one thread per digit");
    __shared__ int warp_cnt[RS_WARPS][256];
    __shared__ long long base[256];
    __shared__ long long dpre[256];
    __shared__ long long wtot[RS_WARPS];
    const long long n = *d_n;
    const long long tiles = vx_ceil_div(n, RS_TILE);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    {   // exclusive prefix of the digit totals (thread d owns digit d)
        const long long c = dtot[threadIdx.x];
        long long inc = c;
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) wtot[warp] = inc;
        __syncthreads();
        long long before = 0;
        for (int q = 0; q < warp; ++q) before += wtot[q];
        dpre[threadIdx.x] = before + inc - c;
        __syncthreads();
    }
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        base[threadIdx.x] = dpre[threadIdx.x] + off[(long long)threadIdx.x * tiles_cap + t];
        __syncthreads();
        for (int r = 0; r < RS_ROUNDS; ++r) {
            for (int w = 0; w < RS_WARPS; ++w) warp_cnt[w][threadIdx.x] = 0;
            __syncthreads();
            const long long e = t * RS_TILE + (long long)r * RS_THREADS + threadIdx.x;
            const bool valid = e < n;
            const unsigned key = valid ? keys[e] : 0u;
            const int val = valid ? vals[e] : 0;
            const unsigned dig = valid ? ((key >> shift) & 255u) : 256u;   // 256: no digit
            const unsigned peers = __match_any_sync(0xffffffffu, dig);
            const int rank = __popc(peers & lt_mask);
            if (valid && rank == 0) warp_cnt[warp][dig] = __popc(peers);
            __syncthreads();
            // thread d turns the per-warp counts of digit d into warp offsets
            {
                const int d = threadIdx.x;
                int run = 0;
                for (int w = 0; w < RS_WARPS; ++w) {
                    const int c = warp_cnt[w][d];
                    warp_cnt[w][d] = run;
                    run += c;
                }
                __syncthreads();
                if (valid) {
                    const long long pos = base[dig] + warp_cnt[warp][dig] + rank;
                    okeys[pos] = key;
                    ovals[pos] = val;
                }
                __syncthreads();
                base[d] += run;
            }
            __syncthreads();
        }
    }
}

// Sorts keys/vals (count *d_n) by bits [0, nbits) of the key.  Buffers
// alternate between (k0,v0) and (k1,v1); the return value tells which pair
// holds the result (0 or 1).  hist holds 256 * tiles_cap entries, off
// 256 * (tiles_cap + 1) (the digit totals follow the offsets).
int vx_radix_sort(const VxLaunch &L, const long long *d_n, unsigned *k0, int *v0, unsigned *k1, int *v1,
                  int nbits, int *hist, long long *off, long long tiles_cap) {
    const int grid = L.num_sms * 4;
    int cur = 0;
    for (int shift = 0; shift < nbits; shift += 8) {
        unsigned *ki = cur ? k1 : k0, *ko = cur ? k0 : k1;
        int *vi = cur ? v1 : v0, *vo = cur ? v0 : v1;
        vx_launch_pdl(k_rs_hist, grid, RS_THREADS, 0, L.stream, d_n, ki, shift, hist, tiles_cap); VX_COUNT(L);
        vx_launch_pdl(k_rs_scan, 256, RS_SCAN_T, 0, L.stream, d_n, hist, off, tiles_cap, off + 256 * tiles_cap);
        VX_COUNT(L);
        vx_launch_pdl(k_rs_scatter, grid, RS_THREADS, 0, L.stream, d_n, ki, vi, ko, vo, shift, off, tiles_cap,
                                                         off + 256 * tiles_cap);
        VX_COUNT(L);
        cur ^= 1;
    }
    return cur;
}

long long vx_rs_tiles_cap(long long cap) { return cap / RS_TILE + 2; }
