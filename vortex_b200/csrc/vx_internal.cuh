// vx_internal.cuh — shared device structures, helpers and stage launchers of
// libvortex_b200.  Every stage reads the live particle count from device
// memory (VxScalars::n), so a whole step is launched without host round
// trips and the launch shapes do not depend on the particle count.
//
// Floating-point contract: the library is compiled with -fmad=false; every
// fused multiply-add is an explicit fma()/fmaf(), the same calls the CPU
// oracle makes.  This keeps the 3-nearest distances, compaction, collapse
// pairing and merge, and the advection bit-identical to the oracle.
#pragma once

#include <cuda_runtime.h>
#include <utility>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <type_traits>
#include <vector>

#include "../../include/vortex_b200.h"

#define VX_TWO_PI 6.283185307179586
#define VX_PI 3.141592653589793

// ---------------------------------------------------------------------------
// Particle storage view.  Element i of x/y/g is at [i*ps], of vx/vy at
// [i*vs]: structure-of-arrays (ps = vs = 1) for the native engine, the
// reference's AoS Vortex/PVortex records (ps = 3, vs = 2) for the
// unit_1.cuh-compatible entry points.
struct VxView {
    double *x, *y, *g;
    long long ps;
    double *vx, *vy;
    long long vs;
    double *d;
};

// Resolved run parameters (reference: __constant__ symbols filled by
// init_device_conf_values, src/unit_1.cu:20-44,1220-1252).
struct VxParams {
    double dt, nu, rho;
    double eps, eps2;
    double r_diff2, r_same2, max_ve_g;
    double x_min, x_max, y_min, y_max;          // wake window
    double px_min, px_max, py_min, py_max;      // profile bbox (left endpoints)
    double wall_x0, wall_x1, wall_y0, wall_y1;  // birth-point bbox grown by 5 L_max
    double wall_h;                              // side of the wall panel-list cells
    int wall_nx, wall_ny;                       // wall cells (0: no lists)
    double hit_x0, hit_y0, hit_h;               // hitting-test panel lists: grid origin, cell side
    int hit_nx, hit_ny;                         // hitting cells (0: no lists)
    double rc_x, rc_y;
    double drop_eps;
    double diff_cutoff;
    // birth right-hand side of the bulk form: vortices farther than
    // sqrt(b_rfar2) from the body centre (bc_x, bc_y) enter through one
    // local expansion about that centre (birth_far != 0)
    double bc_x, bc_y, b_rfar2;
    int birth_far;
    int fmm_leaf;          // quadtree depth aims at this many vortices per leaf
    int fmm_p;             // expansion terms of the quadtree FMM (8, 12, 16 or 20)
    int P;
    int n_of_points;
    int birth_mode;
    int prec;
};

// Device-resident scalars of one body.
struct VxScalars {
    long long n;           // live particle count
    long long n0;          // count before this step's birth
    long long step;        // completed steps
    long long incr_steps;  // V_inf ramp length (src/main.c:586-592,654-659)
    double vinf[2];
    double dvinf[2];
    double dg;             // circulation absorbed by the last convection
    double fx, fy, m;      // force and moment of the last step
    double raw[4];         // unscaled sums of dg, Fx, Fy, M of the last convection
    // compaction
    long long c_n0, c_m, c_H, c_scan_m;
    // collapse
    long long col_n_before;
    int col_done;
    int ncand;
    double gx0, gy0, gh;
    long long gnx, gny, gncells;
    int err;
    int cnwide;            // diffusion targets whose cut-off exceeds the item window
    int cnhuge;            // of those, the ones whose window spans more than WIDE_ROWS rows each side
    long long bf_nnear;    // birth sources inside the far-field radius
    // neighbour-list grid of the bulk form (vortex diffusion)
    double cx0, cy0, ch, chy;   // origin, cell width and cell height
    long long cnx, cny, cncells, cnitems;
    // quadtree of the bulk-form Biot-Savart (vx_fmm.cu)
    double fx0, fy0, fside;
    long long fnleaves, fs;
    long long fnsub;       // cells of the level below the leaves (4 per leaf): the 3-nearest grid
    int fL, fnflag;
    int fnbrute;           // flagged targets left to the whole-set 3-nearest scan
    int bk_nmid, bk_nbig;  // buckets of 17..128 / more elements in the running bucket order (vx_sort.cu)
    long long fcnt_off;    // offset of the leaf level in the quadtree's count array
    unsigned long long fsq;   // sum over the quarter-leaf cells of count^2 at the last tree build (depth rule)
    int fLcap;                // deepest level the depth rule may deepen to (0: none): set when a deepened tree
                              // left too many targets to the exact 3-nearest search
    // pair evaluations executed by the bulk-form near-field and diffusion
    // kernels since the counters were last cleared
    unsigned long long pairs_bs, pairs_diff;
    // grid-wide steps inside one launch (vx_last_block, vx_scan_lookback):
    // the arrival counter of the last-block pattern, and the running scan's
    // tile ticket, finished-block count and epoch (all at rest between
    // launches: the counters at zero, the epoch advanced once per scan)
    unsigned sync_ctr, scan_ticket, scan_done, scan_epoch;
};

enum {
    VX_DERR_RESOLVE = 1,     // collapse resolution did not converge
    VX_DERR_GRID = 2,        // collapse grid did not fit its cell capacity
    VX_DERR_SCAN = 4,        // a look-back scan gave up waiting on a predecessor tile
};

// Device scratch of one body.  Sizes are in elements.
struct VxWork {
    long long cap;           // particle capacity the arrays below were sized for
    long long bytes;         // device bytes the arrays below take
    // compaction
    int *cmp_cnt;
    long long *cmp_off;
    int *hole_pos, *hole_src, *tail_src;
    double *hx, *hy, *hg, *tx, *ty;
    // collapse
    long long cells_cap;
    int *cellid, *cell_cnt, *cell_start, *sorted;
    int *col, *in_cnt, *has_app, *first_app, *cand, *cstate, *cdec;
    double *mx, *my, *mg;
    // pair partial sums
    double *part;
    long long part_cap;      // doubles
    float4 *src32;           // packed FP32 sources (bulk form)
    // birth
    double *rhs_part;        // [chunks][P32][2]
    long long rhs_part_cap;
    double *R, *gamma;
    // birth far field: per-block expansion partials, near-source counts /
    // offsets, the near sources (x, y, G), the summed coefficients
    double *bf_part;
    int *bf_cnt;
    long long *bf_off;
    float4 *bf_near;
    double *bf_coef;
    // reductions
    double *red;             // [blocks][4]
    unsigned long long *box; // [blocks][4] bounding-box keys of the grids' first pass
    // neighbour-list grid (bulk form): radix-sort buffers, cells, sorted sources
    unsigned *key0, *key1;
    int *val0, *val1;
    int *cg_cnt, *cg_start;
    float4 *srt;
    int2 *items;             // (row, first sorted slot) of each target segment
    long long items_cap;
    int *cg_wide;            // sorted slots of the diffusion targets summed one warp each
    int *cg_huge;            // sorted slots of those summed one block each
    int *bk_mid, *bk_big;    // buckets of 17..128 / more than 128 elements (vx_bucket_order)
    // quadtree: counts and expansions of every level up to fmm_lmax
    int fmm_lmax;
    int *fmm_cnt, *fmm_start, *fmm_flags, *fmm_brute;
    int *fmm_sub_cnt, *fmm_sub_start;   // counts / starts of the level below the leaves
    int fmm_p;               // expansion terms the two arrays below were sized for
    double *fmm_M, *fmm_L;   // complex FP64 pairs, fmm_p per cell
    // tile words of the look-back scans (zeroed when allocated)
    unsigned long long *scan_tiles;
    long long scan_tiles_cap;
};

constexpr int VX_FMM_P = 16;              // default expansion terms of the quadtree FMM (vx_fmm.cu)
inline bool vx_fmm_order_ok(int p) { return p == 8 || p == 12 || p == 16 || p == 20; }

// Compaction chunk size (elements per scan chunk).
constexpr int VX_CHUNK = 2048;
constexpr int VX_RED_BLOCKS = 592;   // 4 x 148 SMs: fixed, so sums are deterministic
constexpr int VX_THREADS = 256;

// ---------------------------------------------------------------------------
// helpers
__host__ __device__ inline long long vx_ceil_div(long long a, long long b) { return (a + b - 1) / b; }
__host__ __device__ inline long long vx_round32(long long v) { return (v + 31) / 32 * 32; }
__host__ __device__ inline long long vx_pow2_ceil(long long n) {
    long long q = 1;
    while (q < n) q <<= 1;
    return q;
}

// Result-defining partitions.  Sums split into partitions (force sums,
// diffusion-grid mean, birth far field and right-hand side, pair-kernel
// source chunks) round differently for different splits, so every split is a
// function of the body's own count, taken on the device inside the kernel
// that uses it (never of the host's running bound of the count, which
// depends on when the host last looked): equal states give equal bits,
// whatever ran before or beside.  Grids stay the host's choice.
//
// SMs' worth of partitions for n sources: one per 2048 (n rounded up to a
// power of two), at least 4, at most the device's sms.
__host__ __device__ inline int vx_body_sms(long long n, int sms) {
    const long long q = vx_pow2_ceil(n) / 2048;
    return (int)(q < 4 ? 4 : (q > sms ? sms : q));
}
// Partitions of the force sums and of the diffusion-grid mean.
__host__ __device__ inline int vx_body_parts(long long n, int sms, int cap) {
    const int q = 4 * vx_body_sms(n, sms);
    return q < cap ? q : cap;
}
// Source chunks of the pair kernels: about 8 work items per SM over tiles
// of `tile` targets, 1 to 64.
__host__ __device__ inline int vx_ksplit(long long n, int tile, int sms) {
    const long long tiles = vx_ceil_div(n > 0 ? n : 1, tile);
    long long k = vx_ceil_div(8LL * sms, tiles);
    return (int)(k < 1 ? 1 : (k > 64 ? 64 : k));
}
// Source chunks of the birth right-hand side for P panels and n0 sources:
// enough (panel tile, chunk) items for every SM to hold several blocks,
// within the partial-sum buffer (sms * 4 chunks), one per 1024 sources (n0
// rounded up to a power of two) at most.
__host__ __device__ inline int vx_rhs_chunks(long long n0, int P, int sms) {
    const long long tiles = (P + 127) / 128;
    long long want = (long long)sms * 16 / tiles;
    if (want < 1) want = 1;
    if (want > (long long)sms * 4) want = (long long)sms * 4;
    long long bysrc = vx_ceil_div(vx_pow2_ceil(n0), 1024);
    if (bysrc < 1) bysrc = 1;
    return (int)(want < bysrc ? want : bysrc);
}

// Keep the 3 smallest squared distances (src/kernel.cu:941-953): the result
// is the same for any visiting order.
template <typename T>
__device__ __forceinline__ void vx_nn3_insert(T &d1, T &d2, T &d3, T r2) {
    if (d3 > r2) {
        d3 = r2;
        T t = fmin(d3, d2); d3 = fmax(d3, d2); d2 = t;
        t = fmin(d1, d2); d2 = fmax(d1, d2); d1 = t;
    }
}

// The same 3 smallest squared distances without a branch (FP32, five
// min/max per value): the new value moves each kept one up by at most one
// place, so the three updates read only the previous values.
__device__ __forceinline__ void vx_nn3_insert_bf(float &d1, float &d2, float &d3, float r2) {
    d3 = fminf(d3, fmaxf(d2, r2));
    d2 = fminf(d2, fmaxf(d1, r2));
    d1 = fminf(d1, r2);
}

// Packed FP32 pairs (PTX f32x2, sm_100): one instruction computes the same
// operation on two values held in one 64-bit register; the low half is the
// first.
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2_pack(float a, float b) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(f2 v, float &a, float &b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b) {
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// Monotonic unsigned key of a double (for atomicMin on signed values).
__device__ __forceinline__ unsigned long long vx_dkey(double v) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double vx_dunkey(unsigned long long k) {
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

// ---------------------------------------------------------------------------
// Grid-wide steps inside one launch.  Both helpers count a body's own blocks
// (nblk = the body's share of the launch), so they work the same in a single
// body's launch and in a launch over many bodies.
//
// vx_last_block: true in the block that arrives last of the body's nblk
// blocks; `ctr` counts arrivals and is left at zero.  Every block's global
// writes before its arrival are visible to that block, which reads them
// through L2 (__ldcg), never through an L1 line it may hold from before.
__device__ __forceinline__ bool vx_last_block(unsigned *ctr, unsigned nblk) {
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ctr, 1u);
        s_last = t == nblk - 1;
        if (s_last) atomicExch(ctr, 0u);
    }
    __syncthreads();
    const bool last = s_last != 0;
    if (last) __threadfence();
    return last;
}

// vx_scan_lookback: one-pass exclusive scan of non-negative int counts
// (decoupled look-back).  Blocks take tiles of VX_SCAN_T x PER consecutive
// counts in ticket order; each tile publishes its own sum, then walks back
// over its predecessors' published words (32 at a time, one per lane) adding
// their sums until it meets an inclusive prefix, and publishes its own.  A
// tile only waits on tiles whose tickets were taken before its own, so on
// blocks that are already running: the scan needs no co-residency.
//   tiles[t] = (stamp << 34) | (state << 32) | value, state 1 = the tile's
//   own sum, 2 = the inclusive prefix.  The stamp (1 .. 2^30 - 1) changes
//   with every scan of the body, so a word left by an earlier scan never
//   counts, nor does zeroed memory.
// A wait is bounded: after VX_SCAN_SPIN polls the scan sets VX_DERR_SCAN and
// takes the missing sums as 0 (the step then reports the flag).
// load(i) gives count i; store(i0, val, run) gets a thread's PER counts from
// i0 (PER-aligned; entries at or past `count` are 0) and the scan value at i0;
// total(sum) is called once, by one thread, with the sum of all counts.
// The block must have VX_SCAN_T threads.  Totals below 2^32.
constexpr int VX_SCAN_T = 256;
constexpr int VX_SCAN_SPIN = 1 << 20;

__device__ __forceinline__ void vx_scan_publish(unsigned long long *p, unsigned stamp, unsigned state,
                                                unsigned value) {
    const unsigned long long w = ((unsigned long long)stamp << 34) | ((unsigned long long)state << 32) | value;
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ unsigned long long vx_scan_peek(const unsigned long long *p) {
    unsigned long long w;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    return w;
}

template <int PER, typename Load, typename Store, typename Total>
__device__ void vx_scan_lookback(unsigned nblk, long long count, VxScalars *S, unsigned long long *tiles,
                                 Load load, Store store, Total total) {
    constexpr int NW = VX_SCAN_T / 32;
    constexpr long long TILE = (long long)VX_SCAN_T * PER;
    __shared__ long long s_tile;
    __shared__ unsigned s_warp[NW];
    __shared__ unsigned long long s_prefix;
    const unsigned stamp = 1u + S->scan_epoch % 0x3fffffffu;
    const long long ntiles = (count + TILE - 1) / TILE;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long t;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(&S->scan_ticket, 1u);
        __syncthreads();
        t = s_tile;
        if (t >= ntiles) break;
        const long long i0 = t * TILE + (long long)threadIdx.x * PER;
        unsigned val[PER];
        unsigned loc = 0;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            val[q] = i0 + q < count ? (unsigned)load(i0 + q) : 0u;
            loc += val[q];
        }
        unsigned inc = loc;   // inclusive scan over the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            unsigned wv = lane < NW ? s_warp[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned u = __shfl_up_sync(0xffffffffu, wv, o);
                if (lane >= o) wv += u;
            }
            if (lane < NW) s_warp[lane] = wv;
            const unsigned agg = __shfl_sync(0xffffffffu, wv, NW - 1);
            unsigned long long prefix = 0;
            if (t == 0) {
                if (lane == 0) vx_scan_publish(&tiles[0], stamp, 2u, agg);
            } else {
                if (lane == 0) vx_scan_publish(&tiles[t], stamp, 1u, agg);
                long long j = t - 1;
                int spins = 0;
                for (;;) {
                    const long long idx = j - lane;
                    const unsigned long long wd =
                        idx >= 0 ? vx_scan_peek(&tiles[idx]) : (((unsigned long long)stamp << 34) | (2ull << 32));
                    const unsigned st = (unsigned)(wd >> 32) & 3u;
                    const bool ready = (unsigned)(wd >> 34) == stamp && st != 0u;
                    if (!__all_sync(0xffffffffu, ready)) {
                        if (++spins > VX_SCAN_SPIN) {
                            if (lane == 0) atomicOr(&S->err, VX_DERR_SCAN);
                            break;
                        }
                        __nanosleep(32);
                        continue;
                    }
                    const unsigned pm = __ballot_sync(0xffffffffu, st == 2u);
                    const int stop = pm ? __ffs(pm) - 1 : 31;
                    unsigned long long v = lane <= stop ? (wd & 0xffffffffull) : 0ull;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    prefix += v;
                    if (pm) break;
                    j -= 32;
                }
                if (lane == 0) vx_scan_publish(&tiles[t], stamp, 2u, (unsigned)(prefix + agg));
            }
            if (lane == 0) s_prefix = prefix;
        }
        __syncthreads();
        const unsigned long long run = s_prefix + (warp ? s_warp[warp - 1] : 0u) + inc - loc;
        store(i0, val, (long long)run);
        if (t == ntiles - 1 && threadIdx.x == VX_SCAN_T - 1) total((long long)(run + loc));
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (ntiles == 0 && t == 0) total(0LL);
        __threadfence();
        if (atomicAdd(&S->scan_done, 1u) == nblk - 1) {
            S->scan_ticket = 0;
            S->scan_done = 0;
            S->scan_epoch += 1;
        }
    }
}

// Programmatic dependent launch (sm_90+): a kernel launched by vx_launch_pdl
// or vx_launch may be scheduled while its predecessor on the stream is still
// finishing, which hides the launch gap between the many short kernels of a
// step.  Every such kernel starts with VX_PDL_WAIT(), which returns once the
// predecessor has completed and its writes are visible; nothing is read or
// written before it.  (In a kernel launched the ordinary way the wait returns
// at once.)
#define VX_PDL_WAIT() asm volatile("griddepcontrol.wait;" ::: "memory")
template <typename... K, typename... A>
inline cudaError_t vx_launch_pdl(void (*kernel)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                 A &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}
#define VX_COUNT(L) do { if ((L).launches) ++*(L).launches; } while (0)

// ---------------------------------------------------------------------------
// Kernel bodies and the two ways they are launched.
//
// A step kernel is written as a device function `k_name_body(VxBlkB<T,B> vb,
// args...)` that uses vb.x / vb.n where a kernel would use blockIdx.x /
// gridDim.x (T, B: its launch bounds, 0 for none).  Two kernels run it:
//  * `k_name(args...)`, the body's own __global__ wrapper (vb = blockIdx.x,
//    gridDim.x): one body, arguments as kernel parameters;
//  * `k_many<body>(slot)`: many bodies in one launch.  The slot (device
//    memory) holds, per body, the first block of its range and its argument
//    pack; block b of the launch finds its body by a binary search over the
//    block ranges and runs the body with vb = (b - first, count).  Each body
//    sees exactly the blocks and arguments it would see launched alone, so
//    its results are the same.
template <int MAXT, int MINB>
struct VxBlkB {
    unsigned x, n;   // block index within this body's launch, blocks of this body's launch
};
using VxBlk = VxBlkB<0, 0>;
#define VX_DEVK __device__ __forceinline__

// Argument pack: a plain nested struct (the same layout in host and device
// code), built on the host and read on the device.
template <typename... A>
struct VxPack {};
template <typename H, typename... T>
struct VxPack<H, T...> {
    H h;
    VxPack<T...> t;
};
template <typename... A>
struct VxPackMake;
template <>
struct VxPackMake<> {
    static VxPack<> make() { return {}; }
};
template <typename H, typename... T>
struct VxPackMake<H, T...> {
    static VxPack<H, T...> make(const H &h, const T &...t) {
        VxPack<H, T...> p;
        p.h = h;
        p.t = VxPackMake<T...>::make(t...);
        return p;
    }
};
template <auto DEV, typename BK, typename... Done>
__device__ __forceinline__ void vx_apply(BK vb, const VxPack<> &, const Done &...d) {
    DEV(vb, d...);
}
template <auto DEV, typename BK, typename H, typename... T, typename... Done>
__device__ __forceinline__ void vx_apply(BK vb, const VxPack<H, T...> &p, const Done &...d) {
    vx_apply<DEV>(vb, p.t, d..., p.h);
}

// One multi-body launch (device memory): nb bodies, body i owns blocks
// [first[i], first[i+1]), its arguments at packs + i * stride.
struct VxSlot {
    int nb;
    int pad;
    long long stride;
    const int *first;
    const unsigned char *packs;
};

template <auto DEV, int MAXT, int MINB, typename... A>
__device__ __forceinline__ void vx_many_body(const VxSlot *sd) {
    VX_PDL_WAIT();
    const int nb = sd->nb;
    const int *first = sd->first;
    const unsigned bid = blockIdx.x;
    if (bid >= (unsigned)first[nb]) return;
    int lo = 0, hi = nb;
    while (hi - lo > 1) {
        const int m = (lo + hi) >> 1;
        if ((unsigned)first[m] <= bid) lo = m; else hi = m;
    }
    const VxBlkB<MAXT, MINB> vb{bid - (unsigned)first[lo], (unsigned)(first[lo + 1] - first[lo])};
    const VxPack<A...> &p = *reinterpret_cast<const VxPack<A...> *>(sd->packs + (long long)lo * sd->stride);
    vx_apply<DEV>(vb, p);
}
template <auto DEV, typename... A>
__global__ void k_many(const VxSlot *sd) { vx_many_body<DEV, 0, 0, A...>(sd); }
template <auto DEV, int MAXT, typename... A>
__global__ void __launch_bounds__(MAXT) k_many_t(const VxSlot *sd) { vx_many_body<DEV, MAXT, 0, A...>(sd); }
template <auto DEV, int MAXT, int MINB, typename... A>
__global__ void __launch_bounds__(MAXT, MINB) k_many_tb(const VxSlot *sd) {
    vx_many_body<DEV, MAXT, MINB, A...>(sd);
}

// A launch recorded instead of issued (building a multi-body step): the
// single-body kernel (identity), its multi-body kernel, the shape and the
// argument pack (bytes in the recorder's arena).
struct VxRecLaunch {
    const void *key;
    const void *many;
    dim3 grid, block;
    size_t smem;
    size_t off, size;
};
struct VxRecorder {
    std::vector<VxRecLaunch> launches;
    std::vector<unsigned char> arena;
    void add(const void *key, const void *many, dim3 grid, dim3 block, size_t smem, const void *pack,
             size_t size) {
        const size_t off = (arena.size() + 15) / 16 * 16;
        arena.resize(off + size);
        memcpy(arena.data() + off, pack, size);
        launches.push_back(VxRecLaunch{key, many, grid, block, smem, off, size});
    }
};

// Per-kernel device times: events around every launch, read back by kernel
// once the work has finished.
struct VxKernelTimer {
    struct Rec {
        const void *key;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get() {
        cudaEvent_t e = nullptr;
        if (!pool.empty()) {
            e = pool.back();
            pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    }
};

// ---------------------------------------------------------------------------
// Launch context: stream + launch counter shared by all stage launchers.
struct VxLaunch {
    cudaStream_t stream;
    long long *launches;   // host counter (may be null)
    // SMs the launch grids are sized for.  A step of a small body sizes them
    // for a share of the GPU that follows its source count (grid-stride
    // kernels: same results, fewer idle blocks, so the kernels of many
    // small bodies on concurrent streams overlap); full_sms (0: num_sms)
    // stays the device's count: the all-pairs sums' grid, and the SM count
    // the result-defining partitions are derived from on the device
    // (vx_body_parts, vx_ksplit, vx_rhs_chunks), so a body gets the same
    // results whatever share of the GPU it runs on.
    int num_sms;
    int full_sms = 0;
    // optional events recorded around the Biot-Savart and diffusion pair
    // kernels: [0,1] Biot-Savart, [2,3] diffusion (null: not recorded)
    cudaEvent_t pair_ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // recording instead of launching (multi-body steps), per-kernel timing
    VxRecorder *rec = nullptr;
    VxKernelTimer *kt = nullptr;
};
inline int vx_full_sms(const VxLaunch &L) { return L.full_sms > 0 ? L.full_sms : L.num_sms; }
#define VX_EV(L, k) do { if ((L).pair_ev[k] && !(L).rec) cudaEventRecord((L).pair_ev[k], (L).stream); } while (0)

// Launch kernel K (the __global__ wrapper of body DEV) for one body: with
// programmatic dependent launch, or recorded into L.rec, or bracketed by
// timing events into L.kt.
template <auto K, auto DEV, typename SigD = decltype(DEV)>
struct VxLauncher;
// The argument a body takes by reference (a large parameter struct) is
// stored and passed by value in the pack and to the single kernel; the
// body then reads the pack (or the kernel's parameter space) in place
// instead of holding a copy in registers.
template <typename T>
using vx_arg_t = std::remove_cv_t<std::remove_reference_t<T>>;
template <auto K, auto DEV, int MAXT, int MINB, typename... A0>
struct VxLauncher<K, DEV, void (*)(VxBlkB<MAXT, MINB>, A0...)> {
    static const void *many() {
        if constexpr (MAXT > 0 && MINB > 0) return (const void *)&k_many_tb<DEV, MAXT, MINB, vx_arg_t<A0>...>;
        else if constexpr (MAXT > 0) return (const void *)&k_many_t<DEV, MAXT, vx_arg_t<A0>...>;
        else return (const void *)&k_many<DEV, vx_arg_t<A0>...>;
    }
    template <typename... Args>
    static cudaError_t go(const VxLaunch &L, dim3 grid, dim3 block, size_t smem, Args &&...args) {
        if (L.launches) ++*L.launches;
        if (L.rec) {
            const VxPack<vx_arg_t<A0>...> p = VxPackMake<vx_arg_t<A0>...>::make(static_cast<vx_arg_t<A0>>(args)...);
            L.rec->add((const void *)K, many(), grid, block, smem, &p, sizeof(p));
            return cudaSuccess;
        }
        cudaEvent_t ea = nullptr, eb = nullptr;
        if (L.kt) {
            ea = L.kt->get();
            eb = L.kt->get();
            cudaEventRecord(ea, L.stream);
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = L.stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(&cfg, K, static_cast<vx_arg_t<A0>>(args)...);
        if (L.kt) {
            cudaEventRecord(eb, L.stream);
            L.kt->recs.push_back(VxKernelTimer::Rec{(const void *)K, ea, eb});
        }
        return e;
    }
};
template <auto K, auto DEV, typename... Args>
inline cudaError_t vx_launch(const VxLaunch &L, dim3 grid, dim3 block, size_t smem, Args &&...args) {
    return VxLauncher<K, DEV>::go(L, grid, block, smem, std::forward<Args>(args)...);
}


// Stage launchers (each returns the first CUDA error it saw).
cudaError_t vx_launch_step_begin(const VxLaunch &L, VxScalars *S);
// minv / minv_t: the inverted panel system and its transpose, stride P+1
cudaError_t vx_launch_birth(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                            VxWork &w, const vx_panel *pan, const double *minv, const double *minv_t,
                            int rhs_chunks);
cudaError_t vx_transpose_square(const VxLaunch &L, const double *A, double *At, long long nr);
cudaError_t vx_launch_velocity(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                               VxWork &w);
cudaError_t vx_launch_diffusion(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                                VxWork &w);
// wstart/widx: per wall cell, the panels that can act on a particle in the
// cell (CSR, ascending panel index); null: every panel is tested
cudaError_t vx_launch_wall(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                           const vx_panel *pan, const int *wstart = nullptr, const int *widx = nullptr);
cudaError_t vx_launch_advect(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                             VxWork &w, const vx_panel *pan,
                             const int *hstart = nullptr, const int *hidx = nullptr);
// count_step: the compaction of a whole step also advances the step index.
cudaError_t vx_launch_compact(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                              VxWork &w, bool count_step = false);
cudaError_t vx_launch_collapse(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                               VxWork &w, int pass, int n_col);
cudaError_t vx_launch_probe(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                            VxWork &w, const double *px, const double *py, long long pstride,
                            long long np, double *out_vx, double *out_vy, long long ostride,
                            int ksplit);
// Panel system on the device: L (P+1)^2 then Gauss-Jordan inverse.
// d_L_out (nullable) receives a copy of the influence matrix before elimination.
cudaError_t vx_build_matrix(const VxLaunch &L, const vx_panel *d_pan, int P, double *d_minv,
                            double *d_work, int *d_flag, double *d_L_out,
                            int robust = 0);
// robust: 0 the reference's pivot rule, 1 Gauss-Jordan with partial
// pivoting, 3 blocked LU with partial pivoting (vx_invert_lu).
// A (n x n) -> Inv = A^-1 by blocked LU with partial pivoting; A is
// overwritten, piv holds n ints; *flag set on a pivot below 1e-12.
cudaError_t vx_invert_lu(const VxLaunch &L, double *A, double *Inv, long long n, int *piv, int *flag);
cudaError_t vx_launch_birth_ld(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                               VxWork &w, const vx_panel *pan, const double *minv, long long ld,
                               int rhs_chunks);
cudaError_t vx_launch_step_end(const VxLaunch &L, VxScalars *S);
cudaError_t vx_launch_compact_skip(const VxLaunch &L, const VxParams &p, const VxView &v,
                                   VxScalars *S, VxWork &w, const int *skip, bool count_step = false);
void vx_params_from_conf(const vx_conf *c, const vx_panel *pan, int P, VxParams *p);
void vx_set_error(const char *fmt, ...);
void vx_keep_pool(int device);
void vx_trim_pool(int device);
vx_status vx_work_alloc(VxWork &w, std::vector<void *> &allocs, long long cap, int P32, int num_sms,
                        cudaStream_t stream = nullptr, int fmm_p = VX_FMM_P);
long long vx_work_bytes(long long cap, int P32, int num_sms, int fmm_p = VX_FMM_P);
// What the bucket order writes beside each element's final slot k (element
// j, bucket key b): nothing (mode 0), the quadtree's FP32 source (mode 1:
// position relative to the centre of leaf b / 4, G masked beyond n, the
// leaf's column), or the diffusion grid's (mode 2: position relative to the
// centre of cell b, G, d).  zero_counts: the bucket counts are left at zero
// instead of restored.
struct VxGather {
    int mode = 0;
    int zero_counts = 0;
    VxView v = {};
    const VxScalars *S = nullptr;
    float4 *srt = nullptr;
};
__device__ __forceinline__ void vx_gather_slot(const VxGather &gt, long long k, long long j, unsigned b) {
    const VxScalars *S = gt.S;
    const VxView &v = gt.v;
    if (gt.mode == 1) {
        const unsigned m = 1u << S->fL;
        const double h = S->fside / (double)m;
        const unsigned leaf = b >> 2, col = leaf % m, row = leaf / m;
        const double ccx = S->fx0 + ((double)col + 0.5) * h, ccy = S->fy0 + ((double)row + 0.5) * h;
        gt.srt[k] = make_float4((float)(v.x[j * v.ps] - ccx), (float)(v.y[j * v.ps] - ccy),
                                j < S->n ? (float)v.g[j * v.ps] : 0.0f, (float)col);
    } else if (gt.mode == 2) {
        const long long nx = S->cnx;
        const double ccx = S->cx0 + ((double)(b % nx) + 0.5) * S->ch, ccy = S->cy0 + ((double)(b / nx) + 0.5) * S->chy;
        gt.srt[k] = make_float4((float)(v.x[j * v.ps] - ccx), (float)(v.y[j * v.ps] - ccy), (float)v.g[j * v.ps],
                                (float)v.d[j]);
    }
}
// Stable order by bucket from bucket counts (used up, then restored or
// zeroed) and starts: (okey, oval) = keys and element indices in bucket
// order, elements of a bucket in index order, and the gather of gt at each
// element's final slot (vx_sort.cu).
cudaError_t vx_bucket_order(const VxLaunch &L, VxScalars *S, const long long *d_n, const long long *d_nbuckets,
                            const unsigned *key, const int *start, int *cnt, const long long *d_cnt_off,
                            unsigned *okey, int *oval, int *mid, int *big, int *scratch,
                            const VxGather &gt = VxGather());
int vx_fmm_max_level(long long cap);
long long vx_fmm_cells(int lmax);         // cells of all levels 0..lmax
constexpr int VX_BF_P = 48;          // terms of the birth far-field expansion
constexpr double VX_BF_RHO = 1.5;    // far-field sources lie beyond VX_BF_RHO body radii of its centre
constexpr int VX_BF_MAX_BLOCKS = 1024;
cudaError_t vx_launch_velocity_fmm(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                                   VxWork &w);
cudaError_t vx_launch_diffusion_cells(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                                      VxWork &w);
void vx_work_free(VxWork &w, std::vector<void *> &allocs, cudaStream_t stream = nullptr);

// Split factor so that (target tiles x source chunks) fills the GPU.
