// vx_cells.cu — uniform cell grid with a stable cell ordering, and the
// bulk-form vortex diffusion over it.
//
// The diffusive velocity (reference diffusion_Kernel, src/kernel.cu:985-1029)
// sums G_j exp(-r/d_i) terms; beyond r = c d_i (c = diff_cutoff, default 16)
// a term is below e^-c of its strength, and in a uniform cloud all of them
// together about (c+1) e^-c = 2e-6 of the sum's magnitude, so the bulk form
// sums only the pairs within c d_i.  Particles are binned into
// rectangular cells (their size tracks the mean 3-nearest distance), put in
// cell order with each cell's particles in index order (vx_bucket_order:
// every sum then has a fixed order), and gathered into one float4 per
// particle (x, y, G, d).
//
// Cells are c mean(d) / 16 wide and c mean(d) / 4 high: tall rows keep a
// warp's 32 targets on a short stretch of its row (the window is the
// targets' circles swept along that stretch), narrow columns let each row's
// range follow the circles closely (against square cells of c mean(d) / 8:
// 11 % fewer pair evaluations on the benchmark wake and on Gaussian clouds).
// Work item = one warp's 32 consecutive
// cell-sorted targets of one grid row.  The warp scans the rows within its
// largest cut-off radius; in each row it needs only the union of its targets'
// own column ranges (target i reaches the columns within sqrt(R_i^2 - gy^2)
// of its x, gy its vertical gap to the row: the window follows the targets'
// own cut-off circles, not the largest one), and those columns are one
// contiguous range of the sorted array, staged through the warp's shared
// memory 32 sources at a time.  A
// target whose radius exceeds CG_KCAP rows (an isolated vortex with a large
// d) would widen its warp's window for all 32 targets; unless the item's
// other targets are about as wide (the sparse outskirts of a cloud: the
// window, up to CG_KMAX rows, then serves them all) it is left out of the
// window and summed alone by one warp (k_diff_wide).  So is a target more
// than 64 d from its item's first cell (items of a row that crosses the body
// hold targets on both sides of it): the item's frame would cost it FP32
// digits (an error of order |offset| 6e-8 / d), its own cell's frame does
// not.  Each target is owned by one warp, so the velocity is updated in place
// with no partial sums.
#include "vx_internal.cuh"

constexpr int CG_T = 256;
constexpr int CG_W = 32;       // targets per work item (one warp)
#ifndef VX_CG_DIV_X
#define VX_CG_DIV_X 16
#endif
#ifndef VX_CG_DIV_Y
#define VX_CG_DIV_Y 4
#endif
constexpr int CG_DIV_X = VX_CG_DIV_X;    // cell width = cut-off radius at the mean d / CG_DIV_X
constexpr int CG_DIV_Y = VX_CG_DIV_Y;    // cell height = cut-off radius at the mean d / CG_DIV_Y
constexpr int CG_KCAP = 2 * CG_DIV_Y;    // a target's radius, in rows, that needs no company (twice the mean radius)
constexpr int CG_KMAX = 3 * CG_DIV_Y;    // widest window of a work item, in rows
#ifndef VX_DIFF_FRAME_D
#define VX_DIFF_FRAME_D 64.0f          // farthest a target may sit from its item's frame, in units of its d
#endif

// Start of the diffusion stage, one launch: per partition the bounding-box
// keys (into box[]) and the sum of d (into red[]); the block that finishes
// last combines them, resets the stage's counters and sizes the grid.  The
// sum of d is split into nparts fixed partitions whatever the grid (a
// partition past the last particle adds 0) and the partition sums are added
// in a fixed tree, so the mean spacing, and the grid built from it, do not
// depend on the launch's grid.  Cell width c * mean(d) / CG_DIV_X, height
// c * mean(d) / CG_DIV_Y, both grown until the grid fits cells_cap.
VX_DEVK void k_cg_prep_body(VxBlkB<CG_T, 0> vb, const VxView &v, VxScalars *S, double *red, unsigned long long *box,
                            int sms, double cutoff, long long cells_cap) {
    __shared__ unsigned long long sk[4][CG_T];
    __shared__ double sd[CG_T];
    const long long n = S->n;
    const int nparts = vx_body_parts(n, sms, VX_RED_BLOCKS);
    for (unsigned part = vb.x; part < (unsigned)nparts; part += vb.n) {
        if ((long long)part * blockDim.x >= n) {
            if (threadIdx.x == 0) red[part] = 0.0;
            continue;
        }
        unsigned long long k[4] = {~0ull, ~0ull, ~0ull, ~0ull};
        double dsum = 0.0;
        for (long long i = part * (long long)blockDim.x + threadIdx.x; i < n;
             i += (long long)nparts * blockDim.x) {
            const double x = v.x[i * v.ps], y = v.y[i * v.ps];
            k[0] = min(k[0], vx_dkey(x));
            k[1] = min(k[1], vx_dkey(-x));
            k[2] = min(k[2], vx_dkey(y));
            k[3] = min(k[3], vx_dkey(-y));
            dsum += v.d[i];
        }
        for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = k[q];
        sd[threadIdx.x] = dsum;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) {
                for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = min(sk[q][threadIdx.x], sk[q][threadIdx.x + o]);
                sd[threadIdx.x] += sd[threadIdx.x + o];
            }
            __syncthreads();
        }
        if (threadIdx.x < 4) box[4 * part + threadIdx.x] = sk[threadIdx.x][0];
        if (threadIdx.x == 0) red[part] = sd[0];
        __syncthreads();
    }
    if (!vx_last_block(&S->sync_ctr, vb.n)) return;
    unsigned long long k[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    double dpart = 0.0;
    for (int b = threadIdx.x; b < nparts; b += CG_T) {
        dpart += __ldcg(&red[b]);
        if ((long long)b * CG_T < n)
            for (int q = 0; q < 4; ++q) k[q] = min(k[q], __ldcg(&box[4 * b + q]));
    }
    for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = k[q];
    sd[threadIdx.x] = dpart;
    __syncthreads();
    for (int o = CG_T / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = min(sk[q][threadIdx.x], sk[q][threadIdx.x + o]);
            sd[threadIdx.x] += sd[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    S->cnwide = 0;
    S->cnhuge = 0;
    S->bk_nmid = S->bk_nbig = 0;
    S->cnitems = 0;
    if (n == 0) { S->cncells = 0; S->cnx = S->cny = 0; return; }
    const double dsum = sd[0];
    const double x0 = vx_dunkey(sk[0][0]), x1 = -vx_dunkey(sk[1][0]);
    const double y0 = vx_dunkey(sk[2][0]), y1 = -vx_dunkey(sk[3][0]);
    double hy = cutoff * (dsum / (double)n) / (double)CG_DIV_Y;
    if (!(hy > 0.0)) hy = 1e-3;
    double hx = hy * ((double)CG_DIV_Y / (double)CG_DIV_X);
    long long nx = -1, ny = -1;
    for (int it = 0; it < 400; ++it) {
        const double fx = floor((x1 - x0) / hx) + 1.0, fy = floor((y1 - y0) / hy) + 1.0;
        if (fx * fy <= (double)cells_cap) { nx = (long long)fx; ny = (long long)fy; break; }
        hx *= 1.25;
        hy *= 1.25;
    }
    if (nx < 0) { S->err |= VX_DERR_GRID; S->cncells = 0; return; }
    S->cx0 = x0; S->cy0 = y0; S->ch = hx; S->chy = hy;
    S->cnx = nx; S->cny = ny; S->cncells = nx * ny;
}
__global__ void __launch_bounds__(CG_T) k_cg_prep(VxView v, VxScalars *S, double *red, unsigned long long *box,
                                                  int sms, double cutoff, long long cells_cap) {
    VX_PDL_WAIT();
    k_cg_prep_body(VxBlkB<CG_T, 0>{blockIdx.x, gridDim.x}, v, S, red, box, sms, cutoff, cells_cap);
}

__device__ __forceinline__ long long cg_cell(const VxScalars *S, double x, double y) {
    long long cx = (long long)floor((x - S->cx0) / S->ch);
    long long cy = (long long)floor((y - S->cy0) / S->chy);
    cx = cx < 0 ? 0 : (cx >= S->cnx ? S->cnx - 1 : cx);
    cy = cy < 0 ? 0 : (cy >= S->cny ? S->cny - 1 : cy);
    return cy * S->cnx + cx;
}

// Cell of every particle, counted per cell (the counts are zero between
// steps: the bucket order leaves them at zero once the order is built).
VX_DEVK void k_cg_cellid_body(VxBlkB<0, 0> vb, const VxView &v, const VxScalars *S, unsigned *key, int *val, int *cnt) {
    const long long n = S->n;
    if (S->cncells == 0) return;
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        const long long c = cg_cell(S, v.x[i * v.ps], v.y[i * v.ps]);
        key[i] = (unsigned)c;
        val[i] = (int)i;
        atomicAdd(&cnt[c], 1);
    }
}
__global__ void k_cg_cellid(VxView v, const VxScalars *S, unsigned *key, int *val, int *cnt) {
    VX_PDL_WAIT();
    k_cg_cellid_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, key, val, cnt);
}

// Cell starts: one-pass scan of the counts, start[cncells] = n.
VX_DEVK void k_cg_scan_body(VxBlkB<VX_SCAN_T, 0> vb, VxScalars *S, const int *cnt, int *start,
                            unsigned long long *tiles) {
    const long long nc = S->cncells;
    vx_scan_lookback<VX_CHUNK / VX_SCAN_T>(
        vb.n, nc, S, tiles, [&](long long i) { return cnt[i]; },
        [&](long long i0, const unsigned *val, long long run) {
#pragma unroll
            for (int q = 0; q < VX_CHUNK / VX_SCAN_T; ++q) {
                if (i0 + q < nc) start[i0 + q] = (int)run;
                run += val[q];
            }
        },
        [&](long long) { start[nc] = (int)S->n; });
}
__global__ void __launch_bounds__(VX_SCAN_T) k_cg_scan(VxScalars *S, const int *cnt, int *start,
                                                       unsigned long long *tiles) {
    VX_PDL_WAIT();
    k_cg_scan_body(VxBlkB<VX_SCAN_T, 0>{blockIdx.x, gridDim.x}, S, cnt, start, tiles);
}

// Work items: each row's sorted range cut into segments of CG_W targets, as
// (row, first sorted slot); one-pass scan of the rows' item counts, one row
// per thread.
VX_DEVK void k_cg_items_body(VxBlkB<VX_SCAN_T, 0> vb, VxScalars *S, const int *start, int2 *items, long long items_cap,
                             unsigned long long *tiles) {
    const long long ny = S->cny, nx = S->cnx;
    vx_scan_lookback<1>(
        vb.n, ny, S, tiles,
        [&](long long r) { return (start[(r + 1) * nx] - start[r * nx] + CG_W - 1) / CG_W; },
        [&](long long r, const unsigned *val, long long run) {
            if (r >= ny) return;
            const int s0 = start[r * nx];
            for (unsigned q = 0; q < val[0]; ++q)
                if (run + q < items_cap) items[run + q] = make_int2((int)r, s0 + (int)q * CG_W);
        },
        [&](long long tot) {
            S->cnitems = tot <= items_cap ? tot : 0;
            if (tot > items_cap) S->err |= VX_DERR_GRID;
        });
}
__global__ void __launch_bounds__(VX_SCAN_T) k_cg_items(VxScalars *S, const int *start, int2 *items,
                                                        long long items_cap, unsigned long long *tiles) {
    VX_PDL_WAIT();
    k_cg_items_body(VxBlkB<VX_SCAN_T, 0>{blockIdx.x, gridDim.x}, S, start, items, items_cap, tiles);
}

__device__ __forceinline__ float vx_rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float vx_ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// One diffusion pair in FP32: target (relative position, 1/d folded into
// ndd = -log2(e)/d, R2 = (c d)^2) and source (relative position, G).  Pairs
// closer than 0.001 eps (the target itself) and beyond the cut-off add 0.
__device__ __forceinline__ void diff_pair(float tx, float ty, float R2, float ndd, float thr2, float4 s,
                                          float &s2x, float &s2y, float &s1) {
    const float dx = tx - s.x, dy = ty - s.y;
    const float r2 = fmaf(dx, dx, dy * dy);
    const bool use = (r2 > thr2) & (r2 < R2);
    const float rd = vx_rsqrt_approx(r2);
    const float e = vx_ex2_approx(r2 * rd * ndd);
    const float ge = use ? s.z * e : 0.0f;
    const float m = use ? ge * rd : 0.0f;
    s2x = fmaf(-m, dx, s2x);
    s2y = fmaf(-m, dy, s2y);
    s1 += ge;
}

// Cells of row offset dy that can hold a source within R of a target whose x
// (relative to the centre of column `ocol`) lies in [xlo, xhi]; false if none
// (cells hx wide and hy high).
__device__ __forceinline__ bool diff_window(int dy, float R, float xlo, float xhi, float hx, float hy,
                                            long long ocol, long long nx, long long &c0, long long &c1) {
    const float gy = (float)max(abs(dy) - 1, 0) * hy;   // vertical gap to that row
    const float hw2 = R * R - gy * gy;
    if (!(hw2 >= 0.0f)) return false;
    const float hw = sqrtf(hw2) * 1.0001f + 1e-3f * hx;  // margin over FP32 rounding
    c0 = max(ocol + (long long)floorf((xlo - hw) / hx + 0.5f), 0LL);
    c1 = min(ocol + (long long)floorf((xhi + hw) / hx + 0.5f), nx - 1);
    return c0 <= c1;
}

// Two diffusion pairs (one target, sources a and b of a staged slot).  Each
// pair needs one rsqrt and one 2^x, both on the MUFU pipe.  A degree-5
// polynomial 2^x on the FMA and integer pipes (round by adding 1.5 * 2^23,
// exponent added to the bit pattern) for one or both pairs of a step was
// measured 30 % slower on the whole kernel: those pipes then limit.
// 2^x of both halves on the FMA pipe (Cody-Waite reduction to the nearest
// integer k by adding 1.5 * 2^23, f = x - k in [-1/2, 1/2], then a degree-5
// polynomial p(f) ~ 2^f whose coefficients were fitted here for least
// relative error on [-1/2, 1/2] (7.5e-8; 2.3e-7 after FP32 rounding, as
// ex2.approx), and k added to p's exponent field by one integer
// multiply-add).  The halves are clamped to -125 first, so the exponent
// stays normal; for x that low the value is below 3e-38 either way.
__device__ __forceinline__ f2 diff_exp2_fma(float xa, float xb) {
    const f2 X = f2_pack(fmaxf(xa, -125.0f), fmaxf(xb, -125.0f));
    const f2 MAGIC = f2_pack(12582912.0f, 12582912.0f);
    const f2 T = f2_add(X, MAGIC);
    const f2 F = f2_sub(X, f2_sub(T, MAGIC));
    f2 P = f2_pack(1.3276184150891887e-3f, 1.3276184150891887e-3f);
    P = f2_fma(P, F, f2_pack(9.675540302623352e-3f, 9.675540302623352e-3f));
    P = f2_fma(P, F, f2_pack(5.5507141714826916e-2f, 5.5507141714826916e-2f));
    P = f2_fma(P, F, f2_pack(2.402211974958503e-1f, 2.402211974958503e-1f));
    P = f2_fma(P, F, f2_pack(6.931469665054077e-1f, 6.931469665054077e-1f));
    P = f2_fma(P, F, f2_pack(1.000000071646687f, 1.000000071646687f));
    float pa, pb, ta, tb;
    f2_unpack(P, pa, pb);
    f2_unpack(T, ta, tb);
    return f2_pack(__uint_as_float(__float_as_uint(pa) + (__float_as_uint(ta) << 23)),
                   __uint_as_float(__float_as_uint(pb) + (__float_as_uint(tb) << 23)));
}

#ifndef VX_DIFF_POLY_EVERY
#define VX_DIFF_POLY_EVERY 0   // every k-th pair step takes its 2^x on the FMA pipe (0: none)
#endif
// Two diffusion pairs (one target, sources a and b: SX = (x_a, x_b), SY,
// G likewise) in packed FP32.
template <bool POLY = false>
__device__ __forceinline__ void diff_pair2(f2 SX, f2 SY, f2 G, f2 TX, f2 TY, f2 NDD, float thr2, f2 &S2X, f2 &S2Y,
                                           f2 &S1) {
    const f2 DX = f2_sub(TX, SX), DY = f2_sub(TY, SY);
    const f2 R2 = f2_fma(DX, DX, f2_mul(DY, DY));
    float r2a, r2b;
    f2_unpack(R2, r2a, r2b);
    const f2 RD = f2_pack(vx_rsqrt_approx(fmaxf(r2a, thr2)), vx_rsqrt_approx(fmaxf(r2b, thr2)));
    const f2 ARG = f2_mul(f2_mul(R2, RD), NDD);
    float aa, ab;
    f2_unpack(ARG, aa, ab);
    float ea, eb;
    if (POLY) {
        f2_unpack(diff_exp2_fma(aa, ab), ea, eb);
    } else {
        ea = vx_ex2_approx(aa);
        eb = vx_ex2_approx(ab);
    }
    ea = r2a > thr2 ? ea : 0.0f;
    eb = r2b > thr2 ? eb : 0.0f;
    const f2 GE = f2_mul(G, f2_pack(ea, eb));
    const f2 M = f2_mul(GE, RD);
    S2X = f2_fma(M, DX, S2X);   // sums of +m dx, +m dy: negated by the caller
    S2Y = f2_fma(M, DY, S2Y);
    S1 = f2_add(S1, GE);
}

// Vortex diffusion over the cell grid (bulk form), one warp per work item of
// CG_W targets, one per lane; each step of the inner loop takes two sources
// in packed FP32 pairs.  Per pair: r^2, 1/r = rsqrt(max(r^2, thr^2)),
// e = 2^(-log2(e) r / d_i); the pair adds G e (I1) and G e (r_i - r_j) / r
// (I2) unless r <= 0.001 eps.  Every source of the warp's window enters (the
// window covers all sources within c d_i of each target; the ones beyond
// weigh below e^-c).
//
// The window is one column range per grid row.  The warp first lists the
// rows (a lane per row: first source, x and y offsets) with an exclusive scan
// of their lengths in shared memory, then walks the concatenated ranges in
// chunks of 32 sources, each lane finding its source's row by advancing a
// cursor over the scan; so a chunk spans row boundaries and only the last one
// of the window is padded (with G = 0, which adds exactly 0) — padding every
// row to 32 instead costs about 12 % more pair evaluations on the benchmark
// wake.  A source's x offset is its column minus the item's first column:
// the cell key minus (row * nx + first column), no division.
#ifndef VX_DIFF_UNROLL
#define VX_DIFF_UNROLL 16   // unrolled steps of the pair loop of k_diff_cells
#endif
#define VX_PRAGMA_(x) _Pragma(#x)
#define VX_UNROLL(n) VX_PRAGMA_(unroll n)
#ifndef VX_DIFF_MINB
#define VX_DIFF_MINB 2   // minimum resident blocks per SM requested for k_diff_cells
#endif
struct DiffRow {
    int j0;          // first source of the row's column range
    int pre;         // sources of the rows before it (the entry after the last row holds the total)
    unsigned base;   // row * nx + the item's first column (cell keys wrap modulo 2^32 alike)
    float oy;        // row offset * cell height
};
constexpr int DIFF_ROWS = 2 * CG_KMAX + 2;   // rows of the widest window, and the total
VX_DEVK void k_diff_cells_body(VxBlkB<CG_T, VX_DIFF_MINB> vb, const VxParams &p, const VxView &v, VxScalars *S,
                               const float4 *srt, const unsigned *skey,
                               const int *sorted, const int *start,
                               const int2 *items, int *wide) {
    // per warp 32 staged sources as x[32], y[32], G[32]: one 16-byte shared
    // load brings four sources' x (or y, or G)
    __shared__ float4 sx[CG_T / 4], sy[CG_T / 4], sg[CG_T / 4];
    __shared__ DiffRow srow[CG_T / 32][DIFF_ROWS];
    const int lane = threadIdx.x & 31;
    float4 *wx = sx + ((threadIdx.x & ~31) >> 2), *wy = sy + ((threadIdx.x & ~31) >> 2),
           *wg = sg + ((threadIdx.x & ~31) >> 2);
    DiffRow *wrow = srow[threadIdx.x >> 5];
    const long long nitems = S->cnitems, nx = S->cnx, ny = S->cny;
    const double hyd = S->chy;
    const float hx = (float)S->ch, hy = (float)hyd;
    const float cut = (float)p.diff_cutoff;
    const float thr2 = (float)(0.001 * p.eps) * (float)(0.001 * p.eps);
    const float log2e = 1.4426950408889634f;
    const long long wpb = CG_T / 32;
    unsigned long long pairs = 0;
    for (long long it = vb.x * wpb + (threadIdx.x >> 5); it < nitems; it += vb.n * wpb) {
        const int2 item = items[it];
        const long long row = item.x;
        const long long row_end = start[(row + 1) * nx];
        const long long last = min((long long)item.y + CG_W, row_end);
        const long long t = item.y + lane;
        const bool valid = t < last;
        float4 me = valid ? srt[t] : make_float4(0.f, 0.f, 0.f, 1.f);
        // coordinates relative to the centre of the item's first cell
        const unsigned key0 = skey[item.y];
        const long long ocol = (long long)key0 - row * nx;
        if (valid) me.x += (float)(int)(skey[t] - key0) * hx;   // as for the sources below
        const float R = cut * me.w;
        // a target far from the item's first cell (an item whose row crosses
        // the body holds targets on both sides of it) would lose FP32 digits
        // in the item's frame: beyond 64 d it is summed alone, in the frame
        // of its own cell, as the wide targets are
        const bool far_frame = valid && fabsf((float)(int)(skey[t] - key0)) * hx > VX_DIFF_FRAME_D * me.w;
        // a radius beyond CG_KCAP cells stays in the item (up to CG_KMAX) while
        // it is at most twice the item's mean: the window then serves targets
        // about as wide as itself; an outlier is summed alone
        float rsum = valid && !far_frame ? R : 0.0f;
        int rcnt = valid && !far_frame ? 1 : 0;
        for (int o = 16; o > 0; o >>= 1) {
            rsum += __shfl_xor_sync(0xffffffffu, rsum, o);
            rcnt += __shfl_xor_sync(0xffffffffu, rcnt, o);
        }
        const float rmean = rsum / (float)max(rcnt, 1);
        const bool too_wide = R > (float)CG_KMAX * hy || (R > (float)CG_KCAP * hy && R > 2.0f * rmean);
        const bool is_wide = valid && (too_wide || far_frame);
        if (is_wide) wide[atomicAdd(&S->cnwide, 1)] = (int)t;
        const bool act = valid && !is_wide;
        float rmax = act ? R : 0.0f;
        for (int o = 16; o > 0; o >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        const int nact = __popc(__ballot_sync(0xffffffffu, act));
        if (nact == 0) continue;
        const f2 TX = f2_pack(me.x, me.x), TY = f2_pack(me.y, me.y);
        const float nd = -log2e / me.w;
        const f2 NDD = f2_pack(nd, nd);
        // rows -kk..kk (kk <= CG_KMAX: a non-wide target's radius is at most CG_KMAX cells)
        const int kk = min((int)ceilf(rmax / hy), CG_KMAX);
        const int nrows = 2 * kk + 1;
        int total = 0;
        for (int r0 = 0; r0 < nrows; r0 += 32) {
            // columns of row r0 + lane: the union of the active targets' own
            // ranges in that row, each within sqrt(R^2 - gy^2) of the
            // target's x (gy its vertical gap to the row, less a margin over
            // FP32 rounding), column offsets from the item's first column
            int mc0 = 0, mc1 = -1;
            const int rn = min(32, nrows - r0);
            for (int q = 0; q < rn; ++q) {
                const float fy = (float)(r0 + q - kk) * hy;
                int lo = 0x7fffffff, hi = -0x7fffffff;
                if (act) {
                    const float gy = fmaxf(fmaxf(fy - 0.5f * hy - me.y, me.y - fy - 0.5f * hy) - 1e-3f * hy, 0.0f);
                    const float w2 = R * R - gy * gy;
                    if (w2 >= 0.0f) {
                        const float hw = sqrtf(w2) * 1.0001f + 1e-3f * hx;
                        lo = (int)floorf((me.x - hw) / hx + 0.5f);
                        hi = (int)floorf((me.x + hw) / hx + 0.5f);
                    }
                }
                lo = __reduce_min_sync(0xffffffffu, lo);
                hi = __reduce_max_sync(0xffffffffu, hi);
                if (lane == q) { mc0 = lo; mc1 = hi; }
            }
            const int r = r0 + lane;
            DiffRow e = {0, 0, 0u, 0.0f};
            int len = 0;
            if (r < nrows && mc0 <= mc1) {
                const int dy = r - kk;
                const long long rr = row + dy;
                const long long c0 = max(ocol + mc0, 0LL), c1 = min(ocol + (long long)mc1, nx - 1);
                if (rr >= 0 && rr < ny && c0 <= c1) {
                    e.j0 = start[rr * nx + c0];
                    len = start[rr * nx + c1 + 1] - e.j0;
                    e.base = (unsigned)(rr * nx + ocol);
                    e.oy = (float)((double)dy * hyd);
                }
            }
            int inc = len;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += u;
            }
            e.pre = total + inc - len;
            if (r < nrows) wrow[r] = e;
            total += __shfl_sync(0xffffffffu, inc, 31);
        }
        if (lane == 0) wrow[nrows].pre = total;
        __syncwarp();
        double I2x = 0.0, I2y = 0.0, I1 = 0.0;
        int rc = 0;   // this lane's row cursor (rows only advance as the chunks do)
        // the next chunk's source is loaded before the current chunk's pairs
        // run, so its L2 latency overlaps them
        float4 qn = make_float4(0.f, 0.f, 0.f, 0.f);
        unsigned kn = 0u;
        if (lane < total) {
            while (rc < nrows - 1 && wrow[rc + 1].pre <= lane) ++rc;
            const int j = wrow[rc].j0 + (lane - wrow[rc].pre);
            qn = srt[j];
            kn = skey[j];
        }
        for (int jt = 0; jt < total; jt += 32) {
            const int f = jt + lane;
            float x = 0.f, y = 0.f, gq = 0.f;
            if (f < total) {
                const DiffRow e = wrow[rc];
                x = qn.x + (float)(int)(kn - e.base) * hx;
                y = qn.y + e.oy;
                gq = qn.z;
            }
            reinterpret_cast<float *>(wx)[lane] = x;
            reinterpret_cast<float *>(wy)[lane] = y;
            reinterpret_cast<float *>(wg)[lane] = gq;
            __syncwarp();
            if (f + 32 < total) {
                while (rc < nrows - 1 && wrow[rc + 1].pre <= f + 32) ++rc;
                const int j = wrow[rc].j0 + (f + 32 - wrow[rc].pre);
                qn = srt[j];
                kn = skey[j];
            }
            f2 S2X = 0ull, S2Y = 0ull, S1 = 0ull;   // +0.0f in both halves
            // sources 2q and 2q + 1 are one pair step, in index order, so
            // each packed half sums the even (odd) sources in order
            VX_UNROLL(VX_DIFF_UNROLL)
            for (int q4 = 0; q4 < 8; ++q4) {
                const ulonglong2 X = *reinterpret_cast<const ulonglong2 *>(wx + q4);
                const ulonglong2 Y = *reinterpret_cast<const ulonglong2 *>(wy + q4);
                const ulonglong2 G = *reinterpret_cast<const ulonglong2 *>(wg + q4);
#pragma unroll
                for (int h2 = 0; h2 < 2; ++h2) {
                    const int q = 2 * q4 + h2;
                    const f2 SXp = h2 ? X.y : X.x, SYp = h2 ? Y.y : Y.x, Gp = h2 ? G.y : G.x;
                    if (VX_DIFF_POLY_EVERY > 0 && q % (VX_DIFF_POLY_EVERY > 0 ? VX_DIFF_POLY_EVERY : 1) ==
                                                      VX_DIFF_POLY_EVERY - 1)
                        diff_pair2<true>(SXp, SYp, Gp, TX, TY, NDD, thr2, S2X, S2Y, S1);
                    else
                        diff_pair2<false>(SXp, SYp, Gp, TX, TY, NDD, thr2, S2X, S2Y, S1);
                }
            }
            __syncwarp();
            float a, b;   // the two halves are added in FP32, then carried in FP64
            f2_unpack(S2X, a, b); I2x -= (double)(a + b);
            f2_unpack(S2Y, a, b); I2y -= (double)(a + b);
            f2_unpack(S1, a, b); I1 += (double)(a + b);
        }
        __syncwarp();   // the row list is rewritten by the next item
        pairs += (unsigned long long)total * (unsigned long long)nact;
        if (act && fabs(I1) > 1e-5) {
            const long long i = sorted[t];
            const double dd = (double)me.w;
            v.vx[i * v.vs] += -p.nu * I2x / (I1 * dd);
            v.vy[i * v.vs] += -p.nu * I2y / (I1 * dd);
        }
    }
    if (lane == 0 && pairs) atomicAdd(&S->pairs_diff, pairs);
}
__global__ void __launch_bounds__(CG_T, VX_DIFF_MINB) k_diff_cells(VxParams p, VxView v, VxScalars *S,
                                                                   const float4 *srt, const unsigned *skey,
                                                                   const int *sorted, const int *start,
                                                                   const int2 *items, int *wide) {
    VX_PDL_WAIT();
    k_diff_cells_body(VxBlkB<CG_T, VX_DIFF_MINB>{blockIdx.x, gridDim.x}, p, v, S, srt, skey, sorted, start, items, wide);
}

// Targets left out of the work items (radius beyond CG_KCAP rows).  Most
// have windows of about a thousand sources inside their circles (the sparse
// edge of a Gaussian cloud: about 1 % of its vortices): one warp each
// (k_diff_wide), the lanes taking the concatenated sources of 32 rows at a
// time.  A vortex whose window spans more than WIDE_ROWS rows each side (up
// to the whole grid: a vortex flung far from the cloud) is passed on to
// k_diff_huge: one block of WIDE_T threads each, its warps taking the rows in
// batches of equal height.  FP32 pair sums per lane over at most 16 sources,
// FP64 beyond (fixed order).
constexpr int WIDE_ROWS = 16 * CG_DIV_Y;   // sixteen mean cut-off radii
constexpr int WIDE_T = 512;

// Rows dy0 .. dy0 + nr - 1 (nr <= 32) of one target's window: lane l lists
// row dy0 + l (its column range clipped to the target's own circle) in the
// warp's row table (first source, offset in the concatenation, cell-key base,
// y offset; entry 32 holds the total), and the lanes take the concatenated
// sources 32 at a time, so rows of a few sources (the window of an isolated
// vortex is mostly empty rows and short ranges) do not idle the warp.  FP32
// sums per lane, carried into FP64 every 16 sources.
constexpr int WIDE_TABLE = 33;
__device__ __forceinline__ void wide_rows32(const VxScalars *S, const float4 *srt, const unsigned *skey,
                                            const int *start, const float4 me, long long row, long long ocol,
                                            float R, float R2, float ndd, float thr2, long long dy0, int nr,
                                            int lane, DiffRow *wrow, double &I2x, double &I2y, double &I1,
                                            unsigned long long &pairs) {
    const long long nx = S->cnx, ny = S->cny;
    const double hyd = S->chy;
    const float hx = (float)S->ch, hy = (float)hyd;
    DiffRow e = {0, 0, 0u, 0.0f};
    int len = 0;
    if (lane < nr) {
        const long long dy = dy0 + lane, rr = row + dy;
        long long c0, c1;
        if (rr >= 0 && rr < ny && diff_window((int)dy, R, me.x, me.x, hx, hy, ocol, nx, c0, c1)) {
            e.j0 = start[rr * nx + c0];
            len = start[rr * nx + c1 + 1] - e.j0;
            e.base = (unsigned)(rr * nx + ocol);   // cell keys wrap modulo 2^32 alike
            e.oy = (float)((double)dy * hyd);
        }
    }
    int inc = len;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    const int total = __shfl_sync(0xffffffffu, inc, 31);
    e.pre = inc - len;
    wrow[lane] = e;
    if (lane == 0) wrow[32].pre = total;
    __syncwarp();
    pairs += (unsigned long long)total;
    float s2x = 0.f, s2y = 0.f, s1 = 0.f;
    int rc = 0, cnt = 0;
    for (int f = lane; f < total; f += 32) {
        while (wrow[rc + 1].pre <= f) ++rc;   // entry 32 (the total) stops it
        const DiffRow r = wrow[rc];
        const int j = r.j0 + (f - r.pre);
        float4 q = srt[j];
        q.x += (float)(int)(skey[j] - r.base) * hx;
        q.y += r.oy;
        diff_pair(me.x, me.y, R2, ndd, thr2, q, s2x, s2y, s1);
        if (++cnt == 16) {
            I2x += (double)s2x; I2y += (double)s2y; I1 += (double)s1;
            s2x = s2y = s1 = 0.f;
            cnt = 0;
        }
    }
    I2x += (double)s2x; I2y += (double)s2y; I1 += (double)s1;
    __syncwarp();   // the table is rewritten by the next call
}

__device__ __forceinline__ void wide_apply(const VxParams &p, VxView v, const int *sorted, long long t, float d,
                                           double I2x, double I2y, double I1) {
    if (fabs(I1) > 1e-5) {
        const long long i = sorted[t];
        const double dd = (double)d;
        v.vx[i * v.vs] += -p.nu * I2x / (I1 * dd);
        v.vy[i * v.vs] += -p.nu * I2y / (I1 * dd);
    }
}

VX_DEVK void k_diff_wide_body(VxBlkB<CG_T, 0> vb, const VxParams &p, const VxView &v, VxScalars *S, const float4 *srt,
                              const unsigned *skey, const int *sorted, const int *start,
                              const int *wide, int *huge) {
    __shared__ DiffRow stab[CG_T / 32][WIDE_TABLE];
    const int lane = threadIdx.x & 31;
    DiffRow *wrow = stab[threadIdx.x >> 5];
    const long long nx = S->cnx, ny = S->cny;
    const float hy = (float)S->chy;
    const unsigned unx = (unsigned)nx;
    const float cut = (float)p.diff_cutoff;
    const float thr2 = (float)(0.001 * p.eps) * (float)(0.001 * p.eps);
    const float log2e = 1.4426950408889634f;
    const int nw = S->cnwide;
    const int warps = (vb.n * blockDim.x) >> 5;
    unsigned long long pairs = 0;
    for (int f = (vb.x * blockDim.x + threadIdx.x) >> 5; f < nw; f += warps) {
        const long long t = wide[f];
        const float4 me = srt[t];
        const long long ocol = (long long)(skey[t] % unx), row = (long long)(skey[t] / unx);
        const float R = cut * me.w, R2 = R * R, ndd = -log2e / me.w;
        const long long kk = min((long long)ceilf(R / hy), ny);
        if (kk > WIDE_ROWS) {
            if (lane == 0) huge[atomicAdd(&S->cnhuge, 1)] = (int)t;
            continue;
        }
        double I2x = 0.0, I2y = 0.0, I1 = 0.0;
        for (long long dy0 = -kk; dy0 <= kk; dy0 += 32)
            wide_rows32(S, srt, skey, start, me, row, ocol, R, R2, ndd, thr2, dy0, (int)min(32LL, kk - dy0 + 1),
                        lane, wrow, I2x, I2y, I1, pairs);
        for (int o = 16; o > 0; o >>= 1) {
            I2x += __shfl_xor_sync(0xffffffffu, I2x, o);
            I2y += __shfl_xor_sync(0xffffffffu, I2y, o);
            I1 += __shfl_xor_sync(0xffffffffu, I1, o);
        }
        if (lane == 0) wide_apply(p, v, sorted, t, me.w, I2x, I2y, I1);
    }
    if (lane == 0 && pairs) atomicAdd(&S->pairs_diff, pairs);   // every lane counted the same pairs
}
__global__ void __launch_bounds__(CG_T) k_diff_wide(VxParams p, VxView v, VxScalars *S, const float4 *srt,
                                                    const unsigned *skey, const int *sorted, const int *start,
                                                    const int *wide, int *huge) {
    VX_PDL_WAIT();
    k_diff_wide_body(VxBlkB<CG_T, 0>{blockIdx.x, gridDim.x}, p, v, S, srt, skey, sorted, start, wide, huge);
}

VX_DEVK void k_diff_huge_body(VxBlkB<WIDE_T, 0> vb, const VxParams &p, const VxView &v, VxScalars *S, const float4 *srt,
                              const unsigned *skey, const int *sorted, const int *start,
                              const int *huge) {
    constexpr int NWARP = WIDE_T / 32;
    __shared__ double sred[3][NWARP];
    __shared__ DiffRow stab[NWARP][WIDE_TABLE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long nx = S->cnx, ny = S->cny;
    const float hy = (float)S->chy;
    const unsigned unx = (unsigned)nx;
    const float cut = (float)p.diff_cutoff;
    const float thr2 = (float)(0.001 * p.eps) * (float)(0.001 * p.eps);
    const float log2e = 1.4426950408889634f;
    const int nh = S->cnhuge;
    unsigned long long pairs = 0;
    for (int f = vb.x; f < nh; f += vb.n) {
        const long long t = huge[f];
        const float4 me = srt[t];
        const long long ocol = (long long)(skey[t] % unx), row = (long long)(skey[t] / unx);
        const float R = cut * me.w, R2 = R * R, ndd = -log2e / me.w;
        const long long kk = min((long long)ceilf(R / hy), ny);
        double I2x = 0.0, I2y = 0.0, I1 = 0.0;
        // every warp takes batches of rpw rows (all warps busy whatever the window's height)
        const long long rpw = min(32LL, (2 * kk + 1 + NWARP - 1) / NWARP);
        for (long long dy0 = -kk + rpw * warp; dy0 <= kk; dy0 += rpw * NWARP)
            wide_rows32(S, srt, skey, start, me, row, ocol, R, R2, ndd, thr2, dy0, (int)min(rpw, kk - dy0 + 1),
                        lane, stab[warp], I2x, I2y, I1, pairs);
        for (int o = 16; o > 0; o >>= 1) {
            I2x += __shfl_xor_sync(0xffffffffu, I2x, o);
            I2y += __shfl_xor_sync(0xffffffffu, I2y, o);
            I1 += __shfl_xor_sync(0xffffffffu, I1, o);
        }
        if (lane == 0) { sred[0][warp] = I2x; sred[1][warp] = I2y; sred[2][warp] = I1; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0, c = 0.0;
            for (int w = 0; w < NWARP; ++w) { a += sred[0][w]; b += sred[1][w]; c += sred[2][w]; }
            wide_apply(p, v, sorted, t, me.w, a, b, c);
        }
        __syncthreads();
    }
    if (lane == 0 && pairs) atomicAdd(&S->pairs_diff, pairs);   // a warp's lanes counted the same rows
}
__global__ void __launch_bounds__(WIDE_T) k_diff_huge(VxParams p, VxView v, VxScalars *S, const float4 *srt,
                                                      const unsigned *skey, const int *sorted, const int *start,
                                                      const int *huge) {
    VX_PDL_WAIT();
    k_diff_huge_body(VxBlkB<WIDE_T, 0>{blockIdx.x, gridDim.x}, p, v, S, srt, skey, sorted, start, huge);
}

// Build the grid and run the bulk diffusion (scratch from w).
cudaError_t vx_launch_diffusion_cells(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                                      VxWork &w) {
    const int grid = L.num_sms * 4;
    // partitions of the mean spacing follow the body's count on the device
    // (vx_body_parts), the grid the SMs this launch is given
    vx_launch<k_cg_prep, k_cg_prep_body>(L, std::min(VX_RED_BLOCKS, L.num_sms * 4), CG_T, 0, v, S, w.red, w.box,
                                         vx_full_sms(L), p.diff_cutoff, w.cells_cap);
    vx_launch<k_cg_cellid, k_cg_cellid_body>(L, grid, CG_T, 0, v, S, w.key0, w.val0, w.cg_cnt);
    vx_launch<k_cg_scan, k_cg_scan_body>(L, grid, VX_SCAN_T, 0, S, w.cg_cnt, w.cg_start, w.scan_tiles);

    // cell order: each cell's vortices in index order (a stable sort by cell),
    // the FP32 sources gathered at their slots on the way; the cell counts
    // are left at zero for the next step's count
    VxGather gt;
    gt.mode = 2;
    gt.zero_counts = 1;
    gt.v = v;
    gt.S = S;
    gt.srt = w.srt;
    vx_bucket_order(L, S, &S->n, &S->cncells, w.key0, w.cg_start, w.cg_cnt, nullptr, w.key1, w.val1, w.bk_mid, w.bk_big,
                    w.val0, gt);
    const unsigned *skey = w.key1;
    const int *sorted = w.val1;
    vx_launch<k_cg_items, k_cg_items_body>(L, grid, VX_SCAN_T, 0, S, w.cg_start, w.items, w.items_cap, w.scan_tiles);

    VX_EV(L, 2);
    vx_launch<k_diff_cells, k_diff_cells_body>(L, L.num_sms * 8, CG_T, 0, p, v, S, w.srt, skey, sorted, w.cg_start, w.items, w.cg_wide);

    vx_launch<k_diff_wide, k_diff_wide_body>(L, L.num_sms * 4, CG_T, 0, p, v, S, w.srt, skey, sorted, w.cg_start, w.cg_wide, w.cg_huge);

    vx_launch<k_diff_huge, k_diff_huge_body>(L, L.num_sms * 2, WIDE_T, 0, p, v, S, w.srt, skey, sorted, w.cg_start, w.cg_huge);

    VX_EV(L, 3);
    return cudaGetLastError();
}
