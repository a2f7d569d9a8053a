// vx_fmm.cu — bulk-form Biot-Savart velocity by a quadtree fast multipole
// method, with the mean 3-nearest distance from the near field.
//
// Replaces, for the bulk form, the direct O(N^2) sum of the reference's
// shared_Kernel (src/kernel.cu:875-983); the reference's own tree
// (src/kernel.cu:78-763, src/unit_1.cu:686-960) is off in every shipped
// configuration, so the direct sum is the parity target.
//
// With z = x + i y, the conjugate velocity induced by vortices j is
//   u - i v = 1/(2 pi i) sum_j G_j / (z - z_j)         (|z - z_j| >= eps)
// and the core smoothing max(r^2, eps^2) only acts closer than eps.  The
// leaves are at least eps wide, so every pair that goes through expansions
// is farther apart than eps and sees the plain Cauchy kernel.
//
// Tree: uniform levels 0..L over the particles' square bounding box, dense
// row-major cell arrays per level.  Expansions in FP64, scaled by the cell
// side s (w = (z - c)/s keeps every coefficient O(1)) and by factorials:
//   multipole  B_k  = (1/k!) sum_j G_j w_j^k               (P2M)
//   field      f(z) = sum_k k! B_k s^k (z - c)^-(k+1)
//   local      f(z) = sum_l A_l u^l / l!,  u = (z - c)/s      (M2L, L2L, L2P)
// M2L between two cells of one level with integer offset t = (c_T - c_S)/s
// is then a Hankel product (no binomials):
//   A_l += ((-1)^l / s) sum_k B_k H_{k+l},  H_j = j! t^-(j+1),
// and the shifts M2M / L2L use E_p = d^p / p! for the child offset d:
//   B_k(parent) = sum_m E_{k-m} 2^-m B_m(child),
//   A_l(child)  = 2^-l sum_{j>=l} E_{j-l} A_j(parent).
// Interaction list: children of the parent's 3x3 neighbours that are not
// neighbours of the cell.  Near field: the 3x3 leaves around a target's leaf,
// direct FP32 with the core smoothing; the 3 nearest come from there and are
// exact when the third distance is below the leaf side (nothing outside the
// 3x3 block can be closer); the few targets that fail the test are redone by
// a ring search over the leaves.
#include <algorithm>

#include "vx_internal.cuh"

// Expansion terms P: a template parameter of the kernels that hold
// expansions, one of VX_FMM_ORDERS (run-time choice, VxParams::fmm_p).
constexpr int FMM_PMAX = 20;
constexpr int FMM_T = 256;
constexpr int FMM_W = 32;        // targets per near-field work item (one warp)

struct cplx {
    double r, i;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.r * s, a.i * s}; }
__device__ __forceinline__ cplx cinv(cplx a) {
    const double d = a.r * a.r + a.i * a.i;
    return {a.r / d, -a.i / d};
}

__host__ __device__ inline long long fmm_level_off(int l) { return ((1LL << (2 * l)) - 1) / 3; }

// 1/k for k = 1..FMM_PMAX (folded at compile time)
__constant__ double c_fmm_inv[FMM_PMAX + 1] = {0.0,      1.0,      1.0 / 2,  1.0 / 3,  1.0 / 4,  1.0 / 5,
                                               1.0 / 6,  1.0 / 7,  1.0 / 8,  1.0 / 9,  1.0 / 10, 1.0 / 11,
                                               1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17,
                                               1.0 / 18, 1.0 / 19, 1.0 / 20};
// M2L blocks stage their tables in dynamic shared memory (over 48 KB at P = 20)
extern __shared__ __align__(16) unsigned char vx_fmm_dyn[];

// ---------------------------------------------------------------------------
// Start of the velocity stage, one launch: the count arrays zeroed to their
// capacity, the bounding box (per-block keys into part[], combined by the
// last block), then, in the last block, the stage's counters and the tree:
// square box, depth L = ceil(log4(n / leaf)) within [2, Lmax], deepened while
// the leaf occupancy a vortex sees would reach 2 leaf, reduced until the leaf
// side is at least eps.  The occupancy a vortex sees is sum(c^2) / n over the
// cells; the last build measured it over its quarter-leaf cells (k_fmm_leafid),
// and at the density it implies, a leaf of side a holds rho a^2.  A clustered
// cloud (a dense wall layer, a Gaussian core) then gets the depth its dense
// part needs rather than the one its bounding box implies; a uniform one
// keeps ceil(log4(n / leaf)).  The first build of a body (no measurement yet)
// uses the box rule alone.  Deepening stops one level above a build whose
// 3-nearest pass left more than 0.5 % of its targets to the exact search.
VX_DEVK void k_fmm_prep_body(VxBlkB<FMM_T, 0> vb, const VxView &v, VxScalars *S, double eps, int Lmax, int leaf, int *cnt,
                             long long ncnt, int *subcnt, long long nsub, unsigned long long *part) {
    __shared__ unsigned long long sk[4][FMM_T];
    const long long n = S->n;
    for (long long c = vb.x * (long long)blockDim.x + threadIdx.x; c < ncnt + nsub;
         c += (long long)vb.n * blockDim.x) {
        if (c < ncnt) cnt[c] = 0;
        else subcnt[c - ncnt] = 0;
    }
    unsigned long long k[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        const double x = v.x[i * v.ps], y = v.y[i * v.ps];
        k[0] = min(k[0], vx_dkey(x)); k[1] = min(k[1], vx_dkey(-x));
        k[2] = min(k[2], vx_dkey(y)); k[3] = min(k[3], vx_dkey(-y));
    }
    for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = k[q];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = min(sk[q][threadIdx.x], sk[q][threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x < 4) part[4 * vb.x + threadIdx.x] = sk[threadIdx.x][0];
    if (!vx_last_block(&S->sync_ctr, vb.n)) return;
    for (int q = 0; q < 4; ++q) k[q] = ~0ull;
    for (unsigned b = threadIdx.x; b < vb.n; b += blockDim.x)
        for (int q = 0; q < 4; ++q) k[q] = min(k[q], __ldcg(&part[4 * b + q]));
    for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = k[q];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 4; ++q) sk[q][threadIdx.x] = min(sk[q][threadIdx.x], sk[q][threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    // the last build's quarter-cell occupancy, sources, box, depth and the
    // targets its 3-nearest pass left to the exact search
    const unsigned long long q2 = S->fsq;
    const long long s_prev = S->fs;
    const double side_prev = S->fside;
    const int L_prev = S->fL;
    const long long flags_prev = S->fnflag;
    S->fsq = 0;
    S->fnflag = 0;
    S->fnbrute = 0;
    S->bk_nmid = S->bk_nbig = 0;
    const double x0 = vx_dunkey(sk[0][0]), x1 = -vx_dunkey(sk[1][0]);
    const double y0 = vx_dunkey(sk[2][0]), y1 = -vx_dunkey(sk[3][0]);
    double side = fmax(x1 - x0, y1 - y0);
    side = side * (1.0 + 1e-9) + 1e-12;
    // the depth's ceiling follows the count, not the store's capacity (the
    // arrays are sized for the capacity's ceiling, which is never lower), so
    // the tree does not depend on when the store grew
    int Lc = 2;
    while (Lc < 10 && (double)(1LL << (2 * Lc)) * 8.0 < (double)vx_round32(n)) ++Lc;
    Lmax = min(Lmax, Lc);
    int L = 2;
    while (L < Lmax && (double)(1LL << (2 * L)) * (double)leaf < (double)n) ++L;
    // a tree deep enough for a dense region leaves the sparse rest of the
    // cloud with quarters too small for their 3 nearest: once a build left
    // more than 0.5 % of its targets to the exact search, the depth rule
    // deepens no further than one level above that build, from then on
    if (q2 > 0 && s_prev > 0 && L_prev >= 3 && flags_prev * 200 > s_prev)
        S->fLcap = S->fLcap > 0 ? min(S->fLcap, L_prev - 1) : L_prev - 1;
    const int Ldeep = S->fLcap > 0 ? max(L, min(Lmax, S->fLcap)) : Lmax;
    if (q2 > 0 && s_prev > 0 && side_prev > 0.0 && L_prev >= 1) {
        const double qa = side_prev / (double)(2LL << L_prev);                      // quarter side then
        const double rho = (double)q2 / (double)s_prev / (qa * qa) * ((double)vx_round32(n) / (double)s_prev);
        while (L < Ldeep) {
            const double a = side / (double)(1LL << L);
            if (rho * a * a < 2.0 * (double)leaf) break;
            ++L;
        }
    }
    while (L > 2 && side / (double)(1LL << L) < eps) --L;
    // a box smaller than 4 eps: no pair may use an expansion, all near field
    if (side / 4.0 < eps) L = 1;
    S->fx0 = 0.5 * (x0 + x1) - 0.5 * side;
    S->fy0 = 0.5 * (y0 + y1) - 0.5 * side;
    S->fside = side;
    S->fL = L;
    S->fcnt_off = fmm_level_off(L);
    S->fnleaves = 1LL << (2 * L);
    S->fnsub = 4 * S->fnleaves;
    S->fs = vx_round32(n);   // sources include the round-32 padding (3-nearest)
}
__global__ void __launch_bounds__(FMM_T) k_fmm_prep(VxView v, VxScalars *S, double eps, int Lmax, int leaf, int *cnt,
                                                    long long ncnt, int *subcnt, long long nsub,
                                                    unsigned long long *part) {
    VX_PDL_WAIT();
    k_fmm_prep_body(VxBlkB<FMM_T, 0>{blockIdx.x, gridDim.x}, v, S, eps, Lmax, leaf, cnt, ncnt, subcnt, nsub, part);
}

__device__ __forceinline__ long long fmm_leaf(const VxScalars *S, double x, double y) {
    const long long m = 1LL << S->fL;
    const double h = S->fside / (double)m;
    long long ix = (long long)floor((x - S->fx0) / h), iy = (long long)floor((y - S->fy0) / h);
    ix = ix < 0 ? 0 : (ix >= m ? m - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= m ? m - 1 : iy);
    return iy * m + ix;
}

// Cell of the level below the leaves of every source slot [0, s), as the
// key 4 leaf + child (child = 2 (row & 1) + (column & 1) at that level), so
// that sorting by it keeps each leaf's sources contiguous, its four quarters
// one after the other; counts per key.  The leaf of the key is the one
// fmm_leaf gives (x / (h/2) is exactly 2 (x / h)).
__device__ __forceinline__ unsigned fmm_subkey(const VxScalars *S, double x, double y) {
    const long long m2 = 2LL << S->fL;
    const double h2 = 0.5 * (S->fside / (double)(m2 >> 1));
    long long ix = (long long)floor((x - S->fx0) / h2), iy = (long long)floor((y - S->fy0) / h2);
    ix = ix < 0 ? 0 : (ix >= m2 ? m2 - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= m2 ? m2 - 1 : iy);
    const long long leaf = (iy >> 1) * (m2 >> 1) + (ix >> 1);
    return (unsigned)(4 * leaf + 2 * (iy & 1) + (ix & 1));
}

// The sum of count^2 over the cells (the next build's depth rule) comes from
// the same increments: a cell's count going from c to c + 1 adds 2 c + 1.
VX_DEVK void k_fmm_leafid_body(VxBlkB<0, 0> vb, const VxView &v, VxScalars *S, unsigned *key, int *val, int *subcnt) {
    const long long s = S->fs;
    unsigned long long sq = 0;
    for (long long j = vb.x * (long long)blockDim.x + threadIdx.x; j < s;
         j += (long long)vb.n * blockDim.x) {
        const unsigned k = fmm_subkey(S, v.x[j * v.ps], v.y[j * v.ps]);
        key[j] = k;
        val[j] = (int)j;
        sq += 2ull * (unsigned)atomicAdd(&subcnt[k], 1) + 1ull;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0 && sq) atomicAdd(&S->fsq, sq);
}
__global__ void k_fmm_leafid(VxView v, VxScalars *S, unsigned *key, int *val, int *subcnt) {
    VX_PDL_WAIT();
    k_fmm_leafid_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, key, val, subcnt);
}

// Starts of the quarters (one-pass scan of their counts), and with them the
// leaf counts (the tree's leaf level: the sum of a leaf's four quarters) and
// the leaf starts (its first quarter's); both end with the sources' total.
VX_DEVK void k_fmm_scan_body(VxBlkB<VX_SCAN_T, 0> vb, VxScalars *S, const int *subcnt, int *substart, int *cnt,
                             int *start, unsigned long long *tiles) {
    constexpr int PER = VX_CHUNK / VX_SCAN_T;   // a multiple of 4: a thread holds whole leaves
    const long long len = S->fnsub, nl = S->fnleaves;
    int *leafcnt = cnt + fmm_level_off(S->fL);
    vx_scan_lookback<PER>(
        vb.n, len, S, tiles, [&](long long i) { return subcnt[i]; },
        [&](long long i0, const unsigned *val, long long run) {
#pragma unroll
            for (int q = 0; q < PER; q += 4) {
                if (i0 + q >= len) break;
                const long long leaf = (i0 + q) >> 2;
                leafcnt[leaf] = (int)(val[q] + val[q + 1] + val[q + 2] + val[q + 3]);
                start[leaf] = (int)run;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    substart[i0 + q + e] = (int)run;
                    run += val[q + e];
                }
            }
        },
        [&](long long) {
            substart[len] = (int)S->fs;
            start[nl] = (int)S->fs;
        });
}
__global__ void __launch_bounds__(VX_SCAN_T) k_fmm_scan(VxScalars *S, const int *subcnt, int *substart, int *cnt,
                                                        int *start, unsigned long long *tiles) {
    VX_PDL_WAIT();
    k_fmm_scan_body(VxBlkB<VX_SCAN_T, 0>{blockIdx.x, gridDim.x}, S, subcnt, substart, cnt, start, tiles);
}

// Shift table shared by M2M and L2L, built per block in shared memory:
// E[q][p] = d_q^p / p! for the child offsets d_q = (+-1 +- i)/4 (in units of
// the parent side), q = (dy > 0) * 2 + (dx > 0).
template <int P>
__device__ __forceinline__ void fmm_shift_table(cplx (*se)[P]) {
    if (threadIdx.x < 4) {
        const int q = threadIdx.x;
        const cplx dd = {(q & 1) ? 0.25 : -0.25, (q >> 1) ? 0.25 : -0.25};
        cplx pw = {1.0, 0.0};
        for (int p = 0; p < P; ++p) { se[q][p] = pw; pw = cscale(cmul(pw, dd), c_fmm_inv[p + 1]); }
    }
}

// P2M of leaf c (level L, m leaves a side), by one warp: each lane expands
// its own vortices (FP64 positions), then a fixed butterfly sums the lanes.
// An empty leaf is not written (nothing reads its expansion).
template <int P>
__device__ __forceinline__ void fmm_p2m_leaf(const VxView &v, const VxScalars *S, const int *start,
                                             const int *sorted, cplx *ML, long long c, long long m, int lane) {
    const int j0 = start[c], j1 = start[c + 1];
    if (j0 == j1) return;
    const long long n = S->n;
    const double h = S->fside / (double)m;
    cplx b[P];
#pragma unroll
    for (int k = 0; k < P; ++k) b[k] = {0.0, 0.0};
    const double cx = S->fx0 + ((double)(c % m) + 0.5) * h, cy = S->fy0 + ((double)(c / m) + 0.5) * h;
    for (int q = j0 + lane; q < j1; q += 32) {
        const long long j = sorted[q];
        if (j >= n) continue;
        const double gj = v.g[j * v.ps];
        const cplx w = {(v.x[j * v.ps] - cx) / h, (v.y[j * v.ps] - cy) / h};
        cplx pw = {gj, 0.0};   // G w^k / k!
#pragma unroll
        for (int k = 0; k < P; ++k) {
            b[k] = cadd(b[k], pw);
            pw = cscale(cmul(pw, w), c_fmm_inv[k + 1]);
        }
    }
    // reduce-scatter over the warp: at each halving the lane keeps the half
    // of its values selected by its lane bit and adds the partner's copy of
    // it (31 shuffles instead of 160 for an all-reduce of 32 values);
    // afterwards lane q holds value q = coefficient q/2, part q&1
    // (in groups of 16 coefficients, the last one padded with zeros)
#pragma unroll
    for (int g0 = 0; g0 < P; g0 += 16) {
        double vv[32];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int kk = min(g0 + k, P - 1);
            vv[2 * k] = g0 + k < P ? b[kk].r : 0.0;
            vv[2 * k + 1] = g0 + k < P ? b[kk].i : 0.0;
        }
#pragma unroll
        for (int half = 16; half > 0; half >>= 1) {
            const bool up = (lane & half) != 0;
#pragma unroll
            for (int i = 0; i < half; ++i) {
                const double send = up ? vv[i] : vv[i + half];
                const double keep = up ? vv[i + half] : vv[i];
                vv[i] = keep + __shfl_xor_sync(0xffffffffu, send, half);
            }
        }
        if (g0 + (lane >> 1) < P) reinterpret_cast<double *>(ML + c * P)[2 * g0 + lane] = vv[0];
    }
}

// M2M of coefficient k of cell c of level l from its 4 children at level
// l+1; the thread of coefficient 0 also writes the cell's vortex count (the
// sum of its children's).  Children are read through L2: in the fused
// upward kernels another block of the same launch may have written them.
template <int P>
__device__ __forceinline__ void fmm_m2m_cell(const cplx (*se)[P], int *cnt, cplx *M, int l, long long c, int k) {
    const long long m = 1LL << l, m2 = 2 * m;
    cplx *Mp = M + fmm_level_off(l) * P;
    const cplx *Mc = M + fmm_level_off(l + 1) * P;
    int *cp = cnt + fmm_level_off(l);
    const int *cc = cnt + fmm_level_off(l + 1);
    const long long ix = c % m, iy = c / m;
    int nq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) nq[q] = __ldcg(&cc[(2 * iy + (q >> 1)) * m2 + 2 * ix + (q & 1)]);
    const int np = nq[0] + nq[1] + nq[2] + nq[3];
    if (k == 0) cp[c] = np;
    cplx b = {0.0, 0.0};
    if (np > 0) {
        for (int q = 0; q < 4; ++q) {
            const long long child = (2 * iy + (q >> 1)) * m2 + 2 * ix + (q & 1);
            if (nq[q] == 0) continue;
            // unrolled over the P terms (those above k predicated off), so
            // the child's coefficients are loaded together, not one L2
            // round trip per term
#pragma unroll
            for (int mm = 0; mm < P; ++mm) {
                if (mm <= k) {
                    const double2 t = __ldcg(reinterpret_cast<const double2 *>(&Mc[child * P + mm]));
                    b = cadd(b, cscale(cmul(se[q][k - mm], cplx{t.x, t.y}), ldexp(1.0, -mm)));
                }
            }
        }
    }
    Mp[c * P + k] = b;
}

// M2M of levels hi-1 down to lo inside the subtree of cell r of level lo (one
// block; a barrier between levels).
template <int P>
__device__ __forceinline__ void fmm_m2m_subtree(const cplx (*se)[P], int *cnt, cplx *M, int lo, int hi, long long r) {
    const long long mlo = 1LL << lo, rx = r % mlo, ry = r / mlo;
    for (int l = hi - 1; l >= lo; --l) {
        const long long sl = 1LL << (l - lo), m = 1LL << l;
        for (long long e = threadIdx.x; e < sl * sl * P; e += blockDim.x) {
            const long long q = e / P;
            const long long c = (ry * sl + q / sl) * m + rx * sl + q % sl;
            fmm_m2m_cell<P>(se, cnt, M, l, c, (int)(e % P));
        }
        __syncthreads();
    }
}

constexpr int FMM_UP = 3;   // levels of the upward pass per fused launch
constexpr int FMM_TOP = 3;  // levels below this one are left to the last block of the upward pass

// Upward pass, first part: a block takes a cell r of level lo = max(L - 3, 0),
// computes P2M at the leaves of its subtree (one warp per leaf), then M2M of
// the 3 levels above them.
template <int P>
VX_DEVK void k_fmm_up_body(VxBlkB<128, 4> vb, const VxView &v, const VxScalars *S, const int *start, const int *sorted,
                           int *cnt, cplx *M) {
    __shared__ cplx se[4][P];
    const int L = S->fL;
    const int lo = max(L - FMM_UP, 0);
    const long long m = 1LL << L, mlo = 1LL << lo, sl = 1LL << (L - lo);
    cplx *ML = M + fmm_level_off(L) * P;
    fmm_shift_table<P>(se);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (long long r = vb.x; r < mlo * mlo; r += vb.n) {
        const long long rx = r % mlo, ry = r / mlo;
        for (long long q = warp; q < sl * sl; q += nw)
            fmm_p2m_leaf<P>(v, S, start, sorted, ML, (ry * sl + q / sl) * m + rx * sl + q % sl, m, lane);
        __syncthreads();
        fmm_m2m_subtree<P>(se, cnt, M, lo, L, r);
    }
}
template <int P>
__global__ void __launch_bounds__(128) k_fmm_up(VxView v, const VxScalars *S, const int *start, const int *sorted,
                                                int *cnt, cplx *M) {
    VX_PDL_WAIT();
    k_fmm_up_body<P>(VxBlkB<128, 4>{blockIdx.x, gridDim.x}, v, S, start, sorted, cnt, M);
}

// Upward pass, the rest: M2M of the levels from L - 4 up to 3 by subtrees
// as above (a block per cell of level 3), then the block that finishes last
// runs levels 2, 1 and 0.
template <int P>
VX_DEVK void k_fmm_up_top_body(VxBlkB<128, 0> vb, VxScalars *S, int *cnt, cplx *M) {
    __shared__ cplx se[4][P];
    const int hi = max(S->fL - FMM_UP, 0);
    const int lo = min(FMM_TOP, hi);
    if (hi == 0) return;
    fmm_shift_table<P>(se);
    __syncthreads();
    for (long long r = vb.x; r < (1LL << (2 * lo)); r += vb.n) fmm_m2m_subtree<P>(se, cnt, M, lo, hi, r);
    if (lo == 0 || !vx_last_block(&S->sync_ctr, vb.n)) return;
    for (int l = lo - 1; l >= 0; --l) {
        for (long long e = threadIdx.x; e < (1LL << (2 * l)) * P; e += blockDim.x)
            fmm_m2m_cell<P>(se, cnt, M, l, e / P, (int)(e % P));
        __syncthreads();
    }
}
template <int P>
__global__ void __launch_bounds__(128) k_fmm_up_top(VxScalars *S, int *cnt, cplx *M) {
    VX_PDL_WAIT();
    k_fmm_up_top_body<P>(VxBlkB<128, 0>{blockIdx.x, gridDim.x}, S, cnt, M);
}

// M2L at level l (2 <= l <= L) plus L2L from level l-1.  A block takes a
// 4 x 4 tile of target cells (two parents wide); the interaction lists of the
// tile draw on the 8 x 8 source cells around it (children of the parents'
// neighbours), whose multipoles are staged once in shared memory.  The
// Hankel entries H_j = j! t^-(j+1) of the 40 integer offsets t are tabulated
// per block.  Thread (cell, coefficient group cg, part pt) sums the G
// coefficients G cg .. G cg + G - 1 (G = 8 where it divides the order, else
// 4) over the interactions u = pt, pt + 4, ... of the cell's list, with a
// sliding window over the Hankel entries: per term one shared load of the
// source coefficient and one of the window's new entry serve 4 G FP64 FMAs
// (with G = 4 the two shared loads per 16 FMAs bound the loop).  The four
// parts (adjacent lanes) are then reduce-scattered in a fixed tree, so part
// pt ends with coefficients G cg + (G / 4) pt onwards; every coefficient is
// the same sum, in the same order, whatever G.
//
// The levels up to M2L_SMALL have few cells each: their M2L parts are
// independent of one another and run in one launch over all their tiles
// (k_fmm_m2l_small), then their L2L level by level (k_fmm_l2l_small); deeper
// levels take one launch each (k_fmm_m2l_l2l), M2L and L2L together.
constexpr int M2L_TILE = 4;
constexpr int M2L_SRC = 2 * M2L_TILE;   // 8 x 8 staged source cells
constexpr int M2L_SMALL = 6;
template <int P> __host__ __device__ constexpr int m2l_group() { return P % 8 == 0 ? 8 : 4; }   // coefficients a thread sums
template <int P> __host__ __device__ constexpr int m2l_threads() { return M2L_TILE * M2L_TILE * 4 * (P / m2l_group<P>()); }
#ifndef VX_M2L_MINB
#define VX_M2L_MINB 0   // minimum resident blocks per SM requested for the M2L kernels (0: none)
#endif

template <int P>
struct M2LShared {
    cplx sh[49][2 * P - 1];   // offset (dx, dy) in [-3, 3]^2 at (dy+3)*7 + dx+3
    cplx se[4][P];
    cplx sm[M2L_SRC * M2L_SRC][P];
    int sc[M2L_SRC * M2L_SRC];
};

template <int P>
__device__ void m2l_tables(M2LShared<P> &T) {
    fmm_shift_table<P>(T.se);
    for (int q = threadIdx.x; q < 49; q += blockDim.x) {
        const int dx = q % 7 - 3, dy = q / 7 - 3;
        if (abs(dx) <= 1 && abs(dy) <= 1) continue;   // neighbours: never an interaction
        const cplx ti = cinv(cplx{(double)dx, (double)dy});
        cplx tp = ti;
        double fact = 1.0;   // j!
        for (int j = 0; j < 2 * P - 1; ++j) {
            T.sh[q][j] = cscale(tp, fact);
            tp = cmul(tp, ti);
            fact *= (double)(j + 1);
        }
    }
}

// M2L of tile t of level l for this thread's (cell, lc); the block's threads
// all take part.  Returns whether the cell exists; *c its index, *busy
// whether it holds vortices, *a its scaled M2L coefficient lc.
template <int P>
__device__ bool m2l_tile(const VxScalars *S, const int *cnt, const cplx *M, int l, long long t, M2LShared<P> &T,
                         long long &c, bool &busy, int &lc0, cplx (&a)[2]) {
    constexpr int G = m2l_group<P>(), NC = G / 4, TPC = 4 * (P / G);   // threads per cell
    const long long m = 1LL << l;
    const long long tiles1 = vx_ceil_div(m, (long long)M2L_TILE);
    const double s = S->fside / (double)m;
    const cplx *Ml = M + fmm_level_off(l) * P;
    const int *cl = cnt + fmm_level_off(l);
    const int cell = threadIdx.x / TPC;
    const int cg = (threadIdx.x % TPC) >> 2, pt = threadIdx.x & 3;
    lc0 = G * cg + NC * pt;
    const long long tx0 = (t % tiles1) * M2L_TILE, ty0 = (t / tiles1) * M2L_TILE;
    const long long sx0 = tx0 - 2, sy0 = ty0 - 2;   // staged region origin
    const long long ix = tx0 + cell % M2L_TILE, iy = ty0 + cell / M2L_TILE;
    const bool live = ix < m && iy < m;
    c = live ? iy * m + ix : 0;
    // the barrier: the previous tile is done with sm / sc, tables are built;
    // a tile with no vortex under any of its cells is skipped (an empty
    // cell's local expansion is never read: L2L and L2P read busy cells only)
    if (!__syncthreads_or(live && cl[c] > 0)) {
        busy = false;
        return false;
    }
    for (int e = threadIdx.x; e < M2L_SRC * M2L_SRC * P; e += blockDim.x) {
        const int q = e / P, k = e % P;
        const long long qx = sx0 + q % M2L_SRC, qy = sy0 + q / M2L_SRC;
        const bool in = qx >= 0 && qx < m && qy >= 0 && qy < m;
        const long long src = qy * m + qx;
        const int n = in ? cl[src] : 0;
        if (k == 0) T.sc[q] = n;
        T.sm[q][k] = n > 0 ? Ml[src * P + k] : cplx{0.0, 0.0};
    }
    __syncthreads();
    busy = live && cl[c] > 0;
    const long long px = ix >> 1, py = iy >> 1;
    double v[2 * G];   // (re, im) of coefficients G cg + j
#pragma unroll
    for (int j = 0; j < 2 * G; ++j) v[j] = 0.0;
    if (busy) {
        for (int u = pt; u < 36; u += 4) {
            const long long qy = 2 * (py - 1) + u / 6, qx = 2 * (px - 1) + u % 6;
            if (qx < 0 || qx >= m || qy < 0 || qy >= m) continue;
            if (llabs(qx - ix) <= 1 && llabs(qy - iy) <= 1) continue;   // neighbours: near field
            const int q = (int)((qy - sy0) * M2L_SRC + (qx - sx0));
            if (T.sc[q] == 0) continue;
            const cplx *H = T.sh[(int)(iy - qy + 3) * 7 + (int)(ix - qx + 3)] + G * cg;   // H_{k + G cg + j}
            const cplx *B = T.sm[q];
            cplx h[G];
#pragma unroll
            for (int j = 0; j < G; ++j) h[j] = H[j];
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const cplx b = B[k];
#pragma unroll
                for (int j = 0; j < G; ++j) {
                    v[2 * j] = fma(b.r, h[j].r, fma(-b.i, h[j].i, v[2 * j]));
                    v[2 * j + 1] = fma(b.r, h[j].i, fma(b.i, h[j].r, v[2 * j + 1]));
                }
                if (k + 1 < P) {
#pragma unroll
                    for (int j = 0; j + 1 < G; ++j) h[j] = h[j + 1];
                    h[G - 1] = H[k + G];
                }
            }
        }
    }
    // reduce-scatter over the four parts (all lanes take part): first with
    // the part two lanes away (halves of the G coefficients), then with the
    // neighbouring part (halves of those): (p0 + p2) + (p1 + p3) for each
#pragma unroll
    for (int lvl = 0; lvl < 2; ++lvl) {
        const int half = G >> lvl, x = 2 >> lvl;
        const bool up = (pt & x) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const double send = up ? v[i] : v[i + half];
            const double keep = up ? v[i + half] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, x);
        }
    }
#pragma unroll
    for (int i = 0; i < NC; ++i) {
        a[i] = {v[2 * i], v[2 * i + 1]};
        if (busy) a[i] = cscale(a[i], (((lc0 + i) & 1) ? -1.0 : 1.0) / s);
    }
    return live;
}

// L2L of coefficient lc of cell (ix, iy) of level l from its parent's local
// expansion Lp (level l-1).
template <int P>
__device__ __forceinline__ cplx l2l_term(const cplx *Lp, const cplx (*se)[P], long long m, long long ix,
                                         long long iy, int lc) {
    const long long parent = (iy >> 1) * (m >> 1) + (ix >> 1);
    const int q = (int)((iy & 1) * 2 + (ix & 1));
    cplx acc = {0.0, 0.0};
#pragma unroll
    for (int j = 0; j < P; ++j)   // unrolled, the terms below lc predicated off: the loads issue together
        if (j >= lc) acc = cadd(acc, cmul(Lp[parent * P + j], se[q][j - lc]));
    return cscale(acc, ldexp(1.0, -lc));
}

template <int P>
VX_DEVK void k_fmm_m2l_l2l_body(VxBlkB<m2l_threads<P>(), 0> vb, const VxScalars *S, const int *cnt, const cplx *M,
                                cplx *Loc, int l) {
    constexpr int NC = m2l_group<P>() / 4;
    M2LShared<P> &T = *reinterpret_cast<M2LShared<P> *>(vx_fmm_dyn);
    if (l > S->fL) return;
    m2l_tables<P>(T);
    const long long m = 1LL << l;
    const long long tiles1 = vx_ceil_div(m, (long long)M2L_TILE);
    cplx *Ll = Loc + fmm_level_off(l) * P;
    const cplx *Lp = Loc + fmm_level_off(l - 1) * P;
    for (long long t = vb.x; t < tiles1 * tiles1; t += vb.n) {
        long long c;
        bool busy;
        int lc0;
        cplx a[2];
        if (!m2l_tile<P>(S, cnt, M, l, t, T, c, busy, lc0, a)) continue;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            if (busy && l > 2) a[i] = cadd(a[i], l2l_term<P>(Lp, T.se, m, c % m, c / m, lc0 + i));
            Ll[c * P + lc0 + i] = a[i];
        }
    }
}
template <int P>
__global__ void __launch_bounds__(m2l_threads<P>(), VX_M2L_MINB) k_fmm_m2l_l2l(const VxScalars *S, const int *cnt, const cplx *M,
                                                       cplx *Loc, int l) {
    VX_PDL_WAIT();
    k_fmm_m2l_l2l_body<P>(VxBlkB<m2l_threads<P>(), 0>{blockIdx.x, gridDim.x}, S, cnt, M, Loc, l);
}

// M2L (without L2L) of levels 2 .. min(M2L_SMALL, L): blocks over the tiles
// of all of them.
template <int P>
VX_DEVK void k_fmm_m2l_small_body(VxBlkB<m2l_threads<P>(), 0> vb, const VxScalars *S, const int *cnt, const cplx *M,
                                  cplx *Loc) {
    constexpr int NC = m2l_group<P>() / 4;
    M2LShared<P> &T = *reinterpret_cast<M2LShared<P> *>(vx_fmm_dyn);
    const int hi = min(S->fL, M2L_SMALL);
    if (hi < 2) return;
    m2l_tables<P>(T);
    long long total = 0;
    for (int l = 2; l <= hi; ++l) total += vx_ceil_div(1LL << (2 * l), (long long)(M2L_TILE * M2L_TILE));
    for (long long b = vb.x; b < total; b += vb.n) {
        int l = 2;
        long long t = b;
        while (t >= vx_ceil_div(1LL << (2 * l), (long long)(M2L_TILE * M2L_TILE))) {
            t -= vx_ceil_div(1LL << (2 * l), (long long)(M2L_TILE * M2L_TILE));
            ++l;
        }
        long long c;
        bool busy;
        int lc0;
        cplx a[2];
        if (!m2l_tile<P>(S, cnt, M, l, t, T, c, busy, lc0, a)) continue;
#pragma unroll
        for (int i = 0; i < NC; ++i) Loc[(fmm_level_off(l) + c) * P + lc0 + i] = a[i];
    }
}
template <int P>
__global__ void __launch_bounds__(m2l_threads<P>(), VX_M2L_MINB) k_fmm_m2l_small(const VxScalars *S, const int *cnt, const cplx *M,
                                                         cplx *Loc) {
    VX_PDL_WAIT();
    k_fmm_m2l_small_body<P>(VxBlkB<m2l_threads<P>(), 0>{blockIdx.x, gridDim.x}, S, cnt, M, Loc);
}

// L2L into levels 3 .. min(M2L_SMALL, L), one launch: a block takes a cell
// of level 3 and walks down its subtree level by level (a barrier between
// levels), one thread per (cell, coefficient).
template <int P>
VX_DEVK void k_fmm_l2l_small_body(VxBlkB<256, 0> vb, const VxScalars *S, const int *cnt, cplx *Loc) {
    __shared__ cplx se[4][P];
    const int hi = min(S->fL, M2L_SMALL);
    if (hi < 3) return;
    fmm_shift_table<P>(se);
    __syncthreads();
    for (long long r = vb.x; r < 64; r += vb.n) {
        const long long rx = r % 8, ry = r / 8;
        for (int l = 3; l <= hi; ++l) {
            const long long sl = 1LL << (l - 3), m = 1LL << l;
            const int *cl = cnt + fmm_level_off(l);
            cplx *Ll = Loc + fmm_level_off(l) * P;
            const cplx *Lp = Loc + fmm_level_off(l - 1) * P;
            for (long long e = threadIdx.x; e < sl * sl * P; e += blockDim.x) {
                const long long q = e / P;
                const int lc = (int)(e % P);
                const long long c = (ry * sl + q / sl) * m + rx * sl + q % sl;
                if (cl[c] > 0) Ll[c * P + lc] = cadd(Ll[c * P + lc], l2l_term<P>(Lp, se, m, c % m, c / m, lc));
            }
            __syncthreads();
        }
    }
}
template <int P>
__global__ void __launch_bounds__(256) k_fmm_l2l_small(const VxScalars *S, const int *cnt, cplx *Loc) {
    VX_PDL_WAIT();
    k_fmm_l2l_small_body<P>(VxBlkB<256, 0>{blockIdx.x, gridDim.x}, S, cnt, Loc);
}

// Near field (FP32, core smoothing) + far field (L2P, FP64): one warp per
// work item of up to FMM_W targets of one leaf.  All of them share the 3 x 3
// leaves around it, whose sources the warp stages 32 at a time (three
// contiguous runs of the leaf-sorted array), coordinates relative to the
// item's leaf centre.  The 3 nearest come from their own pass
// (k_fmm_nn3_sub) over the finer grid of quarter leaves.
__device__ __forceinline__ float vx_rcp_approx2(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Two near-field pairs (one target, sources a and b of a staged slot) in
// packed FP32: core-smoothed Biot-Savart terms.  The target's own slot adds
// 0 (dx = dy = 0), so no pair is skipped.  One reciprocal serves both pairs:
// 1/a = b (1/(a b)), 1/b = a (1/(a b)) (a b stays within FP32 range: padding
// sources sit 1e12 away, and both padded gives 1/inf = 0, G = 0).
__device__ __forceinline__ void near_pair2(f2 SX, f2 SYs, f2 G, f2 TX, f2 TY, float eps2, f2 &SY, f2 &SXN) {
    const f2 DX = f2_sub(TX, SX), DY = f2_sub(TY, SYs);
    const f2 R2 = f2_fma(DX, DX, f2_mul(DY, DY));
    float r2a, r2b;
    f2_unpack(R2, r2a, r2b);
    const float ra = fmaxf(r2a, eps2), rb = fmaxf(r2b, eps2);
    const float q = vx_rcp_approx2(ra * rb);
    const f2 MM = f2_mul(G, f2_mul(f2_pack(rb, ra), f2_pack(q, q)));
    SY = f2_fma(MM, DX, SY);
    SXN = f2_fma(MM, DY, SXN);   // sum of +mm dy: negated by the caller
}

#ifndef VX_NEAR_MINB
#define VX_NEAR_MINB 2   // minimum resident blocks per SM requested for k_fmm_near (at most 128 registers)
#endif
template <int P>
VX_DEVK void k_fmm_near_body(VxBlkB<FMM_T, VX_NEAR_MINB> vb, const VxParams &p, const VxView &v, VxScalars *S, const float4 *srt,
                             const int *sorted, const int *start, const int2 *items, const cplx *Loc) {
    // per warp 32 staged sources as x[32], y[32], G[32]: one 16-byte shared
    // load brings four sources' x (or y, or G)
    __shared__ float4 sx[FMM_T / 4], sy[FMM_T / 4], sg[FMM_T / 4];
    const int lane = threadIdx.x & 31;
    float4 *wx = sx + ((threadIdx.x & ~31) >> 2), *wy = sy + ((threadIdx.x & ~31) >> 2),
           *wg = sg + ((threadIdx.x & ~31) >> 2);
    const long long n = S->n;
    const int L = S->fL;
    const long long m = 1LL << L;
    const double h = S->fside / (double)m;
    const float eps2 = (float)p.eps2;
    const long long nitems = S->cnitems;
    const cplx *LL = Loc + fmm_level_off(L) * P;
    const long long wpb = FMM_T / 32;
    for (long long it = vb.x * wpb + (threadIdx.x >> 5); it < nitems; it += vb.n * wpb) {
        const int2 item = items[it];
        const long long leaf = item.x;
        const long long row = leaf / m, col = leaf % m;
        const long long last = min((long long)item.y + FMM_W, (long long)start[leaf + 1]);
        const long long t = item.y + lane;
        const bool valid = t < last;
        const float4 me = valid ? srt[t] : make_float4(0.f, 0.f, 0.f, 0.f);   // relative to the leaf centre
        const long long j_self = valid ? sorted[t] : -1;
        const long long c0 = max(col - 1, 0LL), c1 = min(col + 1, m - 1);
        const f2 TX = f2_pack(me.x, me.x), TY = f2_pack(me.y, me.y);
        double ax = 0.0, ay = 0.0;
        // the 3 x 3 leaves are three contiguous runs (rows row-1..row+1 of
        // columns c0..c1), walked as one stream in chunks of 32 sources, so
        // only the stream's last chunk is padded
        const long long r_lo = max(row - 1, 0LL), r_hi = min(row + 1, m - 1);
        int rj0[3], rpre[4];
        float roy[3];
        rpre[0] = 0;
        for (int r = 0; r < 3; ++r) {
            const long long rr = r_lo + r;
            int len = 0;
            rj0[r] = 0;
            roy[r] = 0.f;
            if (rr <= r_hi) {
                rj0[r] = start[rr * m + c0];
                len = start[rr * m + c1 + 1] - rj0[r];
                roy[r] = (float)((double)(rr - row) * h);
            }
            rpre[r + 1] = rpre[r] + len;
        }
        const int total = rpre[3];
        // source f of the stream: its slot in the leaf-sorted array and the
        // y offset of its row; the x offset of its column, (column - col) h
        // with the difference -1, 0 or 1, is exact in FP32
        const float hf = (float)h, colf = (float)col;
        auto src_of = [&](int f, float &oy) {
            const bool in0 = f < rpre[1], in1 = f < rpre[2];
            oy = in0 ? roy[0] : (in1 ? roy[1] : roy[2]);
            return in0 ? rj0[0] + f : (in1 ? rj0[1] + (f - rpre[1]) : rj0[2] + (f - rpre[2]));
        };
        // the next chunk's source is loaded before the current chunk's pairs run
        float4 qn = make_float4(1e12f, 1e12f, 0.f, colf);
        float oyn = 0.f;
        if (lane < total) qn = srt[src_of(lane, oyn)];
        for (int jt = 0; jt < total; jt += 32) {
            // padding: G = 0 sources far away add exactly 0
            const float4 q = qn;
            const float oy = oyn;
            const int fnext = jt + 32 + lane;
            if (fnext < total) qn = srt[src_of(fnext, oyn)];
            float x = 1e12f, y = 1e12f, g = 0.f;
            if (jt + lane < total) {
                x = q.x + (q.w - colf) * hf;
                y = q.y + oy;
                g = q.z;
            }
            reinterpret_cast<float *>(wx)[lane] = x;
            reinterpret_cast<float *>(wy)[lane] = y;
            reinterpret_cast<float *>(wg)[lane] = g;
            __syncwarp();
            f2 SY = 0ull, SXN = 0ull;   // +0.0f in both halves
#pragma unroll
            for (int q4 = 0; q4 < 8; ++q4) {   // sources 2q, 2q + 1 a pair step, in index order
                const ulonglong2 X = *reinterpret_cast<const ulonglong2 *>(wx + q4);
                const ulonglong2 Y = *reinterpret_cast<const ulonglong2 *>(wy + q4);
                const ulonglong2 G = *reinterpret_cast<const ulonglong2 *>(wg + q4);
                near_pair2(X.x, Y.x, G.x, TX, TY, eps2, SY, SXN);
                near_pair2(X.y, Y.y, G.y, TX, TY, eps2, SY, SXN);
            }
            __syncwarp();
            float a, b;   // the two halves are added in FP32, then carried in FP64
            f2_unpack(SXN, a, b); ax -= (double)(a + b);
            f2_unpack(SY, a, b); ay += (double)(a + b);
        }
        {   // executed near-field pairs: every target of the item sees the same 3x3 leaves
            const unsigned long long nv = __popc(__ballot_sync(0xffffffffu, valid));
            if (lane == 0) atomicAdd(&S->pairs_bs, (unsigned long long)total * nv);
        }
        if (valid && j_self < n) {
            // far field: f(z) = sum a_l u^l at the target's leaf (none below depth 2)
            cplx f = {0.0, 0.0};
            if (L >= 2) {
                const double xd = v.x[j_self * v.ps], yd = v.y[j_self * v.ps];
                const cplx u = {(xd - (S->fx0 + ((double)col + 0.5) * h)) / h,
                                (yd - (S->fy0 + ((double)row + 0.5) * h)) / h};
                // f = sum_l A_l u^l / l!, nested as A_0 + (u/1)(A_1 + (u/2)(A_2 + ...))
                f = LL[leaf * P + P - 1];
                for (int l = P - 2; l >= 0; --l)
                    f = cadd(cmul(f, cscale(u, c_fmm_inv[l + 1])), LL[leaf * P + l]);
            }
            // u - i v = f / (2 pi i): vx = Im f / 2pi, vy = Re f / 2pi
            v.vx[j_self * v.vs] = (ax + f.i) / VX_TWO_PI + S->vinf[0];
            v.vy[j_self * v.vs] = (ay + f.r) / VX_TWO_PI + S->vinf[1];
        }
    }
}
template <int P>
__global__ void __launch_bounds__(FMM_T, VX_NEAR_MINB) k_fmm_near(VxParams p, VxView v, VxScalars *S, const float4 *srt,
                                                   const int *sorted, const int *start, const int2 *items,
                                                   const cplx *Loc) {
    VX_PDL_WAIT();
    k_fmm_near_body<P>(VxBlkB<FMM_T, VX_NEAR_MINB>{blockIdx.x, gridDim.x}, p, v, S, srt, sorted, start, items, Loc);
}

// The 3 nearest sources of every live target (the reference's padded
// launch: sources include the round-32 slots after the live ones; the
// target itself excluded), one thread per target, over the 3 x 3 quarter
// leaves around its own quarter (each quarter a contiguous run of the
// sorted sources; coordinates relative to the target's leaf centre,
// computed as the near field computes them).  Exact when the third distance
// is below the quarter's side (every source outside the 3 x 3 block is
// farther); the others go to the ring search over leaves (k_fmm_nn3_fix).
VX_DEVK void k_fmm_nn3_sub_body(VxBlkB<FMM_T, 0> vb, const VxView &v, VxScalars *S, const float4 *srt, const unsigned *skey,
                                const int *sorted, const int *substart, int *flag_list) {
    const long long s = S->fs, n = S->n;
    const int m = 1 << S->fL, m2 = 2 * m;
    const double h = S->fside / (double)m;
    const float sq2 = (float)(0.25 * h * h);   // (quarter side)^2
    for (long long t = vb.x * (long long)blockDim.x + threadIdx.x; t < s; t += (long long)vb.n * blockDim.x) {
        const int j = sorted[t];
        if (j >= n) continue;
        const unsigned key = skey[t];
        const int leaf = (int)(key >> 2), col = leaf % m, row = leaf / m;
        const int ix2 = 2 * col + (int)(key & 1), iy2 = 2 * row + (int)((key >> 1) & 1);
        const float4 me = srt[t];
        float d1 = 1e5f, d2 = 1e5f, d3 = 1e5f;
        const int y0 = max(iy2 - 1, 0), y1 = min(iy2 + 1, m2 - 1);
        const int x0 = max(ix2 - 1, 0), x1 = min(ix2 + 1, m2 - 1);
        // a source's offset to the target's leaf centre: (its leaf's column -
        // col) h and (its leaf's row - row) h, differences of -1, 0 or 1, so
        // exact in FP32 and the same for every source of a quarter
        const float hf = (float)h, hq = 0.5f * hf;
        // the target's own quarter first, then its four edge neighbours, then
        // the corners; a quarter whose box lies farther than the third
        // distance found so far (with a margin over FP32 rounding) cannot
        // hold one of the 3 nearest and is not read: in a dense region the
        // own quarter alone usually settles them.  (A quarter X2 spans
        // [(X2 - 2 col - 1) hq, (X2 - 2 col) hq] in the leaf frame.)
#pragma unroll 1
        for (int o = 0; o < 9; ++o) {
            const int ddx = (o == 1 || o == 5 || o == 7) ? -1 : ((o == 2 || o == 6 || o == 8) ? 1 : 0);
            const int ddy = (o == 3 || o == 5 || o == 6) ? -1 : ((o == 4 || o == 7 || o == 8) ? 1 : 0);
            const int X2 = ix2 + ddx, Y2 = iy2 + ddy;
            if (X2 < x0 || X2 > x1 || Y2 < y0 || Y2 > y1) continue;
            if (o > 0) {
                const float qx = (float)(X2 - 2 * col), qy = (float)(Y2 - 2 * row);
                const float gx = fmaxf(fmaxf((qx - 1.0f) * hq - me.x, me.x - qx * hq), 0.0f);
                const float gy = fmaxf(fmaxf((qy - 1.0f) * hq - me.y, me.y - qy * hq), 0.0f);
                if (fmaf(gx, gx, gy * gy) > 1.0001f * d3) continue;
            }
            const int lr = Y2 >> 1;
            const float oy = (float)(lr - row) * hf;
            const float ox = (float)((X2 >> 1) - col) * hf;
            const int k = 4 * (lr * m + (X2 >> 1)) + 2 * (Y2 & 1) + (X2 & 1);
            const int q1 = substart[k + 1];
            for (int qq = substart[k]; qq < q1; ++qq) {
                if (qq == t) continue;
                const float2 q = *reinterpret_cast<const float2 *>(srt + qq);   // x, y of the source
                const float dx = me.x - (q.x + ox), dy = me.y - (q.y + oy);
                vx_nn3_insert_bf(d1, d2, d3, fmaf(dx, dx, dy * dy));
            }
        }
        v.d[j] = (double)((sqrtf(d1) + sqrtf(d2) + sqrtf(d3)) / 3);
        if (!(d3 < sq2)) {   // a closer source could lie outside the 3x3 quarters
            const int slot = atomicAdd(&S->fnflag, 1);
            flag_list[slot] = (int)t;
        }
    }
}
__global__ void __launch_bounds__(FMM_T) k_fmm_nn3_sub(VxView v, VxScalars *S, const float4 *srt, const unsigned *skey,
                                                      const int *sorted, const int *substart, int *flag_list) {
    VX_PDL_WAIT();
    k_fmm_nn3_sub_body(VxBlkB<FMM_T, 0>{blockIdx.x, gridDim.x}, v, S, srt, skey, sorted, substart, flag_list);
}

// Targets whose third-nearest distance reached the leaf side: exact 3
// nearest by a ring search over the leaves (one warp per target).  Ring k
// holds the 8k leaves at Chebyshev distance k from the target's leaf; every
// source outside rings 0..k lies at least k*h from the target (a source
// clamped into an edge leaf lies farther out than that leaf), so the search
// stops once the third distance is below (k h)^2 or the rings cover the grid.
// Coordinates are relative to the target's leaf centre, as in the near field.
// The search stops after NN3_RINGS rings: an isolated vortex (one flung out
// of the wake) would need rings over much of the grid, which one warp walks
// for a millisecond or more; such targets go to k_fmm_nn3_brute instead, a
// block scanning every source.
constexpr int NN3_RINGS = 6;
__device__ __forceinline__ void fmm_ring_cell(int k, int q, int &dx, int &dy) {
    if (k == 0) { dx = dy = 0; return; }
    const int w = 2 * k + 1;
    if (q < w) { dx = q - k; dy = -k; return; }
    q -= w;
    if (q < w) { dx = q - k; dy = k; return; }
    q -= w;
    if (q < w - 2) { dx = -k; dy = q - k + 1; return; }
    q -= w - 2;
    dx = k; dy = q - k + 1;
}

// The targets the ring search left over, by one block: each scans every
// source slot (FP64 differences, as the direct pass).
__device__ void fmm_nn3_brute_block(VxView v, VxScalars *S, const int *brute_list) {
    __shared__ float sd[3][FMM_T / 32];
    const int nb = __ldcg(&S->fnbrute);
    const long long fs = S->fs;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = 0; b < nb; ++b) {
        const long long i = __ldcg(&brute_list[b]);
        const double xi = v.x[i * v.ps], yi = v.y[i * v.ps];
        float d1 = 1e5f, d2 = 1e5f, d3 = 1e5f;
        for (long long j = threadIdx.x; j < fs; j += blockDim.x) {
            if (j == i) continue;
            const double dx = xi - v.x[j * v.ps], dy = yi - v.y[j * v.ps];
            vx_nn3_insert_bf(d1, d2, d3, (float)fma(dx, dx, dy * dy));
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float e1 = __shfl_xor_sync(0xffffffffu, d1, o);
            const float e2 = __shfl_xor_sync(0xffffffffu, d2, o);
            const float e3 = __shfl_xor_sync(0xffffffffu, d3, o);
            vx_nn3_insert_bf(d1, d2, d3, e1);
            vx_nn3_insert_bf(d1, d2, d3, e2);
            vx_nn3_insert_bf(d1, d2, d3, e3);
        }
        if (lane == 0) { sd[0][warp] = d1; sd[1][warp] = d2; sd[2][warp] = d3; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < FMM_T / 32; ++w) {
                vx_nn3_insert_bf(d1, d2, d3, sd[0][w]);
                vx_nn3_insert_bf(d1, d2, d3, sd[1][w]);
                vx_nn3_insert_bf(d1, d2, d3, sd[2][w]);
            }
            v.d[i] = (double)((sqrtf(d1) + sqrtf(d2) + sqrtf(d3)) / 3);
        }
        __syncthreads();
    }
}

VX_DEVK void k_fmm_nn3_fix_body(VxBlkB<0, 0> vb, const VxView &v, VxScalars *S, const float4 *srt, const int *sorted,
                                const int *start, const int *flag_list, int *brute_list) {
    const int nf = S->fnflag;
    const long long m = 1LL << S->fL;
    const double h = S->fside / (double)m;
    const int lane = threadIdx.x & 31;
    const int warps = (vb.n * blockDim.x) >> 5;
    for (int f = (vb.x * blockDim.x + threadIdx.x) >> 5; f < nf; f += warps) {
        const long long t = flag_list[f];
        const long long i = sorted[t];
        const long long leaf = fmm_leaf(S, v.x[i * v.ps], v.y[i * v.ps]);
        const long long cx = leaf % m, cy = leaf / m;
        const float4 me = srt[t];
        const long long kmax = max(max(cx, m - 1 - cx), max(cy, m - 1 - cy));
        float d1 = 1e5f, d2 = 1e5f, d3 = 1e5f;
        bool found = false;
        for (long long k = 0; k <= min(kmax, (long long)NN3_RINGS); ++k) {
            const int ncell = k == 0 ? 1 : (int)(8 * k);
            for (int q = lane; q < ncell; q += 32) {
                int dx, dy;
                fmm_ring_cell((int)k, q, dx, dy);
                const long long X = cx + dx, Y = cy + dy;
                if (X < 0 || X >= m || Y < 0 || Y >= m) continue;
                const float ox = (float)((double)dx * h), oy = (float)((double)dy * h);
                const long long c = Y * m + X;
                for (long long j = start[c]; j < start[c + 1]; ++j) {
                    if (j == t) continue;
                    const float4 s = srt[j];
                    const float ddx = me.x - (s.x + ox), ddy = me.y - (s.y + oy);
                    vx_nn3_insert<float>(d1, d2, d3, fmaf(ddx, ddx, ddy * ddy));
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const float e1 = __shfl_xor_sync(0xffffffffu, d1, o);
                const float e2 = __shfl_xor_sync(0xffffffffu, d2, o);
                const float e3 = __shfl_xor_sync(0xffffffffu, d3, o);
                vx_nn3_insert<float>(d1, d2, d3, e1);
                vx_nn3_insert<float>(d1, d2, d3, e2);
                vx_nn3_insert<float>(d1, d2, d3, e3);
            }
            // every lane holds the merged three; keep them in lane 0 only so
            // that the next ring merges disjoint sets
            const float kh = (float)((double)k * h);
            const bool done = d3 < kh * kh || k == kmax;
            if (lane != 0) d1 = d2 = d3 = 1e5f;
            if (done) { found = true; break; }
        }
        if (lane == 0) {
            if (found) v.d[i] = (double)((sqrtf(d1) + sqrtf(d2) + sqrtf(d3)) / 3);
            else brute_list[atomicAdd(&S->fnbrute, 1)] = (int)i;
        }
    }
    // the rare targets no ring settled: the block that finishes last scans
    // every source for them
    if (vx_last_block(&S->sync_ctr, vb.n)) fmm_nn3_brute_block(v, S, brute_list);
}
__global__ void k_fmm_nn3_fix(VxView v, VxScalars *S, const float4 *srt, const int *sorted,
                              const int *start, const int *flag_list, int *brute_list) {
    VX_PDL_WAIT();
    k_fmm_nn3_fix_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, srt, sorted, start, flag_list, brute_list);
}

// The 3 nearest of the targets the ring search left (original indices in
// brute_list) over every source slot [0, fs): one block per target, each
// thread keeping the three smallest of its stride, merged over the warp and
// the block (the same set of sources as the ring search, so the same three).

// Near-field work items: every leaf's targets in chunks of FMM_W, leaves in
// index order (row-major), as (leaf, first target slot); one-pass scan of
// the leaves' item counts, each thread writing its leaves' items.
VX_DEVK void k_fmm_items_body(VxBlkB<VX_SCAN_T, 0> vb, VxScalars *S, const int *start, int2 *items,
                              long long items_cap, unsigned long long *tiles) {
    constexpr int PER = 4;
    const long long nl = S->fnleaves;
    vx_scan_lookback<PER>(
        vb.n, nl, S, tiles, [&](long long c) { return (start[c + 1] - start[c] + FMM_W - 1) / FMM_W; },
        [&](long long c0, const unsigned *val, long long run) {
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const long long c = c0 + q;
                if (c >= nl) break;
                const int j0 = start[c];
                for (unsigned k = 0; k < val[q]; ++k, ++run)
                    if (run < items_cap) items[run] = make_int2((int)c, j0 + (int)k * FMM_W);
            }
        },
        [&](long long tot) {
            // the item buffer holds s/32 + cells items, so this never truncates
            if (tot > items_cap) S->err |= VX_DERR_GRID;
            S->cnitems = tot <= items_cap ? tot : items_cap;
        });
}
__global__ void __launch_bounds__(VX_SCAN_T) k_fmm_items(VxScalars *S, const int *start, int2 *items,
                                                         long long items_cap, unsigned long long *tiles) {
    VX_PDL_WAIT();
    k_fmm_items_body(VxBlkB<VX_SCAN_T, 0>{blockIdx.x, gridDim.x}, S, start, items, items_cap, tiles);
}

long long vx_fmm_cells(int lmax) { return fmm_level_off(lmax + 1); }

int vx_fmm_max_level(long long cap) {
    int L = 2;
    while (L < 10 && (double)(1LL << (2 * L)) * 8.0 < (double)cap) ++L;
    return L;
}

template <int P>
static cudaError_t velocity_fmm(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S, VxWork &w) {
    constexpr int M2L_T = m2l_threads<P>();
    constexpr size_t M2L_SMEM = sizeof(M2LShared<P>);
    if (M2L_SMEM > 48 * 1024 && !L.rec) {   // opt in to more than 48 KB of shared memory (once per device)
        static bool done[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev >= 0 && dev < 64 && !done[dev]) {
            cudaFuncSetAttribute(k_fmm_m2l_l2l<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M2L_SMEM);
            cudaFuncSetAttribute(k_fmm_m2l_small<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M2L_SMEM);
            done[dev] = true;
        }
    }
    const int grid = L.num_sms * 4;
    const int Lmax = w.fmm_lmax;
    const int pgrid = std::min(grid, VX_RED_BLOCKS);   // 4 box keys per block
    vx_launch<k_fmm_prep, k_fmm_prep_body>(L, pgrid, FMM_T, 0, v, S, p.eps, Lmax, p.fmm_leaf > 0 ? p.fmm_leaf : 32,
                                           w.fmm_cnt, vx_fmm_cells(Lmax), w.fmm_sub_cnt, 1LL << (2 * (Lmax + 1)),
                                           w.box);
    vx_launch<k_fmm_leafid, k_fmm_leafid_body>(L, grid, FMM_T, 0, v, S, w.key0, w.val0, w.fmm_sub_cnt);
    vx_launch<k_fmm_scan, k_fmm_scan_body>(L, grid, VX_SCAN_T, 0, S, (const int *)w.fmm_sub_cnt, w.fmm_sub_start,
                                           w.fmm_cnt, w.fmm_start, w.scan_tiles);
    // source order: by quarter-leaf, each quarter's sources in index order
    // (a stable sort by the key 4 leaf + child; each leaf stays contiguous),
    // the FP32 sources gathered at their slots on the way
    VxGather gt;
    gt.mode = 1;
    gt.v = v;
    gt.S = S;
    gt.srt = w.srt;
    vx_bucket_order(L, S, &S->fs, &S->fnsub, w.key0, w.fmm_sub_start, w.fmm_sub_cnt, nullptr, w.key1, w.val1,
                    w.bk_mid, w.bk_big, w.val0, gt);
    const unsigned *skey = w.key1;
    const int *sorted = w.val1;
    // upward pass: P2M + M2M of the 3 levels above the leaves by subtrees,
    // then the levels above those (two launches whatever the depth)
    const int gup = (int)std::min<long long>(grid * 4, 1LL << (2 * std::max(Lmax - FMM_UP, 0)));
    vx_launch<k_fmm_up<P>, k_fmm_up_body<P>>(L, gup, 128, 0, v, S, w.fmm_start, sorted, w.fmm_cnt, (cplx *)w.fmm_M);
    vx_launch<k_fmm_up_top<P>, k_fmm_up_top_body<P>>(L, 1 << (2 * FMM_TOP), 128, 0, S, w.fmm_cnt, (cplx *)w.fmm_M);
    {
        long long tiles = 0;
        for (int l = 2; l <= std::min(Lmax, M2L_SMALL); ++l) tiles += vx_ceil_div(1LL << (2 * l), 16LL);
        if (tiles > 0) {
            vx_launch<k_fmm_m2l_small<P>, k_fmm_m2l_small_body<P>>(L, (int)std::min<long long>(grid * 2, tiles), M2L_T, M2L_SMEM, S, w.fmm_cnt, (const cplx *)w.fmm_M, (cplx *)w.fmm_L);
            vx_launch<k_fmm_l2l_small<P>, k_fmm_l2l_small_body<P>>(L, 64, 256, 0, S, w.fmm_cnt, (cplx *)w.fmm_L);
        }
    }
    for (int l = M2L_SMALL + 1; l <= Lmax; ++l) {
        const long long t1 = vx_ceil_div(1LL << l, (long long)M2L_TILE);
        const int g = (int)std::min<long long>(grid * 2, t1 * t1);
        vx_launch<k_fmm_m2l_l2l<P>, k_fmm_m2l_l2l_body<P>>(L, g, M2L_T, M2L_SMEM, S, w.fmm_cnt, (const cplx *)w.fmm_M, (cplx *)w.fmm_L, l);

    }
    vx_launch<k_fmm_items, k_fmm_items_body>(L, grid, VX_SCAN_T, 0, S, w.fmm_start, w.items, w.items_cap, w.scan_tiles);

    VX_EV(L, 0);
    vx_launch<k_fmm_near<P>, k_fmm_near_body<P>>(L, L.num_sms * 8, FMM_T, 0, p, v, S, w.srt, sorted, w.fmm_start,
                                                 w.items, (const cplx *)w.fmm_L);
    VX_EV(L, 1);
    vx_launch<k_fmm_nn3_sub, k_fmm_nn3_sub_body>(L, grid, FMM_T, 0, v, S, w.srt, skey, sorted,
                                                 (const int *)w.fmm_sub_start, w.fmm_flags);

    vx_launch<k_fmm_nn3_fix, k_fmm_nn3_fix_body>(L, grid, FMM_T, 0, v, S, w.srt, sorted, w.fmm_start, w.fmm_flags, w.fmm_brute);


    return cudaGetLastError();
}

cudaError_t vx_launch_velocity_fmm(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                                   VxWork &w) {
    switch (p.fmm_p) {
    case 8: return velocity_fmm<8>(L, p, v, S, w);
    case 12: return velocity_fmm<12>(L, p, v, S, w);
    case 20: return velocity_fmm<20>(L, p, v, S, w);
    default: return velocity_fmm<16>(L, p, v, S, w);
    }
}
