// vx_collapse.cu — merging of close vortex pairs, two passes (opposite signs,
// then same sign), each repeated up to n_col times while the count changes.
//
// Reference: first_setka_Kernel/second_setka_Kernel src/kernel.cu:1180-1235
// (COL[i] = smallest j > i that qualifies, an O(N^2) scan per thread),
// first_collapse_Kernel/second_collapse_Kernel src/kernel.cu:1237-1271 (one
// thread merges in index order), pass loop src/unit_1.cu:1137-1216.
//
// Here:
//  * COL comes from a uniform cell grid with cells no smaller than the merge
//    radius (counting sort into cells, 3x3 neighbourhood query).  The distance
//    test is the same FP64 expression as the oracle's, so COL is identical.
//  * The serial merge is resolved in parallel.  Candidate i (COL[i] >= 0) is
//    applied iff no applied candidate points at i; rounds decide every
//    candidate whose in-pointing candidates are all decided.  An applied i
//    merges with the original j only if it is the smallest applied candidate
//    pointing at j; later ones merge with (0, 1e10) as the serial loop does,
//    which re-rounds their position.
//  * Compaction then runs as after convection.
// A round is six launches before the compaction: prep (box, bookkeeping and
// grid in one, the last block finishing), count, a one-pass scan of the cell
// counts, scatter, query, and settle (resolution, merge and write-back in
// one block).
#include <limits.h>

#include "vx_internal.cuh"

// Start of a round: the bounding box (per-block keys into part[], combined
// by the last block), the round's bookkeeping and the cell grid.  A round
// after one that removed nothing (or after a failed one) does nothing: the
// pass has converged.  Cell side h = r (1 + 1e-6): any pair closer than r is
// in neighbouring cells; when the box would need more than cells_cap cells,
// h grows.
VX_DEVK void k_col_prep_body(VxBlkB<VX_THREADS, 0> vb, const VxView &v, VxScalars *S, int reset, double r2,
                             long long cells_cap, unsigned long long *part) {
    const bool done = reset ? false : (S->col_done || S->n == S->col_n_before);
    if (done) {
        if (vb.x == 0 && threadIdx.x == 0) S->col_done = 1;
        return;
    }
    __shared__ unsigned long long sh[4][VX_THREADS];
    const long long n = S->n;
    unsigned long long k[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        const double x = v.x[i * v.ps], y = v.y[i * v.ps];
        k[0] = min(k[0], vx_dkey(x));
        k[1] = min(k[1], vx_dkey(-x));
        k[2] = min(k[2], vx_dkey(y));
        k[3] = min(k[3], vx_dkey(-y));
    }
    for (int q = 0; q < 4; ++q) sh[q][threadIdx.x] = k[q];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 4; ++q) sh[q][threadIdx.x] = min(sh[q][threadIdx.x], sh[q][threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x < 4) part[4 * vb.x + threadIdx.x] = sh[threadIdx.x][0];
    if (!vx_last_block(&S->sync_ctr, vb.n)) return;
    for (int q = 0; q < 4; ++q) k[q] = ~0ull;
    for (unsigned b = threadIdx.x; b < vb.n; b += blockDim.x)
        for (int q = 0; q < 4; ++q) k[q] = min(k[q], __ldcg(&part[4 * b + q]));
    for (int q = 0; q < 4; ++q) sh[q][threadIdx.x] = k[q];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 4; ++q) sh[q][threadIdx.x] = min(sh[q][threadIdx.x], sh[q][threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    S->col_done = 0;
    S->col_n_before = n;
    S->ncand = 0;
    if (n == 0) { S->gncells = 0; S->gnx = S->gny = 0; return; }
    const double x0 = vx_dunkey(sh[0][0]), x1 = -vx_dunkey(sh[1][0]);
    const double y0 = vx_dunkey(sh[2][0]), y1 = -vx_dunkey(sh[3][0]);
    // side = the collapse radius: the 3 x 3 search is exact and sees the
    // fewest candidates (a side at the mean spacing, with a quarter of the
    // cells to count and scan, was measured slower: the query dominates)
    double h = sqrt(r2) * (1.0 + 1e-6);
    long long nx = -1, ny = -1;
    for (int it = 0; it < 200; ++it) {
        double fx = floor((x1 - x0) / h) + 1.0, fy = floor((y1 - y0) / h) + 1.0;
        if (fx * fy <= (double)cells_cap) { nx = (long long)fx; ny = (long long)fy; break; }
        h *= 1.25;
    }
    if (nx < 0) { S->err |= VX_DERR_GRID; S->gncells = 0; S->col_done = 1; return; }
    S->gx0 = x0; S->gy0 = y0; S->gh = h;
    S->gnx = nx; S->gny = ny; S->gncells = nx * ny;
}
__global__ void __launch_bounds__(VX_THREADS) k_col_prep(VxView v, VxScalars *S, int reset, double r2,
                                                         long long cells_cap, unsigned long long *part) {
    VX_PDL_WAIT();
    k_col_prep_body(VxBlkB<VX_THREADS, 0>{blockIdx.x, gridDim.x}, v, S, reset, r2, cells_cap, part);
}

__device__ __forceinline__ void vx_cell_of(const VxScalars *S, double x, double y, long long &cx,
                                           long long &cy) {
    cx = (long long)floor((x - S->gx0) / S->gh);
    cy = (long long)floor((y - S->gy0) / S->gh);
    cx = cx < 0 ? 0 : (cx >= S->gnx ? S->gnx - 1 : cx);
    cy = cy < 0 ? 0 : (cy >= S->gny ? S->gny - 1 : cy);
}

VX_DEVK void k_col_count_body(VxBlkB<0, 0> vb, const VxView &v, const VxScalars *S, int *cellid, int *cnt, int *in_cnt,
                              int *has_app, int *first_app) {
    if (S->col_done) return;
    const long long n = S->n;
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        long long cx, cy;
        vx_cell_of(S, v.x[i * v.ps], v.y[i * v.ps], cx, cy);
        const long long c = cy * S->gnx + cx;
        cellid[i] = (int)c;
        atomicAdd(&cnt[c], 1);
        in_cnt[i] = 0;
        has_app[i] = 0;
        first_app[i] = INT_MAX;
    }
}
__global__ void k_col_count(VxView v, const VxScalars *S, int *cellid, int *cnt, int *in_cnt,
                            int *has_app, int *first_app) {
    VX_PDL_WAIT();
    k_col_count_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, cellid, cnt, in_cnt, has_app, first_app);
}

// Cell starts: exclusive scan of the counts in one pass, start[gncells] = n.
VX_DEVK void k_col_scan_body(VxBlkB<VX_SCAN_T, 0> vb, VxScalars *S, const int *cnt, int *start,
                             unsigned long long *tiles) {
    if (S->col_done) return;
    const long long nc = S->gncells;
    vx_scan_lookback<VX_CHUNK / VX_SCAN_T>(
        vb.n, nc, S, tiles, [&](long long i) { return cnt[i]; },
        [&](long long i0, const unsigned *val, long long run) {
#pragma unroll
            for (int q = 0; q < VX_CHUNK / VX_SCAN_T; ++q) {
                if (i0 + q < nc) start[i0 + q] = (int)run;
                run += val[q];
            }
        },
        [&](long long tot) { start[nc] = (int)tot; });
}
__global__ void __launch_bounds__(VX_SCAN_T) k_col_scan(VxScalars *S, const int *cnt, int *start,
                                                        unsigned long long *tiles) {
    VX_PDL_WAIT();
    k_col_scan_body(VxBlkB<VX_SCAN_T, 0>{blockIdx.x, gridDim.x}, S, cnt, start, tiles);
}

// A slot of the cell-sorted copy: position, strength and index of the vortex
// (32 bytes, one DRAM sector, written by one thread).
struct __align__(32) ColRec {
    double x, y, g;
    long long i;
};

// Each cell's slots from its start, counting its count back down to zero
// (the zero the next pass's count starts from); the slot gets a copy of the
// vortex (ColRec), so that the query reads its candidates as contiguous runs.
VX_DEVK void k_col_scatter_body(VxBlkB<0, 0> vb, const VxView &v, const VxScalars *S, const int *cellid, const int *start,
                                int *cnt, ColRec *rec) {
    if (S->col_done) return;
    const long long n = S->n;
    for (long long i = vb.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)vb.n * blockDim.x) {
        const int c = cellid[i];
        const int k = start[c] + atomicSub(&cnt[c], 1) - 1;
        double2 *r = reinterpret_cast<double2 *>(rec + k);
        r[0] = make_double2(v.x[i * v.ps], v.y[i * v.ps]);
        r[1] = make_double2(v.g[i * v.ps], __longlong_as_double(i));
    }
}
__global__ void k_col_scatter(VxView v, const VxScalars *S, const int *cellid, const int *start, int *cnt,
                              ColRec *rec) {
    VX_PDL_WAIT();
    k_col_scatter_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, v, S, cellid, start, cnt, rec);
}

// COL[i] = smallest j > i in the 3x3 cell neighbourhood that qualifies.  The
// targets are taken in cell order (slot k0 of the cell-sorted copy), so
// neighbouring threads read the same cells and sources, all as contiguous
// runs of the copy (a row's three cells are one run); each target's answer
// does not depend on the order.  The target's cell is recomputed from its
// position by the count's expression.
template <int PASS>
VX_DEVK void k_col_query_body(VxBlkB<VX_THREADS, 4> vb, const VxParams &p, VxScalars *S, const int *start, const ColRec *rec,
                              int *col, int *in_cnt, int *cand) {
    if (S->col_done) return;
    const long long n = S->n;
    const long long gnx = S->gnx, gny = S->gny;
    const double rd2 = p.r_diff2, rs2 = p.r_same2, mvg = p.max_ve_g;
    for (long long k0 = vb.x * (long long)blockDim.x + threadIdx.x; k0 < n;
         k0 += (long long)vb.n * blockDim.x) {
        const double2 m0 = reinterpret_cast<const double2 *>(rec + k0)[0];
        const double2 m1 = reinterpret_cast<const double2 *>(rec + k0)[1];
        const double xi = m0.x, yi = m0.y, gi = m1.x;
        const long long i = __double_as_longlong(m1.y);
        long long cx, cy;
        vx_cell_of(S, xi, yi, cx, cy);
        int best = INT_MAX;
        for (long long yy = max(cy - 1, 0LL); yy <= min(cy + 1, gny - 1); ++yy) {
            const long long r0 = yy * gnx;
            const int k1 = start[r0 + min(cx + 1, gnx - 1) + 1];
            for (int k = start[r0 + max(cx - 1, 0LL)]; k < k1; ++k) {
                const double2 q1 = reinterpret_cast<const double2 *>(rec + k)[1];
                const int j = (int)__double_as_longlong(q1.y);
                if (j <= i || j >= best) continue;
                const double2 q0 = reinterpret_cast<const double2 *>(rec + k)[0];
                const double gj = q1.x;
                const double dx = xi - q0.x, dy = yi - q0.y;
                const double r2 = fma(dx, dx, dy * dy);
                bool ok;
                if (PASS == 1) ok = (gi * gj < 0) && (r2 < rd2);
                else ok = (gi * gj > 0) && (r2 < rs2) && (fabs(gi + gj) < mvg);
                if (ok) best = j;
            }
        }
        if (best != INT_MAX) {
            col[i] = best;
            atomicAdd(&in_cnt[best], 1);
            const int slot = atomicAdd(&S->ncand, 1);
            cand[slot] = (int)i;
        } else {
            col[i] = -1;
        }
    }
}
template <int PASS>
__global__ void k_col_query(VxParams p, VxScalars *S, const int *start, const ColRec *rec, int *col, int *in_cnt,
                            int *cand) {
    VX_PDL_WAIT();
    k_col_query_body<PASS>(VxBlkB<VX_THREADS, 4>{blockIdx.x, gridDim.x}, p, S, start, rec, col, in_cnt, cand);
}

// Settles the candidates in one block: rounds over the candidate list decide
// each one (cstate: 0 undecided, 1 applied, 2 consumed before its turn), then
// every applied candidate's merged vortex is computed from the positions as
// they were, then written (after a barrier: a merge may read a partner that
// another merge removes).
template <int PASS>
VX_DEVK void k_col_settle_body(VxBlkB<1024, 0> vb, const VxView &v, VxScalars *S, const int *cand, const int *col,
                               int *in_cnt, int *has_app, int *first_app, int *cstate, int *cdec, double *mx,
                               double *my, double *mg) {
    if (S->col_done) return;
    __shared__ int undecided;
    const int nc = S->ncand;
    for (int k = threadIdx.x; k < nc; k += blockDim.x) cstate[k] = 0;
    __syncthreads();
    const int max_rounds = nc + 2;
    int round = 0;
    for (; round < max_rounds; ++round) {
        for (int k = threadIdx.x; k < nc; k += blockDim.x) {
            int d = 0;
            if (cstate[k] == 0) {
                const int i = cand[k];
                if (has_app[i]) d = 2;
                else if (in_cnt[i] == 0) d = 1;
            }
            cdec[k] = d;
        }
        if (threadIdx.x == 0) undecided = 0;
        __syncthreads();
        for (int k = threadIdx.x; k < nc; k += blockDim.x) {
            if (cstate[k] != 0) continue;
            const int d = cdec[k];
            if (d == 0) { atomicAdd(&undecided, 1); continue; }
            cstate[k] = d;
            const int i = cand[k], j = col[i];
            atomicSub(&in_cnt[j], 1);
            if (d == 1) {
                has_app[j] = 1;
                atomicMin(&first_app[j], i);
            }
        }
        __syncthreads();
        if (undecided == 0) break;
        __syncthreads();
    }
    if (round >= max_rounds) {
        if (threadIdx.x == 0) {
            S->err |= VX_DERR_RESOLVE;
            S->col_done = 1;
        }
        return;
    }
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
        if (cstate[k] != 1) continue;
        const long long i = cand[k], j = col[i];
        const double xi = v.x[i * v.ps], yi = v.y[i * v.ps], gi = v.g[i * v.ps];
        double xj = 1e10, yj = 1e10, gj = 0.0;
        if (first_app[j] == i) { xj = v.x[j * v.ps]; yj = v.y[j * v.ps]; gj = v.g[j * v.ps]; }
        if (PASS == 1) {
            const double ai = fabs(gi), aj = fabs(gj);
            const double mn = ai + aj;
            mx[k] = (xi * ai + xj * aj) / fabs(mn);
            my[k] = (yi * ai + yj * aj) / fabs(mn);
            mg[k] = gi + gj;
        } else {
            const double ng = gi + gj;
            mx[k] = (xi * gi + xj * gj) / ng;
            my[k] = (yi * gi + yj * gj) / ng;
            mg[k] = ng;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
        if (cstate[k] != 1) continue;
        const long long i = cand[k], j = col[i];
        v.x[i * v.ps] = mx[k]; v.y[i * v.ps] = my[k]; v.g[i * v.ps] = mg[k];
        v.x[j * v.ps] = 1e10; v.y[j * v.ps] = 1e10; v.g[j * v.ps] = 0.0;
    }
}
template <int PASS>
__global__ void __launch_bounds__(1024) k_col_settle(VxView v, VxScalars *S, const int *cand, const int *col,
                                                     int *in_cnt, int *has_app, int *first_app, int *cstate,
                                                     int *cdec, double *mx, double *my, double *mg) {
    VX_PDL_WAIT();
    k_col_settle_body<PASS>(VxBlkB<1024, 0>{blockIdx.x, gridDim.x}, v, S, cand, col, in_cnt, has_app, first_app,
                            cstate, cdec, mx, my, mg);
}

cudaError_t vx_launch_collapse(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                               VxWork &w, int pass, int n_col) {
    const double r2 = pass == 1 ? p.r_diff2 : p.r_same2;
    if (!(r2 > 0.0) || n_col <= 0) return cudaSuccess;   // no pair can qualify
    const int grid = std::min(L.num_sms * 4, VX_RED_BLOCKS);   // 4 box keys per block
    // the cell-sorted copy (32 bytes a vortex) lives in the pair kernels'
    // partial-sum buffer, unused by collapse (at least 5 doubles a slot)
    ColRec *rec = reinterpret_cast<ColRec *>(w.part);
    for (int cc = 0; cc < n_col; ++cc) {
        vx_launch<k_col_prep, k_col_prep_body>(L, grid, VX_THREADS, 0, v, S, cc == 0, r2, w.cells_cap, w.box);
        vx_launch<k_col_count, k_col_count_body>(L, grid, VX_THREADS, 0, v, S, w.cellid, w.cell_cnt, w.in_cnt, w.has_app, w.first_app);
        vx_launch<k_col_scan, k_col_scan_body>(L, grid, VX_SCAN_T, 0, S, w.cell_cnt, w.cell_start, w.scan_tiles);
        vx_launch<k_col_scatter, k_col_scatter_body>(L, grid, VX_THREADS, 0, v, S, w.cellid, w.cell_start, w.cell_cnt, rec);
        if (pass == 1) {
            vx_launch<k_col_query<1>, k_col_query_body<1>>(L, grid, VX_THREADS, 0, p, S, w.cell_start, (const ColRec *)rec, w.col, w.in_cnt, w.cand);
            vx_launch<k_col_settle<1>, k_col_settle_body<1>>(L, 1, 1024, 0, v, S, w.cand, w.col, w.in_cnt, w.has_app, w.first_app, w.cstate, w.cdec, w.mx, w.my, w.mg);
        } else {
            vx_launch<k_col_query<2>, k_col_query_body<2>>(L, grid, VX_THREADS, 0, p, S, w.cell_start, (const ColRec *)rec, w.col, w.in_cnt, w.cand);
            vx_launch<k_col_settle<2>, k_col_settle_body<2>>(L, 1, 1024, 0, v, S, w.cand, w.col, w.in_cnt, w.has_app, w.first_app, w.cstate, w.cdec, w.mx, w.my, w.mg);
        }
        vx_launch_compact_skip(L, p, v, S, w, &S->col_done);
    }
    return cudaGetLastError();
}
