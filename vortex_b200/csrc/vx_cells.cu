// vx_cells.cu — uniform cell grid with a stable cell ordering, and the
// bulk-form vortex diffusion over it.
//
// The diffusive velocity (reference diffusion_Kernel, src/kernel.cu:985-1029)
// sums G_j exp(-r/d_i) terms; beyond r = c d_i (c = diff_cutoff, default 30)
// a term is below e^-c of its strength, so the bulk form sums only those
// pairs.  Particles are binned into square cells of side h (h tracks the
// mean 3-nearest distance), cell ids are sorted stably (radix sort: equal ids
// keep index order, so every sum has a fixed order), and the cell-sorted
// particles (x, y, G, d) are gathered into one float4 per particle.
//
// Work item = up to 256 cell-sorted targets of one grid row.  The item scans
// the rows within its largest cut-off radius; in every row the columns it
// needs are one contiguous range of the sorted array, staged through shared
// memory 256 sources at a time.  Each target is owned by one item, so the
// velocity is updated in place with no partial sums.
#include "vx_internal.cuh"

int vx_radix_sort(const VxLaunch &L, const long long *d_n, unsigned *k0, int *v0, unsigned *k1, int *v1,
                  int nbits, int *hist, long long *off, long long tiles_cap);

constexpr int CG_T = 256;

__global__ void k_cg_begin(VxScalars *S) {
    S->cb[0] = S->cb[1] = S->cb[2] = S->cb[3] = ~0ull;
}

// Bounding box of the live particles and per-block sums of d (fixed grid:
// the mean below is reproducible).
__global__ void __launch_bounds__(CG_T) k_cg_bbox(VxView v, VxScalars *S, double *red) {
    __shared__ unsigned long long sk[4][CG_T];
    __shared__ double sd[CG_T];
    const long long n = S->n;
    unsigned long long k[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    double dsum = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
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
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; ++q) atomicMin(&S->cb[q], sk[q][0]);
        red[blockIdx.x] = sd[0];
    }
}

// Cell side h = c * mean(d) / 4, grown until the grid fits cells_cap.
__global__ void k_cg_params(VxScalars *S, const double *red, int nblocks, double cutoff, long long cells_cap) {
    const long long n = S->n;
    S->cnitems = 0;
    if (n == 0) { S->cncells = 0; S->cnx = S->cny = 0; return; }
    double dsum = 0.0;
    for (int b = 0; b < nblocks; ++b) dsum += red[b];
    const double x0 = vx_dunkey(S->cb[0]), x1 = -vx_dunkey(S->cb[1]);
    const double y0 = vx_dunkey(S->cb[2]), y1 = -vx_dunkey(S->cb[3]);
    double h = cutoff * (dsum / (double)n) / 4.0;
    if (!(h > 0.0)) h = 1e-3;
    long long nx = -1, ny = -1;
    for (int it = 0; it < 400; ++it) {
        const double fx = floor((x1 - x0) / h) + 1.0, fy = floor((y1 - y0) / h) + 1.0;
        if (fx * fy <= (double)cells_cap) { nx = (long long)fx; ny = (long long)fy; break; }
        h *= 1.25;
    }
    if (nx < 0) { S->err |= VX_DERR_GRID; S->cncells = 0; return; }
    S->cx0 = x0; S->cy0 = y0; S->ch = h;
    S->cnx = nx; S->cny = ny; S->cncells = nx * ny;
}

__device__ __forceinline__ long long cg_cell(const VxScalars *S, double x, double y) {
    long long cx = (long long)floor((x - S->cx0) / S->ch);
    long long cy = (long long)floor((y - S->cy0) / S->ch);
    cx = cx < 0 ? 0 : (cx >= S->cnx ? S->cnx - 1 : cx);
    cy = cy < 0 ? 0 : (cy >= S->cny ? S->cny - 1 : cy);
    return cy * S->cnx + cx;
}

__global__ void k_cg_zero(const VxScalars *S, int *cnt) {
    const long long nc = S->cncells;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
         c += (long long)gridDim.x * blockDim.x)
        cnt[c] = 0;
}

__global__ void k_cg_cellid(VxView v, const VxScalars *S, unsigned *key, int *val, int *cnt) {
    const long long n = S->n;
    if (S->cncells == 0) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long c = cg_cell(S, v.x[i * v.ps], v.y[i * v.ps]);
        key[i] = (unsigned)c;
        val[i] = (int)i;
        atomicAdd(&cnt[c], 1);
    }
}

// Exclusive scan of cnt[0, len) into start[], start[len] = total: chunk
// sums, one-block scan of the chunk sums, per-chunk apply.
__global__ void __launch_bounds__(CG_T) k_scan_sum(const long long *len_p, const int *cnt, int *csum) {
    __shared__ int sh[CG_T];
    const long long len = *len_p, nch = vx_ceil_div(len, VX_CHUNK);
    for (long long c = blockIdx.x; c < nch; c += gridDim.x) {
        int k = 0;
        for (long long q = c * VX_CHUNK + threadIdx.x; q < min(len, (c + 1) * VX_CHUNK); q += blockDim.x) k += cnt[q];
        sh[threadIdx.x] = k;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) csum[c] = sh[0];
        __syncthreads();
    }
}

__global__ void k_scan_top(const long long *len_p, const int *csum, long long *coff) {
    __shared__ long long sh[1024];
    __shared__ long long carry;
    const long long nch = vx_ceil_div(*len_p, VX_CHUNK);
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < nch; base += blockDim.x) {
        const long long c = base + threadIdx.x;
        const long long val = c < nch ? csum[c] : 0;
        sh[threadIdx.x] = val;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {
            long long t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (c < nch) coff[c] = carry + sh[threadIdx.x] - val;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += sh[threadIdx.x];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(CG_T) k_scan_apply(const long long *len_p, const int *cnt, const long long *coff,
                                                     int *start, const long long *total_p) {
    constexpr int PER = VX_CHUNK / CG_T;
    __shared__ int sh[CG_T];
    const long long len = *len_p, nch = vx_ceil_div(len, VX_CHUNK);
    if (blockIdx.x == 0 && threadIdx.x == 0) start[len] = (int)*total_p;
    for (long long c = blockIdx.x; c < nch; c += gridDim.x) {
        const long long b = c * VX_CHUNK + (long long)threadIdx.x * PER;
        int val[PER], loc = 0;
#pragma unroll
        for (int q = 0; q < PER; ++q) { val[q] = (b + q < len) ? cnt[b + q] : 0; loc += val[q]; }
        sh[threadIdx.x] = loc;
        __syncthreads();
        for (int o = 1; o < CG_T; o <<= 1) {
            int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        long long run = coff[c] + sh[threadIdx.x] - loc;
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (b + q < len) start[b + q] = (int)run;
            run += val[q];
        }
    }
}

// Cell-sorted particles (x, y relative to their cell centre, G, d).  Keeping
// FP32 positions relative to the cell keeps the pair differences accurate to
// FP32 rounding of the local spacing rather than of the absolute position.
__global__ void k_cg_gather(VxView v, const VxScalars *S, const int *sorted, const unsigned *skey, float4 *srt) {
    const long long n = S->n, nx = S->cnx;
    const double h = S->ch;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const long long i = sorted[k];
        const long long c = skey[k];
        const double ccx = S->cx0 + ((double)(c % nx) + 0.5) * h, ccy = S->cy0 + ((double)(c / nx) + 0.5) * h;
        srt[k] = make_float4((float)(v.x[i * v.ps] - ccx), (float)(v.y[i * v.ps] - ccy), (float)v.g[i * v.ps],
                             (float)v.d[i]);
    }
}

// Exclusive scan of the per-row item counts (single block, runs per thread).
__global__ void k_cg_row_scan(const VxScalars *S, const int *in, long long *out) {
    __shared__ long long sh[1024];
    const long long len = S->cny;
    const long long per = vx_ceil_div(len, (long long)blockDim.x);
    const long long b = threadIdx.x * per, e = min(len, b + per);
    long long local = 0;
    for (long long q = b; q < e; ++q) local += in[q];
    sh[threadIdx.x] = local;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        long long t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    long long run = sh[threadIdx.x] - local;
    for (long long q = b; q < e; ++q) {
        out[q] = run;
        run += in[q];
    }
}

// Work items: each row's sorted range cut into segments of CG_T targets.
__global__ void k_cg_row_items(const VxScalars *S, const int *start, int *row_items) {
    const long long ny = S->cny, nx = S->cnx;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ny;
         r += (long long)gridDim.x * blockDim.x) {
        const int cnt = start[(r + 1) * nx] - start[r * nx];
        row_items[r] = (cnt + CG_T - 1) / CG_T;
    }
}

__global__ void k_cg_items(VxScalars *S, const int *start, const int *row_items, const long long *row_off,
                           int2 *items, long long items_cap) {
    const long long ny = S->cny, nx = S->cnx;
    if (blockIdx.x == 0 && threadIdx.x == 0 && ny > 0) {
        const long long tot = row_off[ny - 1] + row_items[ny - 1];
        S->cnitems = tot <= items_cap ? tot : 0;
        if (tot > items_cap) S->err |= VX_DERR_GRID;
    }
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ny;
         r += (long long)gridDim.x * blockDim.x) {
        const long long o = row_off[r];
        const int s0 = start[r * nx];
        for (int q = 0; q < row_items[r]; ++q)
            if (o + q < items_cap) items[o + q] = make_int2((int)r, s0 + q * CG_T);
    }
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

// Vortex diffusion over the cell grid (bulk form).
__global__ void __launch_bounds__(CG_T) k_diff_cells(VxParams p, VxView v, VxScalars *S, const float4 *srt,
                                                     const unsigned *skey, const int *sorted, const int *start,
                                                     const int2 *items) {
    __shared__ float4 sm[CG_T];
    __shared__ float s_rmax;
    const long long nitems = S->cnitems, nx = S->cnx, ny = S->cny;
    const float h = (float)S->ch;
    const float cut = (float)p.diff_cutoff;
    const float thr2 = (float)(0.001 * p.eps) * (float)(0.001 * p.eps);
    const float log2e = 1.4426950408889634f;
    for (long long it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 item = items[it];
        const long long row = item.x;
        const long long row_end = start[(row + 1) * nx];
        const long long last = min((long long)item.y + CG_T, row_end);
        const long long t = item.y + threadIdx.x;
        const bool valid = t < last;
        float4 me = valid ? srt[t] : make_float4(0.f, 0.f, 0.f, 1.f);
        // coordinates relative to the centre of the item's first cell
        const long long ocol = (long long)(skey[item.y] % (unsigned)nx);
        if (valid) me.x += (float)((double)((long long)(skey[t] % (unsigned)nx) - ocol) * (double)S->ch);
        const float R = cut * me.w;
        const float R2 = R * R;
        const float ndd = -log2e / me.w;
        __syncthreads();
        if (threadIdx.x == 0) s_rmax = 0.0f;
        __syncthreads();
        if (valid) atomicMax((int *)&s_rmax, __float_as_int(R));   // R >= 0: int order = float order
        __syncthreads();
        const float rmax = s_rmax;
        const long long kk = min((long long)ceilf(rmax / h), max(nx, ny));
        const long long ca = (long long)(skey[item.y] % (unsigned)nx);
        const long long cbb = (long long)(skey[last - 1] % (unsigned)nx);
        const long long c0 = max(ca - kk, 0LL), c1 = min(cbb + kk, nx - 1);
        const long long r0 = max(row - kk, 0LL), r1 = min(row + kk, ny - 1);
        double I2x = 0.0, I2y = 0.0, I1 = 0.0;
        unsigned long long scanned = 0;
        for (long long rr = r0; rr <= r1; ++rr) {
            const long long j0 = start[rr * nx + c0], j1 = start[rr * nx + c1 + 1];
            scanned += (unsigned long long)(j1 - j0);
            const float oy = (float)((double)(rr - row) * (double)S->ch);
            for (long long jt = j0; jt < j1; jt += CG_T) {
                __syncthreads();
                if (jt + threadIdx.x < j1) {
                    float4 q = srt[jt + threadIdx.x];
                    const long long sc = (long long)(skey[jt + threadIdx.x] % (unsigned)nx);
                    q.x += (float)((double)(sc - ocol) * (double)S->ch);
                    q.y += oy;
                    sm[threadIdx.x] = q;
                }
                __syncthreads();
                const int cnt = (int)min((long long)CG_T, j1 - jt);
                float s2x = 0.f, s2y = 0.f, s1 = 0.f;
#pragma unroll 4
                for (int q = 0; q < cnt; ++q) {
                    const float4 s = sm[q];
                    const float dx = me.x - s.x, dy = me.y - s.y;
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
                I2x += (double)s2x; I2y += (double)s2y; I1 += (double)s1;
            }
        }
        if (threadIdx.x == 0) atomicAdd(&S->pairs_diff, scanned * (unsigned long long)(last - item.y));
        if (valid && fabs(I1) > 1e-5) {
            const long long i = sorted[t];
            const double dd = (double)me.w;
            v.vx[i * v.vs] += -p.nu * I2x / (I1 * dd);
            v.vy[i * v.vs] += -p.nu * I2y / (I1 * dd);
        }
    }
}

static int bits_for(long long cells) {
    int b = 1;
    while ((1LL << b) < cells && b < 32) ++b;
    return ((b + 7) / 8) * 8;
}

// Build the grid and run the bulk diffusion.  Scratch from w; the collapse
// chunk arrays are reused (the passes run one after the other on one stream).
cudaError_t vx_launch_diffusion_cells(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                                      VxWork &w) {
    const int grid = L.num_sms * 4;
    k_cg_begin<<<1, 1, 0, L.stream>>>(S); VX_COUNT(L);
    k_cg_bbox<<<VX_RED_BLOCKS, CG_T, 0, L.stream>>>(v, S, w.red); VX_COUNT(L);
    k_cg_params<<<1, 1, 0, L.stream>>>(S, w.red, VX_RED_BLOCKS, p.diff_cutoff, w.cells_cap); VX_COUNT(L);
    k_cg_zero<<<grid, CG_T, 0, L.stream>>>(S, w.cg_cnt); VX_COUNT(L);
    k_cg_cellid<<<grid, CG_T, 0, L.stream>>>(v, S, w.key0, w.val0, w.cg_cnt); VX_COUNT(L);
    k_scan_sum<<<grid, CG_T, 0, L.stream>>>(&S->cncells, w.cg_cnt, w.cell_chunk_cnt); VX_COUNT(L);
    k_scan_top<<<1, 1024, 0, L.stream>>>(&S->cncells, w.cell_chunk_cnt, w.cell_chunk_off); VX_COUNT(L);
    k_scan_apply<<<grid, CG_T, 0, L.stream>>>(&S->cncells, w.cg_cnt, w.cell_chunk_off, w.cg_start, &S->n);
    VX_COUNT(L);
    const int nb = bits_for(w.cells_cap);
    const int cur = vx_radix_sort(L, &S->n, w.key0, w.val0, w.key1, w.val1, nb, w.rs_hist, w.rs_off,
                                  w.rs_tiles_cap);
    const unsigned *skey = cur ? w.key1 : w.key0;
    const int *sorted = cur ? w.val1 : w.val0;
    k_cg_gather<<<grid, CG_T, 0, L.stream>>>(v, S, sorted, skey, w.srt); VX_COUNT(L);
    k_cg_row_items<<<grid, CG_T, 0, L.stream>>>(S, w.cg_start, w.row_items); VX_COUNT(L);
    k_cg_row_scan<<<1, 1024, 0, L.stream>>>(S, w.row_items, w.row_item_off); VX_COUNT(L);
    k_cg_items<<<grid, CG_T, 0, L.stream>>>(S, w.cg_start, w.row_items, w.row_item_off, w.items, w.items_cap);
    VX_COUNT(L);
    VX_EV(L, 2);
    k_diff_cells<<<L.num_sms * 8, CG_T, 0, L.stream>>>(p, v, S, w.srt, skey, sorted, w.cg_start, w.items);
    VX_EV(L, 3);
    VX_COUNT(L);
    return cudaGetLastError();
}
