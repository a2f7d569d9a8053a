// vx_engine.cu — the vx_sim handle and the native C ABI (include/vortex_b200.h).
//
// A handle keeps one body resident on its device: panels, the inverted
// panel system, SoA particle arrays (x, y, G, Vx, Vy, d) and scratch.  The
// live count stays in device memory; the host keeps only an upper bound
// (births add P per step, nothing else adds) and reads the true count back
// when the store may have to grow.  A step is launched as a fixed sequence,
// so after the first call it is recorded into a CUDA graph and replayed.
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cxxabi.h>

#include <algorithm>
#include <map>
#include <string>
#include <cstddef>
#include <vector>

#include "vx_sim.cuh"

static thread_local std::string g_err;

void vx_set_error(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

extern "C" const char *vx_last_error(void) { return g_err.c_str(); }

// Stream-ordered allocations (growth of the particle arrays, the batch's
// gather buffer) come from the device's default pool.  With the pool's
// default release threshold of 0, every stream or event synchronize hands the
// pool's free memory back to the driver, so the next growth maps fresh pages
// inside a step; keeping the freed memory in the pool makes a regrowth reuse it.
void vx_keep_pool(int device) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) { cudaGetLastError(); return; }
    unsigned long long keep = ~0ull;
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) cudaGetLastError();
}

// A destroyed handle's stream-ordered memory goes back to the driver (the
// pool keeps it otherwise, out of reach of plain cudaMalloc callers).
void vx_trim_pool(int device) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) { cudaGetLastError(); return; }
    if (cudaMemPoolTrimTo(pool, 0) != cudaSuccess) cudaGetLastError();
}

extern "C" const char *vx_status_str(vx_status s) {
    switch (s) {
    case VX_OK: return "ok";
    case VX_ERR_CUDA: return "CUDA error";
    case VX_ERR_ARG: return "bad argument";
    case VX_ERR_IO: return "I/O error";
    case VX_ERR_SINGULAR: return "singular panel system";
    case VX_ERR_NOMEM: return "out of memory";
    case VX_ERR_DEVICE: return "device error flag";
    case VX_ERR_BUDGET: return "HBM budget exceeded";
    }
    return "unknown";
}

#define CU(call)                                                                            \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            vx_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? VX_ERR_NOMEM : VX_ERR_CUDA;            \
        }                                                                                   \
    } while (0)

static VxLaunch launch_of(vx_sim *s) {
    VxLaunch L;
    L.stream = s->stream;
    L.launches = &s->launches;
    L.num_sms = s->num_sms;
    return L;
}

static VxView view_of(vx_sim *s) {
    VxView v;
    v.x = s->x; v.y = s->y; v.g = s->g; v.ps = 1;
    v.vx = s->vx; v.vy = s->vy; v.vs = 1;
    v.d = s->d;
    return v;
}

// ---------------------------------------------------------------------------
// parameters (reference init_device_conf_values, src/unit_1.cu:1220-1252)
void vx_params_from_conf(const vx_conf *c, const vx_panel *pan, int P, VxParams *p) {
    memset(p, 0, sizeof(*p));
    p->dt = c->dt;
    p->nu = c->viscosity;
    p->rho = c->rho;
    p->eps = c->ve_size;
    p->eps2 = c->ve_size * c->ve_size;
    p->r_diff2 = c->r_col_diff_sign * c->r_col_diff_sign * p->eps2;
    p->r_same2 = c->r_col_same_sign * c->r_col_same_sign * p->eps2;
    p->max_ve_g = c->max_ve_g;
    p->x_min = c->x_min; p->x_max = c->x_max; p->y_min = c->y_min; p->y_max = c->y_max;
    // profile bbox from the left endpoints, started from the window's
    // opposite edges (src/main.c:235-254)
    double xmn = c->x_max, xmx = c->x_min, ymn = c->y_max, ymx = c->y_min;
    double bx0 = 1e300, bx1 = -1e300, by0 = 1e300, by1 = -1e300, lmax = 0.0;
    for (int i = 0; i < P; ++i) {
        double xx = pan[i].left[0], yy = pan[i].left[1];
        if (xx < xmn) xmn = xx;
        if (xx > xmx) xmx = xx;
        if (yy < ymn) ymn = yy;
        if (yy > ymx) ymx = yy;
        bx0 = std::min(bx0, pan[i].birth[0]); bx1 = std::max(bx1, pan[i].birth[0]);
        by0 = std::min(by0, pan[i].birth[1]); by1 = std::max(by1, pan[i].birth[1]);
        lmax = std::max(lmax, pan[i].length);
    }
    p->px_min = xmn; p->px_max = xmx; p->py_min = ymn; p->py_max = ymx;
    // a particle farther than 5 L_max from every birth point gets no wall term
    const double m = 5.0 * lmax * (1.0 + 1e-9) + 1e-12;
    p->wall_x0 = bx0 - m; p->wall_x1 = bx1 + m; p->wall_y0 = by0 - m; p->wall_y1 = by1 + m;
    p->rc_x = c->rc_x; p->rc_y = c->rc_y;
    p->drop_eps = c->drop_eps;
    p->diff_cutoff = c->diff_cutoff;
    // body centre and radius (all endpoints) for the birth far field: the
    // expansion about the centre converges at ratio 1/2 on the panels for
    // vortices beyond twice the radius
    if (P > 0) {
        double ex0 = 1e300, ex1 = -1e300, ey0 = 1e300, ey1 = -1e300;
        for (int i = 0; i < P; ++i)
            for (const double *e : {pan[i].left, pan[i].right}) {
                ex0 = std::min(ex0, e[0]); ex1 = std::max(ex1, e[0]);
                ey0 = std::min(ey0, e[1]); ey1 = std::max(ey1, e[1]);
            }
        p->bc_x = 0.5 * (ex0 + ex1);
        p->bc_y = 0.5 * (ey0 + ey1);
        double r2 = 0.0;
        for (int i = 0; i < P; ++i)
            for (const double *e : {pan[i].left, pan[i].right})
                r2 = std::max(r2, (e[0] - p->bc_x) * (e[0] - p->bc_x) + (e[1] - p->bc_y) * (e[1] - p->bc_y));
        p->b_rfar2 = VX_BF_RHO * VX_BF_RHO * r2 * (1.0 + 1e-12);
        p->birth_far = (c->precision == VX_PREC_FP32 && c->fmm) ? 1 : 0;
    }
    p->fmm_leaf = c->fmm_leaf > 0 ? c->fmm_leaf : 32;
    p->fmm_p = vx_fmm_order_ok(c->fmm_p) ? c->fmm_p : VX_FMM_P;
    p->P = P;
    p->n_of_points = (int)c->n_of_points;
    p->birth_mode = c->birth_offset_mode;
    p->prec = c->precision;
}

extern "C" vx_status vx_conf_default(vx_conf *c) {
    if (!c) return VX_ERR_ARG;
    memset(c, 0, sizeof(*c));
    c->log_level = 3;
    c->v_inf_incr_steps = 1;
    c->precision = VX_PREC_FP64;
    c->birth_offset_mode = VX_BIRTH_REF;
    c->drop_eps = 1e-12;
    c->diff_cutoff = 16.0;
    c->fmm = 1;
    c->fmm_leaf = 32;
    return VX_OK;
}

// ---------------------------------------------------------------------------
__global__ void k_fill_tail(double *x, double *y, double *g, long long from, long long to) {
    VX_PDL_WAIT();
    for (long long i = from + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < to;
         i += (long long)gridDim.x * blockDim.x) {
        x[i] = 4.0e5 + (double)i;
        y[i] = 4.0e5 + (double)i;
        g[i] = 0.0;
    }
}

// Device allocation of `count` elements, counted (rounded to the 256-byte
// allocation granularity) into *bytes; with allocs == nullptr only counted,
// or, with a carving cursor, taken from one block allocated before (a
// body's scratch is one allocation: a growth that re-sizes it costs two
// allocator calls, not forty, which matters when a batch of bodies grows at
// once).  With a stream the allocation is stream-ordered (cudaMallocAsync):
// growing one body's store then never waits for the other bodies' streams,
// as a cudaFree would.
struct WorkCarve {
    char *next;
};
template <typename T>
static vx_status dalloc(std::vector<void *> *allocs, long long *bytes, T **p, long long count,
                        cudaStream_t stream, WorkCarve *cv = nullptr) {
    void *q = nullptr;
    if (count < 1) count = 1;
    const long long nb = ((long long)sizeof(T) * count + 255) / 256 * 256;
    *bytes += nb;
    if (cv) {
        *p = reinterpret_cast<T *>(cv->next);
        cv->next += nb;
        return VX_OK;
    }
    if (!allocs) { *p = nullptr; return VX_OK; }
    if (stream)
        CU(cudaMallocAsync(&q, sizeof(T) * (size_t)count, stream));
    else
        CU(cudaMalloc(&q, sizeof(T) * (size_t)count));
    allocs->push_back(q);
    *p = (T *)q;
    return VX_OK;
}

// dalloc, then zeroed in stream order.
template <typename T>
static vx_status dalloc_zero(std::vector<void *> *allocs, long long *bytes, T **p, long long count,
                             cudaStream_t stream, WorkCarve *cv = nullptr) {
    vx_status st = dalloc(allocs, bytes, p, count, stream, cv);
    if (st != VX_OK || (!allocs && !cv)) return st;
    CU(cudaMemsetAsync(*p, 0, sizeof(T) * (size_t)(count < 1 ? 1 : count), stream));
    return VX_OK;
}

void vx_work_free(VxWork &w, std::vector<void *> &allocs, cudaStream_t stream) {
    for (void *q : allocs) {
        if (stream)
            cudaFreeAsync(q, stream);
        else
            cudaFree(q);
    }
    allocs.clear();
    memset(&w, 0, sizeof(w));
}

// Scratch for a particle capacity `cap` and a panel count padded to P32
// (allocs == nullptr: only count the bytes into w.bytes).
static vx_status work_alloc_impl(VxWork &w, std::vector<void *> *allocs, long long cap, int P32, int num_sms,
                                 cudaStream_t stream, int fmm_p, WorkCarve *cv = nullptr) {
    w.cap = cap;
    w.fmm_p = fmm_p;
    w.bytes = 0;
    const long long nch = cap / VX_CHUNK + 2;
    vx_status st;
#define A(ptr, n) if ((st = dalloc(allocs, &w.bytes, &(ptr), (n), stream, cv)) != VX_OK) return st
    A(w.cmp_cnt, nch); A(w.cmp_off, nch);
    A(w.hole_pos, cap); A(w.hole_src, cap); A(w.tail_src, cap);
    A(w.hx, cap); A(w.hy, cap); A(w.hg, cap); A(w.tx, cap); A(w.ty, cap);
    w.cells_cap = std::max(4 * cap, 65536LL);
    A(w.cellid, cap); A(w.cell_start, w.cells_cap + 1); A(w.sorted, cap);
    // the collapse grid's cell counts are zero between passes (the scatter
    // that consumes them counts them back down), so they start at zero
    if ((st = dalloc_zero(allocs, &w.bytes, &w.cell_cnt, w.cells_cap, stream, cv)) != VX_OK) return st;
    A(w.col, cap); A(w.in_cnt, cap); A(w.has_app, cap); A(w.first_app, cap);
    A(w.cand, cap); A(w.cstate, cap); A(w.cdec, cap);
    A(w.mx, cap); A(w.my, cap); A(w.mg, cap);
    // pair partials: K * n <= num_sms*8*tile + n for the split K the launchers pick
    w.part_cap = 5LL * ((long long)num_sms * 8 * 1024 + cap + 1024);
    A(w.part, w.part_cap);
    A(w.src32, cap);
    w.rhs_part_cap = (long long)num_sms * 4 * P32 * 2;
    A(w.rhs_part, w.rhs_part_cap);
    A(w.R, P32); A(w.gamma, P32);
    A(w.bf_part, 2LL * VX_BF_P * VX_BF_MAX_BLOCKS); A(w.bf_cnt, VX_BF_MAX_BLOCKS);
    A(w.bf_off, VX_BF_MAX_BLOCKS + 1); A(w.bf_near, cap); A(w.bf_coef, 2 * VX_BF_P);
    A(w.red, VX_RED_BLOCKS * 4); A(w.box, VX_RED_BLOCKS * 4);
    // neighbour-list grid of the bulk form
    A(w.key0, cap); A(w.key1, cap); A(w.val0, cap); A(w.val1, cap);
    A(w.cg_start, w.cells_cap + 1);
    // the diffusion grid's cell counts are zero between steps (its bucket
    // order leaves them so), so they start at zero
    if ((st = dalloc_zero(allocs, &w.bytes, &w.cg_cnt, w.cells_cap, stream, cv)) != VX_OK) return st;
    A(w.srt, cap);
    w.items_cap = cap / 32 + w.cells_cap + 2;
    A(w.items, w.items_cap);
    A(w.cg_wide, cap); A(w.cg_huge, cap); A(w.bk_mid, cap / 16 + 2); A(w.bk_big, cap / 128 + 2);
    // quadtree of the bulk-form Biot-Savart
    w.fmm_lmax = vx_fmm_max_level(cap);
    A(w.fmm_cnt, vx_fmm_cells(w.fmm_lmax));
    A(w.fmm_start, (1LL << (2 * w.fmm_lmax)) + 1);
    A(w.fmm_flags, cap); A(w.fmm_brute, cap);
    A(w.fmm_sub_cnt, 1LL << (2 * (w.fmm_lmax + 1)));
    A(w.fmm_sub_start, (1LL << (2 * (w.fmm_lmax + 1))) + 1);
    A(w.fmm_M, 2LL * fmm_p * vx_fmm_cells(w.fmm_lmax));
    A(w.fmm_L, 2LL * fmm_p * vx_fmm_cells(w.fmm_lmax));
    // the longest scan: cells of a grid, quarter-leaves, or rows at one per thread
    w.scan_tiles_cap = std::max(std::max(w.cells_cap, 1LL << (2 * (w.fmm_lmax + 1))), cap) / VX_SCAN_T + 2;
    if ((st = dalloc_zero(allocs, &w.bytes, &w.scan_tiles, w.scan_tiles_cap, stream, cv)) != VX_OK) return st;
#undef A
    return VX_OK;
}

vx_status vx_work_alloc(VxWork &w, std::vector<void *> &allocs, long long cap, int P32, int num_sms,
                        cudaStream_t stream, int fmm_p) {
    vx_work_free(w, allocs, stream);
    const long long bytes = vx_work_bytes(cap, P32, num_sms, fmm_p);
    void *block = nullptr;
    if (stream)
        CU(cudaMallocAsync(&block, (size_t)bytes, stream));
    else
        CU(cudaMalloc(&block, (size_t)bytes));
    allocs.push_back(block);
    WorkCarve cv{static_cast<char *>(block)};
    return work_alloc_impl(w, nullptr, cap, P32, num_sms, stream, fmm_p, &cv);
}

long long vx_work_bytes(long long cap, int P32, int num_sms, int fmm_p) {
    VxWork w;
    memset(&w, 0, sizeof(w));
    work_alloc_impl(w, nullptr, cap, P32, num_sms, nullptr, fmm_p);
    return w.bytes;
}

static void free_work(vx_sim *s) { vx_work_free(s->w, s->work_allocs, s->stream); }

static vx_status alloc_work(vx_sim *s, long long cap) {
    return vx_work_alloc(s->w, s->work_allocs, cap, s->P32, s->num_sms, s->stream, s->prm.fmm_p);
}

static void drop_graph(vx_sim *s) {
    for (auto &g : s->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = vx_sim::StepGraph();
    }
}

// Grow the particle store to at least `need` slots, keeping every slot's
// content (the dead tail matters: it enters the next 3-nearest search).
// The capacity a growth to at least `need` slots gives: it adds at least
// one increment (inc_step, 8192 at least) or a quarter; the first store gets
// the same margin beyond what its cloud needs, so a new body does not grow
// within its first steps.
static long long grown_cap(const vx_sim *s, long long need) {
    const long long inc = std::max<long long>(s->conf.inc_step, 8192);
    long long ncap = s->cap > 0 ? std::max(need, s->cap + inc) : std::max(need + inc, (long long)(need * 1.25));
    ncap = std::max(ncap, (long long)(s->cap * 1.25));
    return vx_ceil_div(ncap, 8192) * 8192;
}

static vx_status grow(vx_sim *s, long long need) {
    const long long ncap = grown_cap(s, need);
    double *arr[6] = {s->x, s->y, s->g, s->vx, s->vy, s->d};
    double *nar[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int k = 0; k < 6; ++k) {
        cudaError_t e = cudaMallocAsync(&nar[k], sizeof(double) * ncap, s->stream);   // stream-ordered: see dalloc
        if (e == cudaSuccess)
            e = s->cap > 0 ? cudaMemcpyAsync(nar[k], arr[k], sizeof(double) * s->cap, cudaMemcpyDeviceToDevice,
                                             s->stream)
                           : cudaMemsetAsync(nar[k], 0, sizeof(double) * ncap, s->stream);
        if (e != cudaSuccess) {
            // the store stays as it was: release the new arrays made so far
            for (int q = 0; q <= k; ++q)
                if (nar[q]) cudaFreeAsync(nar[q], s->stream);
            vx_set_error("growing the particle store to %lld slots: %s", ncap, cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? VX_ERR_NOMEM : VX_ERR_CUDA;
        }
    }
    k_fill_tail<<<s->num_sms * 4, 256, 0, s->stream>>>(nar[0], nar[1], nar[2], s->cap, ncap);
    ++s->launches;
    CU(cudaGetLastError());
    for (int k = 0; k < 6; ++k)
        if (arr[k]) CU(cudaFreeAsync(arr[k], s->stream));
    s->x = nar[0]; s->y = nar[1]; s->g = nar[2]; s->vx = nar[3]; s->vy = nar[4]; s->d = nar[5];
    s->cap = ncap;
    drop_graph(s);
    return alloc_work(s, ncap);
}

static vx_status read_scalars(vx_sim *s) {
    CU(cudaMemcpyAsync(s->h_S, s->d_S, sizeof(VxScalars), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->n_upper = s->h_S->n;
    if (s->h_S->err) {
        vx_set_error("device error flag 0x%x", s->h_S->err);
        return VX_ERR_DEVICE;
    }
    return VX_OK;
}

static long long need_for(vx_sim *s, long long n) { return vx_round32(n + s->P) + 64; }

static vx_status ensure_capacity(vx_sim *s) {
    if (need_for(s, s->n_upper) <= s->cap) return VX_OK;
    vx_status st = read_scalars(s);
    if (st != VX_OK) return st;
    if (need_for(s, s->n_upper) <= s->cap) return VX_OK;
    return grow(s, need_for(s, s->n_upper));
}

// Launch shapes of a step follow the host's upper bound of the source count
// rounded up to a power of two, so that they (and the step graph holding
// them) change only when that bound crosses one, not every few steps.  They
// are grids only: the partitions that fix summation orders are derived on
// the device from the body's own count.
static int rhs_chunks_for(vx_sim *s) { return vx_rhs_chunks(s->n_upper, s->P, s->num_sms); }

// SMs a step's grid-stride launches are sized for: one per 2048 sources of
// the rounded bound, at least 4, at most the device's.
static int step_sms_for(vx_sim *s) { return vx_body_sms(s->n_upper + s->P, s->num_sms); }

VxLaunch vx_sim_launch(vx_sim *s) { return launch_of(s); }
long long vx_sim_need(vx_sim *s, long long n) { return need_for(s, n); }
long long vx_sim_grow_bytes(vx_sim *s, long long need) {
    const long long ncap = grown_cap(s, need);
    return 6LL * 8 * ncap + vx_work_bytes(ncap, s->P32, s->num_sms, s->prm.fmm_p) + 6 * 256;
}
vx_status vx_sim_grow(vx_sim *s, long long need) { return grow(s, need); }
vx_status vx_sim_read_scalars(vx_sim *s) { return read_scalars(s); }
int vx_sim_step_sms(vx_sim *s) { return step_sms_for(s); }
int vx_sim_rhs_chunks(vx_sim *s) { return rhs_chunks_for(s); }

// ---------------------------------------------------------------------------
// Wall panel lists: cells of side 5 L_max (1 % margin) over the birth-point
// box grown by 5 L_max; each panel is listed in the 3 x 3 cells around its
// birth point, in ascending panel order.
static vx_status build_wall_lists(vx_sim *s, const vx_panel *pan, int P) {
    VxParams &p = s->prm;
    double lmax = 0.0;
    for (int i = 0; i < P; ++i) lmax = std::max(lmax, pan[i].length);
    if (P <= 0 || !(lmax > 0.0)) { p.wall_nx = p.wall_ny = 0; return VX_OK; }
    const double h = 5.0 * lmax * 1.01;
    const long long nx = std::max(1LL, (long long)std::ceil((p.wall_x1 - p.wall_x0) / h));
    const long long ny = std::max(1LL, (long long)std::ceil((p.wall_y1 - p.wall_y0) / h));
    if (nx * ny > (1LL << 24)) { p.wall_nx = p.wall_ny = 0; return VX_OK; }   // degenerate: test all
    std::vector<std::vector<int>> cells((size_t)(nx * ny));
    for (int f = 0; f < P; ++f) {
        const long long cx = std::min(std::max((long long)std::floor((pan[f].birth[0] - p.wall_x0) / h), 0LL), nx - 1);
        const long long cy = std::min(std::max((long long)std::floor((pan[f].birth[1] - p.wall_y0) / h), 0LL), ny - 1);
        for (long long yy = std::max(cy - 1, 0LL); yy <= std::min(cy + 1, ny - 1); ++yy)
            for (long long xx = std::max(cx - 1, 0LL); xx <= std::min(cx + 1, nx - 1); ++xx)
                cells[(size_t)(yy * nx + xx)].push_back(f);
    }
    std::vector<int> start((size_t)(nx * ny + 1), 0), idx;
    for (size_t c = 0; c < cells.size(); ++c) {
        start[c] = (int)idx.size();
        idx.insert(idx.end(), cells[c].begin(), cells[c].end());
    }
    start[cells.size()] = (int)idx.size();
    if (idx.empty()) idx.push_back(0);
    s->wall_bytes = (long long)sizeof(int) * (long long)(start.size() + idx.size());
    if (cudaMalloc(&s->d_wstart, sizeof(int) * start.size()) != cudaSuccess) return VX_ERR_NOMEM;
    if (cudaMalloc(&s->d_widx, sizeof(int) * idx.size()) != cudaSuccess) return VX_ERR_NOMEM;
    if (cudaMemcpy(s->d_wstart, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->d_widx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return VX_ERR_CUDA;
    p.wall_h = h;
    p.wall_nx = (int)nx;
    p.wall_ny = (int)ny;
    return VX_OK;
}

// Hitting-test panel lists: a grid over the bounding box of all panel
// endpoints (cells of side 4 L_max, at most 512 per side); each panel is
// listed, in ascending order, in every cell its own bounding box touches.
static vx_status build_hit_lists(vx_sim *s, const vx_panel *pan, int P) {
    VxParams &p = s->prm;
    p.hit_nx = p.hit_ny = 0;
    double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300, lmax = 0.0;
    for (int i = 0; i < P; ++i) {
        for (const double *e : {pan[i].left, pan[i].right}) {
            x0 = std::min(x0, e[0]); x1 = std::max(x1, e[0]);
            y0 = std::min(y0, e[1]); y1 = std::max(y1, e[1]);
        }
        lmax = std::max(lmax, pan[i].length);
    }
    if (P <= 0 || !(lmax > 0.0)) return VX_OK;
    double h = 4.0 * lmax;
    h = std::max(h, std::max(x1 - x0, y1 - y0) / 512.0);
    const double pad = 1e-9 * std::max(1.0, std::max(fabs(x0), fabs(x1)) + std::max(fabs(y0), fabs(y1)));
    x0 -= pad; y0 -= pad;
    const long long nx = (long long)std::floor((x1 + pad - x0) / h) + 1;
    const long long ny = (long long)std::floor((y1 + pad - y0) / h) + 1;
    std::vector<std::vector<int>> cells((size_t)(nx * ny));
    for (int f = 0; f < P; ++f) {
        const double bx0 = std::min(pan[f].left[0], pan[f].right[0]), bx1 = std::max(pan[f].left[0], pan[f].right[0]);
        const double by0 = std::min(pan[f].left[1], pan[f].right[1]), by1 = std::max(pan[f].left[1], pan[f].right[1]);
        const long long cx0 = std::max(0LL, (long long)std::floor((bx0 - x0) / h) - 1);
        const long long cx1 = std::min(nx - 1, (long long)std::floor((bx1 - x0) / h) + 1);
        const long long cy0 = std::max(0LL, (long long)std::floor((by0 - y0) / h) - 1);
        const long long cy1 = std::min(ny - 1, (long long)std::floor((by1 - y0) / h) + 1);
        for (long long yy = cy0; yy <= cy1; ++yy)
            for (long long xx = cx0; xx <= cx1; ++xx) cells[(size_t)(yy * nx + xx)].push_back(f);
    }
    std::vector<int> start((size_t)(nx * ny + 1), 0), idx;
    for (size_t c = 0; c < cells.size(); ++c) {
        start[c] = (int)idx.size();
        idx.insert(idx.end(), cells[c].begin(), cells[c].end());
    }
    start[cells.size()] = (int)idx.size();
    if (idx.empty()) idx.push_back(0);
    s->wall_bytes += (long long)sizeof(int) * (long long)(start.size() + idx.size());
    if (cudaMalloc(&s->d_hstart, sizeof(int) * start.size()) != cudaSuccess) return VX_ERR_NOMEM;
    if (cudaMalloc(&s->d_hidx, sizeof(int) * idx.size()) != cudaSuccess) return VX_ERR_NOMEM;
    if (cudaMemcpy(s->d_hstart, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->d_hidx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return VX_ERR_CUDA;
    p.hit_x0 = x0;
    p.hit_y0 = y0;
    p.hit_h = h;
    p.hit_nx = (int)nx;
    p.hit_ny = (int)ny;
    return VX_OK;
}

extern "C" vx_status vx_create(const vx_conf *conf, const vx_panel *pan, int64_t P, int device,
                               vx_sim **out) {
    if (!conf || !pan || P < 2 || !out) { vx_set_error("vx_create: bad arguments"); return VX_ERR_ARG; }
    if (conf->dt <= 0 || conf->ve_size <= 0 || conf->n_of_points < 1) {
        vx_set_error("vx_create: dt, ve_size and n_of_points must be positive");
        return VX_ERR_ARG;
    }
    for (int64_t i = 0; i < P; ++i) {
        if (pan[i].n_of_rpanel >= (uint32_t)P || pan[i].n_of_lpanel >= (uint32_t)P) {
            vx_set_error("vx_create: panel %lld has a neighbour index outside [0,%lld)", (long long)i,
                         (long long)P);
            return VX_ERR_ARG;
        }
    }
    vx_sim *s = new vx_sim();
    s->conf = *conf;
    s->device = device;
    s->P = (int)P;
    s->P32 = (int)vx_round32(P);
    *out = nullptr;
    auto fail = [&](vx_status st) { vx_destroy(s); return st; };
    if (cudaSetDevice(device) != cudaSuccess) { vx_set_error("cudaSetDevice(%d) failed", device); return fail(VX_ERR_CUDA); }
    vx_keep_pool(device);
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(VX_ERR_CUDA);
    vx_params_from_conf(conf, pan, (int)P, &s->prm);
    std::vector<vx_panel> hp(s->P32);
    memset(hp.data(), 0, sizeof(vx_panel) * s->P32);
    memcpy(hp.data(), pan, sizeof(vx_panel) * P);
    if (cudaMalloc(&s->d_pan, sizeof(vx_panel) * s->P32) != cudaSuccess) return fail(VX_ERR_NOMEM);
    if (cudaMemcpy(s->d_pan, hp.data(), sizeof(vx_panel) * s->P32, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(VX_ERR_CUDA);
    if (cudaMalloc(&s->d_S, sizeof(VxScalars)) != cudaSuccess) return fail(VX_ERR_NOMEM);
    if (cudaMallocHost(&s->h_S, sizeof(VxScalars)) != cudaSuccess) return fail(VX_ERR_NOMEM);
    memset(s->h_S, 0, sizeof(VxScalars));
    // V_inf ramp (src/main.c:585-592): with a ramp the flow starts at rest
    s->h_S->incr_steps = conf->v_inf_incr_steps;
    if (conf->v_inf_incr_steps > 0) {
        s->h_S->dvinf[0] = conf->v_inf_x / (double)conf->v_inf_incr_steps;
        s->h_S->dvinf[1] = conf->v_inf_y / (double)conf->v_inf_incr_steps;
    } else {
        s->h_S->vinf[0] = conf->v_inf_x;
        s->h_S->vinf[1] = conf->v_inf_y;
    }
    if (cudaMemcpy(s->d_S, s->h_S, sizeof(VxScalars), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(VX_ERR_CUDA);
    if (build_wall_lists(s, pan, (int)P) != VX_OK) return fail(VX_ERR_NOMEM);
    if (build_hit_lists(s, pan, (int)P) != VX_OK) return fail(VX_ERR_NOMEM);
    // panel system on the device
    const long long S1 = P + 1;
    if (cudaMalloc(&s->d_minv, sizeof(double) * S1 * S1) != cudaSuccess) return fail(VX_ERR_NOMEM);
    double *work = nullptr;
    int *flag = nullptr;
    if (cudaMalloc(&work, sizeof(double) * (2 * S1 * S1 + S1)) != cudaSuccess) return fail(VX_ERR_NOMEM);
    if (cudaMalloc(&flag, sizeof(int)) != cudaSuccess) { cudaFree(work); return fail(VX_ERR_NOMEM); }
    VxLaunch L = launch_of(s);
    const int mode = conf->gj_pivot == 1 ? 1 : (conf->gj_pivot == 3 ? 3 : 0);
    cudaError_t e = vx_build_matrix(L, s->d_pan, (int)P, s->d_minv, work, flag, nullptr, mode);
    int hflag = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess && hflag && conf->gj_pivot == 2) {   // the reference's rule failed: pivot properly
        e = vx_build_matrix(L, s->d_pan, (int)P, s->d_minv, work, flag, nullptr, 1);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    }
    if (e == cudaSuccess && cudaMalloc(&s->d_minvT, sizeof(double) * S1 * S1) != cudaSuccess)
        e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = vx_transpose_square(L, s->d_minv, s->d_minvT, S1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(work);
    cudaFree(flag);
    if (e != cudaSuccess) { vx_set_error("panel system: %s", cudaGetErrorString(e)); return fail(VX_ERR_CUDA); }
    if (hflag) { vx_set_error("panel system is singular (pivot < 1e-12)"); return fail(VX_ERR_SINGULAR); }
    vx_status st = grow(s, std::max<long long>(need_for(s, 0), conf->inc_step > 0 ? conf->inc_step : 8192));
    if (st != VX_OK) return fail(st);
    *out = s;
    return VX_OK;
}

extern "C" vx_status vx_destroy(vx_sim *s) {
    if (!s) return VX_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    drop_graph(s);
    free_work(s);   // stream-ordered, as allocated
    double *arr[6] = {s->x, s->y, s->g, s->vx, s->vy, s->d};
    for (double *a : arr) if (a) cudaFreeAsync(a, s->stream);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->d_pan) cudaFree(s->d_pan);
    if (s->d_minv) cudaFree(s->d_minv);
    if (s->d_minvT) cudaFree(s->d_minvT);
    if (s->d_wstart) cudaFree(s->d_wstart);
    if (s->d_widx) cudaFree(s->d_widx);
    if (s->d_hstart) cudaFree(s->d_hstart);
    if (s->d_hidx) cudaFree(s->d_hidx);
    if (s->d_S) cudaFree(s->d_S);
    if (s->h_S) cudaFreeHost(s->h_S);
    if (s->d_probe) cudaFree(s->d_probe);
    if (s->d_pts) cudaFree(s->d_pts);
    if (s->d_St) cudaFree(s->d_St);
    if (s->d_pred) cudaFree(s->d_pred);
    for (auto &e : s->ev) if (e) cudaEventDestroy(e);
    for (auto &e : s->pev) if (e) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
    vx_trim_pool(s->device);
    delete s;
    return VX_OK;
}

// ---------------------------------------------------------------------------
static vx_status set_count(vx_sim *s, long long n) {
    CU(cudaMemcpyAsync(s->h_S, s->d_S, sizeof(VxScalars), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->h_S->n = n;
    s->h_S->n0 = n >= s->P ? n - s->P : 0;   // the last P count as this step's newborns
    s->h_S->fsq = 0;                          // a new cloud: the quadtree depth starts from the box rule
    s->h_S->fLcap = 0;
    CU(cudaMemcpyAsync(s->d_S, s->h_S, sizeof(VxScalars), cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->n_upper = n;
    return VX_OK;
}

extern "C" vx_status vx_set_particles(vx_sim *s, const double *x, const double *y, const double *g,
                                      int64_t n) {
    if (!s || n < 0 || (n > 0 && (!x || !y || !g))) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    if (need_for(s, n) > s->cap) {
        vx_status st = grow(s, need_for(s, n));
        if (st != VX_OK) return st;
    }
    if (n > 0) {
        CU(cudaMemcpyAsync(s->x, x, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
        CU(cudaMemcpyAsync(s->y, y, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
        CU(cudaMemcpyAsync(s->g, g, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    }
    return set_count(s, n);
}

extern "C" vx_status vx_set_velocity(vx_sim *s, const double *vx, const double *vy, const double *d,
                                     int64_t n) {
    if (!s || n < 0 || n > s->cap) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    if (n > 0) {
        if (vx) CU(cudaMemcpyAsync(s->vx, vx, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
        if (vy) CU(cudaMemcpyAsync(s->vy, vy, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
        if (d) CU(cudaMemcpyAsync(s->d, d, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    }
    CU(cudaStreamSynchronize(s->stream));
    return VX_OK;
}

extern "C" vx_status vx_get_count(vx_sim *s, int64_t *n) {
    if (!s || !n) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    vx_status st = read_scalars(s);
    *n = s->h_S->n;
    return st;
}

extern "C" vx_status vx_get_particles(vx_sim *s, double *x, double *y, double *g, int64_t cap,
                                      int64_t *n) {
    if (!s || !n) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    vx_status st = read_scalars(s);
    if (st != VX_OK) return st;
    long long m = s->h_S->n;
    *n = m;
    if (cap < m) return x ? VX_ERR_ARG : VX_OK;
    if (m > 0 && x && y && g) {
        CU(cudaMemcpyAsync(x, s->x, sizeof(double) * m, cudaMemcpyDeviceToHost, s->stream));
        CU(cudaMemcpyAsync(y, s->y, sizeof(double) * m, cudaMemcpyDeviceToHost, s->stream));
        CU(cudaMemcpyAsync(g, s->g, sizeof(double) * m, cudaMemcpyDeviceToHost, s->stream));
        CU(cudaStreamSynchronize(s->stream));
    }
    return VX_OK;
}

// Raw slots [0, count) including the dead tail (for parity tests).
extern "C" vx_status vx_get_slots(vx_sim *s, double *x, double *y, double *g, int64_t count) {
    if (!s || count < 0 || count > s->cap) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    CU(cudaMemcpyAsync(x, s->x, sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(y, s->y, sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(g, s->g, sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return VX_OK;
}

// Write raw slots [0, count) (tail included) and set the live count.
extern "C" vx_status vx_set_slots(vx_sim *s, const double *x, const double *y, const double *g,
                                  int64_t count, int64_t n) {
    if (!s || count < 0 || n < 0 || n > count) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    if (need_for(s, count) > s->cap) {
        vx_status st = grow(s, need_for(s, count));
        if (st != VX_OK) return st;
    }
    CU(cudaMemcpyAsync(s->x, x, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
    CU(cudaMemcpyAsync(s->y, y, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
    CU(cudaMemcpyAsync(s->g, g, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
    return set_count(s, n);
}

extern "C" vx_status vx_get_velocity(vx_sim *s, double *vx, double *vy, double *d, int64_t cap) {
    if (!s) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    vx_status st = read_scalars(s);
    if (st != VX_OK) return st;
    long long m = std::min<long long>(s->h_S->n, cap);
    if (m > 0) {
        if (vx) CU(cudaMemcpyAsync(vx, s->vx, sizeof(double) * m, cudaMemcpyDeviceToHost, s->stream));
        if (vy) CU(cudaMemcpyAsync(vy, s->vy, sizeof(double) * m, cudaMemcpyDeviceToHost, s->stream));
        if (d) CU(cudaMemcpyAsync(d, s->d, sizeof(double) * m, cudaMemcpyDeviceToHost, s->stream));
        CU(cudaStreamSynchronize(s->stream));
    }
    return VX_OK;
}

extern "C" vx_status vx_get_forces(vx_sim *s, double out4[4]) {
    if (!s || !out4) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    vx_status st = read_scalars(s);
    out4[0] = s->h_S->dg; out4[1] = s->h_S->fx; out4[2] = s->h_S->fy; out4[3] = s->h_S->m;
    return st;
}

// n, n0, step, vinf x/y, dg, fx, fy, m
extern "C" vx_status vx_get_state(vx_sim *s, double out9[9]) {
    if (!s || !out9) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    vx_status st = read_scalars(s);
    const VxScalars &h = *s->h_S;
    double v[9] = {(double)h.n, (double)h.n0, (double)h.step, h.vinf[0], h.vinf[1], h.dg, h.fx, h.fy, h.m};
    memcpy(out9, v, sizeof(v));
    return st;
}

static vx_status patch_scalars(vx_sim *s, void (*fn)(VxScalars *, const double *), const double *a) {
    CU(cudaMemcpyAsync(s->h_S, s->d_S, sizeof(VxScalars), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    fn(s->h_S, a);
    CU(cudaMemcpyAsync(s->d_S, s->h_S, sizeof(VxScalars), cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return VX_OK;
}

extern "C" vx_status vx_set_vinf(vx_sim *s, double vx, double vy) {
    if (!s) return VX_ERR_ARG;
    double a[2] = {vx, vy};
    return patch_scalars(s, [](VxScalars *h, const double *q) { h->vinf[0] = q[0]; h->vinf[1] = q[1]; }, a);
}

extern "C" vx_status vx_set_dg(vx_sim *s, double dg) {
    if (!s) return VX_ERR_ARG;
    return patch_scalars(s, [](VxScalars *h, const double *q) { h->dg = q[0]; }, &dg);
}

// Absolute step index (restart from a KadrNNNNNN file sets it).
extern "C" vx_status vx_set_step_index(vx_sim *s, int64_t step) {
    if (!s || step < 0) return VX_ERR_ARG;
    double a = (double)step;
    return patch_scalars(s, [](VxScalars *h, const double *q) { h->step = (long long)q[0]; }, &a);
}

// Replace the inverted panel system (row-major (P+1)^2, e.g. a matrix file
// the caller loaded) and its transposed copy.
extern "C" vx_status vx_set_matrix(vx_sim *s, const double *minv) {
    if (!s || !minv) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    const long long S1 = s->P + 1;
    CU(cudaMemcpy(s->d_minv, minv, sizeof(double) * S1 * S1, cudaMemcpyHostToDevice));
    CU(vx_transpose_square(launch_of(s), s->d_minv, s->d_minvT, S1));
    CU(cudaStreamSynchronize(s->stream));
    return VX_OK;
}

// ---------------------------------------------------------------------------
// Binary checkpoint of a body: what the next step reads from the previous
// ones, at full precision (the reference's text frames keep 6 decimals and
// drop d_g, the forces and the V_inf ramp): every slot (x, y, G in FP64) up
// to the capacity, the tail beyond the live vortices included (the plain
// form's 3-nearest search reads the round-up slots after the live ones, as
// the reference's does), the step index, the current V_inf, d_g and the
// last forces with their raw sums, and the last quadtree build's occupancy
// record (the bulk form's next depth follows from it).  The file names the
// body it belongs to by its panel count, its form (FP64 / FP32) and a hash of
// its panels; loading into another body fails.  Version 1 files (no
// quadtree record) load with the depth rule starting afresh.
namespace {
struct CkptHead {
    char magic[8];           // "VXCKPT1"
    int32_t version, P, prec, pad;
    int64_t n, n0, step, slots;
    double vinf[2], dg, fx, fy, m, raw[4];
    uint64_t panel_hash;     // FNV-1a of the panel records
    // version 2: the last quadtree build (sum of count^2 over its quarter
    // cells, its sources, box side and depth) and the depth rule's ceiling
    uint64_t tree_sq;
    int64_t tree_s;
    double tree_side;
    int32_t tree_L, tree_Lcap;
};
constexpr size_t kCkptHeadV1 = offsetof(CkptHead, tree_sq);
const char kCkptMagic[8] = {'V', 'X', 'C', 'K', 'P', 'T', '1', 0};

vx_status panel_hash(vx_sim *s, uint64_t *h) {
    std::vector<vx_panel> pan((size_t)s->P);
    CU(cudaMemcpy(pan.data(), s->d_pan, sizeof(vx_panel) * (size_t)s->P, cudaMemcpyDeviceToHost));
    uint64_t v = 1469598103934665603ull;
    const unsigned char *b = reinterpret_cast<const unsigned char *>(pan.data());
    for (size_t i = 0; i < sizeof(vx_panel) * pan.size(); ++i) { v ^= b[i]; v *= 1099511628211ull; }
    *h = v;
    return VX_OK;
}
}  // namespace

extern "C" vx_status vx_checkpoint_save(vx_sim *s, const char *path) {
    if (!s || !path) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    vx_status st = read_scalars(s);
    if (st != VX_OK) return st;
    const VxScalars h = *s->h_S;
    CkptHead hd;
    memset(&hd, 0, sizeof(hd));
    memcpy(hd.magic, kCkptMagic, 8);
    hd.version = 2; hd.P = s->P; hd.prec = s->prm.prec;
    hd.tree_sq = h.fsq; hd.tree_s = h.fs; hd.tree_side = h.fside; hd.tree_L = h.fL; hd.tree_Lcap = h.fLcap;
    hd.n = h.n; hd.n0 = h.n0; hd.step = h.step; hd.slots = s->cap;
    hd.vinf[0] = h.vinf[0]; hd.vinf[1] = h.vinf[1];
    hd.dg = h.dg; hd.fx = h.fx; hd.fy = h.fy; hd.m = h.m;
    for (int q = 0; q < 4; ++q) hd.raw[q] = h.raw[q];
    if ((st = panel_hash(s, &hd.panel_hash)) != VX_OK) return st;
    const long long ns = hd.slots;
    std::vector<double> a((size_t)(3 * ns));
    if (ns > 0) {
        CU(cudaMemcpy(a.data(), s->x, sizeof(double) * ns, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(a.data() + ns, s->y, sizeof(double) * ns, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(a.data() + 2 * ns, s->g, sizeof(double) * ns, cudaMemcpyDeviceToHost));
    }
    FILE *f = fopen(path, "wb");
    if (!f) { vx_set_error("cannot open %s for writing", path); return VX_ERR_ARG; }
    const bool ok = fwrite(&hd, sizeof(hd), 1, f) == 1 &&
                    (a.empty() || fwrite(a.data(), sizeof(double), a.size(), f) == a.size());
    if (fclose(f) != 0 || !ok) { vx_set_error("writing %s failed", path); return VX_ERR_ARG; }
    return VX_OK;
}

extern "C" vx_status vx_checkpoint_load(vx_sim *s, const char *path) {
    if (!s || !path) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    FILE *f = fopen(path, "rb");
    if (!f) { vx_set_error("cannot open %s", path); return VX_ERR_ARG; }
    CkptHead hd;
    memset(&hd, 0, sizeof(hd));
    bool head_ok = fread(&hd, kCkptHeadV1, 1, f) == 1 && memcmp(hd.magic, kCkptMagic, 8) == 0 &&
                   (hd.version == 1 || hd.version == 2) && hd.n >= 0 && hd.slots >= hd.n;
    if (head_ok && hd.version == 2)
        head_ok = fread(reinterpret_cast<char *>(&hd) + kCkptHeadV1, sizeof(hd) - kCkptHeadV1, 1, f) == 1;
    if (!head_ok) {
        fclose(f);
        vx_set_error("%s is not a checkpoint of this library", path);
        return VX_ERR_ARG;
    }
    uint64_t hh = 0;
    vx_status st = panel_hash(s, &hh);
    if (st != VX_OK) { fclose(f); return st; }
    if (hd.P != s->P || hd.prec != s->prm.prec || hd.panel_hash != hh) {
        fclose(f);
        vx_set_error("%s belongs to another body (%d panels, form %d) than this one (%d panels, form %d)", path,
                     hd.P, hd.prec, s->P, s->prm.prec);
        return VX_ERR_ARG;
    }
    const long long ns = hd.slots;
    std::vector<double> a((size_t)(3 * ns));
    const bool ok = a.empty() || fread(a.data(), sizeof(double), a.size(), f) == a.size();
    fclose(f);
    if (!ok) { vx_set_error("%s is truncated", path); return VX_ERR_ARG; }
    if ((st = vx_set_slots(s, a.data(), a.data() + ns, a.data() + 2 * ns, ns, hd.n)) != VX_OK) return st;
    CU(cudaMemcpyAsync(s->h_S, s->d_S, sizeof(VxScalars), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    VxScalars *h = s->h_S;
    h->n0 = hd.n0; h->step = hd.step;
    h->vinf[0] = hd.vinf[0]; h->vinf[1] = hd.vinf[1];
    h->dg = hd.dg; h->fx = hd.fx; h->fy = hd.fy; h->m = hd.m;
    for (int q = 0; q < 4; ++q) h->raw[q] = hd.raw[q];
    h->fsq = hd.tree_sq;
    h->fLcap = hd.tree_Lcap;
    if (hd.tree_sq) { h->fs = hd.tree_s; h->fside = hd.tree_side; h->fL = hd.tree_L; }
    CU(cudaMemcpyAsync(s->d_S, s->h_S, sizeof(VxScalars), cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return VX_OK;
}

extern "C" vx_status vx_get_matrix(vx_sim *s, double *minv) {
    if (!s || !minv) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    const long long S1 = s->P + 1;
    CU(cudaMemcpy(minv, s->d_minv, sizeof(double) * S1 * S1, cudaMemcpyDeviceToHost));
    return VX_OK;
}

// ---------------------------------------------------------------------------
static cudaError_t launch_stages(vx_sim *s, unsigned mask, bool whole_step, VxRecorder *rec = nullptr,
                                 int share = 0) {
    VxLaunch L = launch_of(s);
    L.num_sms = step_sms_for(s);
    if (share > 0) L.num_sms = std::min(share, L.num_sms);
    L.full_sms = s->num_sms;
    L.rec = rec;
    if (rec) L.launches = nullptr;
    if (!rec) L.kt = s->kt;
    VxView v = view_of(s);
    const VxParams &p = s->prm;
    cudaError_t e = cudaSuccess;
    const bool timed = s->timing && !whole_step && !rec;
    if (timed)
        for (int k = 0; k < 4; ++k) L.pair_ev[k] = s->pev[k];
    auto ev = [&](int k) { if (timed) cudaEventRecord(s->ev[k], s->stream); };
    ev(0);
    if (mask & VX_STAGE_BIRTH) {
        if ((e = vx_launch_step_begin(L, s->d_S)) != cudaSuccess) return e;
        if ((e = vx_launch_birth(L, p, v, s->d_S, s->w, s->d_pan, s->d_minv, s->d_minvT, rhs_chunks_for(s))) != cudaSuccess) return e;
    }
    ev(1);
    if (mask & VX_STAGE_VELOCITY) {
        // bulk form: quadtree FMM (vx_fmm.cu); plain form: direct sum
        if (p.prec == VX_PREC_FP32 && s->conf.fmm)
            e = vx_launch_velocity_fmm(L, p, v, s->d_S, s->w);
        else
            e = vx_launch_velocity(L, p, v, s->d_S, s->w);
        if (e != cudaSuccess) return e;
    }
    ev(2);
    if (mask & VX_STAGE_DIFFUSION)
        if ((e = vx_launch_diffusion(L, p, v, s->d_S, s->w)) != cudaSuccess) return e;
    ev(3);
    if (mask & VX_STAGE_WALL)
        if ((e = vx_launch_wall(L, p, v, s->d_S, s->d_pan, s->d_wstart, s->d_widx)) != cudaSuccess) return e;
    ev(4);
    if (mask & VX_STAGE_ADVECT)
        if ((e = vx_launch_advect(L, p, v, s->d_S, s->w, s->d_pan, s->d_hstart, s->d_hidx)) != cudaSuccess) return e;
    if (mask & VX_STAGE_COMPACT)
        if ((e = vx_launch_compact(L, p, v, s->d_S, s->w, whole_step)) != cudaSuccess) return e;
    if (mask & VX_STAGE_COLLAPSE1)
        if ((e = vx_launch_collapse(L, p, v, s->d_S, s->w, 1, (int)s->conf.n_col)) != cudaSuccess) return e;
    if (mask & VX_STAGE_COLLAPSE2)
        if ((e = vx_launch_collapse(L, p, v, s->d_S, s->w, 2, (int)s->conf.n_col)) != cudaSuccess) return e;
    // a whole step is counted by its main compaction (no kernel after it
    // reads the step index), else by a kernel of its own
    if (whole_step && !(mask & VX_STAGE_COMPACT)) e = vx_launch_step_end(L, s->d_S);
    ev(5);
    return e;
}

cudaError_t vx_sim_launch_stages(vx_sim *s, unsigned mask, bool whole_step, VxRecorder *rec, int share) {
    return launch_stages(s, mask, whole_step, rec, share);
}

extern "C" vx_status vx_stage(vx_sim *s, unsigned mask) {
    if (!s) return VX_ERR_ARG;
    if (s->in_batch) { vx_set_error("vx_stage: the body belongs to a batch (step it with vx_batch_step)"); return VX_ERR_ARG; }
    CU(cudaSetDevice(s->device));
    vx_status st = ensure_capacity(s);
    if (st != VX_OK) return st;
    CU(launch_stages(s, mask, false));
    if (mask & VX_STAGE_BIRTH) s->n_upper += s->P;
    return read_scalars(s);
}

static vx_status step_once(vx_sim *s) {
    vx_status st = ensure_capacity(s);
    if (st != VX_OK) return st;
    if (s->timing) {
        // timed steps run eagerly so per-stage events can be recorded
        CU(launch_stages(s, VX_STAGE_ALL, false));
        CU(vx_launch_step_end(launch_of(s), s->d_S));
        s->n_upper += s->P;
        return VX_OK;
    }
    if (!s->use_graph) {
        CU(launch_stages(s, VX_STAGE_ALL, true));
        s->n_upper += s->P;
        return VX_OK;
    }
    const int rc = rhs_chunks_for(s), sms = step_sms_for(s);
    vx_sim::StepGraph *sg = nullptr;
    for (auto &g : s->graphs)
        if (g.exec && g.rhs == rc && g.sms == sms) sg = &g;
    if (!sg) {
        sg = &s->graphs[0];
        for (auto &g : s->graphs)
            if (!g.exec || (sg->exec && g.used < sg->used)) sg = &g;
        if (sg->exec) cudaGraphExecDestroy(sg->exec);
        *sg = vx_sim::StepGraph();
        cudaGraph_t graph;
        long long before = s->launches;
        CU(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = launch_stages(s, VX_STAGE_ALL, true);
        cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            vx_set_error("graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
            return VX_ERR_CUDA;
        }
        sg->launches = s->launches - before;
        s->launches = before;
        e = cudaGraphInstantiate(&sg->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            sg->exec = nullptr;
            vx_set_error("graph instantiate: %s", cudaGetErrorString(e));
            return VX_ERR_CUDA;
        }
        sg->rhs = rc;
        sg->sms = sms;
    }
    sg->used = ++s->graph_clock;
    CU(cudaGraphLaunch(sg->exec, s->stream));
    s->launches += sg->launches;
    s->n_upper += s->P;
    return VX_OK;
}

extern "C" vx_status vx_step(vx_sim *s, int64_t nsteps) {
    if (!s || nsteps < 0) return VX_ERR_ARG;
    if (s->in_batch) { vx_set_error("vx_step: the body belongs to a batch (step it with vx_batch_step)"); return VX_ERR_ARG; }
    CU(cudaSetDevice(s->device));
    for (int64_t k = 0; k < nsteps; ++k) {
        vx_status st = step_once(s);
        if (st != VX_OK) return st;
        if (s->timing) {
            CU(cudaEventSynchronize(s->ev[5]));
            float t;
            for (int q = 0; q < 5; ++q) {
                cudaEventElapsedTime(&t, s->ev[q], s->ev[q + 1]);
                s->t_acc[q] += t;
            }
            cudaEventElapsedTime(&t, s->pev[0], s->pev[1]);
            s->t_acc[5] += t;
            cudaEventElapsedTime(&t, s->pev[2], s->pev[3]);
            s->t_acc[6] += t;
            cudaEventElapsedTime(&t, s->ev[0], s->ev[5]);
            s->t_acc[7] += t;
        }
    }
    CU(cudaGetLastError());
    return VX_OK;
}

extern "C" vx_status vx_sync(vx_sim *s) {
    if (!s) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    return read_scalars(s);
}

extern "C" vx_status vx_set_graph(vx_sim *s, int enable) {
    if (!s) return VX_ERR_ARG;
    s->use_graph = enable != 0;
    if (!s->use_graph) drop_graph(s);
    return VX_OK;
}

extern "C" vx_status vx_set_timing(vx_sim *s, int enable) {
    if (!s) return VX_ERR_ARG;
    s->timing = enable != 0;
    if (s->timing && !s->ev[0]) {
        for (auto &e : s->ev) CU(cudaEventCreate(&e));
        for (auto &e : s->pev) CU(cudaEventCreate(&e));
    }
    for (double &t : s->t_acc) t = 0.0;
    return VX_OK;
}

// Pair evaluations executed by the bulk-form near-field (FMM) and
// neighbour-list diffusion kernels since the last clear.
extern "C" vx_status vx_get_pair_counts(vx_sim *s, double out2[2], int clear) {
    if (!s || !out2) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    CU(cudaMemcpyAsync(s->h_S, s->d_S, sizeof(VxScalars), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    out2[0] = (double)s->h_S->pairs_bs;
    out2[1] = (double)s->h_S->pairs_diff;
    if (clear) {
        s->h_S->pairs_bs = s->h_S->pairs_diff = 0;
        CU(cudaMemcpyAsync(s->d_S, s->h_S, sizeof(VxScalars), cudaMemcpyHostToDevice, s->stream));
        CU(cudaStreamSynchronize(s->stream));
    }
    return VX_OK;
}

extern "C" vx_status vx_get_tree_info(vx_sim *s, double out6[6]) {
    if (!s || !out6) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    CU(cudaMemcpyAsync(s->h_S, s->d_S, sizeof(VxScalars), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    const VxScalars &h = *s->h_S;
    out6[0] = (double)h.fL;
    out6[1] = h.fL >= 0 ? h.fside / (double)(1LL << h.fL) : 0.0;
    out6[2] = (double)h.fnflag;
    out6[3] = h.ch;
    out6[4] = (double)h.cnx;
    out6[5] = (double)h.cny;
    return VX_OK;
}

extern "C" vx_status vx_get_timing(vx_sim *s, double out8[8]) {
    if (!s || !out8) return VX_ERR_ARG;
    for (int k = 0; k < 8; ++k) out8[k] = s->t_acc[k];
    return VX_OK;
}

extern "C" vx_status vx_get_launch_count(vx_sim *s, int64_t *count) {
    if (!s || !count) return VX_ERR_ARG;
    *count = s->launches;
    return VX_OK;
}

// Device bytes held by fixed-size parts of a body: panels, the inverted
// system and its transpose, scalars (the Gauss-Jordan work area of vx_create
// is transient and counted by the estimate only).
static long long fixed_bytes(long long P) {
    const long long P32 = vx_round32(P), S1 = P + 1;
    return P32 * (long long)sizeof(vx_panel) + 2 * S1 * S1 * 8 + (long long)sizeof(VxScalars) + 4096;
}

static long long cap_after_growth(long long need, long long inc_step) {
    const long long inc = std::max<long long>(inc_step, 8192);
    return vx_ceil_div(std::max<long long>((long long)(need * 1.25), need + inc), 8192) * 8192;
}

extern "C" vx_status vx_estimate_bytes(const vx_conf *c, int64_t P, int64_t n_max, int device, int64_t *out) {
    if (!c || !out || P < 2 || n_max < 0) return VX_ERR_ARG;
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) sms = 148;
    const long long need = vx_round32(n_max + P) + 64;
    const long long cap = cap_after_growth(need, c->inc_step);
    const long long S1 = P + 1;
    const long long transient = (2 * S1 * S1 + S1) * 8;     // Gauss-Jordan work area at creation
    const long long wall = 4LL * (9 * P + 4096);              // wall panel lists (bound)
    const int fp = vx_fmm_order_ok(c->fmm_p) ? c->fmm_p : VX_FMM_P;
    *out = 6 * 8 * cap + vx_work_bytes(cap, (int)vx_round32(P), sms, fp) + fixed_bytes(P) + transient + wall;
    return VX_OK;
}

extern "C" vx_status vx_get_device_bytes(vx_sim *s, int64_t *out) {
    if (!s || !out) return VX_ERR_ARG;
    *out = 6 * 8 * s->cap + s->w.bytes + fixed_bytes(s->P) + s->wall_bytes;
    return VX_OK;
}

// Advance several bodies (same device) by nsteps: each step is launched on
// every body's own stream before the next step, so the bodies' kernels
// overlap on the device.  Asynchronous like vx_step.
extern "C" vx_status vx_step_many(vx_sim *const *sims, int count, int64_t nsteps) {
    if ((!sims && count > 0) || count < 0 || nsteps < 0) return VX_ERR_ARG;
    for (int i = 0; i < count; ++i)
        if (!sims[i]) return VX_ERR_ARG;
    for (int64_t k = 0; k < nsteps; ++k)
        for (int i = 0; i < count; ++i) {
            vx_status st = vx_step(sims[i], 1);
            if (st != VX_OK) return st;
        }
    return VX_OK;
}

extern "C" vx_status vx_set_fmm(vx_sim *s, int fmm, int leaf) {
    if (!s || leaf < 1) return VX_ERR_ARG;
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    s->conf.fmm = fmm != 0;
    s->conf.fmm_leaf = leaf;
    s->prm.fmm_leaf = leaf;
    s->prm.birth_far = (s->prm.prec == VX_PREC_FP32 && s->conf.fmm && s->P > 0) ? 1 : 0;
    drop_graph(s);
    return VX_OK;
}

// Expansion terms of the bulk form's quadtree FMM (8, 12, 16 or 20); the
// expansion arrays are re-sized and the step graph re-captured.
extern "C" vx_status vx_set_fmm_order(vx_sim *s, int p) {
    if (!s || !vx_fmm_order_ok(p)) {
        vx_set_error("vx_set_fmm_order: %d terms (8, 12, 16 or 20)", p);
        return VX_ERR_ARG;
    }
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    if (p == s->prm.fmm_p) return VX_OK;
    s->conf.fmm_p = p;
    s->prm.fmm_p = p;
    drop_graph(s);
    return alloc_work(s, s->cap);
}

// The stream the handle launches on (for callers that time with events).
extern "C" void *vx_get_stream(vx_sim *s) { return s ? (void *)s->stream : nullptr; }

VX_DEVK void k_points_begin_body(VxBlkB<0, 0> vb, VxScalars *S, long long n) {
    S->n = n;
    S->n0 = n;   // no point counts as born this step: no force terms
}
__global__ void k_points_begin(VxScalars *S, long long n) {
    VX_PDL_WAIT();
    k_points_begin_body(VxBlkB<0, 0>{blockIdx.x, gridDim.x}, S, n);
}

// Passive points (tracers) moved one time step with the given velocities by
// the vortices' convection kernel: the same wall absorption (g set to 0) and
// window removal (moved to -2e5, g = 0), no force terms, and the body's own
// state and force sums untouched.  Host arrays in and out.
extern "C" vx_status vx_move_points(vx_sim *s, double *x, double *y, double *g, const double *u,
                                    const double *v, int64_t n) {
    if (!s || n < 0 || (n > 0 && (!x || !y || !g || !u || !v))) return VX_ERR_ARG;
    if (n == 0) return VX_OK;
    CU(cudaSetDevice(s->device));
    if (!s->d_St) {
        CU(cudaMalloc(&s->d_St, sizeof(VxScalars)));
        CU(cudaMemset(s->d_St, 0, sizeof(VxScalars)));
        CU(cudaMalloc(&s->d_pred, sizeof(double) * 4 * VX_RED_BLOCKS));
    }
    if (s->pts_cap < n) {
        if (s->d_pts) cudaFree(s->d_pts);
        s->d_pts = nullptr;
        s->pts_cap = 0;
        CU(cudaMalloc(&s->d_pts, sizeof(double) * 5 * n));
        s->pts_cap = n;
    }
    double *dx = s->d_pts, *dy = dx + n, *dg = dy + n, *du = dg + n, *dv = du + n;
    const double *src[5] = {x, y, g, u, v};
    double *dst[5] = {dx, dy, dg, du, dv};
    for (int q = 0; q < 5; ++q)
        CU(cudaMemcpyAsync(dst[q], src[q], sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    vx_launch_pdl(k_points_begin, 1, 1, 0, s->stream, s->d_St, (long long)n);
    VxView pv;
    pv.x = dx; pv.y = dy; pv.g = dg; pv.ps = 1;
    pv.vx = du; pv.vy = dv; pv.vs = 1;
    pv.d = nullptr;
    VxWork tw = s->w;
    tw.red = s->d_pred;
    CU(vx_launch_advect(launch_of(s), s->prm, pv, s->d_St, tw, s->d_pan, s->d_hstart, s->d_hidx));
    CU(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(g, dg, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return VX_OK;
}

extern "C" vx_status vx_probe(vx_sim *s, const double *px, const double *py, int64_t np, double *ovx,
                              double *ovy) {
    if (!s || np < 0 || (np > 0 && (!px || !py || !ovx || !ovy))) return VX_ERR_ARG;
    if (np == 0) return VX_OK;
    CU(cudaSetDevice(s->device));
    if (s->probe_cap < np) {
        if (s->d_probe) cudaFree(s->d_probe);
        s->d_probe = nullptr;
        CU(cudaMalloc(&s->d_probe, sizeof(double) * 4 * np));
        s->probe_cap = np;
    }
    double *dpx = s->d_probe, *dpy = dpx + np, *dvx = dpy + np, *dvy = dvx + np;
    CU(cudaMemcpyAsync(dpx, px, sizeof(double) * np, cudaMemcpyHostToDevice, s->stream));
    CU(cudaMemcpyAsync(dpy, py, sizeof(double) * np, cudaMemcpyHostToDevice, s->stream));
    const int tile = s->prm.prec == VX_PREC_FP32 ? 1024 : 512;
    const int K = vx_ksplit(np, tile, s->num_sms);
    CU(vx_launch_probe(launch_of(s), s->prm, view_of(s), s->d_S, s->w, dpx, dpy, 1, np, dvx, dvy, 1, K));
    CU(cudaMemcpyAsync(ovx, dvx, sizeof(double) * np, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(ovy, dvy, sizeof(double) * np, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return VX_OK;
}

// Device time of every kernel of `nsteps` steps launched stage by stage with
// an event pair around each launch (instrumentation: the events keep
// consecutive kernels from overlapping, and each time includes the event
// overhead, about a microsecond).  Kernels are named by their demangled
// names without parameters; names: '\n'-separated into a buffer of
// names_cap bytes; ms[k], counts[k]: total time and launches of kernel k;
// *nk: kernels found (at most cap are written).
extern "C" vx_status vx_kernel_times(vx_sim *s, int64_t nsteps, char *names, int64_t names_cap, double *ms,
                                     int64_t *counts, int64_t cap, int64_t *nk) {
    if (!s || nsteps < 1 || !names || names_cap < 1 || !ms || !counts || cap < 0 || !nk) return VX_ERR_ARG;
    if (s->in_batch) { vx_set_error("vx_kernel_times: the body belongs to a batch"); return VX_ERR_ARG; }
    CU(cudaSetDevice(s->device));
    VxKernelTimer kt;
    s->kt = &kt;
    vx_status st = VX_OK;
    for (int64_t k = 0; k < nsteps && st == VX_OK; ++k) {
        if ((st = ensure_capacity(s)) != VX_OK) break;
        const cudaError_t e = launch_stages(s, VX_STAGE_ALL, true);
        if (e != cudaSuccess) { vx_set_error("vx_kernel_times: %s", cudaGetErrorString(e)); st = VX_ERR_CUDA; }
        s->n_upper += s->P;
    }
    s->kt = nullptr;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    std::map<std::string, std::pair<double, long long>> acc;
    std::vector<std::string> order;
    std::map<const void *, std::string> name_of;
    for (const auto &r : kt.recs) {
        auto it = name_of.find(r.key);
        if (it == name_of.end()) {
            const char *raw = nullptr;
            std::string nm = "?";
            if (cudaFuncGetName(&raw, r.key) == cudaSuccess && raw) {
                int ok = -1;
                char *dm = abi::__cxa_demangle(raw, nullptr, nullptr, &ok);
                nm = (ok == 0 && dm) ? std::string(dm) : std::string(raw);
                free(dm);
                const size_t par = nm.find('(');
                if (par != std::string::npos) nm = nm.substr(0, par);
                if (nm.rfind("void ", 0) == 0) nm = nm.substr(5);
            }
            it = name_of.emplace(r.key, nm).first;
        }
        float t = 0.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&t, r.a, r.b);
        auto a = acc.find(it->second);
        if (a == acc.end()) {
            order.push_back(it->second);
            a = acc.emplace(it->second, std::make_pair(0.0, 0LL)).first;
        }
        a->second.first += t;
        a->second.second += 1;
    }
    for (const auto &r : kt.recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (cudaEvent_t ev : kt.pool) cudaEventDestroy(ev);
    if (st != VX_OK) return st;
    CU(e);
    std::string all;
    int64_t k = 0;
    for (const std::string &nm : order) {
        if (k < cap) {
            ms[k] = acc[nm].first;
            counts[k] = acc[nm].second;
            all += nm;
            all += '\n';
        }
        ++k;
    }
    *nk = k;
    const size_t nb = std::min<size_t>(all.size(), (size_t)names_cap - 1);
    memcpy(names, all.data(), nb);
    names[nb] = 0;
    return VX_OK;
}
