// vx_advect.cu — convection r <- r + V dt, absorption of vortices that cross
// the wall, removal of vortices that leave the window, per-particle force
// and moment terms, and their deterministic reduction.
//
// Reference: step_Kernel src/kernel.cu:1090-1143, hitting :1357-1431,
// summ_Kernel :1144-1157.  The reference sums serially in one thread; here
// each thread of a fixed partition accumulates a fixed strided subset,
// partitions reduce in a fixed tree and the launch's last block adds the
// partition sums in order, so the result is run-to-run identical.
#include <algorithm>

#include "vx_internal.cuh"

// Segment (x2,y2)->(x1,y1) against one panel: on a crossing, sets hit and
// keeps the crossing nearest to (x2,y2) (the lower panel index on a tie,
// which is the reference's choice when it scans panels in index order).
__device__ __forceinline__ void vx_hit_panel(const vx_panel &q, int i, double A, double B, double D, double x1,
                                             double y1, double x2, double y2, bool &hit, double &minDist,
                                             int &minN) {
    const double thr = 1e-12;
    double r0 = A * q.left[0] + B * q.left[1] + D;
    double r1 = A * q.right[0] + B * q.right[1] + D;
    if (fabs(r0) < thr) r0 = 0.0;
    if (fabs(r1) < thr) r1 = 0.0;
    if (r0 * r1 <= 0) {
        double A1 = q.right[1] - q.left[1];
        double B1 = q.left[0] - q.right[0];
        double D1 = q.left[1] * q.right[0] - q.left[0] * q.right[1];
        double r2 = A1 * x1 + B1 * y1 + D1;
        double r3 = A1 * x2 + B1 * y2 + D1;
        if (fabs(r2) < thr) r2 = 0.0;
        if (fabs(r3) < thr) r3 = 0.0;
        if (r2 * r3 <= 0) {
            hit = true;
            double den = A * B1 - B * A1;
            double X = (B * D1 - D * B1) / den;
            double Y = (A1 * D - D1 * A) / den;
            double d2 = (x2 - X) * (x2 - X) + (y2 - Y) * (y2 - Y);
            if (d2 < minDist || (d2 == minDist && minN >= 0 && i < minN)) { minDist = d2; minN = i; }
        }
    }
}

// Segment (x2,y2)->(x1,y1) against the panels; nearest crossing wins.  With
// hit lists (hstart/hidx: per cell of a grid over the body, every panel whose
// bounding box touches the cell) only the panels listed in the cells under
// the segment's bounding box are tested: a panel the segment crosses touches
// that box, so the set of crossings, and the nearest one, are unchanged.
__device__ bool vx_hitting(const VxParams &p, const vx_panel *pan, double x1, double y1, double x2,
                           double y2, int *hitpan, const int *hstart = nullptr, const int *hidx = nullptr) {
    double minDist = 25.0;
    int minN = -1;
    bool hit = !(((x1 < p.px_min) && (x2 < p.px_min)) || ((x1 > p.px_max) && (x2 > p.px_max)) ||
                 ((y1 < p.py_min) && (y2 < p.py_min)) || ((y1 > p.py_max) && (y2 > p.py_max)));
    if (hit) {
        hit = false;
        const double A = y2 - y1, B = x1 - x2, D = y1 * x2 - x1 * y2;
        bool done = false;
        if (hstart) {
            const double fx0 = (fmin(x1, x2) - p.hit_x0) / p.hit_h, fx1 = (fmax(x1, x2) - p.hit_x0) / p.hit_h;
            const double fy0 = (fmin(y1, y2) - p.hit_y0) / p.hit_h, fy1 = (fmax(y1, y2) - p.hit_y0) / p.hit_h;
            if (fx1 < 0.0 || fy1 < 0.0 || fx0 >= (double)p.hit_nx || fy0 >= (double)p.hit_ny) {
                done = true;   // the segment misses the grid, which holds every panel
            } else {
                const int cx0 = max((int)floor(fx0), 0), cx1 = min((int)floor(fx1), p.hit_nx - 1);
                const int cy0 = max((int)floor(fy0), 0), cy1 = min((int)floor(fy1), p.hit_ny - 1);
                if ((cx1 - cx0 + 1) * (cy1 - cy0 + 1) <= 16) {
                    for (int cy = cy0; cy <= cy1; ++cy)
                        for (int cx = cx0; cx <= cx1; ++cx) {
                            const int c = cy * p.hit_nx + cx;
                            for (int q = hstart[c]; q < hstart[c + 1]; ++q) {
                                const int i = hidx[q];
                                vx_hit_panel(pan[i], i, A, B, D, x1, y1, x2, y2, hit, minDist, minN);
                            }
                        }
                    done = true;
                }
            }
        }
        if (!done)
            for (int i = 0; i < p.P; ++i) vx_hit_panel(pan[i], i, A, B, D, x1, y1, x2, y2, hit, minDist, minN);
    }
    *hitpan = minN;
    return hit;
}

// True when vx_hitting would test every panel for this segment (it lies in
// the profile box, and with hit lists its bounding box covers more than 16
// cells of the grid).  k_advect gives such a segment to its whole warp.
__device__ __forceinline__ bool vx_hit_all_panels(const VxParams &p, double x1, double y1, double x2, double y2,
                                                  const int *hstart) {
    if (((x1 < p.px_min) && (x2 < p.px_min)) || ((x1 > p.px_max) && (x2 > p.px_max)) ||
        ((y1 < p.py_min) && (y2 < p.py_min)) || ((y1 > p.py_max) && (y2 > p.py_max)))
        return false;
    if (!hstart) return false;   // without lists every segment scans the panels itself
    const double fx0 = (fmin(x1, x2) - p.hit_x0) / p.hit_h, fx1 = (fmax(x1, x2) - p.hit_x0) / p.hit_h;
    const double fy0 = (fmin(y1, y2) - p.hit_y0) / p.hit_h, fy1 = (fmax(y1, y2) - p.hit_y0) / p.hit_h;
    if (fx1 < 0.0 || fy1 < 0.0 || fx0 >= (double)p.hit_nx || fy0 >= (double)p.hit_ny) return false;
    const int cx0 = max((int)floor(fx0), 0), cx1 = min((int)floor(fx1), p.hit_nx - 1);
    const int cy0 = max((int)floor(fy0), 0), cy1 = min((int)floor(fy1), p.hit_ny - 1);
    return (cx1 - cx0 + 1) * (cy1 - cy0 + 1) > 16;
}

__device__ __forceinline__ double vx_block_sum(double v, double *sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

// Partition `part` of `nparts` (the particles a block of a grid of nparts
// blocks would take) and its four block sums into red[4 part ..].
__device__ __forceinline__ void advect_part(unsigned part, unsigned nparts, const VxParams &p, const VxView &v,
                                            const VxScalars *S, const vx_panel *pan, double *red,
                                            const int *hstart, const int *hidx) {
    __shared__ double sh[VX_THREADS];
    const long long n = S->n;
    const long long n_new0 = S->n0;   // vortices born this step: [n0, n)
    const int lane = threadIdx.x & 31;
    double sdg = 0.0, sfx = 0.0, sfy = 0.0, sm = 0.0;
    // whole warps step together (lane i of the warp takes particle base + i),
    // so a long segment can be handed to the warp
    for (long long base = part * (long long)blockDim.x + (threadIdx.x & ~31); base < n;
         base += (long long)nparts * blockDim.x) {
        const long long i = base + lane;
        const bool valid = i < n;
        const long long k = i * v.ps;
        double x = valid ? v.x[k] : 0.0, y = valid ? v.y[k] : 0.0, gi = valid ? v.g[k] : 0.0;
        double fx = 0.0, fy = 0.0, m = 0.0;
        if (i >= n_new0) {
            double dx = x - p.rc_x, dy = y - p.rc_y;
            fx = gi * (-y);
            fy = gi * x;
            m = gi * fma(dx, dx, dy * dy);
        }
        const double xn = valid ? fma(v.vx[i * v.vs], p.dt, x) : 0.0;
        const double yn = valid ? fma(v.vy[i * v.vs], p.dt, y) : 0.0;
        // segments whose box covers many hit-grid cells: every panel, tested
        // by the whole warp (lanes over panels, then the nearest crossing,
        // the lower index on a tie: the sequential scan's answer)
        const bool all = valid && gi != 0 && vx_hit_all_panels(p, xn, yn, x, y, hstart);
        unsigned want = __ballot_sync(0xffffffffu, all);
        bool whit = false;
        int whp = -1;
        while (want) {
            const int src = __ffs(want) - 1;
            want &= want - 1;
            const double x1 = __shfl_sync(0xffffffffu, xn, src), y1 = __shfl_sync(0xffffffffu, yn, src);
            const double x2 = __shfl_sync(0xffffffffu, x, src), y2 = __shfl_sync(0xffffffffu, y, src);
            const double A = y2 - y1, B = x1 - x2, D = y1 * x2 - x1 * y2;
            bool h = false;
            double md = 25.0;
            int mn = -1;
            for (int q = lane; q < p.P; q += 32) vx_hit_panel(pan[q], q, A, B, D, x1, y1, x2, y2, h, md, mn);
            h = __any_sync(0xffffffffu, h);
            for (int o = 16; o > 0; o >>= 1) {
                const double od = __shfl_xor_sync(0xffffffffu, md, o);
                const int on = __shfl_xor_sync(0xffffffffu, mn, o);
                if (on >= 0 && (od < md || (od == md && (mn < 0 || on < mn)))) { md = od; mn = on; }
            }
            if (lane == src) { whit = h; whp = mn; }
        }
        int hp = -1;
        bool hit = false;
        if (all) { hit = whit; hp = whp; }
        else if (valid && gi != 0) hit = vx_hitting(p, pan, xn, yn, x, y, &hp, hstart, hidx);
        if (!valid) continue;
        if (hit) {
            if (hp >= 0) {   // the reference reads panels[-1] when no crossing is nearer than 5
                const double cx = pan[hp].contr[0], cy = pan[hp].contr[1];
                const double dx = cx - p.rc_x, dy = cy - p.rc_y;
                fx -= gi * (-cy);
                fy -= gi * cx;
                m -= gi * fma(dx, dx, dy * dy);
            }
            sdg += gi;
            gi = 0.0;
        }
        double xo = xn, yo = yn;
        if (gi != 0 && (xn > p.x_max || xn < p.x_min || yn > p.y_max || yn < p.y_min)) {
            xo = -2.0e5; yo = -2.0e5; gi = 0.0;
        }
        v.x[k] = xo; v.y[k] = yo; v.g[k] = gi;
        sfx += fx; sfy += fy; sm += m;
    }
    double t;
    t = vx_block_sum(sdg, sh); if (threadIdx.x == 0) red[part * 4 + 0] = t;
    t = vx_block_sum(sfx, sh); if (threadIdx.x == 0) red[part * 4 + 1] = t;
    t = vx_block_sum(sfy, sh); if (threadIdx.x == 0) red[part * 4 + 2] = t;
    t = vx_block_sum(sm, sh);  if (threadIdx.x == 0) red[part * 4 + 3] = t;
}
// The particles are split into nparts fixed partitions (block-strided, as a
// grid of nparts blocks would take them) whatever the grid: each block takes
// partitions blockIdx, blockIdx + grid, ...; a partition past the last
// particle has zero sums.  The partial sums, and so the totals, do not depend
// on the grid the kernel runs with.  The block that finishes last adds the
// partition sums: thread t adds partitions t, t + 256, ... in order, then a
// fixed shared-memory tree, so the result is run-to-run identical.
VX_DEVK void k_advect_body(VxBlkB<VX_THREADS, 0> vb, const VxParams &p, const VxView &v, VxScalars *S, const vx_panel *pan,
                           double *red, const int *hstart, const int *hidx, int sms) {
    const long long n = S->n;
    const int nparts = vx_body_parts(n, sms, VX_RED_BLOCKS);
    for (unsigned q = vb.x; q < (unsigned)nparts; q += vb.n) {
        if ((long long)q * blockDim.x >= n) {
            if (threadIdx.x < 4) red[q * 4 + threadIdx.x] = 0.0;
            continue;
        }
        advect_part(q, (unsigned)nparts, p, v, S, pan, red, hstart, hidx);
    }
    if (!vx_last_block(&S->sync_ctr, vb.n)) return;
    __shared__ double sh[VX_THREADS];
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x)
        for (int q = 0; q < 4; ++q) a[q] += __ldcg(&red[b * 4 + q]);
    for (int q = 0; q < 4; ++q) a[q] = vx_block_sum(a[q], sh);
    if (threadIdx.x != 0) return;
    for (int q = 0; q < 4; ++q) S->raw[q] = a[q];
    S->dg = a[0];
    S->fx = a[1] * (p.rho / p.dt);
    S->fy = a[2] * (p.rho / p.dt);
    S->m = a[3] * (p.rho / (2 * p.dt));
}
__global__ void __launch_bounds__(VX_THREADS) k_advect(VxParams p, VxView v, VxScalars *S, const vx_panel *pan,
                                                       double *red, const int *hstart, const int *hidx, int sms) {
    VX_PDL_WAIT();
    k_advect_body(VxBlkB<VX_THREADS, 0>{blockIdx.x, gridDim.x}, p, v, S, pan, red, hstart, hidx, sms);
}

cudaError_t vx_launch_advect(const VxLaunch &L, const VxParams &p, const VxView &v, VxScalars *S,
                             VxWork &w, const vx_panel *pan, const int *hstart, const int *hidx) {
    if (p.hit_nx <= 0 || p.hit_ny <= 0) hstart = hidx = nullptr;
    // partitions of the force sums follow the body's count on the device
    // (vx_body_parts), the grid the SMs this launch is given
    const int grid = std::min(VX_RED_BLOCKS, L.num_sms * 4);
    vx_launch<k_advect, k_advect_body>(L, grid, VX_THREADS, 0, p, v, S, pan, w.red, hstart, hidx, vx_full_sms(L));
    return cudaGetLastError();
}
