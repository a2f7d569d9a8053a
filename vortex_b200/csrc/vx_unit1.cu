// vx_unit1.cu — the reference's step API (include/unit_1.cuh:15-55) on top
// of this library's kernels, declared in include/vortex_b200_unit1.h.
//
// The kernels take a strided view of the particle arrays, so they run
// directly on the caller's AoS records (vortex = x, y, G: stride 3 doubles;
// velocity: stride 2) without conversion.  Precision follows the plain FP64
// form unless VORTEX_B200_PRECISION=fp32 is set in the environment.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <cmath>
#include <vector>

#include "../../include/vortex_b200_unit1.h"
#include "vx_internal.cuh"

static_assert(sizeof(vxu_conf_t) == 1792, "conf_t layout");
static_assert(offsetof(vxu_conf_t, pr_file) == 184 && offsetof(vxu_conf_t, birth_quant) == 440 &&
                  offsetof(vxu_conf_t, v_inf_incr_steps) == 472 && offsetof(vxu_conf_t, log_file) == 488 &&
                  offsetof(vxu_conf_t, log_level) == 1000 && offsetof(vxu_conf_t, rel_t) == 1776 &&
                  offsetof(vxu_conf_t, no_log_buf) == 1785,
              "conf_t layout");
static_assert(sizeof(vxu_vortex) == 24 && sizeof(vxu_velocity) == 16 && sizeof(vx_panel) == 120,
              "record layouts");

// The host driver's configuration (src/main.c:17).  A definition in the
// executable that loads this library takes precedence over this one.
extern "C" {
struct vxu_conf_t conf;
int current_step = 0;   // src/main.c:18-19, read by the tracer entry points
int first_step = 0;
}

namespace {

struct Ctx {
    bool ready = false;
    VxParams prm;
    int num_sms = 148;
    VxScalars *d_S = nullptr;
    VxScalars *h_S = nullptr;
    VxWork w;
    std::vector<void *> allocs;
    long long w_cap = 0;
    int w_P32 = 0;
    const void *wall_for = nullptr;
    long long launches = 0;
};
Ctx U;

VxLaunch launch0() {
    VxLaunch L;
    L.stream = 0;
    L.launches = &U.launches;
    L.num_sms = U.num_sms;
    return L;
}

int cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return 0;
    fprintf(stderr, "vortex_b200: %s: %s\n", what, cudaGetErrorString(e));
    vx_set_error("%s: %s", what, cudaGetErrorString(e));
    return 1;
}
#define CK(call) do { if (cuda_fail((call), #call)) return 1; } while (0)

int setup_params() {
    vx_conf c;
    vx_conf_default(&c);
    c.dt = conf.dt;
    c.viscosity = conf.viscosity;
    c.rho = conf.rho;
    c.ve_size = conf.ve_size;
    c.r_col_diff_sign = conf.r_col_diff_sign;
    c.r_col_same_sign = conf.r_col_same_sign;
    c.max_ve_g = conf.max_ve_g;
    c.x_min = conf.x_min; c.x_max = conf.x_max; c.y_min = conf.y_min; c.y_max = conf.y_max;
    c.rc_x = conf.rc_x; c.rc_y = conf.rc_y;
    c.n_of_points = (int64_t)conf.n_of_points;
    c.n_col = (int64_t)conf.n_col;
    const char *prec = getenv("VORTEX_B200_PRECISION");
    c.precision = (prec && !strcmp(prec, "fp32")) ? VX_PREC_FP32 : VX_PREC_FP64;
    vx_params_from_conf(&c, nullptr, 0, &U.prm);
    // the driver computed the profile box from the left endpoints (src/main.c:235-254)
    U.prm.px_min = conf.profile_x_min; U.prm.px_max = conf.profile_x_max;
    U.prm.py_min = conf.profile_y_min; U.prm.py_max = conf.profile_y_max;
    U.prm.P = (int)conf.birth_quant;
    U.prm.wall_x0 = -1e300; U.prm.wall_x1 = 1e300; U.prm.wall_y0 = -1e300; U.prm.wall_y1 = 1e300;
    U.wall_for = nullptr;
    if (!U.d_S) {
        if (cuda_fail(cudaMalloc(&U.d_S, sizeof(VxScalars)), "cudaMalloc")) return 1;
        if (cuda_fail(cudaMallocHost(&U.h_S, sizeof(VxScalars)), "cudaMallocHost")) return 1;
        memset(U.h_S, 0, sizeof(VxScalars));
        if (cuda_fail(cudaMemcpy(U.d_S, U.h_S, sizeof(VxScalars), cudaMemcpyHostToDevice), "cudaMemcpy")) return 1;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&U.num_sms, cudaDevAttrMultiProcessorCount, dev);
    U.ready = true;
    return 0;
}

int ensure_ready() { return U.ready ? 0 : setup_params(); }

int ensure_work(long long slots) {
    const int P32 = (int)vx_round32(std::max(U.prm.P, 1));
    if (slots + 64 <= U.w_cap && P32 == U.w_P32) return 0;
    long long cap = vx_ceil_div(std::max(slots + 64, U.w_cap * 5 / 4), 8192) * 8192;
    if (vx_work_alloc(U.w, U.allocs, cap, P32, U.num_sms) != VX_OK) return 1;
    U.w_cap = cap;
    U.w_P32 = P32;
    return 0;
}

// The wall term is skipped beyond 5 L_max of every birth point; the box
// comes from the caller's device panels.
int ensure_wall_box(const vx_panel *d_pan) {
    if (U.wall_for == d_pan) return 0;
    const int P = U.prm.P;
    std::vector<vx_panel> hp(P);
    CK(cudaMemcpy(hp.data(), d_pan, sizeof(vx_panel) * P, cudaMemcpyDeviceToHost));
    double bx0 = 1e300, bx1 = -1e300, by0 = 1e300, by1 = -1e300, lmax = 0.0;
    for (const vx_panel &q : hp) {
        bx0 = std::min(bx0, q.birth[0]); bx1 = std::max(bx1, q.birth[0]);
        by0 = std::min(by0, q.birth[1]); by1 = std::max(by1, q.birth[1]);
        lmax = std::max(lmax, q.length);
    }
    const double m = 5.0 * lmax * (1.0 + 1e-9) + 1e-12;
    U.prm.wall_x0 = bx0 - m; U.prm.wall_x1 = bx1 + m; U.prm.wall_y0 = by0 - m; U.prm.wall_y1 = by1 + m;
    U.wall_for = d_pan;
    return 0;
}

__global__ void k_u_set(VxScalars *S, long long n, long long n0, const double *vinf, const double *dg) {
    VX_PDL_WAIT();
    S->n = n;
    S->n0 = n0;
    if (vinf) { S->vinf[0] = vinf[0]; S->vinf[1] = vinf[1]; }
    if (dg) S->dg = dg[0];
}

// summ_Kernel (src/kernel.cu:1144-1157): d_g overwritten, F and M accumulated
// onto the caller's values and then scaled.
__global__ void k_u_sums(VxParams p, const VxScalars *S, double *d_g, double *F, double *M) {
    VX_PDL_WAIT();
    if (d_g) d_g[0] = S->raw[0];
    if (F) {
        F[0] = (F[0] + S->raw[1]) * (p.rho / p.dt);
        F[1] = (F[1] + S->raw[2]) * (p.rho / p.dt);
    }
    if (M) M[0] = (M[0] + S->raw[3]) * (p.rho / (2 * p.dt));
}

__global__ void k_u_tail(double *pos, long long from, long long to) {
    VX_PDL_WAIT();
    for (long long i = from + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < to;
         i += (long long)gridDim.x * blockDim.x) {
        pos[3 * i] = 4.0e5 + (double)i;
        pos[3 * i + 1] = 4.0e5 + (double)i;
        pos[3 * i + 2] = 0.0;
    }
}

VxView aos_view(vxu_vortex *pos, vxu_velocity *vel, double *d) {
    VxView v;
    v.x = (double *)pos; v.y = v.x + 1; v.g = v.x + 2; v.ps = 3;
    v.vx = vel ? (double *)vel : nullptr; v.vy = vel ? v.vx + 1 : nullptr; v.vs = 2;
    v.d = d;
    return v;
}

int write_matrix(const char *name, const double *A, size_t S) {
    FILE *f = fopen(name, "w");
    if (!f) return 2;
    fprintf(f, "%zu\n", S);
    for (size_t i = 0; i < S; ++i) {
        for (size_t j = 0; j < S; ++j) fprintf(f, "%lf\t", A[i * S + j]);
        fprintf(f, "\n");
    }
    fclose(f);
    return 0;
}

}  // namespace

extern "C" {

int init_device_conf_values(void) { return setup_params(); }

double *matr_creation(vx_panel *panels, size_t s, size_t birth) {
    if (!panels || s < 2 || birth < s) return nullptr;
    const long long S1 = (long long)s + 1;
    vx_panel *d_pan = nullptr;
    double *d_minv = nullptr, *d_work = nullptr, *d_L = nullptr;
    int *d_flag = nullptr;
    double *MM = nullptr;
    std::vector<double> L(S1 * S1), M(S1 * S1);
    int hflag = 1;
    bool ok = cudaMalloc(&d_pan, sizeof(vx_panel) * s) == cudaSuccess &&
              cudaMalloc(&d_minv, sizeof(double) * S1 * S1) == cudaSuccess &&
              cudaMalloc(&d_L, sizeof(double) * S1 * S1) == cudaSuccess &&
              cudaMalloc(&d_work, sizeof(double) * (2 * S1 * S1 + S1)) == cudaSuccess &&
              cudaMalloc(&d_flag, sizeof(int)) == cudaSuccess &&
              cudaMemcpy(d_pan, panels, sizeof(vx_panel) * s, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&U.num_sms, cudaDevAttrMultiProcessorCount, dev);
        ok = vx_build_matrix(launch0(), d_pan, (int)s, d_minv, d_work, d_flag, d_L) == cudaSuccess &&
             cudaMemcpy(&hflag, d_flag, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
             cudaMemcpy(L.data(), d_L, sizeof(double) * S1 * S1, cudaMemcpyDeviceToHost) == cudaSuccess &&
             cudaMemcpy(M.data(), d_minv, sizeof(double) * S1 * S1, cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    cudaFree(d_pan); cudaFree(d_minv); cudaFree(d_L); cudaFree(d_work); cudaFree(d_flag);
    if (!ok) return nullptr;
    write_matrix("L.txt", L.data(), S1);
    if (hflag) return nullptr;
    write_matrix("M.txt", M.data(), S1);
    const size_t B1 = birth + 1;
    MM = (double *)calloc(B1 * B1, sizeof(double));
    if (!MM) return nullptr;
    for (long long i = 0; i < S1; ++i)
        for (long long j = 0; j < S1; ++j) MM[i * B1 + j] = M[i * S1 + j];
    return MM;
}

double *load_matrix(size_t *p) {
    if (!p) return nullptr;
    FILE *f = fopen("M.txt", "r");
    if (!f) { fprintf(stderr, "vortex_b200: unable to open matrix file M.txt\n"); return nullptr; }
    size_t S = 0;
    if (fscanf(f, "%zu", &S) != 1 || S < 2) { fclose(f); return nullptr; }
    *p = S - 1;
    std::vector<double> M(S * S);
    for (size_t k = 0; k < S * S; ++k)
        if (fscanf(f, "%lf ", &M[k]) != 1) { fclose(f); return nullptr; }
    fclose(f);
    const size_t birth = (size_t)(32 * std::ceil((double)(*p) / 32));
    const size_t B1 = birth + 1;
    double *MM = (double *)calloc(B1 * B1, sizeof(double));
    if (!MM) return nullptr;
    for (size_t i = 0; i < S; ++i)
        for (size_t j = 0; j < S; ++j) MM[i * B1 + j] = M[i * S + j];
    return MM;
}

int allocate_arrays(vxu_vortex **p_host, vxu_vortex **p_dev, vxu_velocity **v_host, vxu_velocity **v_dev,
                    double **d_dev, size_t size) {
    if (!p_host || !p_dev || !v_host || !v_dev || !d_dev || !size) return 2;
    *p_host = (vxu_vortex *)calloc(size, sizeof(vxu_vortex));
    *v_host = (vxu_velocity *)calloc(size, sizeof(vxu_velocity));
    if (!*p_host || !*v_host) return 1;
    CK(cudaMalloc((void **)p_dev, size * sizeof(vxu_vortex)));
    CK(cudaMemset(*p_dev, 0, size * sizeof(vxu_vortex)));
    CK(cudaMalloc((void **)d_dev, size * sizeof(double)));
    CK(cudaMemset(*d_dev, 0, size * sizeof(double)));
    CK(cudaMalloc((void **)v_dev, size * sizeof(vxu_velocity)));
    CK(cudaMemset(*v_dev, 0, size * sizeof(vxu_velocity)));
    return 0;
}

int randomize_tail(vxu_vortex **p_dev, size_t new_size, size_t increased) {
    if (!p_dev || !*p_dev || increased > new_size) return 2;
    k_u_tail<<<64, 256>>>((double *)*p_dev, (long long)(new_size - increased), (long long)new_size);
    ++U.launches;
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    return 0;
}

int incr_vort_quant(vxu_vortex **p_host, vxu_vortex **p_dev, vxu_velocity **v_host, vxu_velocity **v_dev,
                    double **d_dev, size_t *size) {
    if (!p_host || !p_dev || !v_host || !v_dev || !d_dev || !size) return 2;
    if (*p_host && *p_dev && *v_host && *v_dev && *d_dev) {
        vxu_vortex *np = nullptr;
        const size_t ns = *size + conf.inc_step;
        CK(cudaMalloc((void **)&np, ns * sizeof(vxu_vortex)));
        CK(cudaMemcpy(np, *p_dev, *size * sizeof(vxu_vortex), cudaMemcpyDeviceToDevice));
        *size = ns;
        free(*p_host);
        free(*v_host);
        *p_host = (vxu_vortex *)calloc(ns, sizeof(vxu_vortex));
        *v_host = (vxu_velocity *)calloc(ns, sizeof(vxu_velocity));
        cudaFree(*p_dev);
        cudaFree(*d_dev);
        cudaFree(*v_dev);
        CK(cudaMalloc((void **)d_dev, ns * sizeof(double)));
        CK(cudaMalloc((void **)v_dev, ns * sizeof(vxu_velocity)));
        *p_dev = np;
    } else if (!*p_host && !*p_dev && !*v_host && !*v_dev && !*d_dev) {
        *size = conf.inc_step;
        if (allocate_arrays(p_host, p_dev, v_host, v_dev, d_dev, *size)) return 1;
    } else {
        return 2;
    }
    return randomize_tail(p_dev, *size, conf.inc_step);
}

int vort_creation(vxu_vortex *pos, double (*V_infDev)[2], size_t n_of_birth, size_t n_of_birth_BLOCK_S,
                  size_t n, double *M_Dev, double *d_g, vx_panel *panels) {
    if (!pos || !V_infDev || !M_Dev || !d_g || !panels || n_of_birth < 2) return 2;
    if (ensure_ready()) return 1;
    U.prm.P = (int)n_of_birth;
    if (ensure_work((long long)n + (long long)n_of_birth_BLOCK_S)) return 1;
    k_u_set<<<1, 1>>>(U.d_S, (long long)n, (long long)n, (const double *)V_infDev, d_g);
    ++U.launches;
    const int tiles = (int)vx_ceil_div(n_of_birth, 128);
    const int chunks = (int)std::max(1LL, std::min((long long)U.num_sms * 4 / tiles, vx_ceil_div((long long)n, 2048)));
    CK(vx_launch_birth_ld(launch0(), U.prm, aos_view(pos, nullptr, nullptr), U.d_S, U.w, panels, M_Dev,
                          (long long)n_of_birth_BLOCK_S + 1, chunks));
    CK(cudaDeviceSynchronize());
    return 0;
}

void start_timer(void **start, void **stop) {
    cudaEventCreate((cudaEvent_t *)start);
    cudaEventCreate((cudaEvent_t *)stop);
    cudaEventRecord((cudaEvent_t)*start, 0);
    cudaEventSynchronize((cudaEvent_t)*start);
}

float stop_timer(void *start, void *stop) {
    cudaEventRecord((cudaEvent_t)stop, 0);
    cudaEventSynchronize((cudaEvent_t)stop);
    float t = 0.0f;
    cudaEventElapsedTime(&t, (cudaEvent_t)start, (cudaEvent_t)stop);
    cudaEventDestroy((cudaEvent_t)start);
    cudaEventDestroy((cudaEvent_t)stop);
    return t / 1000;
}

int Speed(vxu_vortex *pos, double (*v_inf)[2], size_t s, vxu_velocity *v, double *d, double nu,
          vx_panel *panels) {
    if (!pos || !v_inf || !v || !d || !panels) return 2;
    if (ensure_ready()) return 1;
    if (ensure_work((long long)s) || ensure_wall_box(panels)) return 1;
    U.prm.nu = nu;
    // the reference evaluates all s slots as targets and sources
    k_u_set<<<1, 1>>>(U.d_S, (long long)s, (long long)s, (const double *)v_inf, nullptr);
    ++U.launches;
    const VxLaunch L = launch0();
    const VxView vw = aos_view(pos, v, d);
    CK(vx_launch_velocity(L, U.prm, vw, U.d_S, U.w));
    CK(vx_launch_diffusion(L, U.prm, vw, U.d_S, U.w));
    CK(vx_launch_wall(L, U.prm, vw, U.d_S, panels));
    CK(cudaDeviceSynchronize());
    return 0;
}

int Step(vxu_vortex *pos, vxu_velocity *V, size_t *n, size_t s, double *d_g, vxu_velocity *F_p, double *M,
         vx_panel *panels) {
    if (!pos || !V || !n || !panels) return 2;
    if (ensure_ready()) return 1;
    if (ensure_work((long long)std::max(s, *n))) return 1;
    const long long nn = (long long)*n, P = U.prm.P;
    // newborns are the last P (the reference tests i >= n - quant in size_t)
    k_u_set<<<1, 1>>>(U.d_S, nn, nn >= P ? nn - P : nn, nullptr, nullptr);
    ++U.launches;
    const VxLaunch L = launch0();
    const VxView vw = aos_view(pos, V, nullptr);
    CK(vx_launch_advect(L, U.prm, vw, U.d_S, U.w, panels));
    k_u_sums<<<1, 1>>>(U.prm, U.d_S, d_g, (double *)F_p, M);
    ++U.launches;
    CK(vx_launch_compact(L, U.prm, vw, U.d_S, U.w));
    CK(vx_launch_collapse(L, U.prm, vw, U.d_S, U.w, 1, (int)conf.n_col));
    CK(vx_launch_collapse(L, U.prm, vw, U.d_S, U.w, 2, (int)conf.n_col));
    CK(cudaMemcpy(U.h_S, U.d_S, sizeof(VxScalars), cudaMemcpyDeviceToHost));
    if (U.h_S->err) {
        fprintf(stderr, "vortex_b200: device error flag 0x%x\n", U.h_S->err);
        return 1;
    }
    *n = (size_t)U.h_S->n;
    return 0;
}

int velocity_control(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *Contr_points,
                     vxu_velocity *V, size_t n_contr) {
    if (!pos || !V_inf || !Contr_points || !V) return 2;
    if (n_contr == 0) return 0;
    if (ensure_ready()) return 1;
    if (ensure_work((long long)std::max(n, n_contr))) return 1;
    k_u_set<<<1, 1>>>(U.d_S, (long long)n, (long long)n, (const double *)V_inf, nullptr);
    ++U.launches;
    const double *px = (const double *)Contr_points;
    double *ov = (double *)V;
    const int tile = U.prm.prec == VX_PREC_FP32 ? 1024 : 512;
    const int K = vx_ksplit((long long)n_contr, tile, U.num_sms);
    CK(vx_launch_probe(launch0(), U.prm, aos_view(pos, nullptr, nullptr), U.d_S, U.w, px, px + 1, 3,
                       (long long)n_contr, ov, ov + 1, 2, K));
    CK(cudaDeviceSynchronize());
    return 0;
}

// Relaxation of inertial tracers towards the carrier velocity
// (second_speed_Kernel, src/kernel.cu:1478-1489); the previous velocity is
// rounded to float there, and so it is here.
__global__ void k_u_relax(const double *pos, const double *venv, double *v, long long nt, double rel_t,
                          double dt) {
    VX_PDL_WAIT();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nt;
         i += (long long)gridDim.x * blockDim.x) {
        if (!pos[3 * i + 2]) { v[2 * i] = 0.0; v[2 * i + 1] = 0.0; continue; }
        const float px = (float)v[2 * i], py = (float)v[2 * i + 1];
        v[2 * i] = (venv[2 * i] - px) / rel_t * dt + px;
        v[2 * i + 1] = (venv[2 * i + 1] - py) / rel_t * dt + py;
    }
}

static void save_vel(const vxu_vortex *d_pos, const vxu_velocity *d_vel, size_t nt, int step, int stage) {
    std::vector<vxu_vortex> P(nt);
    std::vector<vxu_velocity> V(nt);
    if (cudaMemcpy(P.data(), d_pos, nt * sizeof(vxu_vortex), cudaMemcpyDeviceToHost) != cudaSuccess) return;
    if (cudaMemcpy(V.data(), d_vel, nt * sizeof(vxu_velocity), cudaMemcpyDeviceToHost) != cudaSuccess) return;
    char fname[256];
    snprintf(fname, sizeof(fname), "output/vels/Vel%06d_%d.txt", step, stage);
    FILE *f = fopen(fname, "w");
    if (!f) return;
    fprintf(f, "%zu\n", nt);
    for (size_t i = 0; i < nt; ++i)
        fprintf(f, "%zu %lf %lf %lf %lf\n", i, P[i].r[0], P[i].r[1], V[i].v[0], V[i].v[1]);
    fclose(f);
}

// Tracers move with the velocity field and are absorbed by the wall and the
// window like vortices (step_Kernel without the force terms).
static int advect_tracers(vxu_vortex *tp, vxu_velocity *tv, size_t nt, vx_panel *panels) {
    if (ensure_work((long long)nt)) return 1;
    k_u_set<<<1, 1>>>(U.d_S, (long long)nt, (long long)nt, nullptr, nullptr);
    ++U.launches;
    CK(vx_launch_advect(launch0(), U.prm, aos_view(tp, tv, nullptr), U.d_S, U.w, panels));
    CK(cudaDeviceSynchronize());
    return 0;
}

// include/unit_1.cuh:52 — passive tracers (src/unit_1.cu:1271-1298).
int first_speed(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *second_pos,
                vxu_velocity *v_second, size_t *n_second, vx_panel *panels) {
    if (!n_second) return 2;
    if (velocity_control(pos, V_inf, n, second_pos, v_second, *n_second)) return 1;
    save_vel(second_pos, v_second, *n_second, current_step, 5);
    return advect_tracers(second_pos, v_second, *n_second, panels);
}

// include/unit_1.cuh:51 — inertial tracers relaxing towards the carrier
// velocity with time constant rel_t (src/unit_1.cu:1300-1340).
int second_speed(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *second_pos,
                 vxu_velocity *v_second, vxu_velocity *v_env, size_t *n_second, vx_panel *panels) {
    if (!n_second || !v_env) return 2;
    if (velocity_control(pos, V_inf, n, second_pos, v_env, *n_second)) return 1;
    if (current_step == first_step)
        CK(cudaMemcpy(v_second, v_env, sizeof(vxu_velocity) * (*n_second), cudaMemcpyDeviceToDevice));
    save_vel(second_pos, v_env, *n_second, current_step, 4);
    k_u_relax<<<64, 256>>>((const double *)second_pos, (const double *)v_env, (double *)v_second,
                           (long long)*n_second, conf.rel_t, conf.dt);
    ++U.launches;
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    save_vel(second_pos, v_second, *n_second, current_step, 5);
    return advect_tracers(second_pos, v_second, *n_second, panels);
}

// Kernel launches issued by the unit_1.cuh entry points since load.
int64_t vxu_launch_count(void) { return U.launches; }

}  // extern "C"

// ---------------------------------------------------------------------------
// velocity_control_noalloc: velocity_control for callers that must not
// allocate device memory.  Some host programs cannot call cudaMalloc where
// they sample the flow: a process whose device memory is already held by
// another runtime's caching allocator (a cudaMalloc there fails, or forces
// that allocator to release its cache), or a program that reserves a fixed
// device-memory budget at start-up and may not grow past it.  This entry
// point computes the same velocities with its scratch (the per-split partial
// sums of the Biot-Savart kernel and the device scalars) in the fixed
// file-scope array below, which every GPU that loads this library holds
// until the process exits.
//
// Limits and behaviour:
//   * at most VXU_NOALLOC_MAX_POINTS control points per call; more are
//     rejected with return code 2 and a message (nothing is launched);
//   * the plain FP64 form always (the FP32 form needs source scratch that
//     grows with the vortex count); with VORTEX_B200_PRECISION unset its
//     results are bit-identical to velocity_control's;
//   * the core radius is the one velocity_control uses: the value fixed when
//     init_device_conf_values (or the first entry point) ran, or, before
//     that, conf.ve_size at the call;
//   * each call launches on the legacy default stream and ends with a
//     device-wide synchronisation, like the reference's entry points: it
//     must not run while any stream on the device is being captured;
//   * the first call on a device, with that device current, looks up the
//     array's device address (cudaGetSymbolAddress) and the SM count;
//   * every call on a device shares the one array and finds there what the
//     previous call left: the scalars are cleared at the start of each call
//     and the partial sums are fully rewritten before they are read.  Calls
//     that overlap on the same GPU (from several host threads) race on the
//     array and must be serialised by the caller.
namespace {
constexpr long long NA_MAX_POINTS = 4096;   // control points per call
constexpr int NA_MAX_SPLIT = 64;            // source splits (vx_ksplit's cap)
constexpr long long NA_HEAD = ((long long)sizeof(VxScalars) + 255) / 256 * 256 / (long long)sizeof(double);
constexpr long long NA_PART = 2LL * NA_MAX_SPLIT * NA_MAX_POINTS;
constexpr long long NA_WORDS = NA_HEAD + NA_PART;   // 4 MiB + the scalars
constexpr int NA_MAX_DEVICES = 64;
static_assert(NA_MAX_POINTS == VXU_NOALLOC_MAX_POINTS, "header limit");
}  // namespace

// File-scope scratch of velocity_control_noalloc.  In host code this name is
// only a handle for cudaGetSymbolAddress, not a device address.
static __device__ __align__(256) double vx_noalloc_scratch[NA_WORDS];

namespace {
struct NaDevice {
    double *base = nullptr;   // device address of vx_noalloc_scratch
    int num_sms = 0;
};
NaDevice g_na[NA_MAX_DEVICES];
std::mutex g_na_mu;

int na_device(int dev, NaDevice **out) {
    std::lock_guard<std::mutex> lock(g_na_mu);
    NaDevice &d = g_na[dev];
    if (!d.base) {
        void *ptr = nullptr;
        CK(cudaGetSymbolAddress(&ptr, vx_noalloc_scratch));
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        d.num_sms = sms > 0 ? sms : 1;
        d.base = (double *)ptr;
    }
    *out = &d;
    return 0;
}
}  // namespace

extern "C" int velocity_control_noalloc(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *Contr_points,
                                        vxu_velocity *V, size_t n_contr) {
    if (!pos || !V_inf || !Contr_points || !V) return 2;
    if (n_contr == 0) return 0;
    if (n_contr > (size_t)NA_MAX_POINTS) {
        fprintf(stderr, "vortex_b200: velocity_control_noalloc: %zu control points, at most %lld\n", n_contr,
                NA_MAX_POINTS);
        vx_set_error("velocity_control_noalloc: %zu control points, at most %lld", n_contr, NA_MAX_POINTS);
        return 2;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        vx_set_error("velocity_control_noalloc: device %d beyond %d", dev, NA_MAX_DEVICES);
        return 2;
    }
    NaDevice *d = nullptr;
    if (na_device(dev, &d)) return 1;
    VxParams prm;
    memset(&prm, 0, sizeof(prm));
    prm.prec = VX_PREC_FP64;
    prm.eps = U.ready ? U.prm.eps : conf.ve_size;
    prm.eps2 = U.ready ? U.prm.eps2 : conf.ve_size * conf.ve_size;
    VxWork w;
    memset(&w, 0, sizeof(w));
    w.part = d->base + NA_HEAD;
    w.part_cap = NA_PART;
    VxScalars *S = (VxScalars *)d->base;
    VxLaunch L;
    L.stream = 0;
    L.launches = &U.launches;
    L.num_sms = d->num_sms;
    CK(cudaMemsetAsync(S, 0, sizeof(VxScalars), 0));
    k_u_set<<<1, 1>>>(S, (long long)n, (long long)n, (const double *)V_inf, nullptr);
    ++U.launches;
    const double *px = (const double *)Contr_points;
    double *ov = (double *)V;
    const int K = vx_ksplit((long long)n_contr, 512, d->num_sms);
    CK(vx_launch_probe(L, prm, aos_view(pos, nullptr, nullptr), S, w, px, px + 1, 3, (long long)n_contr, ov,
                       ov + 1, 2, K));
    CK(cudaDeviceSynchronize());
    return 0;
}
