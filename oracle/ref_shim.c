/*
 * ref_shim.c — TEST INFRASTRUCTURE.  Host-side glue that lets the reference's
 * own src/unit_1.cu + src/kernel.cu (built unmodified into oracle/_ref by
 * oracle/build_ref.sh) be driven from Python through ctypes.
 *
 * The reference implementation reads globals owned by its src/main.c
 * (conf, current_step, first_step, n, cuda_error, log_lev, flush_log;
 * src/main.c:17-46, src/unit_1.cu:15-18).  This file defines them, plus
 * setters for conf fields and small device-memory helpers that use the same
 * CUDA runtime instance as the reference kernels.
 */
#include "incl.h"
#include <string.h>

struct conf_t conf;
int current_step = 0;
int first_step = 0;
size_t n = 0;
cudaError_t cuda_error = cudaSuccess;

void flush_log(void) {}

void log_lev(uint8_t lev, char *fmt, ...) {
    if (lev > LEV_ERROR) return;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fputc('\n', stderr);
}

#define SET_D(name) if (!strcmp(key, #name)) { conf.name = v; return 0; }
#define SET_U(name) if (!strcmp(key, #name)) { conf.name = (size_t)v; return 0; }

int vxref_conf_reset(void) { memset(&conf, 0, sizeof(conf)); conf.log_level = 1; return 0; }

int vxref_conf_set(const char *key, double v) {
    SET_D(dt) SET_D(viscosity) SET_D(rho) SET_D(v_inf_x) SET_D(v_inf_y)
    SET_D(x_max) SET_D(x_min) SET_D(y_max) SET_D(y_min)
    SET_D(profile_x_min) SET_D(profile_x_max) SET_D(profile_y_min) SET_D(profile_y_max)
    SET_D(ve_size) SET_D(h_col_x) SET_D(h_col_y) SET_D(rc_x) SET_D(rc_y)
    SET_D(r_col_diff_sign) SET_D(r_col_same_sign) SET_D(max_ve_g) SET_D(rel_t)
    SET_U(steps) SET_U(saving_step) SET_U(inc_step) SET_U(n_of_points)
    SET_U(n_col) SET_U(birth_quant) SET_U(v_inf_incr_steps)
    return 1;
}

size_t vxref_sizeof_vortex(void) { return sizeof(Vortex); }
size_t vxref_sizeof_panel(void) { return sizeof(tPanel); }

void *vxref_malloc(size_t bytes) {
    void *p = NULL;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return NULL;
    cudaMemset(p, 0, bytes);
    return p;
}
int vxref_free(void *p) { return cudaFree(p) != cudaSuccess; }
int vxref_h2d(void *dst, const void *src, size_t bytes) {
    return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess;
}
int vxref_d2h(void *dst, const void *src, size_t bytes) {
    return cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess;
}
int vxref_sync(void) { return cudaDeviceSynchronize() != cudaSuccess; }
