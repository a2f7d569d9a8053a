// vx_io.cpp — .conf and profile-file readers (host side of the C ABI).
//
// .conf: "key value" lines; a key matches when the line starts with the key
// followed by one space, anything after the value is ignored, unknown keys
// are ignored (reference read_config, src/main.c:48-115).  Keys this library
// adds: precision (fp64|fp32|0|1), birth_offset_mode (ref|file|half_panel|
// 0|1|2), drop_eps, diff_cutoff, fmm (0|1), fmm_leaf, fmm_p (8|12|16|20),
// gj_pivot (0..3), probe_grid n x0 x1 y0 y1.
//
// Profile: two header lines, the panel count, then that many records
// "n lx ly rx ry cx cy bx by nx ny tx ty len nL nR" (src/main.c:220-256).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/vortex_b200.h"

void vx_set_error(const char *fmt, ...);

static bool key_is(const char *buf, const char *key) {
    size_t k = strlen(key);
    return strncmp(buf, key, k) == 0 && buf[k] == ' ';
}

extern "C" vx_status vx_conf_read(const char *path, vx_conf *c) {
    if (!path || !c) return VX_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) { vx_set_error("unable to open config file %s", path); return VX_ERR_IO; }
    char buf[236];
    while (fgets(buf, sizeof(buf), f)) {
#define U(name) else if (key_is(buf, #name)) { unsigned long long v_ = 0; if (sscanf(buf, "%*s %llu", &v_) == 1) c->name = (int64_t)v_; }
#define D(name) else if (key_is(buf, #name)) { double v_ = 0; if (sscanf(buf, "%*s %lf", &v_) == 1) c->name = v_; }
#define B(name) else if (key_is(buf, #name)) { unsigned v_ = 0; if (sscanf(buf, "%*s %u", &v_) == 1) c->name = (int32_t)(v_ & 0xff); }
#define S(name) else if (key_is(buf, #name)) { char v_[256] = {0}; if (sscanf(buf, "%*s %255s", v_) == 1) { strncpy(c->name, v_, sizeof(c->name) - 1); c->name[sizeof(c->name) - 1] = 0; } }
        if (0) {}
        S(pr_file) S(timings_file) S(kadr_file) S(second_points_file)
        U(steps) U(saving_step) D(dt) U(v_inf_incr_steps) U(inc_step)
        D(viscosity) D(rho) D(v_inf_x) D(v_inf_y) U(n_of_points)
        D(x_max) D(x_min) D(y_max) D(y_min) D(ve_size) U(n_col)
        D(h_col_x) D(h_col_y) D(rc_x) D(rc_y) D(r_col_diff_sign) D(r_col_same_sign)
        B(matrix_load) D(max_ve_g) D(rel_t) B(steady_flow) U(tree_depth) D(theta) B(no_log_buf)
        D(drop_eps) D(diff_cutoff) B(fmm) B(gj_pivot)
        else if (key_is(buf, "fmm_leaf")) { int v_ = 0; if (sscanf(buf, "%*s %d", &v_) == 1 && v_ > 0) c->fmm_leaf = v_; }
        else if (key_is(buf, "fmm_p")) { int v_ = 0; if (sscanf(buf, "%*s %d", &v_) == 1) c->fmm_p = v_; }
        else if (key_is(buf, "precision")) {
            char v[32] = {0};
            if (sscanf(buf, "%*s %31s", v) == 1)
                c->precision = (!strcmp(v, "fp32") || !strcmp(v, "1")) ? VX_PREC_FP32 : VX_PREC_FP64;
        } else if (key_is(buf, "birth_offset_mode")) {
            char v[32] = {0};
            if (sscanf(buf, "%*s %31s", v) == 1) {
                if (!strcmp(v, "file") || !strcmp(v, "1")) c->birth_offset_mode = VX_BIRTH_FILE;
                else if (!strcmp(v, "half_panel") || !strcmp(v, "2")) c->birth_offset_mode = VX_BIRTH_HALF_PANEL;
                else c->birth_offset_mode = VX_BIRTH_REF;
            }
        } else if (key_is(buf, "probe_grid")) {
            int n = 0;
            double b[4] = {0, 0, 0, 0};
            if (sscanf(buf, "%*s %d %lf %lf %lf %lf", &n, &b[0], &b[1], &b[2], &b[3]) == 5) {
                c->n_probes_grid = n;
                memcpy(c->probe_box, b, sizeof(b));
            }
        }
#undef U
#undef D
#undef B
#undef S
    }
    fclose(f);
    return VX_OK;
}

extern "C" vx_status vx_profile_read(const char *path, vx_panel *out, int64_t cap, int64_t *P) {
    if (!path || !P) return VX_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) { vx_set_error("can't open profile file %s", path); return VX_ERR_IO; }
    char buf[255];
    if (!fgets(buf, sizeof(buf), f) || !fgets(buf, sizeof(buf), f)) {
        fclose(f);
        vx_set_error("profile %s: missing header lines", path);
        return VX_ERR_IO;
    }
    unsigned long long p = 0;
    if (fscanf(f, "%llu", &p) != 1 || p < 2) {
        fclose(f);
        vx_set_error("profile %s: bad panel count", path);
        return VX_ERR_IO;
    }
    *P = (int64_t)p;
    if (!out) { fclose(f); return VX_OK; }
    if ((int64_t)p > cap) { fclose(f); vx_set_error("profile %s: %llu panels > capacity", path, p); return VX_ERR_ARG; }
    for (unsigned long long i = 0; i < p; ++i) {
        vx_panel &q = out[i];
        memset(&q, 0, sizeof(q));
        unsigned n = 0, nl = 0, nr = 0;
        int got = fscanf(f, " %u %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %u %u", &n,
                         &q.left[0], &q.left[1], &q.right[0], &q.right[1], &q.contr[0], &q.contr[1],
                         &q.birth[0], &q.birth[1], &q.norm[0], &q.norm[1], &q.tang[0], &q.tang[1],
                         &q.length, &nl, &nr);
        if (got != 16) {
            fclose(f);
            vx_set_error("profile %s: record %llu unreadable", path, i);
            return VX_ERR_IO;
        }
        q.n = n; q.n_of_lpanel = nl; q.n_of_rpanel = nr;
    }
    fclose(f);
    return VX_OK;
}
