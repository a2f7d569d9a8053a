/*
 * vortex_b200_unit1.h — the reference's step API, exported by
 * libvortex_b200.so with the same names, argument meaning and return codes,
 * so the reference's host driver (src/main.c) links against this library in
 * place of its src/unit_1.cu + src/kernel.cu.
 *
 * Every entry point below replaces the declaration at the cited line of the
 * reference's include/unit_1.cuh.  Records use the reference's layouts
 * (include/definitions.h, NO_TREE build): a vortex is 3 doubles (x, y, G),
 * a velocity 2 doubles, a panel the 120-byte vx_panel.  Arrays passed as
 * "device" are device pointers, as in the reference.
 *
 * Like the reference, the implementation reads the run configuration from a
 * global `struct conf_t conf` that the host driver owns (src/main.c:17); the
 * library also defines `conf` so that it can be used without that driver
 * (a definition in the executable takes precedence).  Calls run on the legacy
 * default stream and return after the device work finished; they are not
 * re-entrant (the reference's are not either).
 *
 * Return codes: 0 ok, 1 CUDA failure, 2 bad arguments; matrix functions
 * return NULL on failure.
 */
#ifndef VORTEX_B200_UNIT1_H_
#define VORTEX_B200_UNIT1_H_

#include <stddef.h>
#include <stdint.h>

#include "vortex_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vxu_vortex { double r[2]; double g; } vxu_vortex;   /* Vortex  */
typedef struct vxu_velocity { double v[2]; } vxu_velocity;         /* PVortex */

/* Layout-identical to the reference's struct conf_t without NO_TREE fields
 * (include/definitions.h:105-142): 1792 bytes. */
struct vxu_conf_t {
    size_t steps, saving_step;
    double dt;
    size_t inc_step;
    double viscosity, rho;
    double v_inf_x;
    double v_inf_y;
    size_t n_of_points;
    double x_max, x_min, y_max, y_min;
    double profile_x_min;
    double profile_x_max;
    double profile_y_min;
    double profile_y_max;
    double ve_size;
    size_t n_col;
    double h_col_x, h_col_y;
    double rc_x;
    double rc_y;
    char pr_file[256];
    size_t birth_quant;
    double r_col_diff_sign, r_col_same_sign;
    uint8_t matrix_load;
    size_t v_inf_incr_steps;
    double max_ve_g;
    char log_file[256];
    char config_file[256];
    uint8_t log_level;
    char timings_file[256];
    char kadr_file[256];
    char second_points_file[256];
    double rel_t;
    uint8_t steady_flow;
    uint8_t no_log_buf;
};

/* include/unit_1.cuh:20 — build and invert the panel system; returns a
 * malloc'd (birth+1)^2 row-major matrix (zero padded), or NULL.  Also writes
 * L.txt and M.txt into the working directory, as the reference does. */
double *matr_creation(vx_panel *panels, size_t s, size_t birth);

/* include/unit_1.cuh:23 — read M.txt (first line: size P+1) from the working
 * directory; *p receives P.  Returns the padded matrix or NULL. */
double *load_matrix(size_t *p);

/* include/unit_1.cuh:26 — host and device particle arrays of `size`. */
int allocate_arrays(vxu_vortex **p_host, vxu_vortex **p_dev, vxu_velocity **v_host,
                    vxu_velocity **v_dev, double **d_dev, size_t size);

/* include/unit_1.cuh:28 — fill [new_size-increased, new_size) with far-away
 * G = 0 entries. */
int randomize_tail(vxu_vortex **p_dev, size_t new_size, size_t increased);

/* include/unit_1.cuh:30 — grow the arrays by conf.inc_step (or allocate the
 * first conf.inc_step). */
int incr_vort_quant(vxu_vortex **p_host, vxu_vortex **p_dev, vxu_velocity **v_host,
                    vxu_velocity **v_dev, double **d_dev, size_t *size);

/* include/unit_1.cuh:33 — birth of one vortex per panel at pos[n .. n+P). */
int vort_creation(vxu_vortex *pos, double (*V_infDev)[2], size_t n_of_birth,
                  size_t n_of_birth_BLOCK_S, size_t n, double *M_Dev, double *d_g,
                  vx_panel *panels);

/* include/unit_1.cuh:37,39 — event timer on the legacy stream (seconds). */
void start_timer(void **start, void **stop);
float stop_timer(void *start, void *stop);

/* include/unit_1.cuh:42 — convective + diffusive velocity of the s slots. */
int Speed(vxu_vortex *pos, double (*v_inf)[2], size_t s, vxu_velocity *v, double *d, double nu,
          vx_panel *panels);

/* include/unit_1.cuh:45 — convection, absorption, force sums, compaction and
 * both collapse passes; *n is updated. */
int Step(vxu_vortex *pos, vxu_velocity *V, size_t *n, size_t s, double *d_g, vxu_velocity *F_p,
         double *M, vx_panel *panels);

/* include/unit_1.cuh:47 — copy the configuration into the library. */
int init_device_conf_values(void);

/* include/unit_1.cuh:50 — velocity at n_contr control points. */
int velocity_control(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *Contr_points,
                     vxu_velocity *V, size_t n_contr);

/* include/unit_1.cuh:51 — inertial tracers: carrier velocity into v_env,
 * relaxation of v_second towards it with time constant conf.rel_t, then
 * convection with wall absorption.  Writes output/vels/Vel<step>_4.txt and
 * _5.txt as the reference does. */
int second_speed(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *second_pos,
                 vxu_velocity *v_second, vxu_velocity *v_env, size_t *n_second, vx_panel *panels);

/* include/unit_1.cuh:52 — passive tracers moved with the carrier velocity. */
int first_speed(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *second_pos,
                vxu_velocity *v_second, size_t *n_second, vx_panel *panels);

/* Kernels launched by the entry points above since the library was loaded
 * (no counterpart in the reference; used to show which code ran). */
int64_t vxu_launch_count(void);

/* Control points accepted by velocity_control_noalloc in one call. */
#define VXU_NOALLOC_MAX_POINTS 4096

/* velocity_control without any device allocation.  No counterpart in the
 * reference: it is for host programs that cannot call cudaMalloc where they
 * sample the flow (device memory already held by another runtime's caching
 * allocator, or a device-memory budget fixed at start-up).  Its scratch is a
 * fixed 4 MiB array inside this library, held on every GPU that loads it
 * until exit; the caller passes the inputs and outputs as for
 * velocity_control.
 *   - at most VXU_NOALLOC_MAX_POINTS control points, else returns 2 and
 *     launches nothing;
 *   - plain FP64 form (results identical to velocity_control's when
 *     VORTEX_B200_PRECISION is unset); the core radius is velocity_control's:
 *     the one fixed by init_device_conf_values, or conf.ve_size before it;
 *   - each call launches on the legacy default stream and synchronises the
 *     device, like the reference's entry points: do not call it while any
 *     stream on the device is being captured;
 *   - the first call on a device, with that device current, looks up the
 *     array's device address;
 *   - all calls on one device share the array; calls that overlap on the
 *     same GPU race and must be serialised by the caller. */
int velocity_control_noalloc(vxu_vortex *pos, double (*V_inf)[2], size_t n, vxu_vortex *Contr_points,
                             vxu_velocity *V, size_t n_contr);

#ifdef __cplusplus
}
#endif
#endif /* VORTEX_B200_UNIT1_H_ */
