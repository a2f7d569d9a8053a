/*
 * vortex_b200.h — native C ABI of the B200 vortex-element step library
 * (libvortex_b200.so).
 *
 * One handle (vx_sim) owns one body's resident device state: panels, the
 * inverted panel system, structure-of-arrays particle storage and scratch.
 * vx_step() advances it by whole time steps in the reference's per-step order
 * (src/main.c:676-784 of grechkin-pogrebnyakov/vortex): birth, convective
 * velocity with 3-nearest distance, vortex and wall diffusion, convection with
 * wall absorption, force sums, compaction, collapse of opposite-sign then
 * same-sign pairs.  A step never synchronises with the host unless the
 * particle store has to grow.
 *
 * The reference's own entry points (include/unit_1.cuh:15-55) are exported
 * by the same library; they are declared in vortex_b200_unit1.h.
 *
 * All functions return vx_status; VX_OK is 0.  Handles are not thread-safe;
 * different handles may be used from different threads.
 */
#ifndef VORTEX_B200_H_
#define VORTEX_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vx_status {
    VX_OK = 0,
    VX_ERR_CUDA = 1,        /* a CUDA call failed (message in vx_last_error) */
    VX_ERR_ARG = 2,         /* bad argument (reference: return code 2) */
    VX_ERR_IO = 3,          /* file could not be opened or parsed */
    VX_ERR_SINGULAR = 4,    /* panel system pivot below 1e-12 */
    VX_ERR_NOMEM = 5,       /* device or host allocation failed */
    VX_ERR_DEVICE = 6,      /* a kernel reported an internal error flag */
    VX_ERR_BUDGET = 7       /* request exceeds the server's HBM budget */
} vx_status;

enum { VX_PREC_FP64 = 0, VX_PREC_FP32 = 1 };
/* Where a new vortex is placed: the reference's midpoint + 1e-6 n
 * (include/kernel.cuh:109-116), the profile file's birth column, or the
 * panel midpoint + L/2 n. */
enum { VX_BIRTH_REF = 0, VX_BIRTH_FILE = 1, VX_BIRTH_HALF_PANEL = 2 };

/* Panel record; same 120-byte layout as the reference's tPanel
 * (include/definitions.h:82-103). */
typedef struct vx_panel {
    uint32_t n;
    uint32_t pad_;
    double left[2];
    double right[2];
    double contr[2];
    double birth[2];
    double norm[2];
    double tang[2];
    double length;
    uint32_t n_of_lpanel;
    uint32_t n_of_rpanel;
} vx_panel;

/* Run configuration.  The first block holds the reference's .conf keys
 * (src/main.c:77-111, struct conf_t include/definitions.h:105-142); the
 * second block holds keys this library adds.  Unknown keys in a .conf file
 * are ignored, as in the reference. */
typedef struct vx_conf {
    int64_t steps, saving_step, inc_step, n_of_points, n_col, v_inf_incr_steps, tree_depth;
    double dt, viscosity, rho, v_inf_x, v_inf_y;
    double x_max, x_min, y_max, y_min;
    double ve_size, h_col_x, h_col_y, rc_x, rc_y;
    double r_col_diff_sign, r_col_same_sign, max_ve_g, rel_t, theta;
    int32_t matrix_load, steady_flow, log_level, no_log_buf;
    char pr_file[256];
    char timings_file[256];
    char kadr_file[256];
    char second_points_file[256];
    char log_file[256];
    /* ---- additions ---- */
    int32_t precision;          /* VX_PREC_FP64 (plain) or VX_PREC_FP32 (bulk) */
    int32_t birth_offset_mode;  /* VX_BIRTH_* ; default VX_BIRTH_REF */
    double drop_eps;            /* |G| below this is removed; default 1e-12 */
    double diff_cutoff;         /* bulk form: vortex diffusion ignores pairs
                                   with r > diff_cutoff * d_i (default 16:
                                   each such term weighs below e^-16 = 1.1e-7,
                                   together about (c+1) e^-c = 2e-6 of the
                                   sum's magnitude in a uniform cloud, within
                                   the bulk form's per-particle bound) */
    int32_t n_probes_grid;      /* >0: probes on an n x n grid (box below) */
    int32_t pad1_;
    double probe_box[4];        /* x0, x1, y0, y1 of the probe grid */
    int32_t fmm;                /* bulk form: Biot-Savart by the quadtree
                                   multipole method, and the birth
                                   right-hand side with the vortices beyond
                                   1.5 body radii through one local
                                   expansion about the body (default 1);
                                   0 = direct sums */
    int32_t gj_pivot;           /* panel-system inversion: 0 = the reference's
                                   Gauss-Jordan pivot rule (a pivot below
                                   1e-12 fails, as in the reference);
                                   1 = partial pivoting; 2 = the reference's
                                   rule, partial pivoting if it fails;
                                   3 = blocked LU with partial pivoting
                                   (fastest to build, about 20 kernels
                                   per 32 columns) */
    int32_t fmm_leaf;           /* quadtree depth: mean vortices per leaf
                                   the depth aims at (default 32) */
    int32_t fmm_p;              /* expansion terms of the quadtree FMM: 8, 12, 16
                                   or 20 (0: 16) */
} vx_conf;

typedef struct vx_sim vx_sim;

const char *vx_status_str(vx_status s);
/* Last error message of the calling thread (empty string if none). */
const char *vx_last_error(void);

/* Defaults as the reference's main() leaves them (src/main.c:420-422:
 * zeroed struct, log_level 3, v_inf_incr_steps 1) plus the additions'. */
vx_status vx_conf_default(vx_conf *conf);
/* Parse a .conf file ("key value" lines, prefix-matched keys, trailing
 * comments tolerated; src/main.c:48-115) on top of *conf. */
vx_status vx_conf_read(const char *path, vx_conf *conf);
/* Read a profile file (src/main.c:220-256).  With out == NULL only *P is
 * set; otherwise cap must be >= P. */
vx_status vx_profile_read(const char *path, vx_panel *out, int64_t cap, int64_t *P);

/* Create a body on CUDA device `device`: uploads panels, builds and inverts
 * the panel system on the device.  Particle store starts empty. */
vx_status vx_create(const vx_conf *conf, const vx_panel *panels, int64_t P, int device,
                    vx_sim **out);
vx_status vx_destroy(vx_sim *sim);

/* Host <-> device particle state (x, y, G of the first n particles). */
vx_status vx_set_particles(vx_sim *sim, const double *x, const double *y, const double *g,
                           int64_t n);
vx_status vx_get_particles(vx_sim *sim, double *x, double *y, double *g, int64_t cap,
                           int64_t *n);
vx_status vx_get_count(vx_sim *sim, int64_t *n);
/* Velocity and 3-nearest distance from the last velocity evaluation. */
vx_status vx_get_velocity(vx_sim *sim, double *vx, double *vy, double *d, int64_t cap);
/* Absorbed circulation, force (x, y) and moment of the last step
 * (the reference's d_g, F_p, M after summ_Kernel). */
vx_status vx_get_forces(vx_sim *sim, double out4[4]);
vx_status vx_set_vinf(vx_sim *sim, double vx, double vy);
vx_status vx_set_dg(vx_sim *sim, double dg);
/* The inverted (P+1)^2 panel system, row-major. */
vx_status vx_get_matrix(vx_sim *sim, double *minv);
/* Replace the inverted panel system ((P+1)^2 row-major FP64), e.g. one read
 * from a matrix file as the reference's matrix_load does. */
vx_status vx_set_matrix(vx_sim *sim, const double *minv);

/* Advance nsteps whole steps. */
vx_status vx_step(vx_sim *sim, int64_t nsteps);

/* Individual stages, in step order (for tests and custom drivers). */
enum {
    VX_STAGE_BIRTH = 1u << 0,
    VX_STAGE_VELOCITY = 1u << 1,     /* Biot-Savart + 3-nearest distance */
    VX_STAGE_DIFFUSION = 1u << 2,    /* vortex-vortex diffusive velocity */
    VX_STAGE_WALL = 1u << 3,         /* wall diffusive velocity */
    VX_STAGE_ADVECT = 1u << 4,       /* convection, absorption, force sums */
    VX_STAGE_COMPACT = 1u << 5,
    VX_STAGE_COLLAPSE1 = 1u << 6,    /* opposite signs, n_col rounds */
    VX_STAGE_COLLAPSE2 = 1u << 7,    /* same sign, n_col rounds */
    VX_STAGE_ALL = 0xffu
};
vx_status vx_stage(vx_sim *sim, unsigned stage_mask);

/* Velocity at probe points (host arrays), Biot-Savart + V_inf only
 * (src/kernel.cu:1434-1475). */
vx_status vx_probe(vx_sim *sim, const double *px, const double *py, int64_t np,
                   double *vx, double *vy);

/* Binary checkpoint of a body at full precision (no counterpart in the
 * reference, whose restart frames, src/main.c:175-188 and 558-605, keep six
 * decimals and lose d_g, the forces and the V_inf ramp): the vortices, the
 * step index, the current V_inf, d_g, the last forces and the last quadtree
 * build's occupancy record (the next depth follows from it).  A body continued
 * from a checkpoint steps exactly as the one that wrote it.  Loading checks
 * the panel count, the form and a hash of the panels (VX_ERR_ARG on a
 * mismatch or a damaged file). */
vx_status vx_checkpoint_save(vx_sim *sim, const char *path);
vx_status vx_checkpoint_load(vx_sim *sim, const char *path);

/* Tracer points moved one time step with the velocities (u, v): the
 * convection of the tracers in first_speed / second_speed
 * (src/unit_1.cu:1271-1340, the vortices' step kernel without force terms).
 * A point that crosses the wall gets g = 0; one that leaves the window is
 * moved to (-2e5, -2e5) with g = 0.  Host arrays in and out; the body's
 * vortices and force sums are not changed. */
vx_status vx_move_points(vx_sim *sim, double *x, double *y, double *g, const double *u,
                         const double *v, int64_t n);

/* Record every step into a CUDA graph after the first call and replay it
 * (on by default; 0 turns it off). */
vx_status vx_set_graph(vx_sim *sim, int enable);

/* Device time (ms) accumulated per stage since timing was (re)enabled:
 * out[0] birth, [1] convective velocity, [2] vortex diffusion, [3] wall
 * diffusion, [4] convection + compaction + collapse, [5] the Biot-Savart
 * pair kernel alone, [6] the diffusion pair kernel alone, [7] whole steps.
 * Timed steps run eagerly (no graph) so the events can be recorded. */
vx_status vx_set_timing(vx_sim *sim, int enable);
vx_status vx_get_timing(vx_sim *sim, double out8[8]);
/* Pair evaluations executed by the bulk form's near-field (FMM) and
 * neighbour-list diffusion kernels since the last clear (clear != 0 resets). */
vx_status vx_get_pair_counts(vx_sim *sim, double out2[2], int clear);
/* Spatial structures of the last bulk-form velocity / diffusion pass:
 * out[0] quadtree depth, [1] leaf side, [2] targets redone by the exact
 * 3-nearest search, [3] neighbour-grid cell side, [4] cells in x, [5] in y. */
vx_status vx_get_tree_info(vx_sim *sim, double out6[6]);

/* Device bytes a body with P panels will hold when its particle count
 * reaches n_max (capacity growth included): the admission estimate of
 * vx_server.  vx_get_device_bytes: what a handle holds now. */
vx_status vx_estimate_bytes(const vx_conf *conf, int64_t P, int64_t n_max, int device, int64_t *bytes);
vx_status vx_get_device_bytes(vx_sim *sim, int64_t *bytes);

/* Advance `count` bodies of one device by nsteps; every step is launched on
 * all bodies' streams before the next, so their kernels overlap.  Returns
 * without waiting, like vx_step. */
vx_status vx_step_many(vx_sim *const *sims, int count, int64_t nsteps);

/* ---- Serving (no counterpart in the reference, which runs one body per
 * process): a request loop with continuous batching.  Requests (one body
 * each: conf, panels, starting vortices, step count) wait in arrival order
 * until a slot is free and the device-byte budget holds their
 * vx_estimate_bytes at n + P * nsteps; admitted bodies are created on worker
 * threads (state 1 from admission on) and stay resident, each
 * with at most one step in flight on its own stream; a tick launches the
 * next step of every resident body with none in flight, waits until at
 * least one step has finished, collects every finished step and launches
 * that body's next one, and releases the finished bodies.  Results do not
 * depend on what else runs. */
typedef struct vx_server vx_server;
vx_status vx_server_create(int device, int64_t budget_bytes, int max_active, vx_server **out);
vx_status vx_server_destroy(vx_server *srv);
/* Inputs are copied; VX_ERR_BUDGET if the request alone exceeds the budget. */
vx_status vx_server_submit(vx_server *srv, const vx_conf *conf, const vx_panel *panels, int64_t P,
                           const double *x, const double *y, const double *g, int64_t n, int64_t nsteps,
                           int64_t *id);
/* Admit, launch, collect at least one finished step, retire; counts after
 * the tick. */
vx_status vx_server_tick(vx_server *srv, int64_t *active, int64_t *queued);
/* state: 0 queued, 1 resident, 2 done, 3 failed; forces: (dg, Fx, Fy, M)
 * per completed step, at most cap_steps steps copied. */
vx_status vx_server_result(vx_server *srv, int64_t id, int *state, int64_t *steps_done, double *forces,
                           int64_t cap_steps, int64_t *n_final);
/* Why a failed request (state 3) failed: the first error met, as text
 * (empty otherwise), NUL-terminated within cap bytes. */
vx_status vx_server_failure(vx_server *srv, int64_t id, char *buf, int64_t cap);
/* out[0] finished, [1]/[2] p50/p99 body-step device ms, [3]/[4] p50/p99
 * submit-to-finish s, [5] mean resident bodies per tick, [6] body steps,
 * [7] particle steps, [8] bytes reserved now, [9] ticks. */
vx_status vx_server_stats(vx_server *srv, double out10[10]);
/* How the resident bodies are stepped: 1 (default) as the members of one
 * batch (vx_batch: each kernel of the step once for all of them, joining
 * at the step after their creation, leaving after their last step), 0 each
 * on its own stream.  Only while no body is resident. */
vx_status vx_server_set_batched(vx_server *srv, int on);

/* Batched steps (no counterpart in the reference, which runs one body per
 * process; its step loop is src/main.c:652-785).  A batch advances bodies
 * of one device together: each kernel of the step runs once for all of them
 * (its blocks laid out body after body, each block given its body's
 * arguments), and the whole batched step is one CUDA graph, so a step of
 * the batch takes one launch per kernel of the step, not one per body.
 * Each body's results are bit-identical to stepping it alone with vx_step.
 * While a body belongs to a batch it launches on the batch's stream and is
 * stepped only through vx_batch_step (vx_step and vx_stage refuse it); the
 * other calls on the body work and are ordered after the batch's steps.
 * Destroy the batch before any of its bodies. */
typedef struct vx_batch vx_batch;
vx_status vx_batch_create(vx_sim *const *sims, int count, vx_batch **out);
/* An empty batch on `device`; members join with vx_batch_add. */
vx_status vx_batch_new(int device, vx_batch **out);
/* Membership changes between batched steps: a body joins at the next step
 * (after the work already queued on its own stream), or leaves after the
 * steps already launched and returns to its own stream.  No host wait. */
vx_status vx_batch_add(vx_batch *batch, vx_sim *sim);
vx_status vx_batch_remove(vx_batch *batch, vx_sim *sim);
/* Wait for the last batched step; for each body that took part in it (in
 * the batch's order at that step, *count of them, at most cap written):
 * the body and 5 values, its vortex count, d_g, Fx, Fy and M after the
 * step (gathered on the device and copied back once per step). */
vx_status vx_batch_last_results(vx_batch *batch, vx_sim **members, double *out5, int cap, int *count);
/* The same for batched step `step` (0-based among the batch's steps; the
 * last two launched are kept, so a caller can launch the next step before
 * collecting the previous one). */
vx_status vx_batch_results(vx_batch *batch, int64_t step, vx_sim **members, double *out5, int cap, int *count);
/* Asynchronous like vx_step; bodies grow their stores as needed. */
vx_status vx_batch_step(vx_batch *batch, int64_t nsteps);
/* Wait for the batch's steps; reports the bodies' device error flags. */
vx_status vx_batch_sync(vx_batch *batch);
/* out[0] batched steps, [1] kernels they launched, [2] kernels per batched
 * step now, [3] slot-table rebuilds, [4] graph instantiations, [5] bodies. */
vx_status vx_batch_info(vx_batch *batch, double out6[6]);
/* Host time spent preparing the batched steps so far: out[0] / [1] the
 * longest / total capacity growth, [2] / [3] the longest / total
 * re-recording, merge and upload of the slot tables, [4..7] the longest
 * re-recording, merge + layout, upload and graph build (ms). */
vx_status vx_batch_host_times(vx_batch *batch, double out8[8]);
/* The CUDA stream (cudaStream_t) the batch launches on. */
void *vx_batch_stream(vx_batch *batch);
/* Ends the batch (waits for its steps); the bodies return to their own
 * streams and can be stepped alone again. */
vx_status vx_batch_destroy(vx_batch *batch);

/* Switch the bulk form's far field (fmm: 1 quadtree FMM and birth far
 * field, 0 direct sums) and the quadtree's target vortices per leaf at run
 * time (the autotuner's knobs); the step graph is re-captured. */
vx_status vx_set_fmm(vx_sim *sim, int fmm, int leaf);

/* Validation hook (no counterpart in the reference): the FP32 atan2 the
 * bulk form's birth terms use, evaluated on device arrays of n floats. */
vx_status vx_eval_bulk_atan2(const float *y, const float *x, float *out, int64_t n);

/* Validation hook (no counterpart in the reference): the order the particle
 * grids use, for n keys below nb (device arrays): element indices by key,
 * equal keys in index order (a stable sort by key), written to `order`.
 * Allocates its own scratch. */
vx_status vx_eval_bucket_order(const unsigned *key, int64_t n, int64_t nb, int *order);

/* Number of kernels this handle has launched since creation. */
vx_status vx_get_launch_count(vx_sim *sim, int64_t *count);

/* Instrumentation (no counterpart in the reference): run nsteps steps
 * stage by stage with an event pair around every kernel launch and report
 * each kernel's total device time and launches.  names receives the
 * kernels' names, '\n'-separated (names_cap bytes, NUL-terminated); ms[k] and
 * counts[k] belong to the k-th name; *nkernels is the number of distinct
 * kernels (at most cap are written).  The events keep consecutive kernels
 * from overlapping and add about a microsecond to each time. */
vx_status vx_kernel_times(vx_sim *sim, int64_t nsteps, char *names, int64_t names_cap, double *ms,
                          int64_t *counts, int64_t cap, int64_t *nkernels);

/* Block until the handle's device work is done; reports device error flags. */
vx_status vx_sync(vx_sim *sim);
/* Expansion terms of the bulk form's quadtree FMM (8, 12, 16 or 20; the
 * autotuner's third knob); the step graph is re-captured. */
vx_status vx_set_fmm_order(vx_sim *sim, int p);
/* The CUDA stream (cudaStream_t) the handle launches on. */
void *vx_get_stream(vx_sim *sim);

/* Slot-level access for drivers that manage the padded store themselves:
 * raw slots [0, count), dead tail included; vx_set_slots also sets the live
 * count n (the last P live slots count as this step's newborns). */
vx_status vx_get_slots(vx_sim *sim, double *x, double *y, double *g, int64_t count);
vx_status vx_set_slots(vx_sim *sim, const double *x, const double *y, const double *g,
                       int64_t count, int64_t n);
/* Overwrite velocity / 3-nearest distance of the first n particles (any
 * pointer may be NULL). */
vx_status vx_set_velocity(vx_sim *sim, const double *vx, const double *vy, const double *d,
                          int64_t n);
/* Scalars: n, n before this step's birth, step index, V_inf x/y, d_g, Fx, Fy, M. */
vx_status vx_get_state(vx_sim *sim, double out9[9]);
/* Absolute step index (a restart from KadrNNNNNN.txt sets it). */
vx_status vx_set_step_index(vx_sim *sim, int64_t step);

/* Measured throughput of `device`, the roofline denominators of the pair
 * kernels: mode 0 FP32 FMA, 1 FP64 FMA, 2 packed FP32 pairs (TFLOP/s);
 * 3 rsqrt + ex2 units on the special-function pipe (1e12 units/s). */
vx_status vx_measure_peak(int device, int fp64, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* VORTEX_B200_H_ */
