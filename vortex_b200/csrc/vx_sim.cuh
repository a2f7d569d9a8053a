// vx_sim.cuh — the body handle (vx_sim) and the engine functions the batch
// (vx_batch.cu) shares with the single-body path (vx_engine.cu).
#pragma once

#include "vx_internal.cuh"

struct vx_sim {
    vx_conf conf;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    int P = 0, P32 = 0;
    VxParams prm;
    vx_panel *d_pan = nullptr;
    double *d_minv = nullptr;
    double *d_minvT = nullptr;   // transposed copy read by the birth solve
    int *d_wstart = nullptr, *d_widx = nullptr;   // wall panel lists per wall cell
    int *d_hstart = nullptr, *d_hidx = nullptr;   // hitting-test panel lists per cell
    long long wall_bytes = 0;
    VxScalars *d_S = nullptr;
    VxScalars *h_S = nullptr;     // pinned mirror
    long long cap = 0;
    double *x = nullptr, *y = nullptr, *g = nullptr, *vx = nullptr, *vy = nullptr, *d = nullptr;
    VxWork w;
    std::vector<void *> work_allocs;
    long long n_upper = 0;
    long long launches = 0;
    // step graphs: a few instantiated shapes, least recently used evicted
    // (the source count moves a shape key back and forth across a power of
    // two; capacity growth drops them all)
    bool use_graph = true;
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        int rhs = -1, sms = -1;
        long long launches = 0, used = 0;
    };
    StepGraph graphs[4];
    long long graph_clock = 0;
    // timing
    bool timing = false;
    cudaEvent_t ev[6] = {};     // stage boundaries
    cudaEvent_t pev[4] = {};    // around the two pair kernels
    double t_acc[8] = {};
    // probe scratch
    double *d_probe = nullptr;
    long long probe_cap = 0;
    // moved-point scratch (vx_move_points): x, y, g, u, v; own scalars and
    // block partials, so the body's force sums stay as they are
    double *d_pts = nullptr;
    long long pts_cap = 0;
    VxScalars *d_St = nullptr;
    double *d_pred = nullptr;
    // member of a batch (vx_batch_create): the handle launches on the
    // batch's stream meanwhile (own_stream kept), and steps only through it
    bool in_batch = false;
    cudaStream_t own_stream = nullptr;
    // per-kernel timing of eagerly launched steps (vx_kernel_times)
    VxKernelTimer *kt = nullptr;
};


// Engine internals (vx_engine.cu).
VxLaunch vx_sim_launch(vx_sim *s);
long long vx_sim_need(vx_sim *s, long long n);     // slots a step starting with n vortices needs
vx_status vx_sim_grow(vx_sim *s, long long need);
long long vx_sim_grow_bytes(vx_sim *s, long long need);   // device bytes the store and scratch of that growth take
vx_status vx_sim_read_scalars(vx_sim *s);
int vx_sim_step_sms(vx_sim *s);
int vx_sim_rhs_chunks(vx_sim *s);
// Launch (or, with rec, record) the stages of one step; share > 0: the SMs
// the scaled grid-stride launches are sized for (at most the body's own).
cudaError_t vx_sim_launch_stages(vx_sim *s, unsigned mask, bool whole_step, VxRecorder *rec, int share);
