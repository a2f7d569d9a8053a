// vx_serve.cpp — continuous-batching request loop over resident bodies.
//
// A request is one simulation (conf, panels, starting vortices, number of
// steps).  Requests wait in arrival order until a slot is free and the
// device-byte budget holds their estimate (vx_estimate_bytes at the largest
// particle count the run can reach: start + P per step); then the body is
// created (on worker threads: building a body's panel system takes tens of
// milliseconds, during which the loop keeps relaunching the resident bodies)
// and stays resident until its last step.  Each body has at most one
// step in flight on its own stream; a tick launches the next step of every
// resident body that has none in flight, waits until at least one step has
// finished, collects every finished step (forces, count) and launches that
// body's next step at once.  So no body waits for the slowest one: bodies of
// different sizes overlap on the device and a small body takes many steps
// while a large one takes one.  Finished bodies are released at once, which
// frees their slot and budget for the next arrivals.  Each body runs in its
// own handle with deterministic kernels, so its results do not depend on what
// else runs.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <condition_variable>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/vortex_b200.h"

void vx_set_error(const char *fmt, ...);

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    vx_conf conf;
    std::vector<vx_panel> pan;
    std::vector<double> x, y, g;
    int64_t steps = 0;
    int64_t est_bytes = 0;
    int state = 0;            // 0 queued, 1 resident, 2 done, 3 failed
    vx_sim *sim = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool inflight = false;    // a step launched and not yet collected
    vx_status create_st = VX_OK;   // set by the worker thread
    std::string create_err;        // the worker's error text when create_st != VX_OK
    int64_t done_steps = 0;
    std::vector<double> forces;   // 4 per step: dg, Fx, Fy, M
    int64_t n_final = 0;
    double t_submit = 0, t_admit = 0, t_finish = 0;
};

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)std::floor(pos), hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (pos - (double)lo) * (v[hi] - v[lo]);
}

}  // namespace

struct vx_server {
    int device = 0;
    int64_t budget = 0, used = 0;
    int max_active = 1;
    int64_t next_id = 1;
    std::deque<Request *> queue;
    std::vector<Request *> active;
    // body creation on worker threads: admitted requests go to to_create,
    // come back in created; `creating` (loop thread only) counts those away
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request *> to_create;
    std::vector<Request *> created;
    bool stop = false;
    int creating = 0;
    std::map<int64_t, Request *> all;
    std::vector<double> step_ms;      // device time of every body step
    std::vector<double> ttc_s;        // submit -> finish of every finished request
    double active_sum = 0.0;
    int64_t ticks = 0, body_steps = 0;
    double particle_steps = 0.0;      // sum over body steps of the particle count
};

// Launch the next step of resident body r on its stream, between its events.
static void launch_step(vx_server *S, Request *r) {
    cudaStream_t st = (cudaStream_t)vx_get_stream(r->sim);
    cudaEventRecord(r->e0, st);
    if (vx_step(r->sim, 1) != VX_OK) {
        r->state = 3;
        return;
    }
    cudaEventRecord(r->e1, st);
    r->inflight = true;
}

// Collect r's finished step: its device time, forces and count.
static void collect_step(vx_server *S, Request *r) {
    r->inflight = false;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->e0, r->e1);
    double st9[9];
    if (vx_get_state(r->sim, st9) != VX_OK) {
        r->state = 3;
        return;
    }
    const int64_t n = (int64_t)st9[0];
    S->step_ms.push_back(ms);
    S->body_steps += 1;
    S->particle_steps += (double)n;
    r->forces.insert(r->forces.end(), st9 + 5, st9 + 9);
    r->done_steps += 1;
    if (r->done_steps == r->steps) {
        r->n_final = n;
        r->state = 2;
    }
}

static vx_status release(vx_server *S, Request *r) {
    if (r->sim) vx_destroy(r->sim);
    r->sim = nullptr;
    if (r->e0) cudaEventDestroy(r->e0);
    if (r->e1) cudaEventDestroy(r->e1);
    r->e0 = r->e1 = nullptr;
    S->used -= r->est_bytes;
    return VX_OK;
}

extern "C" vx_status vx_server_create(int device, int64_t budget_bytes, int max_active, vx_server **out) {
    if (!out || budget_bytes <= 0 || max_active < 1) return VX_ERR_ARG;
    vx_server *S = new vx_server;
    S->device = device;
    S->budget = budget_bytes;
    S->max_active = max_active;
    *out = S;
    return VX_OK;
}

constexpr int CREATE_THREADS = 4;

// Worker thread: create admitted bodies, taken in admission order.
static void create_loop(vx_server *S) {
    cudaSetDevice(S->device);
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv.wait(lk, [S] { return S->stop || !S->to_create.empty(); });
            if (S->to_create.empty()) return;   // stop, nothing left
            r = S->to_create.front();
            S->to_create.pop_front();
        }
        vx_status st = vx_create(&r->conf, r->pan.data(), (int64_t)r->pan.size(), S->device, &r->sim);
        if (st == VX_OK && !r->x.empty())
            st = vx_set_particles(r->sim, r->x.data(), r->y.data(), r->g.data(), (int64_t)r->x.size());
        if (st == VX_OK && (cudaEventCreate(&r->e0) != cudaSuccess || cudaEventCreate(&r->e1) != cudaSuccess))
            st = VX_ERR_CUDA;
        if (st == VX_OK && r->sim && vx_sync(r->sim) != VX_OK) st = VX_ERR_CUDA;
        r->create_st = st;
        // the error text is thread-local: keep the worker's for the loop thread
        if (st != VX_OK) r->create_err = vx_last_error();
        std::lock_guard<std::mutex> lk(S->mu);
        S->created.push_back(r);
    }
}

static void stop_worker(vx_server *S) {
    if (S->workers.empty()) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        for (Request *r : S->to_create) r->create_st = VX_ERR_ARG;   // never created
        for (Request *r : S->to_create) S->created.push_back(r);
        S->to_create.clear();
    }
    S->cv.notify_all();
    for (auto &t : S->workers) t.join();
    S->workers.clear();
}

extern "C" vx_status vx_server_destroy(vx_server *S) {
    if (!S) return VX_OK;
    cudaSetDevice(S->device);
    stop_worker(S);
    for (auto &kv : S->all) {
        if (kv.second->state == 1) release(S, kv.second);
        delete kv.second;
    }
    delete S;
    return VX_OK;
}

// Queue a request; inputs are copied.  VX_ERR_BUDGET if the request alone
// can never fit the budget.
extern "C" vx_status vx_server_submit(vx_server *S, const vx_conf *conf, const vx_panel *pan, int64_t P,
                                      const double *x, const double *y, const double *g, int64_t n,
                                      int64_t nsteps, int64_t *id) {
    if (!S || !conf || !pan || P < 2 || n < 0 || nsteps < 1 || !id || (n > 0 && (!x || !y || !g)))
        return VX_ERR_ARG;
    Request *r = new Request;
    r->conf = *conf;
    r->pan.assign(pan, pan + P);
    r->x.assign(x, x + n);
    r->y.assign(y, y + n);
    r->g.assign(g, g + n);
    r->steps = nsteps;
    vx_status st = vx_estimate_bytes(conf, P, n + P * nsteps, S->device, &r->est_bytes);
    if (st != VX_OK) { delete r; return st; }
    if (r->est_bytes > S->budget) {
        vx_set_error("request needs about %lld device bytes, budget %lld", (long long)r->est_bytes,
                     (long long)S->budget);
        delete r;
        return VX_ERR_BUDGET;
    }
    r->id = S->next_id++;
    r->t_submit = now_s();
    S->queue.push_back(r);
    S->all[r->id] = r;
    *id = r->id;
    return VX_OK;
}

// Bodies the worker has finished creating join the resident set (or fail).
static void take_created(vx_server *S) {
    std::vector<Request *> got;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        got.swap(S->created);
    }
    for (Request *r : got) {
        --S->creating;
        if (r->create_st != VX_OK) {
            // the caller of the tick reads the reason through vx_last_error
            vx_set_error("request %lld: body creation failed: %s", (long long)r->id,
                         r->create_err.empty() ? vx_status_str(r->create_st) : r->create_err.c_str());
            release(S, r);
            r->state = 3;
            r->t_finish = now_s();
            continue;
        }
        std::vector<double>().swap(r->x);
        std::vector<double>().swap(r->y);
        std::vector<double>().swap(r->g);
        r->forces.reserve((size_t)(4 * r->steps));
        r->t_admit = now_s();
        S->active.push_back(r);
    }
}

// Admit what fits, launch and collect steps as above, retire the
// finished ones.  *active: bodies resident after the tick; *queued: waiting.
extern "C" vx_status vx_server_tick(vx_server *S, int64_t *active, int64_t *queued) {
    if (!S) return VX_ERR_ARG;
    if (cudaSetDevice(S->device) != cudaSuccess) return VX_ERR_CUDA;
    // admission in arrival order (slots and budget are held from here on)
    while (!S->queue.empty() && (int)S->active.size() + S->creating < S->max_active &&
           S->used + S->queue.front()->est_bytes <= S->budget) {
        Request *r = S->queue.front();
        S->queue.pop_front();
        S->used += r->est_bytes;
        r->state = 1;
        ++S->creating;
        if ((int)S->workers.size() < std::min(CREATE_THREADS, S->creating)) S->workers.emplace_back(create_loop, S);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->to_create.push_back(r);
        }
        S->cv.notify_one();
    }
    take_created(S);
    // the next step of every resident body with none in flight
    for (Request *r : S->active)
        if (r->state == 1 && !r->inflight) launch_step(S, r);
    // wait until some step in flight has finished (whichever comes first:
    // a small body's step is not held back by a large one's)
    for (;;) {
        bool pending = S->creating > 0, any = false;
        if (pending) {
            std::lock_guard<std::mutex> lk(S->mu);
            any = !S->created.empty();
        }
        for (Request *r : S->active) {
            if (!r->inflight) continue;
            pending = true;
            if (cudaEventQuery(r->e1) != cudaErrorNotReady) any = true;
        }
        if (any || !pending) break;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    // collect every finished step; launch that body's next one at once
    std::vector<Request *> keep;
    for (Request *r : S->active) {
        if (r->inflight && r->state == 1) {
            const cudaError_t q = cudaEventQuery(r->e1);
            if (q == cudaSuccess) {
                collect_step(S, r);
                if (r->state == 1) launch_step(S, r);
            } else if (q != cudaErrorNotReady) {
                r->inflight = false;
                r->state = 3;
            }
        }
        if (r->state == 1) {
            keep.push_back(r);
        } else {
            if (r->inflight) cudaEventSynchronize(r->e1);   // nothing of it may run on after release
            r->t_finish = now_s();
            if (r->state == 2) S->ttc_s.push_back(r->t_finish - r->t_submit);
            release(S, r);
        }
    }
    S->active.swap(keep);
    take_created(S);
    for (Request *r : S->active)
        if (r->state == 1 && !r->inflight) launch_step(S, r);
    S->ticks += 1;
    S->active_sum += (double)S->active.size();
    if (active) *active = (int64_t)S->active.size() + S->creating;
    if (queued) *queued = (int64_t)S->queue.size();
    return VX_OK;
}

// state: 0 queued, 1 resident, 2 done, 3 failed; forces: 4 per completed
// step (dg, Fx, Fy, M), at most cap_steps steps copied; *steps_done.
extern "C" vx_status vx_server_result(vx_server *S, int64_t id, int *state, int64_t *steps_done,
                                      double *forces, int64_t cap_steps, int64_t *n_final) {
    if (!S) return VX_ERR_ARG;
    auto it = S->all.find(id);
    if (it == S->all.end()) return VX_ERR_ARG;
    const Request *r = it->second;
    if (state) *state = r->state;
    if (steps_done) *steps_done = r->done_steps;
    if (forces && cap_steps > 0) {
        const int64_t k = std::min<int64_t>(cap_steps, r->done_steps);
        std::memcpy(forces, r->forces.data(), sizeof(double) * 4 * (size_t)k);
    }
    if (n_final) *n_final = r->n_final;
    return VX_OK;
}

// out[0] finished requests, [1] p50 / [2] p99 body-step device time (ms),
// [3] p50 / [4] p99 submit-to-finish time (s), [5] mean resident bodies per
// tick, [6] body steps, [7] sum of particle counts over body steps,
// [8] device bytes reserved now, [9] ticks.
extern "C" vx_status vx_server_stats(vx_server *S, double out[10]) {
    if (!S || !out) return VX_ERR_ARG;
    out[0] = (double)S->ttc_s.size();
    out[1] = percentile(S->step_ms, 0.50);
    out[2] = percentile(S->step_ms, 0.99);
    out[3] = percentile(S->ttc_s, 0.50);
    out[4] = percentile(S->ttc_s, 0.99);
    out[5] = S->ticks ? S->active_sum / (double)S->ticks : 0.0;
    out[6] = (double)S->body_steps;
    out[7] = S->particle_steps;
    out[8] = (double)S->used;
    out[9] = (double)S->ticks;
    return VX_OK;
}
