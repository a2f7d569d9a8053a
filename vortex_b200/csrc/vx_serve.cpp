// vx_serve.cpp — continuous-batching request loop over resident bodies.
//
// A request is one simulation (conf, panels, starting vortices, number of
// steps).  Requests wait in arrival order until a slot is free and the
// device-byte budget holds their estimate (vx_estimate_bytes at the largest
// particle count the run can reach: start + P per step); then the body is
// created (on worker threads: building a body's panel system takes tens of
// milliseconds, during which the loop keeps stepping the resident bodies)
// and stays resident until its last step.  Finished bodies are released at
// once, which frees their slot and budget for the next arrivals.
//
// Two ways to step the resident bodies:
//  * batched (default): the resident bodies are the members of one vx_batch,
//    so each batched step runs every kernel of the step once for all of them
//    (one CUDA graph).  Bodies join the batch at the step after their
//    creation and leave it after their last step, so requests that arrive
//    while others run are batched with them step by step (iteration-level
//    continuous batching).  The next batched step is launched before the
//    previous one is collected (its results come back in one copy), so the
//    device does not wait for the host between steps.
//  * per-body streams: each body has at most one step in flight on its own
//    stream; a tick launches the next step of every resident body that has
//    none in flight, waits until at least one has finished, collects every
//    finished step and launches that body's next one at once.
// Either way each body runs in its own handle with deterministic kernels, so
// its results do not depend on what else runs (bit-identical alone and in
// the mix).
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
#include <unordered_map>
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
    std::string err;               // why the request failed (state 3)
    int64_t done_steps = 0;
    int64_t launched = 0;     // steps launched (batched form)
    bool in_batch = false;
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
    // batched form
    bool batched = true;
    vx_batch *batch = nullptr;
    struct Flight {
        int64_t step;                     // the batch's step index
        std::vector<Request *> members;
        cudaEvent_t e0, e1;
    };
    std::deque<Flight> flight;
    std::vector<cudaEvent_t> ev_pool;
    int64_t batch_steps = 0;
};

// Launch the next step of resident body r on its stream, between its events.
// A request fails: state 3, with the first reason kept.
static void fail(Request *r, const std::string &why) {
    r->state = 3;
    if (r->err.empty()) r->err = why;
}

static void launch_step(vx_server *S, Request *r) {
    cudaStream_t st = (cudaStream_t)vx_get_stream(r->sim);
    cudaEventRecord(r->e0, st);
    if (vx_step(r->sim, 1) != VX_OK) {
        fail(r, std::string("step: ") + vx_last_error());
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
        fail(r, std::string("state: ") + vx_last_error());
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
    if (r->in_batch && S->batch && r->sim) vx_batch_remove(S->batch, r->sim);
    r->in_batch = false;
    if (r->sim) vx_destroy(r->sim);   // waits for the steps it took part in
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
    if (S->batch) vx_batch_destroy(S->batch);
    for (auto &f : S->flight) {
        cudaEventDestroy(f.e0);
        cudaEventDestroy(f.e1);
    }
    for (cudaEvent_t e : S->ev_pool) cudaEventDestroy(e);
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
            fail(r, "creation: " + (r->create_err.empty() ? std::string(vx_status_str(r->create_st)) : r->create_err));
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

// Admission in arrival order (slots and budget are held from here on); the
// admitted bodies are created on the worker threads.
static void admit(vx_server *S) {
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
}

static bool created_waiting(vx_server *S) {
    if (S->creating == 0) return false;
    std::lock_guard<std::mutex> lk(S->mu);
    return !S->created.empty();
}

// Release every body that is no longer resident (done or failed).
static void retire(vx_server *S) {
    std::vector<Request *> keep;
    for (Request *r : S->active) {
        if (r->state == 1) {
            keep.push_back(r);
            continue;
        }
        if (r->inflight) cudaEventSynchronize(r->e1);   // nothing of it may run on after release
        r->t_finish = now_s();
        if (r->state == 2) S->ttc_s.push_back(r->t_finish - r->t_submit);
        release(S, r);
    }
    S->active.swap(keep);
}

// Per-body streams: launch the next step of every resident body with none
// in flight, wait until some step has finished (whichever comes first: a
// small body's step is not held back by a large one's), collect every
// finished step and launch that body's next one at once.
static void tick_streams(vx_server *S) {
    for (Request *r : S->active)
        if (r->state == 1 && !r->inflight) launch_step(S, r);
    for (;;) {
        bool pending = S->creating > 0, any = created_waiting(S);
        for (Request *r : S->active) {
            if (!r->inflight) continue;
            pending = true;
            if (cudaEventQuery(r->e1) != cudaErrorNotReady) any = true;
        }
        if (any || !pending) break;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    for (Request *r : S->active) {
        if (r->inflight && r->state == 1) {
            const cudaError_t q = cudaEventQuery(r->e1);
            if (q == cudaSuccess) {
                collect_step(S, r);
                if (r->state == 1) launch_step(S, r);
            } else if (q != cudaErrorNotReady) {
                r->inflight = false;
                fail(r, std::string("step event: ") + cudaGetErrorString(q));
            }
        }
    }
    retire(S);
    take_created(S);
    for (Request *r : S->active)
        if (r->state == 1 && !r->inflight) launch_step(S, r);
}

static cudaEvent_t pool_event(vx_server *S) {
    cudaEvent_t e = nullptr;
    if (!S->ev_pool.empty()) {
        e = S->ev_pool.back();
        S->ev_pool.pop_back();
    } else {
        cudaEventCreate(&e);
    }
    return e;
}

// Collect the oldest batched step in flight: per member its count and
// force sums (one copy for all), its step time, completion.
static void collect_flight(vx_server *S) {
    vx_server::Flight f = S->flight.front();
    S->flight.pop_front();
    cudaEventSynchronize(f.e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, f.e0, f.e1);
    S->ev_pool.push_back(f.e0);
    S->ev_pool.push_back(f.e1);
    const size_t room = f.members.size() + S->active.size();   // at least the batch's members at that step
    std::vector<vx_sim *> mem(room);
    std::vector<double> out(5 * room);
    int cnt = 0;
    const vx_status st = vx_batch_results(S->batch, f.step, mem.data(), out.data(), (int)mem.size(), &cnt);
    // the batch lists its members in its own order: match them by body
    std::unordered_map<const vx_sim *, int> at;
    for (int j = 0; st == VX_OK && j < cnt; ++j) at[mem[j]] = j;
    for (Request *r : f.members) {
        if (r->state != 1) continue;
        const auto it = at.find(r->sim);
        if (it == at.end()) {
            fail(r, st != VX_OK ? std::string("batch results: ") + vx_last_error()
                                : std::string("batch results: body not among the step's members"));
            continue;
        }
        const double *o = out.data() + 5 * it->second;
        S->step_ms.push_back(ms);
        S->body_steps += 1;
        S->particle_steps += o[0];
        r->forces.insert(r->forces.end(), o + 1, o + 5);
        r->done_steps += 1;
        if (r->done_steps == r->steps) {
            r->n_final = (int64_t)o[0];
            r->state = 2;
        }
    }
}

// Batched: new bodies join the batch, bodies that have launched all their
// steps leave it, the next batched step is launched (at most two in flight),
// then the oldest step in flight is collected once it has finished (or a
// created body is waiting to join).
static vx_status tick_batched(vx_server *S) {
    if (!S->batch) {
        const vx_status st = vx_batch_new(S->device, &S->batch);
        if (st != VX_OK) return st;
    }
    // keep two batched steps in flight: the host collects one while the
    // device runs the next
    while (S->flight.size() < 2) {
        for (Request *r : S->active) {
            if (r->state == 1 && !r->in_batch && r->launched < r->steps) {
                if (vx_batch_add(S->batch, r->sim) != VX_OK) {
                    fail(r, std::string("batch add: ") + vx_last_error());
                    continue;
                }
                r->in_batch = true;
            }
            if (r->in_batch && (r->launched >= r->steps || r->state != 1)) {
                vx_batch_remove(S->batch, r->sim);   // after the steps in flight
                r->in_batch = false;
            }
        }
        vx_server::Flight f;
        for (Request *r : S->active)
            if (r->in_batch) f.members.push_back(r);
        if (f.members.empty()) break;
        cudaStream_t st = (cudaStream_t)vx_batch_stream(S->batch);
        f.e0 = pool_event(S);
        f.e1 = pool_event(S);
        cudaEventRecord(f.e0, st);
        double info[6];
        vx_batch_info(S->batch, info);
        f.step = (int64_t)info[0];
        if (vx_batch_step(S->batch, 1) != VX_OK) {
            const std::string why = std::string("batch step: ") + vx_last_error();
            for (Request *r : f.members) fail(r, why);
            S->ev_pool.push_back(f.e0);
            S->ev_pool.push_back(f.e1);
            break;
        }
        cudaEventRecord(f.e1, st);
        for (Request *r : f.members) r->launched += 1;
        S->flight.push_back(f);
        S->batch_steps += 1;
    }
    // collect the oldest step once it has finished; with fewer than two in
    // flight and a body waiting to join, do not wait for it
    while (!S->flight.empty()) {
        const bool full = S->flight.size() >= 2;
        if (cudaEventQuery(S->flight.front().e1) == cudaSuccess || full) {
            collect_flight(S);
            break;
        }
        if (created_waiting(S)) break;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    if (S->flight.empty() && S->active.empty() && S->creating > 0) {
        // nothing to step: wait for a body to be created
        while (!created_waiting(S)) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    // a body leaves before its release; its last step has been collected
    for (Request *r : S->active)
        if (r->state != 1 && r->in_batch) {
            vx_batch_remove(S->batch, r->sim);
            r->in_batch = false;
        }
    bool referenced = false;
    std::vector<Request *> keep;
    for (Request *r : S->active) {
        referenced = false;
        for (const auto &fl : S->flight)
            for (Request *q : fl.members) referenced |= (q == r);
        if (r->state == 1 || referenced) {
            keep.push_back(r);
            continue;
        }
        r->t_finish = now_s();
        if (r->state == 2) S->ttc_s.push_back(r->t_finish - r->t_submit);
        release(S, r);
    }
    S->active.swap(keep);
    take_created(S);
    return VX_OK;
}

// Admit what fits, step the resident bodies (batched or per-body streams, as
// above), retire the finished ones.  *active: bodies resident after the
// tick; *queued: waiting.
extern "C" vx_status vx_server_tick(vx_server *S, int64_t *active, int64_t *queued) {
    if (!S) return VX_ERR_ARG;
    if (cudaSetDevice(S->device) != cudaSuccess) return VX_ERR_CUDA;
    admit(S);
    take_created(S);
    if (S->batched) {
        const vx_status st = tick_batched(S);
        if (st != VX_OK) return st;
    } else {
        tick_streams(S);
    }
    S->ticks += 1;
    S->active_sum += (double)S->active.size();
    if (active) *active = (int64_t)S->active.size() + S->creating;
    if (queued) *queued = (int64_t)S->queue.size();
    return VX_OK;
}

// 1: batched steps (default); 0: per-body streams.  Only while nothing is
// resident.
extern "C" vx_status vx_server_set_batched(vx_server *S, int on) {
    if (!S) return VX_ERR_ARG;
    if (!S->active.empty() || S->creating > 0) {
        vx_set_error("vx_server_set_batched: bodies are resident");
        return VX_ERR_ARG;
    }
    S->batched = on != 0;
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

// Why request `id` failed ("" unless its state is 3), NUL-terminated in buf.
extern "C" vx_status vx_server_failure(vx_server *S, int64_t id, char *buf, int64_t cap) {
    if (!S || !buf || cap < 1) return VX_ERR_ARG;
    auto it = S->all.find(id);
    if (it == S->all.end()) return VX_ERR_ARG;
    const std::string &e = it->second->err;
    const size_t k = std::min<size_t>(e.size(), (size_t)(cap - 1));
    std::memcpy(buf, e.data(), k);
    buf[k] = 0;
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
