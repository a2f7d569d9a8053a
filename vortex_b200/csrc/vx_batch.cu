// vx_batch.cu — many bodies advanced together: every kernel of the step runs
// once for all bodies (k_many over the bodies' argument packs), and the whole
// batched step is one CUDA graph.
//
// Each body's step is recorded, not launched: the same stage launchers the
// single-body path runs (vx_sim_launch_stages) append (kernel, grid, block,
// argument pack) to the body's recording.  The recordings are merged into one
// sequence of slots, each one kernel with the bodies that run it at that
// point: a greedy merge that keeps every body's own order (bodies whose
// quadtrees have more levels run their extra level kernels in slots of their
// own).  A slot's bodies share one launch: its blocks are the bodies' own
// grids laid end to end, and k_many gives each block its body's arguments
// and block coordinates, so a body computes exactly what its own launches
// would have computed.  The grids of the scaled grid-stride launches are
// sized for a share of the GPU proportional to the body's capacity; the
// partitions that fix summation orders follow the body's own count on the
// device (vx_body_parts and the like), so results are bit-identical to
// vx_step's.
//
// The slot tables (block ranges and packs) live in one device arena that the
// graph's kernels read; when a body's recording changes (its store grew, a
// launch shape followed its size across a power of two) the arena is
// rewritten by a stream-ordered copy and the graph is re-instantiated only if
// the slot sequence or a grid bound changed.  Capacity: the host keeps an
// upper bound of each body's count (births add P per step) and, when a body
// may outgrow its store, tightens it with the counts of the step before the
// one in flight (copied back after every step), so the pipeline is not
// drained for it; growth is stream-ordered after the steps in flight.
//
// Reference: the step loop this batches is src/main.c:652-785 with Speed /
// Step / vort_creation (src/unit_1.cu:963-1218); the reference runs one body
// per process.
#include <algorithm>
#include <chrono>
#include <map>
#include <string>
#include <vector>

#include "vx_sim.cuh"

#define BCU(call)                                                                           \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            vx_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? VX_ERR_NOMEM : VX_ERR_CUDA;            \
        }                                                                                   \
    } while (0)

namespace {

// What a body's recording depends on besides its (unchanging) parameters.
struct BodyKey {
    long long cap;
    int rhs, sms, share, fmm, leaf, lmax;
    bool operator==(const BodyKey &o) const {
        return cap == o.cap && rhs == o.rhs && sms == o.sms && share == o.share && fmm == o.fmm &&
               leaf == o.leaf && lmax == o.lmax;
    }
};

struct Body {
    vx_sim *s = nullptr;
    VxRecorder rec;
    BodyKey key{};
    bool recorded = false;
};

struct Slot {
    const void *key = nullptr;    // the single-body kernel (identity)
    const void *many = nullptr;   // its multi-body kernel
    dim3 block;
    size_t smem = 0;
    std::vector<int> bodies;      // batch indices
    std::vector<int> launch;      // index of the launch in each body's recording
    long long total = 0;          // blocks of all bodies
    size_t pack = 0;              // bytes of one argument pack
};

// What the instantiated graph holds for a slot.
struct SlotSig {
    const void *many;
    unsigned bx;
    size_t smem;
    long long bound;
};

// What a batched step leaves of each member, gathered into one array that
// is copied back after the step: count, d_g, Fx, Fy, M.
constexpr int GATHER = 5;
__global__ void k_batch_gather(const VxScalars *const *S, double *out, int nb) {
    VX_PDL_WAIT();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
        const VxScalars *q = S[i];
        double *o = out + (long long)GATHER * i;
        o[0] = (double)q->n;
        o[1] = q->dg;
        o[2] = q->fx;
        o[3] = q->fy;
        o[4] = q->m;
    }
}

long long pow2_at_least(long long v) {
    long long q = 1;
    while (q < v) q <<= 1;
    return q;
}

}  // namespace

struct vx_batch {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    std::vector<Body> bodies;
    int share_div = 1;
    std::vector<Slot> slots;
    // device arena: VxSlot[ns] | scalar pointers [nb] | per slot: first[] | packs
    unsigned char *d_arena = nullptr;
    size_t arena_cap = 0;
    std::vector<unsigned char> h_arena;
    unsigned char *h_stage[2] = {nullptr, nullptr};
    size_t stage_cap[2] = {0, 0};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    int stage_idx = 0;
    // graph
    cudaGraphExec_t exec = nullptr;
    std::vector<SlotSig> sig;
    const unsigned char *sig_arena = nullptr;
    const double *sig_gather = nullptr;
    size_t sig_nb = 0;
    // what each step left of its members (GATHER values each), copied back
    // after the step (two steps kept), with the members of that step
    double *d_gather = nullptr;
    double *h_gather[2] = {nullptr, nullptr};
    size_t gather_cap = 0;                  // members the buffers hold
    cudaEvent_t cnt_ev[2] = {nullptr, nullptr};
    long long cnt_step[2] = {-1, -1};
    std::vector<vx_sim *> cnt_members[2];
    long long launched = 0;       // batched steps launched
    long long kernels = 0;        // kernels launched by the batched steps
    long long rebuilds = 0, reinstantiations = 0;
    // host time spent in vx_batch_step's preparation of a step: capacity
    // growth, then re-recording / merging / uploading (max and total, ms)
    double grow_ms_max = 0.0, grow_ms_sum = 0.0, refresh_ms_max = 0.0, refresh_ms_sum = 0.0;
    // the longest of refresh's phases: re-recording, merge + layout, upload, graph build (ms)
    double phase_ms_max[4] = {0.0, 0.0, 0.0, 0.0};
    // pinned buffers outgrown while steps were in flight: freed at destroy
    // (cudaFreeHost waits for the whole device, which would drain the
    // pipeline of batched steps)
    std::vector<void *> retired;
    bool dirty = true;
};

static vx_status free_graph(vx_batch *b) {
    if (b->exec) {
        cudaStreamSynchronize(b->stream);   // no launch of it still running
        cudaGraphExecDestroy(b->exec);
    }
    b->exec = nullptr;
    b->sig.clear();
    return VX_OK;
}

// Merge of the bodies' launch sequences into slots: a common supersequence
// of them, built body by body (longest recordings first) by aligning each
// body's (kernel, block) sequence with the merged one along a longest common
// subsequence; a slot is one entry of the merged sequence, run by every body
// aligned to it.  Bodies whose steps differ (direct or quadtree velocity, a
// quadtree with more levels, the collapse passes) then share every kernel
// their sequences have in common, in order; a greedy merge (the kernel at
// the head of the most sequences first) let a minority group fall behind and
// run the rest of its step in slots of its own (140 slots for the seeded
// 256-body population instead of about 60).
static vx_status merge(vx_batch *b) {
    const int nb = (int)b->bodies.size();
    using Key = std::pair<const void *, unsigned>;
    auto key_at = [&](int i, size_t q) {
        const VxRecLaunch &r = b->bodies[(size_t)i].rec.launches[q];
        return Key(r.key, r.block.x);
    };
    // the merged sequence (each entry a slot key with a stable id) and, per
    // body, the slot id of each of its launches
    std::vector<Key> seq;
    std::vector<int> seq_id;
    std::vector<std::vector<int>> at((size_t)nb);
    int next_id = 0;
    std::vector<int> order((size_t)nb);
    for (int i = 0; i < nb; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return b->bodies[(size_t)a].rec.launches.size() > b->bodies[(size_t)c].rec.launches.size();
    });
    std::vector<int> dp;
    // bodies with the same sequence take the same slots (aligned once)
    std::map<std::vector<Key>, int> seen;
    for (int i : order) {
        const size_t m = seq.size(), n = b->bodies[(size_t)i].rec.launches.size();
        std::vector<Key> mykeys(n);
        for (size_t c = 0; c < n; ++c) mykeys[c] = key_at(i, c);
        const auto hit = seen.find(mykeys);
        if (hit != seen.end()) {
            at[(size_t)i] = at[(size_t)hit->second];
            continue;
        }
        seen.emplace(std::move(mykeys), i);
        // longest common subsequence of seq[a..] and the body's launches[c..]
        dp.assign((m + 1) * (n + 1), 0);
        for (size_t a = m; a-- > 0;)
            for (size_t c = n; c-- > 0;)
                dp[a * (n + 1) + c] = seq[a] == key_at(i, c)
                                          ? dp[(a + 1) * (n + 1) + c + 1] + 1
                                          : std::max(dp[(a + 1) * (n + 1) + c], dp[a * (n + 1) + c + 1]);
        std::vector<Key> ns;
        std::vector<int> nid;
        std::vector<int> &mine = at[(size_t)i];
        mine.assign(n, -1);
        size_t a = 0, c = 0;
        while (a < m || c < n) {
            if (a < m && c < n && seq[a] == key_at(i, c)) {
                ns.push_back(seq[a]); nid.push_back(seq_id[a]);
                mine[c] = seq_id[a];
                ++a; ++c;
            } else if (c == n || (a < m && dp[(a + 1) * (n + 1) + c] >= dp[a * (n + 1) + c + 1])) {
                ns.push_back(seq[a]); nid.push_back(seq_id[a]);
                ++a;
            } else {
                ns.push_back(key_at(i, c)); nid.push_back(next_id);
                mine[c] = next_id++;
                ++c;
            }
        }
        seq.swap(ns);
        seq_id.swap(nid);
    }
    std::vector<int> slot_of((size_t)next_id, -1);
    for (size_t j = 0; j < seq_id.size(); ++j) slot_of[(size_t)seq_id[j]] = (int)j;
    b->slots.assign(seq.size(), Slot());
    for (int i = 0; i < nb; ++i) {
        const auto &L = b->bodies[(size_t)i].rec.launches;
        for (size_t q = 0; q < L.size(); ++q) {
            const VxRecLaunch &r = L[q];
            Slot &sl = b->slots[(size_t)slot_of[(size_t)at[(size_t)i][q]]];
            if (r.grid.y != 1 || r.grid.z != 1 || r.block.y != 1 || r.block.z != 1) {
                vx_set_error("batch: a step kernel with a multi-dimensional launch cannot be batched");
                return VX_ERR_ARG;
            }
            if (sl.bodies.empty()) {
                sl.key = r.key;
                sl.many = r.many;
                sl.block = r.block;
                sl.pack = r.size;
            } else if (r.size != sl.pack || r.many != sl.many) {
                vx_set_error("batch: one kernel recorded with different argument packs");
                return VX_ERR_ARG;
            }
            sl.smem = std::max(sl.smem, r.smem);
            sl.bodies.push_back(i);
            sl.launch.push_back((int)q);
            sl.total += r.grid.x;
        }
    }
    return VX_OK;
}

static size_t align16(size_t v) { return (v + 15) / 16 * 16; }

// Lay out the arena for the current slots on the host (device addresses from
// `base`); returns its size.
static size_t layout(vx_batch *b, unsigned char *base) {
    const size_t ns = b->slots.size(), nb = b->bodies.size();
    size_t off = align16(ns * sizeof(VxSlot));
    const size_t s_off = off;
    off = align16(off + nb * sizeof(VxScalars *));
    std::vector<size_t> first_off(ns), pack_off(ns);
    for (size_t j = 0; j < ns; ++j) {
        first_off[j] = off;
        off = align16(off + (b->slots[j].bodies.size() + 1) * sizeof(int));
    }
    for (size_t j = 0; j < ns; ++j) {
        pack_off[j] = off;
        off = align16(off + b->slots[j].bodies.size() * align16(b->slots[j].pack));
    }
    const size_t size = off;
    b->h_arena.assign(size, 0);
    unsigned char *h = b->h_arena.data();
    VxSlot *hs = reinterpret_cast<VxSlot *>(h);
    for (size_t j = 0; j < ns; ++j) {
        const Slot &sl = b->slots[j];
        VxSlot d;
        d.nb = (int)sl.bodies.size();
        d.pad = 0;
        d.stride = (long long)align16(sl.pack);
        d.first = reinterpret_cast<const int *>(base + first_off[j]);
        d.packs = base + pack_off[j];
        hs[j] = d;
        int *first = reinterpret_cast<int *>(h + first_off[j]);
        long long acc = 0;
        for (size_t q = 0; q < sl.bodies.size(); ++q) {
            const Body &bd = b->bodies[(size_t)sl.bodies[q]];
            const VxRecLaunch &r = bd.rec.launches[(size_t)sl.launch[q]];
            first[q] = (int)acc;
            acc += r.grid.x;
            memcpy(h + pack_off[j] + q * align16(sl.pack), bd.rec.arena.data() + r.off, r.size);
        }
        first[sl.bodies.size()] = (int)acc;
    }
    VxScalars **sp = reinterpret_cast<VxScalars **>(h + s_off);
    for (size_t i = 0; i < nb; ++i) sp[i] = b->bodies[i].s->d_S;
    return size;
}

static const VxScalars *const *scalars_list(vx_batch *b) {
    const size_t ns = b->slots.size();
    return reinterpret_cast<const VxScalars *const *>(b->d_arena + align16(ns * sizeof(VxSlot)));
}

static vx_status build_graph(vx_batch *b) {
    free_graph(b);
    for (const Slot &sl : b->slots) {
        if (sl.smem > 48 * 1024)
            BCU(cudaFuncSetAttribute(sl.many, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sl.smem));
        cudaFuncAttributes fa;
        BCU(cudaFuncGetAttributes(&fa, sl.many));
        if ((int)sl.block.x > fa.maxThreadsPerBlock) {
            vx_set_error("batch: a multi-body kernel takes at most %d threads per block, %u recorded",
                         fa.maxThreadsPerBlock, sl.block.x);
            return VX_ERR_CUDA;
        }
    }
    cudaGraph_t graph;
    BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (size_t j = 0; j < b->slots.size() && e == cudaSuccess; ++j) {
        const Slot &sl = b->slots[j];
        SlotSig g{sl.many, sl.block.x, sl.smem, std::max<long long>(1, pow2_at_least(sl.total))};
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)g.bound);
        cfg.blockDim = sl.block;
        cfg.dynamicSmemBytes = sl.smem;
        cfg.stream = b->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const VxSlot *slot = reinterpret_cast<const VxSlot *>(b->d_arena) + j;
        void *args[1] = {&slot};
        e = cudaLaunchKernelExC(&cfg, sl.many, args);
        b->sig.push_back(g);
    }
    if (e == cudaSuccess) {
        const int nb = (int)b->bodies.size();
        vx_launch_pdl(k_batch_gather, std::max(1, std::min(64, (nb + 255) / 256)), 256, 0, b->stream,
                      scalars_list(b), b->d_gather, nb);
        e = cudaGetLastError();
    }
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        b->sig.clear();
        vx_set_error("batch graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        return VX_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        b->exec = nullptr;
        b->sig.clear();
        vx_set_error("batch graph instantiate: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    b->sig_arena = b->d_arena;
    b->sig_gather = b->d_gather;
    b->sig_nb = b->bodies.size();
    b->reinstantiations += 1;
    return VX_OK;
}

static bool graph_fits(const vx_batch *b) {
    if (!b->exec || b->sig_arena != b->d_arena || b->sig_gather != b->d_gather || b->sig_nb != b->bodies.size() ||
        b->sig.size() != b->slots.size())
        return false;
    for (size_t j = 0; j < b->slots.size(); ++j) {
        const SlotSig &g = b->sig[j];
        const Slot &sl = b->slots[j];
        if (g.many != sl.many || g.bx != sl.block.x || sl.smem > g.smem || sl.total > g.bound) return false;
    }
    return true;
}

// Copy the host arena into the device one: a pinned staging buffer (two,
// used in turn, each reused only after its previous copy finished) and a
// copy ordered on the batch stream after the steps already launched.
static vx_status upload(vx_batch *b) {
    const size_t size = b->h_arena.size();
    const int k = b->stage_idx;
    b->stage_idx ^= 1;
    BCU(cudaEventSynchronize(b->stage_ev[k]));
    if (b->stage_cap[k] < size) {
        if (b->h_stage[k]) b->retired.push_back(b->h_stage[k]);
        b->h_stage[k] = nullptr;
        b->stage_cap[k] = 0;
        const size_t cap = size + size / 2;   // headroom: members' tables grow with them
        BCU(cudaMallocHost(&b->h_stage[k], cap));
        b->stage_cap[k] = cap;
    }
    memcpy(b->h_stage[k], b->h_arena.data(), size);
    BCU(cudaMemcpyAsync(b->d_arena, b->h_stage[k], size, cudaMemcpyHostToDevice, b->stream));
    BCU(cudaEventRecord(b->stage_ev[k], b->stream));
    return VX_OK;
}

// A body's claim on the GPU in a batched step: its store's capacity in
// units of 2048 vortices (the work of every stage grows with the count; the
// capacity changes only when the store grows, which re-records the body
// anyway).  Its share is that claim over the batch's divisor, at most the
// SMs its own step would use: a stage's blocks then carry about the same
// work in every body, and the biggest bodies do not run on alone at the end
// of each stage.
#ifndef VX_BATCH_FILL
#define VX_BATCH_FILL 8   // times the members' scaled launches fill the GPU
#endif
static long long share_demand(const vx_sim *s) { return std::max(1LL, s->cap / 2048); }
static void update_share(vx_batch *b);

static BodyKey key_of(vx_batch *b, vx_sim *s) {
    BodyKey k;
    k.cap = s->cap;
    k.rhs = vx_sim_rhs_chunks(s);
    k.sms = vx_sim_step_sms(s);
    k.share = std::max(1, std::min(k.sms, (int)((share_demand(s) + b->share_div - 1) / b->share_div)));
    k.fmm = s->conf.fmm;
    k.leaf = s->prm.fmm_leaf;
    k.lmax = s->w.fmm_lmax;
    return k;
}

// Re-record the bodies whose recordings are stale, then merge, lay out,
// upload and (if needed) re-instantiate.
static double ms_since(std::chrono::steady_clock::time_point &t) {
    const auto now = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
    return ms;
}

static vx_status refresh(vx_batch *b) {
    auto tp = std::chrono::steady_clock::now();
    auto phase = [&](int q) { b->phase_ms_max[q] = std::max(b->phase_ms_max[q], ms_since(tp)); };
    update_share(b);   // growth moves the members' claims (the divisor has hysteresis)
    bool changed = b->dirty;
    for (Body &bd : b->bodies) {
        const BodyKey k = key_of(b, bd.s);
        if (bd.recorded && k == bd.key) continue;
        bd.rec.launches.clear();
        bd.rec.arena.clear();
        const cudaError_t e = vx_sim_launch_stages(bd.s, VX_STAGE_ALL, true, &bd.rec, k.share);
        if (e != cudaSuccess) {
            vx_set_error("batch: recording a body's step: %s", cudaGetErrorString(e));
            return VX_ERR_CUDA;
        }
        bd.key = k;
        bd.recorded = true;
        changed = true;
    }
    phase(0);
    if (!changed) return VX_OK;
    vx_status st = merge(b);
    if (st != VX_OK) return st;
    size_t need = layout(b, b->d_arena);
    if (need > b->arena_cap) {
        if (b->d_arena) BCU(cudaFreeAsync(b->d_arena, b->stream));   // after the steps in flight
        b->d_arena = nullptr;
        b->arena_cap = 0;
        const size_t cap = std::max(need + need / 2, (size_t)1 << 16);
        BCU(cudaMallocAsync((void **)&b->d_arena, cap, b->stream));
        b->arena_cap = cap;
        need = layout(b, b->d_arena);
    }
    phase(1);
    if ((st = upload(b)) != VX_OK) return st;
    phase(2);
    if (!graph_fits(b) && (st = build_graph(b)) != VX_OK) return st;
    phase(3);
    b->rebuilds += 1;
    b->dirty = false;
    return VX_OK;
}

// Upper bounds of the counts before the next step, from the counts copied
// back after step `launched - 2` (the step before the one in flight);
// bodies that may outgrow their stores grow (stream-ordered).
static vx_status ensure_capacities(vx_batch *b) {
    bool need_counts = false;
    for (Body &bd : b->bodies)
        if (vx_sim_need(bd.s, bd.s->n_upper) > bd.s->cap) need_counts = true;
    if (!need_counts) return VX_OK;
    const long long want = b->launched - 2;
    int k = -1;
    for (int q = 0; q < 2; ++q)
        if (b->cnt_step[q] >= 0 && b->cnt_step[q] >= want && (k < 0 || b->cnt_step[q] < b->cnt_step[k])) k = q;
    if (k < 0)
        for (int q = 0; q < 2; ++q)
            if (b->cnt_step[q] >= 0 && (k < 0 || b->cnt_step[q] > b->cnt_step[k])) k = q;
    if (k >= 0) {
        BCU(cudaEventSynchronize(b->cnt_ev[k]));
        const long long after = b->launched - 1 - b->cnt_step[k];   // steps launched after those counts
        const std::vector<vx_sim *> &mem = b->cnt_members[k];
        for (size_t i = 0; i < mem.size(); ++i) {
            vx_sim *s = mem[i];
            if (!s->in_batch || s->stream != b->stream) continue;   // left the batch since
            const long long bound = (long long)b->h_gather[k][GATHER * i] + after * s->P;
            if (bound < s->n_upper) s->n_upper = bound;
        }
    }
    // the members that grow now take their new stores and scratch from the
    // device's pool: one allocation of their total, given back at once,
    // leaves that memory in the pool (its release threshold keeps it), so
    // their own allocations are served from it instead of each mapping new
    // memory (hundreds of ms when a batch of bodies grows together)
    long long grow_bytes = 0;
    for (Body &bd : b->bodies) {
        vx_sim *s = bd.s;
        const long long need = vx_sim_need(s, s->n_upper);
        if (need > s->cap) grow_bytes += vx_sim_grow_bytes(s, need);
    }
    if (grow_bytes > 0) {
        void *reserve = nullptr;
        if (cudaMallocAsync(&reserve, (size_t)grow_bytes, b->stream) == cudaSuccess)
            cudaFreeAsync(reserve, b->stream);
        else
            cudaGetLastError();   // no room for the whole at once: the members allocate one by one
    }
    for (Body &bd : b->bodies) {
        vx_sim *s = bd.s;
        const long long need = vx_sim_need(s, s->n_upper);
        if (need > s->cap) {
            const vx_status st = vx_sim_grow(s, need);
            if (st != VX_OK) return st;
        }
    }
    return VX_OK;
}

static void release(vx_batch *b) {
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_graph(b);
    for (Body &bd : b->bodies) {
        vx_sim *s = bd.s;
        if (!s || !s->in_batch) continue;
        s->stream = s->own_stream;
        s->own_stream = nullptr;
        s->in_batch = false;
        vx_sim_read_scalars(s);   // the true count again
    }
    if (b->d_arena) cudaFree(b->d_arena);
    if (b->d_gather) cudaFree(b->d_gather);
    for (int k = 0; k < 2; ++k) {
        if (b->h_stage[k]) cudaFreeHost(b->h_stage[k]);
        if (b->h_gather[k]) cudaFreeHost(b->h_gather[k]);
        if (b->stage_ev[k]) cudaEventDestroy(b->stage_ev[k]);
        if (b->cnt_ev[k]) cudaEventDestroy(b->cnt_ev[k]);
    }
    for (void *h : b->retired) cudaFreeHost(h);
    b->retired.clear();
    if (b->stream) cudaStreamDestroy(b->stream);
}

// Members' shares of the GPU: the scaled launches of all members together
// fill it VX_BATCH_FILL times; the divisor is kept while the total demand
// stays within a factor of two of the one it was set for (a new divisor
// changes every member's launch shapes, so all are recorded again).
static void update_share(vx_batch *b) {
    long long demand = 0;
    for (const Body &bd : b->bodies) demand += share_demand(bd.s);
    const int want = (int)std::max(1LL, demand / ((long long)VX_BATCH_FILL * b->num_sms));
    if (want > 2 * b->share_div || 2 * want < b->share_div) b->share_div = want;
}

// Room for `nb` members in the gathered results (the device array is
// stream-ordered: steps in flight still write the old one).  The host copies
// of the last two steps' results are carried over into the larger buffers,
// so a step that is still to be collected keeps its results.
static vx_status gather_room(vx_batch *b, size_t nb) {
    if (nb <= b->gather_cap && b->d_gather) return VX_OK;
    size_t cap = std::max<size_t>(std::max<size_t>(nb, 2 * b->gather_cap), 16);
    for (int k = 0; k < 2; ++k) {
        BCU(cudaEventSynchronize(b->cnt_ev[k]));   // its last copy has landed
        double *old = b->h_gather[k];
        double *grown = nullptr;
        BCU(cudaMallocHost(&grown, sizeof(double) * GATHER * cap));
        if (old) {
            const size_t keep = std::min(b->cnt_members[k].size(), b->gather_cap);
            memcpy(grown, old, sizeof(double) * GATHER * keep);
            b->retired.push_back(old);
        }
        b->h_gather[k] = grown;
    }
    if (b->d_gather) BCU(cudaFreeAsync(b->d_gather, b->stream));
    b->d_gather = nullptr;
    BCU(cudaMallocAsync((void **)&b->d_gather, sizeof(double) * GATHER * cap, b->stream));
    b->gather_cap = cap;
    return VX_OK;
}

extern "C" vx_status vx_batch_new(int device, vx_batch **out) {
    if (!out) return VX_ERR_ARG;
    *out = nullptr;
    BCU(cudaSetDevice(device));
    vx_batch *b = new vx_batch();
    b->device = device;
    auto fail = [&](vx_status st) {
        release(b);
        delete b;
        return st;
    };
    vx_keep_pool(device);
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(VX_ERR_CUDA);
    for (int k = 0; k < 2; ++k)
        if (cudaEventCreateWithFlags(&b->stage_ev[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->cnt_ev[k], cudaEventDisableTiming) != cudaSuccess)
            return fail(VX_ERR_CUDA);
    vx_status st = gather_room(b, 16);
    if (st != VX_OK) return fail(st);
    *out = b;
    return VX_OK;
}

// A body joins at the next batched step: the batch's stream waits for the
// work already queued on the body's own stream (no host wait).
extern "C" vx_status vx_batch_add(vx_batch *b, vx_sim *s) {
    if (!b || !s) return VX_ERR_ARG;
    if (s->device != b->device || s->in_batch) {
        vx_set_error("vx_batch_add: the body is on another device or already in a batch");
        return VX_ERR_ARG;
    }
    BCU(cudaSetDevice(b->device));
    cudaEvent_t e;
    BCU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t err = cudaEventRecord(e, s->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(b->stream, e, 0);
    cudaEventDestroy(e);
    BCU(err);
    Body bd;
    bd.s = s;
    b->bodies.push_back(std::move(bd));
    s->own_stream = s->stream;
    s->stream = b->stream;
    s->in_batch = true;
    vx_status st = gather_room(b, b->bodies.size());
    if (st != VX_OK) return st;
    update_share(b);
    b->dirty = true;
    return VX_OK;
}

// A body leaves after the batched steps already launched: its own stream
// waits for them (no host wait) and it can be stepped alone again.
extern "C" vx_status vx_batch_remove(vx_batch *b, vx_sim *s) {
    if (!b || !s) return VX_ERR_ARG;
    size_t i = 0;
    while (i < b->bodies.size() && b->bodies[i].s != s) ++i;
    if (i == b->bodies.size()) {
        vx_set_error("vx_batch_remove: the body is not in this batch");
        return VX_ERR_ARG;
    }
    BCU(cudaSetDevice(b->device));
    cudaEvent_t e;
    BCU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t err = cudaEventRecord(e, b->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(s->own_stream, e, 0);
    cudaEventDestroy(e);
    BCU(err);
    s->stream = s->own_stream;
    s->own_stream = nullptr;
    s->in_batch = false;
    b->bodies.erase(b->bodies.begin() + (long)i);
    update_share(b);
    b->dirty = true;
    return VX_OK;
}

extern "C" vx_status vx_batch_create(vx_sim *const *sims, int count, vx_batch **out) {
    if (!sims || count < 1 || !out) return VX_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < count; ++i) {
        if (!sims[i] || sims[i]->device != sims[0]->device || sims[i]->in_batch) {
            vx_set_error("vx_batch_create: body %d is null, on another device or already in a batch", i);
            return VX_ERR_ARG;
        }
        for (int j = 0; j < i; ++j)
            if (sims[j] == sims[i]) {
                vx_set_error("vx_batch_create: body %d is listed twice", i);
                return VX_ERR_ARG;
            }
    }
    vx_batch *b = nullptr;
    vx_status st = vx_batch_new(sims[0]->device, &b);
    if (st != VX_OK) return st;
    for (int i = 0; i < count && st == VX_OK; ++i) st = vx_batch_add(b, sims[i]);
    if (st != VX_OK) {
        vx_batch_destroy(b);
        return st;
    }
    *out = b;
    return VX_OK;
}

extern "C" vx_status vx_batch_step(vx_batch *b, int64_t nsteps) {
    if (!b || nsteps < 0) return VX_ERR_ARG;
    BCU(cudaSetDevice(b->device));
    if (b->bodies.empty()) return VX_OK;
    for (int64_t t = 0; t < nsteps; ++t) {
        const auto t0 = std::chrono::steady_clock::now();
        vx_status st = ensure_capacities(b);
        if (st != VX_OK) return st;
        const auto t1 = std::chrono::steady_clock::now();
        if ((st = refresh(b)) != VX_OK) return st;
        const auto t2 = std::chrono::steady_clock::now();
        const double gm = std::chrono::duration<double, std::milli>(t1 - t0).count();
        const double rm = std::chrono::duration<double, std::milli>(t2 - t1).count();
        b->grow_ms_max = std::max(b->grow_ms_max, gm);
        b->grow_ms_sum += gm;
        b->refresh_ms_max = std::max(b->refresh_ms_max, rm);
        b->refresh_ms_sum += rm;
        const int k = (int)(b->launched & 1);
        BCU(cudaEventSynchronize(b->cnt_ev[k]));   // the host buffer of two steps ago has been read
        BCU(cudaGraphLaunch(b->exec, b->stream));
        BCU(cudaMemcpyAsync(b->h_gather[k], b->d_gather, sizeof(double) * GATHER * b->bodies.size(),
                            cudaMemcpyDeviceToHost, b->stream));
        BCU(cudaEventRecord(b->cnt_ev[k], b->stream));
        b->cnt_step[k] = b->launched;
        b->cnt_members[k].clear();
        for (const Body &bd : b->bodies) b->cnt_members[k].push_back(bd.s);
        b->launched += 1;
        b->kernels += (long long)b->slots.size() + 1;
        for (Body &bd : b->bodies) bd.s->n_upper += bd.s->P;
    }
    return VX_OK;
}

// Waits for batched step `step` (the index among the batch's steps; the
// last two launched are kept) and reports, for each body that took part in
// it (in the batch's order at that step), the count and the force sums it
// left: 5 values per body (count, d_g, Fx, Fy, M).
extern "C" vx_status vx_batch_results(vx_batch *b, int64_t step, vx_sim **members, double *out5, int cap,
                                      int *count) {
    if (!b || !count || cap < 0) return VX_ERR_ARG;
    *count = 0;
    const int k = (int)(step & 1);
    if (step < 0 || b->cnt_step[k] != step) {
        vx_set_error("vx_batch_results: step %lld is not one of the last two launched", (long long)step);
        return VX_ERR_ARG;
    }
    BCU(cudaSetDevice(b->device));
    BCU(cudaEventSynchronize(b->cnt_ev[k]));
    const std::vector<vx_sim *> &mem = b->cnt_members[k];
    const int n = (int)std::min<size_t>(mem.size(), (size_t)cap);
    for (int i = 0; i < n; ++i) {
        if (members) members[i] = mem[(size_t)i];
        if (out5) memcpy(out5 + GATHER * i, b->h_gather[k] + GATHER * i, sizeof(double) * GATHER);
    }
    *count = (int)mem.size();
    return VX_OK;
}

extern "C" vx_status vx_batch_last_results(vx_batch *b, vx_sim **members, double *out5, int cap, int *count) {
    if (!b || !count) return VX_ERR_ARG;
    *count = 0;
    if (b->launched == 0) return VX_OK;
    return vx_batch_results(b, b->launched - 1, members, out5, cap, count);
}

extern "C" vx_status vx_batch_sync(vx_batch *b) {
    if (!b) return VX_ERR_ARG;
    BCU(cudaSetDevice(b->device));
    BCU(cudaStreamSynchronize(b->stream));
    for (Body &bd : b->bodies) {
        const vx_status st = vx_sim_read_scalars(bd.s);
        if (st != VX_OK) return st;
    }
    return VX_OK;
}

// out[0] batched steps, [1] kernels launched by them, [2] kernels per step
// now (slots + the count gather), [3] slot-table rebuilds, [4] graph
// instantiations, [5] bodies.
extern "C" vx_status vx_batch_info(vx_batch *b, double out6[6]) {
    if (!b || !out6) return VX_ERR_ARG;
    out6[0] = (double)b->launched;
    out6[1] = (double)b->kernels;
    out6[2] = (double)b->slots.size() + 1;
    out6[3] = (double)b->rebuilds;
    out6[4] = (double)b->reinstantiations;
    out6[5] = (double)b->bodies.size();
    return VX_OK;
}

// Host time of the steps' preparation: out[0] / [1] the longest / total
// capacity growth, [2] / [3] the longest / total re-recording, merge and
// upload, [4..7] the longest re-recording, merge + layout, upload and graph
// build (ms).
extern "C" vx_status vx_batch_host_times(vx_batch *b, double out8[8]) {
    if (!b || !out8) return VX_ERR_ARG;
    out8[0] = b->grow_ms_max;
    out8[1] = b->grow_ms_sum;
    out8[2] = b->refresh_ms_max;
    out8[3] = b->refresh_ms_sum;
    for (int q = 0; q < 4; ++q) out8[4 + q] = b->phase_ms_max[q];
    return VX_OK;
}

extern "C" void *vx_batch_stream(vx_batch *b) { return b ? (void *)b->stream : nullptr; }

extern "C" vx_status vx_batch_destroy(vx_batch *b) {
    if (!b) return VX_OK;
    cudaSetDevice(b->device);
    release(b);
    vx_trim_pool(b->device);
    delete b;
    return VX_OK;
}
