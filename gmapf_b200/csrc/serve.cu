// serve.cu -- serving form: agent retargets admitted continuously.
//
// The reference has no serving form: a retarget (SetAgentTargPos,
// src/GMAPF.cu:238-253) waits for the next AsyncStep, whose KernelSearch runs
// the frame's requests to completion (PathFinder.h:508-598).  Here a retarget
// becomes a query the moment it is submitted:
//   - the host fixes its start (the triangle under the agent's position at
//     submission) and target, and appends it to a device ring whose capacity
//     is set by free device memory (one path row per entry plus the search
//     state); queries beyond the capacity wait on the host until entries are
//     released;
//   - each poll launches the queries admitted since the previous launch as a
//     micro-batch on one of kStreams streams that is idle; every stream owns
//     its own range of search slots, so up to kStreams batches run at once
//     and queries that arrive while others run start without waiting for
//     them (a persistent launch over its batch: warps take queries as they
//     free up);
//   - each completion writes a done word into host-mapped memory after its
//     results; latency = the host time a poll sees it - the arrival time;
//   - a finished query's result moves to a per-agent stash (unless a newer
//     query of the same agent was submitted), which frees its ring entry; at
//     the next frame boundary a kernel installs the stashed paths into their
//     agents, ahead of the frame's compaction and mover.  Until then an agent
//     keeps its previous motion.
// A query's result depends only on its start, target and the map, so it is
// the same alone and among any other queries.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>

#include "internal.h"

namespace gmapf_b200 {

#define SCK(x)                                                                       \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            err = std::string(#x) + " failed: " + cudaGetErrorString(e_);            \
            return GMAPF_E_CUDA;                                                     \
        }                                                                            \
    } while (0)

namespace {

enum SlotState : unsigned char { SLOT_FREE = 0, SLOT_ADMITTED, SLOT_STASHING };

struct Waiting {
    int agent, start, tnode;
    float tx, ty;
    long long arrival_ns;
    unsigned sub;  // the agent's submission number
};

struct SlotInfo {
    int agent = -1, tnode = -1;
    float tx = 0, ty = 0;
    long long arrival_ns = 0;
    unsigned sub = 0;
};

// a stashed result to install: agent, target triangle and position
struct ApplyRec {
    int agent, tnode;
    float tx, ty;
};

// finished queries -> the per-agent stash (one block per query): {slot, agent}
__global__ void k_serve_stash(const int2* recs, int n, const int* found, const int* lens, const int* pool,
                              long long stride, int2* stash_fl, int* stash_path) {
    const int k = blockIdx.x;
    if (k >= n) return;
    const int2 r = recs[k];
    const int f = found[r.x];
    const int L = f ? lens[r.x] : 0;
    const bool ok = L >= 0 && L <= stride;
    if (ok)
        for (int i = threadIdx.x; i < L; i += blockDim.x)
            stash_path[(long long)r.y * stride + i] = pool[(long long)r.x * stride + i];
    if (threadIdx.x == 0) stash_fl[r.y] = make_int2(f, ok ? L : -1);
}

// install stashed results into their agents (one block per agent)
__global__ void k_serve_apply(const ApplyRec* recs, int n, const int2* stash_fl, const int* stash_path,
                              long long stride, int* paths, int* state, int* step_idx, int* path_len, int* targ,
                              float2* targ_pos) {
    const int k = blockIdx.x;
    if (k >= n) return;
    const ApplyRec r = recs[k];
    const int2 fl = stash_fl[r.agent];
    const int f = fl.x;
    const int L = f ? fl.y : 0;
    const bool ok = L >= 0 && L <= stride;
    if (ok)
        for (int i = threadIdx.x; i < L; i += blockDim.x)
            paths[(long long)r.agent * stride + i] = stash_path[(long long)r.agent * stride + i];
    if (threadIdx.x == 0) {
        targ[r.agent] = r.tnode;
        targ_pos[r.agent] = make_float2(r.tx, r.ty);
        path_len[r.agent] = ok ? L : 0;
        // PathFinder.h:268-289: found -> Move from step -1, else Idle with the
        // step index left as it was; an empty path means the agent already
        // stands in the target triangle
        const bool move = f && ok && L > 0;
        if (move) step_idx[r.agent] = -1;
        state[r.agent] = move ? GMAPF_AGENT_MOVE : GMAPF_AGENT_IDLE;
    }
}

}  // namespace

constexpr int kStreams = 8;

struct Service {
    int cap = 0;
    // batches
    cudaStream_t st[kStreams] = {};
    cudaEvent_t st_done[kStreams] = {};
    bool st_busy[kStreams] = {};
    int slots_per_stream = 0;
    int* d_wc = nullptr;   // per stream: work counter, query count
    int* h_cnt = nullptr;  // pinned: per stream, the batch's query count
    int* d_err = nullptr;  // per stream: device-side error bits
    int* h_err = nullptr;  // pinned copies
    long long launched = 0;  // queries [launched, tail) admitted, not yet launched
    // admission copies
    cudaStream_t copy = nullptr;
    cudaEvent_t copied = nullptr;
    bool copy_recorded = false;
    // stash
    cudaStream_t stash_stream = nullptr;
    cudaEvent_t stashed = nullptr, applied_ev = nullptr;
    bool stash_in_flight = false, apply_recorded = false;
    std::vector<int> stashing;  // ring entries freed when `stashed` completes
    int2* d_stash_fl = nullptr;  // per agent: found, length
    int* d_stash_path = nullptr; // per agent: path row
    int2* h_stash = nullptr;
    int2* d_stash_recs = nullptr;
    std::vector<void*> dallocs;
    int4* d_ring = nullptr;
    int *d_found = nullptr, *d_len = nullptr, *d_pool = nullptr;
    long long stride = 0;
    unsigned long long* h_done = nullptr;  // host-mapped
    unsigned long long* d_done = nullptr;
    // the service's own search state
    Rec* rec = nullptr;
    unsigned* epoch = nullptr;
    unsigned* gbm = nullptr;
    int slots = 0;
    unsigned long long* d_stats = nullptr;
    // pinned staging
    int4* h_stage = nullptr;
    ApplyRec* h_apply = nullptr;
    ApplyRec* d_apply = nullptr;
    // host bookkeeping
    long long tail = 0, released = 0;
    std::vector<SlotInfo> info;
    std::vector<unsigned char> state;
    std::deque<Waiting> waiting;
    std::vector<unsigned> agent_sub;  // per agent: number of its submissions
    std::vector<int> install;         // agents with a stashed result to install
    std::vector<unsigned char> to_install;
    std::vector<ApplyRec> target;     // per agent: the stashed result's target
    long long pending = 0;  // admitted, not done
    // statistics
    long long submitted = 0, completed = 0, found = 0, applied = 0, stale = 0, launches = 0;
    std::vector<float> lat_ms;
};

namespace {

long long now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

LocateGrid scene_grid(const Context& c, int s) {
    if (!c.is_world) return c.map.view();
    const SceneInfo& si = c.scenes[s];
    LocateGrid g;
    g.x0 = si.gx0;
    g.y0 = si.gy0;
    g.inv = si.ginv;
    g.w = si.gw;
    g.h = si.gh;
    g.start = c.map.gstart.data() + si.gstart_off;
    g.list = c.map.glist.data() + si.glist_off;
    g.degen = c.map.degen.data() + si.degen_off;
    g.ndegen = si.ndegen;
    g.tri = c.map.tri.data() + 3 * (size_t)si.node_base;
    g.n = si.n;
    g.base = si.node_base;
    return g;
}

int scene_of_agent(const Context& c, int a) {
    int lo = 0, hi = (int)c.scenes.size() - 1;
    while (lo < hi) {  // last scene with agent_base <= a
        const int mid = (lo + hi + 1) / 2;
        if (c.scenes[mid].agent_base <= a)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <class T>
int salloc(Service& sv, T** p, size_t count, std::string& err) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        err = std::string("serving buffers: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? GMAPF_E_CAPACITY : GMAPF_E_CUDA;
    }
    sv.dallocs.push_back(*p);
    return GMAPF_OK;
}

#define SALLOC(ptr, count)                          \
    do {                                            \
        int rc_ = salloc(sv, &(ptr), (count), err); \
        if (rc_ != GMAPF_OK) return rc_;            \
    } while (0)

SearchParams serve_params(Context& c, Service& sv, int k) {
    Device& d = c.dev;
    SearchParams p{};
    p.rows = d.rows;
    p.cen = d.cen;
    p.n = c.map.n;
    p.req = sv.d_ring;
    p.req_count_d = sv.d_wc + 2 * k + 1;
    p.work_ctr = sv.d_wc + 2 * k;
    p.T = c.T;
    p.C = c.C;
    p.K = c.K;
    p.rec = sv.rec;
    p.epoch = sv.epoch;
    p.gbm = sv.gbm;
    p.slot_base = k * sv.slots_per_stream;
    p.slots = sv.slots_per_stream;
    p.max_rounds = search_round_limit(c);
    p.promote_rounds = search_promote_rounds(c);
    p.paths = sv.d_pool;
    p.path_stride = sv.stride;
    p.out_found = sv.d_found;
    p.out_len = sv.d_len;
    p.stats = sv.d_stats;
    p.err = sv.d_err + k;
    p.ring_cap = sv.cap;
    p.ring_base = (int)sv.launched;
    p.done = sv.d_done;
    return p;
}

// completions since the last harvest: the latest of each agent goes to the
// stash (its ring entry is freed once the copy is done), superseded ones are
// freed at once; advances `released`
int harvest(Context& c, Service& sv, std::string& err) {
    if (sv.stash_in_flight && cudaEventQuery(sv.stashed) == cudaSuccess) {
        for (int slot : sv.stashing) sv.state[slot] = SLOT_FREE;
        sv.stashing.clear();
        sv.stash_in_flight = false;
    }
    std::vector<int2> fresh;
    long long now = 0;  // one clock reading for the completions seen by this poll
    for (long long q = sv.released; q < sv.tail; q++) {
        const int slot = (int)(q % sv.cap);
        if (sv.state[slot] != SLOT_ADMITTED) continue;
        const unsigned long long v = reinterpret_cast<volatile unsigned long long*>(sv.h_done)[slot];
        if ((v >> 1) != (unsigned long long)(q + 1)) continue;
        const SlotInfo& si = sv.info[slot];
        sv.pending--;
        sv.completed++;
        if (v & 1ull) sv.found++;
        if (now == 0) now = now_ns();
        sv.lat_ms.push_back((float)((double)(now - si.arrival_ns) * 1e-6));
        if (sv.agent_sub[si.agent] == si.sub) {
            fresh.push_back(make_int2(slot, si.agent));
        } else {
            sv.state[slot] = SLOT_FREE;  // a newer query of this agent supersedes it
            sv.stale++;
        }
    }
    if (!fresh.empty()) {
        if (sv.stash_in_flight) {  // one stash batch at a time
            SCK(cudaEventSynchronize(sv.stashed));
            for (int slot : sv.stashing) sv.state[slot] = SLOT_FREE;
            sv.stashing.clear();
        }
        const int n = (int)fresh.size();
        std::memcpy(sv.h_stash, fresh.data(), sizeof(int2) * n);
        SCK(cudaMemcpyAsync(sv.d_stash_recs, sv.h_stash, sizeof(int2) * n, cudaMemcpyHostToDevice, sv.stash_stream));
        // never overwrite a stash row while a frame still installs from it
        if (sv.apply_recorded) SCK(cudaStreamWaitEvent(sv.stash_stream, sv.applied_ev, 0));
        k_serve_stash<<<n, 128, 0, sv.stash_stream>>>(sv.d_stash_recs, n, sv.d_found, sv.d_len, sv.d_pool, sv.stride,
                                                       sv.d_stash_fl, sv.d_stash_path);
        SCK(cudaGetLastError());
        SCK(cudaEventRecord(sv.stashed, sv.stash_stream));
        sv.stash_in_flight = true;
        c.launches++;
        for (const int2& r : fresh) {
            sv.state[r.x] = SLOT_STASHING;
            sv.stashing.push_back(r.x);
            const SlotInfo& si = sv.info[r.x];
            sv.target[r.y] = ApplyRec{r.y, si.tnode, si.tx, si.ty};
            if (!sv.to_install[r.y]) {
                sv.to_install[r.y] = 1;
                sv.install.push_back(r.y);
            }
        }
    }
    while (sv.released < sv.tail && sv.state[(int)(sv.released % sv.cap)] == SLOT_FREE) sv.released++;
    return GMAPF_OK;
}

int admit_and_launch(Context& c, Service& sv, std::string& err) {
    // admit waiting queries into free ring entries
    const long long room = sv.cap - (sv.tail - sv.released);
    const long long n = std::min<long long>(room, (long long)sv.waiting.size());
    if (n > 0) {
        const long long first = sv.tail;
        for (long long k = 0; k < n; k++) {
            const Waiting w = sv.waiting.front();
            sv.waiting.pop_front();
            const int slot = (int)((first + k) % sv.cap);
            sv.h_stage[slot] = make_int4(-1, w.start, w.tnode, slot);
            SlotInfo& si = sv.info[slot];
            si.agent = w.agent;
            si.tnode = w.tnode;
            si.tx = w.tx;
            si.ty = w.ty;
            si.arrival_ns = w.arrival_ns;
            si.sub = w.sub;
            sv.state[slot] = SLOT_ADMITTED;
        }
        // the new entries: one or two contiguous ranges of the ring (their
        // staging entries are not rewritten before the entry is released)
        const int s0 = (int)(first % sv.cap);
        const long long run1 = std::min<long long>(n, sv.cap - s0);
        SCK(cudaMemcpyAsync(sv.d_ring + s0, sv.h_stage + s0, sizeof(int4) * run1, cudaMemcpyHostToDevice, sv.copy));
        if (run1 < n)
            SCK(cudaMemcpyAsync(sv.d_ring, sv.h_stage, sizeof(int4) * (n - run1), cudaMemcpyHostToDevice, sv.copy));
        SCK(cudaEventRecord(sv.copied, sv.copy));
        sv.copy_recorded = true;
        sv.tail += n;
        sv.pending += n;
    }
    // finished batches
    for (int k = 0; k < kStreams; k++) {
        if (!sv.st_busy[k] || cudaEventQuery(sv.st_done[k]) != cudaSuccess) continue;
        sv.st_busy[k] = false;
        if (sv.h_err[k] != 0) {
            err = "serving search: " + device_error_text(sv.h_err[k]);
            sv.h_err[k] = 0;
            return GMAPF_E_DEVICE;
        }
    }
    // the queries admitted since the last launch, as one batch on an idle stream
    if (sv.launched < sv.tail) {
        int k = -1;
        for (int j = 0; j < kStreams && k < 0; j++)
            if (!sv.st_busy[j]) k = j;
        if (k >= 0) {
            const long long cnt = sv.tail - sv.launched;
            sv.h_cnt[k] = (int)cnt;
            cudaStream_t st = sv.st[k];
            if (sv.copy_recorded) SCK(cudaStreamWaitEvent(st, sv.copied, 0));
            SCK(cudaMemsetAsync(sv.d_wc + 2 * k, 0, sizeof(int), st));
            SCK(cudaMemcpyAsync(sv.d_wc + 2 * k + 1, sv.h_cnt + k, sizeof(int), cudaMemcpyHostToDevice, st));
            SearchParams sp = serve_params(c, sv, k);
            const int gpb = c.block_threads / 32;
            const long long warps = std::min<long long>(cnt, sv.slots_per_stream);
            const int blocks = (int)((warps + gpb - 1) / gpb);
            SCK(launch_search(st, sp, blocks, c.block_threads, true, 0, c.dev.vm, c.dev.bm_words));
            SCK(cudaMemcpyAsync(sv.h_err + k, sv.d_err + k, sizeof(int), cudaMemcpyDeviceToHost, st));
            SCK(cudaEventRecord(sv.st_done[k], st));
            sv.st_busy[k] = true;
            sv.launched = sv.tail;
            sv.launches++;
            c.launches++;
        }
    }
    return GMAPF_OK;
}

}  // namespace

int serve_start(Context& c, int max_in_flight, std::string& err) {
    if (c.serve) return GMAPF_OK;
    Device& d = c.dev;
    SCK(cudaSetDevice(d.device));
    Service* psv = new Service();
    c.serve = psv;
    Service& sv = *psv;
    for (int k = 0; k < kStreams; k++) {
        SCK(cudaStreamCreateWithFlags(&sv.st[k], cudaStreamNonBlocking));
        SCK(cudaEventCreateWithFlags(&sv.st_done[k], cudaEventDisableTiming));
    }
    SCK(cudaStreamCreateWithFlags(&sv.copy, cudaStreamNonBlocking));
    SCK(cudaStreamCreateWithFlags(&sv.stash_stream, cudaStreamNonBlocking));
    SCK(cudaEventCreateWithFlags(&sv.copied, cudaEventDisableTiming));
    SCK(cudaEventCreateWithFlags(&sv.stashed, cudaEventDisableTiming));
    SCK(cudaEventCreateWithFlags(&sv.applied_ev, cudaEventDisableTiming));
    const int n = std::max(1, c.map.n);
    sv.stride = d.path_stride;

    // search state: the context's kernel shape, resident slots bounded by a
    // quarter of the free memory
    int sms = 0;
    SCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.device));
    size_t freeb = 0, totalb = 0;
    SCK(cudaMemGetInfo(&freeb, &totalb));
    const int gpb = c.block_threads / 32;
    const int per_sm = search_max_blocks_per_sm(c.T, c.C, c.block_threads, d.vm, d.bm_words);
    if (per_sm <= 0) {
        err = "serving: the search kernel cannot be resident with this shape";
        return GMAPF_E_CAPACITY;
    }
    const double per_slot = (double)n * sizeof(Rec) + (d.vm >= 3 ? 4.0 * d.bm_words : 0.0);
    // the drain launch is persistent while queries keep coming: leave one
    // block per SM for the frames' own kernels
    const int drain_per_sm = per_sm > 1 ? per_sm - 1 : 1;
    long long slots = std::min<long long>((long long)sms * drain_per_sm * gpb, (long long)(0.25 * freeb / per_slot));
    // split over the streams, whole blocks each
    const long long per_stream = (slots / kStreams / gpb) * gpb;
    if (per_stream < gpb) {
        err = "serving: not enough device memory for the search slots";
        return GMAPF_E_CAPACITY;
    }
    sv.slots_per_stream = (int)per_stream;
    sv.slots = (int)(per_stream * kStreams);
    SALLOC(sv.rec, (size_t)sv.slots * n);
    SALLOC(sv.epoch, (size_t)sv.slots);
    if (d.vm >= 3) SALLOC(sv.gbm, (size_t)sv.slots * d.bm_words);
    SALLOC(sv.d_stats, ST_COUNT);

    // ring: admission capacity from free memory (a path row and 16 bytes per entry)
    SCK(cudaMemGetInfo(&freeb, &totalb));
    const double per_entry = (double)sv.stride * 4.0 + 64.0;
    long long cap = std::min<long long>(max_in_flight > 0 ? max_in_flight : 65536, (long long)(0.25 * freeb / per_entry));
    cap = std::min<long long>(cap, 1 << 24);
    if (cap < 1) {
        err = "serving: not enough device memory for the query ring";
        return GMAPF_E_CAPACITY;
    }
    sv.cap = (int)cap;
    SALLOC(sv.d_ring, (size_t)sv.cap);
    SALLOC(sv.d_wc, 2 * kStreams);
    SALLOC(sv.d_err, kStreams);
    SALLOC(sv.d_found, (size_t)sv.cap);
    SALLOC(sv.d_len, (size_t)sv.cap);
    SALLOC(sv.d_pool, (size_t)sv.cap * sv.stride);
    SALLOC(sv.d_apply, (size_t)std::max(1, c.A));
    SALLOC(sv.d_stash_recs, (size_t)sv.cap);
    SALLOC(sv.d_stash_fl, (size_t)std::max(1, c.A));
    SALLOC(sv.d_stash_path, (size_t)std::max(1, c.A) * sv.stride);
    SCK(cudaHostAlloc((void**)&sv.h_done, sizeof(unsigned long long) * sv.cap, cudaHostAllocMapped));
    std::memset(sv.h_done, 0, sizeof(unsigned long long) * sv.cap);
    SCK(cudaHostGetDevicePointer((void**)&sv.d_done, sv.h_done, 0));
    SCK(cudaMallocHost((void**)&sv.h_stage, sizeof(int4) * sv.cap));
    SCK(cudaMallocHost((void**)&sv.h_cnt, sizeof(int) * kStreams));
    SCK(cudaMallocHost((void**)&sv.h_err, sizeof(int) * kStreams));
    SCK(cudaMallocHost((void**)&sv.h_apply, sizeof(ApplyRec) * std::max(1, c.A)));
    SCK(cudaMallocHost((void**)&sv.h_stash, sizeof(int2) * sv.cap));
    std::memset(sv.h_err, 0, sizeof(int) * kStreams);
    sv.info.assign(sv.cap, SlotInfo{});
    sv.state.assign(sv.cap, SLOT_FREE);
    sv.agent_sub.assign(std::max(1, c.A), 0u);
    sv.to_install.assign(std::max(1, c.A), 0);
    sv.target.assign(std::max(1, c.A), ApplyRec{});
    return GMAPF_OK;
}

void serve_free(Context& c) {
    if (!c.serve) return;
    Service& sv = *c.serve;
    for (int k = 0; k < kStreams; k++)
        if (sv.st[k]) cudaStreamSynchronize(sv.st[k]);
    if (sv.copy) cudaStreamSynchronize(sv.copy);
    if (sv.stash_stream) cudaStreamSynchronize(sv.stash_stream);
    for (void* p : sv.dallocs) cudaFree(p);
    void* hp[] = {sv.h_done, sv.h_stage, sv.h_cnt, sv.h_err, sv.h_apply, sv.h_stash};
    for (void* p : hp)
        if (p) cudaFreeHost(p);
    for (int k = 0; k < kStreams; k++) {
        if (sv.st_done[k]) cudaEventDestroy(sv.st_done[k]);
        if (sv.st[k]) cudaStreamDestroy(sv.st[k]);
    }
    for (cudaEvent_t e : {sv.copied, sv.stashed, sv.applied_ev})
        if (e) cudaEventDestroy(e);
    for (cudaStream_t st : {sv.copy, sv.stash_stream})
        if (st) cudaStreamDestroy(st);
    delete c.serve;
    c.serve = nullptr;
}

int serve_submit(Context& c, const int* ids, const gmapf_v2* pos, int n, const int64_t* arrival_ns,
                 std::string& err) {
    Service& sv = *c.serve;
    // validate everything first: a rejected call queues nothing
    std::vector<Waiting> batch(n);
    const long long now = now_ns();
    for (int k = 0; k < n; k++) {
        const int a = ids[k];
        if (a < 0 || a >= c.A) {
            err = "agent id " + std::to_string(a) + " out of range";
            return GMAPF_E_INVALID_ARG;
        }
        const LocateGrid g = scene_grid(c, c.is_world ? scene_of_agent(c, a) : 0);
        const int tnode = locate(g, pos[k].X, pos[k].Y);
        if (tnode < 0) {
            err = "target pos (" + std::to_string(pos[k].X) + ", " + std::to_string(pos[k].Y) + ") is invalid";
            return GMAPF_E_INVALID_POS;
        }
        // the start: the triangle under the agent now (its last known triangle
        // if the position lies in none)
        int start = locate(g, c.m_pos[a].X, c.m_pos[a].Y);
        if (start < 0) start = c.m_cur[a];
        batch[k] = Waiting{a, start, tnode, pos[k].X, pos[k].Y, arrival_ns ? (long long)arrival_ns[k] : now, 0};
    }
    for (Waiting& w : batch) {
        w.sub = ++sv.agent_sub[w.agent];
        sv.waiting.push_back(w);
    }
    sv.submitted += n;
    return admit_and_launch(c, sv, err);
}

int serve_poll(Context& c, std::string& err) {
    Service& sv = *c.serve;
    SCK(cudaSetDevice(c.dev.device));  // the context's GPU, whatever the caller's current one
    int rc = harvest(c, sv, err);
    if (rc) return rc;
    return admit_and_launch(c, sv, err);
}

// frame boundary: install the stashed results (on the frame's stream, before it)
int serve_before_frame(Context& c, cudaStream_t s, std::string& err) {
    Service& sv = *c.serve;
    int rc = serve_poll(c, err);
    if (rc) return rc;
    const int n = (int)sv.install.size();
    if (n == 0) return GMAPF_OK;
    for (int k = 0; k < n; k++) {
        const int a = sv.install[k];
        sv.h_apply[k] = sv.target[a];
        sv.to_install[a] = 0;
    }
    sv.install.clear();
    Device& d = c.dev;
    if (sv.stash_in_flight) SCK(cudaStreamWaitEvent(s, sv.stashed, 0));
    SCK(cudaMemcpyAsync(sv.d_apply, sv.h_apply, sizeof(ApplyRec) * n, cudaMemcpyHostToDevice, s));
    k_serve_apply<<<n, 128, 0, s>>>(sv.d_apply, n, sv.d_stash_fl, sv.d_stash_path, sv.stride, d.paths, d.state,
                                    d.step_idx, d.path_len, d.targ, d.targ_pos);
    SCK(cudaGetLastError());
    SCK(cudaEventRecord(sv.applied_ev, s));
    sv.apply_recorded = true;
    c.launches++;
    sv.applied += n;
    return GMAPF_OK;
}

// after the frame (nothing is held by a finished frame)
void serve_after_frame(Context& c) { (void)c; }

void serve_stats(Context& c, gmapf_serve_stats* out, bool reset) {
    Service& sv = *c.serve;
    std::memset(out, 0, sizeof(*out));
    out->submitted = sv.submitted;
    out->admitted = sv.tail;
    out->completed = sv.completed;
    out->found = sv.found;
    out->applied = sv.applied;
    out->superseded = sv.stale;
    out->waiting = (int64_t)sv.waiting.size();
    out->in_flight = sv.pending;
    out->launches = sv.launches;
    out->capacity = sv.cap;
    out->slots = sv.slots;
    std::vector<float> v = sv.lat_ms;
    if (!v.empty()) {
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) {
            size_t k = (size_t)std::ceil(q / 100.0 * v.size());
            if (k > 0) k--;
            return v[std::min(k, v.size() - 1)];
        };
        double s = 0;
        for (float x : v) s += x;
        out->latency_p50_ms = pct(50);
        out->latency_p99_ms = pct(99);
        out->latency_mean_ms = (float)(s / v.size());
        out->latency_max_ms = v.back();
        out->latency_samples = (int64_t)v.size();
    }
    if (reset) {
        sv.lat_ms.clear();
        sv.submitted = sv.completed = sv.found = sv.applied = sv.stale = sv.launches = 0;
    }
}

int serve_drain(Context& c, double timeout_s, std::string& err) {
    Service& sv = *c.serve;
    const long long t_end = now_ns() + (long long)(timeout_s * 1e9);
    while (sv.pending > 0 || !sv.waiting.empty()) {
        int rc = serve_poll(c, err);
        if (rc) return rc;
        if (now_ns() > t_end) {
            err = "serving: queries still pending after the drain timeout";
            return GMAPF_E_DEVICE_TIMEOUT;
        }
    }
    return GMAPF_OK;
}

int serve_result(Context& c, int agent, int* found, int* len, int* path, int cap, std::string& err) {
    // the agent's stashed result, not yet installed by a frame
    Service& sv = *c.serve;
    SCK(cudaSetDevice(c.dev.device));
    if (!sv.to_install[agent]) {
        err = "no finished, uninstalled query for this agent";
        return GMAPF_E_STATE;
    }
    SCK(cudaEventSynchronize(sv.stashed));
    int2 fl;
    SCK(cudaMemcpy(&fl, sv.d_stash_fl + agent, sizeof(int2), cudaMemcpyDeviceToHost));
    *found = fl.x;
    *len = fl.y;
    const int L = std::min(fl.y, cap);
    if (fl.x && L > 0)
        SCK(cudaMemcpy(path, sv.d_stash_path + (long long)agent * sv.stride, sizeof(int) * L, cudaMemcpyDeviceToHost));
    return GMAPF_OK;
}

}  // namespace gmapf_b200
