// device.cu -- device state and per-frame orchestration.
//
// Reference orchestration: src/GMAPF.cu:72-130 (ManualStart), :255-289
// (AsyncStep), :291-314 (WaitStepEnd); PathFinder.h:354-409 / AgentsMover.h
// :211-252 (module init); PathFinder.h:508-598 / AgentsMover.h:345-424 (phase
// launches).  The reference reads the request and mover counts back to the
// host in the middle of every frame and copies the whole 64-byte-per-agent
// array both ways synchronously.  Here:
//   - agents live on the device as structure-of-arrays; SetAgentTargPos
//     uploads only the changed agents (16 bytes each) before the frame;
//   - batched form: the frame (compaction, persistent search on one stream,
//     mover on a second stream, D2H of positions and states) is one CUDA
//     graph; counts stay on the device;
//   - plain form: the same kernels launched one by one with the reference's
//     host read-back of the counts and one static search launch per chunk
//     of requests.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "internal.h"

namespace gmapf_b200 {

#define CK(x)                                                                        \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            err = std::string(#x) + " failed: " + cudaGetErrorString(e_);            \
            return GMAPF_E_CUDA;                                                     \
        }                                                                            \
    } while (0)

// "device-side check failed: ..." with the names of the error bits set
std::string device_error_text(int e) {
    std::string s = "device-side check failed:";
    if (e & ERR_ROUNDS) s += " a search reached the round limit;";
    if (e & ERR_PATH_CAP) s += " a path did not fit its output row;";
    if (e & ERR_BAD_REQUEST) s += " a request named a triangle outside the map;";
    if (e & ERR_BOUNDS) s += " an index failed its bounds check;";
    return s + " (error bits " + std::to_string(e) + ")";
}

int search_round_limit(const Context& c) {
    return c.opt.round_limit > 0 ? c.opt.round_limit : 4 * c.map.n + 64;
}

int search_promote_rounds(const Context& c) { return c.opt.promote_rounds > 0 ? c.opt.promote_rounds : 512; }

namespace {

// device counters: [8] holds the frame's dt as a float
enum Counter { CT_REQ = 0, CT_MOVE = 1, CT_WORK = 2, CT_ERR = 3, CT_ERR_TARGETS = 4, CT_COUNT = 16 };

template <class T>
int dalloc(Context& c, T** p, size_t count, std::string& err) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) {
        err = std::string("cudaMalloc of ") + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e);
        cudaGetLastError();
        *p = nullptr;
        return e == cudaErrorMemoryAllocation ? GMAPF_E_CAPACITY : GMAPF_E_CUDA;
    }
    c.dev.allocs.push_back((void*)*p);
    // cudaMemset runs on the legacy stream, which the library's non-blocking
    // streams do not wait for: finish it before any kernel can touch the buffer
    e = cudaMemset(*p, 0, bytes);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        err = std::string("cudaMemset failed: ") + cudaGetErrorString(e);
        return GMAPF_E_CUDA;
    }
    return GMAPF_OK;
}

#define DALLOC(ptr, count)                                \
    do {                                                  \
        int rc_ = dalloc(c, &(ptr), (count), err);        \
        if (rc_ != GMAPF_OK) return rc_;                  \
    } while (0)

SearchParams search_params(Context& c) {
    Device& d = c.dev;
    SearchParams p{};
    p.rows = d.rows;
    p.cen = d.cen;
    p.n = c.map.n;
    p.req = d.req;
    p.req_count_d = d.counters + CT_REQ;
    p.req_count_h = 0;
    p.T = c.T;
    p.C = c.C;
    p.K = c.K;
    p.rec = d.rec;
    p.epoch = d.epoch;
    p.slots = d.slots;
    p.gbm = d.gbm;
    p.work_ctr = d.counters + CT_WORK;
    p.max_rounds = search_round_limit(c);
    p.promote_rounds = search_promote_rounds(c);
    p.paths = d.paths;
    p.path_stride = d.path_stride;
    p.ag_state = d.state;
    p.ag_step_idx = d.step_idx;
    p.ag_path_len = d.path_len;
    p.stats = d.stats;
    p.err = d.counters + CT_ERR;
    return p;
}

// The scene table of a plain context: its one map and all its agents.
SceneInfo single_scene(const Context& c) {
    const HostMap& m = c.map;
    SceneInfo si;
    si.node_base = 0;
    si.n = m.n;
    si.agent_base = 0;
    si.A = c.A;
    si.P = c.cfg.PathFinderParallelAgents;
    si.radius = c.cfg.AgentRadius;
    si.speed = c.cfg.AgentSpeed;
    si.bx0 = m.bx0;
    si.by0 = m.by0;
    si.bx1 = m.bx1;
    si.by1 = m.by1;
    si.gx0 = m.gx0;
    si.gy0 = m.gy0;
    si.ginv = m.ginv;
    si.gw = m.gw;
    si.gh = m.gh;
    si.ndegen = (int)m.degen.size();
    return si;
}

// Mover constants of one scene (AgentsMover.h:162,222-224) and its agent grid:
// cells at least 1.0625 collision distances wide and about one agent per
// cell (a scan over the cells is part of every moving frame; the collision
// pass reads the 3x3 cells around each agent, so the cell size changes only
// which agents are read, never the result), at most 2048 per axis; cell ids
// continue from cell_base.
ScenePar scene_par(const Device& d, const SceneInfo& si, int cell_base) {
    ScenePar p{};
    p.cd = si.radius * 2.5f;
    p.cd2 = p.cd * p.cd;
    p.arrive = FLT_EPSILON + si.radius;
    p.speed = si.speed;
    p.clear = d.clearance ? si.radius : 0.f;
    const double w = std::max(1e-3, (double)si.bx1 - si.bx0), h = std::max(1e-3, (double)si.by1 - si.by0);
    double cell = std::max((double)p.cd * 1.0625, 1e-4);
    cell = std::max(cell, std::sqrt(w * h / std::max(1.0, (double)si.A)));
    cell = std::max(cell, std::max(w, h) / 2048.0);
    p.ax0 = si.bx0;
    p.ay0 = si.by0;
    p.ainv = (float)(1.0 / cell);
    p.aw = std::max(1, (int)std::ceil(w / cell) + 1);
    p.ah = std::max(1, (int)std::ceil(h / cell) + 1);
    p.cell_base = cell_base;
    p.loc.x0 = si.gx0;
    p.loc.y0 = si.gy0;
    p.loc.inv = si.ginv;
    p.loc.w = si.gw;
    p.loc.h = si.gh;
    p.loc.start = d.gstart + si.gstart_off;
    p.loc.list = d.glist + si.glist_off;
    p.loc.degen = d.degen + si.degen_off;
    p.loc.ndegen = si.ndegen;
    p.loc.tri = d.tri + 3 * (size_t)si.node_base;
    p.loc.n = si.n;
    p.loc.base = si.node_base;
    return p;
}

MoverParams mover_params(Context& c) {
    Device& d = c.dev;
    MoverParams p{};
    p.A = c.A;
    p.mv_count = d.counters + CT_MOVE;
    p.in_move = d.in_move;
    p.pos = d.pos;
    p.pos_mid = d.pos_mid;
    p.step_pos = d.step_pos;
    p.targ_pos = d.targ_pos;
    p.state = d.state;
    p.cur_node = d.cur;
    p.step_idx = d.step_idx;
    p.step_node = d.step_node;
    p.path_len = d.path_len;
    p.paths = d.paths;
    p.path_stride = d.path_stride;
    p.dt = reinterpret_cast<const float*>(d.counters + 8);
    // V2Float::GetRotated(10): cos/sin of 10 degrees, taken in double, rounded to float
    const double ang = 10.0 * 3.14159265358979323846 / 180.0;
    p.cs = (float)std::cos(ang);
    p.sn = (float)std::sin(ang);
    p.sc = d.scene_par;
    p.agent_scene = d.agent_scene;
    p.cells = d.cells;
    p.cell_of = d.cell_of;
    p.cell_cnt = d.cell_cnt;
    p.cell_start = d.cell_start;
    p.cell_fill = d.cell_fill;
    p.cell_items = d.cell_items;
    p.tri = d.tri;
    p.cen = d.cen;
    p.waypoints = d.waypoints;
    p.n = c.map.n;
    p.stats = d.stats;
    p.err = d.counters + CT_ERR;
    return p;
}

CompactScenes compact_scenes(const Context& c) {
    const Device& d = c.dev;
    return CompactScenes{d.agent_scene, d.scene_abase, d.scene_P, d.scene_first};
}

int pick_slots(Context& c, int& blocks, std::string& err) {
    Device& d = c.dev;
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.device));
    size_t freeb = 0, totalb = 0;
    CK(cudaMemGetInfo(&freeb, &totalb));
    // the search state this context already holds counts as free: a reshape
    // reuses or replaces it
    freeb += (size_t)d.rec_cap * (sizeof(Rec) * std::max(1, c.map.n) + sizeof(unsigned)) +
             (size_t)d.gbm_cap * 4 * (size_t)d.bm_words;
    long long budget = c.opt.search_mem_budget > 0 ? c.opt.search_mem_budget : (40ll << 30);
    budget = std::min<long long>(budget, (long long)(freeb * 0.6));
    const long long per_slot = (long long)std::max(1, c.map.n) * (long long)sizeof(Rec);
    d.bm_words = search_bitmap_words(std::max(1, c.map.n));

    // Candidates: visited placement (1 shared-memory bitmap, 2 stamped
    // records, 3 global bitmap, 4 global bitmap that a search at a batch's
    // tail moves into its block's shared memory) and block size.  The
    // score is the number of resident slots weighted by how close the claim
    // check is: on chip x4, L2 x3, DRAM x2 (the record check misses L2 in
    // every round); placement 4 wins a tie with placement 3 (a frame's tail
    // then checks on chip).
    long long best_score = -1;
    int best_bt = 0;
    int best_vm = 2;
    long long best_slots = 0;
    const int want_vm = c.opt.visited_mode ? c.opt.visited_mode : c.tuned_vm;
    const int want_bt = c.opt.block_threads ? c.opt.block_threads : c.tuned_bt;
    for (int vm = 1; vm <= 4; vm++) {
        if (want_vm != 0 && want_vm != vm) continue;
        const long long mem_slots = budget / (per_slot + (vm >= 3 ? 4ll * d.bm_words : 0));
        // the first of equal scores wins; placement 4 prefers 256-thread blocks
        // (measured faster than 128 on the 160x160 maze: 27.1 against 28.0 ms
        // for a frame batch)
        const int bts3[4] = {128, 64, 32, 256}, bts4[4] = {256, 128, 64, 32};
        for (int bt : (vm == 4 ? bts4 : bts3)) {
            if (want_bt != 0 && bt != want_bt) continue;
            if (bt % c.T) continue;
            const int per_sm = search_max_blocks_per_sm(c.T, c.C, bt, vm, d.bm_words);
            if (per_sm <= 0) continue;
            const int gpb = bt / 32;  // one request slot per warp
            long long slots = std::min((long long)sms * per_sm * gpb, mem_slots);
            slots = (slots / gpb) * gpb;
            if (slots < gpb) continue;
            const long long score = slots * (vm == 1 ? 4 : vm >= 3 ? 3 : 2) + (vm == 4 ? 1 : 0);
            if (score > best_score) {
                best_score = score;
                best_bt = bt;
                best_vm = vm;
                best_slots = slots;
            }
        }
    }
    if (best_score < 0) {
        err = "search kernel cannot be resident with T=" + std::to_string(c.T) + " C=" +
              std::to_string(c.C) + " (shared memory or device memory too small)";
        return GMAPF_E_CAPACITY;
    }
    c.block_threads = best_bt;
    d.vm = best_vm;
    d.slots = (int)best_slots;
    blocks = (int)(best_slots / (best_bt / 32));
    // leave the kernel's shared-memory limit set for the chosen shape
    search_max_blocks_per_sm(c.T, c.C, best_bt, best_vm, d.bm_words);
    return GMAPF_OK;
}

void release(Context& c, void* p) {
    if (!p) return;
    Device& d = c.dev;
    d.allocs.erase(std::remove(d.allocs.begin(), d.allocs.end(), p), d.allocs.end());
    cudaFree(p);
}

// Search state for the shape in c (T, C, visited placement, block size).
// The record and bitmap arrays are kept while the new shape's slots fit
// them (the autotuner reshapes a hundred times; a ~12 GB free, allocation
// and clear each time would take seconds).  Reuse needs no clearing: slot s
// keeps its records together with its query epoch, so an old stamp never
// equals a new epoch (modes 1 and 3 stamp 0, which no mode-2 epoch is), and
// the bitmaps are cleared at the start of every query.
int alloc_search_state(Context& c, std::string& err) {
    Device& d = c.dev;
    int blocks = 0;
    int rc = pick_slots(c, blocks, err);
    if (rc) return rc;
    if (!d.rec || d.slots > d.rec_cap) {
        release(c, d.rec);
        release(c, d.epoch);
        d.rec = nullptr;
        d.epoch = nullptr;
        d.rec_cap = 0;
        DALLOC(d.rec, (size_t)d.slots * std::max(1, c.map.n));
        DALLOC(d.epoch, (size_t)d.slots);
        d.rec_cap = d.slots;
    }
    if (d.vm >= 3 && (!d.gbm || d.slots > d.gbm_cap)) {
        release(c, d.gbm);
        d.gbm = nullptr;
        d.gbm_cap = 0;
        DALLOC(d.gbm, (size_t)d.slots * d.bm_words);
        d.gbm_cap = d.slots;
    }
    return GMAPF_OK;
}

int search_blocks(Context& c) { return c.dev.slots / (c.block_threads / 32); }

void destroy_graph(Context& c) {
    if (c.dev.graph_exec) cudaGraphExecDestroy(c.dev.graph_exec);
    if (c.dev.graph) cudaGraphDestroy(c.dev.graph);
    c.dev.graph_exec = nullptr;
    c.dev.graph = nullptr;
}

// kernels of one frame on the two streams (batched form: captured)
int enqueue_frame(Context& c, bool timing, std::string& err) {
    Device& d = c.dev;
    cudaStream_t s = d.stream, s2 = d.stream2;
    if (timing) CK(cudaEventRecordWithFlags(d.ev[0], s, cudaEventRecordExternal));
    CK(cudaMemsetAsync(d.counters + CT_ERR, 0, sizeof(int), s));
    launch_compact(s, c.A, d.state, d.cur, d.targ, c.cfg.PathFinderParallelAgents, compact_scenes(c), d.req,
                   d.counters + CT_REQ, d.in_move, d.counters + CT_MOVE, d.counters + CT_WORK, d.stats);
    if (timing) CK(cudaEventRecordWithFlags(d.ev[1], s, cudaEventRecordExternal));
    CK(cudaEventRecord(d.ev[5], s));
    CK(cudaStreamWaitEvent(s2, d.ev[5], 0));
    // search branch (requests longest-first when the landmark estimate is on)
    SearchParams sp = search_params(c);
    if (d.lm) {
        launch_order_requests(s, d.req, d.counters + CT_REQ, d.req_sorted, d.req_keys, d.lm, d.lm_count, c.map.n);
        sp.req = d.req_sorted;
    }
    CK(launch_search(s, sp, search_blocks(c), c.block_threads, true, 0, d.vm, d.bm_words));
    if (timing) CK(cudaEventRecordWithFlags(d.ev[2], s, cudaEventRecordExternal));
    // mover branch
    MoverParams mp = mover_params(c);
    if (c.A > 0) {
        CK(cudaMemsetAsync(d.cell_cnt, 0, sizeof(int) * (d.cells + 1), s2));
        launch_funnel(s2, mp);  // path smoothing only
        launch_move_bin(s2, mp);
        launch_cell_scan(s2, mp);
        launch_scatter(s2, mp);
        launch_collide_progress(s2, mp);
    }
    if (timing) CK(cudaEventRecordWithFlags(d.ev[3], s2, cudaEventRecordExternal));
    CK(cudaEventRecord(d.ev[6], s2));
    CK(cudaStreamWaitEvent(s, d.ev[6], 0));
    if (c.A > 0) {
        CK(cudaMemcpyAsync(c.h_pos_stage, d.pos, sizeof(float2) * c.A, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(c.h_state_stage, d.state, sizeof(int) * c.A, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaMemcpyAsync(c.h_small, d.counters, sizeof(int) * CT_COUNT, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(c.h_stats, d.stats, sizeof(unsigned long long) * ST_COUNT, cudaMemcpyDeviceToHost, s));
    if (timing) CK(cudaEventRecordWithFlags(d.ev[4], s, cudaEventRecordExternal));
    return GMAPF_OK;
}

int capture_graph(Context& c, std::string& err) {
    Device& d = c.dev;
    destroy_graph(c);
    CK(cudaStreamBeginCapture(d.stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_frame(c, c.cfg.IsProfiler != 0, err);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(d.stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) {
        err = std::string("graph capture failed: ") + cudaGetErrorString(e);
        return GMAPF_E_CUDA;
    }
    d.graph = g;
    CK(cudaGraphInstantiate(&d.graph_exec, g, 0));
    return GMAPF_OK;
}

int kernels_per_frame(Context& c) {
    return 2 + (c.dev.lm ? 1 : 0) + (c.A > 0 ? 4 + (c.dev.waypoints ? 1 : 0) : 0);
}

}  // namespace

int device_start(Context& c, std::string& err) {
    Device& d = c.dev;
    d.device = c.opt.device;
    CK(cudaSetDevice(d.device));
    CK(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&d.stream2, cudaStreamNonBlocking));
    for (auto& e : d.ev) CK(cudaEventCreate(&e));
    CK(cudaEventCreateWithFlags(&d.frame_done, cudaEventDisableTiming));

    const HostMap& m = c.map;
    const int n = m.n;
    if (c.scenes.empty()) c.scenes.push_back(single_scene(c));
    const int nsc = (int)c.scenes.size();
    int max_scene_n = 1;
    for (const SceneInfo& si : c.scenes) max_scene_n = std::max(max_scene_n, si.n);
    // map
    DALLOC(d.rows, n);
    DALLOC(d.cen, n);
    DALLOC(d.tri, 3 * (size_t)n);
    DALLOC(d.gstart, m.gstart.size());
    DALLOC(d.glist, m.glist.size());
    DALLOC(d.degen, m.degen.size());
    CK(cudaMemcpy(d.rows, m.rows.data(), sizeof(SearchRow) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.cen, m.cen.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.tri, m.tri.data(), sizeof(float2) * 3 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.gstart, m.gstart.data(), sizeof(int) * m.gstart.size(), cudaMemcpyHostToDevice));
    if (!m.glist.empty())
        CK(cudaMemcpy(d.glist, m.glist.data(), sizeof(int) * m.glist.size(), cudaMemcpyHostToDevice));
    if (!m.degen.empty())
        CK(cudaMemcpy(d.degen, m.degen.data(), sizeof(int) * m.degen.size(), cudaMemcpyHostToDevice));

    // agents
    const int A = c.A;
    DALLOC(d.pos, A);
    DALLOC(d.pos_mid, A);
    DALLOC(d.targ_pos, A);
    DALLOC(d.step_pos, A);
    DALLOC(d.state, A);
    DALLOC(d.cur, A);
    DALLOC(d.targ, A);
    DALLOC(d.step_idx, A);
    DALLOC(d.step_node, A);
    DALLOC(d.path_len, A);
    DALLOC(d.in_move, A);
    DALLOC(d.dirty, A);
    d.dirty_cap = A;
    d.path_stride = max_scene_n;  // a path holds at most its scene's triangles
    {
        size_t freeb = 0, totalb = 0;
        CK(cudaMemGetInfo(&freeb, &totalb));
        double need = (double)std::max(1, A) * d.path_stride * sizeof(int);
        if (need > 0.45 * (double)freeb) {
            err = "path buffers (agents x triangles x 4 bytes = " + std::to_string((long long)need) +
                  " bytes) exceed the device memory budget";
            return GMAPF_E_CAPACITY;
        }
    }
    DALLOC(d.paths, (size_t)std::max(1, A) * d.path_stride);
    d.clearance = c.opt.path_smoothing == 2;
    if (c.opt.path_smoothing) {
        size_t freeb = 0, totalb = 0;
        CK(cudaMemGetInfo(&freeb, &totalb));
        const double need = (double)std::max(1, A) * d.path_stride * sizeof(float2);
        if (need > 0.45 * (double)freeb) {
            err = "path smoothing: steering points (agents x triangles x 8 bytes) exceed the device memory budget";
            return GMAPF_E_CAPACITY;
        }
        DALLOC(d.waypoints, (size_t)std::max(1, A) * d.path_stride);
    }
    DALLOC(d.req, std::max(1, c.cfg.PathFinderParallelAgents));
    DALLOC(d.counters, CT_COUNT);
    if (c.opt.order_by_estimate && c.opt.mode == GMAPF_MODE_BATCHED && n > 0 && nsc == 1) {
        // landmark hop distances for the longest-first request order
        std::vector<unsigned short> lm;
        d.lm_count = 8;
        landmark_distances(m, d.lm_count, lm);
        DALLOC(d.lm, lm.size());
        CK(cudaMemcpy(d.lm, lm.data(), sizeof(unsigned short) * lm.size(), cudaMemcpyHostToDevice));
        DALLOC(d.req_sorted, std::max(1, c.cfg.PathFinderParallelAgents));
        DALLOC(d.req_keys, std::max(1, c.cfg.PathFinderParallelAgents));
    }
    DALLOC(d.stats, ST_COUNT);

    std::vector<float2> tp(A);
    std::vector<int> minus(A, -1);
    for (int i = 0; i < A; i++) tp[i] = make_float2(c.m_targ[i].X, c.m_targ[i].Y);
    if (A > 0) {
        CK(cudaMemcpy(d.pos, c.m_pos.data(), sizeof(float2) * A, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.state, c.m_state.data(), sizeof(int) * A, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.cur, c.m_cur.data(), sizeof(int) * A, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.targ, c.m_targ_node.data(), sizeof(int) * A, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.targ_pos, tp.data(), sizeof(float2) * A, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.step_idx, minus.data(), sizeof(int) * A, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.step_node, minus.data(), sizeof(int) * A, cudaMemcpyHostToDevice));
    }

    // scene table and agent grid
    c.scene_par.clear();
    d.cells = 0;
    for (const SceneInfo& si : c.scenes) {
        c.scene_par.push_back(scene_par(d, si, d.cells));
        d.cells += c.scene_par.back().aw * c.scene_par.back().ah;
    }
    DALLOC(d.scene_par, nsc);
    CK(cudaMemcpy(d.scene_par, c.scene_par.data(), sizeof(ScenePar) * nsc, cudaMemcpyHostToDevice));
    if (nsc > 1) {
        std::vector<int> as(std::max(1, A), 0), ab(nsc + 1, 0), sp(nsc, 0);
        for (int s = 0; s < nsc; s++) {
            const SceneInfo& si = c.scenes[s];
            for (int i = 0; i < si.A; i++) as[si.agent_base + i] = s;
            ab[s] = si.agent_base;
            sp[s] = si.P;
        }
        ab[nsc] = A;
        DALLOC(d.agent_scene, std::max(1, A));
        DALLOC(d.scene_abase, nsc + 1);
        DALLOC(d.scene_P, nsc);
        DALLOC(d.scene_first, nsc);
        CK(cudaMemcpy(d.agent_scene, as.data(), sizeof(int) * as.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.scene_abase, ab.data(), sizeof(int) * ab.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.scene_P, sp.data(), sizeof(int) * sp.size(), cudaMemcpyHostToDevice));
    }
    DALLOC(d.cell_of, A);
    DALLOC(d.cell_cnt, (size_t)d.cells + 1);
    DALLOC(d.cell_start, (size_t)d.cells + 1);
    DALLOC(d.cell_fill, (size_t)d.cells + 1);
    DALLOC(d.cell_items, A);

    // pinned host staging
    CK(cudaMallocHost((void**)&c.h_pos_stage, sizeof(float2) * std::max(1, A)));
    CK(cudaMallocHost((void**)&c.h_state_stage, sizeof(int) * std::max(1, A)));
    CK(cudaMallocHost((void**)&c.h_dirty, sizeof(int4) * std::max(1, A)));
    CK(cudaMallocHost((void**)&c.h_small, sizeof(int) * CT_COUNT));
    CK(cudaMallocHost((void**)&c.h_stats, sizeof(unsigned long long) * ST_COUNT));
    CK(cudaMallocHost((void**)&c.h_step, sizeof(float) * 4));
    std::memset(c.h_stats, 0, sizeof(unsigned long long) * ST_COUNT);

    int rc = alloc_search_state(c, err);
    if (rc) return rc;
    CK(cudaDeviceSynchronize());
    return GMAPF_OK;
}

void device_free(Context& c) {
    Device& d = c.dev;
    if (d.stream && cudaSetDevice(d.device) != cudaSuccess) cudaGetLastError();
    serve_free(c);
    if (d.stream) cudaStreamSynchronize(d.stream);
    if (d.stream2) cudaStreamSynchronize(d.stream2);
    destroy_graph(c);
    for (void* p : d.allocs)
        if (p) cudaFree(p);
    d.allocs.clear();
    d.rec = nullptr;  // freed above: a later start allocates anew
    d.epoch = nullptr;
    d.gbm = nullptr;
    d.rec_cap = d.gbm_cap = 0;
    d.slots = 0;
    for (auto& e : d.ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    if (d.frame_done) cudaEventDestroy(d.frame_done);
    d.frame_done = nullptr;
    if (d.stream) cudaStreamDestroy(d.stream);
    if (d.stream2) cudaStreamDestroy(d.stream2);
    d.stream = d.stream2 = nullptr;
    if (d.loc_stream) cudaStreamSynchronize(d.loc_stream), cudaStreamDestroy(d.loc_stream);
    if (d.loc_pts) cudaFree(d.loc_pts);
    if (d.loc_node) cudaFree(d.loc_node);
    if (d.h_loc_pts) cudaFreeHost(d.h_loc_pts);
    if (d.h_loc_node) cudaFreeHost(d.h_loc_node);
    d.loc_stream = nullptr;
    d.loc_pts = nullptr;
    d.loc_node = nullptr;
    d.h_loc_pts = nullptr;
    d.h_loc_node = nullptr;
    d.loc_cap = 0;
    void* hp[] = {c.h_pos_stage, c.h_state_stage, c.h_dirty, c.h_small, c.h_stats, c.h_step};
    for (void* p : hp)
        if (p) cudaFreeHost(p);
    c.h_pos_stage = nullptr;
    c.h_state_stage = nullptr;
    c.h_dirty = nullptr;
    c.h_small = nullptr;
    c.h_stats = nullptr;
    c.h_step = nullptr;
}

int device_async_step(Context& c, float dt, std::string& err) {
    Device& d = c.dev;
    cudaStream_t s = d.stream;
    CK(cudaSetDevice(d.device));
    c.t_step0 = std::chrono::steady_clock::now();
    // changed targets (src/GMAPF.cu:270-278 copies the whole agent array)
    const int nd = (int)c.dirty_recs.size();
    c.pre_done = nd > 0;
    if (nd > 0) {
        std::memcpy(c.h_dirty, c.dirty_recs.data(), sizeof(int4) * nd);
        CK(cudaMemcpyAsync(d.dirty, c.h_dirty, sizeof(int4) * nd, cudaMemcpyHostToDevice, s));
        launch_apply_targets(s, d.dirty, nd, d.state, d.targ, d.targ_pos);
        c.launches += 1;
        for (const int4& r : c.dirty_recs) c.dirty_slot[r.x] = -1;
        c.dirty_recs.clear();
    }
    if (c.serve) {  // serving: finished queries join this frame
        int rc = serve_before_frame(c, s, err);
        if (rc) return rc;
    }
    c.h_step[0] = dt;  // each scene's step is speed * dt, rounded once (AgentsMover.h:63)
    CK(cudaMemcpyAsync(d.counters + 8, c.h_step, sizeof(float), cudaMemcpyHostToDevice, s));

    if (c.opt.mode == GMAPF_MODE_BATCHED) {
        if (!d.graph_exec) {
            int rc = capture_graph(c, err);
            if (rc) return rc;
        }
        CK(cudaGraphLaunch(d.graph_exec, s));
        c.launches += kernels_per_frame(c);
    } else {
        // plain: the reference's shape -- counts read back mid-frame
        const bool timing = c.cfg.IsProfiler != 0;
        if (timing) CK(cudaEventRecord(d.ev[0], s));
        CK(cudaMemsetAsync(d.counters + CT_ERR, 0, sizeof(int), s));
        launch_compact(s, c.A, d.state, d.cur, d.targ, c.cfg.PathFinderParallelAgents, compact_scenes(c), d.req,
                       d.counters + CT_REQ, d.in_move, d.counters + CT_MOVE, d.counters + CT_WORK,
                       d.stats);
        c.launches += 1;
        CK(cudaMemcpyAsync(c.h_small, d.counters, sizeof(int) * CT_COUNT, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (timing) CK(cudaEventRecord(d.ev[1], s));
        const int R = c.h_small[CT_REQ], M = c.h_small[CT_MOVE];
        c.plain_req_count = R;
        c.plain_mv_count = M;
        if (R > 0) {
            SearchParams sp = search_params(c);
            sp.req_count_h = R;
            const int chunk = d.slots;
            for (int base = 0; base < R; base += chunk) {
                const int cnt = std::min(chunk, R - base);
                const int gpb = c.block_threads / 32;
                const int blocks = (cnt + gpb - 1) / gpb;
                CK(launch_search(s, sp, blocks, c.block_threads, false, base, d.vm, d.bm_words));
                c.launches += 1;
            }
        }
        if (timing) CK(cudaEventRecord(d.ev[2], s));
        if (M > 0) {
            MoverParams mp = mover_params(c);
            CK(cudaMemsetAsync(d.cell_cnt, 0, sizeof(int) * (d.cells + 1), s));
            launch_funnel(s, mp);  // path smoothing only
            launch_move_bin(s, mp);
            launch_cell_scan(s, mp);
            launch_scatter(s, mp);
            launch_collide_progress(s, mp);
            c.launches += 4 + (d.waypoints ? 1 : 0);
        }
        if (timing) CK(cudaEventRecord(d.ev[3], s));
        if (c.A > 0) {
            CK(cudaMemcpyAsync(c.h_pos_stage, d.pos, sizeof(float2) * c.A, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(c.h_state_stage, d.state, sizeof(int) * c.A, cudaMemcpyDeviceToHost, s));
        }
        CK(cudaMemcpyAsync(c.h_small, d.counters, sizeof(int) * CT_COUNT, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(c.h_stats, d.stats, sizeof(unsigned long long) * ST_COUNT, cudaMemcpyDeviceToHost, s));
        if (timing) CK(cudaEventRecord(d.ev[4], s));
    }
    CK(cudaEventRecord(d.frame_done, s));
    return GMAPF_OK;
}

bool device_step_ready(Context& c) {
    const cudaError_t e = cudaEventQuery(c.dev.frame_done);
    if (e == cudaErrorNotReady) return false;
    cudaGetLastError();
    return true;  // finished, or failed: WaitStepEnd reports it
}

int device_wait_step(Context& c, std::string& err) {
    Device& d = c.dev;
    CK(cudaSetDevice(d.device));
    CK(cudaStreamSynchronize(d.stream));
    if (c.serve) serve_after_frame(c);
    const auto t1 = std::chrono::steady_clock::now();
    if (c.A > 0) {
        for (int i = 0; i < c.A; i++) {
            c.m_pos[i].X = c.h_pos_stage[i].x;
            c.m_pos[i].Y = c.h_pos_stage[i].y;
        }
        std::memcpy(c.m_state.data(), c.h_state_stage, sizeof(int) * c.A);
    }
    const auto t2 = std::chrono::steady_clock::now();
    unsigned long long delta[ST_COUNT];
    for (int k = 0; k < ST_COUNT; k++) {
        delta[k] = c.h_stats[k] - c.stats_prev[k];
        c.stats_prev[k] = c.h_stats[k];
    }
    gmapf_step_stats& st = c.last;
    st.requests = (int64_t)delta[ST_REQUESTS];
    st.found = (int64_t)delta[ST_FOUND];
    st.expansions = (int64_t)delta[ST_EXPANSIONS];
    st.rounds = (int64_t)delta[ST_ROUNDS];
    st.deg_sum = (int64_t)delta[ST_DEG_SUM];
    st.claims = (int64_t)delta[ST_CLAIMS];
    st.path_nodes = (int64_t)delta[ST_PATH_NODES];
    st.moving = (int64_t)delta[ST_MOVING];
    st.neighbours = (int64_t)delta[ST_NEIGHBOURS];
    st.promoted = (int64_t)delta[ST_PROMOTED];
    st.ms_step_wall = std::chrono::duration<float, std::milli>(t2 - c.t_step0).count();
    st.ms_search = st.ms_mover = st.ms_total_device = 0;
    if (c.cfg.IsProfiler) {
        float a = 0, b = 0, t = 0, cp = 0;
        cudaEventElapsedTime(&cp, d.ev[0], d.ev[1]);
        cudaEventElapsedTime(&a, d.ev[1], d.ev[2]);
        cudaEventElapsedTime(&b, d.ev[c.opt.mode == GMAPF_MODE_BATCHED ? 1 : 2], d.ev[3]);
        cudaEventElapsedTime(&t, d.ev[0], d.ev[4]);
        cudaGetLastError();
        st.ms_search = a;
        st.ms_mover = b;
        st.ms_total_device = t;
        Profiler& p = c.prof;
        p.n++;
        p.sum_wall += st.ms_step_wall;
        p.max_wall = std::max(p.max_wall, st.ms_step_wall);
        p.sum_compact += cp;
        p.max_compact = std::max(p.max_compact, cp);
        if (st.requests > 0) {
            p.n_search++;
            p.sum_search += a;
            p.max_search = std::max(p.max_search, a);
        }
        if (st.moving > 0) {
            p.n_mover++;
            p.sum_mover += b;
            p.max_mover = std::max(p.max_mover, b);
        }
        const float post = std::chrono::duration<float, std::milli>(t2 - t1).count();
        p.sum_post += post;
        p.max_post = std::max(p.max_post, post);
    }
    c.prof.wall_ms.push_back(st.ms_step_wall);
    const int e = c.h_small[CT_ERR];
    const int et = c.h_small[CT_ERR_TARGETS];
    if (et != 0) {  // from device-resident retargets enqueued before this step
        CK(cudaMemsetAsync(d.counters + CT_ERR_TARGETS, 0, sizeof(int), d.stream));
        CK(cudaStreamSynchronize(d.stream));
        err = "device-resident retarget rejected (agent id out of range or position in no triangle)";
        return GMAPF_E_DEVICE;
    }
    if (e != 0) {
        err = device_error_text(e);
        return GMAPF_E_DEVICE;
    }
    return GMAPF_OK;
}

int device_locate_points(Context& c, const gmapf_v2* pts, int n, int* node, std::string& err) {
    Device& d = c.dev;
    if (n <= 0) return GMAPF_OK;
    if (c.scene_par.size() != 1) {
        err = "device point location needs a single-map context";
        return GMAPF_E_STATE;
    }
    CK(cudaSetDevice(d.device));
    if (!d.loc_stream) CK(cudaStreamCreateWithFlags(&d.loc_stream, cudaStreamNonBlocking));
    if (n > d.loc_cap) {
        cudaFree(d.loc_pts);
        cudaFree(d.loc_node);
        cudaFreeHost(d.h_loc_pts);
        cudaFreeHost(d.h_loc_node);
        d.loc_pts = nullptr;
        d.loc_node = nullptr;
        d.h_loc_pts = nullptr;
        d.h_loc_node = nullptr;
        d.loc_cap = 0;
        const int cap = std::max(n, 4096);
        CK(cudaMalloc(&d.loc_pts, sizeof(float2) * cap));
        CK(cudaMalloc(&d.loc_node, sizeof(int) * cap));
        CK(cudaHostAlloc(&d.h_loc_pts, sizeof(float2) * cap, cudaHostAllocDefault));
        CK(cudaHostAlloc(&d.h_loc_node, sizeof(int) * cap, cudaHostAllocDefault));
        d.loc_cap = cap;
    }
    static_assert(sizeof(gmapf_v2) == sizeof(float2), "point layout");
    std::memcpy(d.h_loc_pts, pts, sizeof(float2) * n);
    CK(cudaMemcpyAsync(d.loc_pts, d.h_loc_pts, sizeof(float2) * n, cudaMemcpyHostToDevice, d.loc_stream));
    launch_locate_points(d.loc_stream, c.scene_par[0].loc, d.loc_pts, n, d.loc_node);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(d.h_loc_node, d.loc_node, sizeof(int) * n, cudaMemcpyDeviceToHost, d.loc_stream));
    CK(cudaStreamSynchronize(d.loc_stream));
    std::memcpy(node, d.h_loc_node, sizeof(int) * n);
    c.launches += 1;
    return GMAPF_OK;
}

int device_set_targets_device(Context& c, const int* d_ids, const gmapf_v2* d_pos, int n, int id_base,
                              int id_count, std::string& err) {
    Device& d = c.dev;
    CK(cudaSetDevice(d.device));
    launch_apply_targets_device(d.stream, d_ids, reinterpret_cast<const float2*>(d_pos), n, id_base, id_count,
                                d.scene_par, d.agent_scene, d.state, d.targ, d.targ_pos,
                                d.counters + CT_ERR_TARGETS);
    c.launches += 1;
    CK(cudaGetLastError());
    return GMAPF_OK;
}

int device_search_batch(Context& c, const int* d_starts, const int* d_targets, int n, int* d_found,
                        int* d_lens, int* d_paths, long long path_stride, gmapf_step_stats* out,
                        std::string& err) {
    Device& d = c.dev;
    cudaStream_t s = d.stream;
    CK(cudaSetDevice(d.device));
    if (n > d.breq_cap) {
        for (void* p : {(void*)d.breq, (void*)d.breq_sorted, (void*)d.breq_keys}) {
            if (!p) continue;
            cudaFree(p);
            d.allocs.erase(std::remove(d.allocs.begin(), d.allocs.end(), p), d.allocs.end());
        }
        d.breq = nullptr;
        d.breq_sorted = nullptr;
        d.breq_keys = nullptr;
        DALLOC(d.breq, (size_t)n);
        if (d.lm) {
            DALLOC(d.breq_sorted, (size_t)n);
            DALLOC(d.breq_keys, (size_t)n);
        }
        d.breq_cap = n;
    }
    CK(cudaMemsetAsync(d.counters + CT_ERR, 0, sizeof(int), s));
    CK(cudaMemcpyAsync(c.h_stats, d.stats, sizeof(unsigned long long) * ST_COUNT, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    unsigned long long before[ST_COUNT];
    std::memcpy(before, c.h_stats, sizeof(before));
    launch_prepare_batch(s, d_starts, d_targets, n, c.map.n, d.breq, d.counters + CT_REQ,
                         d.counters + CT_WORK, d.counters + CT_ERR);
    c.launches += 1;
    SearchParams sp = search_params(c);
    sp.req = d.breq;
    if (d.lm && n > 0) {
        launch_order_requests(s, d.breq, d.counters + CT_REQ, d.breq_sorted, d.breq_keys, d.lm, d.lm_count, c.map.n);
        c.launches += 1;
        sp.req = d.breq_sorted;
    }
    sp.paths = d_paths;
    sp.path_stride = path_stride;
    sp.out_found = d_found;
    sp.out_len = d_lens;
    sp.ag_state = nullptr;
    sp.ag_step_idx = nullptr;
    sp.ag_path_len = nullptr;
    if (c.timeline) {
        if (n > c.timeline_rows) {
            err = "the search timeline holds " + std::to_string(c.timeline_rows) + " requests, the batch has " +
                  std::to_string(n);
            return GMAPF_E_INVALID_ARG;
        }
        sp.timeline = c.timeline;
    }
    CK(cudaEventRecord(d.ev[6], s));
    if (n > 0) {
        if (c.opt.mode == GMAPF_MODE_BATCHED) {
            CK(launch_search(s, sp, search_blocks(c), c.block_threads, true, 0, d.vm, d.bm_words));
            c.launches += 1;
        } else {
            sp.req_count_h = n;
            const int gpb = c.block_threads / 32;
            for (int base = 0; base < n; base += d.slots) {
                const int cnt = std::min(d.slots, n - base);
                CK(launch_search(s, sp, (cnt + gpb - 1) / gpb, c.block_threads, false, base, d.vm, d.bm_words));
                c.launches += 1;
            }
        }
    }
    CK(cudaEventRecord(d.ev[7], s));
    CK(cudaMemcpyAsync(c.h_small, d.counters, sizeof(int) * CT_COUNT, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(c.h_stats, d.stats, sizeof(unsigned long long) * ST_COUNT, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, d.ev[6], d.ev[7]));
    c.last_search_ms = ms;
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->requests = n;
        out->found = (int64_t)(c.h_stats[ST_FOUND] - before[ST_FOUND]);
        out->expansions = (int64_t)(c.h_stats[ST_EXPANSIONS] - before[ST_EXPANSIONS]);
        out->rounds = (int64_t)(c.h_stats[ST_ROUNDS] - before[ST_ROUNDS]);
        out->deg_sum = (int64_t)(c.h_stats[ST_DEG_SUM] - before[ST_DEG_SUM]);
        out->claims = (int64_t)(c.h_stats[ST_CLAIMS] - before[ST_CLAIMS]);
        out->path_nodes = (int64_t)(c.h_stats[ST_PATH_NODES] - before[ST_PATH_NODES]);
        out->promoted = (int64_t)(c.h_stats[ST_PROMOTED] - before[ST_PROMOTED]);
        out->ms_search = ms;
        out->ms_total_device = ms;
    }
    // keep the step's delta base consistent with the searches done here
    for (int k = 0; k < ST_COUNT; k++) c.stats_prev[k] += c.h_stats[k] - before[k];
    const int e = c.h_small[CT_ERR];
    if (e != 0) {
        err = device_error_text(e);
        return (e & ERR_BAD_REQUEST) ? GMAPF_E_INVALID_ARG : GMAPF_E_DEVICE;
    }
    return GMAPF_OK;
}

int device_upload_batch_io(Context& c, int n, long long path_stride, std::string& err) {
    Device& d = c.dev;
    if (n > d.bio_cap || (long long)n * path_stride > d.bpaths_cap) {
        void* old[] = {d.bstarts, d.btargets, d.bfound, d.blens, d.bpaths};
        for (void* p : old) {
            if (!p) continue;
            cudaFree(p);
            d.allocs.erase(std::remove(d.allocs.begin(), d.allocs.end(), p), d.allocs.end());
        }
        d.bstarts = d.btargets = d.bfound = d.blens = d.bpaths = nullptr;
        DALLOC(d.bstarts, (size_t)n);
        DALLOC(d.btargets, (size_t)n);
        DALLOC(d.bfound, (size_t)n);
        DALLOC(d.blens, (size_t)n);
        DALLOC(d.bpaths, (size_t)n * path_stride);
        d.bio_cap = n;
        d.bpaths_cap = (long long)n * path_stride;
    }
    return GMAPF_OK;
}

int device_debug_agents(Context& c, gmapf_v2* pos, int* state, int* cur, int* targ, int* step_idx,
                        int* step_node, gmapf_v2* step_pos, int* path_len, std::string& err) {
    Device& d = c.dev;
    const int A = c.A;
    CK(cudaSetDevice(d.device));
    CK(cudaStreamSynchronize(d.stream));
    if (A == 0) return GMAPF_OK;
    if (pos) CK(cudaMemcpy(pos, d.pos, sizeof(float2) * A, cudaMemcpyDeviceToHost));
    if (state) CK(cudaMemcpy(state, d.state, sizeof(int) * A, cudaMemcpyDeviceToHost));
    if (cur) CK(cudaMemcpy(cur, d.cur, sizeof(int) * A, cudaMemcpyDeviceToHost));
    if (targ) CK(cudaMemcpy(targ, d.targ, sizeof(int) * A, cudaMemcpyDeviceToHost));
    if (step_idx) CK(cudaMemcpy(step_idx, d.step_idx, sizeof(int) * A, cudaMemcpyDeviceToHost));
    if (step_node) CK(cudaMemcpy(step_node, d.step_node, sizeof(int) * A, cudaMemcpyDeviceToHost));
    if (step_pos) CK(cudaMemcpy(step_pos, d.step_pos, sizeof(float2) * A, cudaMemcpyDeviceToHost));
    if (path_len) CK(cudaMemcpy(path_len, d.path_len, sizeof(int) * A, cudaMemcpyDeviceToHost));
    return GMAPF_OK;
}

int device_debug_path(Context& c, int id, int* out, int cap, int* out_len, std::string& err) {
    Device& d = c.dev;
    CK(cudaSetDevice(d.device));
    CK(cudaStreamSynchronize(d.stream));
    int L = 0;
    CK(cudaMemcpy(&L, d.path_len + id, sizeof(int), cudaMemcpyDeviceToHost));
    *out_len = L;
    const int k = std::min(L, cap);
    if (k > 0) CK(cudaMemcpy(out, d.paths + (long long)id * d.path_stride, sizeof(int) * k, cudaMemcpyDeviceToHost));
    return GMAPF_OK;
}

// Re-size the search state after the search parameters change (autotuner).
int device_reconfigure_search(Context& c, std::string& err) {
    destroy_graph(c);
    return alloc_search_state(c, err);
}

int device_apply_tuned_shape(Context& c, int T, int C, int vm, int bt, std::string& err) {
    c.T = T;
    c.C = C;
    c.tuned_vm = vm;
    c.tuned_bt = bt;
    return device_reconfigure_search(c, err);
}

// Per-map autotuner (batched form): threads per agent T, queue capacity C,
// visited-state placement and block size.  T and C are parameters of the
// method itself (README.md:98-101: "picked empirically"), so the tuner keeps
// only shapes whose found rate on the sample is within 0.1% of the best one
// and, among those, takes the fastest.  The sample is seeded uniform triangle
// pairs of this navmesh; block size follows from pick_slots for each
// (T, C, placement).
int device_autotune(Context& c, std::string& err) {
    Device& d = c.dev;
    const int n = c.map.n;
    if (n < 2) return GMAPF_OK;
    // the sample is as large as a frame's request batch (2,048..16,384), so
    // that the tuner weighs throughput against the longest searches as a
    // frame does, with its path rows kept under 8 GB and a quarter of the free
    // memory
    size_t freeb = 0, totalb = 0;
    CK(cudaMemGetInfo(&freeb, &totalb));
    const double row_cap = std::min(8e9, 0.25 * (double)freeb);
    int Q = std::min(16384, std::max(2048, c.cfg.PathFinderParallelAgents));
    while (Q > 128 && (double)Q * n * 4 > row_cap) Q /= 2;
    std::vector<int> hs(Q), ht(Q);
    unsigned long long x = 0x9e3779b97f4a7c15ull;
    for (int i = 0; i < Q; i++) {
        x = x * 6364136223846793005ull + 1442695040888963407ull;
        hs[i] = (int)((x >> 33) % (unsigned long long)n);
        x = x * 6364136223846793005ull + 1442695040888963407ull;
        ht[i] = (int)((x >> 33) % (unsigned long long)n);
    }
    int *ds = nullptr, *dt = nullptr, *dfound = nullptr, *dlens = nullptr, *dpaths = nullptr;
    auto release = [&]() {
        for (int* p : {ds, dt, dfound, dlens, dpaths})
            if (p) cudaFree(p);
    };
    if (cudaMalloc(&ds, 4 * Q) != cudaSuccess || cudaMalloc(&dt, 4 * Q) != cudaSuccess ||
        cudaMalloc(&dfound, 4 * Q) != cudaSuccess || cudaMalloc(&dlens, 4 * Q) != cudaSuccess ||
        cudaMalloc(&dpaths, (size_t)4 * Q * n) != cudaSuccess) {
        cudaGetLastError();
        release();
        err = "autotune: cannot allocate the sample buffers";
        return GMAPF_E_CAPACITY;
    }
    if (cudaMemcpyAsync(ds, hs.data(), 4 * Q, cudaMemcpyHostToDevice, d.stream) != cudaSuccess ||
        cudaMemcpyAsync(dt, ht.data(), 4 * Q, cudaMemcpyHostToDevice, d.stream) != cudaSuccess ||
        cudaStreamSynchronize(d.stream) != cudaSuccess) {
        cudaGetLastError();
        release();
        err = "autotune: cannot upload the sample";
        return GMAPF_E_CUDA;
    }

    struct Trial {
        int T, C, vm, bt;
        float ms;
        long long found;
    };
    std::vector<Trial> trials;
    const int T0 = c.T, C0 = c.C;
    // one trial: the sample twice, the faster time kept (a shape that is
    // already three times slower than the best so far is not repeated)
    float best_so_far = 1e30f;
    auto trial = [&](int T, int C, int vm, int bt) {
        c.T = T;
        c.C = C;
        c.tuned_vm = vm;
        c.tuned_bt = bt;
        std::string e2;
        if (device_reconfigure_search(c, e2) != GMAPF_OK) return;  // shape does not fit
        gmapf_step_stats st{};
        float ms = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            if (device_search_batch(c, ds, dt, Q, dfound, dlens, dpaths, n, &st, e2) != GMAPF_OK) return;
            ms = std::min(ms, c.last_search_ms);
            if (ms > 3.0f * best_so_far) break;
        }
        best_so_far = std::min(best_so_far, ms);
        trials.push_back({T, C, c.dev.vm, c.block_threads, ms, (long long)st.found});
    };
    // stage 1: threads per agent x queue capacity x visited placement, block
    // size by occupancy.  The found count depends on (T, C) only, so a shape
    // already below the best found count skips its other placements.
    std::vector<int> Ts = {32, 16, 8, 4, 2}, Cs = {8, 16, 32, 64, 128, 256};  // likely-fast shapes first
    if (std::find(Cs.begin(), Cs.end(), C0) == Cs.end()) Cs.push_back(C0);
    // Fewer threads per agent mean more rounds per query: once the best time
    // at one T is over twice the best so far, the smaller T are not tried.
    long long best_found_so_far = 0;
    for (int T : Ts) {
        float best_at_T = 1e30f;
        for (int C : Cs) {
            bool vm4_fits = false;
            for (int vm : {4, 3, 2, 1}) {
                if (c.opt.visited_mode != 0 && c.opt.visited_mode != vm) continue;
                // placement 4 runs placement 3's rounds until a search is alone in
                // its block, then cheaper ones: where it fits with placement 3's
                // occupancy, 3 is not timed
                if (vm == 3 && vm4_fits) continue;
                const size_t before = trials.size();
                trial(T, C, vm, 0);
                if (trials.size() == before) continue;  // shape does not fit this placement
                if (vm == 4)
                    vm4_fits = search_max_blocks_per_sm(T, C, c.block_threads, 4, d.bm_words) ==
                               search_max_blocks_per_sm(T, C, c.block_threads, 3, d.bm_words);
                best_at_T = std::min(best_at_T, trials.back().ms);
                const long long f = trials.back().found;
                best_found_so_far = std::max(best_found_so_far, f);
                if ((double)f < (double)best_found_so_far * 0.999) break;
            }
        }
        if (best_at_T < 1e30f && best_at_T > 2.0f * best_so_far) break;
    }
    auto choose = [&]() -> const Trial* {
        long long best_found = 0;
        for (const Trial& t : trials) best_found = std::max(best_found, t.found);
        const Trial* pick = nullptr;
        for (const Trial& t : trials)
            if ((double)t.found >= (double)best_found * 0.999 && (!pick || t.ms < pick->ms)) pick = &t;
        return pick;
    };
    // stage 1b: the four fastest eligible shapes timed again (four more runs
    // each), so that shapes within the timing noise are told apart fairly
    {
        long long best_found = 0;
        for (const Trial& t : trials) best_found = std::max(best_found, t.found);
        std::vector<Trial> top;
        for (const Trial& t : trials)
            if ((double)t.found >= (double)best_found * 0.999) top.push_back(t);
        std::sort(top.begin(), top.end(), [](const Trial& a, const Trial& b) { return a.ms < b.ms; });
        if (top.size() > 4) top.resize(4);
        for (int rep = 0; rep < 2; rep++)
            for (const Trial& t : top) trial(t.T, t.C, t.vm, 0);
    }
    // stage 2: block size for the chosen shape
    if (const Trial* p1 = choose(); p1 && c.opt.block_threads == 0) {
        const Trial t1 = *p1;
        for (int bt : {32, 64, 128, 256})
            if (bt != t1.bt) trial(t1.T, t1.C, t1.vm, bt);
    }
    release();
    const Trial* pick = choose();
    c.T = pick ? pick->T : T0;
    c.C = pick ? pick->C : C0;
    c.tuned_vm = pick ? pick->vm : 0;
    c.tuned_bt = pick ? pick->bt : 0;
    if (c.cfg.IsDebug) {
        for (const Trial& t : trials)
            std::printf("[gmapf] autotune T=%d C=%d visited=%d block=%d: %.3f ms, found %lld/%d\n", t.T, t.C, t.vm,
                        t.bt, t.ms, t.found, Q);
        std::printf("[gmapf] autotune picked T=%d C=%d visited=%d block=%d\n", c.T, c.C, c.tuned_vm, c.tuned_bt);
    }
    // the sample's searches do not count toward the frames' statistics
    CK(cudaMemsetAsync(d.stats, 0, sizeof(unsigned long long) * ST_COUNT, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    std::memset(c.h_stats, 0, sizeof(unsigned long long) * ST_COUNT);
    for (int k = 0; k < ST_COUNT; k++) c.stats_prev[k] = 0;
    return device_reconfigure_search(c, err);
}

}  // namespace gmapf_b200
