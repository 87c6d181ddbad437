// internal.h -- host-side structures of the B200 G-MAPF library (not installed).
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gmapf_c.h"
#include "geom.cuh"

namespace gmapf_b200 {

// ------------------------------------------------------------------ device --

// Per-slot visited record of one claimed node, 32 bytes.  With stamped
// records (visited placement 2) `stamp` equals the slot's current query epoch
// iff the node is claimed by that query, so slots are reused across queries
// and frames without clearing; with a visited bitmap the same word holds the
// node's jump ancestor (the nearest proper ancestor at a depth that is a
// multiple of 256, -1 at the root) for a parallel path walk.  `gd` = G << 1 | dir
// (dir 1 = reached from the start, PathNode::FromStart).  anc[0] is the
// parent (PathNode::PrevNodeIdx); anc[k] the (k+1)-th ancestor, so a path
// walk advances six hops per record read.  One 32-byte sector: it is read
// and written as a whole (records.cuh).
struct __align__(32) Rec {
    unsigned stamp;
    int gd;
    int anc[6];
};

enum StatIdx {
    ST_EXPANSIONS = 0,
    ST_ROUNDS,
    ST_DEG_SUM,
    ST_CLAIMS,
    ST_PATH_NODES,
    ST_FOUND,
    ST_REQUESTS,
    ST_MOVING,
    ST_NEIGHBOURS,  // agents examined in the 3x3 grid cells by the collision pass
    ST_PROMOTED,    // searches that moved their visited bitmap into their block's shared memory
    ST_COUNT
};

enum ErrBits {
    ERR_BOUNDS = 1,      // an index failed its bounds check (access skipped)
    ERR_ROUNDS = 2,      // a search exceeded its round limit
    ERR_PATH_CAP = 4,    // a path did not fit its output row
    ERR_BAD_REQUEST = 8  // a request named a node outside the map
};

struct SearchParams {
    const SearchRow* rows;
    const float2* cen;
    int n;
    const int4* req;         // {agent (or -1), start, target, output row}
    const int* req_count_d;  // device count (persistent form)
    int req_count_h;         // host count (plain form)
    int T, C;
    float K;
    Rec* rec;                // slots * n
    unsigned* epoch;         // per slot
    int slots;
    unsigned* gbm;           // visited mode 3: bm_words 32-bit words per slot, global
    int* work_ctr;
    int max_rounds;
    int promote_rounds;      // visited placement 4: rounds before a search may move its bitmap into shared memory
    // outputs
    int* paths;              // row-major, path_stride ints per row
    long long path_stride;
    int* out_found;          // per request (batch API) or null
    int* out_len;            // per request (batch API) or null
    int* ag_state;           // agent arrays (step) or null
    int* ag_step_idx;
    int* ag_path_len;
    unsigned long long* stats;  // ST_COUNT counters
    int* err;
    // search state slots [slot_base, slot_base + slots) of rec/epoch/gbm
    int slot_base;
    // serving ring (ring_cap > 0): request r of this launch is query
    // q = ring_base + r, stored at req[q % ring_cap]; its completion word
    // done[q % ring_cap] = (q + 1) << 1 | found goes to host-mapped memory
    // after the results
    int ring_cap;
    int ring_base;
    unsigned long long* done;
    // diagnostics (batch searches): per output row, the GPU global timer when
    // a warp took the request [2 row] and when its results were written
    // [2 row + 1], or null
    unsigned long long* timeline;
};

// Per-scene constants of the mover and of point location: one entry for a
// context with one map; a scene batch concatenates several maps (global
// triangle ids) and several agent ranges.
struct ScenePar {
    float ax0, ay0, ainv;    // agent grid: origin, inverse cell size
    int aw, ah, cell_base;   // cells per axis, first global cell
    float cd, cd2;           // collision distance (2.5 r) and its square
    float arrive;            // FLT_EPSILON + r
    float speed;
    float clear;             // path smoothing 2: portals narrowed by r at both ends (else 0)
    LocateGrid loc;          // this scene's triangles (found ids are global)
};

struct MoverParams {
    int A;
    const int* mv_count;
    const unsigned char* in_move;
    float2* pos;       // in: previous frame, out: final (collision output)
    float2* pos_mid;   // after move (collision snapshot)
    float2* step_pos;
    const float2* targ_pos;
    int* state;
    int* cur_node;
    int* step_idx;
    int* step_node;
    const int* path_len;
    const int* paths;
    long long path_stride;
    const float* dt;   // frame dt (device scalar, set per frame); step = speed * dt
    float cs, sn;      // rotation by +10 degrees
    const ScenePar* sc;        // per scene
    const int* agent_scene;    // scene of each agent, or null (one scene)
    // agent grid (all scenes' cells, global ids)
    int cells;
    int* cell_of;
    int* cell_cnt;     // cells + 1
    int* cell_start;   // cells + 1
    int* cell_fill;    // cells
    int* cell_items;   // A
    // map
    const float2* tri; // 3 vertices per triangle, global ids
    const float2* cen;
    float2* waypoints; // path smoothing: per agent, per path step, the steering point (null: centroids)
    int n;
    unsigned long long* stats;
    int* err;
};

// kernels.cu
// Scene limits for compaction: agents of scene s are [abase[s], abase[s+1]);
// at most P[s] requests per scene per frame, in ascending agent id.  All null
// for a context with one map (P applies).  first: nscenes ints of scratch.
struct CompactScenes {
    const int* agent_scene;
    const int* abase;
    const int* P;
    int* first;
};
void launch_compact(cudaStream_t s, int A, int* state, const int* cur, const int* targ, int P,
                    const CompactScenes& scn, int4* req, int* req_count, unsigned char* in_move, int* mv_count,
                    int* work_ctr, unsigned long long* stats);
void launch_apply_targets(cudaStream_t s, const int4* recs, int n, int* state, int* targ_node,
                          float2* targ_pos);
// device-resident retargets of agents id_base + ids[k], ids[k] in [0, id_count)
// point location of n points in one map (found ids include g.base; -1: none)
void launch_locate_points(cudaStream_t s, const LocateGrid& g, const float2* pts, int n, int* out);
void launch_apply_targets_device(cudaStream_t s, const int* ids, const float2* pos, int n, int id_base,
                                 int id_count, const ScenePar* sc, const int* agent_scene, int* state,
                                 int* targ_node, float2* targ_pos, int* err);
// requests reordered longest-first by the landmark estimate (keys: scratch, one int per request)
void launch_order_requests(cudaStream_t s, const int4* req_in, const int* req_count, int4* req_out, int* keys,
                           const unsigned short* lm, int L, int n);
void launch_move_bin(cudaStream_t s, const MoverParams& p);
void launch_cell_scan(cudaStream_t s, const MoverParams& p);
void launch_scatter(cudaStream_t s, const MoverParams& p);
void launch_collide_progress(cudaStream_t s, const MoverParams& p);
// path smoothing: funnel corners of the paths that start this frame
void launch_funnel(cudaStream_t s, const MoverParams& p);
void launch_prepare_batch(cudaStream_t s, const int* starts, const int* targets, int n, int nodes,
                          int4* req, int* req_count, int* work_ctr, int* err);
// search.cu
// persistent: groups pull requests from *work_ctr until *req_count_d is reached.
// plain: one request per group, requests [base, base + groups).
// vm (visited state): 1 a 2-bit bitmap per slot in shared memory (bm_words
// 32-bit words per slot), 2 query-stamped records in global memory, 3 a 2-bit
// bitmap per slot in global memory (p.gbm, small enough to stay in L2).
cudaError_t launch_search(cudaStream_t s, const SearchParams& p, int blocks, int block_threads,
                          bool persistent, int req_base, int vm, int bm_words);
size_t search_smem_bytes(int C, int block_threads, int bm_words, int T, int vm);
int search_bitmap_words(int n_nodes);
int search_max_blocks_per_sm(int T, int C, int block_threads, int vm, int bm_words);

// ------------------------------------------------------------------- host --

// One map with its agents inside a context: a plain context has exactly one
// (the whole map and every agent); a scene batch's world has one per scene.
struct SceneInfo {
    int node_base = 0, n = 0;     // global triangle range
    int agent_base = 0, A = 0;    // global agent range
    int P = 0;                    // requests per frame (Config.PathFinderParallelAgents)
    float radius = 0, speed = 0;
    float bx0 = 0, by0 = 0, bx1 = 0, by1 = 0;  // map bounds (agent grid)
    float gx0 = 0, gy0 = 0, ginv = 1;          // point-location grid
    int gw = 1, gh = 1;
    size_t gstart_off = 0, glist_off = 0, degen_off = 0;
    int ndegen = 0;
};

struct HostMap {
    int n = 0;
    std::vector<gmapf_node> nodes;  // as ingested, PCenter recomputed
    std::vector<SearchRow> rows;
    std::vector<float2> tri;        // 3 per node
    std::vector<float2> cen;
    float bx0 = 0, by0 = 0, bx1 = 0, by1 = 0;
    float gx0 = 0, gy0 = 0, ginv = 1;
    int gw = 1, gh = 1;
    std::vector<int> gstart, glist, degen;
    LocateGrid view() const;
};

// hostmap.cpp
void build_host_map(const gmapf_node* nodes, int n, HostMap& out);
// The world map of a scene batch: the scenes' maps one after another with
// global triangle ids; fills each scene's triangle range, bounds and
// point-location grid (offsets into the concatenated grid arrays).
void concat_host_maps(const std::vector<const HostMap*>& maps, HostMap& out, std::vector<SceneInfo>& scenes);
// Hop distances from `count` landmark triangles chosen by farthest-point
// sampling over the neighbour graph (unreachable: 65535), count * n values.
void landmark_distances(const HostMap& m, int count, std::vector<unsigned short>& out);
// navmesh_cdt.cpp: 0 on success, else a gmapf_status with `err` set
int build_navmesh_cdt(const std::vector<float>& verts, const std::vector<unsigned>& edges,
                      std::vector<gmapf_node>& out, std::string& err);

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct Device {
    int device = 0;
    cudaStream_t stream = nullptr, stream2 = nullptr;
    // map
    SearchRow* rows = nullptr;
    float2* cen = nullptr;
    float2* tri = nullptr;
    int *gstart = nullptr, *glist = nullptr, *degen = nullptr;
    // agents
    float2 *pos = nullptr, *pos_mid = nullptr, *targ_pos = nullptr, *step_pos = nullptr;
    int *state = nullptr, *cur = nullptr, *targ = nullptr, *step_idx = nullptr, *step_node = nullptr,
        *path_len = nullptr;
    int* paths = nullptr;
    long long path_stride = 0;
    unsigned char* in_move = nullptr;
    int4* dirty = nullptr;
    int dirty_cap = 0;
    // requests / counters
    int4* req = nullptr;
    int4* req_sorted = nullptr;  // longest-first order (order_by_estimate)
    int* req_keys = nullptr;
    unsigned short* lm = nullptr;  // landmark hop distances, lm_count x n
    int lm_count = 0;
    int4* breq_sorted = nullptr;
    int* breq_keys = nullptr;
    int* counters = nullptr;  // [req_count, mv_count, work_ctr, err, spare...]
    unsigned long long* stats = nullptr;
    // search state
    Rec* rec = nullptr;
    unsigned* epoch = nullptr;
    int slots = 0;
    int vm = 2;                 // visited mode (1, 2 or 3; see launch_search)
    unsigned* gbm = nullptr;    // visited mode 3: slots x bm_words
    int bm_words = 0;           // bitmap words per slot
    int rec_cap = 0, gbm_cap = 0;  // slots the record / bitmap arrays hold (kept across reshapes)
    // agent grid
    int *cell_of = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cell_fill = nullptr,
        *cell_items = nullptr;
    int cells = 0;
    // scenes (ScenePar per scene; the rest only when there is more than one)
    ScenePar* scene_par = nullptr;
    int* agent_scene = nullptr;
    int *scene_abase = nullptr, *scene_P = nullptr, *scene_first = nullptr;
    float2* waypoints = nullptr;  // path smoothing (A x path_stride)
    bool clearance = false;       // path smoothing 2: corners kept one agent radius off the walls
    // batch API scratch
    int4* breq = nullptr;
    int breq_cap = 0;
    int *bstarts = nullptr, *btargets = nullptr, *bfound = nullptr, *blens = nullptr,
        *bpaths = nullptr;
    long long bpaths_cap = 0;
    int bio_cap = 0;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    float graph_dt = -1.0f;
    // events
    cudaEvent_t ev[8] = {};
    cudaEvent_t frame_done = nullptr;  // recorded after each frame's work (step-ready query)
    std::vector<void*> allocs;
    // bulk point location (large host retargets), on its own stream so it never
    // waits behind a running frame; buffers grow to the largest call
    cudaStream_t loc_stream = nullptr;
    float2* loc_pts = nullptr;
    int* loc_node = nullptr;
    float2* h_loc_pts = nullptr;  // pinned
    int* h_loc_node = nullptr;    // pinned
    int loc_cap = 0;
};

struct Profiler {
    std::vector<float> wall_ms;
    float sum_wall = 0, max_wall = 0;
    float sum_pre = 0, max_pre = 0;
    int n_pre = 0;
    float sum_post = 0, max_post = 0;
    float sum_search = 0, max_search = 0;
    float sum_mover = 0, max_mover = 0;
    float sum_compact = 0, max_compact = 0;
    int n = 0, n_search = 0, n_mover = 0;
};

struct Service;  // serve.cu

struct Context {
    bool inited = false, started = false, step_going = false;
    gmapf_config cfg{};
    gmapf_options opt{};
    // map ingestion
    std::vector<float> cdt_v;
    std::vector<unsigned> cdt_e;
    bool map_filled = false;
    uint64_t map_input_hash = 0;  // hash of the CDT input the map was built from (0: given as nodes)
    HostMap map;
    // agents: host mirror (capacity reserved at Init, so pointers stay valid)
    int A = 0;
    std::vector<gmapf_v2> m_pos;
    std::vector<int> m_state, m_cur, m_targ_node;
    std::vector<gmapf_v2> m_targ;
    // pinned staging (allocated at start)
    float2* h_pos_stage = nullptr;
    int* h_state_stage = nullptr;
    int4* h_dirty = nullptr;
    int* h_small = nullptr;            // counters snapshot
    unsigned long long* h_stats = nullptr;
    float* h_step = nullptr;
    std::vector<int4> dirty_recs;
    std::vector<int> dirty_slot;       // agent -> index in dirty_recs or -1
    // maps and agent ranges on the device (filled at start: one entry unless
    // this context is a scene batch's world)
    std::vector<SceneInfo> scenes;
    std::vector<ScenePar> scene_par;  // host copy, device pointers inside
    // effective search parameters
    int T = 4, C = 16, block_threads = 128;
    float K = 1.0f;
    // autotuner's choices where the options leave them open (0: pick by occupancy)
    int tuned_vm = 0, tuned_bt = 0;
    std::string tune_cache;  // autotuner cache file ("" = none)
    unsigned long long* timeline = nullptr;  // caller's device buffer (gmapf_set_search_timeline)
    int timeline_rows = 0;
    int tune_source = 0;     // 0 not tuned, 1 tuned at the start, 2 from the cache
    // device
    Device dev;
    Profiler prof;
    gmapf_step_stats last{};
    unsigned long long stats_prev[ST_COUNT] = {};
    std::chrono::steady_clock::time_point t_step0;
    float pre_ms = 0;
    bool pre_done = false;
    long long launches = 0;
    float last_search_ms = 0;
    // scene batches: a scene context bound to a batch forwards its agent calls
    // to the batch's world (agents [agent_base, agent_base + A), triangles
    // [node_base, node_base + map.n) there)
    int scene_index = -1, agent_base = 0, node_base = 0;
    bool is_world = false;   // the merged context of a batch
    bool detached = false;   // its batch was destroyed
    Service* serve = nullptr;  // serving form (after gmapf_serve_start)
    int plain_req_count = 0, plain_mv_count = 0;
};

// device.cu
// rounds one search may run: the round_limit option, else 4 N + 64 (never
// reached: every round pops a queued node and a node is queued once)
int search_round_limit(const Context& c);
int search_promote_rounds(const Context& c);
// "device-side check failed: ..." naming the ErrBits set in e
std::string device_error_text(int e);
int device_start(Context& c, std::string& err);
void device_free(Context& c);
int device_async_step(Context& c, float dt, std::string& err);
int device_wait_step(Context& c, std::string& err);
bool device_step_ready(Context& c);
int device_search_batch(Context& c, const int* d_starts, const int* d_targets, int n, int* d_found,
                        int* d_lens, int* d_paths, long long path_stride, gmapf_step_stats* st,
                        std::string& err);
int device_debug_agents(Context& c, gmapf_v2* pos, int* state, int* cur, int* targ, int* step_idx,
                        int* step_node, gmapf_v2* step_pos, int* path_len, std::string& err);
int device_debug_path(Context& c, int id, int* out, int cap, int* out_len, std::string& err);
int device_autotune(Context& c, std::string& err);
// use a shape the autotuner picked before (T, C, visited placement, block size)
int device_apply_tuned_shape(Context& c, int T, int C, int vm, int bt, std::string& err);
int device_upload_batch_io(Context& c, int n, long long path_stride, std::string& err);
// the triangle of each of n host points, located on the device with the
// same rule as the host (single-map context, after start); blocks until done
int device_locate_points(Context& c, const gmapf_v2* pts, int n, int* node, std::string& err);
int device_set_targets_device(Context& c, const int* d_ids, const gmapf_v2* d_pos, int n, int id_base,
                              int id_count, std::string& err);

// serve.cu
int serve_start(Context& c, int max_in_flight, std::string& err);
void serve_free(Context& c);
int serve_submit(Context& c, const int* ids, const gmapf_v2* pos, int n, const int64_t* arrival_ns, std::string& err);
int serve_poll(Context& c, std::string& err);
int serve_drain(Context& c, double timeout_s, std::string& err);
int serve_before_frame(Context& c, cudaStream_t s, std::string& err);
void serve_after_frame(Context& c);
void serve_stats(Context& c, gmapf_serve_stats* out, bool reset);
int serve_result(Context& c, int agent, int* found, int* len, int* path, int cap, std::string& err);

// capi.cpp: message returned by gmapf_last_error() on this thread
void set_last_error(const std::string& msg);
// capi.cpp: p is memory a kernel on `device` may access (that GPU's device
// memory, managed memory or mapped host memory); false for pageable host
// memory and for another GPU's device memory
bool gpu_reachable(const void* p, int device);

}  // namespace gmapf_b200
