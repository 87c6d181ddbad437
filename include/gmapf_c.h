/*
 * gmapf_c.h -- C ABI of the B200-native G-MAPF per-frame step.
 *
 * The reference (rosdvp/gmapf) exposes only the C++ class gmapf::GMAPF
 * (include/gmapf/GMAPF.h:30-98) and has no C ABI.  Each entry point below
 * replaces one member of that class; the citation names the member it
 * stands for.  include/gmapf/GMAPF.h in this repository is the header-only
 * C++ wrapper over these functions with the reference's class, method and
 * type names.
 *
 * Conventions: every function returns a gmapf_status (GMAPF_OK == 0);
 * gmapf_last_error() returns a message for the last failure on the calling
 * thread.  Plain pointers and sizes only; no C++ or torch types cross.
 */
#ifndef GMAPF_C_H
#define GMAPF_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gmapf_status {
    GMAPF_OK = 0,
    GMAPF_E_STATE = 1,          /* lifecycle rule broken (not initialised, already started, ...) */
    GMAPF_E_INVALID_POS = 2,    /* a position lies in no navmesh triangle */
    GMAPF_E_CUDA = 3,           /* a CUDA runtime call failed */
    GMAPF_E_CAPACITY = 4,       /* a fixed capacity would be exceeded */
    GMAPF_E_DEVICE_TIMEOUT = 5, /* a wait for device work ran out of time (gmapf_serve_drain) */
    GMAPF_E_INVALID_ARG = 6,    /* bad argument (null pointer, out-of-range id or parameter) */
    GMAPF_E_UNSUPPORTED = 7,    /* feature not compiled in (e.g. the CDT navmesh builder) */
    GMAPF_E_DEVICE = 8          /* a device-side check failed (bounds / consistency) */
} gmapf_status;

typedef enum gmapf_agent_state { /* include/gmapf/Agent.h:7-12 (EAgentState) */
    GMAPF_AGENT_IDLE = 0,
    GMAPF_AGENT_SEARCH = 1,
    GMAPF_AGENT_MOVE = 2
} gmapf_agent_state;

/* include/gmapf/Config.h:5-18 -- same field order, types and layout
 * (7 x 4-byte fields then two bools; 32 bytes with padding). */
typedef struct gmapf_config {
    int32_t AgentsMaxCount;
    float AgentRadius;
    float AgentSpeed;
    int32_t PathFinderParallelAgents;
    int32_t PathFinderThreadsPerAgents;
    int32_t PathFinderQueueCapacity;
    float PathFinderHeuristicK;
    uint8_t IsDebug;
    uint8_t IsProfiler;
} gmapf_config;

/* include/gmapf/misc/V2Float.h:12-16 */
typedef struct gmapf_v2 {
    float X;
    float Y;
} gmapf_v2;

/* include/gmapf/misc/CuNodesMap.h:14-21 (CuNodesMap::Node, 48 bytes,
 * 16-byte aligned): three vertices, the centroid (overwritten on ingest),
 * up to three neighbour ids packed first and padded with -1. */
typedef struct gmapf_node {
    gmapf_v2 P1;
    gmapf_v2 P2;
    gmapf_v2 P3;
    gmapf_v2 PCenter;
    int32_t NeibsIdx[3];
    int32_t _pad;
} gmapf_node;

/* Step forms.  Both run the same per-query arithmetic and give identical
 * results for the same (threads per agent, queue capacity). */
typedef enum gmapf_mode {
    GMAPF_MODE_BATCHED = 0, /* persistent search over a device work queue; step replayed as a CUDA graph */
    GMAPF_MODE_PLAIN = 1    /* one lane group per request in fixed launches; host reads counts back */
} gmapf_mode;

/* Tuning knobs that are not part of the reference Config. */
typedef struct gmapf_options {
    int32_t device;            /* CUDA device ordinal (default 0) */
    int32_t mode;              /* gmapf_mode (default GMAPF_MODE_BATCHED) */
    int32_t block_threads;     /* search block size, 0 = automatic */
    int32_t autotune;          /* 1: pick threads/agent, queue capacity and block size per map at start */
    int64_t search_mem_budget; /* bytes for per-slot search records, 0 = automatic */
    int32_t order_by_estimate; /* 1 (default): batched form serves the searches with the largest
                                  landmark hop-distance estimate first; results do not depend on it */
    int32_t visited_mode;      /* 0 automatic, 1 shared-memory bitmap per slot, 2 stamped global records,
                                  3 global bitmap per slot (L2-resident for maps up to a few 100k triangles),
                                  4 global bitmap per slot; a search still running after promote_rounds
                                  rounds, once enough of its block's warps have finished (a batch's
                                  tail), moves its bitmap into their shared memory (the bitmap, N/4 bytes for
                                  N triangles, has to fit in one block's shared memory; automatic
                                  placement only picks 4 where it does, a forced 4 that does not fit
                                  fails the start with GMAPF_E_CAPACITY) */
    int32_t path_smoothing;    /* 1: agents steer through the corridor's funnel corners (portal edges)
                                  instead of triangle centroids; 2: the same with every portal narrowed
                                  by the agent radius at both ends, so the corners keep that clearance
                                  from the walls (a portal no wider than two radii becomes its midpoint);
                                  the triangle paths and the per-triangle progress stay the reference's.
                                  Off (0) by default: on, agents take different routes from the
                                  reference's (AgentsMover.h:148,174) */
    int32_t round_limit;       /* rounds one search may run before it is stopped, not found, and the
                                  call or step reports GMAPF_E_DEVICE (round-limit bit); 0 = 4 N + 64
                                  for an N-triangle map, which no search reaches (every round pops a
                                  queued node and a node is queued once).  Smaller values bound the
                                  time of one search */
    int32_t promote_rounds;    /* visited mode 4: rounds a search runs on its global bitmap before it
                                  may move it into its block's shared memory, 0 = 512.  Results do not
                                  depend on it */
    int32_t _reserved[1];
} gmapf_options;

typedef struct gmapf_step_stats {
    int64_t requests;       /* path requests served this frame */
    int64_t found;          /* of which found */
    int64_t expansions;     /* nodes expanded */
    int64_t rounds;         /* search rounds summed over requests */
    int64_t deg_sum;        /* sum of the degrees of expanded nodes */
    int64_t claims;         /* nodes claimed */
    int64_t path_nodes;     /* sum of path lengths written */
    int64_t moving;         /* agents in Move at the start of the frame */
    float ms_step_wall;     /* host wall time AsyncStep -> WaitStepEnd */
    float ms_search;        /* device time of the search kernel(s) */
    float ms_mover;         /* device time of the mover kernels */
    float ms_total_device;  /* device time of the whole frame */
    int64_t neighbours;     /* agents read from the 3x3 grid cells by the collision pass (summed over agents) */
    int64_t promoted;       /* searches that moved their visited bitmap into shared memory (visited mode 4) */
} gmapf_step_stats;

typedef struct gmapf_ctx gmapf_ctx;

/* Lifecycle (GMAPF.h:32-37 constructor/destructor) */
gmapf_status gmapf_create(gmapf_ctx** out);
gmapf_status gmapf_destroy(gmapf_ctx* ctx);
const char* gmapf_last_error(void);

/* GMAPF::Init(const Config&)            -- src/GMAPF.cu:58-70 */
gmapf_status gmapf_init(gmapf_ctx* ctx, const gmapf_config* config);
/* tuning knobs; call between gmapf_init and the start */
gmapf_status gmapf_set_options(gmapf_ctx* ctx, const gmapf_options* opts);
gmapf_status gmapf_get_options(gmapf_ctx* ctx, gmapf_options* out);

/* GMAPF::FillMapStart(const V2Float&)   -- src/GMAPF.cu:133-145 */
gmapf_status gmapf_fill_map_start(gmapf_ctx* ctx, float size_x, float size_y);
/* GMAPF::FillMapObstacle(vector<V2Float>) -- src/GMAPF.cu:147-159 */
gmapf_status gmapf_fill_map_obstacle(gmapf_ctx* ctx, const gmapf_v2* vertices, int32_t count);
/* GMAPF::FillMapEnd()                    -- src/GMAPF.cu:161-196 */
gmapf_status gmapf_fill_map_end(gmapf_ctx* ctx);
/* GMAPF::FillMapManually(vector<Node>)   -- src/GMAPF.cu:199-217 */
gmapf_status gmapf_fill_map_manually(gmapf_ctx* ctx, const gmapf_node* nodes, int32_t count);

/* ---- navmesh files (no counterpart in the reference, which triangulates on
 * every FillMapEnd: ~0.45 s on the host at 100k triangles) ----
 * A file holds the built navmesh (the gmapf_node records FillMapEnd makes),
 * a checksum of them and a hash of the FillMapStart/FillMapObstacle input it
 * was built from. */
/* write the context's navmesh */
gmapf_status gmapf_map_save(gmapf_ctx* ctx, const char* path);
/* FillMapManually from a file (checked: magic, version, size, checksum,
 * neighbour ids) */
gmapf_status gmapf_map_load(gmapf_ctx* ctx, const char* path);
/* FillMapEnd through a cache file: when `path` holds a navmesh built from the
 * same FillMapStart/FillMapObstacle input, it is loaded instead of
 * triangulating; otherwise the navmesh is built and written there.  *hit (may
 * be null) tells which happened.  A damaged or foreign file is rebuilt. */
gmapf_status gmapf_fill_map_end_cached(gmapf_ctx* ctx, const char* path, int32_t* hit);

/* GMAPF::AddAgent(const V2Float&)        -- src/GMAPF.cu:219-236 */
gmapf_status gmapf_add_agent(gmapf_ctx* ctx, float x, float y, int32_t* out_id);
/* GMAPF::SetAgentTargPos(int, V2Float)   -- src/GMAPF.cu:238-253
 * (README.md:78 spells it SetAgentTargetPos; both C++ spellings map here) */
gmapf_status gmapf_set_agent_targ_pos(gmapf_ctx* ctx, int32_t agent_id, float x, float y);
/* bulk form of the above: n targets, one call, the same as n calls in order
 * (the first invalid position stops it with GMAPF_E_INVALID_POS, the items
 * before it applied).  From 2,048 targets the points are located on the
 * device once the context is started (on a stream of their own: a running
 * step is not waited for), before that on several host threads. */
gmapf_status gmapf_set_agent_targ_pos_bulk(gmapf_ctx* ctx, const int32_t* ids, const gmapf_v2* pos, int32_t n);
/* device-resident form: ids and positions already in device memory; the
 * target triangles are located on the device (same rule as the host path).
 * Enqueued on the context's stream before the next step; a position in no
 * triangle leaves that agent unchanged and makes the next step report
 * GMAPF_E_DEVICE.  Call after the start, not during a step.  Pageable host
 * memory is refused (GMAPF_E_INVALID_ARG). */
gmapf_status gmapf_set_agent_targ_pos_device(gmapf_ctx* ctx, const int32_t* d_ids, const gmapf_v2* d_pos, int32_t n);

/* GMAPF::ManualStart()                   -- src/GMAPF.cu:72-130 */
gmapf_status gmapf_manual_start(gmapf_ctx* ctx);
/* GMAPF::AsyncStep(float)                -- src/GMAPF.cu:255-289 */
gmapf_status gmapf_async_step(gmapf_ctx* ctx, float delta_time);
/* GMAPF::WaitStepEnd()                   -- src/GMAPF.cu:291-314 */
gmapf_status gmapf_wait_step_end(gmapf_ctx* ctx);
/* No counterpart in the reference: 1 when no step is running or the running
 * step's device work has finished (gmapf_wait_step_end will not block), 0
 * while it runs.  Lets a caller keep serving or preparing input during a
 * step; the step's results still appear only through gmapf_wait_step_end. */
int32_t gmapf_step_ready(gmapf_ctx* ctx);

/* GMAPF::GetAgentPos(int)                -- src/GMAPF.cu:316-319 */
gmapf_status gmapf_get_agent_pos(gmapf_ctx* ctx, int32_t agent_id, gmapf_v2* out);
/* GMAPF::GetAgentState(int)              -- src/GMAPF.cu:321-324 */
gmapf_status gmapf_get_agent_state(gmapf_ctx* ctx, int32_t agent_id, int32_t* out);
/* pointer to the host mirror of all positions (valid until gmapf_destroy;
 * refreshed by gmapf_wait_step_end); backs GMAPF::GetAgentPos's reference */
const gmapf_v2* gmapf_agent_pos_view(gmapf_ctx* ctx);
/* bulk copies of the host mirror */
gmapf_status gmapf_get_agents(gmapf_ctx* ctx, gmapf_v2* pos, int32_t* state, int32_t n);
int32_t gmapf_agent_count(gmapf_ctx* ctx);

/* GMAPF::ProfilerDump()                  -- src/GMAPF.cu:326-356 */
gmapf_status gmapf_profiler_dump(gmapf_ctx* ctx);

/* ---- inspection (tests, benchmarks, tools); not in the reference API ---- */
int32_t gmapf_map_count(gmapf_ctx* ctx);
gmapf_status gmapf_get_map_nodes(gmapf_ctx* ctx, gmapf_node* out, int32_t cap);
/* host point location with CuNodesMap::TryGetNodeIdx semantics (first
 * triangle in index order), grid-accelerated; -1 when outside */
gmapf_status gmapf_locate_points(gmapf_ctx* ctx, const gmapf_v2* pts, int32_t n, int32_t* out_node);
/* full device agent state, downloaded synchronously (no step may be running) */
gmapf_status gmapf_debug_get_agents(gmapf_ctx* ctx, gmapf_v2* pos, int32_t* state, int32_t* cur_node,
                                    int32_t* targ_node, int32_t* step_idx, int32_t* step_node,
                                    gmapf_v2* step_pos, int32_t* path_len);
/* path of one agent (device download); returns its length in *out_len */
gmapf_status gmapf_debug_get_path(gmapf_ctx* ctx, int32_t agent_id, int32_t* out, int32_t cap, int32_t* out_len);
/* statistics of the last completed step */
gmapf_status gmapf_last_step_stats(gmapf_ctx* ctx, gmapf_step_stats* out);
/* wall-time percentiles (ms) over the recorded steps; q in [0,100] */
gmapf_status gmapf_step_time_percentile(gmapf_ctx* ctx, float q, float* out_ms);
gmapf_status gmapf_reset_profiler(gmapf_ctx* ctx);
/* number of kernel launches issued by the library since creation */
int64_t gmapf_kernel_launches(gmapf_ctx* ctx);
/* the CUDA stream (cudaStream_t) the library launches on, for callers that
 * time or order their own work against it; null before the start */
void* gmapf_stream_handle(gmapf_ctx* ctx);
/* effective search shape after the start: threads per agent, queue
 * capacity, block size, visited mode (1 shared bitmap, 2 global records,
 * 3 global bitmap) and resident request slots */
gmapf_status gmapf_search_shape(gmapf_ctx* ctx, int32_t* T, int32_t* C, int32_t* block_threads,
                                int32_t* visited_mode, int32_t* slots);
/* Autotuner cache (no reference counterpart): with a file set, the shape the
 * autotuner picks for this map, GPU, search parameters and options is kept
 * there (one text line) and later starts with the same inputs take it from
 * the file instead of tuning again (the tuning takes seconds on large maps).
 * Set before the start; NULL or "" turns it off.  A file that cannot be read
 * or written only costs the time of tuning. */
gmapf_status gmapf_set_tune_cache(gmapf_ctx* ctx, const char* path);
/* Search timeline (diagnostics, no reference counterpart): with a device
 * buffer of 2 x rows uint64 set, each later gmapf_search_batch_host/_device
 * call of at most `rows` requests writes for request i the GPU global timer
 * (ns) when a warp took it, at [2i], and when its results were written, at
 * [2i + 1].  A larger batch is rejected (GMAPF_E_INVALID_ARG).  NULL turns it
 * off.  Frames are not recorded. */
gmapf_status gmapf_set_search_timeline(gmapf_ctx* ctx, uint64_t* d_timeline, int32_t rows);
/* how the started context's search shape was chosen: 0 the Config's (no
 * autotune), 1 tuned at the start, 2 taken from the autotuner cache */
gmapf_status gmapf_tune_source(gmapf_ctx* ctx, int32_t* source);

/* ---- batched query API: searches only, no agents ---- */
/* Run n independent searches (start/target node ids) with the context's
 * map and search parameters; writes found flags, lengths and paths
 * (path i at paths[i * path_stride]).  Inputs and outputs are host
 * buffers; copies are inside the call. */
gmapf_status gmapf_search_batch_host(gmapf_ctx* ctx, const int32_t* starts, const int32_t* targets,
                                     int32_t n, int32_t* found, int32_t* lens, int32_t* paths,
                                     int32_t path_stride, gmapf_step_stats* stats);
/* Same with device pointers already resident in HBM (no copies); ordered
 * on the context's stream; synchronous.  Buffers must be GPU memory
 * (device, managed or mapped pinned); pageable host memory is refused with
 * GMAPF_E_INVALID_ARG before anything runs. */
gmapf_status gmapf_search_batch_device(gmapf_ctx* ctx, const int32_t* d_starts, const int32_t* d_targets,
                                       int32_t n, int32_t* d_found, int32_t* d_lens, int32_t* d_paths,
                                       int32_t path_stride, gmapf_step_stats* stats);
/* device time (ms) of the last batch search kernel, measured with CUDA
 * events on the launching stream */
gmapf_status gmapf_last_search_ms(gmapf_ctx* ctx, float* out_ms);

/* ---- scene batches: several maps stepped as one ----
 * The reference runs one map per GMAPF instance (a second FillMap* throws
 * "map is already filled", GMAPF.cu:205-206), so a program with several
 * scenes creates several instances and steps them in turn.  A scene batch
 * keeps those instances as they are -- each scene is an ordinary context,
 * initialised, filled and given its agents through the calls above -- and
 * steps all of them with one compaction, one persistent search launch and one
 * mover pass per frame.  Each scene keeps its own Config (radius, speed,
 * PathFinderParallelAgents, agent count); threads per agent, queue capacity
 * and heuristic K must be equal across the scenes (they shape the one search
 * launch).  Results per scene equal those of that scene stepped alone.
 *
 * After gmapf_batch_create the scene contexts stay valid for their per-agent
 * calls (gmapf_set_agent_targ_pos[_bulk], gmapf_get_agent_pos/state,
 * gmapf_get_agents, gmapf_agent_pos_view, gmapf_debug_get_agents/path,
 * gmapf_locate_points and the map queries), with the scene's own agent and
 * triangle ids; stepping, options, statistics and profiling go through the
 * world context that gmapf_batch_world returns (gmapf_manual_start,
 * gmapf_async_step, gmapf_wait_step_end, gmapf_last_step_stats, ...).  On
 * the world, agent and triangle ids are global: scene s's agents start at
 * agent_base and its triangles at node_base (gmapf_batch_scene_base);
 * gmapf_set_agent_targ_pos_device on the world takes global agent ids and
 * locates each target in its agent's scene.  Calls that would change a
 * scene's map, agent set or options, or step it alone, return GMAPF_E_STATE. */
typedef struct gmapf_batch gmapf_batch;
/* Bind n >= 1 scene contexts (initialised, map filled, not started, not in
 * another batch) into a batch; opt (may be null) holds the world's step
 * options (mode, device, block size, visited mode, autotune). */
gmapf_status gmapf_batch_create(gmapf_ctx* const* scenes, int32_t n, const gmapf_options* opt,
                                gmapf_batch** out);
/* Free the world; the scene contexts then answer GMAPF_E_STATE to agent calls
 * and may only be destroyed. */
gmapf_status gmapf_batch_destroy(gmapf_batch* batch);
/* the world context (owned by the batch; do not destroy it) */
gmapf_ctx* gmapf_batch_world(gmapf_batch* batch);
/* first global agent id and first global triangle id of scene s */
gmapf_status gmapf_batch_scene_base(gmapf_batch* batch, int32_t scene, int32_t* agent_base, int32_t* node_base);

/* ---- serving: retargets admitted continuously ----
 * No counterpart in the reference, where a retarget waits for the next
 * AsyncStep and that frame's search (src/GMAPF.cu:238-289).  After
 * gmapf_serve_start, gmapf_serve_submit turns each retarget into a query at
 * once: its start is the triangle under the agent at submission, it enters a
 * device ring (capacity set by free device memory; the rest waits on the
 * host), and each poll launches the newly admitted queries as a batch on one
 * of several streams, each with its own search slots, so queries that arrive
 * while others run start without waiting for them.  Frames keep running: at each AsyncStep the finished queries' paths are
 * installed into their agents (unless a newer query of the same agent was
 * submitted), before the frame's compaction and mover; until then an agent
 * keeps its previous motion.  A query's result depends only on its start,
 * target and the map, so it is the same alone and among any other queries.
 * Latency is measured from the arrival time passed in (host steady clock, see
 * gmapf_clock_ns; now if null) to the poll that sees the query finished.  On a
 * scene batch call these on the world (global agent ids); on a bound scene,
 * gmapf_serve_submit takes the scene's own agent ids. */
typedef struct gmapf_serve_stats {
    int64_t submitted, admitted, completed, found;
    int64_t applied;     /* results installed into agents */
    int64_t superseded;  /* results dropped: a newer query of the same agent came */
    int64_t waiting;     /* submitted, not yet admitted (ring full) */
    int64_t in_flight;   /* admitted, not finished */
    int64_t launches;    /* batch launches */
    int64_t latency_samples;
    int32_t capacity;    /* ring entries (queries in flight at most) */
    int32_t slots;       /* search slots over all serving streams */
    float latency_p50_ms, latency_p99_ms, latency_mean_ms, latency_max_ms;
} gmapf_serve_stats;
/* allocate the ring (at most max_in_flight entries, 0: up to 65,536, fewer if
 * free memory is short) and the serving search state; starts the context */
gmapf_status gmapf_serve_start(gmapf_ctx* ctx, int32_t max_in_flight);
/* queue n retargets (agent ids, target positions, arrival times or null) */
gmapf_status gmapf_serve_submit(gmapf_ctx* ctx, const int32_t* ids, const gmapf_v2* targets, int32_t n,
                                const int64_t* arrival_ns);
/* harvest finished queries, admit waiting ones and launch them; call it
 * often: latency is counted to the poll that sees a query finished */
gmapf_status gmapf_serve_poll(gmapf_ctx* ctx);
/* poll until every submitted query has finished (or timeout_s passes:
 * GMAPF_E_DEVICE_TIMEOUT) */
gmapf_status gmapf_serve_drain(gmapf_ctx* ctx, float timeout_s);
/* counters and latency percentiles since the last reset */
gmapf_status gmapf_serve_get_stats(gmapf_ctx* ctx, gmapf_serve_stats* out, int32_t reset);
/* an agent's finished query not yet installed by a frame: found flag, length
 * and up to cap path triangles (global ids on a world) */
gmapf_status gmapf_serve_result(gmapf_ctx* ctx, int32_t agent, int32_t* found, int32_t* len, int32_t* path,
                                int32_t cap);
/* stop serving and free its memory (pending queries are dropped) */
gmapf_status gmapf_serve_stop(gmapf_ctx* ctx);
/* the host clock arrival times are measured in (steady clock, ns) */
int64_t gmapf_clock_ns(void);

/* ---- searches without any memory allocation ----
 * No counterpart in the reference.  For callers that may not allocate
 * device memory themselves or through the library (an engine that owns every
 * GPU allocation, memory fully reserved, allocation not allowed at the point
 * of the call): no context, no cudaMalloc, no cudaFree.  The caller passes
 * the navmesh (n_nodes gmapf_node records, neighbours packed and -1 padded,
 * as for FillMapManually; centroids are recomputed), the start/target
 * triangle ids and the outputs, all in memory the current GPU can reach
 * (its device memory, managed or mapped pinned; anything else is refused with
 * GMAPF_E_INVALID_ARG before a launch); results equal
 * gmapf_search_batch_device's for the same threads per agent and queue
 * capacity.  found[i] is 1 (found), 0 (not found), -1 for an id outside the
 * navmesh, or -2 when the search reached round_limit rounds before ending
 * (round_limit 0 means the default, 4 n_nodes + 64, which no search
 * reaches); a length above path_stride means path row i was left unwritten.
 * Working memory is one 64 MiB array built into the library (held by every
 * GPU that loads it until exit): the navmesh may have at most 2,097,144
 * triangles, and fewer triangles give more concurrent requests.  Calls share
 * that array: calls that overlap on the GPU race and must be serialized.
 * Enqueued on `stream` (a cudaStream_t, null for the default stream) and
 * asynchronous.  The first call on each device sets up the array's address,
 * and the first call with each (threads per agent, queue capacity) sets the
 * kernel's shared-memory limit, so make those before any stream capture.
 * Errors are read with gmapf_last_error(). */
gmapf_status gmapf_search_batch_noalloc(const gmapf_node* d_nodes, int32_t n_nodes, const int32_t* d_starts,
                                        const int32_t* d_targets, int32_t n_queries, int32_t threads_per_agent,
                                        int32_t queue_capacity, float heuristic_k, int32_t round_limit,
                                        int32_t* d_found, int32_t* d_lens, int32_t* d_paths, int32_t path_stride,
                                        void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GMAPF_C_H */
