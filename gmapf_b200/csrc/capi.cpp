// capi.cpp -- the C ABI (include/gmapf_c.h): lifecycle rules and host-side
// bookkeeping of gmapf::GMAPF (src/GMAPF.cu), with the reference's
// exceptions turned into status codes and a per-thread error message.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>

#include "internal.h"

using namespace gmapf_b200;

namespace gmapf_b200 {

// A pointer a kernel on `device` may be given: device memory of that GPU,
// managed memory or mapped host memory.  Pageable host memory (the usual
// mistake with the *_device entry points) and device memory of another GPU
// are refused before anything is launched, instead of faulting the GPU.
bool gpu_reachable(const void* p, int device) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeUnregistered) return false;
    if (a.type == cudaMemoryTypeDevice && a.device != device) return false;
    return true;
}

}  // namespace gmapf_b200

struct gmapf_batch;

struct gmapf_ctx {
    Context c;
    gmapf_batch* batch = nullptr;  // the batch this scene is bound to
    gmapf_ctx* world = nullptr;    // that batch's world
};

struct gmapf_batch {
    gmapf_ctx* world = nullptr;
    std::vector<gmapf_ctx*> scenes;
};

namespace {

thread_local std::string g_err;

gmapf_status fail(int code, const std::string& msg) {
    g_err = msg;
    return (gmapf_status)code;
}

#define NEED_CTX(ctx) \
    if (!(ctx)) return fail(GMAPF_E_INVALID_ARG, "null context")

// A scene bound to a batch: its agent calls go to the world (null if the
// scene is not bound); a scene whose batch was destroyed answers E_STATE.
#define SCENE_WORLD(ctx, w)                                                                  \
    if ((ctx)->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");   \
    gmapf_ctx* w = (ctx)->world

gmapf_status scene_only(const char* what) {
    return fail(GMAPF_E_STATE, std::string(what) + ": this scene is stepped by its batch (use the batch's world)");
}

// PathFinder threads per agent: the reference packs 128/T requests per block
// (PathFinder.h:559-572) and seeds lanes 0 and 1 (PathFinder.h:168-189).
bool valid_T(int t) { return t == 2 || t == 4 || t == 8 || t == 16 || t == 32; }

int locate_host(const Context& c, float x, float y) {
    LocateGrid g = c.map.view();
    return locate(g, x, y);
}

std::string v2s(float x, float y) {
    char b[96];
    std::snprintf(b, sizeof(b), "(%f, %f)", x, y);
    return b;
}

int add_dirty(Context& c, int id, int node, float x, float y) {
    int4 r;
    r.x = id;
    r.y = node;
    std::memcpy(&r.z, &x, 4);
    std::memcpy(&r.w, &y, 4);
    int& slot = c.dirty_slot[id];
    if (slot >= 0)
        c.dirty_recs[slot] = r;
    else {
        slot = (int)c.dirty_recs.size();
        c.dirty_recs.push_back(r);
    }
    return GMAPF_OK;
}

uint64_t cdt_input_hash(const Context& c);  // navmesh files, below
int autotune_at_start(Context& c, std::string& err);  // autotuner cache, below

gmapf_status start_if_needed(Context& c) {
    if (c.started) return GMAPF_OK;
    if (!c.map_filled) return fail(GMAPF_E_STATE, "map is not filled");
    std::string err;
    int rc = device_start(c, err);
    if (rc) {
        device_free(c);
        return fail(rc, err);
    }
    c.started = true;
    c.tune_source = 0;
    if (c.opt.autotune) {
        rc = autotune_at_start(c, err);
        if (rc) return fail(rc, err);
    }
    return GMAPF_OK;
}

}  // namespace

namespace gmapf_b200 {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace gmapf_b200

extern "C" {

const char* gmapf_last_error(void) { return g_err.c_str(); }

gmapf_status gmapf_create(gmapf_ctx** out) {
    if (!out) return fail(GMAPF_E_INVALID_ARG, "null output pointer");
    *out = new (std::nothrow) gmapf_ctx();
    if (!*out) return fail(GMAPF_E_CAPACITY, "out of host memory");
    (*out)->c.opt.device = 0;
    (*out)->c.opt.mode = GMAPF_MODE_BATCHED;
    (*out)->c.opt.order_by_estimate = 1;
    return GMAPF_OK;
}

gmapf_status gmapf_destroy(gmapf_ctx* ctx) {
    if (!ctx) return GMAPF_OK;
    Context& c = ctx->c;
    if (c.is_world) return fail(GMAPF_E_STATE, "the world context belongs to its batch: destroy the batch");
    if (ctx->batch) {
        auto& v = ctx->batch->scenes;
        v.erase(std::remove(v.begin(), v.end(), ctx), v.end());
    }
    if (c.started && c.scene_index < 0) {  // a batch's scene holds no device state
        if (c.step_going) {
            std::string err;
            device_wait_step(c, err);
            c.step_going = false;
        }
        device_free(c);
    }
    delete ctx;
    return GMAPF_OK;
}

gmapf_status gmapf_init(gmapf_ctx* ctx, const gmapf_config* cfg) {
    NEED_CTX(ctx);
    if (!cfg) return fail(GMAPF_E_INVALID_ARG, "null config");
    Context& c = ctx->c;
    if (c.inited) return fail(GMAPF_E_STATE, "already initialized");
    if (cfg->AgentsMaxCount < 0) return fail(GMAPF_E_INVALID_ARG, "AgentsMaxCount must be >= 0");
    if (!valid_T(cfg->PathFinderThreadsPerAgents))
        return fail(GMAPF_E_INVALID_ARG, "PathFinderThreadsPerAgents must be one of 2, 4, 8, 16, 32");
    // the per-lane queues live in shared memory (12 bytes per entry per thread)
    if (cfg->PathFinderQueueCapacity < 1 || cfg->PathFinderQueueCapacity > 512)
        return fail(GMAPF_E_INVALID_ARG, "PathFinderQueueCapacity must be in [1, 512]");
    if (cfg->PathFinderParallelAgents < 0) return fail(GMAPF_E_INVALID_ARG, "PathFinderParallelAgents must be >= 0");
    c.cfg = *cfg;
    c.T = cfg->PathFinderThreadsPerAgents;
    c.C = cfg->PathFinderQueueCapacity;
    c.K = cfg->PathFinderHeuristicK;
    c.block_threads = 128;
    const int cap = cfg->AgentsMaxCount;
    c.m_pos.reserve(cap);
    c.m_state.reserve(cap);
    c.m_cur.reserve(cap);
    c.m_targ.reserve(cap);
    c.m_targ_node.reserve(cap);
    c.dirty_slot.reserve(cap);
    c.inited = true;
    return GMAPF_OK;
}

gmapf_status gmapf_set_options(gmapf_ctx* ctx, const gmapf_options* o) {
    NEED_CTX(ctx);
    if (!o) return fail(GMAPF_E_INVALID_ARG, "null options");
    Context& c = ctx->c;
    if (c.started) return fail(GMAPF_E_STATE, "options must be set before start");
    if (o->mode != GMAPF_MODE_BATCHED && o->mode != GMAPF_MODE_PLAIN)
        return fail(GMAPF_E_INVALID_ARG, "unknown mode");
    if (o->block_threads != 0 &&
        (o->block_threads < 32 || o->block_threads > 256 || o->block_threads % 32 != 0))
        return fail(GMAPF_E_INVALID_ARG, "block_threads must be 0 or a multiple of 32 in [32, 256]");
    if (o->device < 0) return fail(GMAPF_E_INVALID_ARG, "device must be >= 0");
    if (o->visited_mode < 0 || o->visited_mode > 4)
        return fail(GMAPF_E_INVALID_ARG, "visited_mode must be 0 (automatic), 1, 2, 3 or 4");
    if (o->round_limit < 0) return fail(GMAPF_E_INVALID_ARG, "round_limit must be >= 0 (0: no practical limit)");
    if (o->promote_rounds < 0) return fail(GMAPF_E_INVALID_ARG, "promote_rounds must be >= 0 (0: 512)");
    if (o->path_smoothing < 0 || o->path_smoothing > 2)
        return fail(GMAPF_E_INVALID_ARG, "path_smoothing must be 0 (off), 1 (funnel corners) or 2 (corners one agent radius off the walls)");
    c.opt = *o;
    if (o->block_threads) c.block_threads = o->block_threads;
    return GMAPF_OK;
}

gmapf_status gmapf_get_options(gmapf_ctx* ctx, gmapf_options* out) {
    NEED_CTX(ctx);
    if (!out) return fail(GMAPF_E_INVALID_ARG, "null output");
    *out = ctx->c.opt;
    out->block_threads = ctx->c.block_threads;
    return GMAPF_OK;
}

gmapf_status gmapf_fill_map_start(gmapf_ctx* ctx, float sx, float sy) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    // src/GMAPF.cu:133-145
    c.cdt_v = {0.f, 0.f, 0.f, sy, sx, sy, sx, 0.f};
    c.cdt_e = {0, 1, 1, 2, 2, 3, 3, 0};
    return GMAPF_OK;
}

gmapf_status gmapf_fill_map_obstacle(gmapf_ctx* ctx, const gmapf_v2* v, int32_t count) {
    NEED_CTX(ctx);
    if (count > 0 && !v) return fail(GMAPF_E_INVALID_ARG, "null vertices");
    if (count <= 0) return fail(GMAPF_E_INVALID_ARG, "an obstacle needs at least one vertex");
    Context& c = ctx->c;
    // src/GMAPF.cu:147-159: a closed polygon
    const unsigned start = (unsigned)(c.cdt_v.size() / 2);
    for (int i = 0; i < count; i++) {
        const unsigned idx = (unsigned)(c.cdt_v.size() / 2);
        c.cdt_v.push_back(v[i].X);
        c.cdt_v.push_back(v[i].Y);
        if (i > 0) {
            c.cdt_e.push_back(idx - 1);
            c.cdt_e.push_back(idx);
        }
    }
    c.cdt_e.push_back((unsigned)(c.cdt_v.size() / 2 - 1));
    c.cdt_e.push_back(start);
    return GMAPF_OK;
}

gmapf_status gmapf_fill_map_manually(gmapf_ctx* ctx, const gmapf_node* nodes, int32_t count);

gmapf_status gmapf_fill_map_end(gmapf_ctx* ctx) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.started) return fail(GMAPF_E_STATE, "cannot modify map after start");
    if (c.map_filled) return fail(GMAPF_E_STATE, "map is already filled");
    std::vector<gmapf_node> nodes;
    std::string err;
    int rc = build_navmesh_cdt(c.cdt_v, c.cdt_e, nodes, err);
    if (rc) return fail(rc, err);
    gmapf_status s = gmapf_fill_map_manually(ctx, nodes.data(), (int32_t)nodes.size());
    if (s == GMAPF_OK) c.map_input_hash = cdt_input_hash(c);
    return s;
}

gmapf_status gmapf_fill_map_manually(gmapf_ctx* ctx, const gmapf_node* nodes, int32_t count) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    // src/GMAPF.cu:199-217
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.started) return fail(GMAPF_E_STATE, "cannot modify map after start");
    if (c.map_filled) return fail(GMAPF_E_STATE, "map is already filled");
    if (count < 0 || (count > 0 && !nodes)) return fail(GMAPF_E_INVALID_ARG, "bad node array");
    for (int i = 0; i < count; i++)
        for (int k = 0; k < 3; k++) {
            const int nb = nodes[i].NeibsIdx[k];
            if (nb < -1 || nb >= count)
                return fail(GMAPF_E_INVALID_ARG, "node " + std::to_string(i) + " has neighbour " +
                                                     std::to_string(nb) + " outside the map");
        }
    build_host_map(nodes, count, c.map);
    c.map_filled = true;
    return GMAPF_OK;
}

// ------------------------------------------------------------ navmesh files --

}  // extern "C"

namespace {

const char kMapMagic[8] = {'G', 'M', 'A', 'P', 'F', 'N', 'M', '1'};

struct MapFileHeader {
    char magic[8];
    uint32_t version;
    int32_t count;
    uint64_t input_hash;  // FNV-1a of the FillMapStart/FillMapObstacle input (0: none)
    uint64_t checksum;    // FNV-1a of the node records
};

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < bytes; i++) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

// ---- autotuner cache ----------------------------------------------------
// One text line per tuned (map, GPU, options):
//   gmapf-tune 1 <key, 16 hex digits> <T> <C> <visited placement> <block>
// The key hashes the search graph and its geometry, the search parameters and
// options the tuner reads, the GPU (name, SM count, memory) and this build,
// so a changed map, GPU, option or library never reuses a stale shape.
// Unreadable or foreign lines are skipped; the last matching line wins.
const char kTuneBuild[] = "gmapf-tune 2 " __DATE__ " " __TIME__;

uint64_t tune_key(const Context& c) {
    const HostMap& m = c.map;
    uint64_t h = fnv1a(kTuneBuild, sizeof(kTuneBuild));
    h = fnv1a(&m.n, sizeof(m.n), h);
    h = fnv1a(m.rows.data(), sizeof(SearchRow) * m.rows.size(), h);
    h = fnv1a(m.cen.data(), sizeof(float2) * m.cen.size(), h);
    const int32_t iv[] = {c.cfg.PathFinderParallelAgents, c.cfg.PathFinderThreadsPerAgents,
                          c.cfg.PathFinderQueueCapacity, c.opt.visited_mode, c.opt.block_threads, c.opt.mode};
    h = fnv1a(iv, sizeof(iv), h);
    h = fnv1a(&c.cfg.PathFinderHeuristicK, sizeof(float), h);
    h = fnv1a(&c.opt.search_mem_budget, sizeof(c.opt.search_mem_budget), h);
    cudaDeviceProp pr{};
    if (cudaGetDeviceProperties(&pr, c.dev.device) == cudaSuccess) {
        h = fnv1a(pr.name, std::strlen(pr.name), h);
        h = fnv1a(&pr.multiProcessorCount, sizeof(pr.multiProcessorCount), h);
        h = fnv1a(&pr.totalGlobalMem, sizeof(pr.totalGlobalMem), h);
    } else {
        cudaGetLastError();
    }
    return h;
}

bool tune_lookup(const std::string& path, uint64_t key, int v[4]) {
    std::FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    bool hit = false;
    char line[256];
    while (std::fgets(line, sizeof(line), f)) {
        unsigned long long k = 0;
        int fmt = 0, T = 0, C = 0, vm = 0, bt = 0;
        if (std::sscanf(line, "gmapf-tune %d %16llx %d %d %d %d", &fmt, &k, &T, &C, &vm, &bt) != 6) continue;
        if (fmt != 1 || k != key) continue;
        const bool t_ok = T == 2 || T == 4 || T == 8 || T == 16 || T == 32;
        if (!t_ok || C < 1 || vm < 0 || vm > 4 || bt < 0 || bt > 1024) continue;
        v[0] = T, v[1] = C, v[2] = vm, v[3] = bt;
        hit = true;
    }
    std::fclose(f);
    return hit;
}

void tune_store(const std::string& path, uint64_t key, const Context& c) {
    std::FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return;  // the cache only saves time: a start never fails on it
    std::fprintf(f, "gmapf-tune 1 %016llx %d %d %d %d\n", (unsigned long long)key, c.T, c.C, c.tuned_vm,
                 c.tuned_bt);
    std::fclose(f);
}

int autotune_at_start(Context& c, std::string& err) {
    uint64_t key = 0;
    if (!c.tune_cache.empty()) {
        key = tune_key(c);
        int v[4];
        if (tune_lookup(c.tune_cache, key, v)) {
            const int rc = device_apply_tuned_shape(c, v[0], v[1], v[2], v[3], err);
            if (rc == GMAPF_OK) {
                c.tune_source = 2;
                return GMAPF_OK;
            }
            // the stored shape does not fit this process (memory): tune again
            err.clear();
        }
    }
    const int rc = device_autotune(c, err);
    if (rc) return rc;
    c.tune_source = 1;
    if (!c.tune_cache.empty()) tune_store(c.tune_cache, key, c);
    return GMAPF_OK;
}

uint64_t cdt_input_hash(const Context& c) {
    uint64_t h = fnv1a(c.cdt_v.data(), sizeof(float) * c.cdt_v.size());
    h = fnv1a(c.cdt_e.data(), sizeof(unsigned) * c.cdt_e.size(), h);
    return h ? h : 1;
}

int write_map(const std::vector<gmapf_node>& nodes, uint64_t input_hash, const char* path, std::string& err) {
    MapFileHeader hd{};
    std::memcpy(hd.magic, kMapMagic, 8);
    hd.version = 1;
    hd.count = (int32_t)nodes.size();
    hd.input_hash = input_hash;
    hd.checksum = fnv1a(nodes.data(), sizeof(gmapf_node) * nodes.size());
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        err = std::string("cannot open ") + path + " for writing";
        return GMAPF_E_INVALID_ARG;
    }
    bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1;
    if (ok && !nodes.empty()) ok = std::fwrite(nodes.data(), sizeof(gmapf_node), nodes.size(), f) == nodes.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        err = std::string("cannot write ") + path;
        return GMAPF_E_INVALID_ARG;
    }
    return GMAPF_OK;
}

int read_map(const char* path, std::vector<gmapf_node>& nodes, uint64_t& input_hash, std::string& err) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) {
        err = std::string("cannot open ") + path;
        return GMAPF_E_INVALID_ARG;
    }
    MapFileHeader hd{};
    bool ok = std::fread(&hd, sizeof(hd), 1, f) == 1 && std::memcmp(hd.magic, kMapMagic, 8) == 0 && hd.version == 1 &&
              hd.count >= 0 && hd.count <= (1 << 27);
    if (ok) {
        nodes.resize(hd.count);
        ok = hd.count == 0 || std::fread(nodes.data(), sizeof(gmapf_node), hd.count, f) == (size_t)hd.count;
        char extra;
        ok = ok && std::fread(&extra, 1, 1, f) == 0;  // nothing after the records
    }
    std::fclose(f);
    if (ok) ok = fnv1a(nodes.data(), sizeof(gmapf_node) * nodes.size()) == hd.checksum;
    if (!ok) {
        err = std::string(path) + " is not an intact navmesh file";
        return GMAPF_E_INVALID_ARG;
    }
    input_hash = hd.input_hash;
    return GMAPF_OK;
}

}  // namespace

extern "C" {

gmapf_status gmapf_map_save(gmapf_ctx* ctx, const char* path) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (!path) return fail(GMAPF_E_INVALID_ARG, "null path");
    if (!c.map_filled) return fail(GMAPF_E_STATE, "map is not filled");
    std::string err;
    int rc = write_map(c.map.nodes, c.map_input_hash, path, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_map_load(gmapf_ctx* ctx, const char* path) {
    NEED_CTX(ctx);
    if (!path) return fail(GMAPF_E_INVALID_ARG, "null path");
    std::vector<gmapf_node> nodes;
    uint64_t h = 0;
    std::string err;
    int rc = read_map(path, nodes, h, err);
    if (rc) return fail(rc, err);
    gmapf_status s = gmapf_fill_map_manually(ctx, nodes.data(), (int32_t)nodes.size());
    if (s == GMAPF_OK) ctx->c.map_input_hash = h;
    return s;
}

gmapf_status gmapf_fill_map_end_cached(gmapf_ctx* ctx, const char* path, int32_t* hit) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (!path) return fail(GMAPF_E_INVALID_ARG, "null path");
    if (hit) *hit = 0;
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.started) return fail(GMAPF_E_STATE, "cannot modify map after start");
    if (c.map_filled) return fail(GMAPF_E_STATE, "map is already filled");
    const uint64_t want = cdt_input_hash(c);
    {
        std::vector<gmapf_node> nodes;
        uint64_t h = 0;
        std::string err;
        if (read_map(path, nodes, h, err) == GMAPF_OK && h == want &&
            gmapf_fill_map_manually(ctx, nodes.data(), (int32_t)nodes.size()) == GMAPF_OK) {
            c.map_input_hash = want;
            if (hit) *hit = 1;
            return GMAPF_OK;
        }
    }
    gmapf_status s = gmapf_fill_map_end(ctx);
    if (s != GMAPF_OK) return s;
    std::string err;
    int rc = write_map(c.map.nodes, want, path, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_add_agent(gmapf_ctx* ctx, float x, float y, int32_t* out_id) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    // src/GMAPF.cu:219-236
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.is_world) return fail(GMAPF_E_STATE, "agents are added to the scene contexts");
    if (c.started) return fail(GMAPF_E_STATE, "cannot add agents after start");
    if (!c.map_filled) return fail(GMAPF_E_STATE, "map is not filled");
    if (c.A >= c.cfg.AgentsMaxCount) return fail(GMAPF_E_CAPACITY, "AgentsMaxCount reached");
    const int node = locate_host(c, x, y);
    if (node < 0) return fail(GMAPF_E_INVALID_POS, "initial pos " + v2s(x, y) + " is invalid");
    c.m_pos.push_back(gmapf_v2{x, y});
    c.m_state.push_back(GMAPF_AGENT_IDLE);
    c.m_cur.push_back(node);
    c.m_targ.push_back(gmapf_v2{0.f, 0.f});
    c.m_targ_node.push_back(-1);
    c.dirty_slot.push_back(-1);
    if (out_id) *out_id = c.A;
    c.A++;
    return GMAPF_OK;
}

namespace {
// SetAgentTargPos with the target's triangle already located (node = -2: locate here)
gmapf_status set_target_located(gmapf_ctx* ctx, int32_t id, float x, float y, int node);
}  // namespace

gmapf_status gmapf_set_agent_targ_pos(gmapf_ctx* ctx, int32_t id, float x, float y) {
    return set_target_located(ctx, id, x, y, -2);
}

}  // extern "C"

namespace {
gmapf_status set_target_located(gmapf_ctx* ctx, int32_t id, float x, float y, int located) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    SCENE_WORLD(ctx, w);
    if (c.is_world)
        return fail(GMAPF_E_STATE, "targets are set through the scene contexts (or gmapf_set_agent_targ_pos_device)");
    if (w) {
        if (id < 0 || id >= c.A) return fail(GMAPF_E_INVALID_ARG, "agent id " + std::to_string(id) + " out of range");
        const int node = located == -2 ? locate_host(c, x, y) : located;
        if (node < 0) return fail(GMAPF_E_INVALID_POS, "target pos " + v2s(x, y) + " is invalid");
        Context& wc = w->c;
        const int gid = c.agent_base + id, gnode = c.node_base + node;
        wc.m_state[gid] = GMAPF_AGENT_SEARCH;
        wc.m_targ[gid] = gmapf_v2{x, y};
        wc.m_targ_node[gid] = gnode;
        if (wc.started) add_dirty(wc, gid, gnode, x, y);
        return GMAPF_OK;
    }
    // src/GMAPF.cu:238-253
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (!c.map_filled) return fail(GMAPF_E_STATE, "map is not filled");
    if (id < 0 || id >= c.A) return fail(GMAPF_E_INVALID_ARG, "agent id " + std::to_string(id) + " out of range");
    const int node = located == -2 ? locate_host(c, x, y) : located;
    if (node < 0) return fail(GMAPF_E_INVALID_POS, "target pos " + v2s(x, y) + " is invalid");
    c.m_state[id] = GMAPF_AGENT_SEARCH;
    c.m_targ[id] = gmapf_v2{x, y};
    c.m_targ_node[id] = node;
    if (c.started) add_dirty(c, id, node, x, y);
    return GMAPF_OK;
}
}  // namespace

extern "C" {

gmapf_status gmapf_set_agent_targ_pos_bulk(gmapf_ctx* ctx, const int32_t* ids, const gmapf_v2* pos, int32_t n) {
    NEED_CTX(ctx);
    if (n < 0 || (n > 0 && (!ids || !pos))) return fail(GMAPF_E_INVALID_ARG, "bad bulk arrays");
    Context& c = ctx->c;
    std::vector<int> node(n, -2);
    if (n >= 2048 && c.map_filled && c.started && !c.is_world && !c.detached && !ctx->world) {
        // point location is the cost of a large retarget: on the device (its own
        // stream: a running frame is not waited for), then applied in order
        // below (the first invalid item stops the call)
        std::string err;
        const int rc = device_locate_points(c, pos, n, node.data(), err);
        if (rc) return fail(rc, err);
    } else if (n >= 2048 && c.map_filled && !c.is_world && !c.detached) {
        // before start: split it over host threads
        const LocateGrid g = c.map.view();
        const int nt = std::max(1, std::min<int>(8, (int)std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (int t = 0; t < nt; t++)
            th.emplace_back([&, t]() {
                for (int k = t; k < n; k += nt) node[k] = locate(g, pos[k].X, pos[k].Y);
            });
        for (std::thread& x : th) x.join();
    }
    for (int k = 0; k < n; k++) {
        gmapf_status s = set_target_located(ctx, ids[k], pos[k].X, pos[k].Y, node[k]);
        if (s != GMAPF_OK) return s;
    }
    return GMAPF_OK;
}

gmapf_status gmapf_set_agent_targ_pos_device(gmapf_ctx* ctx, const int32_t* d_ids, const gmapf_v2* d_pos,
                                             int32_t n) {
    NEED_CTX(ctx);
    SCENE_WORLD(ctx, w);
    // a bound scene's ids are its own: offset into the world's agents
    Context& c = w ? w->c : ctx->c;
    const int id_base = w ? ctx->c.agent_base : 0, id_count = w ? ctx->c.A : c.A;
    if (!c.started) return fail(GMAPF_E_STATE, "not started");
    if (c.step_going) return fail(GMAPF_E_STATE, "a step is running");
    if (n < 0 || (n > 0 && (!d_ids || !d_pos))) return fail(GMAPF_E_INVALID_ARG, "bad device arrays");
    if (n > 0 && !(gpu_reachable(d_ids, c.opt.device) && gpu_reachable(d_pos, c.opt.device)))
        return fail(GMAPF_E_INVALID_ARG, "a buffer is not memory the context's GPU can reach (its device memory, managed or mapped pinned)");
    if (n == 0) return GMAPF_OK;
    std::string err;
    int rc = device_set_targets_device(c, d_ids, d_pos, n, id_base, id_count, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_manual_start(gmapf_ctx* ctx) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (ctx->world || c.detached) return scene_only("ManualStart");
    // src/GMAPF.cu:72-130
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.started) return fail(GMAPF_E_STATE, "already started");
    return start_if_needed(c);
}

gmapf_status gmapf_async_step(gmapf_ctx* ctx, float dt) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (ctx->world || c.detached) return scene_only("AsyncStep");
    // src/GMAPF.cu:255-289
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.step_going) return GMAPF_OK;
    gmapf_status s = start_if_needed(c);
    if (s != GMAPF_OK) return s;
    std::string err;
    int rc = device_async_step(c, dt, err);
    if (rc) return fail(rc, err);
    c.step_going = true;
    return GMAPF_OK;
}

gmapf_status gmapf_wait_step_end(gmapf_ctx* ctx) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (ctx->world || c.detached) return scene_only("WaitStepEnd");
    // src/GMAPF.cu:291-314
    if (!c.step_going) return GMAPF_OK;
    std::string err;
    int rc = device_wait_step(c, err);
    c.step_going = false;
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

int32_t gmapf_step_ready(gmapf_ctx* ctx) {
    if (!ctx) return 1;
    if (ctx->world) ctx = ctx->world;
    Context& c = ctx->c;
    if (!c.step_going) return 1;
    return device_step_ready(c) ? 1 : 0;
}

gmapf_status gmapf_get_agent_pos(gmapf_ctx* ctx, int32_t id, gmapf_v2* out) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    SCENE_WORLD(ctx, w);
    if (id < 0 || id >= c.A || !out) return fail(GMAPF_E_INVALID_ARG, "agent id out of range");
    *out = w ? w->c.m_pos[c.agent_base + id] : c.m_pos[id];
    return GMAPF_OK;
}

gmapf_status gmapf_get_agent_state(gmapf_ctx* ctx, int32_t id, int32_t* out) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    SCENE_WORLD(ctx, w);
    if (id < 0 || id >= c.A || !out) return fail(GMAPF_E_INVALID_ARG, "agent id out of range");
    *out = w ? w->c.m_state[c.agent_base + id] : c.m_state[id];
    return GMAPF_OK;
}

const gmapf_v2* gmapf_agent_pos_view(gmapf_ctx* ctx) {
    if (!ctx || ctx->c.detached) return nullptr;
    if (ctx->world) return ctx->world->c.m_pos.data() + ctx->c.agent_base;
    return ctx->c.m_pos.data();
}

gmapf_status gmapf_get_agents(gmapf_ctx* ctx, gmapf_v2* pos, int32_t* state, int32_t n) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    SCENE_WORLD(ctx, w);
    if (n < 0 || n > c.A) return fail(GMAPF_E_INVALID_ARG, "n out of range");
    const Context& src = w ? w->c : c;
    const int b = w ? c.agent_base : 0;
    if (pos) std::memcpy(pos, src.m_pos.data() + b, sizeof(gmapf_v2) * n);
    if (state) std::memcpy(state, src.m_state.data() + b, sizeof(int32_t) * n);
    return GMAPF_OK;
}

int32_t gmapf_agent_count(gmapf_ctx* ctx) { return ctx ? ctx->c.A : 0; }

gmapf_status gmapf_profiler_dump(gmapf_ctx* ctx) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    if (ctx->world) ctx = ctx->world;
    Context& c = ctx->c;
    // src/GMAPF.cu:326-356, same line format
    if (!c.cfg.IsProfiler) return fail(GMAPF_E_STATE, "profiler disabled");
    const Profiler& p = c.prof;
    auto line = [](const char* t, float sum, float mx, int n) {
        std::printf("%s avg: %g max: %g\n", t, n > 0 ? sum / n : 0.0f, mx);
    };
    std::printf("[gmapf]----------------------\n");
    line("[gmapf] step", p.sum_wall, p.max_wall, p.n);
    line("[gmapf] ---step post copy", p.sum_post, p.max_post, p.n);
    std::printf("\n[gmapf] path finder\n");
    line("[gmapf] find requests", p.sum_compact, p.max_compact, p.n);
    line("[gmapf] search", p.sum_search, p.max_search, p.n_search);
    std::printf("\n[gmapf] agents mover\n");
    line("[gmapf] move+collisions+progress", p.sum_mover, p.max_mover, p.n_mover);
    std::printf("[gmapf]----------------------\n");
    std::fflush(stdout);
    return GMAPF_OK;
}

int32_t gmapf_map_count(gmapf_ctx* ctx) { return ctx ? ctx->c.map.n : 0; }

gmapf_status gmapf_get_map_nodes(gmapf_ctx* ctx, gmapf_node* out, int32_t cap) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (!c.map_filled) return fail(GMAPF_E_STATE, "map is not filled");
    if (!out || cap < c.map.n) return fail(GMAPF_E_INVALID_ARG, "output too small");
    std::memcpy(out, c.map.nodes.data(), sizeof(gmapf_node) * c.map.n);
    return GMAPF_OK;
}

gmapf_status gmapf_locate_points(gmapf_ctx* ctx, const gmapf_v2* pts, int32_t n, int32_t* out) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (c.is_world) return fail(GMAPF_E_STATE, "points are located in the scene contexts");
    if (!c.map_filled) return fail(GMAPF_E_STATE, "map is not filled");
    if (n < 0 || (n > 0 && (!pts || !out))) return fail(GMAPF_E_INVALID_ARG, "bad arrays");
    LocateGrid g = c.map.view();
    for (int i = 0; i < n; i++) out[i] = locate(g, pts[i].X, pts[i].Y);
    return GMAPF_OK;
}

gmapf_status gmapf_debug_get_agents(gmapf_ctx* ctx, gmapf_v2* pos, int32_t* state, int32_t* cur,
                                    int32_t* targ, int32_t* step_idx, int32_t* step_node,
                                    gmapf_v2* step_pos, int32_t* path_len) {
    NEED_CTX(ctx);
    SCENE_WORLD(ctx, w);
    if (w) {  // the world's arrays, this scene's slice, triangle ids made local
        Context& wc = w->c;
        const Context& c = ctx->c;
        if (!wc.started) return fail(GMAPF_E_STATE, "not started");
        if (wc.step_going) return fail(GMAPF_E_STATE, "a step is running");
        const int WA = wc.A, b = c.agent_base, A = c.A, nb = c.node_base;
        std::vector<gmapf_v2> p(WA), sp(WA);
        std::vector<int32_t> st(WA), cu(WA), tg(WA), si(WA), sn(WA), pl(WA);
        std::string err;
        int rc = device_debug_agents(wc, p.data(), st.data(), cu.data(), tg.data(), si.data(), sn.data(), sp.data(),
                                     pl.data(), err);
        if (rc) return fail(rc, err);
        auto local = [nb](int v) { return v >= 0 ? v - nb : v; };
        for (int i = 0; i < A; i++) {
            if (pos) pos[i] = p[b + i];
            if (state) state[i] = st[b + i];
            if (cur) cur[i] = local(cu[b + i]);
            if (targ) targ[i] = local(tg[b + i]);
            if (step_idx) step_idx[i] = si[b + i];
            if (step_node) step_node[i] = local(sn[b + i]);
            if (step_pos) step_pos[i] = sp[b + i];
            if (path_len) path_len[i] = pl[b + i];
        }
        return GMAPF_OK;
    }
    Context& c = ctx->c;
    if (!c.started) return fail(GMAPF_E_STATE, "not started");
    if (c.step_going) return fail(GMAPF_E_STATE, "a step is running");
    std::string err;
    int rc = device_debug_agents(c, pos, state, cur, targ, step_idx, step_node, step_pos, path_len, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_debug_get_path(gmapf_ctx* ctx, int32_t id, int32_t* out, int32_t cap, int32_t* out_len) {
    NEED_CTX(ctx);
    SCENE_WORLD(ctx, w);
    Context& c = w ? w->c : ctx->c;
    if (!c.started) return fail(GMAPF_E_STATE, "not started");
    if (c.step_going) return fail(GMAPF_E_STATE, "a step is running");
    if (id < 0 || id >= ctx->c.A || !out_len || (cap > 0 && !out)) return fail(GMAPF_E_INVALID_ARG, "bad arguments");
    std::string err;
    int rc = device_debug_path(c, w ? ctx->c.agent_base + id : id, out, cap, out_len, err);
    if (rc) return fail(rc, err);
    if (w)  // scene-local triangle ids
        for (int k = 0; k < std::min(*out_len, cap); k++) out[k] -= ctx->c.node_base;
    return GMAPF_OK;
}

gmapf_status gmapf_last_step_stats(gmapf_ctx* ctx, gmapf_step_stats* out) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    if (ctx->world) ctx = ctx->world;
    if (!out) return fail(GMAPF_E_INVALID_ARG, "null output");
    *out = ctx->c.last;
    return GMAPF_OK;
}

gmapf_status gmapf_step_time_percentile(gmapf_ctx* ctx, float q, float* out_ms) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    if (ctx->world) ctx = ctx->world;
    if (!out_ms || q < 0 || q > 100) return fail(GMAPF_E_INVALID_ARG, "bad arguments");
    std::vector<float> v = ctx->c.prof.wall_ms;
    if (v.empty()) {
        *out_ms = 0;
        return GMAPF_OK;
    }
    std::sort(v.begin(), v.end());
    // nearest-rank percentile
    size_t k = (size_t)std::ceil(q / 100.0 * v.size());
    if (k > 0) k--;
    if (k >= v.size()) k = v.size() - 1;
    *out_ms = v[k];
    return GMAPF_OK;
}

gmapf_status gmapf_reset_profiler(gmapf_ctx* ctx) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    if (ctx->world) ctx = ctx->world;
    ctx->c.prof = Profiler{};
    return GMAPF_OK;
}

int64_t gmapf_kernel_launches(gmapf_ctx* ctx) {
    if (ctx && ctx->world) ctx = ctx->world;
    return ctx ? ctx->c.launches : 0;
}

void* gmapf_stream_handle(gmapf_ctx* ctx) {
    if (ctx && ctx->world) ctx = ctx->world;
    if (!ctx || !ctx->c.started) return nullptr;
    return (void*)ctx->c.dev.stream;
}

gmapf_status gmapf_set_tune_cache(gmapf_ctx* ctx, const char* path) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (c.started) return fail(GMAPF_E_STATE, "set the autotuner cache before the start");
    c.tune_cache = path ? path : "";
    return GMAPF_OK;
}

gmapf_status gmapf_set_search_timeline(gmapf_ctx* ctx, uint64_t* d_timeline, int32_t rows) {
    NEED_CTX(ctx);
    if (ctx->world || ctx->c.detached) return scene_only("search timeline");
    if (d_timeline && rows <= 0) return fail(GMAPF_E_INVALID_ARG, "timeline rows must be positive");
    if (d_timeline && !gpu_reachable(d_timeline, ctx->c.opt.device))
        return fail(GMAPF_E_INVALID_ARG, "the timeline is not memory the context's GPU can reach (its device memory, managed or mapped pinned)");
    ctx->c.timeline = reinterpret_cast<unsigned long long*>(d_timeline);
    ctx->c.timeline_rows = d_timeline ? rows : 0;
    return GMAPF_OK;
}

gmapf_status gmapf_tune_source(gmapf_ctx* ctx, int32_t* source) {
    NEED_CTX(ctx);
    if (!source) return fail(GMAPF_E_INVALID_ARG, "null output pointer");
    if (ctx->world) ctx = ctx->world;
    if (!ctx->c.started) return fail(GMAPF_E_STATE, "not started");
    *source = ctx->c.tune_source;
    return GMAPF_OK;
}

gmapf_status gmapf_search_shape(gmapf_ctx* ctx, int32_t* T, int32_t* C, int32_t* bt, int32_t* vm,
                                int32_t* slots) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    if (ctx->world) ctx = ctx->world;
    Context& c = ctx->c;
    if (!c.started) return fail(GMAPF_E_STATE, "not started");
    if (T) *T = c.T;
    if (C) *C = c.C;
    if (bt) *bt = c.block_threads;
    if (vm) *vm = c.dev.vm;
    if (slots) *slots = c.dev.slots;
    return GMAPF_OK;
}

gmapf_status gmapf_search_batch_device(gmapf_ctx* ctx, const int32_t* d_starts, const int32_t* d_targets,
                                       int32_t n, int32_t* d_found, int32_t* d_lens, int32_t* d_paths,
                                       int32_t path_stride, gmapf_step_stats* stats) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (ctx->world || c.detached) return scene_only("search batch");
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.step_going) return fail(GMAPF_E_STATE, "a step is running");
    if (n < 0 || path_stride < 1) return fail(GMAPF_E_INVALID_ARG, "bad sizes");
    if (n > 0 && (!d_starts || !d_targets || !d_found || !d_lens || !d_paths))
        return fail(GMAPF_E_INVALID_ARG, "null device pointer");
    const int dv = c.opt.device;
    if (n > 0 && !(gpu_reachable(d_starts, dv) && gpu_reachable(d_targets, dv) && gpu_reachable(d_found, dv) &&
                   gpu_reachable(d_lens, dv) && gpu_reachable(d_paths, dv)))
        return fail(GMAPF_E_INVALID_ARG, "a buffer is not memory the context's GPU can reach (its device memory, managed or mapped pinned)");
    gmapf_status s = start_if_needed(c);
    if (s != GMAPF_OK) return s;
    std::string err;
    int rc = device_search_batch(c, d_starts, d_targets, n, d_found, d_lens, d_paths, path_stride, stats, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_search_batch_host(gmapf_ctx* ctx, const int32_t* starts, const int32_t* targets,
                                     int32_t n, int32_t* found, int32_t* lens, int32_t* paths,
                                     int32_t path_stride, gmapf_step_stats* stats) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (ctx->world || c.detached) return scene_only("search batch");
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.step_going) return fail(GMAPF_E_STATE, "a step is running");
    if (n < 0 || path_stride < 1) return fail(GMAPF_E_INVALID_ARG, "bad sizes");
    if (n > 0 && (!starts || !targets || !found || !lens || !paths))
        return fail(GMAPF_E_INVALID_ARG, "null host pointer");
    for (int i = 0; i < n; i++)
        if (starts[i] < 0 || starts[i] >= c.map.n || targets[i] < 0 || targets[i] >= c.map.n)
            return fail(GMAPF_E_INVALID_ARG, "query " + std::to_string(i) + " names a node outside the map");
    gmapf_status s = start_if_needed(c);
    if (s != GMAPF_OK) return s;
    std::string err;
    int rc = device_upload_batch_io(c, n, path_stride, err);
    if (rc) return fail(rc, err);
    Device& d = c.dev;
    cudaStream_t st = d.stream;
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMemcpyAsync(d.bstarts, starts, sizeof(int) * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.btargets, targets, sizeof(int) * n, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return fail(GMAPF_E_CUDA, std::string("upload failed: ") + cudaGetErrorString(e));
    }
    rc = device_search_batch(c, d.bstarts, d.btargets, n, d.bfound, d.blens, d.bpaths, path_stride, stats, err);
    if (rc) return fail(rc, err);
    if (n > 0) {
        e = cudaMemcpyAsync(found, d.bfound, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(lens, d.blens, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(paths, d.bpaths, sizeof(int) * (size_t)n * path_stride, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(GMAPF_E_CUDA, std::string("download failed: ") + cudaGetErrorString(e));
    }
    return GMAPF_OK;
}

gmapf_status gmapf_last_search_ms(gmapf_ctx* ctx, float* out_ms) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    if (ctx->world) ctx = ctx->world;
    if (!out_ms) return fail(GMAPF_E_INVALID_ARG, "null output");
    *out_ms = ctx->c.last_search_ms;
    return GMAPF_OK;
}

// ------------------------------------------------------------------ serving --

namespace {
// the context that serves: a bound scene's world
gmapf_ctx* serving_ctx(gmapf_ctx* ctx) { return ctx->world ? ctx->world : ctx; }
}  // namespace

gmapf_status gmapf_serve_start(gmapf_ctx* ctx, int32_t max_in_flight) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    if (ctx->world) return scene_only("serve start");
    Context& c = ctx->c;
    if (!c.inited) return fail(GMAPF_E_STATE, "not initialized");
    if (c.step_going) return fail(GMAPF_E_STATE, "a step is running");
    if (max_in_flight < 0) return fail(GMAPF_E_INVALID_ARG, "max_in_flight must be >= 0");
    if (c.serve) return fail(GMAPF_E_STATE, "already serving");
    gmapf_status s = start_if_needed(c);
    if (s != GMAPF_OK) return s;
    std::string err;
    int rc = serve_start(c, max_in_flight, err);
    if (rc) {
        serve_free(c);
        return fail(rc, err);
    }
    return GMAPF_OK;
}

gmapf_status gmapf_serve_submit(gmapf_ctx* ctx, const int32_t* ids, const gmapf_v2* targets, int32_t n,
                                const int64_t* arrival_ns) {
    NEED_CTX(ctx);
    if (ctx->c.detached) return fail(GMAPF_E_STATE, "the scene's batch was destroyed");
    gmapf_ctx* w = serving_ctx(ctx);
    Context& c = w->c;
    if (!c.serve) return fail(GMAPF_E_STATE, "not serving (gmapf_serve_start)");
    if (n < 0 || (n > 0 && (!ids || !targets))) return fail(GMAPF_E_INVALID_ARG, "bad arrays");
    if (n == 0) return GMAPF_OK;
    std::vector<int> gid;
    const int* use = ids;
    if (w != ctx) {  // a bound scene: its own ids, offset into the world
        gid.resize(n);
        for (int k = 0; k < n; k++) {
            if (ids[k] < 0 || ids[k] >= ctx->c.A)
                return fail(GMAPF_E_INVALID_ARG, "agent id " + std::to_string(ids[k]) + " out of range");
            gid[k] = ids[k] + ctx->c.agent_base;
        }
        use = gid.data();
    }
    std::string err;
    int rc = serve_submit(c, use, targets, n, arrival_ns, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_serve_poll(gmapf_ctx* ctx) {
    NEED_CTX(ctx);
    Context& c = serving_ctx(ctx)->c;
    if (!c.serve) return fail(GMAPF_E_STATE, "not serving (gmapf_serve_start)");
    std::string err;
    int rc = serve_poll(c, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_serve_drain(gmapf_ctx* ctx, float timeout_s) {
    NEED_CTX(ctx);
    Context& c = serving_ctx(ctx)->c;
    if (!c.serve) return fail(GMAPF_E_STATE, "not serving (gmapf_serve_start)");
    std::string err;
    int rc = serve_drain(c, timeout_s, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_serve_get_stats(gmapf_ctx* ctx, gmapf_serve_stats* out, int32_t reset) {
    NEED_CTX(ctx);
    if (!out) return fail(GMAPF_E_INVALID_ARG, "null output");
    Context& c = serving_ctx(ctx)->c;
    if (!c.serve) return fail(GMAPF_E_STATE, "not serving (gmapf_serve_start)");
    serve_stats(c, out, reset != 0);
    return GMAPF_OK;
}

gmapf_status gmapf_serve_result(gmapf_ctx* ctx, int32_t agent, int32_t* found, int32_t* len, int32_t* path,
                                int32_t cap) {
    NEED_CTX(ctx);
    Context& c = ctx->c;
    if (ctx->world) return scene_only("serve result");
    if (!c.serve) return fail(GMAPF_E_STATE, "not serving (gmapf_serve_start)");
    if (agent < 0 || agent >= c.A || !found || !len || (cap > 0 && !path))
        return fail(GMAPF_E_INVALID_ARG, "bad arguments");
    std::string err;
    int rc = serve_result(c, agent, found, len, path, cap, err);
    if (rc) return fail(rc, err);
    return GMAPF_OK;
}

gmapf_status gmapf_serve_stop(gmapf_ctx* ctx) {
    NEED_CTX(ctx);
    Context& c = serving_ctx(ctx)->c;
    if (c.step_going) return fail(GMAPF_E_STATE, "a step is running");
    serve_free(c);
    return GMAPF_OK;
}

int64_t gmapf_clock_ns(void) {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// ------------------------------------------------------------ scene batches --

gmapf_status gmapf_batch_create(gmapf_ctx* const* scenes, int32_t n, const gmapf_options* opt, gmapf_batch** out) {
    if (!out) return fail(GMAPF_E_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (n < 1 || !scenes) return fail(GMAPF_E_INVALID_ARG, "a batch needs at least one scene");
    for (int s = 0; s < n; s++) {
        gmapf_ctx* sc = scenes[s];
        const std::string who = "scene " + std::to_string(s);
        if (!sc) return fail(GMAPF_E_INVALID_ARG, who + " is null");
        for (int t = 0; t < s; t++)
            if (scenes[t] == sc) return fail(GMAPF_E_INVALID_ARG, who + " is listed twice");
        const Context& c = sc->c;
        if (c.is_world) return fail(GMAPF_E_INVALID_ARG, who + " is a batch's world");
        if (sc->world || c.detached) return fail(GMAPF_E_STATE, who + " already belongs to a batch");
        if (!c.inited) return fail(GMAPF_E_STATE, who + " is not initialized");
        if (!c.map_filled) return fail(GMAPF_E_STATE, who + " has no map");
        if (c.started) return fail(GMAPF_E_STATE, who + " is already started");
        const Context& c0 = scenes[0]->c;
        if (c.T != c0.T || c.C != c0.C || c.K != c0.K)
            return fail(GMAPF_E_INVALID_ARG, who + ": threads per agent, queue capacity and heuristic K must equal "
                                                   "scene 0's (they shape the one search launch)");
    }
    if (opt) {
        if (opt->mode != GMAPF_MODE_BATCHED && opt->mode != GMAPF_MODE_PLAIN)
            return fail(GMAPF_E_INVALID_ARG, "unknown mode");
        if (opt->block_threads != 0 &&
            (opt->block_threads < 32 || opt->block_threads > 256 || opt->block_threads % 32 != 0))
            return fail(GMAPF_E_INVALID_ARG, "block_threads must be 0 or a multiple of 32 in [32, 256]");
        if (opt->visited_mode < 0 || opt->visited_mode > 4)
            return fail(GMAPF_E_INVALID_ARG, "visited_mode must be 0 (automatic), 1, 2, 3 or 4");
        if (opt->device < 0) return fail(GMAPF_E_INVALID_ARG, "device must be >= 0");
        if (opt->round_limit < 0) return fail(GMAPF_E_INVALID_ARG, "round_limit must be >= 0");
        if (opt->promote_rounds < 0) return fail(GMAPF_E_INVALID_ARG, "promote_rounds must be >= 0");
        if (opt->path_smoothing < 0 || opt->path_smoothing > 2)
            return fail(GMAPF_E_INVALID_ARG, "path_smoothing must be 0, 1 or 2");
    }
    gmapf_batch* b = new (std::nothrow) gmapf_batch();
    gmapf_ctx* w = new (std::nothrow) gmapf_ctx();
    if (!b || !w) {
        delete b;
        delete w;
        return fail(GMAPF_E_CAPACITY, "out of host memory");
    }
    Context& wc = w->c;
    const Context& c0 = scenes[0]->c;
    wc.is_world = true;
    wc.opt.device = 0;
    wc.opt.mode = GMAPF_MODE_BATCHED;
    wc.opt.order_by_estimate = 1;
    if (opt) wc.opt = *opt;
    if (wc.opt.block_threads) wc.block_threads = wc.opt.block_threads;
    // world map and scene table
    std::vector<const HostMap*> maps;
    for (int s = 0; s < n; s++) maps.push_back(&scenes[s]->c.map);
    concat_host_maps(maps, wc.map, wc.scenes);
    // world config: the search shape of the scenes, summed capacities
    wc.cfg = c0.cfg;
    wc.cfg.AgentsMaxCount = 0;
    wc.cfg.PathFinderParallelAgents = 0;
    wc.cfg.IsDebug = 0;
    wc.cfg.IsProfiler = 0;
    int A = 0;
    for (int s = 0; s < n; s++) {
        const Context& c = scenes[s]->c;
        SceneInfo& si = wc.scenes[s];
        si.agent_base = A;
        si.A = c.A;
        si.P = c.cfg.PathFinderParallelAgents;
        si.radius = c.cfg.AgentRadius;
        si.speed = c.cfg.AgentSpeed;
        wc.cfg.AgentsMaxCount += c.A;
        wc.cfg.PathFinderParallelAgents += std::min(c.cfg.PathFinderParallelAgents, std::max(c.A, 1));
        wc.cfg.IsDebug |= c.cfg.IsDebug;
        wc.cfg.IsProfiler |= c.cfg.IsProfiler;
        A += c.A;
    }
    wc.T = c0.T;
    wc.C = c0.C;
    wc.K = c0.K;
    // world agents: the scenes' agents one after another, triangle ids made global
    wc.m_pos.reserve(A);
    wc.m_state.reserve(A);
    wc.m_cur.reserve(A);
    wc.m_targ.reserve(A);
    wc.m_targ_node.reserve(A);
    for (int s = 0; s < n; s++) {
        const Context& c = scenes[s]->c;
        const int nb = wc.scenes[s].node_base;
        for (int i = 0; i < c.A; i++) {
            wc.m_pos.push_back(c.m_pos[i]);
            wc.m_state.push_back(c.m_state[i]);
            wc.m_cur.push_back(c.m_cur[i] >= 0 ? c.m_cur[i] + nb : -1);
            wc.m_targ.push_back(c.m_targ[i]);
            wc.m_targ_node.push_back(c.m_targ_node[i] >= 0 ? c.m_targ_node[i] + nb : -1);
        }
    }
    wc.dirty_slot.assign(A, -1);
    wc.A = A;
    wc.inited = true;
    wc.map_filled = true;
    // bind the scenes
    for (int s = 0; s < n; s++) {
        gmapf_ctx* sc = scenes[s];
        sc->batch = b;
        sc->world = w;
        sc->c.scene_index = s;
        sc->c.agent_base = wc.scenes[s].agent_base;
        sc->c.node_base = wc.scenes[s].node_base;
        sc->c.started = true;  // no more map, agent or option changes
        b->scenes.push_back(sc);
    }
    b->world = w;
    *out = b;
    return GMAPF_OK;
}

gmapf_status gmapf_batch_destroy(gmapf_batch* b) {
    if (!b) return GMAPF_OK;
    for (gmapf_ctx* sc : b->scenes) {
        sc->batch = nullptr;
        sc->world = nullptr;
        sc->c.detached = true;
    }
    Context& wc = b->world->c;
    if (wc.started) {
        if (wc.step_going) {
            std::string err;
            device_wait_step(wc, err);
            wc.step_going = false;
        }
        device_free(wc);
    }
    delete b->world;
    delete b;
    return GMAPF_OK;
}

gmapf_ctx* gmapf_batch_world(gmapf_batch* b) { return b ? b->world : nullptr; }

gmapf_status gmapf_batch_scene_base(gmapf_batch* b, int32_t scene, int32_t* agent_base, int32_t* node_base) {
    if (!b) return fail(GMAPF_E_INVALID_ARG, "null batch");
    const Context& wc = b->world->c;
    if (scene < 0 || scene >= (int)wc.scenes.size()) return fail(GMAPF_E_INVALID_ARG, "scene out of range");
    if (agent_base) *agent_base = wc.scenes[scene].agent_base;
    if (node_base) *node_base = wc.scenes[scene].node_base;
    return GMAPF_OK;
}

}  // extern "C"
