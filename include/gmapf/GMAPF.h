// gmapf/GMAPF.h -- header-only C++ front-end of the B200 G-MAPF library with
// the reference's public names and signatures (rosdvp/gmapf
// include/gmapf/GMAPF.h:30-98, Config.h:5-18, Agent.h:7-12,
// misc/V2Float.h:12-16, misc/CuNodesMap.h:14-21), over the C ABI in
// gmapf_c.h.  Code written against the reference compiles against this
// header and links with libgmapf_b200.so.
//
// Errors: the reference throws std::exception("message") (an MSVC extension,
// src/GMAPF.cu:75-329); this wrapper throws gmapf::Error, a
// std::runtime_error carrying the C status, so `catch (std::exception&)`
// keeps working and what() returns the message.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../gmapf_c.h"

namespace gmapf {

// include/gmapf/misc/V2Float.h:12-16 (layout; arithmetic is not needed by the API)
struct V2Float {
    float X = 0;
    float Y = 0;
    V2Float() = default;
    V2Float(float x, float y) : X(x), Y(y) {}
};

// include/gmapf/Agent.h:7-12
enum class EAgentState { Idle = 0, Search = 1, Move = 2 };

// include/gmapf/Config.h:5-18
struct Config {
    int AgentsMaxCount;
    float AgentRadius;
    float AgentSpeed;
    int PathFinderParallelAgents;
    int PathFinderThreadsPerAgents;
    int PathFinderQueueCapacity;
    float PathFinderHeuristicK;
    bool IsDebug = false;
    bool IsProfiler = false;
};

// include/gmapf/misc/CuNodesMap.h:14-21 (CuNodesMap::Node)
class CuNodesMap {
public:
    constexpr static int INVALID = -1;
    constexpr static int NEIBS_MAX_COUNT = 3;
    struct alignas(16) Node {
        V2Float P1;
        V2Float P2;
        V2Float P3;
        V2Float PCenter;
        int NeibsIdx[NEIBS_MAX_COUNT];
    };
};
static_assert(sizeof(CuNodesMap::Node) == sizeof(gmapf_node), "Node layout");
static_assert(sizeof(V2Float) == sizeof(gmapf_v2), "V2Float layout");

class Error : public std::runtime_error {
public:
    Error(gmapf_status s, const std::string& m) : std::runtime_error(m), status(s) {}
    gmapf_status status;
};

class GMAPF {
public:
    GMAPF() {
        check(gmapf_create(&_ctx));
    }
    GMAPF(const GMAPF&) = delete;
    GMAPF(GMAPF&&) = delete;
    GMAPF& operator=(GMAPF&) = delete;
    GMAPF& operator=(GMAPF&&) = delete;
    ~GMAPF() { gmapf_destroy(_ctx); }  // waits for a running step, frees everything

    void Init(const Config& c) {
        gmapf_config cc{};
        cc.AgentsMaxCount = c.AgentsMaxCount;
        cc.AgentRadius = c.AgentRadius;
        cc.AgentSpeed = c.AgentSpeed;
        cc.PathFinderParallelAgents = c.PathFinderParallelAgents;
        cc.PathFinderThreadsPerAgents = c.PathFinderThreadsPerAgents;
        cc.PathFinderQueueCapacity = c.PathFinderQueueCapacity;
        cc.PathFinderHeuristicK = c.PathFinderHeuristicK;
        cc.IsDebug = c.IsDebug ? 1 : 0;
        cc.IsProfiler = c.IsProfiler ? 1 : 0;
        check(gmapf_init(_ctx, &cc));
    }
    void ManualStart() { check(gmapf_manual_start(_ctx)); }

    int AddAgent(const V2Float& currPos) {
        int32_t id = -1;
        check(gmapf_add_agent(_ctx, currPos.X, currPos.Y, &id));
        return id;
    }
    void SetAgentTargPos(int agentId, const V2Float& targPos) {
        check(gmapf_set_agent_targ_pos(_ctx, agentId, targPos.X, targPos.Y));
    }
    // README.md:78 spelling
    void SetAgentTargetPos(int agentId, const V2Float& targPos) { SetAgentTargPos(agentId, targPos); }

    void FillMapStart(const V2Float& mapSize) { check(gmapf_fill_map_start(_ctx, mapSize.X, mapSize.Y)); }
    // README.md:66 calls it with two numbers
    void FillMapStart(float sizeX, float sizeY) { check(gmapf_fill_map_start(_ctx, sizeX, sizeY)); }
    void FillMapObstacle(const std::vector<V2Float>& vertices) {
        check(gmapf_fill_map_obstacle(_ctx, reinterpret_cast<const gmapf_v2*>(vertices.data()),
                                      (int32_t)vertices.size()));
    }
    void FillMapEnd() { check(gmapf_fill_map_end(_ctx)); }
    void FillMapManually(const std::vector<CuNodesMap::Node>& nodes) {
        std::vector<gmapf_node> n(nodes.size());
        for (size_t i = 0; i < nodes.size(); i++) {
            n[i].P1 = {nodes[i].P1.X, nodes[i].P1.Y};
            n[i].P2 = {nodes[i].P2.X, nodes[i].P2.Y};
            n[i].P3 = {nodes[i].P3.X, nodes[i].P3.Y};
            n[i].PCenter = {nodes[i].PCenter.X, nodes[i].PCenter.Y};
            for (int k = 0; k < 3; k++) n[i].NeibsIdx[k] = nodes[i].NeibsIdx[k];
            n[i]._pad = 0;
        }
        check(gmapf_fill_map_manually(_ctx, n.data(), (int32_t)n.size()));
    }

    void AsyncStep(float deltaTime) { check(gmapf_async_step(_ctx, deltaTime)); }
    void WaitStepEnd() { check(gmapf_wait_step_end(_ctx)); }

    // a reference into the host mirror, refreshed by WaitStepEnd (src/GMAPF.cu:316-319)
    const V2Float& GetAgentPos(int agentId) {
        if (agentId < 0 || agentId >= gmapf_agent_count(_ctx)) throw Error(GMAPF_E_INVALID_ARG, "agent id out of range");
        return reinterpret_cast<const V2Float*>(gmapf_agent_pos_view(_ctx))[agentId];
    }
    EAgentState GetAgentState(int agentId) {
        int32_t s = 0;
        check(gmapf_get_agent_state(_ctx, agentId, &s));
        return static_cast<EAgentState>(s);
    }

    void ProfilerDump() const { check(gmapf_profiler_dump(_ctx)); }

    // ---- extensions (no counterpart in the reference; see gmapf_c.h) ----
    // step form, visited placement, autotuner, path smoothing (before the start)
    void SetOptions(const gmapf_options& o) { check(gmapf_set_options(_ctx, &o)); }
    // autotuner cache file (before the start); "" turns it off
    void SetTuneCache(const std::string& path) { check(gmapf_set_tune_cache(_ctx, path.c_str())); }
    // 0: the Config's shape, 1: tuned at the start, 2: from the autotuner cache
    int TuneSource() const {
        int32_t v = 0;
        check(gmapf_tune_source(_ctx, &v));
        return v;
    }
    gmapf_options Options() const {
        gmapf_options o{};
        check(gmapf_get_options(_ctx, &o));
        return o;
    }
    // FillMapEnd through a navmesh cache file; returns true when the cache was used
    bool FillMapEndCached(const std::string& path) {
        int32_t hit = 0;
        check(gmapf_fill_map_end_cached(_ctx, path.c_str(), &hit));
        return hit != 0;
    }
    void MapSave(const std::string& path) const { check(gmapf_map_save(_ctx, path.c_str())); }
    void MapLoad(const std::string& path) { check(gmapf_map_load(_ctx, path.c_str())); }
    // true when no step runs or its device work is done (WaitStepEnd will not block)
    bool StepReady() const { return gmapf_step_ready(_ctx) != 0; }
    // serving: retargets searched as soon as they are submitted
    void ServeStart(int maxInFlight = 0) { check(gmapf_serve_start(_ctx, maxInFlight)); }
    void ServeSubmit(const std::vector<int>& agentIds, const std::vector<V2Float>& targets) {
        if (agentIds.size() != targets.size()) throw Error(GMAPF_E_INVALID_ARG, "ids and targets differ in length");
        check(gmapf_serve_submit(_ctx, agentIds.data(), reinterpret_cast<const gmapf_v2*>(targets.data()),
                                 (int32_t)agentIds.size(), nullptr));
    }
    void ServePoll() { check(gmapf_serve_poll(_ctx)); }
    void ServeDrain(float timeoutSeconds = 60.0f) { check(gmapf_serve_drain(_ctx, timeoutSeconds)); }
    gmapf_serve_stats ServeStats(bool reset = false) {
        gmapf_serve_stats st{};
        check(gmapf_serve_get_stats(_ctx, &st, reset ? 1 : 0));
        return st;
    }

    // the C context, for the extensions in gmapf_c.h
    gmapf_ctx* handle() const { return _ctx; }

    static void check(gmapf_status s) {
        if (s != GMAPF_OK) throw Error(s, std::string("[gmapf] ") + gmapf_last_error());
    }

private:
    gmapf_ctx* _ctx = nullptr;
};

// Several scenes stepped as one (gmapf_batch_*): each scene is a GMAPF that
// was initialised, filled and given its agents; afterwards the scenes keep
// their per-agent calls (SetAgentTargPos, GetAgentPos, GetAgentState, ...)
// with their own ids, and frames run here.  The scenes must outlive the batch.
class SceneBatch {
public:
    explicit SceneBatch(const std::vector<GMAPF*>& scenes, const gmapf_options* options = nullptr) {
        std::vector<gmapf_ctx*> h;
        for (GMAPF* g : scenes) h.push_back(g->handle());
        GMAPF::check(gmapf_batch_create(h.data(), (int32_t)h.size(), options, &_b));
    }
    SceneBatch(const SceneBatch&) = delete;
    SceneBatch& operator=(const SceneBatch&) = delete;
    ~SceneBatch() { gmapf_batch_destroy(_b); }

    void ManualStart() { GMAPF::check(gmapf_manual_start(world())); }
    void AsyncStep(float deltaTime) { GMAPF::check(gmapf_async_step(world(), deltaTime)); }
    void WaitStepEnd() { GMAPF::check(gmapf_wait_step_end(world())); }
    bool StepReady() const { return gmapf_step_ready(world()) != 0; }
    // serving on the whole batch (agent ids global: see SceneBase)
    void ServeStart(int maxInFlight = 0) { GMAPF::check(gmapf_serve_start(world(), maxInFlight)); }
    void ServeDrain(float timeoutSeconds = 60.0f) { GMAPF::check(gmapf_serve_drain(world(), timeoutSeconds)); }
    gmapf_serve_stats ServeStats(bool reset = false) {
        gmapf_serve_stats st{};
        GMAPF::check(gmapf_serve_get_stats(world(), &st, reset ? 1 : 0));
        return st;
    }
    // first global agent id and triangle id of a scene
    void SceneBase(int scene, int* agentBase, int* nodeBase) const {
        GMAPF::check(gmapf_batch_scene_base(_b, scene, agentBase, nodeBase));
    }
    gmapf_ctx* world() const { return gmapf_batch_world(_b); }

private:
    gmapf_batch* _b = nullptr;
};

}  // namespace gmapf
