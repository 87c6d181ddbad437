// Reference-style client of include/gmapf/GMAPF.h (the drop-in C++ API).
//   wrapper_demo cpu   lifecycle and error rules, no GPU needed
//   wrapper_demo gpu   zig-zag map, agents in a row heading north, N steps;
//                      prints "agent x y state" lines for the oracle check
//   wrapper_demo batch the same as two scenes of one SceneBatch (different
//                      radii), then served retargets on one scene;
//                      prints "scene s agent x y state" lines and the counts
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "gmapf/GMAPF.h"

using namespace gmapf;

static void zigzag(GMAPF& g) {
    g.FillMapStart({1000, 1000});
    for (int i = 2; i <= 8; i++) {
        float y0 = i * 100.0f, y1 = y0 + 10;
        float x0 = i % 2 == 0 ? 100.0f : 0.0f, x1 = i % 2 == 0 ? 1000.0f : 100.0f;
        g.FillMapObstacle({{x0, y0}, {x0, y1}, {x1, y1}, {x1, y0}});
    }
    g.FillMapEnd();
}

static Config config(int agents) {
    Config c;
    c.AgentsMaxCount = agents;
    c.AgentSpeed = 1;
    c.AgentRadius = 2;
    c.PathFinderParallelAgents = agents;
    c.PathFinderThreadsPerAgents = 4;
    c.PathFinderQueueCapacity = 16;
    c.PathFinderHeuristicK = 1;
    c.IsProfiler = true;
    return c;
}

int main(int argc, char** argv) {
    const bool gpu = argc > 1 && (std::strcmp(argv[1], "gpu") == 0 || std::strcmp(argv[1], "batch") == 0);
    if (!gpu) {
        GMAPF g;
        g.Init(config(8));
        zigzag(g);
        int thrown = 0;
        try {
            g.FillMapEnd();
        } catch (const std::exception& e) {  // reference callers catch std::exception
            thrown += std::strstr(e.what(), "already filled") != nullptr;
        }
        try {
            g.AddAgent({500, 205});  // inside a wall
        } catch (const Error& e) {
            thrown += e.status == GMAPF_E_INVALID_POS;
        }
        int id = g.AddAgent({10, 10});
        g.SetAgentTargetPos(id, {10, 950});
        const V2Float& p = g.GetAgentPos(id);
        std::printf("cpu ok thrown=%d id=%d pos=%g,%g state=%d\n", thrown, id, p.X, p.Y, (int)g.GetAgentState(id));
        return thrown == 2 ? 0 : 1;
    }
    if (std::strcmp(argv[1], "batch") == 0) {
        const int A = 128, steps = 120;
        GMAPF a, b;
        Config ca = config(A), cb = config(A);
        cb.AgentRadius = 1.5f;
        a.Init(ca);
        b.Init(cb);
        zigzag(a);
        zigzag(b);
        for (int i = 0; i < A; i++) {
            a.AddAgent({i / 5.0f + 1.0f, 1.0f});
            b.AddAgent({i / 4.0f + 2.0f, 3.0f});
        }
        for (int i = 0; i < A; i++) {
            a.SetAgentTargetPos(i, {i / 5.0f + 1.0f, 950.0f});
            b.SetAgentTargetPos(i, {990.0f - i / 4.0f, 600.0f});
        }
        SceneBatch batch({&a, &b});
        batch.ManualStart();
        for (int s = 0; s < steps; s++) {
            batch.AsyncStep(1.0f / 60.0f);
            batch.WaitStepEnd();
        }
        GMAPF* sc[2] = {&a, &b};
        for (int k = 0; k < 2; k++)
            for (int i = 0; i < A; i++) {
                const V2Float& p = sc[k]->GetAgentPos(i);
                std::printf("scene %d agent %d %.9g %.9g %d\n", k, i, p.X, p.Y, (int)sc[k]->GetAgentState(i));
            }
        // served retargets through scene b's own ids
        batch.ServeStart();
        std::vector<int> ids;
        std::vector<V2Float> to;
        for (int i = 0; i < 16; i++) {
            ids.push_back(i);
            to.push_back({50.0f + i, 150.0f});
        }
        b.ServeSubmit(ids, to);
        batch.ServeDrain();
        batch.AsyncStep(1.0f / 60.0f);
        batch.WaitStepEnd();
        const gmapf_serve_stats st = batch.ServeStats();
        std::printf("served completed=%lld found=%lld applied=%lld\n", (long long)st.completed, (long long)st.found,
                    (long long)st.applied);
        return 0;
    }
    const int A = 256, steps = 120;
    GMAPF g;
    g.Init(config(A));
    zigzag(g);
    for (int i = 0; i < A; i++) g.AddAgent({i / 5.0f + 1.0f, 1.0f});
    for (int i = 0; i < A; i++) g.SetAgentTargetPos(i, {i / 5.0f + 1.0f, 950.0f});
    g.ManualStart();
    for (int s = 0; s < steps; s++) {
        g.AsyncStep(1.0f / 60.0f);
        g.WaitStepEnd();
    }
    for (int i = 0; i < A; i++) {
        const V2Float& p = g.GetAgentPos(i);
        std::printf("agent %d %.9g %.9g %d\n", i, p.X, p.Y, (int)g.GetAgentState(i));
    }
    g.ProfilerDump();
    return 0;
}
