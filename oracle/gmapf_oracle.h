/*
 * gmapf_oracle.h -- CPU oracle for the G-MAPF per-frame step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * It restates, in plain single-threaded C++17 per query (and a std::thread
 * pool across queries), the reference algorithm of rosdvp/gmapf:
 *   search          include/gmapf/PathFinder.h:138-251 (KernelSearch)
 *   bounded queue   include/gmapf/misc/CuQueue.h:33-70
 *   visited claims  include/gmapf/misc/CuVisitedMap.h:45-54
 *   path layout     include/gmapf/PathFinder.h:253-307 (KernelBuildPath)
 *   request rules   include/gmapf/PathFinder.h:76-117 (KernelFindRequests)
 *   move            include/gmapf/AgentsMover.h:51-71
 *   collisions      include/gmapf/AgentsMover.h:73-129
 *   path progress   include/gmapf/AgentsMover.h:131-177
 *   geometry        include/gmapf/misc/CuNodesMap.h:46-112, V2Float.h:23-55
 *   centroid        src/GMAPF.cu:215
 * with the reference's data races replaced by one fixed total order, the
 * deterministic tie-break (F, then G, then node id) and Jacobi collisions
 * summed in ascending agent id.  Every floating-point expression is evaluated
 * in IEEE binary32 with no contraction (built with -ffp-contract=off).
 *
 * Parity pin: the container and geometry semantics are checked against the
 * reference's own __host__ __device__ code compiled on the host
 * (oracle/ref/, output in oracle/_ref/); the searches themselves are
 * race-by-design in the reference, so the per-query search order is pinned
 * only through those container semantics and through property tests
 * (valid, connected paths; found/not-found against BFS reachability).
 */
#ifndef GMAPF_ORACLE_H
#define GMAPF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_map orc_map;
typedef struct orc_world orc_world;

typedef struct orc_search_stats {
    long long rounds;      /* search rounds (all lanes pop once per round) */
    long long expansions;  /* nodes popped and expanded */
    long long claims;      /* nodes claimed in the visited map */
    long long deg_sum;     /* sum over expansions of the expanded node's degree */
} orc_search_stats;

/* Map: tri = 6 floats per node (P1.x P1.y P2.x P2.y P3.x P3.y),
 * nbr = 3 ints per node, -1 padded (CuNodesMap::Node::NeibsIdx). */
orc_map* orc_map_create(const float* tri, const int* nbr, int n);
void orc_map_destroy(orc_map* m);
int orc_map_count(const orc_map* m);
void orc_map_centroids(const orc_map* m, float* out_xy);
int orc_locate_linear(const orc_map* m, float x, float y);
int orc_locate(const orc_map* m, float x, float y);
/* orc_locate for n points (xy interleaved) */
void orc_locate_batch(const orc_map* m, const float* xy, int n, int* out);

/* Navmesh of a FillMapStart(size) + FillMapObstacle(...) + FillMapEnd()
 * sequence (navmesh_oracle.cpp): obstacle o has obst_counts[o] vertices,
 * taken in order from obst_xy (xy interleaved).  Writes 6 floats and 3
 * neighbour ids per triangle and returns the triangle count; -1 when it
 * exceeds cap, -2 when built without the CDT headers, -3 when CDT fails. */
int orc_navmesh_build(float size_x, float size_y, const float* obst_xy, const int* obst_counts, int n_obst,
                      float* out_tri, int* out_nbr, int cap);
int orc_in_node(const orc_map* m, float x, float y, int node);
float orc_dist_sqr(const orc_map* m, int a, int b);

/* One search.  Returns 1 found, 0 not found, -1 if path_cap is too small. */
int orc_search(const orc_map* m, int start, int target, int T, int C, float K,
               int* path, int path_cap, int* path_len, orc_search_stats* st);

/* Many independent searches on `threads` host threads.  paths_out holds
 * n * path_stride ints; path i lives at paths_out[i*path_stride]. */
int orc_search_batch(const orc_map* m, const int* starts, const int* targets, int n,
                     int T, int C, float K, int* found, int* lens, int* paths_out,
                     int path_stride, orc_search_stats* st_total, int threads);

/* Bounded queue simulator (CuQueue semantics with the (F,G,id) tie-break).
 * ops[k] = 1: push item number (next unpushed); 0: pop.  Popped ids are
 * written to out_popped (-1 when the queue was empty); the final contents in
 * pop order to out_final.  Returns the final size. */
int orc_queue_sim(const float* F, const int* G, const int* id, int n_items,
                  const int* ops, int n_ops, int C, int* out_popped, int* out_final);

/* The same searches with the reference's own orders emulated, for path-cost
 * comparisons: fifo = 1 orders each queue by F alone, equal F first in first
 * out (CuQueue.h:39-63); seed != 0 takes the lanes of each neighbour slot of
 * a round in a seeded random order, as the reference's threads race inside
 * each claim and frontier append (PathFinder.h:198-231).  fifo = 0 and
 * seed = 0 is orc_search_batch. */
int orc_search_batch_order(const orc_map* m, const int* starts, const int* targets, int n,
                           int T, int C, float K, int fifo, unsigned long long seed, int* found,
                           int* lens, int* paths_out, int path_stride, orc_search_stats* st_total,
                           int threads);

/* orc_queue_sim with the reference's own key when fifo = 1 (F alone, equal F
 * first in first out). */
int orc_queue_sim_order(const float* F, const int* G, const int* id, int n_items,
                        const int* ops, int n_ops, int C, int fifo, int* out_popped, int* out_final);

/* Cost references */
int orc_bfs_hops(const orc_map* m, int s, int t);
double orc_dijkstra_len(const orc_map* m, int s, int t);
double orc_path_len(const orc_map* m, int start, const int* path, int L);

/* World: the full per-frame step (AsyncStep + WaitStepEnd semantics). */
orc_world* orc_world_create(const orc_map* m, int agents_max, float radius, float speed,
                            int parallel_agents, int T, int C, float K);
void orc_world_destroy(orc_world* w);
/* path smoothing (not in the reference): 1 steer through funnel corners, 2 the
 * same with every portal narrowed by the agent radius at both ends */
void orc_world_set_smoothing(orc_world* w, int mode);
int orc_world_add_agent(orc_world* w, float x, float y);
int orc_world_set_target(orc_world* w, int id, float x, float y);
void orc_world_step(orc_world* w, float dt, int threads);
int orc_world_count(const orc_world* w);
void orc_world_get(const orc_world* w, float* pos, int* state, int* cur_node,
                   int* targ_node, int* step_idx, int* step_node, float* step_pos,
                   int* path_len);
int orc_world_get_path(const orc_world* w, int id, int* out, int cap);
void orc_world_last_stats(const orc_world* w, long long* out6);
/* Overwrite the full agent state (used to start the oracle from a GPU state). */
void orc_world_set(orc_world* w, int id, float px, float py, int state, int cur_node,
                   float tx, float ty, int targ_node, int step_idx, int step_node,
                   float sx, float sy, const int* path, int path_len);

#ifdef __cplusplus
}
#endif
#endif
