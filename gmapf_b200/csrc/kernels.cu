// kernels.cu -- request compaction, target upload and the agents mover.
//
// Reference kernels restated here:
//   KernelFindRequests        include/gmapf/PathFinder.h:76-117
//   KernelFindMovingAgents    include/gmapf/AgentsMover.h:29-49
//   KernelMoveAgents          include/gmapf/AgentsMover.h:51-71
//   KernelResolveCollisions   include/gmapf/AgentsMover.h:73-129
//   KernelUpdatePathProgress  include/gmapf/AgentsMover.h:131-177
// Agents are stored as structure-of-arrays.  Compaction is stable (requests
// in ascending agent id).  Collisions read one snapshot of the positions
// after the move and write a second buffer (Jacobi); each agent sums its
// contributions in ascending neighbour id, found through a counting-sort
// uniform grid whose cells are at least 1.0625 collision distances wide, so
// the 3x3 neighbourhood holds every agent the reference's all-pairs loop
// would accept.
#include <cuda_runtime.h>

#include "internal.h"

namespace gmapf_b200 {

namespace {

constexpr int kCompactThreads = 1024;

// Per-scene request limits (a scene batch): scene s takes its Search agents in
// ascending id up to P[s] (each scene is its own PathFinder, PathFinder.h:76-117).
// first[s] records how many Search agents precede the scene's first agent.
__global__ void __launch_bounds__(kCompactThreads)
    k_compact(int A, int* state, const int* cur, const int* targ, int P, CompactScenes scn, int4* req,
              int* req_count, unsigned char* in_move, int* mv_count, int* work_ctr, unsigned long long* stats) {
    __shared__ int warp_tot[32];
    __shared__ int warp_totm[32];
    __shared__ int warp_toto[32];
    __shared__ int base_s, base_m, base_o;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const bool scenes = scn.agent_scene != nullptr;
    if (tid == 0) {
        base_s = 0;
        base_m = 0;
        base_o = 0;
    }
    __syncthreads();
    for (int b = 0; b < A; b += kCompactThreads) {
        const int i = b + tid;
        bool isS = false, isM = false;
        int cu = 0, ta = 0;
        if (i < A) {
            const int st = state[i];
            if (st == GMAPF_AGENT_SEARCH) {
                cu = cur[i];
                ta = targ[i];
                if (cu == ta) {
                    state[i] = GMAPF_AGENT_IDLE;  // PathFinder.h:91-95
                } else {
                    isS = true;
                }
            }
            isM = st == GMAPF_AGENT_MOVE;
            in_move[i] = isM ? 1 : 0;
        }
        const unsigned bs = __ballot_sync(0xffffffffu, isS);
        const unsigned bm = __ballot_sync(0xffffffffu, isM);
        if (lane == 0) {
            warp_tot[warp] = __popc(bs);
            warp_totm[warp] = __popc(bm);
        }
        __syncthreads();
        if (warp == 0) {
            int v = warp_tot[lane], vm = warp_totm[lane];
            // inclusive scans over the 32 warp totals
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, v, o);
                int tm = __shfl_up_sync(0xffffffffu, vm, o);
                if (lane >= o) {
                    v += t;
                    vm += tm;
                }
            }
            warp_tot[lane] = v;  // inclusive
            warp_totm[lane] = vm;
        }
        __syncthreads();
        const int wpre = (warp == 0) ? 0 : warp_tot[warp - 1];
        const int gpos = base_s + wpre + __popc(bs & lt);  // Search agents before i
        if (!scenes) {
            if (isS && gpos < P) req[gpos] = make_int4(i, cu, ta, i);  // over capacity: stays Search
        } else {
            const int sidx = i < A ? scn.agent_scene[i] : 0;
            if (i < A && i == scn.abase[sidx]) scn.first[sidx] = gpos;
            __syncthreads();
            const bool ok = isS && gpos - scn.first[sidx] < scn.P[sidx];
            const unsigned bo = __ballot_sync(0xffffffffu, ok);
            if (lane == 0) warp_toto[warp] = __popc(bo);
            __syncthreads();
            if (warp == 0) {
                int v = warp_toto[lane];
                for (int o = 1; o < 32; o <<= 1) {
                    int t = __shfl_up_sync(0xffffffffu, v, o);
                    if (lane >= o) v += t;
                }
                warp_toto[lane] = v;
            }
            __syncthreads();
            const int opos = base_o + (warp == 0 ? 0 : warp_toto[warp - 1]) + __popc(bo & lt);
            if (ok) req[opos] = make_int4(i, cu, ta, i);
        }
        __syncthreads();
        if (tid == 0) {
            base_s += warp_tot[31];
            base_m += warp_totm[31];
            if (scenes) base_o += warp_toto[31];
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int R = scenes ? base_o : (base_s < P ? base_s : P);
        *req_count = R;
        *mv_count = base_m;
        *work_ctr = 0;
        stats[ST_REQUESTS] += (unsigned long long)R;
        stats[ST_MOVING] += (unsigned long long)base_m;
    }
}

__global__ void k_apply_targets(const int4* recs, int n, int* state, int* targ_node,
                                float2* targ_pos) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int4 r = recs[k];  // {agent, node, x bits, y bits}
    state[r.x] = GMAPF_AGENT_SEARCH;
    targ_node[r.x] = r.y;
    targ_pos[r.x] = make_float2(__int_as_float(r.z), __int_as_float(r.w));
}

// device-resident retargets: locate each target on the device (the host
// path's CuNodesMap::TryGetNodeIdx rule) and mark the agent Search
__global__ void k_apply_targets_device(const int* ids, const float2* pos, int n, int id_base, int id_count,
                                       const ScenePar* sc, const int* agent_scene, int* state, int* targ_node,
                                       float2* targ_pos, int* err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int lid = ids[k];
    const float2 p = pos[k];
    if (lid < 0 || lid >= id_count) {
        atomicOr(err, ERR_BAD_REQUEST);
        return;
    }
    const int id = id_base + lid;
    const int node = locate(sc[agent_scene ? agent_scene[id] : 0].loc, p.x, p.y);
    if (node < 0) {
        atomicOr(err, ERR_BAD_REQUEST);
        return;
    }
    state[id] = GMAPF_AGENT_SEARCH;
    targ_node[id] = node;
    targ_pos[id] = p;
}

__global__ void k_prepare_batch(const int* starts, const int* targets, int n, int nodes, int4* req,
                                int* req_count, int* work_ctr, int* err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) {
        *req_count = n;
        *work_ctr = 0;
    }
    if (k >= n) return;
    int s = starts[k], t = targets[k];
    if (s < 0 || s >= nodes || t < 0 || t >= nodes) atomicOr(err, ERR_BAD_REQUEST);
    req[k] = make_int4(-1, s, t, k);
}

// Orders requests longest-first for the persistent search: the estimate is
// the landmark lower bound on the hop distance, max_l |d_l(s) - d_l(t)|, and
// requests are bucketed by it in descending order.  Results do not depend
// on the order (every request writes only its own row and agent).
constexpr int kOrderBuckets = 1024;

__global__ void __launch_bounds__(1024) k_order_requests(const int4* req_in, const int* req_count, int4* req_out,
                                                         int* keys, const unsigned short* lm, int L, int n) {
    __shared__ int hist[kOrderBuckets];
    __shared__ int wmax[32];
    __shared__ int gmax;
    const int tid = threadIdx.x;
    const int R = *req_count;
    int mx = 0;
    for (int i = tid; i < R; i += blockDim.x) {
        const int4 q = req_in[i];
        int est = 0;
        if (q.y >= 0 && q.y < n && q.z >= 0 && q.z < n) {
            for (int l = 0; l < L; l++) {
                const int a = lm[(size_t)l * n + q.y], b = lm[(size_t)l * n + q.z];
                const int e = (a == 65535 || b == 65535) ? 65535 : abs(a - b);
                est = max(est, e);
            }
        }
        keys[i] = est;
        mx = max(mx, est);
    }
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((tid & 31) == 0) wmax[tid >> 5] = mx;
    hist[tid] = 0;
    __syncthreads();
    if (tid < 32) {
        int v = wmax[tid];
        for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (tid == 0) gmax = v;
    }
    __syncthreads();
    const long long den = max(1, gmax);
    for (int i = tid; i < R; i += blockDim.x) {
        const int b = (kOrderBuckets - 1) - (int)(((long long)keys[i] * (kOrderBuckets - 1)) / den);
        keys[i] = b;
        atomicAdd(hist + b, 1);
    }
    __syncthreads();
    // exclusive scan of the histogram (one value per thread)
    int v = hist[tid];
    const int lane = tid & 31, w = tid >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wmax[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = wmax[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wmax[lane] = s;  // inclusive warp sums
    }
    __syncthreads();
    hist[tid] = x - v + (w > 0 ? wmax[w - 1] : 0);
    __syncthreads();
    for (int i = tid; i < R; i += blockDim.x) {
        const int pos = atomicAdd(hist + keys[i], 1);
        req_out[pos] = req_in[i];
    }
}

// move (AgentsMover.h:51-71) fused with the agent-grid histogram
__global__ void k_move_bin(MoverParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (*p.mv_count == 0) return;  // AgentsMover.h:296-297
    if (i >= p.A) return;
    const ScenePar& sc = p.sc[p.agent_scene ? p.agent_scene[i] : 0];
    float2 c = p.pos[i];
    const float step = GM_FMUL(sc.speed, *p.dt);
    if (p.in_move[i] && p.step_idx[i] != -1) {
        const float2 s = p.step_pos[i];
        const float dx = GM_FSUB(s.x, c.x), dy = GM_FSUB(s.y, c.y);
        const float len = GM_FSQRT(GM_FADD(GM_FMUL(dx, dx), GM_FMUL(dy, dy)));
        if (len <= step) {
            c = s;
        } else {
            c.x = GM_FADD(c.x, GM_FMUL(GM_FDIV(dx, len), step));
            c.y = GM_FADD(c.y, GM_FMUL(GM_FDIV(dy, len), step));
        }
    }
    p.pos_mid[i] = c;
    int cell = -1;
    if (gm_isfinite(c.x) && gm_isfinite(c.y)) {
        const int cx = grid_cell(c.x, sc.ax0, sc.ainv, sc.aw);
        const int cy = grid_cell(c.y, sc.ay0, sc.ainv, sc.ah);
        cell = sc.cell_base + cy * sc.aw + cx;
        atomicAdd(p.cell_cnt + cell, 1);
    }
    p.cell_of[i] = cell;
}

// exclusive scan of the cell histogram, one block: each thread sums a run of
// cells, the runs are scanned with warp shuffles (two block barriers), then
// each thread writes its run's starts
__global__ void __launch_bounds__(1024) k_cell_scan(MoverParams p) {
    if (*p.mv_count == 0) return;
    __shared__ int wsum[32];
    const int cells = p.cells;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int per = (cells + 1023) / 1024;
    const int b = tid * per, e = min(b + per, cells);
    int s = 0;
#pragma unroll 8
    for (int k = b; k < e; k++) s += p.cell_cnt[k];  // unrolled: the loads of a run are in flight together
    int x = s;  // inclusive scan of the runs within the warp
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int v = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        wsum[lane] = v;  // inclusive warp totals
    }
    __syncthreads();
    int run = x - s + (w > 0 ? wsum[w - 1] : 0);
#pragma unroll 8
    for (int k = b; k < e; k++) {
        p.cell_start[k] = run;
        p.cell_fill[k] = run;
        run += p.cell_cnt[k];
    }
    if (tid == 1023) p.cell_start[cells] = wsum[31];
}

__global__ void k_scatter(MoverParams p) {
    if (*p.mv_count == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.A) return;
    const int c = p.cell_of[i];
    if (c < 0) return;
    const int k = atomicAdd(p.cell_fill + c, 1);
    p.cell_items[k] = i;
}

constexpr int kMaxLocal = 16;

// collisions (AgentsMover.h:73-129) + path progress (AgentsMover.h:131-177)
__global__ void k_collide_progress(MoverParams p) {
    if (*p.mv_count == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.A) return;
    const ScenePar& sc = p.sc[p.agent_scene ? p.agent_scene[i] : 0];
    const float2 me = p.pos_mid[i];
    float2 np = me;
    const int c = p.cell_of[i];
    unsigned examined = 0;  // agents of the 3x3 cells read (the agent itself included)
    if (c >= 0) {
        const int lc = c - sc.cell_base;  // cell within the agent's scene
        const int cx = lc % sc.aw, cy = lc / sc.aw;
        const int x0 = max(cx - 1, 0), x1 = min(cx + 1, sc.aw - 1);
        const int y0 = max(cy - 1, 0), y1 = min(cy + 1, sc.ah - 1);
        int ids[kMaxLocal];
        float vxs[kMaxLocal], vys[kMaxLocal];
        int cnt = 0;
        bool overflow = false;
        for (int yy = y0; yy <= y1; yy++)
            for (int xx = x0; xx <= x1; xx++) {
                const int cc = sc.cell_base + yy * sc.aw + xx;
                examined += p.cell_start[cc + 1] - p.cell_start[cc];
                for (int k = p.cell_start[cc], e = p.cell_start[cc + 1]; k < e; k++) {
                    const int j = p.cell_items[k];
                    if (j == i) continue;
                    const float2 o = p.pos_mid[j];
                    const float dx = GM_FSUB(me.x, o.x), dy = GM_FSUB(me.y, o.y);
                    const float d2 = GM_FADD(GM_FMUL(dx, dx), GM_FMUL(dy, dy));
                    if (!(d2 < sc.cd2)) continue;
                    if (cnt >= kMaxLocal) {
                        overflow = true;
                        continue;
                    }
                    const float d = GM_FSQRT(d2);
                    const float shift = GM_FSUB(sc.cd, d);
                    const float vx = GM_FMUL(GM_FDIV(dx, d), shift);
                    const float vy = GM_FMUL(GM_FDIV(dy, d), shift);
                    // insertion keeps ids ascending
                    int k2 = cnt++;
                    while (k2 > 0 && ids[k2 - 1] > j) {
                        ids[k2] = ids[k2 - 1];
                        vxs[k2] = vxs[k2 - 1];
                        vys[k2] = vys[k2 - 1];
                        k2--;
                    }
                    ids[k2] = j;
                    vxs[k2] = vx;
                    vys[k2] = vy;
                }
            }
        float sx = 0.f, sy = 0.f;
        int total = 0;
        if (!overflow) {
            for (int k = 0; k < cnt; k++) {
                sx = GM_FADD(sx, vxs[k]);
                sy = GM_FADD(sy, vys[k]);
            }
            total = cnt;
        } else {
            // dense crowd: take contributors in ascending id by repeated minimum search
            int last = -1;
            for (;;) {
                int best = 0x7fffffff;
                float bvx = 0.f, bvy = 0.f;
                for (int yy = y0; yy <= y1; yy++)
                    for (int xx = x0; xx <= x1; xx++) {
                        const int cc = sc.cell_base + yy * sc.aw + xx;
                        for (int k = p.cell_start[cc], e = p.cell_start[cc + 1]; k < e; k++) {
                            const int j = p.cell_items[k];
                            if (j == i || j <= last || j >= best) continue;
                            const float2 o = p.pos_mid[j];
                            const float dx = GM_FSUB(me.x, o.x), dy = GM_FSUB(me.y, o.y);
                            const float d2 = GM_FADD(GM_FMUL(dx, dx), GM_FMUL(dy, dy));
                            if (!(d2 < sc.cd2)) continue;
                            const float d = GM_FSQRT(d2);
                            const float shift = GM_FSUB(sc.cd, d);
                            best = j;
                            bvx = GM_FMUL(GM_FDIV(dx, d), shift);
                            bvy = GM_FMUL(GM_FDIV(dy, d), shift);
                        }
                    }
                if (best == 0x7fffffff) break;
                sx = GM_FADD(sx, bvx);
                sy = GM_FADD(sy, bvy);
                total++;
                last = best;
            }
        }
        if (total > 0) {
            const float fc = (float)total;
            const float ax = GM_FDIV(sx, fc), ay = GM_FDIV(sy, fc);
            const float rx = GM_FSUB(GM_FMUL(ax, p.cs), GM_FMUL(ay, p.sn));
            const float ry = GM_FADD(GM_FMUL(ax, p.sn), GM_FMUL(ay, p.cs));
            const float px = GM_FADD(me.x, rx), py = GM_FADD(me.y, ry);
            if (locate(sc.loc, px, py) >= 0) np = make_float2(px, py);
        }
    }
    p.pos[i] = np;
    {  // counter of the agents examined (the mover's per-agent traffic), one atomic per warp
        const unsigned m = __activemask();
        const unsigned tot = __reduce_add_sync(m, examined);
        if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(p.stats + ST_NEIGHBOURS, (unsigned long long)tot);
    }

    if (!p.in_move[i]) return;
    // path progress
    const int* path = p.paths + (long long)i * p.path_stride;
    const int L = p.path_len[i];
    int si = p.step_idx[i];
    if (si == -1) {
        if (L < 1) {
            atomicOr(p.err, ERR_BOUNDS);
            return;
        }
        const int nd = path[0];
        p.step_idx[i] = 0;
        p.step_node[i] = nd;
        p.step_pos[i] = p.waypoints ? p.waypoints[(long long)i * p.path_stride] : p.cen[nd];
        return;
    }
    const int sn = p.step_node[i];
    if (sn < 0 || sn >= p.n) {
        atomicOr(p.err, ERR_BOUNDS);
        return;
    }
    const bool inside = point_in_tri(np.x, np.y, p.tri[3 * sn], p.tri[3 * sn + 1], p.tri[3 * sn + 2]);
    bool at_point = false;  // path smoothing: the steering point reached
    if (p.waypoints && !inside) {
        const float2 s = p.step_pos[i];
        const float dx = GM_FSUB(s.x, np.x), dy = GM_FSUB(s.y, np.y);
        at_point = GM_FSQRT(GM_FADD(GM_FMUL(dx, dx), GM_FMUL(dy, dy))) <= sc.arrive;
    }
    if (!inside && !at_point) return;
    if (inside) {
        p.cur_node[i] = sn;
        if (si < L) si += 1;
    } else {
        // a straight run to a funnel corner may cross thin corridor triangles
        // between two frames: skip every step that steers to the same point
        const float2 s = p.step_pos[i];
        const float2* wp = p.waypoints + (long long)i * p.path_stride;
        int cur = p.cur_node[i];
        while (si < L && wp[si].x == s.x && wp[si].y == s.y) cur = path[si++];
        p.cur_node[i] = cur;
    }
    p.step_idx[i] = si;
    if (si == L) {
        const float2 t = p.targ_pos[i];
        const float dx = GM_FSUB(t.x, np.x), dy = GM_FSUB(t.y, np.y);
        const float len = GM_FSQRT(GM_FADD(GM_FMUL(dx, dx), GM_FMUL(dy, dy)));
        if (len > sc.arrive)
            p.step_pos[i] = t;
        else
            p.state[i] = GMAPF_AGENT_IDLE;
    } else {
        const int nd = path[si];
        p.step_node[i] = nd;
        p.step_pos[i] = p.waypoints ? p.waypoints[(long long)i * p.path_stride + si] : p.cen[nd];
    }
}

// ---- path smoothing (opt-in): the simple stupid funnel (M. Mononen, 2010)
// over the corridor of a path.  Portal 0 is the agent's position, portal k
// (1..L) the edge shared by triangles k-1 and k of the corridor (triangle 0 =
// the start triangle, triangle k = path[k-1]), portal L+1 the target
// position.  Step k of the path (heading into path[k]) steers to the first
// funnel corner at a portal index >= k+1.

// twice the signed area of (a, b, c): > 0 when c lies left of a -> b
__device__ __forceinline__ float area2(float2 a, float2 b, float2 c) {
    const float bx = GM_FSUB(b.x, a.x), by = GM_FSUB(b.y, a.y);
    const float cx = GM_FSUB(c.x, a.x), cy = GM_FSUB(c.y, a.y);
    return GM_FSUB(GM_FMUL(bx, cy), GM_FMUL(cx, by));
}

__device__ __forceinline__ bool veq(float2 a, float2 b) { return a.x == b.x && a.y == b.y; }

// path smoothing 2: both ends of an edge portal moved inward by c (the agent
// radius), so that the funnel's corners keep that distance from the walls; a
// portal no wider than 2c becomes its midpoint
__device__ __forceinline__ void narrow_portal(float2& l, float2& r, float c) {
    if (!(c > 0.f)) return;
    const float dx = GM_FSUB(r.x, l.x), dy = GM_FSUB(r.y, l.y);
    const float w = GM_FSQRT(GM_FADD(GM_FMUL(dx, dx), GM_FMUL(dy, dy)));
    if (w > GM_FADD(c, c)) {
        const float t = GM_FDIV(c, w);
        const float ox = GM_FMUL(dx, t), oy = GM_FMUL(dy, t);
        l = make_float2(GM_FADD(l.x, ox), GM_FADD(l.y, oy));
        r = make_float2(GM_FSUB(r.x, ox), GM_FSUB(r.y, oy));
    } else {
        const float mx = GM_FMUL(GM_FADD(l.x, r.x), 0.5f), my = GM_FMUL(GM_FADD(l.y, r.y), 0.5f);
        l = r = make_float2(mx, my);
    }
}

// portal k as (left, right) seen travelling from triangle k-1 to triangle k;
// triangles that share no edge give their centroid as a point portal
__device__ void corridor_portal(const MoverParams& p, const int* path, int start_tri, int L, float2 sp, float2 ep,
                                int k, float clear, float2& left, float2& right) {
    if (k <= 0) {
        left = right = sp;
        return;
    }
    if (k > L) {
        left = right = ep;
        return;
    }
    const int u = k == 1 ? start_tri : path[k - 2];
    const int v = path[k - 1];
    if (u < 0 || u >= p.n || v < 0 || v >= p.n) {
        left = right = ep;
        return;
    }
    const float2* A = p.tri + 3 * (size_t)u;
    const float2* B = p.tri + 3 * (size_t)v;
    float2 s0 = make_float2(0.f, 0.f), s1 = s0;
    int cnt = 0;
    for (int a = 0; a < 3; a++) {
        const float2 va = A[a];
        if (veq(va, B[0]) || veq(va, B[1]) || veq(va, B[2])) {
            if (cnt == 0) s0 = va;
            if (cnt == 1) s1 = va;
            cnt++;
        }
    }
    if (cnt < 2) {
        left = right = p.cen[v];
        return;
    }
    if (area2(p.cen[u], p.cen[v], s0) > 0.f) {
        left = s0;
        right = s1;
    } else {
        left = s1;
        right = s0;
    }
    narrow_portal(left, right, clear);
}

// one thread per agent whose path starts this frame (in Move at the frame's
// start, step index -1): fills its path row of steering points
__global__ void k_funnel(MoverParams p) {
    if (*p.mv_count == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.A) return;
    if (!p.in_move[i] || p.step_idx[i] != -1) return;
    const int L = p.path_len[i];
    if (L < 1 || L > p.path_stride) return;
    const int* path = p.paths + (long long)i * p.path_stride;
    float2* wp = p.waypoints + (long long)i * p.path_stride;
    const float2 sp = p.pos[i], ep = p.targ_pos[i];
    const int st = p.cur_node[i];
    const float clear = p.sc[p.agent_scene ? p.agent_scene[i] : 0].clear;
    float2 apex = sp, fl = sp, fr = sp;
    int apex_i = 0, left_i = 0, right_i = 0, filled = 0;
    const int max_iter = 4 * (L + 2) + 16;  // every restart moves the apex forward
    int iter = 0;
    bool capped = false;
    for (int k = 1; k <= L + 1; k++) {
        if (++iter > max_iter) {
            capped = true;
            break;
        }
        float2 l, r;
        corridor_portal(p, path, st, L, sp, ep, k, clear, l, r);
        if (area2(apex, fr, r) >= 0.f) {  // right edge moves inward
            if (veq(apex, fr) || area2(apex, fl, r) < 0.f) {
                fr = r;
                right_i = k;
            } else {  // crosses the left edge: its end is a corner
                for (const int upto = min(left_i, L); filled < upto; filled++) wp[filled] = fl;
                apex = fl;
                apex_i = left_i;
                fr = fl = apex;
                right_i = left_i = apex_i;
                k = apex_i;
                continue;
            }
        }
        if (area2(apex, fl, l) <= 0.f) {  // left edge moves inward
            if (veq(apex, fl) || area2(apex, fr, l) > 0.f) {
                fl = l;
                left_i = k;
            } else {  // crosses the right edge
                for (const int upto = min(right_i, L); filled < upto; filled++) wp[filled] = fr;
                apex = fr;
                apex_i = right_i;
                fl = fr = apex;
                left_i = right_i = apex_i;
                k = apex_i;
                continue;
            }
        }
    }
    for (; filled < L; filled++) {
        const int nd = path[filled];
        wp[filled] = (capped && nd >= 0 && nd < p.n) ? p.cen[nd] : ep;
    }
}

// GMAPF.cu:227,244 -> CuNodesMap.h:53-66 for a batch of points: the first
// containing triangle in ascending id, through the point-location grid
__global__ void k_locate_points(LocateGrid g, const float2* pts, int n, int* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = locate(g, pts[i].x, pts[i].y);
}

inline int blocks_for(int n, int bt) { return (n + bt - 1) / bt; }

}  // namespace

void launch_compact(cudaStream_t s, int A, int* state, const int* cur, const int* targ, int P,
                    const CompactScenes& scn, int4* req, int* req_count, unsigned char* in_move, int* mv_count,
                    int* work_ctr, unsigned long long* stats) {
    k_compact<<<1, kCompactThreads, 0, s>>>(A, state, cur, targ, P, scn, req, req_count, in_move, mv_count,
                                            work_ctr, stats);
}

void launch_apply_targets(cudaStream_t s, const int4* recs, int n, int* state, int* targ_node,
                          float2* targ_pos) {
    if (n <= 0) return;
    k_apply_targets<<<blocks_for(n, 256), 256, 0, s>>>(recs, n, state, targ_node, targ_pos);
}

void launch_locate_points(cudaStream_t s, const LocateGrid& g, const float2* pts, int n, int* out) {
    if (n <= 0) return;
    k_locate_points<<<blocks_for(n, 256), 256, 0, s>>>(g, pts, n, out);
}

void launch_apply_targets_device(cudaStream_t s, const int* ids, const float2* pos, int n, int id_base,
                                 int id_count, const ScenePar* sc, const int* agent_scene, int* state,
                                 int* targ_node, float2* targ_pos, int* err) {
    if (n <= 0) return;
    k_apply_targets_device<<<blocks_for(n, 256), 256, 0, s>>>(ids, pos, n, id_base, id_count, sc, agent_scene,
                                                              state, targ_node, targ_pos, err);
}

void launch_prepare_batch(cudaStream_t s, const int* starts, const int* targets, int n, int nodes,
                          int4* req, int* req_count, int* work_ctr, int* err) {
    k_prepare_batch<<<blocks_for(n > 0 ? n : 1, 256), 256, 0, s>>>(starts, targets, n, nodes, req,
                                                                   req_count, work_ctr, err);
}

void launch_order_requests(cudaStream_t s, const int4* req_in, const int* req_count, int4* req_out, int* keys,
                           const unsigned short* lm, int L, int n) {
    k_order_requests<<<1, 1024, 0, s>>>(req_in, req_count, req_out, keys, lm, L, n);
}

void launch_move_bin(cudaStream_t s, const MoverParams& p) {
    k_move_bin<<<blocks_for(p.A, 256), 256, 0, s>>>(p);
}

void launch_cell_scan(cudaStream_t s, const MoverParams& p) { k_cell_scan<<<1, 1024, 0, s>>>(p); }

void launch_scatter(cudaStream_t s, const MoverParams& p) {
    k_scatter<<<blocks_for(p.A, 256), 256, 0, s>>>(p);
}

void launch_funnel(cudaStream_t s, const MoverParams& p) {
    if (p.A <= 0 || !p.waypoints) return;
    k_funnel<<<blocks_for(p.A, 128), 128, 0, s>>>(p);
}

void launch_collide_progress(cudaStream_t s, const MoverParams& p) {
    k_collide_progress<<<blocks_for(p.A, 128), 128, 0, s>>>(p);
}

}  // namespace gmapf_b200
