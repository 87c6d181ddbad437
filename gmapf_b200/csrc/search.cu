// search.cu -- bidirectional bounded-queue A* over the navmesh triangle graph.
//
// Method (reference: include/gmapf/PathFinder.h:138-251, CuQueue.h:33-70,
// CuVisitedMap.h:45-54, path layout PathFinder.h:253-307):
//   - T lanes per path request (T in {2,4,8,16,32}); lane q owns bounded
//     priority queue q of capacity C;
//   - lane 0 is seeded with the start, lane 1 with the target (F = K*h(s,t));
//   - each round every lane with a non-empty queue pops its minimum and
//     expands up to three neighbours: G' = G+1, F' = G' + K*h where h is the
//     squared centroid distance to the far end (target for nodes reached from
//     the start, start otherwise);
//   - a neighbour not yet claimed by this query is claimed (record written)
//     and appended to the round's frontier; a neighbour already claimed from
//     the other side is a meeting point; the first one ends the search;
//   - frontier item i is pushed into queue i mod T; a full queue evicts its
//     maximum, or drops the new item when it is not smaller than the maximum;
//   - all queues empty: not found.
// Determinism (the reference resolves these with racing atomics): queue
// order is (F, G, node id); within a round candidates are taken slot-major
// (neighbour slot 0 of lanes 0..T-1, then slot 1, then slot 2); the first
// candidate of a node claims it and the first conflicting candidate is the
// meeting pair.
//
// B200 mapping -- one warp per request:
//   - threads 0..T-1 own the T queues (sorted rings in shared memory,
//     maximum at the head and minimum at the tail: pop and eviction are O(1),
//     an insertion moves only the entries smaller than the new one -- the
//     reference's sorted array without its O(C) eviction shift);
//   - candidate c = slot*T + lane of a round is handled by warp thread
//     c mod 32 in pass c / 32 (one pass for T <= 8, two for T = 16, three for
//     T = 32), so thread order is candidate order and a single
//     __match_any_sync per pass resolves every claim of the pass: the lowest
//     fresh thread of a node claims it, later ones see the claim;
//   - visited state, one of four placements: a 2-bit-per-node bitmap
//     (claimed, side) per slot in shared memory; the same bitmap per slot in
//     global memory, sized to stay in L2 and cleared per query; that global
//     bitmap, moved into the shares of its block's finished warps by a search
//     still running at a batch's tail; or the
//     32-byte records themselves, stamped with the query epoch (no clearing
//     between queries, but one DRAM round trip per round);
//   - for T >= 16 the expanded node's parent (carried in its frontier entry)
//     is not a candidate: it is claimed from the same side, so it changes
//     nothing;
//   - the items a lane received but did not select are inserted into its
//     ring at the start of the next round, read from the frontier that is
//     still in place (no registers held across the round), and the ring's
//     cached minimum is reloaded only when the ring changed;
//   - records (G, parent and five further ancestors; with a visited bitmap
//     also the jump ancestor, the nearest ancestor at a depth that is a
//     multiple of 256) are written once per claimed node, each as one 32-byte
//     access; the path walk reads one record per six hops, on all lanes at
//     once between the jump ancestors; a node's record is read when it is
//     expanded, in flight together with its row (T <= 8) or with its
//     neighbours' visited state (T >= 16);
//   - idle warps refill from a device work counter (persistent form) or
//     stop (plain form).
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>

#include "internal.h"
#include "records.cuh"
#include "region_plan.cuh"

namespace gmapf_b200 {

namespace {

// (F, G, id) lexicographic; gd = G << 1 | dir
__device__ __forceinline__ bool key_less(float fa, int ga, int ia, float fb, int gb, int ib) {
    // G<<1|dir with the side bit set orders and ties exactly as G does
    const int Ga = ga | 1, Gb = gb | 1;
    return fa != fb ? fa < fb : (Ga != Gb ? Ga < Gb : ia < ib);
}

// A queued node: its key (F, G<<1|dir, id).
constexpr int kEntryWords = 3;

// Per-lane sorted ring in shared memory: entry k of lane q is (F, G<<1|dir)
// as one 8-byte word at fg[k*T + q] and the node id at id[k*T + q].
struct Ring {
    int* base;
    int T;
    int q;
    int C;
    __device__ __forceinline__ int at(int k) const {  // k in [0, 2C)
        return (k >= C ? k - C : k) * T + q;
    }
    __device__ __forceinline__ int2* fg() const { return reinterpret_cast<int2*>(base); }
    __device__ __forceinline__ int* id() const { return base + 2 * C * T; }
};

// bounded push (CuQueue.h:33-63 with the (F,G,id) order) into a ring holding
// at most cap entries, kept in descending order (minimum at the tail)
__device__ __forceinline__ void ring_push(const Ring& r, int& beg, int& size, int cap, float F, int gd, int id) {
    if (cap <= 0) return;
    if (size == cap) {
        const int k0 = r.at(beg);
        const int2 e = r.fg()[k0];
        if (!key_less(F, gd, id, __int_as_float(e.x), e.y, r.id()[k0]))
            return;                            // not below the maximum: dropped
        beg = (beg + 1 == r.C) ? 0 : beg + 1;  // evict the maximum
        size--;
    }
    int i = size - 1;
    while (i >= 0) {
        const int k = r.at(beg + i);
        const int2 e = r.fg()[k];
        const int ei = r.id()[k];
        if (!key_less(__int_as_float(e.x), e.y, ei, F, gd, id)) break;
        const int k1 = r.at(beg + i + 1);
        r.fg()[k1] = e;
        r.id()[k1] = ei;
        i--;
    }
    const int k1 = r.at(beg + i + 1);
    r.fg()[k1] = make_int2(__float_as_int(F), gd);
    r.id()[k1] = id;
    size++;
}

__device__ __forceinline__ int2 ld_state(const Rec* r) {
    return __ldcg(reinterpret_cast<const int2*>(r));
}

// 2-bit visited state: bit 0 = claimed, bit 1 = reached from the start
__device__ __forceinline__ int bm_bits(unsigned w, int n) { return (int)((w >> ((n & 15) << 1)) & 3u); }
__device__ __forceinline__ int bm_get(const unsigned* bm, int n) { return bm_bits(bm[n >> 4], n); }

// SHARED: the bitmap is in shared memory; otherwise in global memory, set by
// a reduction that returns nothing (no register or scoreboard held for it)
template <bool SHARED>
__device__ __forceinline__ void bm_set(unsigned* bm, int n, int dir) {
    const unsigned bit = (1u | ((unsigned)dir << 1)) << ((n & 15) << 1);
    if constexpr (SHARED)
        atomicOr(bm + (n >> 4), bit);
    else
        asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(bm + (n >> 4)), "r"(bit) : "memory");
}

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Serving ring: publish query q's completion after its results (lane 0,
// after the warp's writes are ordered by __syncwarp)
__device__ __forceinline__ void ring_complete(const SearchParams& p, int slot_row, int q, int found) {
    __threadfence_system();
    reinterpret_cast<volatile unsigned long long*>(p.done)[slot_row] =
        ((unsigned long long)(unsigned)(q + 1) << 1) | (unsigned long long)(found ? 1 : 0);
}

// per-warp shared-memory regions in 4-byte words, rounded to 16 bytes
__host__ __device__ __forceinline__ size_t search_queue_words(int C, int T) {
    return ((size_t)kEntryWords * C * T + 3) & ~(size_t)3;
}
// The round's frontier (3T entries: the queue key (F, G<<1|dir, id) and, for
// T >= 16, the claimed node's parent) and, for T >= 16, the owner lane of
// each of the 3T compacted candidates.  A node's parent is claimed from its
// side, so when the node is expanded the parent can be neither a claim nor a
// meeting point: for T >= 16 a node that arrives from the last frontier (the
// usual case: a search's queues hold few entries better than its newest)
// leaves its parent out of the round's candidates, which shortens the
// compacted pass without changing any claim, meet or frontier position.
__host__ __device__ __forceinline__ size_t search_frontier_words(int T) {
    return ((size_t)(kEntryWords + (T >= 16 ? 1 : 0)) * 3 * T + (T >= 16 ? 3 * (size_t)T : 0) + 3) & ~(size_t)3;
}


// Record word 0 in the bitmap placements: the nearest proper ancestor whose
// depth (G) is a multiple of kJumpDepth, -1 at a search's root.
constexpr int kJumpDepth = 256;

// Path output: depth d of the start side at out[d - 1] (d >= 1), depth d of
// the target side at out[gS + gT - d] (d >= 0).
__device__ __forceinline__ int path_pos(int side, int d, int gS, int gT) {
    return side == 0 ? d - 1 : gS + gT - d;
}

// Writes the path nodes at depths dx-1 down to b of one side, reading the
// records from node x (depth dx) down: six nodes per record.
__device__ __forceinline__ void walk_segment(const Rec* rec, int n_nodes, int* out, int side, int x, int dx, int b,
                                             int gS, int gT, int* err) {
    int g = dx;
    while (g > b) {
        if (x < 0 || x >= n_nodes) {
            atomicOr(err, ERR_BOUNDS);
            break;
        }
        int4 a, c;
        ld_rec(rec + x, a, c);
        const int anc[6] = {a.z, a.w, c.x, c.y, c.z, c.w};
#pragma unroll
        for (int j = 0; j < 6; j++) {
            const int d = g - 1 - j;
            if (d >= b) out[path_pos(side, d, gS, gT)] = anc[j];
        }
        x = anc[5];
        g -= 6;
    }
}

// Path walk of one warp.  With jump ancestors (records of the bitmap
// placements), lanes 0 and 1 first follow each side's jump chain from the
// meeting node, writing the checkpoints (the path nodes at depths that are
// multiples of kJumpDepth) to their output positions; then the segments
// between checkpoints, kJumpDepth hops each, are walked by all lanes at once.
// A path of g hops per side takes about g / kJumpDepth + kJumpDepth / 6
// dependent record reads instead of g / 6.  Without jump ancestors (stamped
// records) lanes 0 and 1 walk their sides from the meeting node.
template <bool JUMP>
__device__ __forceinline__ void walk_path(const Rec* rec, int n_nodes, int* out, int mS, int gS, int mT, int gT,
                                          int lane, int* err) {
    if (lane == 0 && gS >= 1) out[gS - 1] = mS;
    if (lane == 1) out[gS] = mT;
    if constexpr (!JUMP) {
        if (lane < 2)
            walk_segment(rec, n_nodes, out, lane, lane == 0 ? mS : mT, lane == 0 ? gS : gT, lane == 0 ? 1 : 0, gS,
                         gT, err);
    } else {
        // checkpoints k*D, k = 1..K of each side: K = (g - 1) / D
        int kc = 0;
        bool bad = false;
        if (lane < 2) {
            const int g = lane == 0 ? gS : gT;
            int x = lane == 0 ? mS : mT;
            kc = g >= 1 ? (g - 1) / kJumpDepth : 0;
            for (int k = kc; k >= 1; k--) {
                if (x < 0 || x >= n_nodes) {
                    bad = true;
                    break;
                }
                x = (int)__ldcg(&rec[x].stamp);  // the nearest ancestor at a multiple of D: depth k*D
                out[path_pos(lane, k * kJumpDepth, gS, gT)] = x;
            }
        }
        if (__any_sync(kFull, bad)) {
            if (lane == 0) atomicOr(err, ERR_BOUNDS);
            return;
        }
        const int kS = __shfl_sync(kFull, kc, 0), kT = __shfl_sync(kFull, kc, 1);
        __syncwarp();  // the checkpoints are written
        // segment k of a side: k = 0 from the meeting node down to depth kD + 1
        // (or the side's last depth), k >= 1 from the checkpoint at depth kD
        const int m = kS + 1 + kT + 1;
        for (int i = lane; i < m; i += 32) {
            const int side = i <= kS ? 0 : 1;
            const int k = side == 0 ? i : i - (kS + 1);
            const int kk = side == 0 ? kS : kT;
            const int last = side == 0 ? 1 : 0;
            int x, dx, b;
            if (k == 0) {
                x = side == 0 ? mS : mT;
                dx = side == 0 ? gS : gT;
                b = kk >= 1 ? kk * kJumpDepth + 1 : last;
            } else {
                dx = k * kJumpDepth;
                x = out[path_pos(side, dx, gS, gT)];
                b = k == 1 ? last : (k - 1) * kJumpDepth + 1;
            }
            walk_segment(rec, n_nodes, out, side, x, dx, b, gS, gT, err);
        }
    }
}

// VM: visited placement (1 shared-memory bitmap, 2 stamped records, 3 global
// bitmap, 4 global bitmap that a search still running at a batch's tail
// moves into the shared memory of its block's finished warps).  In modes 1, 3 and 4 a bit set by one thread is
// seen by the others after the next __syncwarp (bar.warp.sync orders memory
// among its threads).
//
// Placement 4: the block's shared memory holds each warp's queues and
// frontier contiguously, plus a pad sized so that all shares but one, with
// the pad, can hold one visited bitmap.  A search runs on its slot's global
// bitmap (placement 3's rounds); from p.promote_rounds rounds on, every 256
// rounds, it checks whether enough warps of its block have left the
// persistent loop (the work queue is empty: they never come back) for a run
// of their shares to hold its bitmap.  If so, and no other search of the
// block is in shared memory, it copies its bitmap into that run (its queues
// and frontier move to another free share when its own lies in the run) and
// runs its remaining rounds with the claim checks in shared memory
// (placement 1's rounds), then returns to its own share.  Alone, a round with
// the check in shared memory is ~15-18% shorter on the 101,698-triangle maze,
// and a frame's tail is its longest searches running on a nearly idle GPU.
// Results do not depend on where the bitmap is.
template <int T, int VM>
__global__ void __launch_bounds__(256, 3) k_search(SearchParams p, int persistent, int req_base, int bm_words) {
    constexpr bool SMEMV = VM == 1;  // bitmap in shared memory
    constexpr bool BMV = VM != 2;    // visited state in a bitmap (shared or global)
    constexpr bool JUMP = VM != 2;   // record word 0: the jump ancestor (else the query stamp)
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;                 // warp in block
    const int wpb = blockDim.x >> 5;                  // warps per block
    const int slot = blockIdx.x * wpb + wib;          // one request slot per warp
    const int n_nodes = p.n;
    const float K = p.K;
    const int C = p.C;
    // placement 4: the warps of this block that have left the persistent loop
    // (or never entered it; their shares stay free) and the warp whose search
    // runs in the block's shared memory (-1: none)
    __shared__ unsigned block_left;
    __shared__ int block_mover;
    if constexpr (VM == 4) {
        if (threadIdx.x == 0) {
            const int valid = max(0, min(wpb, p.slots - (int)blockIdx.x * wpb));
            block_left = (wpb >= 32 ? 0xffffffffu : ((1u << wpb) - 1u)) & ~((valid >= 32 ? 0xffffffffu : (1u << valid) - 1u));
            block_mover = -1;
        }
        __syncthreads();
    }

    // shared memory: [queues of every warp][frontiers of every warp][bitmaps]
    // (placement 4: [queues | frontier] of each warp, then the pad), each
    // per-warp region a whole number of 16-byte words
    const size_t qblk = search_queue_words(C, T), fblk = search_frontier_words(T);
    int* base = reinterpret_cast<int*>(smem);
    Ring ring;
    ring.base = VM == 4 ? base + (size_t)wib * (qblk + fblk) : base + (size_t)wib * qblk;
    ring.T = T;
    ring.q = lane < T ? lane : 0;
    ring.C = C;
    // word w of frontier item i at fr[w*3T + i]
    int* fr = VM == 4 ? ring.base + qblk : base + (size_t)wpb * qblk + (size_t)wib * fblk;
    unsigned* bm = SMEMV ? reinterpret_cast<unsigned*>(base + (size_t)wpb * (qblk + fblk)) + (size_t)wib * bm_words
                         : nullptr;

    if (slot >= p.slots) return;  // whole warps
    if (VM == 3 || VM == 4) bm = p.gbm + (size_t)(p.slot_base + slot) * bm_words;
    Rec* rec = p.rec + (size_t)(p.slot_base + slot) * n_nodes;
    const unsigned lt_mask = (1u << lane) - 1u;

    for (int iter = 0;; iter++) {
        // ------------------------------------------------------------ fetch
        int r, R;
        if (persistent) {
            int v = 0;
            if (lane == 0) v = atomicAdd(p.work_ctr, 1);
            r = __shfl_sync(kFull, v, 0);
            R = *p.req_count_d;
        } else {
            if (iter > 0) break;
            r = req_base + slot;
            R = p.req_count_h;
        }
        if (r >= R) break;
        // ring entries are rewritten by host copies over time: read past L1
        const int4 rq = p.ring_cap > 0 ? __ldcg(p.req + ((p.ring_base + r) % p.ring_cap)) : p.req[r];
        const int agent = rq.x, start = rq.y, target = rq.z, orow = rq.w;
        if (start < 0 || start >= n_nodes || target < 0 || target >= n_nodes || start == target) {
            const bool bad = start != target || start < 0 || start >= n_nodes;
            if (lane == 0) {  // bad request: not found; start == target: found, empty path
                if (p.timeline) p.timeline[2 * (long long)orow] = p.timeline[2 * (long long)orow + 1] = global_timer_ns();
                if (bad) atomicOr(p.err, ERR_BAD_REQUEST);
                if (p.out_found) p.out_found[orow] = bad ? 0 : 1;
                if (p.out_len) p.out_len[orow] = 0;
                if (agent >= 0 && p.ag_state) {
                    p.ag_state[agent] = GMAPF_AGENT_IDLE;
                    p.ag_path_len[agent] = 0;
                }
                if (!bad) atomicAdd(p.stats + ST_FOUND, 1ull);
                if (p.done) ring_complete(p, orow, p.ring_base + r, bad ? 0 : 1);
            }
            continue;
        }

        if (p.timeline && lane == 0) p.timeline[2 * (long long)orow] = global_timer_ns();
        unsigned ep = 0;
        if (VM == 2) {
            unsigned e = 0;
            if (lane == 0) e = p.epoch[p.slot_base + slot] + 1u;
            e = __shfl_sync(kFull, e, 0);
            if (e == 0u) {  // 2^32 queries in this slot: wipe its records once
                for (long long k = lane; k < (long long)n_nodes * 2; k += 32)
                    __stcg(reinterpret_cast<int4*>(rec) + k, make_int4(0, 0, 0, 0));
                e = 1u;
            }
            if (lane == 0) p.epoch[p.slot_base + slot] = e;
            ep = e;
        } else if (SMEMV) {
            uint4* b4 = reinterpret_cast<uint4*>(bm);
            for (int k = lane; k < (bm_words >> 2); k += 32) b4[k] = make_uint4(0, 0, 0, 0);
        } else {  // placements 3 and 4
            uint4* b4 = reinterpret_cast<uint4*>(bm);
            for (int k = lane; k < (bm_words >> 2); k += 32) __stcg(b4 + k, make_uint4(0, 0, 0, 0));
        }
        __syncwarp();
        const float2 cs = p.cen[start];
        const float2 ct = p.cen[target];
        const float f0 = GM_FMUL(dist_sqr(cs.x, cs.y, ct.x, ct.y), K);
        // Lane q's queue (lanes < T) is kept as: the node selected for the
        // coming round (uid/ugd, -1 if none), the ring in shared memory with its
        // minimum cached in registers (tF/tgd/tid), and up to three received
        // items waiting to be inserted (px*).  Pushing a round's items and then
        // popping the minimum equals selecting the minimum of (ring ∪ items)
        // first and inserting the rest with capacity C-1, so the insertion can
        // run while the next round's loads are in flight.
        int qbeg = 0, qsize = 0;
        int uid = -1, ugd = 0;
        int upar = -1;  // the selected node's parent when it came from the last frontier (-1: unknown)
        float tF = 0.f;
        int tgd = 0, tid = -1;
        bool pop_tail = false;
        bool pv[3] = {false, false, false};  // received items waiting for insertion
        bool more = false;                   // warp-uniform: the last round claimed more than T nodes
        if (lane < 2) {  // PathFinder.h:168-189: lane 0 seeds the start, lane 1 the target
            const int node = lane == 0 ? start : target;
            const int gd = lane == 0 ? 1 : 0;
            uid = node;
            ugd = gd;
            st_rec(rec + node, JUMP ? 0xffffffffu : ep, gd, -1, -1, -1, -1, -1, -1);
            if (BMV) bm_set<SMEMV>(bm, node, gd);
        }
        (void)f0;  // the seeds' F never takes part in a comparison: each seed is alone in its queue
        __syncwarp();

        unsigned expansions = 0, deg_sum = 0, claims = 2, rounds = 0;
        int found = 0, mS = -1, gS = 0, mT = -1, gT = 0;
        int next_check = p.promote_rounds;  // placement 4: the round of the next room-in-block check

        // ------------------------------------------------------------ rounds
        // The rounds with the claim checks in placement VX (1 shared, 2
        // records, 3 global bitmap) on bitmap bmx.  Returns true when the
        // search has ended, false when (placement 4) enough warps of its block
        // have left for its bitmap to fit in their shares.
        auto run_rounds = [&](auto vtag, unsigned* bmx) -> bool {
          constexpr int VX = decltype(vtag)::value;
          constexpr bool SMX = VX == 1;
          for (;;) {
            rounds++;
            // lanes < T expand the node selected at the end of the previous round
            const int idu = (lane < T) ? uid : -1;
            const int gdu = ugd;

            int nwin = 0;
            bool meet = false;
            int mu = 0, mgu = 0, mn = 0, mgn = 0, mgn_known = 0;

            // One claim pass over up to 32 candidates, in candidate order by
            // thread index: visited state, the lowest fresh thread of a node
            // claims it, the first conflicting thread is the meeting pair.
            auto resolve = [&](bool valid, int cu, int cgdu, int n, float cx, float cy, const int4& ra,
                               const int4& rb, int2 cst, bool later_pass) {
                const int du = cgdu & 1;
                const int ngd = cgdu + 2;  // (G + 1) << 1 | dir
                bool prev = false;
                int pside = 0, pgd = 0, pknown = 0;  // earlier claim: side, G<<1|side if known
                if (valid) {
                    if (VX == 1) {  // includes earlier passes of this round
                        const int st = bm_get(bmx, n);
                        prev = (st & 1) != 0;
                        pside = st >> 1;
                    } else if (VX == 3) {  // word loaded at the start of the round
                        const int st = bm_bits((unsigned)cst.x, n);
                        prev = (st & 1) != 0;
                        pside = st >> 1;
                    } else {
                        prev = (unsigned)cst.x == ep;
                        pgd = cst.y;
                        pside = pgd & 1;
                        pknown = 1;
                    }
                    if (VX == 2 && later_pass && !prev) {  // claimed by an earlier pass of this round
                        int hit = -1;
                        for (int w = 0; w < nwin; w++) hit = (fr[6 * T + w] == n) ? w : hit;
                        if (hit >= 0) {
                            prev = true;
                            pgd = fr[3 * T + hit];
                            pside = pgd & 1;
                            pknown = 1;
                        }
                    }
                }
                const bool fresh = valid && !prev;
                const unsigned dm = __ballot_sync(kFull, du);  // candidates' sides
                const unsigned mm = __match_any_sync(kFull, fresh ? n : -1);
                const int leader = __ffs(mm) - 1;
                const bool win = fresh && leader == lane;
                const bool dup = fresh && !win;  // same node as a lower candidate of this pass
                const bool conflict = dup ? (int)((dm >> leader) & 1u) != du : (prev && pside != du);
                const unsigned cm = __ballot_sync(kFull, conflict);
                if (!meet && cm != 0u) {  // warp-uniform
                    const int lgd = __shfl_sync(kFull, ngd, leader);
                    const int cgd = dup ? lgd : pgd;
                    const int cknown = dup ? 1 : pknown;
                    const int ml = __ffs(cm) - 1;
                    mu = __shfl_sync(kFull, cu, ml);
                    mgu = __shfl_sync(kFull, cgdu, ml);
                    mn = __shfl_sync(kFull, n, ml);
                    mgn = __shfl_sync(kFull, cgd, ml);
                    mgn_known = __shfl_sync(kFull, cknown, ml);
                    meet = true;
                }
                const unsigned wm = __ballot_sync(kFull, win);
                if (win) {
                    const int idx = nwin + __popc(wm & lt_mask);
                    const float farx = du ? ct.x : cs.x;
                    const float fary = du ? ct.y : cs.y;
                    const float hh = dist_sqr(cx, cy, farx, fary);
                    const float F = GM_FADD((float)(ngd >> 1), GM_FMUL(hh, K));
                    fr[idx] = __float_as_int(F);
                    fr[3 * T + idx] = ngd;
                    fr[6 * T + idx] = n;
                    if constexpr (T >= 16) fr[9 * T + idx] = cu;  // its parent: same side, never a claim or a meet
                    if (BMV) bm_set<SMX>(bmx, n, du);
                    // ancestors 1..5 of n = ancestors 0..4 of the popped node
                    // the jump ancestor: the parent when its depth is a multiple of
                    // kJumpDepth, else the parent's jump ancestor (its record word 0)
                    const unsigned w0 = JUMP ? (((cgdu >> 1) & (kJumpDepth - 1)) == 0 ? (unsigned)cu : (unsigned)ra.x) : ep;
                    st_rec(rec + n, w0, ngd, cu, ra.z, ra.w, rb.x, rb.y, rb.z);
                }
                nwin += __popc(wm);
                __syncwarp();
            };

            // deferred queue work of the previous round, placed where the loads
            // issued before it are still in flight
            auto deferred_queue_work = [&]() {
                if (lane < T) {
                    const bool touched = pop_tail || pv[0] || (more && (pv[1] || pv[2]));
                    if (pop_tail) qsize--;
                    // the last round's frontier is still in place: read the items from it
                    if (pv[0]) ring_push(ring, qbeg, qsize, C - 1, __int_as_float(fr[lane]), fr[3 * T + lane], fr[6 * T + lane]);
                    if (more) {  // items lane + T, lane + 2T exist only when nwin > T
                        if (pv[1])
                            ring_push(ring, qbeg, qsize, C - 1, __int_as_float(fr[lane + T]), fr[4 * T + lane],
                                      fr[7 * T + lane]);
                        if (pv[2])
                            ring_push(ring, qbeg, qsize, C - 1, __int_as_float(fr[lane + 2 * T]), fr[5 * T + lane],
                                      fr[8 * T + lane]);
                    }
                    if (touched && qsize > 0) {  // an untouched ring keeps its cached minimum
                        const int k = ring.at(qbeg + qsize - 1);
                        const int2 e = ring.fg()[k];
                        tF = __int_as_float(e.x);
                        tgd = e.y;
                        tid = ring.id()[k];
                    }
                }
            };

            if constexpr (T <= 8) {
                // one pass: thread c = slot*T + lane handles candidate c directly
                const int c = lane, sl = c / T, qq = c - sl * T;
                const int cu = __shfl_sync(kFull, idu, qq & 31);
                const int cgdu = __shfl_sync(kFull, gdu, qq & 31);
                bool valid = c < 3 * T && cu >= 0;
                int n = -1;
                float cx = 0.f, cy = 0.f;
                int4 ra = make_int4(0, 0, -1, -1), rb = make_int4(-1, -1, -1, -1);
                int2 cst = make_int2(0, 0);
                if (valid) {
                    const SearchRow* rw = p.rows + cu;
                    const int4 r0 = __ldg(reinterpret_cast<const int4*>(rw));
                    const float2 cc = __ldg(reinterpret_cast<const float2*>(&rw->x0) + sl);
                    ld_rec(rec + cu, ra, rb);  // the popped node's ancestors
                    n = (sl == 0) ? r0.x : (sl == 1) ? r0.y : r0.z;
                    valid = sl < r0.w;
                    cx = cc.x;
                    cy = cc.y;
                    if (sl == 0) {
                        expansions++;
                        deg_sum += (unsigned)r0.w;
                    }
                    if (VX == 2 && valid) cst = ld_state(rec + n);  // claims of earlier rounds
                    if (VX == 3 && valid) cst.x = (int)__ldcg(bmx + (n >> 4));
                }
                deferred_queue_work();
                resolve(valid, cu, cgdu, n, cx, cy, ra, rb, cst, false);
            } else {
                // compacted candidates: slot-major (slot 0 of every expanding lane,
                // then slot 1, then slot 2) -- usually one pass of at most 32
                int4 r0 = make_int4(-1, -1, -1, 0);
                if (idu >= 0) r0 = __ldg(reinterpret_cast<const int4*>(p.rows + idu));
                deferred_queue_work();
                // the popped node's parent is claimed from its side: it can be
                // neither a claim nor a meet, so it is left out of the candidates
                const bool k0 = idu >= 0 && r0.w > 0 && r0.x != upar;
                const bool k1 = idu >= 0 && r0.w > 1 && r0.y != upar;
                const bool k2 = idu >= 0 && r0.w > 2 && r0.z != upar;
                const unsigned b0 = __ballot_sync(kFull, k0);
                const unsigned b1 = __ballot_sync(kFull, k1);
                const unsigned b2 = __ballot_sync(kFull, k2);
                if (idu >= 0) {
                    expansions++;
                    deg_sum += (unsigned)r0.w;
                }
                const int n0 = __popc(b0), n1 = __popc(b1), total = n0 + n1 + __popc(b2);
                // each owner writes its lane at its candidates' compacted positions
                // (a ballot rank is one popc; the inverse, the n-th set bit, is not)
                int* oix = fr + 12 * T;
                if (k0) oix[__popc(b0 & lt_mask)] = lane;
                if (k1) oix[n0 + __popc(b1 & lt_mask)] = lane;
                if (k2) oix[n0 + n1 + __popc(b2 & lt_mask)] = lane;
                __syncwarp();
                for (int base = 0; base < total; base += 32) {  // warp-uniform
                    const int t = base + lane;
                    const int sl = t < n0 ? 0 : (t < n0 + n1 ? 1 : 2);
                    const int qq = t < total ? (oix[t] & 31) : 0;  // the candidate's owner lane
                    const int cu = __shfl_sync(kFull, idu, qq);
                    const int cgdu = __shfl_sync(kFull, gdu, qq);
                    const int na = __shfl_sync(kFull, r0.x, qq);
                    const int nb = __shfl_sync(kFull, r0.y, qq);
                    const int nc = __shfl_sync(kFull, r0.z, qq);
                    int n = sl == 0 ? na : (sl == 1 ? nb : nc);
                    const bool valid = t < total && (unsigned)cu < (unsigned)n_nodes && (unsigned)n < (unsigned)n_nodes;
                    if (!valid) n = -1;
                    float cx = 0.f, cy = 0.f;
                    int4 ra = make_int4(0, 0, -1, -1), rb = make_int4(-1, -1, -1, -1);
                    int2 cst = make_int2(0, 0);
                    if (valid) {
                        const float2 cc = __ldg(reinterpret_cast<const float2*>(&p.rows[cu].x0) + sl);
                        ld_rec(rec + cu, ra, rb);
                        cx = cc.x;
                        cy = cc.y;
                        if (VX == 2) cst = ld_state(rec + n);
                        if (VX == 3) cst.x = (int)__ldcg(bmx + (n >> 4));
                    }
                    resolve(valid, cu, cgdu, n, cx, cy, ra, rb, cst, base > 0);
                }
            }
            claims += (unsigned)nwin;
            bool ended = false;
            if (meet) {
                if (!mgn_known) {  // side came from the bitmap: read G from the record
                    int g = 0;
                    if (lane == 0) g = ld_state(rec + mn).y;
                    mgn = __shfl_sync(kFull, g, 0);
                }
                if (mgu & 1) {  // PathFinder.h:226-227
                    mS = mu;
                    gS = mgu >> 1;
                    mT = mn;
                    gT = mgn >> 1;
                } else {
                    mS = mn;
                    gS = mgn >> 1;
                    mT = mu;
                    gT = mgu >> 1;
                }
                found = 1;
                ended = true;
            } else {
                // frontier item i goes to queue i mod T (items lane, lane+T, lane+2T);
                // select the next pop in registers
                int best = -1;  // -1: the ring's minimum; 0..2: a received item
                bool have = lane < T && qsize > 0;
                float bF = tF;
                int bg = tgd, bi = tid;
                more = nwin > T;
                // branch-free (an absent item reads slot 0 and is ignored):
                // selects instead of a divergent branch per item, 5% of a round
                auto take = [&](int j) {
                    const int i = lane + j * T;
                    pv[j] = lane < T && i < nwin;
                    const int ii = pv[j] ? i : 0;
                    const float xF = __int_as_float(fr[ii]);
                    const int xg = fr[3 * T + ii], xi = fr[6 * T + ii];
                    const bool better = pv[j] && (!have || key_less(xF, xg, xi, bF, bg, bi));
                    best = better ? j : best;
                    have = have || better;
                    bF = better ? xF : bF;
                    bg = better ? xg : bg;
                    bi = better ? xi : bi;
                };
                take(0);
                if (more) {
                    take(1);
                    take(2);
                } else {
                    pv[1] = false;
                    pv[2] = false;
                }
                uid = have ? bi : -1;
                ugd = bg;
                pop_tail = have && best < 0;  // otherwise the ring is untouched by the pop
                if constexpr (T >= 16) upar = (have && best >= 0) ? fr[9 * T + lane + best * T] : -1;
#pragma unroll
                for (int j = 0; j < 3; j++) pv[j] = pv[j] && j != best;  // the rest waits for insertion
                if (!__any_sync(kFull, uid >= 0))
                    ended = true;
                else if ((int)rounds >= p.max_rounds) {  // still running after its last allowed round
                    if (lane == 0) atomicOr(p.err, ERR_ROUNDS);
                    ended = true;
                }
            }
            __syncwarp();  // frontier reads done before the next round rewrites it
            if (ended) return true;
            if constexpr (VM == 4 && VX == 3) {
                // at promote_rounds rounds, then every 256: enough shares free
                // (their count; where the bitmap goes is worked out outside)?
                if ((int)rounds == next_check) {  // warp-uniform
                    next_check += 256;
                    int room = 0;
                    if (lane == 0)
                        room = __popc(*reinterpret_cast<volatile unsigned*>(&block_left) | (1u << wib)) >=
                               region_shares_needed(bm_words, wpb, (int)(qblk + fblk));
                    if (__shfl_sync(kFull, room, 0)) return false;
                }
            }
          }
        };
        if constexpr (VM == 4) {
            int move_plan = -1;
            while (!run_rounds(std::integral_constant<int, 3>{}, bm)) {
                if (lane == 0) {
                    move_plan = region_plan(*reinterpret_cast<volatile unsigned*>(&block_left), wib, wpb,
                                            (int)(qblk + fblk), bm_words,
                                            (int)search_pad_words(bm_words, wpb, (int)(qblk + fblk)));
                    if (move_plan >= 0 && atomicCAS(&block_mover, -1, wib) != -1) move_plan = -1;
                }
                move_plan = __shfl_sync(kFull, move_plan, 0);
                if (move_plan >= 0) break;  // else back to the rounds: the next check in 256
            }
            if (move_plan >= 0) {
                // shares of warps that have left hold the bitmap from share
                // `first` on; this warp's queues and frontier move to share `home`
                // when its own share lies in that run (the deferred items stay in
                // place in the frontier); the search goes on there
                __threadfence_block();
                const int first = move_plan & 0xff, home = move_plan >> 8;
                if (home != wib) {
                    const int4* from = reinterpret_cast<const int4*>(ring.base);
                    int4* to = reinterpret_cast<int4*>(base + (size_t)home * (qblk + fblk));
                    for (int k = lane; k < (int)((qblk + fblk) >> 2); k += 32) to[k] = from[k];
                    __syncwarp();
                    ring.base = base + (size_t)home * (qblk + fblk);
                    fr = ring.base + qblk;
                }
                unsigned* region = reinterpret_cast<unsigned*>(base + (size_t)first * (qblk + fblk));
                const uint4* g4 = reinterpret_cast<const uint4*>(bm);
                uint4* s4 = reinterpret_cast<uint4*>(region);
                for (int k = lane; k < (bm_words >> 2); k += 32) s4[k] = __ldcg(g4 + k);
                __syncwarp();
                run_rounds(std::integral_constant<int, 1>{}, region);
                // back to the warp's own share (the next query starts afresh) and
                // the block's shared memory free for another search
                ring.base = base + (size_t)wib * (qblk + fblk);
                fr = ring.base + qblk;
                __syncwarp();
                __threadfence_block();
                if (lane == 0) {
                    atomicExch(&block_mover, -1);
                    atomicAdd(p.stats + ST_PROMOTED, 1ull);
                }
            }
        } else {
            run_rounds(std::integral_constant<int, VM>{}, bm);
        }

        // ------------------------------------------------------------ path walk
        int L = 0;
        if (found) {
            L = gS + gT + 1;
            const int row = (agent >= 0) ? agent : orow;
            if ((long long)L > p.path_stride) {
                if (lane == 0) atomicOr(p.err, ERR_PATH_CAP);
            } else {
                walk_path<JUMP>(rec, n_nodes, p.paths + (long long)row * p.path_stride, mS, gS, mT, gT, lane, p.err);
            }
        }
        __syncwarp();
        // results, agent update (PathFinder.h:268-289) and counters
        const unsigned ex = __reduce_add_sync(kFull, expansions);
        const unsigned ds = __reduce_add_sync(kFull, deg_sum);
        if (lane == 0) {
            if (p.out_found) p.out_found[orow] = found;
            if (p.out_len) p.out_len[orow] = L;
            if (agent >= 0 && p.ag_state) {
                // PathFinder.h:268-289: not found -> Idle with the path step
                // index left as it was; found -> Move from step -1
                p.ag_state[agent] = found ? GMAPF_AGENT_MOVE : GMAPF_AGENT_IDLE;
                if (found) p.ag_step_idx[agent] = -1;
                p.ag_path_len[agent] = L;
            }
            atomicAdd(p.stats + ST_EXPANSIONS, (unsigned long long)ex);
            atomicAdd(p.stats + ST_DEG_SUM, (unsigned long long)ds);
            atomicAdd(p.stats + ST_ROUNDS, (unsigned long long)rounds);
            atomicAdd(p.stats + ST_CLAIMS, (unsigned long long)claims);
            atomicAdd(p.stats + ST_PATH_NODES, (unsigned long long)L);
            atomicAdd(p.stats + ST_FOUND, (unsigned long long)found);
            if (p.done) ring_complete(p, orow, p.ring_base + r, found);
            if (p.timeline) p.timeline[2 * (long long)orow + 1] = global_timer_ns();
        }
    }
    if constexpr (VM == 4) {  // this warp uses its block's shared memory no more
        __syncwarp();
        __threadfence_block();
        if (lane == 0) atomicOr(&block_left, 1u << wib);
    }
}

template <int T, int VM>
cudaError_t launch_t(cudaStream_t s, const SearchParams& p, int blocks, int bt, bool persistent,
                     int req_base, int bm_words) {
    // the dynamic shared-memory limit was raised when the search state was
    // sized (no attribute calls here: this may run under stream capture)
    const size_t smem = search_smem_bytes(p.C, bt, bm_words, T, VM);
    if (blocks <= 0) return cudaSuccess;
    k_search<T, VM><<<blocks, bt, smem, s>>>(p, persistent ? 1 : 0, req_base, bm_words);
    return cudaGetLastError();
}

// The dynamic shared-memory limit is an attribute of the kernel on a device,
// shared by every context of the process: it is only ever raised, so a
// context sized for a small map never lowers the limit under a live context
// sized for a larger one.
std::mutex g_smem_attr_mu;

template <int T, int VM>
int& smem_attr(int device) {
    static int limit[64] = {};
    return limit[device & 63];
}

template <int T, int VM>
int occupancy_t(int C, int bt, int bm_words) {
    if (bt > 256) return 0;  // the kernel's launch bounds
    const size_t smem = search_smem_bytes(C, bt, bm_words, T, VM);
    if (smem > 227 * 1024) return 0;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    {
        std::lock_guard<std::mutex> lock(g_smem_attr_mu);
        int& limit = smem_attr<T, VM>(device);
        if ((int)smem > limit) {
            if (cudaFuncSetAttribute(k_search<T, VM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess) {
                cudaGetLastError();
                return 0;
            }
            limit = (int)smem;
        }
    }
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search<T, VM>, bt, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

template <int VM>
cudaError_t launch_v(cudaStream_t s, const SearchParams& p, int blocks, int bt, bool persistent,
                     int req_base, int bm_words) {
    switch (p.T) {
        case 2: return launch_t<2, VM>(s, p, blocks, bt, persistent, req_base, bm_words);
        case 4: return launch_t<4, VM>(s, p, blocks, bt, persistent, req_base, bm_words);
        case 8: return launch_t<8, VM>(s, p, blocks, bt, persistent, req_base, bm_words);
        case 16: return launch_t<16, VM>(s, p, blocks, bt, persistent, req_base, bm_words);
        case 32: return launch_t<32, VM>(s, p, blocks, bt, persistent, req_base, bm_words);
        default: return cudaErrorInvalidValue;
    }
}

template <int VM>
int occupancy_v(int T, int C, int bt, int bm_words) {
    switch (T) {
        case 2: return occupancy_t<2, VM>(C, bt, bm_words);
        case 4: return occupancy_t<4, VM>(C, bt, bm_words);
        case 8: return occupancy_t<8, VM>(C, bt, bm_words);
        case 16: return occupancy_t<16, VM>(C, bt, bm_words);
        case 32: return occupancy_t<32, VM>(C, bt, bm_words);
        default: return 0;
    }
}

}  // namespace

// per-block dynamic shared memory, per warp: T queues of C entries (12 B),
// a frontier of 3T entries (12 B) and, in visited mode 1, the visited bitmap;
// in visited mode 4 a pad so that all but the first warp's share can hold one
// bitmap
size_t search_smem_bytes(int C, int bt, int bm_words, int T, int vm) {
    const size_t warps = (size_t)bt / 32;
    const size_t per_warp = search_queue_words(C, T) + search_frontier_words(T);
    const size_t pad = vm == 4 ? search_pad_words(bm_words, (int)warps, (int)per_warp) : 0;
    return 4 * (warps * (per_warp + (vm == 1 ? (size_t)bm_words : 0)) + pad);
}

int search_bitmap_words(int n_nodes) {
    const int w = (n_nodes + 15) / 16;
    return (w + 3) & ~3;  // whole uint4 for the clear
}

int search_max_blocks_per_sm(int T, int C, int bt, int vm, int bm_words) {
    switch (vm) {
        case 1: return occupancy_v<1>(T, C, bt, bm_words);
        case 2: return occupancy_v<2>(T, C, bt, 0);
        case 3: return occupancy_v<3>(T, C, bt, 0);
        case 4: return occupancy_v<4>(T, C, bt, bm_words);
        default: return 0;
    }
}

cudaError_t launch_search(cudaStream_t s, const SearchParams& p, int blocks, int bt, bool persistent,
                          int req_base, int vm, int bm_words) {
    switch (vm) {
        case 1: return launch_v<1>(s, p, blocks, bt, persistent, req_base, bm_words);
        case 2: return launch_v<2>(s, p, blocks, bt, persistent, req_base, 0);
        case 3: return launch_v<3>(s, p, blocks, bt, persistent, req_base, bm_words);
        case 4: return launch_v<4>(s, p, blocks, bt, persistent, req_base, bm_words);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace gmapf_b200
