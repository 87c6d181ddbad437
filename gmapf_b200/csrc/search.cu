// search.cu -- bidirectional bounded-queue A* over the navmesh triangle graph.
//
// Method (reference: include/gmapf/PathFinder.h:138-251, CuQueue.h:33-70,
// CuVisitedMap.h:45-54, path layout PathFinder.h:253-307):
//   - one lane group of T threads (T in {2,4,8,16,32}, inside one warp) per
//     path request; lane q owns bounded priority queue q of capacity C;
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
// meeting pair.  Same-slot duplicates are resolved with __match_any_sync,
// earlier-slot duplicates with the round's winner list in shared memory.
//
// B200 layout: the per-lane queues are binary min-heaps in shared memory,
// element k of thread t at [k * blockDim + t] (bank = lane: conflict-free);
// the map is read as 48-byte SearchRows through the read-only path; visited
// state is a 32-byte record per (slot, node) stamped with the query epoch so
// nothing is cleared between queries; records carry six ancestors so the
// path walk reads one record per six hops.
#include <cuda_runtime.h>

#include "internal.h"

namespace gmapf_b200 {

namespace {

struct HeapRef {
    float* F;
    int* GD;
    int* ID;
    int stride;  // blockDim.x
    int t;       // thread index
    __device__ __forceinline__ int at(int k) const { return k * stride + t; }
};

// (F, G, id) lexicographic; gd = G << 1 | dir
__device__ __forceinline__ bool key_less(float fa, int ga, int ia, float fb, int gb, int ib) {
    if (fa != fb) return fa < fb;
    int Ga = ga >> 1, Gb = gb >> 1;
    if (Ga != Gb) return Ga < Gb;
    return ia < ib;
}

__device__ __forceinline__ void heap_pop(const HeapRef& h, int& size, float& F, int& gd, int& id) {
    F = h.F[h.at(0)];
    gd = h.GD[h.at(0)];
    id = h.ID[h.at(0)];
    int n = --size;
    if (n == 0) return;
    float xf = h.F[h.at(n)];
    int xg = h.GD[h.at(n)], xi = h.ID[h.at(n)];
    int i = 0;
    for (;;) {
        int c = 2 * i + 1;
        if (c >= n) break;
        float cf = h.F[h.at(c)];
        int cg = h.GD[h.at(c)], ci = h.ID[h.at(c)];
        if (c + 1 < n) {
            float df = h.F[h.at(c + 1)];
            int dg = h.GD[h.at(c + 1)], di = h.ID[h.at(c + 1)];
            if (key_less(df, dg, di, cf, cg, ci)) {
                c = c + 1;
                cf = df;
                cg = dg;
                ci = di;
            }
        }
        if (!key_less(cf, cg, ci, xf, xg, xi)) break;
        h.F[h.at(i)] = cf;
        h.GD[h.at(i)] = cg;
        h.ID[h.at(i)] = ci;
        i = c;
    }
    h.F[h.at(i)] = xf;
    h.GD[h.at(i)] = xg;
    h.ID[h.at(i)] = xi;
}

__device__ __forceinline__ void heap_sift_up(const HeapRef& h, int i, float xf, int xg, int xi) {
    while (i > 0) {
        int p = (i - 1) >> 1;
        float pf = h.F[h.at(p)];
        int pg = h.GD[h.at(p)], pi = h.ID[h.at(p)];
        if (!key_less(xf, xg, xi, pf, pg, pi)) break;
        h.F[h.at(i)] = pf;
        h.GD[h.at(i)] = pg;
        h.ID[h.at(i)] = pi;
        i = p;
    }
    h.F[h.at(i)] = xf;
    h.GD[h.at(i)] = xg;
    h.ID[h.at(i)] = xi;
}

// Bounded push (CuQueue.h:33-63 with the (F,G,id) order): below capacity the
// item is inserted; at capacity the maximum (always a leaf of the min-heap)
// is replaced by the item when the item is smaller, else the item is dropped.
__device__ __forceinline__ void heap_push(const HeapRef& h, int& size, int cap, float F, int gd,
                                          int id) {
    if (size < cap) {
        heap_sift_up(h, size, F, gd, id);
        size++;
        return;
    }
    int m = size >> 1;
    float mf = h.F[h.at(m)];
    int mg = h.GD[h.at(m)], mi = h.ID[h.at(m)];
    for (int k = m + 1; k < size; k++) {
        float kf = h.F[h.at(k)];
        int kg = h.GD[h.at(k)], ki = h.ID[h.at(k)];
        if (key_less(mf, mg, mi, kf, kg, ki)) {
            m = k;
            mf = kf;
            mg = kg;
            mi = ki;
        }
    }
    if (!key_less(F, gd, id, mf, mg, mi)) return;
    heap_sift_up(h, m, F, gd, id);
}

__device__ __forceinline__ int2 ld_state(const Rec* r) {
    return __ldcg(reinterpret_cast<const int2*>(r));
}

__device__ __forceinline__ void ld_rec(const Rec* r, int4& a, int4& b) {
    a = __ldcg(reinterpret_cast<const int4*>(r));
    b = __ldcg(reinterpret_cast<const int4*>(r) + 1);
}

__device__ __forceinline__ void st_rec(Rec* r, unsigned stamp, int gd, int a0, int a1, int a2,
                                       int a3, int a4, int a5) {
    __stcg(reinterpret_cast<int4*>(r), make_int4((int)stamp, gd, a0, a1));
    __stcg(reinterpret_cast<int4*>(r) + 1, make_int4(a2, a3, a4, a5));
}

template <int T>
__global__ void __launch_bounds__(256) k_search(SearchParams p, int persistent, int req_base) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int q = tid & (T - 1);
    const int gbase_lane = lane & ~(T - 1);
    const unsigned gmask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << gbase_lane);
    const int C = p.C;
    const int groups_per_block = B / T;
    const int group = tid / T;
    const int slot = blockIdx.x * groups_per_block + group;
    const int n_nodes = p.n;

    HeapRef h;
    h.F = reinterpret_cast<float*>(smem);
    h.GD = reinterpret_cast<int*>(h.F + (size_t)C * B);
    h.ID = h.GD + (size_t)C * B;
    h.stride = B;
    h.t = tid;
    int* wId = h.ID + (size_t)C * B;
    int* wGD = wId + 3 * B;
    float* wF = reinterpret_cast<float*>(wGD + 3 * B);
    const int wb = group * 3 * T;  // this group's winner list

    if (slot >= p.slots) return;  // whole groups: slot is group-uniform
    Rec* rec = p.rec + (size_t)slot * n_nodes;
    const float K = p.K;

    for (int iter = 0;; iter++) {
        int r;
        int R;
        if (persistent) {
            int v = 0;
            if (q == 0) v = atomicAdd(p.work_ctr, 1);
            r = __shfl_sync(gmask, v, gbase_lane);
            R = *p.req_count_d;
        } else {
            if (iter > 0) break;
            r = req_base + slot;
            R = p.req_count_h;
        }
        if (r >= R) break;

        const int4 rq = p.req[r];
        const int agent = rq.x, start = rq.y, target = rq.z, orow = rq.w;
        if (start < 0 || start >= n_nodes || target < 0 || target >= n_nodes) {
            if (q == 0) {
                atomicOr(p.err, ERR_BAD_REQUEST);
                if (p.out_found) p.out_found[r] = 0;
                if (p.out_len) p.out_len[r] = 0;
                if (agent >= 0 && p.ag_state) {
                    p.ag_state[agent] = GMAPF_AGENT_IDLE;
                    p.ag_path_len[agent] = 0;
                }
            }
            continue;
        }

        if (start == target) {  // already there: found, empty path (never a step request)
            if (q == 0) {
                if (p.out_found) p.out_found[r] = 1;
                if (p.out_len) p.out_len[r] = 0;
                atomicAdd(p.stats + ST_FOUND, 1ull);
            }
            continue;
        }

        // epoch of this query in this slot (slot-private; no atomics needed)
        unsigned ep = 0;
        if (q == 0) ep = p.epoch[slot] + 1u;
        ep = __shfl_sync(gmask, ep, gbase_lane);
        if (ep == 0u) {  // 2^32 queries in this slot: wipe its records once
            for (long long k = q; k < (long long)n_nodes * 2; k += T)
                __stcg(reinterpret_cast<int4*>(rec) + k, make_int4(0, 0, 0, 0));
            __syncwarp(gmask);
            ep = 1u;
        }
        if (q == 0) p.epoch[slot] = ep;

        const float2 cs = p.cen[start];
        const float2 ct = p.cen[target];
        const float f0 = GM_FMUL(dist_sqr(cs.x, cs.y, ct.x, ct.y), K);

        int hsize = 0;
        if (q == 0) {  // PathFinder.h:168-178
            heap_push(h, hsize, C, f0, (0 << 1) | 1, start);
            st_rec(rec + start, ep, 1, -1, -1, -1, -1, -1, -1);
        } else if (q == 1) {  // PathFinder.h:179-189
            heap_push(h, hsize, C, f0, (0 << 1) | 0, target);
            st_rec(rec + target, ep, 0, -1, -1, -1, -1, -1, -1);
        }
        __syncwarp(gmask);

        unsigned expansions = 0, deg_sum = 0, claims = (q == 0) ? 2u : 0u;
        unsigned rounds = 0;
        int found = 0, mS = -1, gS = 0, mT = -1, gT = 0;

        for (;;) {
            rounds++;
            if ((int)rounds > p.max_rounds) {
                if (q == 0) atomicOr(p.err, ERR_ROUNDS);
                break;
            }
            const bool has = hsize > 0;
            float Fu = 0.f;
            int gdu = 0, idu = 0;
            if (has) heap_pop(h, hsize, Fu, gdu, idu);

            int deg = 0;
            int nid0 = -1, nid1 = -1, nid2 = -1;
            float nx0 = 0, ny0 = 0, nx1 = 0, ny1 = 0, nx2 = 0, ny2 = 0;
            int4 ra = make_int4(0, 0, -1, -1), rb = make_int4(-1, -1, -1, -1);
            if (has) {
                const int4* rp = reinterpret_cast<const int4*>(p.rows + idu);
                const int4 r0 = __ldg(rp);
                const float4 r1 = __ldg(reinterpret_cast<const float4*>(rp + 1));
                const float4 r2 = __ldg(reinterpret_cast<const float4*>(rp + 2));
                ld_rec(rec + idu, ra, rb);
                nid0 = r0.x;
                nid1 = r0.y;
                nid2 = r0.z;
                deg = r0.w;
                nx0 = r1.x;
                ny0 = r1.y;
                nx1 = r1.z;
                ny1 = r1.w;
                nx2 = r2.x;
                ny2 = r2.y;
                expansions++;
                deg_sum += (unsigned)deg;
            }
            const int du = gdu & 1;
            const int Gn = (gdu >> 1) + 1;
            const int ngd = (Gn << 1) | du;
            const float farx = du ? ct.x : cs.x;
            const float fary = du ? ct.y : cs.y;

            // previous-round claim state of every candidate (one L2 round trip)
            int2 s0 = make_int2(0, 0), s1 = make_int2(0, 0), s2 = make_int2(0, 0);
            if (deg > 0) s0 = ld_state(rec + nid0);
            if (deg > 1) s1 = ld_state(rec + nid1);
            if (deg > 2) s2 = ld_state(rec + nid2);
            __syncwarp(gmask);  // every load of the round precedes every write

            int nwin = 0;
            bool meet = false;
#pragma unroll
            for (int s = 0; s < 3; s++) {
                const int n = (s == 0) ? nid0 : (s == 1) ? nid1 : nid2;
                const int2 st = (s == 0) ? s0 : (s == 1) ? s1 : s2;
                const float cx = (s == 0) ? nx0 : (s == 1) ? nx1 : nx2;
                const float cy = (s == 0) ? ny0 : (s == 1) ? ny1 : ny2;
                const bool valid = s < deg;
                bool prev = valid && (unsigned)st.x == ep;
                int pgd = st.y;
                if (valid && !prev) {  // claimed earlier in this round (earlier slot)
                    for (int w = 0; w < nwin; w++) {
                        if (wId[wb + w] == n) {
                            prev = true;
                            pgd = wGD[wb + w];
                            break;
                        }
                    }
                }
                const bool fresh = valid && !prev;
                const int key = fresh ? n : (-1 - lane);
                const unsigned mm = __match_any_sync(gmask, key);
                const int leader = __ffs(mm) - 1;
                const bool win = fresh && leader == lane;
                const int lgd = __shfl_sync(gmask, ngd, leader);
                int cgd = 0;
                bool conflict = false;
                if (fresh && !win) {
                    cgd = lgd;
                    conflict = (lgd & 1) != du;
                } else if (prev) {
                    cgd = pgd;
                    conflict = (pgd & 1) != du;
                }
                const unsigned cm = __ballot_sync(gmask, conflict) & gmask;
                if (!meet && cm != 0u) {  // group-uniform
                    const int ml = __ffs(cm) - 1;
                    const int mu = __shfl_sync(gmask, idu, ml);
                    const int mgu = __shfl_sync(gmask, gdu, ml);
                    const int mn = __shfl_sync(gmask, n, ml);
                    const int mgn = __shfl_sync(gmask, cgd, ml);
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
                    meet = true;
                }
                const unsigned wm = __ballot_sync(gmask, win) & gmask;
                if (win) {
                    const int idx = nwin + __popc(wm & ((1u << lane) - 1u));
                    const float hh = dist_sqr(cx, cy, farx, fary);
                    const float F = GM_FADD((float)Gn, GM_FMUL(hh, K));
                    wId[wb + idx] = n;
                    wGD[wb + idx] = ngd;
                    wF[wb + idx] = F;
                    st_rec(rec + n, ep, ngd, idu, ra.z, ra.w, rb.x, rb.y, rb.z);
                }
                nwin += __popc(wm);
                __syncwarp(gmask);
            }
            if (q == 0) claims += (unsigned)nwin;
            if (meet) {
                found = 1;
                break;
            }
            for (int i = q; i < nwin; i += T) heap_push(h, hsize, C, wF[wb + i], wGD[wb + i], wId[wb + i]);
            const bool any = __any_sync(gmask, hsize > 0);
            __syncwarp(gmask);  // winner list reads done before the next round
            if (!any) break;
        }

        // path reconstruction (PathFinder.h:276-306)
        int L = 0;
        if (found) {
            L = gS + gT + 1;
            const int row = (agent >= 0) ? agent : orow;
            if ((long long)L > p.path_stride) {
                if (q == 0) atomicOr(p.err, ERR_PATH_CAP);
            } else {
                int* out = p.paths + (long long)row * p.path_stride;
                if (q == 0) {
                    // start side: depths gS..1 at positions gS-1..0
                    int x = mS, g = gS;
                    if (g >= 1) out[g - 1] = x;
                    while (g > 1) {
                        if (x < 0 || x >= n_nodes) {
                            atomicOr(p.err, ERR_BOUNDS);
                            break;
                        }
                        int4 a, b;
                        ld_rec(rec + x, a, b);
                        const int anc[6] = {a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
                        for (int j = 0; j < 6; j++) {
                            const int d = g - 1 - j;
                            if (d >= 1) out[d - 1] = anc[j];
                        }
                        x = anc[5];
                        g -= 6;
                    }
                } else if (q == 1) {
                    // target side: depths gT..0 at positions gS..gS+gT
                    int x = mT, g = gT;
                    out[gS] = x;
                    while (g > 0) {
                        if (x < 0 || x >= n_nodes) {
                            atomicOr(p.err, ERR_BOUNDS);
                            break;
                        }
                        int4 a, b;
                        ld_rec(rec + x, a, b);
                        const int anc[6] = {a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
                        for (int j = 0; j < 6; j++) {
                            const int d = g - 1 - j;
                            if (d >= 0) out[gS + gT - d] = anc[j];
                        }
                        x = anc[5];
                        g -= 6;
                    }
                }
            }
        }
        __syncwarp(gmask);
        // results, agent update (PathFinder.h:268-289) and counters
        const unsigned ex = __reduce_add_sync(gmask, expansions);
        const unsigned ds = __reduce_add_sync(gmask, deg_sum);
        if (q == 0) {
            if (p.out_found) p.out_found[r] = found;
            if (p.out_len) p.out_len[r] = L;
            if (agent >= 0 && p.ag_state) {
                p.ag_state[agent] = found ? GMAPF_AGENT_MOVE : GMAPF_AGENT_IDLE;
                p.ag_step_idx[agent] = -1;
                p.ag_path_len[agent] = L;
            }
            atomicAdd(p.stats + ST_EXPANSIONS, (unsigned long long)ex);
            atomicAdd(p.stats + ST_DEG_SUM, (unsigned long long)ds);
            atomicAdd(p.stats + ST_ROUNDS, (unsigned long long)rounds);
            atomicAdd(p.stats + ST_CLAIMS, (unsigned long long)claims);
            atomicAdd(p.stats + ST_PATH_NODES, (unsigned long long)L);
            atomicAdd(p.stats + ST_FOUND, (unsigned long long)found);
        }
    }
}

template <int T>
cudaError_t launch_t(cudaStream_t s, const SearchParams& p, int blocks, int bt, bool persistent,
                     int req_base) {
    // the dynamic shared-memory limit was raised by search_max_blocks_per_sm
    // when the search state was sized (no attribute calls here: this may run
    // under stream capture)
    size_t smem = search_smem_bytes(T, p.C, bt);
    if (blocks <= 0) return cudaSuccess;
    k_search<T><<<blocks, bt, smem, s>>>(p, persistent ? 1 : 0, req_base);
    return cudaGetLastError();
}

}  // namespace

size_t search_smem_bytes(int T, int C, int bt) {
    (void)T;
    return (size_t)C * bt * 12 + (size_t)3 * bt * 12;
}

int search_max_blocks_per_sm(int T, int C, int bt) {
    int nb = 0;
    size_t smem = search_smem_bytes(T, C, bt);
    cudaError_t e = cudaSuccess;
    switch (T) {
        case 2:
            cudaFuncSetAttribute(k_search<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search<2>, bt, smem);
            break;
        case 4:
            cudaFuncSetAttribute(k_search<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search<4>, bt, smem);
            break;
        case 8:
            cudaFuncSetAttribute(k_search<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search<8>, bt, smem);
            break;
        case 16:
            cudaFuncSetAttribute(k_search<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search<16>, bt, smem);
            break;
        case 32:
            cudaFuncSetAttribute(k_search<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search<32>, bt, smem);
            break;
        default:
            return 0;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

cudaError_t launch_search(cudaStream_t s, const SearchParams& p, int blocks, int bt, bool persistent,
                          int req_base) {
    switch (p.T) {
        case 2: return launch_t<2>(s, p, blocks, bt, persistent, req_base);
        case 4: return launch_t<4>(s, p, blocks, bt, persistent, req_base);
        case 8: return launch_t<8>(s, p, blocks, bt, persistent, req_base);
        case 16: return launch_t<16>(s, p, blocks, bt, persistent, req_base);
        case 32: return launch_t<32>(s, p, blocks, bt, persistent, req_base);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace gmapf_b200
