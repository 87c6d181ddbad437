// noalloc.cu -- path searches that allocate no memory.
//
// For callers that must not allocate device memory at all: a game engine or
// host application that owns every GPU allocation through its own allocator
// or budget, code running where an allocation would stall or fail (memory
// already fully reserved, allocation forbidden while other work is captured
// or in flight), or a plug-in that may only touch buffers it is handed.
// They pass the navmesh, the queries and the output buffers in device memory
// and this entry point runs the same bidirectional bounded-queue search as
// the rest of the library (same order, same results), using as its only
// working memory one fixed array compiled into the library.
//
// That array (g_scratch, kScratchBytes) is a file-scope __device__ array:
// every GPU that loads the library holds it until the process exits.  It
// holds a small header (work counter, query counter) and the search records
// of the concurrent request slots (32 bytes per navmesh triangle per slot).
// Calls share it and it keeps the previous call's contents: the work counter
// is cleared by each call, and records are stamped with a 64-bit query
// number that never repeats (it would take centuries of queries to wrap), so
// a stale record is never mistaken for a live one, whatever the earlier
// calls' navmesh sizes were.  Two calls that overlap on the GPU (different
// streams, or different host threads) race on it and give wrong results:
// serialize them.
//
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current), clears it and sets the
// kernel's shared-memory limit for its (threads per agent, queue capacity);
// make that first call, and the first call with each new shape, before any
// stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <unordered_map>

#include "internal.h"

namespace gmapf_b200 {
namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB per device
constexpr size_t kHeaderBytes = 256;
constexpr int kMaxDevices = 64;

// header: 32-bit work counter at byte 0, 64-bit query counter at byte 8
constexpr size_t kWorkOff = 0, kQueryOff = 8;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct DeviceSetup {
    bool ready = false;
    unsigned char* scratch = nullptr;  // device address of g_scratch
    int sms = 0;
    std::unordered_map<int, int> blocks_per_sm;  // (T, C) -> resident one-warp blocks per SM
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

constexpr unsigned kFull = 0xffffffffu;
// queue / frontier entry: F, G<<1|dir, id, ancestors 1..4
constexpr int kEntry = 7;

// Search record of this kernel: the 64-bit stamp of the query that claimed
// the node, G<<1|dir and ancestors 1..5 (anc[0] is the parent).  32 bytes,
// read and written as one sector like the library's other records.
struct __align__(32) NRec {
    unsigned lo, hi;
    int gd;
    int anc[5];
};
static_assert(sizeof(NRec) == 32, "one sector per record");

__device__ __forceinline__ int4 ld_head(const NRec* r) {  // {stamp lo, stamp hi, gd, parent}
    return __ldcg(reinterpret_cast<const int4*>(r));
}
__device__ __forceinline__ void ld_nrec(const NRec* r, int4& a, int4& b) {
    asm volatile("ld.global.cg.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
                 : "l"(r));
}
__device__ __forceinline__ void st_nrec(NRec* r, unsigned long long stamp, int gd, int a0, int a1, int a2, int a3,
                                        int a4) {
    asm volatile("st.global.cg.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(r), "r"((unsigned)stamp),
                 "r"((unsigned)(stamp >> 32)), "r"(gd), "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(a4)
                 : "memory");
}

__device__ __forceinline__ bool less3(float fa, int ga, int ia, float fb, int gb, int ib) {
    if (fa != fb) return fa < fb;
    if ((ga >> 1) != (gb >> 1)) return (ga >> 1) < (gb >> 1);
    return ia < ib;
}

// centroid of a navmesh node: ((P1 + P2) + P3) / 3, src/GMAPF.cu:215
__device__ __forceinline__ float2 node_centroid(const gmapf_node* nodes, int i) {
    const gmapf_node& nd = nodes[i];
    const float sx = __fadd_rn(__fadd_rn(nd.P1.X, nd.P2.X), nd.P3.X);
    const float sy = __fadd_rn(__fadd_rn(nd.P1.Y, nd.P2.Y), nd.P3.Y);
    return make_float2(__fdiv_rn(sx, 3.0f), __fdiv_rn(sy, 3.0f));
}

struct NoAllocArgs {
    const gmapf_node* nodes;
    int n;
    const int* starts;
    const int* targets;
    int nq;
    int T, C;
    float K;
    int max_rounds;
    int* found;
    int* lens;
    int* paths;
    long long stride;
    unsigned char* scratch;  // device address of g_scratch
    int slots;
};

// One warp per request; the same rounds, claim order and queue rules as the
// main search kernel (include/gmapf/PathFinder.h:138-251 with the (F, G, id)
// order), with the visited state in stamped scratch records.
template <int T>
__global__ void __launch_bounds__(32) k_search_noalloc(NoAllocArgs a) {
    constexpr int NP = (3 * T + 31) / 32;
    extern __shared__ __align__(16) int sm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int slot = blockIdx.x * wpb + wib;
    if (slot >= a.slots) return;
    const int C = a.C, n_nodes = a.n;
    const int qwords = kEntry * C * T;
    int* q = sm + wib * (qwords + kEntry * 3 * T);  // ring: word w of entry k of lane l at [(w*C+k)*T+l]
    int* fr = q + qwords;                           // frontier: word w of item i at [w*3T+i]
    unsigned* work = reinterpret_cast<unsigned*>(a.scratch + kWorkOff);
    unsigned long long* qctr = reinterpret_cast<unsigned long long*>(a.scratch + kQueryOff);
    NRec* rec = reinterpret_cast<NRec*>(a.scratch + kHeaderBytes) + (size_t)slot * n_nodes;
    const unsigned lt = (1u << lane) - 1u;

    auto at = [&](int k) { return (k >= C ? k - C : k) * T + (lane < T ? lane : 0); };
    auto key_at = [&](int k, float& f, int& gd, int& id) {
        f = __int_as_float(q[k]);
        gd = q[C * T + k];
        id = q[2 * C * T + k];
    };

    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(work, 1);
        r = __shfl_sync(kFull, r, 0);
        if (r >= a.nq) break;
        const int start = a.starts[r], target = a.targets[r];
        if (start < 0 || start >= n_nodes || target < 0 || target >= n_nodes || start == target) {
            if (lane == 0) {  // bad query: found = -1; start == target: found, empty path
                a.found[r] = (start == target && start >= 0 && start < n_nodes) ? 1 : -1;
                a.lens[r] = 0;
            }
            continue;
        }
        unsigned long long ep = 0;
        if (lane == 0) ep = atomicAdd(qctr, 1ull) + 1ull;  // never repeats: stale records never match
        ep = __shfl_sync(kFull, ep, 0);
        const unsigned ep_lo = (unsigned)ep, ep_hi = (unsigned)(ep >> 32);
        const float2 cs = node_centroid(a.nodes, start), ct = node_centroid(a.nodes, target);
        const float f0 = __fmul_rn(dist_sqr(cs.x, cs.y, ct.x, ct.y), a.K);
        int beg = 0, size = 0;
        if (lane < 2) {  // PathFinder.h:168-189: lane 0 seeds the start, lane 1 the target
            const int node = lane == 0 ? start : target;
            const int k = at(0);
            q[k] = __float_as_int(f0);
            q[C * T + k] = lane == 0 ? 1 : 0;
            q[2 * C * T + k] = node;
            for (int j = 0; j < 4; j++) q[(3 + j) * C * T + k] = -1;
            size = 1;
            st_nrec(rec + node, ep, lane == 0 ? 1 : 0, -1, -1, -1, -1, -1);
        }
        __syncwarp();
        int found = 0, mS = 0, gS = 0, mT = 0, gT = 0, rounds = 0;
        bool capped = false;
        for (;;) {
            rounds++;
            int idu = -1, gdu = 0, uk = 0;
            if (lane < T && size > 0) {
                uk = at(beg + size - 1);
                gdu = q[C * T + uk];
                idu = q[2 * C * T + uk];
                size--;
            }
            int nwin = 0;
            bool meet = false;
            int mu = 0, mgu = 0, mn = 0, mgn = 0;
#pragma unroll
            for (int pass = 0; pass < NP; pass++) {
                const int c = pass * 32 + lane, s = c / T, qq = c - s * T;
                const int cu = __shfl_sync(kFull, idu, qq & 31);
                const int cgdu = __shfl_sync(kFull, gdu, qq & 31);
                const int cuk = __shfl_sync(kFull, uk, qq & 31);
                bool valid = c < 3 * T && cu >= 0;
                int n = -1;
                if (valid) {
                    int deg = 0;
                    while (deg < 3 && a.nodes[cu].NeibsIdx[deg] != -1) deg++;
                    valid = s < deg;
                    if (valid) n = a.nodes[cu].NeibsIdx[s];
                    valid = valid && n >= 0 && n < n_nodes;  // caller-provided ids: never index out of range
                }
                const int du = cgdu & 1, ngd = (((cgdu >> 1) + 1) << 1) | du;
                bool prev = false;
                int pgd = 0;
                if (valid) {
                    const int4 h = ld_head(rec + n);
                    prev = (unsigned)h.x == ep_lo && (unsigned)h.y == ep_hi;
                    pgd = h.z;
                }
                const bool fresh = valid && !prev;
                const unsigned mm = __match_any_sync(kFull, fresh ? n : (-1 - lane));
                const int leader = __ffs(mm) - 1;
                const bool win = fresh && leader == lane;
                const int lgd = __shfl_sync(kFull, ngd, leader);
                bool conflict = false;
                int cgd = 0;
                if (fresh && !win) {
                    cgd = lgd;
                    conflict = (lgd & 1) != du;
                } else if (prev) {
                    cgd = pgd;
                    conflict = (pgd & 1) != du;
                }
                const unsigned cm = __ballot_sync(kFull, conflict);
                if (!meet && cm != 0u) {
                    const int ml = __ffs(cm) - 1;
                    mu = __shfl_sync(kFull, cu, ml);
                    mgu = __shfl_sync(kFull, cgdu, ml);
                    mn = __shfl_sync(kFull, n, ml);
                    mgn = __shfl_sync(kFull, cgd, ml);
                    meet = true;
                }
                const unsigned wm = __ballot_sync(kFull, win);
                if (win) {
                    const int idx = nwin + __popc(wm & lt);
                    const float2 cn = node_centroid(a.nodes, n);
                    const float2 far = du ? ct : cs;
                    const float F = __fadd_rn((float)(ngd >> 1), __fmul_rn(dist_sqr(cn.x, cn.y, far.x, far.y), a.K));
                    int ua[4];
                    for (int j = 0; j < 4; j++) ua[j] = q[(3 + j) * C * T + cuk];
                    fr[idx] = __float_as_int(F);
                    fr[3 * T + idx] = ngd;
                    fr[6 * T + idx] = n;
                    fr[9 * T + idx] = cu;
                    for (int j = 0; j < 3; j++) fr[(4 + j) * 3 * T + idx] = ua[j];
                    st_nrec(rec + n, ep, ngd, cu, ua[0], ua[1], ua[2], ua[3]);
                }
                nwin += __popc(wm);
                __syncwarp();
            }
            bool ended = false;
            if (meet) {
                if (mgu & 1) {
                    mS = mu; gS = mgu >> 1; mT = mn; gT = mgn >> 1;
                } else {
                    mS = mn; gS = mgn >> 1; mT = mu; gT = mgu >> 1;
                }
                found = 1;
                ended = true;
            } else {
                if (lane < T) {
                    for (int i = lane; i < nwin; i += T) {
                        int e[kEntry];
                        for (int w = 0; w < kEntry; w++) e[w] = fr[w * 3 * T + i];
                        const float ef = __int_as_float(e[0]);
                        bool keep = true;
                        if (size == C) {  // bounded: evict the maximum or drop
                            float mf;
                            int mg, mi;
                            key_at(at(beg), mf, mg, mi);
                            if (!less3(ef, e[1], e[2], mf, mg, mi)) keep = false;
                            else {
                                beg = (beg + 1 == C) ? 0 : beg + 1;
                                size--;
                            }
                        }
                        if (keep) {
                            int j = size - 1;
                            while (j >= 0) {
                                float kf;
                                int kg, ki;
                                const int k = at(beg + j);
                                key_at(k, kf, kg, ki);
                                if (!less3(kf, kg, ki, ef, e[1], e[2])) break;
                                const int k1 = at(beg + j + 1);
                                for (int w = 0; w < kEntry; w++) q[w * C * T + k1] = q[w * C * T + k];
                                j--;
                            }
                            const int k1 = at(beg + j + 1);
                            for (int w = 0; w < kEntry; w++) q[w * C * T + k1] = e[w];
                            size++;
                        }
                    }
                }
                if (!__any_sync(kFull, size > 0)) ended = true;
                if (!ended && rounds >= a.max_rounds) {  // the round limit: reported as found = -2
                    ended = true;
                    capped = true;
                }
            }
            __syncwarp();
            if (ended) break;
        }
        int L = 0;
        if (found) {
            L = gS + gT + 1;
            if ((long long)L <= a.stride && lane < 2) {
                // lane 0: start side, depths gS..1 at positions gS-1..0;
                // lane 1: target side, depths gT..0 at positions gS..gS+gT;
                // each record read gives five more ancestors
                int* out = a.paths + (long long)r * a.stride;
                int x = lane == 0 ? mS : mT, g = lane == 0 ? gS : gT;
                const int stop = lane == 0 ? 1 : 0;
                if (lane == 0) {
                    if (g >= 1) out[g - 1] = x;
                } else {
                    out[gS] = x;
                }
                while (g > stop && x >= 0 && x < n_nodes) {
                    int4 p0, p1;
                    ld_nrec(rec + x, p0, p1);
                    const int anc[5] = {p0.w, p1.x, p1.y, p1.z, p1.w};
                    for (int j = 0; j < 5; j++) {
                        const int d = g - 1 - j;
                        if (d >= stop) {
                            if (lane == 0) out[d - 1] = anc[j];
                            else out[gS + gT - d] = anc[j];
                        }
                    }
                    x = anc[4];
                    g -= 5;
                }
            }
        }
        __syncwarp();
        if (lane == 0) {
            a.found[r] = capped ? -2 : found;
            a.lens[r] = L;  // a length above path_stride means the row was left unwritten
        }
    }
}

size_t smem_per_warp(int T, int C) { return (size_t)4 * kEntry * T * (C + 3); }

template <int T>
cudaError_t run_t(const NoAllocArgs& a, int blocks, cudaStream_t s) {
    k_search_noalloc<T><<<blocks, 32, smem_per_warp(T, a.C), s>>>(a);
    return cudaGetLastError();
}

template <int T>
int occupancy(int C) {
    const size_t smem = smem_per_warp(T, C);
    if (smem > 227 * 1024) return 0;
    if (cudaFuncSetAttribute(k_search_noalloc<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_search_noalloc<T>, 32, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

int occupancy_any(int T, int C) {
    switch (T) {
        case 2: return occupancy<2>(C);
        case 4: return occupancy<4>(C);
        case 8: return occupancy<8>(C);
        case 16: return occupancy<16>(C);
        case 32: return occupancy<32>(C);
        default: return 0;
    }
}

gmapf_status fail(gmapf_status s, const char* what) {
    set_last_error(what);  // read with gmapf_last_error()
    return s;
}

}  // namespace
}  // namespace gmapf_b200

using namespace gmapf_b200;

extern "C" gmapf_status gmapf_search_batch_noalloc(const gmapf_node* d_nodes, int32_t n_nodes,
                                                   const int32_t* d_starts, const int32_t* d_targets,
                                                   int32_t n_queries, int32_t threads_per_agent,
                                                   int32_t queue_capacity, float heuristic_k,
                                                   int32_t round_limit, int32_t* d_found, int32_t* d_lens,
                                                   int32_t* d_paths, int32_t path_stride, void* stream) {
    const int T = threads_per_agent, C = queue_capacity;
    if (!(T == 2 || T == 4 || T == 8 || T == 16 || T == 32))
        return fail(GMAPF_E_INVALID_ARG, "threads_per_agent must be one of 2, 4, 8, 16, 32");
    if (C < 1 || C > 512) return fail(GMAPF_E_INVALID_ARG, "queue_capacity must be in [1, 512]");
    if (n_nodes < 1 || n_queries < 0 || path_stride < 1 || round_limit < 0)
        return fail(GMAPF_E_INVALID_ARG, "need n_nodes >= 1, n_queries >= 0, path_stride >= 1, round_limit >= 0");
    if ((size_t)n_nodes * sizeof(NRec) > kScratchBytes - kHeaderBytes)
        return fail(GMAPF_E_CAPACITY,
                    "navmesh too large for the built-in 64 MiB scratch (at most 2,097,144 triangles)");
    if (n_queries > 0 && (!d_nodes || !d_starts || !d_targets || !d_found || !d_lens || !d_paths))
        return fail(GMAPF_E_INVALID_ARG, "null device pointer");
    if (n_queries == 0) return GMAPF_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return fail(GMAPF_E_CUDA, "no usable current CUDA device");
    }
    // a kernel given pageable host memory or another GPU's memory would
    // fault: refuse it here (the check allocates nothing)
    const void* bufs[6] = {d_nodes, d_starts, d_targets, d_found, d_lens, d_paths};
    for (const void* b : bufs)
        if (!gpu_reachable(b, dev))
            return fail(GMAPF_E_INVALID_ARG,
                        "a buffer is not memory the current GPU can reach (its device memory, managed or mapped "
                        "pinned)");
    DeviceSetup* ds = &g_setup[dev];
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!ds->ready) {  // once per device, with that device current
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
            if (e != cudaSuccess || !ptr) {
                cudaGetLastError();
                return fail(GMAPF_E_CUDA, "cudaGetSymbolAddress of the scratch array failed");
            }
            if (cudaDeviceGetAttribute(&ds->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
                cudaGetLastError();
                return fail(GMAPF_E_CUDA, "cudaDeviceGetAttribute failed");
            }
            // records start unclaimed: zero them once (query stamps start at 1)
            if (cudaMemsetAsync(ptr, 0, kScratchBytes, s) != cudaSuccess) {
                cudaGetLastError();
                return fail(GMAPF_E_CUDA, "clearing the scratch array failed");
            }
            ds->scratch = static_cast<unsigned char*>(ptr);
            ds->ready = true;
        }
        // the kernel attribute and occupancy query run once per (T, C) on
        // this device; later calls make no CUDA calls besides the launch
        const int key = T * 1024 + C;
        auto it = ds->blocks_per_sm.find(key);
        if (it == ds->blocks_per_sm.end()) it = ds->blocks_per_sm.emplace(key, occupancy_any(T, C)).first;
        per_sm = it->second;
    }
    if (per_sm <= 0) return fail(GMAPF_E_CAPACITY, "queues do not fit in shared memory for this T and C");
    const long long by_mem = (long long)((kScratchBytes - kHeaderBytes) / ((size_t)n_nodes * sizeof(NRec)));
    long long slots = (long long)ds->sms * per_sm;  // one warp (one request slot) per block
    slots = std::min(slots, by_mem);
    slots = std::min(slots, (long long)n_queries);
    if (slots < 1) slots = 1;
    const int blocks = (int)slots;

    // the work counter must start at zero for every call
    if (cudaMemsetAsync(ds->scratch + kWorkOff, 0, sizeof(unsigned), s) != cudaSuccess) {
        cudaGetLastError();
        return fail(GMAPF_E_CUDA, "clearing the work counter failed");
    }
    NoAllocArgs a;
    a.nodes = d_nodes;
    a.n = n_nodes;
    a.starts = d_starts;
    a.targets = d_targets;
    a.nq = n_queries;
    a.T = T;
    a.C = C;
    a.K = heuristic_k;
    // the default limit, 4 n + 64 rounds, is never reached: every round pops
    // a queued node, and a node is queued at most once (when it is claimed)
    a.max_rounds = round_limit > 0 ? round_limit : (int)std::min<long long>(4ll * n_nodes + 64, 0x7fffffff);
    a.found = d_found;
    a.lens = d_lens;
    a.paths = d_paths;
    a.stride = path_stride;
    a.scratch = ds->scratch;
    a.slots = (int)slots;
    cudaError_t e;
    switch (T) {
        case 2: e = run_t<2>(a, blocks, s); break;
        case 4: e = run_t<4>(a, blocks, s); break;
        case 8: e = run_t<8>(a, blocks, s); break;
        case 16: e = run_t<16>(a, blocks, s); break;
        default: e = run_t<32>(a, blocks, s); break;
    }
    if (e != cudaSuccess) return fail(GMAPF_E_CUDA, cudaGetErrorString(e));
    return GMAPF_OK;
}
