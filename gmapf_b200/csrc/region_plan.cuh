// region_plan.cuh -- where a search moves its visited bitmap in its block's
// shared memory (visited placement 4).  Host and device code: the kernel calls
// it, and a host program checks it over every case (tests/cpp/region_plan_check.cu).
#pragma once

#include <cstddef>

namespace gmapf_b200 {

// Words after the last warp's share so that all but one share and the pad
// hold one bitmap of bm_words words (a multiple of 4 words).
__host__ __device__ __forceinline__ size_t search_pad_words(int bm_words, int warps, int per_warp) {
    const long long rest = (long long)bm_words - (long long)(warps - 1) * per_warp;
    return rest > 0 ? (size_t)((rest + 3) & ~3ll) : 0;
}

// The fewest shares (with the pad after the last) that hold the bitmap: a
// search checks this cheap count in its round loop and works out a plan only
// when at least that many shares are free; no plan needs fewer.
__host__ __device__ __forceinline__ int region_shares_needed(int bm_words, int wpb, int share) {
    const int rest = bm_words - (int)search_pad_words(bm_words, wpb, share);
    return rest > 0 ? (rest + share - 1) / share : 0;
}

__host__ __device__ __forceinline__ int lowest_set_bit(unsigned x) {  // 1-based, 0 for none
#ifdef __CUDA_ARCH__
    return __ffs(x);
#else
    return __builtin_ffs((int)x);
#endif
}

// Where a search of warp `me` can put its bitmap (bm words) in its block's
// shared memory, given the warps that have left (`left`, whose shares are
// free for good).  Shares are `share` words each, `pad` words follow the last
// one.  The bitmap takes a run of free shares (this warp's own share may be
// in it), the last run of the block also using the pad; when this warp's
// share is in the run, its queues move to a free share outside it.  Returns
// first | home << 8 (the bitmap starts at share `first`, the queues live in
// share `home`), or -1 when there is no room.
static __host__ __device__ __noinline__ int region_plan(unsigned left, int me, int wpb, int share, int bm,
                                                        int pad) {
    if (pad >= bm) return wpb | (me << 8);  // the pad alone (one-warp blocks)
    const unsigned usable = left | (1u << me);
    for (int first = wpb - 1; first >= 0; first--) {
        // the run [first, last] with the smallest last that holds the bitmap
        long long room = 0;
        int last = first;
        for (; last < wpb; last++) {
            if (!((usable >> last) & 1u)) break;
            room += share + (last == wpb - 1 ? pad : 0);
            if (room >= bm) break;
        }
        if (last >= wpb || room < bm || !((usable >> last) & 1u)) continue;
        const unsigned run = (last - first >= 31 ? 0xffffffffu : ((2u << (last - first)) - 1u)) << first;
        if (!((run >> me) & 1u)) return first | (me << 8);
        const unsigned outside = left & ~run;  // another free share for this warp's queues
        if (outside) return first | ((lowest_set_bit(outside) - 1) << 8);
    }
    return -1;
}

}  // namespace gmapf_b200
