// Host check of region_plan (visited placement 4): for every block size up to
// 8 warps, several share, pad and bitmap sizes, every mask of warps that have
// left and every warp still running, a plan must keep the bitmap inside the
// block's shared memory, cover only free shares (or the warp's own), and put
// the warp's queues in its own share or in a free share outside the bitmap;
// a warp whose block-mates have all left must always get a plan, and the
// round loop's count of free shares must never turn away a plan.  Built with
// nvcc as host code and run by tests/test_region_plan.py.
#include <cstdio>

#include "region_plan.cuh"

using gmapf_b200::region_plan;
using gmapf_b200::region_shares_needed;
using gmapf_b200::search_pad_words;

int main() {
    long long cases = 0, plans = 0;
    const int shares[] = {64, 1000, 2016, 3000};
    for (int wpb = 1; wpb <= 8; wpb++)
        for (int share : shares) {
            const int bms[] = {16, 1020, 4000, 6360, 2016 * wpb, 25000};
            for (int bm : bms) {
                const int pad = (int)search_pad_words(bm, wpb, share);
                const long long total = (long long)wpb * share + pad;
                for (unsigned left = 0; left < (1u << wpb); left++)
                    for (int me = 0; me < wpb; me++) {
                        if ((left >> me) & 1u) continue;  // a running warp has not left
                        cases++;
                        const int r = region_plan(left, me, wpb, share, bm, pad);
                        const bool alone = (left | (1u << me)) == (1u << wpb) - 1u;
                        if (r < 0) {
                            if (alone) {
                                std::printf("FAIL alone without a plan: wpb=%d share=%d bm=%d me=%d\n", wpb, share,
                                            bm, me);
                                return 1;
                            }
                            continue;
                        }
                        plans++;
                        // the round loop's cheap count must let every plan through
                        if (__builtin_popcount(left | (1u << me)) < region_shares_needed(bm, wpb, share)) {
                            std::printf("FAIL count vetoes a plan: wpb=%d share=%d bm=%d left=%x me=%d\n", wpb,
                                        share, bm, left, me);
                            return 1;
                        }
                        const int first = r & 0xff, home = r >> 8;
                        const long long start = (long long)first * share, end = start + bm;
                        bool ok = first >= 0 && first <= wpb && home >= 0 && home < wpb && end <= total;
                        bool home_in_run = false;
                        for (int w = 0; w < wpb && ok; w++) {
                            const bool touched = (long long)w * share < end && (long long)(w + 1) * share > start;
                            if (touched && w != me && !((left >> w) & 1u)) ok = false;  // a running warp's share
                            if (touched && w == home) home_in_run = true;
                        }
                        if (home != me && !((left >> home) & 1u)) ok = false;
                        if (home_in_run) ok = false;
                        if (!ok) {
                            std::printf("FAIL wpb=%d share=%d bm=%d left=%x me=%d plan=%d\n", wpb, share, bm, left,
                                        me, r);
                            return 1;
                        }
                    }
            }
        }
    std::printf("ok %lld cases, %lld plans\n", cases, plans);
    return 0;
}
