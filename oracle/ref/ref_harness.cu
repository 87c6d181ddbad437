// ref_harness.cu -- runs the reference's own __host__ __device__ container
// and geometry code on the CPU, to pin the oracle (test infrastructure only).
//
// Compiled by oracle/ref/build_ref.sh against the reference headers where
// they lie (include/gmapf/misc/CuQueue.h, CuNodesMap.h, V2Float.h); output
// goes to oracle/_ref/ only.  Reads a small text protocol on stdin:
//   Q <cap> <nops>   then nops lines "u <F> <id>" (push) or "o" (pop)
//                    -> popped ids, then the final contents in pop order
//   M <n>            then n lines "x1 y1 x2 y2 x3 y3 nb0 nb1 nb2": load a map
//   C                -> centroids ((P1+P2+P3)/3.0f, src/GMAPF.cu:215) as hex bits
//   P <k>            then k lines "x y": CuNodesMap::TryGetNodeIdx
//   I <k>            then k lines "x y node": CuNodesMap::IsInNode
//   D <k>            then k lines "a b": CuNodesMap::GetDistSqr as hex bits
//   R <k>            then k lines "x y": V2Float::GetRotated(10) as hex bits
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gmapf/misc/V2Float.h"
#include "gmapf/misc/CuNodesMap.h"
#include "gmapf/misc/CuQueue.h"

using namespace gmapf;

struct Item {
    int NodeIdx;
    float F;
    int G;
};

static unsigned bits(float f) {
    unsigned u;
    std::memcpy(&u, &f, 4);
    return u;
}

int main() {
    char cmd[8];
    std::vector<char> mapBlob;
    int mapN = 0;
    while (std::scanf("%7s", cmd) == 1) {
        if (cmd[0] == 'Q') {
            int cap, nops;
            std::scanf("%d %d", &cap, &nops);
            std::vector<char> blob(CuQueue<Item>::EvalSize(cap));
            CuQueue<Item> q(blob.data());
            q.Mark(cap);
            std::printf("Q");
            for (int k = 0; k < nops; k++) {
                char op[4];
                std::scanf("%3s", op);
                if (op[0] == 'u') {
                    Item it;
                    std::scanf("%f %d", &it.F, &it.NodeIdx);
                    it.G = 0;
                    q.Push(it);
                } else {
                    if (q.Count() == 0)
                        std::printf(" -1");
                    else
                        std::printf(" %d", q.Pop().NodeIdx);
                }
            }
            std::printf(" |");
            while (q.Count() > 0) std::printf(" %d", q.Pop().NodeIdx);
            std::printf("\n");
        } else if (cmd[0] == 'M') {
            std::scanf("%d", &mapN);
            mapBlob.assign(CuNodesMap::EvalSize(mapN), 0);
            CuNodesMap m(mapBlob.data());
            m.Mark(mapN);
            for (int i = 0; i < mapN; i++) {
                CuNodesMap::Node& nd = m.At(i);
                std::scanf("%f %f %f %f %f %f %d %d %d", &nd.P1.X, &nd.P1.Y, &nd.P2.X, &nd.P2.Y, &nd.P3.X,
                           &nd.P3.Y, &nd.NeibsIdx[0], &nd.NeibsIdx[1], &nd.NeibsIdx[2]);
                nd.PCenter = (nd.P1 + nd.P2 + nd.P3) / 3.0f;
            }
        } else if (cmd[0] == 'C') {
            CuNodesMap m(mapBlob.data());
            std::printf("C");
            for (int i = 0; i < mapN; i++) {
                V2Float c = m.GetPos(i);
                std::printf(" %08x %08x", bits(c.X), bits(c.Y));
            }
            std::printf("\n");
        } else if (cmd[0] == 'P') {
            CuNodesMap m(mapBlob.data());
            int k;
            std::scanf("%d", &k);
            std::printf("P");
            for (int i = 0; i < k; i++) {
                V2Float p;
                std::scanf("%f %f", &p.X, &p.Y);
                int idx = -1;
                if (!m.TryGetNodeIdx(p, &idx)) idx = -1;
                std::printf(" %d", idx);
            }
            std::printf("\n");
        } else if (cmd[0] == 'I') {
            CuNodesMap m(mapBlob.data());
            int k;
            std::scanf("%d", &k);
            std::printf("I");
            for (int i = 0; i < k; i++) {
                V2Float p;
                int node;
                std::scanf("%f %f %d", &p.X, &p.Y, &node);
                std::printf(" %d", m.IsInNode(p, node) ? 1 : 0);
            }
            std::printf("\n");
        } else if (cmd[0] == 'D') {
            CuNodesMap m(mapBlob.data());
            int k;
            std::scanf("%d", &k);
            std::printf("D");
            for (int i = 0; i < k; i++) {
                int a, b;
                std::scanf("%d %d", &a, &b);
                std::printf(" %08x", bits(m.GetDistSqr(a, b)));
            }
            std::printf("\n");
        } else if (cmd[0] == 'R') {
            int k;
            std::scanf("%d", &k);
            std::printf("R");
            for (int i = 0; i < k; i++) {
                V2Float v;
                std::scanf("%f %f", &v.X, &v.Y);
                V2Float r = v.GetRotated(10);
                std::printf(" %08x %08x", bits(r.X), bits(r.Y));
            }
            std::printf("\n");
        }
    }
    return 0;
}
