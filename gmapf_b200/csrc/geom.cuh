// geom.cuh -- navmesh geometry shared by host and device code.
//
// Every floating-point expression is spelled with explicit round-to-nearest
// operations on the device (__fmul_rn/__fadd_rn/... are never contracted into
// FMA) and compiled with -ffp-contract=off on the host, so host and device
// give bit-identical answers and both match the reference's IEEE binary32
// formulas:
//   GetSign / IsPointInTriangle    include/gmapf/misc/CuNodesMap.h:97-112
//   GetDistSqr (V2Float::DistSqr)  include/gmapf/misc/CuNodesMap.h:74-80, V2Float.h:50-55
//   TryGetNodeIdx (first match)    include/gmapf/misc/CuNodesMap.h:53-66
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#if defined(__CUDA_ARCH__)
#define GM_FMUL(a, b) __fmul_rn((a), (b))
#define GM_FADD(a, b) __fadd_rn((a), (b))
#define GM_FSUB(a, b) __fsub_rn((a), (b))
#define GM_FDIV(a, b) __fdiv_rn((a), (b))
#define GM_FSQRT(a) __fsqrt_rn((a))
#else
#define GM_FMUL(a, b) ((float)(a) * (float)(b))
#define GM_FADD(a, b) ((float)(a) + (float)(b))
#define GM_FSUB(a, b) ((float)(a) - (float)(b))
#define GM_FDIV(a, b) ((float)(a) / (float)(b))
#define GM_FSQRT(a) sqrtf((float)(a))
#endif

namespace gmapf_b200 {

constexpr int kInvalid = -1;

// Per-node search row: the node's neighbours (packed, -1 padded) with the
// count of leading valid ones and each neighbour's centroid.  48 bytes,
// 16-byte aligned: expanding a node reads one row.
struct __align__(16) SearchRow {
    int n0, n1, n2, deg;
    float x0, y0, x1, y1;
    float x2, y2;
    int pad0, pad1;
};
static_assert(sizeof(SearchRow) == 48, "search row layout");

// Point-location grid: every non-degenerate triangle is listed, in ascending
// id, in each cell its padded bounding box touches; degenerate triangles
// (zero signed area) are checked for every query.  With the lists ascending,
// the first containing triangle is the one the reference's linear scan finds.
struct LocateGrid {
    float x0, y0, inv;
    int w, h;
    const int* start;   // w*h+1
    const int* list;    // triangle ids local to this map
    const int* degen;
    int ndegen;
    const float2* tri;  // 3 vertices per triangle of this map
    int n;
    int base;           // added to a found id (first global id of this map in a scene batch)
};

__host__ __device__ inline float get_sign(float p1x, float p1y, float p2x, float p2y, float p3x,
                                          float p3y) {
    float a = GM_FMUL(GM_FSUB(p1x, p3x), GM_FSUB(p2y, p3y));
    float b = GM_FMUL(GM_FSUB(p2x, p3x), GM_FSUB(p1y, p3y));
    return GM_FSUB(a, b);
}

__host__ __device__ inline bool point_in_tri(float px, float py, float2 v1, float2 v2, float2 v3) {
    float d1 = get_sign(px, py, v1.x, v1.y, v2.x, v2.y);
    float d2 = get_sign(px, py, v2.x, v2.y, v3.x, v3.y);
    float d3 = get_sign(px, py, v3.x, v3.y, v1.x, v1.y);
    bool isNeg = (d1 < 0) || (d2 < 0) || (d3 < 0);
    bool isPos = (d1 > 0) || (d2 > 0) || (d3 > 0);
    return !(isNeg && isPos);
}

__host__ __device__ inline float dist_sqr(float ax, float ay, float bx, float by) {
    float x = GM_FSUB(ax, bx);
    float y = GM_FSUB(ay, by);
    return GM_FADD(GM_FMUL(x, x), GM_FMUL(y, y));
}

// Cell coordinate along one axis, clamped to [0, cells-1].  Monotonic in x,
// which is what makes the padded-bounding-box listing complete.
__host__ __device__ inline int grid_cell(float x, float x0, float inv, int cells) {
    float f = floorf(GM_FMUL(GM_FSUB(x, x0), inv));
    f = fminf(fmaxf(f, 0.0f), (float)(cells - 1));
    return (int)f;
}

__host__ __device__ inline bool gm_isfinite(float x) { return x - x == 0.0f; }

__host__ __device__ inline int locate_linear(const LocateGrid& g, float px, float py) {
    for (int i = 0; i < g.n; i++)
        if (point_in_tri(px, py, g.tri[3 * i], g.tri[3 * i + 1], g.tri[3 * i + 2])) return i + g.base;
    return -1;
}

__host__ __device__ inline int locate(const LocateGrid& g, float px, float py) {
    if (!gm_isfinite(px) || !gm_isfinite(py)) return locate_linear(g, px, py);
    int cx = grid_cell(px, g.x0, g.inv, g.w);
    int cy = grid_cell(py, g.y0, g.inv, g.h);
    int c = cy * g.w + cx;
    int best = -1;
    for (int k = g.start[c], e = g.start[c + 1]; k < e; k++) {
        int i = g.list[k];
        if (point_in_tri(px, py, g.tri[3 * i], g.tri[3 * i + 1], g.tri[3 * i + 2])) {
            best = i;
            break;
        }
    }
    for (int k = 0; k < g.ndegen; k++) {
        int i = g.degen[k];
        if (best >= 0 && i > best) break;
        if (point_in_tri(px, py, g.tri[3 * i], g.tri[3 * i + 1], g.tri[3 * i + 2])) {
            best = i;
            break;
        }
    }
    return best >= 0 ? best + g.base : -1;
}

}  // namespace gmapf_b200
