/*
 * gmapf_oracle.cpp -- CPU oracle for the G-MAPF per-frame step.
 *
 * TEST INFRASTRUCTURE ONLY (see gmapf_oracle.h).  Build with
 * -ffp-contract=off so that every a*b+c stays two IEEE roundings, exactly as
 * the CUDA kernels spell it with __fmul_rn/__fadd_rn.
 *
 * Determinism rules this file fixes (the reference leaves them to atomics):
 *   - queue order: ascending (F, G, node id); pop takes the minimum; a push
 *     into a full queue evicts the maximum or drops the new item when it is
 *     not smaller than the maximum (CuQueue.h:33-63 with F ties broken by G
 *     then id instead of FIFO);
 *   - candidates of one round are taken slot-major: neighbour slot 0 of lanes
 *     0..T-1, then slot 1, then slot 2 (the lock-step order of one warp
 *     executing PathFinder.h:198-231); the first candidate of a node claims it
 *     (CuVisitedMap.h:45-54) and its frontier position is its rank among the
 *     round's claims;
 *   - the first conflicting candidate in that order is the meeting pair
 *     (PathFinder.h:219-229);
 *   - frontier item i goes to lane i mod T (PathFinder.h:236-240);
 *   - requests are taken in ascending agent id up to the capacity
 *     (PathFinder.h:85-116); collisions use positions after the move for all
 *     reads (Jacobi) and sum contributions in ascending agent id
 *     (AgentsMover.h:96-113).
 */
#include "gmapf_oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <queue>
#include <thread>
#include <vector>

namespace {

/* ------------------------------------------------------------------ map --- */

struct Map {
    int n = 0;
    std::vector<float> t;   /* 6 per node */
    std::vector<float> cx, cy;
    std::vector<int> nb;    /* 3 per node */
    std::vector<int> deg;   /* leading valid neighbours (search stops at first -1) */
    /* point-location grid: triangles listed in ascending id in every cell their
     * (padded) bounding box touches; degenerate triangles checked everywhere */
    float gx0 = 0, gy0 = 0, gcell = 1, ginv = 1;
    int gw = 1, gh = 1;
    std::vector<int> gstart, glist, degenerate;
};

/* CuNodesMap.h:109-112 */
inline float get_sign(float p1x, float p1y, float p2x, float p2y, float p3x, float p3y) {
    float a = (p1x - p3x) * (p2y - p3y);
    float b = (p2x - p3x) * (p1y - p3y);
    return a - b;
}

/* CuNodesMap.h:97-107 */
inline bool point_in_tri(const float* v, float px, float py) {
    float d1 = get_sign(px, py, v[0], v[1], v[2], v[3]);
    float d2 = get_sign(px, py, v[2], v[3], v[4], v[5]);
    float d3 = get_sign(px, py, v[4], v[5], v[0], v[1]);
    bool isNeg = (d1 < 0) || (d2 < 0) || (d3 < 0);
    bool isPos = (d1 > 0) || (d2 > 0) || (d3 > 0);
    return !(isNeg && isPos);
}

inline float dist_sqr(const Map& m, int a, int b) {
    /* CuNodesMap.h:74-80 -> V2Float.h:50-55 */
    float x = m.cx[a] - m.cx[b];
    float y = m.cy[a] - m.cy[b];
    float xx = x * x;
    float yy = y * y;
    return xx + yy;
}

int locate_linear(const Map& m, float px, float py) {
    /* CuNodesMap.h:53-66: the first triangle in index order */
    for (int i = 0; i < m.n; i++)
        if (point_in_tri(&m.t[6 * i], px, py)) return i;
    return -1;
}

void build_grid(Map& m) {
    if (m.n == 0) return;
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    for (int i = 0; i < m.n; i++)
        for (int k = 0; k < 3; k++) {
            x0 = std::min(x0, m.t[6 * i + 2 * k]);
            x1 = std::max(x1, m.t[6 * i + 2 * k]);
            y0 = std::min(y0, m.t[6 * i + 2 * k + 1]);
            y1 = std::max(y1, m.t[6 * i + 2 * k + 1]);
        }
    double w = std::max(1e-3, (double)x1 - x0), h = std::max(1e-3, (double)y1 - y0);
    double cell = std::sqrt(w * h / std::max(1, m.n));
    cell = std::max(cell, std::max(w, h) / 4096.0);
    m.gcell = (float)cell;
    m.ginv = (float)(1.0 / cell);
    m.gx0 = x0;
    m.gy0 = y0;
    m.gw = std::max(1, (int)std::ceil(w / cell) + 1);
    m.gh = std::max(1, (int)std::ceil(h / cell) + 1);
    std::vector<int> cnt((size_t)m.gw * m.gh + 1, 0);
    auto cell_range = [&](int i, int& cx0, int& cy0, int& cx1, int& cy1) {
        const float* v = &m.t[6 * i];
        double bx0 = std::min({v[0], v[2], v[4]}), bx1 = std::max({v[0], v[2], v[4]});
        double by0 = std::min({v[1], v[3], v[5]}), by1 = std::max({v[1], v[3], v[5]});
        double pad = 0.01 * cell + 1e-3 + 1e-5 * std::max(std::fabs(bx1), std::fabs(by1));
        cx0 = std::max(0, (int)std::floor((bx0 - pad - m.gx0) / cell));
        cy0 = std::max(0, (int)std::floor((by0 - pad - m.gy0) / cell));
        cx1 = std::min(m.gw - 1, (int)std::floor((bx1 + pad - m.gx0) / cell));
        cy1 = std::min(m.gh - 1, (int)std::floor((by1 + pad - m.gy0) / cell));
    };
    m.degenerate.clear();
    std::vector<char> degen(m.n, 0);
    for (int i = 0; i < m.n; i++) {
        const float* v = &m.t[6 * i];
        if (get_sign(v[0], v[1], v[2], v[3], v[4], v[5]) == 0.0f) {
            degen[i] = 1;
            m.degenerate.push_back(i);
            continue;
        }
        int a, b, c, d;
        cell_range(i, a, b, c, d);
        for (int y = b; y <= d; y++)
            for (int x = a; x <= c; x++) cnt[(size_t)y * m.gw + x + 1]++;
    }
    for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
    m.gstart = cnt;
    m.glist.assign(cnt.back(), 0);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < m.n; i++) {
        if (degen[i]) continue;
        int a, b, c, d;
        cell_range(i, a, b, c, d);
        for (int y = b; y <= d; y++)
            for (int x = a; x <= c; x++) m.glist[fill[(size_t)y * m.gw + x]++] = i;
    }
}

int locate(const Map& m, float px, float py) {
    if (!std::isfinite(px) || !std::isfinite(py)) return locate_linear(m, px, py);
    int cx = (int)std::floor(((double)px - m.gx0) / m.gcell);
    int cy = (int)std::floor(((double)py - m.gy0) / m.gcell);
    cx = std::min(std::max(cx, 0), m.gw - 1);
    cy = std::min(std::max(cy, 0), m.gh - 1);
    size_t c = (size_t)cy * m.gw + cx;
    int best = -1;
    for (int k = m.gstart[c]; k < m.gstart[c + 1]; k++) {
        int i = m.glist[k];
        if (point_in_tri(&m.t[6 * i], px, py)) { best = i; break; }
    }
    for (int i : m.degenerate) {
        if (best >= 0 && i > best) break;
        if (point_in_tri(&m.t[6 * i], px, py)) { best = i; break; }
    }
    return best;
}

/* ---------------------------------------------------------------- queue --- */

struct QItem {
    float F;
    int G;
    int id;
    int dir;  /* 1 = from start, 0 = from target (PathNode::FromStart) */
};

inline bool qless(const QItem& a, const QItem& b) {
    if (a.F != b.F) return a.F < b.F;
    if (a.G != b.G) return a.G < b.G;
    return a.id < b.id;
}

/* Bounded queue kept in descending key order, minimum at the back, as the
 * reference's CuQueue (CuQueue.h:33-70).  fifo: the reference's own key, F
 * alone: a new item goes after every queued item with a larger F, so equal F
 * leave first in first out and a full queue evicts the newest of the maximal
 * F (CuQueue.h:39-63); otherwise the (F, G, id) order the kernels use. */
struct BQueue {
    std::vector<QItem> d;
    int cap = 0;
    bool fifo = false;
    void reset(int c, bool f = false) { d.clear(); cap = c; fifo = f; d.reserve(c + 1); }
    bool empty() const { return d.empty(); }
    QItem pop() { QItem x = d.back(); d.pop_back(); return x; }
    void push(const QItem& it) {
        /* position: after every element that is greater than `it` */
        auto pos = fifo ? std::lower_bound(d.begin(), d.end(), it,
                                           [](const QItem& a, const QItem& b) { return a.F > b.F; })
                        : std::lower_bound(d.begin(), d.end(), it,
                                           [](const QItem& a, const QItem& b) { return qless(b, a); });
        if ((int)d.size() < cap) {
            d.insert(pos, it);
            return;
        }
        if (pos == d.begin()) return;      /* not smaller than the maximum: dropped */
        d.insert(pos, it);
        d.erase(d.begin());                /* evict the maximum */
    }
};

/* --------------------------------------------------------------- search --- */

struct SearchScratch {
    std::vector<uint32_t> stamp;
    std::vector<int> dir, g, prev;
    uint32_t epoch = 0;
    std::vector<BQueue> q;
    std::vector<QItem> frontier;
    void ensure(int n, int T) {
        if ((int)stamp.size() < n) {
            stamp.assign(n, 0);
            dir.assign(n, 0);
            g.assign(n, 0);
            prev.assign(n, 0);
            epoch = 0;
        }
        if ((int)q.size() < T) q.resize(T);
    }
};

/* The reference's own orders, emulated for path-cost comparisons (the
 * kernels follow the deterministic order): fifo = its queue key (above);
 * seed != 0 = within each neighbour slot of a round, the expanding lanes in a
 * seeded random order: the reference's threads take their slots in step but
 * race inside each claim and frontier append (atomicExch, atomicAdd;
 * PathFinder.h:198-231), so claims, the meeting pair and frontier positions
 * follow that order. */
struct SearchOrder {
    int fifo = 0;
    uint64_t seed = 0;
};

inline uint64_t mix64(uint64_t x) {  /* splitmix64 finaliser */
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

int search(const Map& m, int start, int target, int T, int C, float K, SearchScratch& s,
           std::vector<int>& path, orc_search_stats* st, const SearchOrder& ord = SearchOrder()) {
    s.ensure(m.n, T);
    path.clear();
    if (start == target) return 1; /* already there: found, empty path */
    if (++s.epoch == 0) {
        std::fill(s.stamp.begin(), s.stamp.end(), 0u);
        s.epoch = 1;
    }
    const uint32_t ep = s.epoch;
    for (int q = 0; q < T; q++) s.q[q].reset(C, ord.fifo != 0);
    orc_search_stats loc{0, 0, 0, 0};
    uint64_t rng = ord.seed ? mix64(ord.seed ^ ((uint64_t)(uint32_t)start << 32 | (uint32_t)target)) : 0;
    std::vector<int> cand_q, cand_s;  /* racing order: candidates (lane, slot) in order */

    auto claim = [&](int n, int d, int G, int pv) {
        s.stamp[n] = ep;
        s.dir[n] = d;
        s.g[n] = G;
        s.prev[n] = pv;
        loc.claims++;
    };
    /* PathFinder.h:168-189: lane 0 seeds the start, lane 1 the target */
    float f0 = dist_sqr(m, start, target) * K;
    s.q[0].push(QItem{f0, 0, start, 1});
    claim(start, 1, 0, -1);
    if (T > 1) {
        s.q[1].push(QItem{f0, 0, target, 0});
        claim(target, 0, 0, -1);
    }

    int found = 0, mS = -1, mT = -1;
    std::vector<QItem> popped(T);
    std::vector<char> has(T);
    for (;;) {
        loc.rounds++;
        for (int q = 0; q < T; q++) {
            has[q] = !s.q[q].empty();
            if (has[q]) {
                popped[q] = s.q[q].pop();
                loc.expansions++;
                loc.deg_sum += m.deg[popped[q].id];
            }
        }
        s.frontier.clear();
        bool meet = false;
        /* candidate order: slot-major, lanes ascending (deterministic) or in a
         * random order within each slot (Fisher-Yates) */
        cand_q.clear();
        cand_s.clear();
        if (ord.seed) {
            std::vector<int> lanes;
            for (int slot = 0; slot < 3; slot++) {
                lanes.clear();
                for (int q = 0; q < T; q++)
                    if (has[q] && slot < m.deg[popped[q].id]) lanes.push_back(q);
                for (int k = (int)lanes.size() - 1; k > 0; k--) {
                    rng = mix64(rng);
                    std::swap(lanes[k], lanes[(int)(rng % (uint64_t)(k + 1))]);
                }
                for (int q : lanes) {
                    cand_q.push_back(q);
                    cand_s.push_back(slot);
                }
            }
        }
        const int ncand = ord.seed ? (int)cand_q.size() : 3 * T;
        for (int c = 0; c < ncand; c++) {
            {
                const int q = ord.seed ? cand_q[c] : c % T;
                const int slot = ord.seed ? cand_s[c] : c / T;
                if (!has[q]) continue;
                const QItem& u = popped[q];
                if (slot >= m.deg[u.id]) continue;
                int nbn = m.nb[3 * u.id + slot];
                int far = u.dir ? target : start;
                float h = dist_sqr(m, nbn, far);
                int G = u.G + 1;
                float hk = h * K;
                float F = (float)G + hk;
                if (s.stamp[nbn] != ep) {
                    claim(nbn, u.dir, G, u.id);
                    s.frontier.push_back(QItem{F, G, nbn, u.dir});
                } else if (!meet && s.dir[nbn] != u.dir) {
                    meet = true;
                    mS = u.dir ? u.id : nbn;
                    mT = u.dir ? nbn : u.id;
                }
            }
        }
        if (meet) {
            found = 1;
            break;
        }
        for (size_t i = 0; i < s.frontier.size(); i++) s.q[i % T].push(s.frontier[i]);
        bool any = false;
        for (int q = 0; q < T; q++) any = any || !s.q[q].empty();
        if (!any) break;
    }
    path.clear();
    if (found) {
        /* PathFinder.h:276-306 */
        int gs = s.g[mS], gt = s.g[mT];
        int L = gs + gt + 1;
        path.assign(L, -1);
        int idx = gs - 1;
        for (int x = mS; x != start; x = s.prev[x]) path[idx--] = x;
        idx = gs;
        int x = mT;
        for (; x != target; x = s.prev[x]) path[idx++] = x;
        path[idx] = target;
    }
    if (st) {
        st->rounds += loc.rounds;
        st->expansions += loc.expansions;
        st->claims += loc.claims;
        st->deg_sum += loc.deg_sum;
    }
    return found;
}

template <class F>
void parallel_for(int n, int threads, F&& fn) {
    if (threads <= 1 || n < 2) {
        for (int i = 0; i < n; i++) fn(i, 0);
        return;
    }
    threads = std::min(threads, n);
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++)
        th.emplace_back([&, t] {
            for (;;) {
                int i = next.fetch_add(1);
                if (i >= n) break;
                fn(i, t);
            }
        });
    for (auto& x : th) x.join();
}

/* ---------------------------------------------------------------- world --- */

enum { IDLE = 0, SEARCH = 1, MOVE = 2 };

struct Agent {
    float px, py;
    int cur;
    float tx, ty;
    int targ;
    int state;
    std::vector<int> path;
    int step_idx, step_node;
    float sx, sy;
    std::vector<float> wp;  /* path smoothing: steering point per path step (x, y) */
};

struct World {
    const Map* m;
    int max_agents;
    float radius, speed, cd, cd2;
    int P, T, C;
    float K;
    float cs, sn;
    std::vector<Agent> a;
    long long last[6] = {0, 0, 0, 0, 0, 0};
};

}  // namespace

struct orc_map : Map {};
struct orc_world : World {
    int smoothing = 0;
};

namespace {

/* ---- path smoothing: portals of the corridor, then the simple stupid funnel
 * (M. Mononen, 2010).  twice the signed area of (a, b, c), > 0 when c is left
 * of a -> b; every product and difference rounded to binary32 on its own. */
float orient2(float ax, float ay, float bx, float by, float cx, float cy) {
    float ux = bx - ax, uy = by - ay;
    float vx = cx - ax, vy = cy - ay;
    float p1 = ux * vy;
    float p2 = vx * uy;
    return p1 - p2;
}

/* portals 0..L+1: the start point, the shared edges (left, right as seen from
 * the earlier triangle's centroid towards the later one's), the end point */
/* path smoothing 2: both ends of an edge portal moved inward by c (the agent
 * radius); a portal no wider than 2c becomes its midpoint */
void narrow_portal(float& lx, float& ly, float& rx, float& ry, float c) {
    if (!(c > 0.0f)) return;
    const float dx = rx - lx, dy = ry - ly;
    const float xx = dx * dx, yy = dy * dy;
    const float w = std::sqrt(xx + yy);
    if (w > c + c) {
        const float t = c / w;
        const float ox = dx * t, oy = dy * t;
        lx = lx + ox;
        ly = ly + oy;
        rx = rx - ox;
        ry = ry - oy;
    } else {
        const float mx = (lx + rx) * 0.5f, my = (ly + ry) * 0.5f;
        lx = rx = mx;
        ly = ry = my;
    }
}

void corridor(const Map& m, int start_tri, const std::vector<int>& path, float sx, float sy, float ex, float ey,
              float clear, std::vector<float>& lx, std::vector<float>& ly, std::vector<float>& rx,
              std::vector<float>& ry) {
    const int L = (int)path.size();
    lx.assign(L + 2, 0);
    ly.assign(L + 2, 0);
    rx.assign(L + 2, 0);
    ry.assign(L + 2, 0);
    lx[0] = rx[0] = sx;
    ly[0] = ry[0] = sy;
    lx[L + 1] = rx[L + 1] = ex;
    ly[L + 1] = ry[L + 1] = ey;
    for (int k = 1; k <= L; k++) {
        const int u = k == 1 ? start_tri : path[k - 2], v = path[k - 1];
        const float* A = &m.t[6 * (size_t)u];
        const float* B = &m.t[6 * (size_t)v];
        float sh[4];
        int cnt = 0;
        for (int a = 0; a < 3; a++) {
            bool in_b = false;
            for (int b = 0; b < 3; b++) in_b = in_b || (A[2 * a] == B[2 * b] && A[2 * a + 1] == B[2 * b + 1]);
            if (in_b && cnt < 2) {
                sh[2 * cnt] = A[2 * a];
                sh[2 * cnt + 1] = A[2 * a + 1];
            }
            if (in_b) cnt++;
        }
        if (cnt < 2) {
            lx[k] = rx[k] = m.cx[v];
            ly[k] = ry[k] = m.cy[v];
            continue;
        }
        const bool first_left = orient2(m.cx[u], m.cy[u], m.cx[v], m.cy[v], sh[0], sh[1]) > 0.0f;
        const int li = first_left ? 0 : 1, ri = 1 - li;
        lx[k] = sh[2 * li];
        ly[k] = sh[2 * li + 1];
        rx[k] = sh[2 * ri];
        ry[k] = sh[2 * ri + 1];
        narrow_portal(lx[k], ly[k], rx[k], ry[k], clear);
    }
}

/* steering point of each path step: the first funnel corner at a portal index
 * past the step's portal (step k crosses portal k + 1) */
void funnel_points(const Map& m, Agent& ag, float clear) {
    const int L = (int)ag.path.size();
    std::vector<float> lx, ly, rx, ry;
    corridor(m, ag.cur, ag.path, ag.px, ag.py, ag.tx, ag.ty, clear, lx, ly, rx, ry);
    std::vector<float> cx, cy;
    std::vector<int> ci;  /* corners and their portal indices */
    float apx = ag.px, apy = ag.py, flx = apx, fly = apy, frx = apx, fry = apy;
    int apex = 0, lft = 0, rgt = 0;
    int guard = 0;
    const int max_guard = 4 * (L + 2) + 16;
    bool capped = false;
    int k = 1;
    while (k <= L + 1) {
        if (++guard > max_guard) {
            capped = true;
            break;
        }
        bool restart = false;
        if (orient2(apx, apy, frx, fry, rx[k], ry[k]) >= 0.0f) {
            if ((apx == frx && apy == fry) || orient2(apx, apy, flx, fly, rx[k], ry[k]) < 0.0f) {
                frx = rx[k];
                fry = ry[k];
                rgt = k;
            } else {
                cx.push_back(flx);
                cy.push_back(fly);
                ci.push_back(lft);
                apx = flx;
                apy = fly;
                apex = lft;
                restart = true;
            }
        }
        if (!restart && orient2(apx, apy, flx, fly, lx[k], ly[k]) <= 0.0f) {
            if ((apx == flx && apy == fly) || orient2(apx, apy, frx, fry, lx[k], ly[k]) > 0.0f) {
                flx = lx[k];
                fly = ly[k];
                lft = k;
            } else {
                cx.push_back(frx);
                cy.push_back(fry);
                ci.push_back(rgt);
                apx = frx;
                apy = fry;
                apex = rgt;
                restart = true;
            }
        }
        if (restart) {
            flx = frx = apx;
            fly = fry = apy;
            lft = rgt = apex;
            k = apex + 1;
        } else {
            k++;
        }
    }
    ag.wp.assign(2 * (size_t)L, 0.0f);
    size_t c = 0;
    for (int step = 0; step < L; step++) {
        while (c < ci.size() && ci[c] < step + 1) c++;
        if (c < ci.size()) {
            ag.wp[2 * step] = cx[c];
            ag.wp[2 * step + 1] = cy[c];
        } else if (capped) {
            ag.wp[2 * step] = m.cx[ag.path[step]];
            ag.wp[2 * step + 1] = m.cy[ag.path[step]];
        } else {
            ag.wp[2 * step] = ag.tx;
            ag.wp[2 * step + 1] = ag.ty;
        }
    }
}

}  // namespace

extern "C" {

orc_map* orc_map_create(const float* tri, const int* nbr, int n) {
    auto* m = new orc_map();
    m->n = n;
    m->t.assign(tri, tri + 6 * (size_t)n);
    m->nb.assign(nbr, nbr + 3 * (size_t)n);
    m->cx.resize(n);
    m->cy.resize(n);
    m->deg.resize(n);
    for (int i = 0; i < n; i++) {
        const float* v = &m->t[6 * i];
        /* GMAPF.cu:215: (P1 + P2 + P3) / 3.0f, left to right */
        float sx = v[0] + v[2];
        sx = sx + v[4];
        float sy = v[1] + v[3];
        sy = sy + v[5];
        m->cx[i] = sx / 3.0f;
        m->cy[i] = sy / 3.0f;
        int d = 0;
        while (d < 3 && m->nb[3 * i + d] != -1) d++;
        m->deg[i] = d;
    }
    build_grid(*m);
    return m;
}

void orc_map_destroy(orc_map* m) { delete m; }
int orc_map_count(const orc_map* m) { return m->n; }

void orc_map_centroids(const orc_map* m, float* out) {
    for (int i = 0; i < m->n; i++) {
        out[2 * i] = m->cx[i];
        out[2 * i + 1] = m->cy[i];
    }
}

int orc_locate_linear(const orc_map* m, float x, float y) { return locate_linear(*m, x, y); }
int orc_locate(const orc_map* m, float x, float y) { return locate(*m, x, y); }
void orc_locate_batch(const orc_map* m, const float* xy, int n, int* out) {
    for (int i = 0; i < n; i++) out[i] = locate(*m, xy[2 * i], xy[2 * i + 1]);
}
int orc_in_node(const orc_map* m, float x, float y, int node) {
    return point_in_tri(&m->t[6 * node], x, y) ? 1 : 0;
}
float orc_dist_sqr(const orc_map* m, int a, int b) { return dist_sqr(*m, a, b); }

int orc_search(const orc_map* m, int start, int target, int T, int C, float K, int* path,
               int path_cap, int* path_len, orc_search_stats* st) {
    SearchScratch s;
    std::vector<int> p;
    int f = search(*m, start, target, T, C, K, s, p, st);
    *path_len = (int)p.size();
    if ((int)p.size() > path_cap) return -1;
    std::copy(p.begin(), p.end(), path);
    return f;
}

int orc_search_batch(const orc_map* m, const int* starts, const int* targets, int n, int T,
                     int C, float K, int* found, int* lens, int* paths_out, int path_stride,
                     orc_search_stats* st_total, int threads) {
    threads = std::max(1, threads);
    std::vector<SearchScratch> scratch(threads);
    std::vector<orc_search_stats> st(threads, orc_search_stats{0, 0, 0, 0});
    std::atomic<int> overflow{0};
    parallel_for(n, threads, [&](int i, int t) {
        std::vector<int> p;
        found[i] = search(*m, starts[i], targets[i], T, C, K, scratch[t], p, &st[t]);
        lens[i] = (int)p.size();
        if (paths_out) {
            if ((int)p.size() > path_stride) overflow = 1;
            else std::copy(p.begin(), p.end(), paths_out + (size_t)i * path_stride);
        }
    });
    if (st_total) {
        for (auto& x : st) {
            st_total->rounds += x.rounds;
            st_total->expansions += x.expansions;
            st_total->claims += x.claims;
            st_total->deg_sum += x.deg_sum;
        }
    }
    return overflow ? -1 : 0;
}

int orc_search_batch_order(const orc_map* m, const int* starts, const int* targets, int n, int T,
                           int C, float K, int fifo, unsigned long long seed, int* found, int* lens,
                           int* paths_out, int path_stride, orc_search_stats* st_total, int threads) {
    threads = std::max(1, threads);
    SearchOrder ord;
    ord.fifo = fifo;
    ord.seed = seed;
    std::vector<SearchScratch> scratch(threads);
    std::vector<orc_search_stats> st(threads, orc_search_stats{0, 0, 0, 0});
    std::atomic<int> overflow{0};
    parallel_for(n, threads, [&](int i, int t) {
        std::vector<int> p;
        found[i] = search(*m, starts[i], targets[i], T, C, K, scratch[t], p, &st[t], ord);
        lens[i] = (int)p.size();
        if (paths_out) {
            if ((int)p.size() > path_stride) overflow = 1;
            else std::copy(p.begin(), p.end(), paths_out + (size_t)i * path_stride);
        }
    });
    if (st_total) {
        for (auto& x : st) {
            st_total->rounds += x.rounds;
            st_total->expansions += x.expansions;
            st_total->claims += x.claims;
            st_total->deg_sum += x.deg_sum;
        }
    }
    return overflow ? -1 : 0;
}

int orc_queue_sim_order(const float* F, const int* G, const int* id, int n_items, const int* ops,
                        int n_ops, int C, int fifo, int* out_popped, int* out_final) {
    BQueue q;
    q.reset(C, fifo != 0);
    int next = 0, npop = 0;
    for (int k = 0; k < n_ops; k++) {
        if (ops[k] == 1) {
            if (next < n_items) {
                q.push(QItem{F[next], G[next], id[next], 0});
                next++;
            }
        } else {
            out_popped[npop++] = q.empty() ? -1 : q.pop().id;
        }
    }
    int sz = (int)q.d.size();
    for (int i = 0; i < sz; i++) out_final[i] = q.d[sz - 1 - i].id;
    return sz;
}

int orc_queue_sim(const float* F, const int* G, const int* id, int n_items, const int* ops,
                  int n_ops, int C, int* out_popped, int* out_final) {
    BQueue q;
    q.reset(C);
    int next = 0, npop = 0;
    for (int k = 0; k < n_ops; k++) {
        if (ops[k] == 1) {
            if (next < n_items) {
                q.push(QItem{F[next], G[next], id[next], 0});
                next++;
            }
        } else {
            out_popped[npop++] = q.empty() ? -1 : q.pop().id;
        }
    }
    int sz = (int)q.d.size();
    for (int i = 0; i < sz; i++) out_final[i] = q.d[sz - 1 - i].id;
    return sz;
}

int orc_bfs_hops(const orc_map* m, int s, int t) {
    std::vector<int> d(m->n, -1);
    std::deque<int> dq;
    d[s] = 0;
    dq.push_back(s);
    while (!dq.empty()) {
        int u = dq.front();
        dq.pop_front();
        if (u == t) return d[u];
        for (int k = 0; k < m->deg[u]; k++) {
            int v = m->nb[3 * u + k];
            if (d[v] < 0) {
                d[v] = d[u] + 1;
                dq.push_back(v);
            }
        }
    }
    return -1;
}

double orc_dijkstra_len(const orc_map* m, int s, int t) {
    std::vector<double> d(m->n, INFINITY);
    using E = std::pair<double, int>;
    std::priority_queue<E, std::vector<E>, std::greater<E>> pq;
    d[s] = 0;
    pq.push({0.0, s});
    while (!pq.empty()) {
        auto [du, u] = pq.top();
        pq.pop();
        if (du > d[u]) continue;
        if (u == t) return du;
        for (int k = 0; k < m->deg[u]; k++) {
            int v = m->nb[3 * u + k];
            double dx = (double)m->cx[u] - m->cx[v], dy = (double)m->cy[u] - m->cy[v];
            double nd = du + std::sqrt(dx * dx + dy * dy);
            if (nd < d[v]) {
                d[v] = nd;
                pq.push({nd, v});
            }
        }
    }
    return -1.0;
}

double orc_path_len(const orc_map* m, int start, const int* path, int L) {
    double len = 0;
    int prev = start;
    for (int i = 0; i < L; i++) {
        double dx = (double)m->cx[prev] - m->cx[path[i]], dy = (double)m->cy[prev] - m->cy[path[i]];
        len += std::sqrt(dx * dx + dy * dy);
        prev = path[i];
    }
    return len;
}

orc_world* orc_world_create(const orc_map* m, int agents_max, float radius, float speed,
                            int parallel_agents, int T, int C, float K) {
    auto* w = new orc_world();
    w->m = m;
    w->max_agents = agents_max;
    w->radius = radius;
    w->speed = speed;
    w->cd = radius * 2.5f;       /* AgentsMover.h:222-223 */
    w->cd2 = w->cd * w->cd;
    w->P = parallel_agents;
    w->T = T;
    w->C = C;
    w->K = K;
    /* V2Float::GetRotated(10) (V2Float.h:39-47): cos/sin of 10 degrees, the
     * constants taken once in double precision and rounded to float */
    double ang = 10.0 * 3.14159265358979323846 / 180.0;
    w->cs = (float)std::cos(ang);
    w->sn = (float)std::sin(ang);
    w->a.reserve(agents_max);
    return w;
}

void orc_world_destroy(orc_world* w) { delete w; }
void orc_world_set_smoothing(orc_world* w, int mode) { w->smoothing = mode == 2 ? 2 : (mode ? 1 : 0); }
int orc_world_count(const orc_world* w) { return (int)w->a.size(); }

int orc_world_add_agent(orc_world* w, float x, float y) {
    if ((int)w->a.size() >= w->max_agents) return -1;
    int n = locate(*w->m, x, y);
    if (n < 0) return -1;
    Agent ag{};
    ag.px = x;
    ag.py = y;
    ag.cur = n;
    ag.state = IDLE;
    ag.targ = -1;
    ag.step_idx = -1;
    ag.step_node = -1;
    w->a.push_back(ag);
    return (int)w->a.size() - 1;
}

int orc_world_set_target(orc_world* w, int id, float x, float y) {
    int n = locate(*w->m, x, y);
    if (n < 0) return -1;
    Agent& ag = w->a[id];
    ag.state = SEARCH;
    ag.tx = x;
    ag.ty = y;
    ag.targ = n;
    return 0;
}

void orc_world_set(orc_world* w, int id, float px, float py, int state, int cur_node, float tx,
                   float ty, int targ_node, int step_idx, int step_node, float sx, float sy,
                   const int* path, int path_len) {
    Agent& ag = w->a[id];
    ag.px = px;
    ag.py = py;
    ag.state = state;
    ag.cur = cur_node;
    ag.tx = tx;
    ag.ty = ty;
    ag.targ = targ_node;
    ag.step_idx = step_idx;
    ag.step_node = step_node;
    ag.sx = sx;
    ag.sy = sy;
    ag.path.assign(path, path + path_len);
}

void orc_world_step(orc_world* w, float dt, int threads) {
    const Map& m = *w->m;
    auto& A = w->a;
    const int n = (int)A.size();
    threads = std::max(1, threads);

    /* 1. requests (PathFinder.h:85-116), ascending agent id */
    std::vector<int> req;
    for (int i = 0; i < n; i++) {
        Agent& ag = A[i];
        if (ag.state != SEARCH) continue;
        if (ag.cur == ag.targ) {
            ag.state = IDLE;
            continue;
        }
        if ((int)req.size() >= w->P) continue; /* stays in Search for the next frame */
        req.push_back(i);
    }
    /* 2. moving agents (AgentsMover.h:39-48) */
    std::vector<int> mv;
    for (int i = 0; i < n; i++)
        if (A[i].state == MOVE) mv.push_back(i);
    /* path smoothing: steering points of the paths that start this frame,
     * from the agents' positions at the frame's start */
    if (w->smoothing)
        for (int i : mv)
            if (A[i].step_idx == -1 && !A[i].path.empty()) funnel_points(m, A[i], w->smoothing == 2 ? w->radius : 0.0f);

    /* 3. searches + path build (PathFinder.h:253-307) */
    std::vector<SearchScratch> scratch(threads);
    std::vector<orc_search_stats> st(threads, orc_search_stats{0, 0, 0, 0});
    std::vector<int> fnd(req.size());
    parallel_for((int)req.size(), threads, [&](int r, int t) {
        Agent& ag = A[req[r]];
        fnd[r] = search(m, ag.cur, ag.targ, w->T, w->C, w->K, scratch[t], ag.path, &st[t]);
        if (fnd[r]) {
            ag.state = MOVE;
            ag.step_idx = -1;
        } else {
            ag.state = IDLE;
            ag.path.clear();
        }
    });
    long long nf = 0;
    for (int f : fnd) nf += f;
    w->last[0] = (long long)req.size();
    w->last[1] = nf;
    w->last[2] = 0;
    w->last[3] = 0;
    for (auto& x : st) {
        w->last[2] += x.expansions;
        w->last[3] += x.rounds;
    }
    w->last[4] = (long long)mv.size();
    w->last[5] = 0;

    if (mv.empty()) return; /* AgentsMover.h:296-297 */

    /* 4a. move (AgentsMover.h:51-71) */
    const float step = w->speed * dt;
    for (int i : mv) {
        Agent& ag = A[i];
        if (ag.step_idx == -1) continue;
        float dx = ag.sx - ag.px, dy = ag.sy - ag.py;
        float dxx = dx * dx, dyy = dy * dy;
        float len = std::sqrt(dxx + dyy);
        if (len <= step) {
            ag.px = ag.sx;
            ag.py = ag.sy;
        } else {
            float qx = dx / len, qy = dy / len;
            float mx = qx * step, my = qy * step;
            ag.px = ag.px + mx;
            ag.py = ag.py + my;
        }
    }

    /* 4b. collisions over all agents (AgentsMover.h:73-129), Jacobi reads */
    std::vector<float> ox(n), oy(n);
    for (int i = 0; i < n; i++) {
        ox[i] = A[i].px;
        oy[i] = A[i].py;
    }
    /* neighbour candidates from a uniform grid of cells >= 1.0625 * cd: every
     * pair closer than cd lies in adjacent cells, so the candidate set is a
     * superset of the all-pairs set and sorting it by id restores its order */
    float gx0 = INFINITY, gy0 = INFINITY, gx1 = -INFINITY, gy1 = -INFINITY;
    for (int i = 0; i < n; i++) {
        if (!std::isfinite(ox[i]) || !std::isfinite(oy[i])) continue;
        gx0 = std::min(gx0, ox[i]);
        gx1 = std::max(gx1, ox[i]);
        gy0 = std::min(gy0, oy[i]);
        gy1 = std::max(gy1, oy[i]);
    }
    std::vector<float> nx(n), ny(n);
    long long ncoll = 0;
    if (gx0 <= gx1) {
        double cell = std::max((double)w->cd * 1.0625, 1e-6);
        double span = std::max((double)gx1 - gx0, (double)gy1 - gy0);
        cell = std::max(cell, span / 2048.0);
        int gw = (int)((gx1 - gx0) / cell) + 1, gh = (int)((gy1 - gy0) / cell) + 1;
        std::vector<int> head((size_t)gw * gh, -1), nxt(n, -1), cellof(n, -1);
        for (int i = n - 1; i >= 0; i--) {
            if (!std::isfinite(ox[i]) || !std::isfinite(oy[i])) continue;
            int cx = std::min(gw - 1, (int)(((double)ox[i] - gx0) / cell));
            int cy = std::min(gh - 1, (int)(((double)oy[i] - gy0) / cell));
            size_t c = (size_t)cy * gw + cx;
            cellof[i] = (int)c;
            nxt[i] = head[c];
            head[c] = i;
        }
        std::vector<long long> cc(threads, 0);
        parallel_for(n, threads, [&](int i, int t) {
            nx[i] = ox[i];
            ny[i] = oy[i];
            if (cellof[i] < 0) return;
            int cx = cellof[i] % gw, cy = cellof[i] / gw;
            std::vector<int> cand;
            for (int yy = std::max(0, cy - 1); yy <= std::min(gh - 1, cy + 1); yy++)
                for (int xx = std::max(0, cx - 1); xx <= std::min(gw - 1, cx + 1); xx++)
                    for (int j = head[(size_t)yy * gw + xx]; j >= 0; j = nxt[j])
                        if (j != i) cand.push_back(j);
            std::sort(cand.begin(), cand.end());
            float sx = 0, sy = 0;
            int cnt = 0;
            for (int j : cand) {
                float dx = ox[i] - ox[j], dy = oy[i] - oy[j];
                float dxx = dx * dx, dyy = dy * dy;
                float d2 = dxx + dyy;
                if (d2 < w->cd2) {
                    float d = std::sqrt(d2);
                    float shift = w->cd - d;
                    float qx = dx / d, qy = dy / d;
                    float vx = qx * shift, vy = qy * shift;
                    sx = sx + vx;
                    sy = sy + vy;
                    cnt++;
                }
            }
            if (cnt == 0) return;
            cc[t]++;
            float fc = (float)cnt;
            float ax = sx / fc, ay = sy / fc;
            float r1 = ax * w->cs, r2 = ay * w->sn, r3 = ax * w->sn, r4 = ay * w->cs;
            float rx = r1 - r2, ry = r3 + r4;
            float px = ox[i] + rx, py = oy[i] + ry;
            if (locate(m, px, py) >= 0) {
                nx[i] = px;
                ny[i] = py;
            }
        });
        for (auto c : cc) ncoll += c;
    } else {
        for (int i = 0; i < n; i++) {
            nx[i] = ox[i];
            ny[i] = oy[i];
        }
    }
    for (int i = 0; i < n; i++) {
        A[i].px = nx[i];
        A[i].py = ny[i];
    }
    w->last[5] = ncoll;

    /* 4c. path progress (AgentsMover.h:131-177) */
    const float arrive = FLT_EPSILON + w->radius;
    for (int i : mv) {
        Agent& ag = A[i];
        if (ag.step_idx == -1) {
            ag.step_idx = 0;
            ag.step_node = ag.path[0];
            ag.sx = w->smoothing ? ag.wp[0] : m.cx[ag.step_node];
            ag.sy = w->smoothing ? ag.wp[1] : m.cy[ag.step_node];
            continue;
        }
        const bool inside = point_in_tri(&m.t[6 * ag.step_node], ag.px, ag.py);
        bool at_point = false; /* path smoothing: the steering point reached */
        if (w->smoothing && !inside) {
            float dx = ag.sx - ag.px, dy = ag.sy - ag.py;
            float dxx = dx * dx, dyy = dy * dy;
            at_point = std::sqrt(dxx + dyy) <= arrive;
        }
        if (!inside && !at_point) continue;
        int L = (int)ag.path.size();
        if (inside) {
            ag.cur = ag.step_node;
            if (ag.step_idx < L) ag.step_idx += 1;
        } else {
            /* skip the steps that steer to the point just reached */
            while (ag.step_idx < L && ag.wp[2 * ag.step_idx] == ag.sx && ag.wp[2 * ag.step_idx + 1] == ag.sy) {
                ag.cur = ag.path[ag.step_idx];
                ag.step_idx++;
            }
        }
        if (ag.step_idx == L) {
            float dx = ag.tx - ag.px, dy = ag.ty - ag.py;
            float dxx = dx * dx, dyy = dy * dy;
            if (std::sqrt(dxx + dyy) > arrive) {
                ag.sx = ag.tx;
                ag.sy = ag.ty;
            } else {
                ag.state = IDLE;
            }
        } else {
            ag.step_node = ag.path[ag.step_idx];
            ag.sx = w->smoothing ? ag.wp[2 * ag.step_idx] : m.cx[ag.step_node];
            ag.sy = w->smoothing ? ag.wp[2 * ag.step_idx + 1] : m.cy[ag.step_node];
        }
    }
}

void orc_world_get(const orc_world* w, float* pos, int* state, int* cur_node, int* targ_node,
                   int* step_idx, int* step_node, float* step_pos, int* path_len) {
    for (size_t i = 0; i < w->a.size(); i++) {
        const Agent& ag = w->a[i];
        if (pos) { pos[2 * i] = ag.px; pos[2 * i + 1] = ag.py; }
        if (state) state[i] = ag.state;
        if (cur_node) cur_node[i] = ag.cur;
        if (targ_node) targ_node[i] = ag.targ;
        if (step_idx) step_idx[i] = ag.step_idx;
        if (step_node) step_node[i] = ag.step_node;
        if (step_pos) { step_pos[2 * i] = ag.sx; step_pos[2 * i + 1] = ag.sy; }
        if (path_len) path_len[i] = (int)ag.path.size();
    }
}

int orc_world_get_path(const orc_world* w, int id, int* out, int cap) {
    const auto& p = w->a[id].path;
    int L = (int)p.size();
    for (int i = 0; i < std::min(L, cap); i++) out[i] = p[i];
    return L;
}

void orc_world_last_stats(const orc_world* w, long long* out6) {
    for (int k = 0; k < 6; k++) out6[k] = w->last[k];
}

}  // extern "C"
