// hostmap.cpp -- navmesh ingestion on the host: centroids, search rows and
// the point-location grid.
//
// Centroid: ((P1 + P2) + P3) / 3.0f per component, as src/GMAPF.cu:215
// (FillMapManually overwrites PCenter).  Neighbour lists are read as the
// reference's search reads them: up to the first -1 (PathFinder.h:198-201).
// Compiled with -ffp-contract=off.
#include <algorithm>
#include <cmath>

#include "internal.h"

namespace gmapf_b200 {

LocateGrid HostMap::view() const {
    LocateGrid g;
    g.x0 = gx0;
    g.y0 = gy0;
    g.inv = ginv;
    g.w = gw;
    g.h = gh;
    g.start = gstart.data();
    g.list = glist.data();
    g.degen = degen.data();
    g.ndegen = (int)degen.size();
    g.tri = tri.data();
    g.n = n;
    g.base = 0;
    return g;
}

void build_host_map(const gmapf_node* nodes, int n, HostMap& m) {
    m.n = n;
    m.nodes.assign(nodes, nodes + n);
    m.rows.assign(n, SearchRow{});
    m.tri.assign(3 * (size_t)n, make_float2(0, 0));
    m.cen.assign(n, make_float2(0, 0));
    for (int i = 0; i < n; i++) {
        gmapf_node& nd = m.nodes[i];
        float sx = nd.P1.X + nd.P2.X;
        sx = sx + nd.P3.X;
        float sy = nd.P1.Y + nd.P2.Y;
        sy = sy + nd.P3.Y;
        nd.PCenter.X = sx / 3.0f;
        nd.PCenter.Y = sy / 3.0f;
        m.cen[i] = make_float2(nd.PCenter.X, nd.PCenter.Y);
        m.tri[3 * i] = make_float2(nd.P1.X, nd.P1.Y);
        m.tri[3 * i + 1] = make_float2(nd.P2.X, nd.P2.Y);
        m.tri[3 * i + 2] = make_float2(nd.P3.X, nd.P3.Y);
    }
    for (int i = 0; i < n; i++) {
        const gmapf_node& nd = m.nodes[i];
        SearchRow r{};
        int nb[3] = {-1, -1, -1};
        int d = 0;
        while (d < 3 && nd.NeibsIdx[d] != -1) {
            nb[d] = nd.NeibsIdx[d];
            d++;
        }
        r.n0 = nb[0];
        r.n1 = nb[1];
        r.n2 = nb[2];
        r.deg = d;
        float2 c0 = nb[0] >= 0 ? m.cen[nb[0]] : make_float2(0, 0);
        float2 c1 = nb[1] >= 0 ? m.cen[nb[1]] : make_float2(0, 0);
        float2 c2 = nb[2] >= 0 ? m.cen[nb[2]] : make_float2(0, 0);
        r.x0 = c0.x;
        r.y0 = c0.y;
        r.x1 = c1.x;
        r.y1 = c1.y;
        r.x2 = c2.x;
        r.y2 = c2.y;
        r.pad0 = r.pad1 = 0;
        m.rows[i] = r;
    }

    // bounding box and point-location grid (about one triangle per cell)
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    for (const float2& v : m.tri) {
        if (!std::isfinite(v.x) || !std::isfinite(v.y)) continue;
        x0 = std::min(x0, v.x);
        x1 = std::max(x1, v.x);
        y0 = std::min(y0, v.y);
        y1 = std::max(y1, v.y);
    }
    if (!(x0 <= x1)) {
        x0 = y0 = 0;
        x1 = y1 = 1;
    }
    m.bx0 = x0;
    m.by0 = y0;
    m.bx1 = x1;
    m.by1 = y1;
    double w = std::max(1e-3, (double)x1 - x0), h = std::max(1e-3, (double)y1 - y0);
    double cell = std::sqrt(w * h / std::max(1, n));
    cell = std::max(cell, std::max(w, h) / 4096.0);
    m.gx0 = x0;
    m.gy0 = y0;
    m.ginv = (float)(1.0 / cell);
    m.gw = std::max(1, std::min(4096, (int)std::ceil(w / cell) + 1));
    m.gh = std::max(1, std::min(4096, (int)std::ceil(h / cell) + 1));
    const float pad = (float)(0.01 * cell + 1e-3 + 1e-5 * std::max(std::fabs((double)x1), std::fabs((double)y1)));

    std::vector<int> cnt((size_t)m.gw * m.gh + 1, 0);
    std::vector<char> isdeg(n, 0);
    m.degen.clear();
    auto range = [&](int i, int& a, int& b, int& c, int& d) {
        const float2* v = &m.tri[3 * (size_t)i];
        float bx0 = std::min({v[0].x, v[1].x, v[2].x}), bx1 = std::max({v[0].x, v[1].x, v[2].x});
        float by0 = std::min({v[0].y, v[1].y, v[2].y}), by1 = std::max({v[0].y, v[1].y, v[2].y});
        a = grid_cell(bx0 - pad, m.gx0, m.ginv, m.gw);
        c = grid_cell(bx1 + pad, m.gx0, m.ginv, m.gw);
        b = grid_cell(by0 - pad, m.gy0, m.ginv, m.gh);
        d = grid_cell(by1 + pad, m.gy0, m.ginv, m.gh);
    };
    for (int i = 0; i < n; i++) {
        const float2* v = &m.tri[3 * (size_t)i];
        bool finite = true;
        for (int k = 0; k < 3; k++) finite = finite && std::isfinite(v[k].x) && std::isfinite(v[k].y);
        if (!finite || get_sign(v[0].x, v[0].y, v[1].x, v[1].y, v[2].x, v[2].y) == 0.0f) {
            isdeg[i] = 1;
            m.degen.push_back(i);
            continue;
        }
        int a, b, c, d;
        range(i, a, b, c, d);
        for (int y = b; y <= d; y++)
            for (int x = a; x <= c; x++) cnt[(size_t)y * m.gw + x + 1]++;
    }
    for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
    m.gstart = cnt;
    m.glist.assign(cnt.back(), 0);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < n; i++) {
        if (isdeg[i]) continue;
        int a, b, c, d;
        range(i, a, b, c, d);
        for (int y = b; y <= d; y++)
            for (int x = a; x <= c; x++) m.glist[fill[(size_t)y * m.gw + x]++] = i;
    }
}

}  // namespace gmapf_b200

namespace gmapf_b200 {

// Breadth-first hop distances over the search's neighbour lists (leading
// valid entries).  Used only to order requests longest-first; the order
// does not change any result.
static void bfs_hops(const HostMap& m, int src, std::vector<unsigned short>& d) {
    d.assign(m.n, 65535);
    std::vector<int> q;
    q.reserve(m.n);
    d[src] = 0;
    q.push_back(src);
    for (size_t h = 0; h < q.size(); h++) {
        const int u = q[h];
        const SearchRow& r = m.rows[u];
        const int nb[3] = {r.n0, r.n1, r.n2};
        for (int k = 0; k < r.deg; k++) {
            const int v = nb[k];
            if (d[v] == 65535) {
                d[v] = (unsigned short)std::min(65534, d[u] + 1);
                q.push_back(v);
            }
        }
    }
}

void landmark_distances(const HostMap& m, int count, std::vector<unsigned short>& out) {
    out.assign((size_t)count * std::max(0, m.n), 65535);
    if (m.n == 0 || count <= 0) return;
    std::vector<unsigned short> d;
    std::vector<unsigned> best(m.n, 0xffffffffu);  // distance to the nearest landmark so far
    bfs_hops(m, 0, d);
    int next = 0;
    for (int i = 0; i < m.n; i++)
        if (d[i] != 65535 && d[i] > d[next]) next = i;
    for (int l = 0; l < count; l++) {
        bfs_hops(m, next, d);
        std::copy(d.begin(), d.end(), out.begin() + (size_t)l * m.n);
        int far = next;
        for (int i = 0; i < m.n; i++) {
            best[i] = std::min<unsigned>(best[i], d[i]);
            if (best[i] != 65535 && best[i] > best[far]) far = i;
        }
        next = far;
    }
}

void concat_host_maps(const std::vector<const HostMap*>& maps, HostMap& out, std::vector<SceneInfo>& scenes) {
    out = HostMap{};
    scenes.assign(maps.size(), SceneInfo{});
    int base = 0;
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    for (size_t s = 0; s < maps.size(); s++) {
        const HostMap& m = *maps[s];
        SceneInfo& si = scenes[s];
        si.node_base = base;
        si.n = m.n;
        si.bx0 = m.bx0;
        si.by0 = m.by0;
        si.bx1 = m.bx1;
        si.by1 = m.by1;
        si.gx0 = m.gx0;
        si.gy0 = m.gy0;
        si.ginv = m.ginv;
        si.gw = m.gw;
        si.gh = m.gh;
        si.gstart_off = out.gstart.size();
        si.glist_off = out.glist.size();
        si.degen_off = out.degen.size();
        si.ndegen = (int)m.degen.size();
        // grid cell lists keep scene-local ids: the scene's LocateGrid adds node_base
        out.gstart.insert(out.gstart.end(), m.gstart.begin(), m.gstart.end());
        out.glist.insert(out.glist.end(), m.glist.begin(), m.glist.end());
        out.degen.insert(out.degen.end(), m.degen.begin(), m.degen.end());
        for (int i = 0; i < m.n; i++) {
            gmapf_node nd = m.nodes[i];
            for (int k = 0; k < 3; k++)
                if (nd.NeibsIdx[k] >= 0) nd.NeibsIdx[k] += base;
            out.nodes.push_back(nd);
            SearchRow r = m.rows[i];
            if (r.n0 >= 0) r.n0 += base;
            if (r.n1 >= 0) r.n1 += base;
            if (r.n2 >= 0) r.n2 += base;
            out.rows.push_back(r);
            out.cen.push_back(m.cen[i]);
            for (int k = 0; k < 3; k++) out.tri.push_back(m.tri[3 * (size_t)i + k]);
        }
        x0 = std::min(x0, m.bx0);
        y0 = std::min(y0, m.by0);
        x1 = std::max(x1, m.bx1);
        y1 = std::max(y1, m.by1);
        base += m.n;
    }
    out.n = base;
    out.bx0 = x0;
    out.by0 = y0;
    out.bx1 = x1;
    out.by1 = y1;
    // the world has no single point-location grid: locating goes through the scenes
    out.gx0 = out.gy0 = 0;
    out.ginv = 1;
    out.gw = out.gh = 1;
}

}  // namespace gmapf_b200
