/*
 * navmesh_oracle.cpp -- the oracle's own navmesh build (FillMapStart /
 * FillMapObstacle / FillMapEnd).
 *
 * TEST INFRASTRUCTURE ONLY (see gmapf_oracle.h): it lets the CPU baseline
 * and bench.py's reference arm build the benchmark maps without the product
 * library.  The reference triangulates with the CDT library it vendors
 * (artem-ogre/CDT, header-only, MPL-2.0, no version string in its tree);
 * this file is compiled against those same headers (ORC_HAVE_CDT, include
 * directory given at build time), so the triangles, their order and the
 * neighbour lists are the reference's own.  Steps restated:
 *   map border: vertices (0,0) (0,sy) (sx,sy) (sx,0), edges 0-1 1-2 2-3 3-0
 *     (src/GMAPF.cu:133-145);
 *   each obstacle: its vertices appended, consecutive ones joined by edges,
 *     the last joined to the first (src/GMAPF.cu:147-159);
 *   RemoveDuplicatesAndRemapEdges, Triangulation<float>(Auto, TryResolve,
 *     1.0), insert vertices, insert edges, eraseOuterTrianglesAndHoles, then
 *     per triangle its three vertices and the neighbours that exist, in CDT
 *     order, packed first and padded with -1 (src/GMAPF.cu:161-196).
 */
#include "gmapf_oracle.h"

#include <exception>
#include <vector>

#ifdef ORC_HAVE_CDT
#include "CDT/CDT.h"
#endif

extern "C" int orc_navmesh_build(float size_x, float size_y, const float* obst_xy, const int* obst_counts,
                                 int n_obst, float* out_tri, int* out_nbr, int cap) {
#ifndef ORC_HAVE_CDT
    (void)size_x; (void)size_y; (void)obst_xy; (void)obst_counts; (void)n_obst; (void)out_tri; (void)out_nbr;
    (void)cap;
    return -2;
#else
    try {
        std::vector<CDT::V2d<float>> verts = {CDT::V2d<float>::make(0.f, 0.f), CDT::V2d<float>::make(0.f, size_y),
                                              CDT::V2d<float>::make(size_x, size_y),
                                              CDT::V2d<float>::make(size_x, 0.f)};
        std::vector<CDT::Edge> edges = {CDT::Edge(0, 1), CDT::Edge(1, 2), CDT::Edge(2, 3), CDT::Edge(3, 0)};
        size_t k = 0;
        for (int o = 0; o < n_obst; o++) {
            const unsigned first = (unsigned)verts.size();
            for (int i = 0; i < obst_counts[o]; i++, k++) {
                verts.push_back(CDT::V2d<float>::make(obst_xy[2 * k], obst_xy[2 * k + 1]));
                if (i > 0) edges.emplace_back((unsigned)verts.size() - 2, (unsigned)verts.size() - 1);
            }
            edges.emplace_back((unsigned)verts.size() - 1, first);
        }
        CDT::RemoveDuplicatesAndRemapEdges(verts, edges);
        CDT::Triangulation<float> cdt(CDT::VertexInsertionOrder::Auto, CDT::IntersectingConstraintEdges::TryResolve,
                                      1.0f);
        cdt.insertVertices(verts);
        cdt.insertEdges(edges);
        cdt.eraseOuterTrianglesAndHoles();
        const int n = (int)cdt.triangles.size();
        if (n > cap) return -1;
        for (int t = 0; t < n; t++) {
            const auto& tr = cdt.triangles[t];
            for (int v = 0; v < 3; v++) {
                out_tri[6 * t + 2 * v] = cdt.vertices[tr.vertices[v]].x;
                out_tri[6 * t + 2 * v + 1] = cdt.vertices[tr.vertices[v]].y;
            }
            int m = 0;
            for (int i = 0; i < 3; i++)
                if (tr.neighbors[i] != CDT::noNeighbor) out_nbr[3 * t + m++] = (int)tr.neighbors[i];
            while (m < 3) out_nbr[3 * t + m++] = -1;
        }
        return n;
    } catch (const std::exception&) {
        return -3;
    }
#endif
}
