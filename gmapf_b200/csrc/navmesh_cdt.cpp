// navmesh_cdt.cpp -- FillMapEnd's navmesh build on the host.
//
// The reference triangulates with the CDT library it vendors (artem-ogre/CDT,
// MPL-2.0, header-only).  This file is compiled against those same headers,
// taken from an include directory given at build time (GMAPF_HAVE_CDT), so
// the triangle set, its order and every neighbour list are the reference's
// own.  The call sequence and the neighbour packing follow src/GMAPF.cu:161-196:
//   RemoveDuplicatesAndRemapEdges -> Triangulation<float>(Auto, TryResolve, 1.0f)
//   -> insertVertices -> insertEdges -> eraseOuterTrianglesAndHoles;
//   per triangle: its three vertices, then the neighbours that exist, in
//   CDT order, packed first and padded with -1.
// Without the headers the library builds without this step and FillMapEnd
// reports GMAPF_E_UNSUPPORTED (FillMapManually still works).
#include <stdexcept>

#include "internal.h"

#ifdef GMAPF_HAVE_CDT
#include "CDT/CDT.h"
#endif

namespace gmapf_b200 {

int build_navmesh_cdt(const std::vector<float>& verts, const std::vector<unsigned>& edges,
                      std::vector<gmapf_node>& out, std::string& err) {
#ifndef GMAPF_HAVE_CDT
    (void)verts;
    (void)edges;
    (void)out;
    err = "navmesh builder (CDT) not compiled into this library; use FillMapManually";
    return GMAPF_E_UNSUPPORTED;
#else
    try {
        std::vector<CDT::V2d<float>> v;
        v.reserve(verts.size() / 2);
        for (size_t i = 0; i + 1 < verts.size(); i += 2) v.push_back(CDT::V2d<float>::make(verts[i], verts[i + 1]));
        std::vector<CDT::Edge> e;
        e.reserve(edges.size() / 2);
        for (size_t i = 0; i + 1 < edges.size(); i += 2) e.emplace_back(edges[i], edges[i + 1]);

        CDT::RemoveDuplicatesAndRemapEdges(v, e);
        CDT::Triangulation<float> cdt(CDT::VertexInsertionOrder::Auto,
                                      CDT::IntersectingConstraintEdges::TryResolve, 1.0f);
        cdt.insertVertices(v);
        cdt.insertEdges(e);
        cdt.eraseOuterTrianglesAndHoles();

        out.clear();
        out.reserve(cdt.triangles.size());
        for (const auto& tr : cdt.triangles) {
            const auto& a = cdt.vertices[tr.vertices[0]];
            const auto& b = cdt.vertices[tr.vertices[1]];
            const auto& c = cdt.vertices[tr.vertices[2]];
            gmapf_node nd{};
            nd.P1 = gmapf_v2{a.x, a.y};
            nd.P2 = gmapf_v2{b.x, b.y};
            nd.P3 = gmapf_v2{c.x, c.y};
            int k = 0;
            for (int i = 0; i < 3; i++)
                if (tr.neighbors[i] != CDT::noNeighbor) nd.NeibsIdx[k++] = (int32_t)tr.neighbors[i];
            for (; k < 3; k++) nd.NeibsIdx[k] = -1;
            nd._pad = 0;
            out.push_back(nd);
        }
        return GMAPF_OK;
    } catch (const std::exception& ex) {
        err = std::string("navmesh triangulation failed: ") + ex.what();
        return GMAPF_E_INVALID_ARG;
    }
#endif
}

}  // namespace gmapf_b200
