/*
 * cloth_oracle.cpp — CPU oracle for the per-substep PBD cloth step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that tests/ compares the CUDA
 * path against, and the "port" CPU baseline of bench.py. The shipped library
 * (solidcloth_b200/) never includes, links or calls it.
 *
 * It restates, function by function, the SolidCloth reference code on the hot
 * path (file:line cited at each function), in the same floating-point
 * operation order, so that with -ffp-contract=off it reproduces the reference
 * build (oracle/_ref) bit for bit. On top of the reference's sequential
 * Gauss-Seidel order it accepts an explicit constraint order (orc_set_tri_order
 * / orc_set_bend_order) and the GPU's contact colouring (orc_set_contact_order),
 * so that it can also run "check mode": the same sequential sweep in the order
 * the coloured GPU sweep realises.
 */
#include "cloth_oracle.h"
#include "oracle_math.h"

#include <vector>
#include <array>
#include <cstdint>
#include <cstring>
#include <memory>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
static int omp_threads() { return omp_get_max_threads(); }
static int omp_thread() { return omp_get_thread_num(); }
#else
static int omp_threads() { return 1; }
static int omp_thread() { return 0; }
#endif

using namespace orc;
typedef uint32_t u32;

namespace orc { bool g_portable_math = false; }

namespace {

const V3 kGravity = {0.f, -9.8f, 0.f}; /* Physics/Common.h:18 */

enum { CF_VERTICES = 1, CF_TRIANGLES = 2, CF_SELF = 4, CF_WALLS = 8, CF_EDGES = 16 };
enum { ATF_VERTICES = 1, ATF_TRIANGLES = 2, ATF_EDGES = 4 };

/* ------------------------------------------------------------------ mesh */
struct Edge
{
    V3 n = {0, 0, 0};
    u32 i1 = 0, i2 = 0;
    int t1 = -1, t2 = -1;
    int origIdx = 0;
    bool swapped = false;
};

struct Topo
{
    std::vector<V3> verts;
    std::vector<u32> idx;
    std::vector<V3> normals;
    std::vector<V3> triN;
    std::vector<std::array<u32, 3>> triE;
    std::vector<Edge> edges;
    std::vector<std::vector<int>> vtxRing, edgeRing;

    int ntris() const { return (int)idx.size() / 3; }

    /* Mesh::ComputeNormals, angle-weighted (Geometry/Mesh.cpp:10-63) */
    void compute_normals()
    {
        normals.assign(verts.size(), v3(0, 0, 0));
        triN.resize(idx.size() / 3);
        for (size_t i = 0; i < idx.size(); i += 3)
        {
            const int i1 = idx[i], i2 = idx[i + 1], i3 = idx[i + 2];
            V3 a = verts[i1], b = verts[i2], c = verts[i3];
            V3 n = cross(b - a, c - a);
            V3 nt = normalized(n);
            triN[i / 3] = nt;
            V3 e1 = normalized(b - a), e2 = normalized(c - b), e3 = normalized(a - c);
            float c1 = -dot(e1, e3), c2 = -dot(e1, e2), c3 = -dot(e2, e3);
            float s1 = len(cross(e1, -e3)), s2 = len(cross(e2, -e1)), s3 = len(cross(e3, -e1));
            float t1 = std::fabs(c1) > 1 ? (float)std::fabs(std::atan2((double)s1, (double)c1)) : step_acos(c1);
            float t2 = std::fabs(c2) > 1 ? (float)std::fabs(std::atan2((double)s2, (double)c2)) : step_acos(c2);
            float t3 = std::fabs(c3) > 1 ? (float)std::fabs(std::atan2((double)s3, (double)c3)) : step_acos(c3);
            normals[i1] += t1 * nt;
            normals[i2] += t2 * nt;
            normals[i3] += t3 * nt;
        }
        for (size_t i = 0; i < verts.size(); i++)
        {
            if (len(normals[i]) == 0) continue;
            normals[i] = normalized(normals[i]);
        }
    }

    /* Mesh::ConstructEdges (Geometry/Mesh.cpp:65-147). std::sort with the same
       (i1, i2) comparator on the same input order reproduces the reference's
       (unstable) ordering of the two half-edges of each interior edge. */
    void construct_edges()
    {
        edges.clear();
        int numEdges = (int)idx.size();
        std::vector<Edge> dup(numEdges);
        triE.assign(idx.size() / 3, {0, 0, 0});
        for (int i = 0; i < numEdges; i++)
        {
            int i1 = idx[i];
            int i2;
            if ((i + 1) % 3 == 0)
            {
                i2 = idx[i - 2];
                triE[i / 3][2] = (u32)i;
                triE[i / 3][1] = (u32)(i - 1);
                triE[i / 3][0] = (u32)(i - 2);
            }
            else
                i2 = idx[i + 1];
            bool swapped = false;
            if (i1 > i2) { std::swap(i1, i2); swapped = true; }
            Edge e;
            e.i1 = i1; e.i2 = i2; e.swapped = swapped; e.t1 = i / 3; e.t2 = -1;
            e.n = triN[i / 3];
            e.origIdx = i;
            dup[i] = e;
        }
        std::sort(dup.begin(), dup.end(), [](const Edge& a, const Edge& b) {
            return a.i1 < b.i1 || (a.i1 == b.i1 && a.i2 < b.i2);
        });
        Edge cur = dup[0];
        std::vector<int> map(dup.size(), -1);
        map[cur.origIdx] = 0;
        for (size_t i = 1; i < dup.size(); i++)
        {
            if (dup[i].i1 == dup[i - 1].i1 && dup[i].i2 == dup[i - 1].i2)
            {
                map[dup[i].origIdx] = (int)edges.size();
                cur.t2 = dup[i].t1;
                cur.n = normalized(triN[cur.t1] + triN[cur.t2]);
                continue;
            }
            edges.push_back(cur);
            cur = dup[i];
            map[cur.origIdx] = (int)edges.size();
        }
        edges.push_back(cur);
        for (size_t t = 0; t < triE.size(); t++)
            for (int j = 0; j < 3; j++) triE[t][j] = map[triE[t][j]];
    }

    /* ConstructVertexOneRings / ConstructEdgeOneRings (Geometry/Mesh.cpp:149-179) */
    void construct_rings(bool vtx, bool edge)
    {
        if (vtx) vtxRing.assign(verts.size(), {});
        if (edge) edgeRing.assign(verts.size(), {});
        for (size_t i = 0; i < edges.size(); i++)
        {
            if (vtx) { vtxRing[edges[i].i1].push_back(edges[i].i2); vtxRing[edges[i].i2].push_back(edges[i].i1); }
            if (edge) { edgeRing[edges[i].i1].push_back((int)i); edgeRing[edges[i].i2].push_back((int)i); }
        }
    }

    /* Mesh::AreAdjacent / IsBorderEdge / IsBorderVertex (Geometry/Mesh.h:237-263) */
    bool adjacent(int a, int b) const
    {
        for (int v : vtxRing[a]) if (v == b) return true;
        return false;
    }
    bool border_edge(int e) const { return edges[e].t2 < 0; }
    bool border_vertex(int v) const
    {
        if (v < 0) return false;
        for (int e : edgeRing[v]) if (border_edge(e)) return true;
        return false;
    }
};

/* ---------------------------------------------------------- Voronoi tests */
/* TestPointInTriangleVoronoiRegion (Geometry/VoronoiRegions.cpp:11-35). The
   chained comparison is kept: (signbit1 == signbit2) == signbit3. */
bool in_triangle_vr(V3 p, const Topo& m, int tri)
{
    V3 v1 = m.verts[m.idx[tri * 3]], v2 = m.verts[m.idx[tri * 3 + 1]], v3_ = m.verts[m.idx[tri * 3 + 2]];
    V3 e1 = v2 - v1, e2 = v3_ - v2, e3 = v1 - v3_;
    V3 n = m.triN[tri];
    V3 h1 = cross(e1, n), h2 = cross(e2, n), h3 = cross(e3, n);
    float d1 = dot(h1, p - v1), d2 = dot(h2, p - v2), d3 = dot(h3, p - v3_);
    bool s1 = std::signbit(d1), s2 = std::signbit(d2), s3 = std::signbit(d3);
    return (s1 == s2) == s3;
}

/* TestPointInEdgeVoronoiRegion, eps 0.002 (Geometry/VoronoiRegions.cpp:37-82) */
bool in_edge_vr(V3 p, const Topo& m, int eid, float eps = 0.002f)
{
    const Edge& ed = m.edges[eid];
    V3 a = m.verts[ed.i1], b = m.verts[ed.i2];
    V3 e = normalized(b - a);
    float d3 = dot(e, p - a), d4 = dot(e, p - b);
    if (d3 < 0 || d4 > 0) return false;
    if (ed.swapped) e = -e;
    if (ed.t2 >= 0)
    {
        V3 h1 = normalized(cross(e, m.triN[ed.t1]));
        V3 h2 = normalized(-cross(e, m.triN[ed.t2]));
        float d1 = dot(h1, p - a), d2 = dot(h2, p - a);
        if (d1 < -eps || d2 < -eps) return false;
    }
    else
    {
        V3 h1 = normalized(cross(e, m.triN[ed.t1]));
        if (dot(h1, p - a) < -eps) return false;
    }
    return true;
}

/* TestPointInVertexVoronoiRegion (Geometry/VoronoiRegions.cpp:84-113) */
bool in_vertex_vr(V3 p, const Topo& m, int vid)
{
    V3 v = m.verts[vid];
    float side = 1;
    if (dot(m.normals[vid], p - v) < 0) side = -1;
    const float eps = 0.1f;
    for (int ei : m.edgeRing[vid])
    {
        const Edge& ed = m.edges[ei];
        V3 e = normalized(m.verts[ed.i1] - m.verts[ed.i2]);
        if ((int)ed.i2 != vid) e = -e;
        float d = dot(e, p - v);
        if (side > 0 && d < -eps) return false;
        if (side < 0 && d > eps) return false;
    }
    return true;
}

/* ------------------------------------------------------- closest points */
struct TriInfo /* ClosestTriangleToPoint (Geometry/ClosestPointOnMesh.h:21-33) */
{
    V3 cp = {0, 0, 0}, normal = {0, 0, 0}, bary = {0, 0, 0};
    float distance = FLT_MAX;
    int tri = -1, vtx = -1, feature = -1, region = -1, regionType = -1;
    float side = FLT_MAX;
};

struct EdgeInfo /* ClosestEdgeToSegment (Geometry/ClosestPointOnMesh.h:44-56) */
{
    V3 cpMesh = {0, 0, 0}, cpSegm = {0, 0, 0}, normal = {0, 0, 0};
    float cs[2] = {0, 0}, cm[2] = {0, 0};
    int edge1 = -1, edge = -1;
    float distance = -FLT_MAX;
    int region = -1;
    float side = FLT_MAX;
};

struct VtxInfo /* ClosestVertexToTriangle (Geometry/ClosestPointOnMesh.h:66-75) */
{
    V3 cpMesh = {0, 0, 0}, cpTri = {0, 0, 0}, normal = {0, 0, 0}, bary = {0, 0, 0};
    float distance = -FLT_MAX;
    int vertex = -1, region = 0;
};

/* ClosestPointsOnMeshToPoint, brute force with Voronoi filters and
   first-feature dedup (Geometry/ClosestPointOnMesh.cpp:142-246) */
void closest_points_on_mesh_to_point(V3 p, const Topo& m, std::vector<TriInfo>& out, float maxDist, int idx)
{
    bool isBorder = m.border_vertex(idx);
    for (int i = 0; i < m.ntris(); i++)
    {
        int i0 = m.idx[i * 3], i1 = m.idx[i * 3 + 1], i2 = m.idx[i * 3 + 2];
        V3 a = m.verts[i0], b = m.verts[i1], c = m.verts[i2];
        V3 coords, pt;
        int region = closest_pt_point_triangle(p, a, b, c, pt, coords);
        bool inVR = idx >= 0 ? in_vertex_vr(pt, m, idx) : false;
        V3 delta = p - pt;
        float dist = len(delta);
        if (dist > maxDist) continue;
        if (dist == 0) continue;
        TriInfo r;
        if (region == TR_FACE_INTERIOR)
        {
            if (!(inVR || in_triangle_vr(p, m, i))) continue;
            r.regionType = 0;
        }
        if (region == TR_EDGE_AB)
        {
            int e = m.triE[i][0];
            if (!m.border_edge(e) && !(inVR || in_edge_vr(p, m, e))) continue;
            r.regionType = 1; r.feature = e;
        }
        if (region == TR_EDGE_BC)
        {
            int e = m.triE[i][1];
            if (!m.border_edge(e) && !(inVR || in_edge_vr(p, m, e))) continue;
            r.regionType = 1; r.feature = e;
        }
        if (region == TR_EDGE_AC)
        {
            int e = m.triE[i][2];
            if (!m.border_edge(e) && !(inVR || in_edge_vr(p, m, e))) continue;
            r.regionType = 1; r.feature = e;
        }
        if (region == TR_VERTEX_A)
        {
            if (!isBorder && !(inVR || in_vertex_vr(p, m, i0))) continue;
            r.regionType = 2; r.feature = i0;
        }
        if (region == TR_VERTEX_B)
        {
            if (!isBorder && !(inVR || in_vertex_vr(p, m, i1))) continue;
            r.regionType = 2; r.feature = i1;
        }
        if (region == TR_VERTEX_C)
        {
            if (!isBorder && !(inVR || in_vertex_vr(p, m, i2))) continue;
            r.regionType = 2; r.feature = i2;
        }
        if (r.feature >= 0)
        {
            bool found = false;
            for (const TriInfo& o : out)
                if (r.regionType == o.regionType && r.feature == o.feature) { found = true; break; }
            if (found) continue;
        }
        r.distance = dist;
        r.tri = i;
        r.cp = pt;
        r.bary = coords;
        r.normal = (1.f / dist) * delta;
        r.region = region;
        r.side = signed_volume(p, a, b, c);
        out.push_back(r);
    }
}

/* CheckAdjacency (Geometry/ClosestPointsBetweenMeshes.cpp:441-461) */
bool check_adjacency(const Topo& m, int vtx, int tri, int region)
{
    int i1 = m.idx[tri * 3], i2 = m.idx[tri * 3 + 1], i3 = m.idx[tri * 3 + 2];
    if (i1 == vtx || i2 == vtx || i3 == vtx) return true;
    if (region == TR_VERTEX_A && m.adjacent(vtx, i1)) return true;
    if (region == TR_VERTEX_B && m.adjacent(vtx, i2)) return true;
    if (region == TR_VERTEX_C && m.adjacent(vtx, i3)) return true;
    if (region == TR_EDGE_AB && (m.adjacent(vtx, i1) && m.adjacent(vtx, i2))) return true;
    if (region == TR_EDGE_BC && (m.adjacent(vtx, i2) && m.adjacent(vtx, i3))) return true;
    if (region == TR_EDGE_AC && (m.adjacent(vtx, i1) && m.adjacent(vtx, i3))) return true;
    return false;
}

/* ClosestPointOnMeshToSegment with e2 = the query edge: nearest non-adjacent
   edge of higher index (Geometry/ClosestPointOnMesh.cpp:499-542) */
void closest_edge_to_segment_self(V3 p, V3 q, const Topo& m, EdgeInfo& r, int e2)
{
    float distMin = FLT_MAX;
    const Edge& ed2 = m.edges[e2];
    for (int e1 = e2 + 1; e1 < (int)m.edges.size(); e1++)
    {
        u32 i1 = m.edges[e1].i1, i2 = m.edges[e1].i2;
        if (i1 == ed2.i1 || i1 == ed2.i2 || i2 == ed2.i1 || i2 == ed2.i2) continue;
        V3 a = m.verts[i1], b = m.verts[i2];
        float ps, pm;
        V3 cs, cm;
        int region = closest_pt_segm_segm(p, q, a, b, ps, pm, cs, cm);
        float dist = len(cs - cm);
        if (dist != 0 && dist < distMin)
        {
            distMin = dist;
            r.edge = e1;
            r.distance = dist;
            r.cpMesh = cm;
            r.cpSegm = cs;
            r.cs[0] = 1.0f - ps; r.cs[1] = ps;
            r.cm[0] = 1.0f - pm; r.cm[1] = pm;
            r.normal = normalized(cm - cs);
            r.side = signed_volume(p, q, a, b);
            r.region = region;
        }
    }
}

bool same_triangle(const Topo& m, int vtx, int tri)
{
    if (tri < 0) return false;
    return vtx == (int)m.idx[tri * 3] || vtx == (int)m.idx[tri * 3 + 1] || vtx == (int)m.idx[tri * 3 + 2];
}

/* CheckEdgeAdjacency (Geometry/ClosestPointsBetweenMeshes.cpp:474-536) */
bool check_edge_adjacency(EdgeInfo& info, const Topo& m, int i1, int i2, const Edge& edge1)
{
    const float eps = 1e-5f;
    int e = info.edge;
    if (e < 0) return true;
    const Edge& edge2 = m.edges[e];
    if (i1 == (int)edge2.i1 || i1 == (int)edge2.i2 || i2 == (int)edge2.i1 || i2 == (int)edge2.i2)
    { info.distance = FLT_MAX; return true; }
    if ((info.region & ER_VERTEX_P1) != 0 || info.cs[0] < eps)
        if (same_triangle(m, i1, edge2.t1) || same_triangle(m, i1, edge2.t2)) { info.distance = FLT_MAX; return true; }
    if ((info.region & ER_VERTEX_Q1) != 0 || info.cs[1] < eps)
        if (same_triangle(m, i2, edge2.t1) || same_triangle(m, i2, edge2.t2)) { info.distance = FLT_MAX; return true; }
    if ((info.region & ER_VERTEX_P2) != 0 || info.cm[0] < eps)
        if (same_triangle(m, edge2.i1, edge1.t1) || same_triangle(m, edge2.i1, edge1.t2)) { info.distance = FLT_MAX; return true; }
    if ((info.region & ER_VERTEX_Q2) != 0 || info.cm[1] < eps)
        if (same_triangle(m, edge2.i2, edge1.t1) || same_triangle(m, edge2.i2, edge1.t2)) { info.distance = FLT_MAX; return true; }
    return false;
}

/* ------------------------------------------------------- static mesh tree */
struct TreeNode
{
    Box box;
    std::vector<u32> tris, verts, edges;
    int left = -1, right = -1;
};

struct MeshCollider
{
    Topo m;
    std::vector<TreeNode> nodes; /* nodes[0] = root once built */
    bool built = false;

    /* SplitNode with exclusive child assignment (Geometry/AabbTree.cpp:9-134) */
    void split(int ni, int level, int maxLevel, float tol)
    {
        const size_t maxPrims = 40;
        if (nodes[ni].tris.size() < maxPrims && nodes[ni].verts.size() < maxPrims && nodes[ni].edges.size() < maxPrims)
            return;
        V3 ext = nodes[ni].box.mx - nodes[ni].box.mn;
        int dir = 0;
        float mxv = ext.x;
        if (ext.y > mxv) { mxv = ext.y; dir = 1; }
        if (ext.z > mxv) { mxv = ext.z; dir = 2; }
        float center = 0.5f * (comp(nodes[ni].box.mn, dir) + comp(nodes[ni].box.mx, dir));
        TreeNode L, R;
        for (u32 t : nodes[ni].tris)
        {
            Box b;
            b.add(m.verts[m.idx[t * 3]]); b.add(m.verts[m.idx[t * 3 + 1]]); b.add(m.verts[m.idx[t * 3 + 2]]);
            b.extrude(tol);
            if (comp(b.mn, dir) <= center) { L.tris.push_back(t); L.box.add(b); }
            else { R.tris.push_back(t); R.box.add(b); }
        }
        for (u32 e : nodes[ni].edges)
        {
            Box b;
            b.add(m.verts[m.edges[e].i1]); b.add(m.verts[m.edges[e].i2]);
            b.extrude(tol);
            if (comp(b.mn, dir) <= center) { L.edges.push_back(e); L.box.add(b); }
            else { R.edges.push_back(e); R.box.add(b); }
        }
        for (u32 v : nodes[ni].verts)
        {
            Box b;
            b.add(m.verts[v]);
            b.extrude(tol);
            if (comp(m.verts[v], dir) <= center) { L.verts.push_back(v); L.box.add(b); }
            else { R.verts.push_back(v); R.box.add(b); }
        }
        nodes[ni].tris.clear(); nodes[ni].edges.clear(); nodes[ni].verts.clear();
        bool hasL = !(L.tris.empty() && L.verts.empty() && L.edges.empty());
        bool hasR = !(R.tris.empty() && R.verts.empty() && R.edges.empty());
        if (hasL) { nodes.push_back(L); nodes[ni].left = (int)nodes.size() - 1; }
        if (hasR) { nodes.push_back(R); nodes[ni].right = (int)nodes.size() - 1; }
        if (level < maxLevel)
        {
            int l = nodes[ni].left, r = nodes[ni].right;
            if (l >= 0) split(l, level + 1, maxLevel, tol);
            if (r >= 0) split(r, level + 1, maxLevel, tol);
        }
    }

    /* ComputeMeshTree (Geometry/AabbTree.cpp:136-178); CollisionMesh::Update
       builds it once, lazily, with maxLevel 20 and tol = thickness
       (Physics/Common.h:124-137). */
    void build(float tol)
    {
        nodes.clear();
        TreeNode root;
        for (V3 v : m.verts) { root.box.mn = vmin(root.box.mn, v); root.box.mx = vmax(root.box.mx, v); }
        for (u32 i = 0; i < (u32)m.ntris(); i++) root.tris.push_back(i);
        for (u32 i = 0; i < (u32)m.verts.size(); i++) root.verts.push_back(i);
        for (u32 i = 0; i < (u32)m.edges.size(); i++) root.edges.push_back(i);
        nodes.push_back(root);
        split(0, 1, 20, tol);
        built = true;
    }

    /* ClosestTriKernel + ClosestPointOnMeshToPointRec, useDelta = true
       (Geometry/ClosestPointOnMesh.cpp:99-126, 262-302) */
    void point_rec(V3 p, int ni, float& minDist, TriInfo& r) const
    {
        const TreeNode& n = nodes[ni];
        for (u32 tri : n.tris)
        {
            V3 a = m.verts[m.idx[tri * 3]], b = m.verts[m.idx[tri * 3 + 1]], c = m.verts[m.idx[tri * 3 + 2]];
            V3 coords, pt;
            int region = closest_pt_point_triangle(p, a, b, c, pt, coords);
            V3 delta = p - pt;
            float dist = len(delta);
            if (dist == 0) continue;
            if (dist < minDist)
            {
                minDist = dist;
                r.distance = dist; r.tri = tri; r.cp = pt; r.bary = coords;
                r.normal = (1.f / dist) * delta;
                r.region = region;
            }
        }
        if (n.left < 0 && n.right < 0) return;
        float dl = n.left >= 0 ? nodes[n.left].box.dist(p) : FLT_MAX;
        float dr = n.right >= 0 ? nodes[n.right].box.dist(p) : FLT_MAX;
        if (dl < dr)
        {
            if (dl < minDist) point_rec(p, n.left, minDist, r);
            if (dr < minDist) point_rec(p, n.right, minDist, r);
        }
        else
        {
            if (dr < minDist) point_rec(p, n.right, minDist, r);
            if (dl < minDist) point_rec(p, n.left, minDist, r);
        }
    }

    /* ClosestPointOnMeshToTriangleRec (Geometry/ClosestPointOnMesh.cpp:393-452) */
    void tri_rec(V3 a, V3 b, V3 c, int ni, float& minDist, VtxInfo& r) const
    {
        const TreeNode& n = nodes[ni];
        for (u32 v : n.verts)
        {
            V3 bary, cp;
            int region = closest_pt_point_triangle(m.verts[v], a, b, c, cp, bary);
            V3 delta = cp - m.verts[v];
            float dist = len(delta);
            if (dist == 0) continue;
            if (dist < minDist)
            {
                minDist = dist;
                r.vertex = v; r.cpMesh = m.verts[v]; r.cpTri = cp; r.bary = bary;
                r.normal = (1.f / dist) * delta;
                r.distance = dist; r.region = region;
            }
        }
        if (n.left < 0 && n.right < 0) return;
        Box tb;
        tb.add(a); tb.add(b); tb.add(c);
        float dl = n.left >= 0 ? nodes[n.left].box.dist(tb) : FLT_MAX;
        float dr = n.right >= 0 ? nodes[n.right].box.dist(tb) : FLT_MAX;
        if (dl < dr)
        {
            if (dl < minDist) tri_rec(a, b, c, n.left, minDist, r);
            if (dr < minDist) tri_rec(a, b, c, n.right, minDist, r);
        }
        else
        {
            if (dr < minDist) tri_rec(a, b, c, n.right, minDist, r);
            if (dl < minDist) tri_rec(a, b, c, n.left, minDist, r);
        }
    }

    /* ComputeEdgeNormal (Geometry/ClosestPointOnMesh.cpp:483-497) */
    V3 edge_normal(int e, float param) const
    {
        V3 n = m.edges[e].n;
        if (param == 0.f) n = m.normals[m.edges[e].i1];
        if (param == 1.f) n = m.normals[m.edges[e].i2];
        return n;
    }

    /* ClosestPointOnMeshToSegmentEdgeRec, useDelta = false
       (Geometry/ClosestPointOnMesh.cpp:589-659) */
    void seg_rec(V3 p, V3 q, int ni, float& minDist, EdgeInfo& r) const
    {
        const TreeNode& n = nodes[ni];
        for (u32 i : n.edges)
        {
            V3 a = m.verts[m.edges[i].i1], b = m.verts[m.edges[i].i2];
            float ps, pm;
            V3 cs, cm;
            int region = closest_pt_segm_segm(p, q, a, b, ps, pm, cs, cm);
            V3 delta = cm - cs;
            float dist = len(delta);
            if (dist == 0) continue;
            if (dist < minDist)
            {
                minDist = dist;
                r.distance = dist; r.edge = i; r.cpMesh = cm; r.cpSegm = cs;
                r.cs[0] = 1.0f - ps; r.cs[1] = ps; r.cm[0] = 1.0f - pm; r.cm[1] = pm;
                r.normal = edge_normal(i, pm);
                r.region = region;
            }
        }
        if (n.left < 0 && n.right < 0) return;
        Box eb;
        eb.add(p); eb.add(q);
        float dl = n.left >= 0 ? nodes[n.left].box.dist(eb) : FLT_MAX;
        float dr = n.right >= 0 ? nodes[n.right].box.dist(eb) : FLT_MAX;
        if (dl < dr)
        {
            if (dl < minDist) seg_rec(p, q, n.left, minDist, r);
            if (dr < minDist) seg_rec(p, q, n.right, minDist, r);
        }
        else
        {
            if (dr < minDist) seg_rec(p, q, n.right, minDist, r);
            if (dl < minDist) seg_rec(p, q, n.left, minDist, r);
        }
    }
};

/* ------------------------------------------------------------- SDF grid */
struct GridSDF /* Geometry/SDF.h:13-251, SDF.cpp:10-40,210-256 */
{
    int nc[3], nv[3];
    std::vector<float> val;
    std::vector<V3> grad;
    Box box;
    V3 steps;

    int index(int x, int y, int z) const { return x + y * nv[0] + z * nv[0] * nv[1]; }
    bool out(int x, int y, int z) const { return x > nc[0] || y > nc[1] || z > nc[2] || x < 0 || y < 0 || z < 0; }
    float value_at(int x, int y, int z) const { return out(x, y, z) ? 0.f : val[index(x, y, z)]; }
    V3 grad_at(int x, int y, int z) const { return out(x, y, z) ? v3(0, 0, 0) : grad[index(x, y, z)]; }

    void create(int x, int y, int z, const Box& b)
    {
        box = b;
        nc[0] = x; nc[1] = y; nc[2] = z;
        for (int k = 0; k < 3; k++) nv[k] = nc[k] + 1;
        val.assign((size_t)nv[0] * nv[1] * nv[2], 0.f);
        V3 ext = box.mx - box.mn;
        V3 invRes = v3(1.f / nc[0], 1.f / nc[1], 1.f / nc[2]);
        steps = v3(ext.x * invRes.x, ext.y * invRes.y, ext.z * invRes.z);
    }

    void compute_gradient()
    {
        grad.assign(val.size(), v3(0, 0, 0));
        auto set = [&](int x, int y, int z, V3 g) { if (!out(x, y, z)) grad[index(x, y, z)] = g; };
        for (int x = 0; x < nc[0]; x++)
        {
            for (int y = 0; y < nc[1]; y++)
            {
                for (int z = 0; z < nc[2]; z++)
                {
                    float v = value_at(x, y, z);
                    float dfdx = (value_at(x + 1, y, z) - v) / steps.x;
                    float dfdy = (value_at(x, y + 1, z) - v) / steps.y;
                    float dfdz = (value_at(x, y, z + 1) - v) / steps.z;
                    set(x, y, z, v3(dfdx, dfdy, dfdz));
                }
                int z = nc[2];
                set(x, y, z, grad_at(x, y, z - 1));
            }
            int y = nc[1];
            for (int z = 0; z <= nc[2]; z++) set(x, y, z, grad_at(x, y - 1, z));
        }
        int x = nc[0];
        for (int y = 0; y <= nc[1]; y++)
            for (int z = 0; z <= nc[2]; z++) set(x, y, z, grad_at(x - 1, y, z));
    }

    void coords(V3 p, int& x, int& y, int& z, float& fx, float& fy, float& fz) const
    {
        float rx = (p.x - box.mn.x) / steps.x;
        float ry = (p.y - box.mn.y) / steps.y;
        float rz = (p.z - box.mn.z) / steps.z;
        x = (int)floorf(rx); y = (int)floorf(ry); z = (int)floorf(rz);
        fx = std::fabs(rx - x); fy = std::fabs(ry - y); fz = std::fabs(rz - z);
    }

    /* SDF::GetValue(Vector3), trilinear with the zero border (SDF.h:138-155) */
    float value(V3 p) const
    {
        int x, y, z; float fx, fy, fz;
        coords(p, x, y, z, fx, fy, fz);
        if (out(x, y, z)) return FLT_MAX;
        return (1.f - fx) * (1.f - fy) * (1.f - fz) * value_at(x, y, z) +
               (1.f - fx) * (1.f - fy) * fz * value_at(x, y, z + 1) +
               (1.f - fx) * fy * (1.f - fz) * value_at(x, y + 1, z) +
               (1.f - fx) * fy * fz * value_at(x, y + 1, z + 1) +
               fx * (1.f - fy) * (1.f - fz) * value_at(x + 1, y, z) +
               fx * (1.f - fy) * fz * value_at(x + 1, y, z + 1) +
               fx * fy * (1.f - fz) * value_at(x + 1, y + 1, z) +
               fx * fy * fz * value_at(x + 1, y + 1, z + 1);
    }

    /* SDF::GetGrad(Vector3) (SDF.h:119-136) */
    V3 gradient(V3 p) const
    {
        int x, y, z; float fx, fy, fz;
        coords(p, x, y, z, fx, fy, fz);
        if (out(x, y, z)) return v3(0, 0, 0);
        return (1.f - fx) * (1.f - fy) * (1.f - fz) * grad_at(x, y, z) +
               (1.f - fx) * (1.f - fy) * fz * grad_at(x, y, z + 1) +
               (1.f - fx) * fy * (1.f - fz) * grad_at(x, y + 1, z) +
               (1.f - fx) * fy * fz * grad_at(x, y + 1, z + 1) +
               fx * (1.f - fy) * (1.f - fz) * grad_at(x + 1, y, z) +
               fx * (1.f - fy) * fz * grad_at(x + 1, y, z + 1) +
               fx * fy * (1.f - fz) * grad_at(x + 1, y + 1, z) +
               fx * fy * fz * grad_at(x + 1, y + 1, z + 1);
    }
};

/* ---------------------------------------------------------- cloth state */
struct Tri /* Physics/ClothTypes.h:37-62 (solver fields) */
{
    u32 i1, i2, i3;
    float du1, du2, dv1, dv2, det, invDet, lu0, lv0, lu2, lv2, area;
};
struct Bend { u32 i1, i2, i3, i4; };

struct VContact { int idx, feature, mesh; V3 point, normal; float depth, lambda, lambdaF; };
/* item: the cloth triangle / edge; slot: the collider's index among the sphere,
   mesh and SDF colliders (for the static contact colouring of check mode) */
struct TContact { u32 i1, i2, i3; int feature, mesh; V3 point, normal; float w1, w2, w3, lambda, lambdaF; int item = -1, slot = 0; };
struct EContact { u32 i1, i2; int feature, mesh; V3 point, normal; float w1, w2, lambda, lambdaF; int item = -1, slot = 0; };
struct SContact { u32 i1, i2, i3, i4; V3 normal; float w1, w2, w3, side, lambda, lambdaF, error; };

struct Collider
{
    int type; /* 1 walls, 3 sphere, 4 mesh, 7 sdf (Physics/Common.h:20-29) */
    Box walls;
    V3 center;
    float radius;
    int sdf = -1, mesh = -1;
};

struct Cloth
{
    /* parameters, defaults as Physics/ClothModel.cpp:10-36 */
    float unit = 10, thickness = 0.3f, tolerance = 0.2f, shear = 5e8f, bendStiff = 5.f, stretch = 2e10f;
    float poisson = 0.5f, friction = 0.4f, drag = 1.f, selfShrink = 0.9f, selfThreshold = 0.003f, area = 10.f;
    int iterations = 50, substeps = 1, flags = 0, bendFreq = 2;
    bool fem = false, dihedral = true;
    bool ccd = false;

    int N = 0;
    std::vector<V3> pos, prev, vel;
    std::vector<float> invMass;
    std::vector<V3> uv;
    std::vector<Tri> tris;
    std::vector<Bend> bends;
    struct Link { u32 i1, i2; float len, stiffness; };   /* Physics/ClothTypes.h:94-99 */
    std::vector<Link> links;
    Topo mesh, prevMesh;

    std::vector<int> triOrder, bendOrder, linkOrder;
    int contactOrder = 0;

    std::vector<Collider> colliders;
    std::vector<std::unique_ptr<GridSDF>> sdfs;
    std::vector<std::unique_ptr<MeshCollider>> meshes;

    std::vector<VContact> contacts;
    std::vector<TContact> triContacts;
    std::vector<EContact> edgeContacts;
    std::vector<SContact> selfTris, selfEdges;
    int lastIterations = 0;

    /* ---- setup ---- */
    /* ClothModel::AddTriangle (Physics/ClothModel.cpp:54-92) */
    void add_triangle(u32 i1, u32 i2, u32 i3)
    {
        Tri t;
        t.i1 = i1; t.i2 = i2; t.i3 = i3;
        float d1x = uv[i2].x - uv[i1].x, d1y = uv[i2].y - uv[i1].y;
        float d2x = uv[i3].x - uv[i1].x, d2y = uv[i3].y - uv[i1].y;
        t.du1 = d1x; t.du2 = d2x; t.dv1 = d1y; t.dv2 = d2y;
        t.det = t.du1 * t.dv2 - t.du2 * t.dv1;
        t.invDet = 0.f;
        if (t.det != 0) t.invDet = 1.f / t.det;
        V3 dx1 = pos[i2] - pos[i1], dx2 = pos[i3] - pos[i1];
        V3 wu = t.invDet * (t.dv2 * dx1 - t.dv1 * dx2);
        V3 wv = t.invDet * (-t.du2 * dx1 + t.du1 * dx2);
        t.lu0 = len(wu);
        t.lv0 = len(wv);
        t.area = 0.5f * t.det;
        t.lu2 = t.lu0 * t.lu0;
        t.lv2 = t.lv0 * t.lv0;
        tris.push_back(t);
    }

    /* ClothModel::AddLink (Physics/ClothModel.inl:12-31): skipped when both ends
       are pinned or the stiffness is zero; rest length from the current positions */
    void add_link(u32 a, u32 b, float stiff)
    {
        if (invMass[a] == 0 && invMass[b] == 0) return;
        if (stiff == 0) return;
        Link l;
        l.i1 = a; l.i2 = b; l.stiffness = stiff;
        l.len = len(pos[a] - pos[b]);
        links.push_back(l);
    }

    /* ClothPatch::Init(grid) (Physics/ClothPatch.cpp:135-246): positions, uv,
       links (stretch, shear and, without dihedral bending, bend links) in the
       reference's creation order, alternating-diagonal triangles, pins, edges
       and bends. */
    void init_grid(int divX, int divY, float inc, V3 offset, bool horizontal, bool attached)
    {
        N = divX * divY;
        pos.assign(N, v3(0, 0, 0)); prev.assign(N, v3(0, 0, 0)); vel.assign(N, v3(0, 0, 0));
        invMass.assign(N, 1.f); uv.assign(N, v3(0, 0, 0));
        tris.clear(); bends.clear(); links.clear();
        mesh = Topo();
        float x = -0.5f * divX * inc;
        const float startY = x;
        std::vector<u32> idxs;
        for (int j = 0, base = 0; j < divX; j++, base += divY)
        {
            pos[base] = v3(x, 0, startY) + offset;
            if (!horizontal) pos[base] = v3(x, startY, 0) + offset;
            prev[base] = pos[base];
            uv[base] = v3(x, 0, 0);
            if (base >= divY)
            {
                add_link(base - divY, base, stretch);
                add_link(base - divY + 1, base, shear);
                if (base >= 2 * divY && !dihedral) add_link(base - 2 * divY, base, bendStiff);
            }
            for (int i = 1; i < divY; i++)
            {
                int idx = base + i;
                if (horizontal) pos[idx] = v3(x, 0, startY + inc * i) + offset;
                else pos[idx] = v3(x, startY + inc * i, 0) + offset; /* incline unsupported */
                prev[idx] = pos[idx];
                uv[idx] = v3(x, inc * i, 0);
                add_link(idx - 1, idx, stretch);
                if (idx > base + 1 && !dihedral) add_link(idx - 2, idx, bendStiff);
                if (idx >= divY)
                {
                    add_link(idx - divY, idx, stretch);
                    if (i < divY - 1) add_link(idx - divY + 1, idx, shear);
                    if (j > 1 && !dihedral) add_link(idx - 2 * divY, idx, bendStiff);
                }
                if (idx > divY) add_link(idx - divY - 1, idx, shear);
                if (idx > base && idx > divY)
                {
                    u32 a = idx - divY - 1, b = idx - divY, c = idx, d = idx - 1;
                    if ((i & 1) == (j & 1))
                    {
                        add_triangle(a, c, b); add_triangle(a, d, c);
                        u32 t[6] = {a, c, b, a, d, c};
                        idxs.insert(idxs.end(), t, t + 6);
                    }
                    else
                    {
                        add_triangle(b, d, c); add_triangle(d, b, a);
                        u32 t[6] = {b, d, c, d, b, a};
                        idxs.insert(idxs.end(), t, t + 6);
                    }
                }
            }
            if (attached && (j == 0 || j == divX - 1)) invMass[base + divY - 1] = 0.f;
            x += inc;
        }
        mesh.verts = pos;
        mesh.idx = idxs;
        mesh.compute_normals();
        mesh.construct_edges();
        mesh.construct_rings(true, true);
        /* ClothModel::AddBendConstraint (Physics/ClothModel.cpp:94-126) */
        for (const Edge& e : mesh.edges)
        {
            if (e.t2 < 0) continue;
            auto opp = [&](int t) {
                const Tri& tr = tris[t];
                if (tr.i1 != e.i1 && tr.i1 != e.i2) return tr.i1;
                if (tr.i2 != e.i1 && tr.i2 != e.i2) return tr.i2;
                return tr.i3;
            };
            Bend b;
            b.i1 = e.i1; b.i2 = e.i2; b.i3 = opp(e.t1); b.i4 = opp(e.t2);
            bends.push_back(b);
        }
        prevMesh = mesh;
    }

    /* ---- step ---- */
    /* ClothModelPBD::Step predict (Physics/ClothPBD.cpp:257-266) */
    void predict(float h)
    {
        for (int i = 0; i < N; i++)
        {
            prev[i] = pos[i];
            if (invMass[i] == 0) continue;
            vel[i] += h * kGravity * unit;
            vel[i] = vel[i] * drag;
            pos[i] += h * vel[i];
        }
    }

    /* ClothModel::WallCollisions (Physics/ClothCollision.cpp:199-220) */
    void wall_collisions(const Box& w)
    {
        const float r = thickness + tolerance;
        for (int i = 0; i < N; i++)
        {
            V3 p = pos[i];
            if (p.y - r <= w.mn.y) add_contact(i, v3(p.x, w.mn.y, p.z), v3(0, 1, 0), -1, -1);
            if (p.x - r <= w.mn.x) add_contact(i, v3(w.mn.x, p.y, p.z), v3(1, 0, 0), -1, -1);
            if (p.x + r >= w.mx.x) add_contact(i, v3(w.mx.x, p.y, p.z), v3(-1, 0, 0), -1, -1);
            if (p.z - r <= w.mn.z) add_contact(i, v3(p.x, p.y, w.mn.z), v3(0, 0, 1), -1, -1);
            if (p.z + r >= w.mx.z) add_contact(i, v3(p.x, p.y, w.mx.z), v3(0, 0, -1), -1, -1);
        }
    }

    /* ClothModel::AddContact (Physics/ClothModel.inl:31-45) */
    void add_contact(int idx, V3 p, V3 n, int feature, int meshId)
    {
        VContact c;
        c.idx = idx; c.point = p; c.normal = n; c.feature = feature; c.mesh = meshId;
        c.depth = thickness - dot(n, pos[idx] - p);
        c.lambda = 0; c.lambdaF = 0;
        contacts.push_back(c);
    }

    /* SDFCollisions<SphereSDF / GridSDF>, vertex, edge and triangle parts with
       handleInside = handleCurrent = handleBorder = false
       (Physics/ClothCollision.cpp:430-580; SphereSDF/GridSDF in
       Physics/ClothCollisionSDF.h:8-55,124-206) */
    void sdf_collisions(const Collider& col, int slot)
    {
        const GridSDF* g = col.type == 7 ? sdfs[col.sdf].get() : nullptr;
        auto queryPoint = [&](V3 p, V3& cp, V3& n, int& feature) -> float {
            if (g)
            {
                float v = g->value(p);
                V3 gr = normalized(g->gradient(p));
                n = gr;
                cp = p - v * gr;
                feature = -3;
                return v;
            }
            V3 delta = p - col.center;
            float l = len(delta);
            delta = (1.f / l) * delta;
            n = delta;
            cp = col.center + col.radius * delta;
            feature = -1;
            return l - col.radius;
        };
        if (flags & CF_VERTICES)
        {
            for (int i = 0; i < N; i++)
            {
                V3 p, n;
                int feature = -1;
                float dist = queryPoint(prev[i], p, n, feature);
                float tv = len(prev[i] - pos[i]);
                float radTol = thickness + std::max(tolerance, tv * 1.1f);
                if (dist < radTol && dist >= 0) add_contact(i, p, n, feature, -1);
            }
        }
        bool handleBorder = (flags & CF_VERTICES) == 0;
        if (flags & CF_EDGES)
        {
            float eps = 0.02f;
            for (size_t i = 0; i < mesh.edges.size(); i++)
            {
                u32 i1 = mesh.edges[i].i1, i2 = mesh.edges[i].i2;
                V3 p = prev[i1], q = prev[i2];
                float c0 = 0, c1 = 0;
                V3 cp = v3(0, 0, 0), n = v3(0, 0, 0);
                float dist;
                if (g)
                    dist = 0; /* GridSDF::QuerySegment is a stub (ClothCollisionSDF.h:141-146) */
                else
                {
                    float t;
                    V3 ps = closest_pt_segm(col.center, p, q, t);
                    V3 delta = ps - col.center;
                    float l = len(delta);
                    delta = (1.f / l) * delta;
                    n = delta;
                    cp = col.center + col.radius * delta;
                    c0 = 1.0f - t; c1 = t;
                    dist = l - col.radius;
                }
                float tv = std::max(len(prev[i1] - pos[i1]), len(prev[i2] - pos[i2]));
                float radTol = thickness + std::max(tolerance, tv * 1.1f);
                if (dist < radTol && dist >= 0 && ((c0 > eps && c0 < 1.f - eps && c1 > eps && c1 < 1.f - eps) || handleBorder))
                {
                    EContact c;
                    c.i1 = i1; c.i2 = i2; c.point = cp; c.normal = n; c.w1 = c0; c.w2 = c1;
                    c.feature = -1; c.mesh = -1; c.lambda = c.lambdaF = 0;
                    c.item = (int)i; c.slot = slot;
                    edgeContacts.push_back(c);
                }
            }
        }
        handleBorder |= (flags & CF_EDGES) == 0;
        if (flags & CF_TRIANGLES)
        {
            float eps = 0.001f;
            for (size_t i = 0; i < tris.size(); i++)
            {
                u32 i1 = tris[i].i1, i2 = tris[i].i2, i3 = tris[i].i3;
                V3 a = prev[i1], b = prev[i2], c = prev[i3];
                V3 cp, n, coords;
                float dist;
                if (g)
                {
                    dist = grid_query_triangle(*g, a, b, c, cp, n, coords);
                }
                else
                {
                    V3 pt;
                    closest_pt_point_triangle(col.center, a, b, c, pt, coords);
                    V3 delta = pt - col.center;
                    float l = len(delta);
                    delta = (1.f / l) * delta;
                    n = delta;
                    cp = col.center + col.radius * delta;
                    dist = l - col.radius;
                }
                float tv = std::max(len(prev[i1] - pos[i1]), std::max(len(prev[i2] - pos[i2]), len(prev[i3] - pos[i3])));
                float radTol = thickness + std::max(tolerance, tv * 1.1f);
                if (dist < radTol && dist >= 0 && ((coords.x > eps && coords.y > eps && coords.z > eps) || handleBorder))
                {
                    TContact t;
                    t.i1 = i1; t.i2 = i2; t.i3 = i3; t.point = cp; t.normal = n;
                    t.w1 = coords.x; t.w2 = coords.y; t.w3 = coords.z;
                    t.feature = -1; t.mesh = -1; t.lambda = t.lambdaF = 0;
                    t.item = (int)i; t.slot = slot;
                    triContacts.push_back(t);
                }
            }
        }
    }

    /* GridSDF::QueryTriangle, Frank-Wolfe (Physics/ClothCollisionSDF.h:148-205) */
    static float grid_query_triangle(const GridSDF& g, V3 a, V3 b, V3 c, V3& cp_out, V3& n, V3& coords)
    {
        V3 cp = 0.33f * (a + b + c);
        float distOld = 0;
        for (int i = 1; i < 100; i++)
        {
            float dist = g.value(cp);
            if (dist == FLT_MAX) return FLT_MAX;
            V3 gr = g.gradient(cp);
            float dA = dot(a, gr), dB = dot(b, gr), dC = dot(c, gr);
            float d = dA;
            V3 s = a;
            if (dB < d) { d = dB; s = b; }
            if (dC < d) { d = dC; s = c; }
            if (distOld > 0)
            {
                float rel = std::fabs(distOld - dist) / distOld;
                if (rel < 0.0001f) break;
            }
            distOld = dist;
            float alpha = 2.f / (i + 2.f);
            cp += alpha * (s - cp);
        }
        float v = g.value(cp);
        V3 gr = normalized(g.gradient(cp));
        n = gr;
        cp_out = cp - v * gr;
        coords = barycentric(a, b, c, cp);
        return v;
    }

    /* ClothModel::MeshCollisions against a static triangle mesh
       (Physics/ClothCollision.cpp:89-197 with
       MeshClosestPoints::ClosestPoints(mesh1, mesh2, tree, r, false),
       Geometry/ClosestPointsBetweenMeshes.cpp:595-695) */
    void mesh_collisions(int meshId, float radTol, const std::vector<float>& tvs, int slot)
    {
        /* The queries are independent (const tree walks); they run in parallel
           and their results are appended in query order, as the serial loops do. */
        MeshCollider& mc = *meshes[meshId];
        if (!mc.built) mc.build(thickness);
        const Topo& cm = prevMesh;
        if (flags & CF_VERTICES)
        {
            std::vector<TriInfo> res(N);
#pragma omp parallel for schedule(dynamic, 64)
            for (int i = 0; i < N; i++)
            {
                float minDist = FLT_MAX;
                mc.point_rec(cm.verts[i], 0, minDist, res[i]);
            }
            for (int i = 0; i < N; i++)
            {
                const TriInfo& info = res[i];
                float dist = info.distance;
                if (dist < radTol && dist >= 0) add_contact(i, info.cp, info.normal, info.tri, meshId);
            }
        }
        if (flags & CF_TRIANGLES)
        {
            const int nt = (int)tris.size();
            std::vector<VtxInfo> res(nt);
#pragma omp parallel for schedule(dynamic, 64)
            for (int j = 0; j < nt; j++)
            {
                u32 a = cm.idx[j * 3], b = cm.idx[j * 3 + 1], c = cm.idx[j * 3 + 2];
                float minDist = FLT_MAX;
                mc.tri_rec(cm.verts[a], cm.verts[b], cm.verts[c], 0, minDist, res[j]);
            }
            for (int j = 0; j < nt; j++)
            {
                const VtxInfo& info = res[j];
                u32 i1 = tris[j].i1, i2 = tris[j].i2, i3 = tris[j].i3;
                float tv = std::max(tvs[i1], std::max(tvs[i2], tvs[i3]));
                float rt = thickness + std::max(tolerance, tv * 1.2f);
                float dist = info.distance;
                if (dist < rt && dist >= 0)
                {
                    TContact t;
                    t.i1 = i1; t.i2 = i2; t.i3 = i3; t.point = info.cpMesh; t.normal = info.normal;
                    t.w1 = info.bary.x; t.w2 = info.bary.y; t.w3 = info.bary.z;
                    t.feature = info.vertex; t.mesh = meshId; t.lambda = t.lambdaF = 0;
                    t.item = j; t.slot = slot;
                    triContacts.push_back(t);
                }
            }
        }
        if (flags & CF_EDGES)
        {
            const int ne = (int)cm.edges.size();
            std::vector<EdgeInfo> res(ne);
#pragma omp parallel for schedule(dynamic, 64)
            for (int e = 0; e < ne; e++)
            {
                res[e].edge1 = e;
                float minDist = FLT_MAX;
                mc.seg_rec(cm.verts[cm.edges[e].i1], cm.verts[cm.edges[e].i2], 0, minDist, res[e]);
            }
            for (int e = 0; e < ne; e++)
            {
                const EdgeInfo& info = res[e];
                float dist = info.distance;
                if (dist < radTol && dist >= 0)
                {
                    EContact c;
                    c.i1 = mesh.edges[e].i1; c.i2 = mesh.edges[e].i2; c.point = info.cpMesh; c.normal = info.normal;
                    c.w1 = info.cs[0]; c.w2 = info.cs[1]; c.feature = info.edge; c.mesh = meshId;
                    c.lambda = c.lambdaF = 0;
                    c.item = e; c.slot = slot;
                    edgeContacts.push_back(c);
                }
            }
        }
    }

    /* MeshCollisions(prevMesh, tree, V|E) with the brute-force self query
       MeshClosestPoints::ClosestPoints(mesh, tree, radTol)
       (Physics/ClothCollision.cpp:41-47,89-197;
       Geometry/ClosestPointsBetweenMeshes.cpp:538-592) */
    void self_collisions(float radTol)
    {
        const Topo& m = prevMesh;
        for (int i = 0; i < N; i++)
        {
            std::vector<TriInfo> res;
            closest_points_on_mesh_to_point(m.verts[i], m, res, radTol, i);
            for (TriInfo& r : res)
            {
                r.vtx = i;
                if (r.tri >= 0 && !check_adjacency(m, i, r.tri, r.region))
                {
                    float dist = r.distance;
                    if (dist < radTol && dist >= 0)
                    {
                        SContact c;
                        c.i1 = m.idx[r.tri * 3]; c.i2 = m.idx[r.tri * 3 + 1]; c.i3 = m.idx[r.tri * 3 + 2]; c.i4 = i;
                        c.normal = r.normal; c.w1 = r.bary.x; c.w2 = r.bary.y; c.w3 = r.bary.z; c.side = r.side;
                        c.lambda = c.lambdaF = 0; c.error = 0;
                        selfTris.push_back(c);
                    }
                }
            }
        }
        for (int i = 0; i < (int)m.edges.size(); i++)
        {
            const Edge& e1 = m.edges[i];
            EdgeInfo info;
            info.edge1 = i;
            closest_edge_to_segment_self(m.verts[e1.i1], m.verts[e1.i2], m, info, i);
            if (!check_edge_adjacency(info, m, e1.i1, e1.i2, e1))
            {
                float dist = info.distance;
                if (dist < radTol && dist >= 0)
                {
                    const Edge& e2 = m.edges[info.edge];
                    SContact c;
                    c.i1 = e1.i1; c.i2 = e1.i2; c.i3 = e2.i1; c.i4 = e2.i2;
                    c.w1 = info.cs[1]; c.w2 = info.cm[1]; c.w3 = 0; c.normal = info.normal; c.side = info.side;
                    c.lambda = c.lambdaF = 0; c.error = 0;
                    selfEdges.push_back(c);
                }
            }
        }
    }

    /* ClothModel::DetectCollisions (Physics/ClothCollision.cpp:17-48) */
    void detect(bool runCCD)
    {
        for (int i = 0; i < N; i++) prevMesh.verts[i] = prev[i];
        contacts.clear(); triContacts.clear(); edgeContacts.clear();
        std::vector<float> tvs(N);
        float maxTv = 0;
        for (int i = 0; i < N; i++)
        {
            tvs[i] = len(pos[i] - prev[i]);
            if (tvs[i] > maxTv) maxTv = tvs[i];
        }
        float radTol = thickness + std::max(tolerance, maxTv * 1.5f);
        int slot = 0;
        for (size_t c = 0; c < colliders.size(); c++)
        {
            const Collider& col = colliders[c];
            if (col.type == 1 && (flags & CF_WALLS)) wall_collisions(col.walls);
            else if (col.type == 3 || col.type == 7) sdf_collisions(col, slot++);
            else if (col.type == 4) mesh_collisions(col.mesh, radTol, tvs, slot++);
        }
        if (flags & CF_SELF)
        {
            selfTris.clear();
            selfEdges.clear();
            self_collisions(radTol);
        }
        if (runCCD) ccd_detect();
    }

    /* ---- solver ---- */
    /* SolveLinks (Physics/ClothPBD.cpp:9-50) for one link; returns |s err| or -1 */
    float solve_link(const Link& link, float k, float omega)
    {
        const float w1 = invMass[link.i1], w2 = invMass[link.i2];
        if (w1 + w2 == 0) return -1;
        const float mu = 1.f / (w1 + w2);
        V3 delta = pos[link.i1] - pos[link.i2];
        const float len0 = link.len;
        const float l = len(delta);
        if (l == 0 || std::isnan(l) || std::isinf(l)) return -1;
        const float err = l - len0;
        delta = (1 / l) * delta;
        const float epsilon = len0 / (k * link.stiffness);
        const float s = 1.f / (1.f + mu * epsilon);
        const float lambda = err * mu * s;
        const V3 fc = omega * lambda * delta;
        pos[link.i1] = pos[link.i1] - w1 * fc;
        pos[link.i2] = pos[link.i2] + w2 * fc;
        return std::fabs(s * err);
    }

    /* SolveTriangles (Physics/ClothPBD.cpp:52-108) for one triangle */
    void solve_triangle(const Tri& tri, float h2, float epsUV)
    {
        V3& x1 = pos[tri.i1]; V3& x2 = pos[tri.i2]; V3& x3 = pos[tri.i3];
        float w1 = invMass[tri.i1], w2 = invMass[tri.i2], w3 = invMass[tri.i3];
        V3 dx1 = x2 - x1, dx2 = x3 - x1;
        V3 wu = tri.invDet * (tri.dv2 * dx1 - tri.dv1 * dx2);
        V3 wv = tri.invDet * (-tri.du2 * dx1 + tri.du1 * dx2);
        float err, diag, lambda;
        V3 q1, q2, q3;
        q2 = (tri.invDet * tri.dv2) * wu;
        q3 = (-tri.invDet * tri.dv1) * wu;
        q1 = -q2 - q3;
        diag = dot(w1 * q1, q1) + dot(w2 * q2, q2) + dot(w3 * q3, q3);
        err = 0.5f * (dot(wu, wu) - tri.lu2);
        lambda = -err / diag;
        x1 += (w1 * lambda) * q1; x2 += (w2 * lambda) * q2; x3 += (w3 * lambda) * q3;

        q2 = (-tri.invDet * tri.du2) * wv;
        q3 = (tri.invDet * tri.du1) * wv;
        q1 = -q2 - q3;
        diag = dot(w1 * q1, q1) + dot(w2 * q2, q2) + dot(w3 * q3, q3);
        err = 0.5f * (dot(wv, wv) - tri.lv2);
        lambda = -err / diag;
        x1 += (w1 * lambda) * q1; x2 += (w2 * lambda) * q2; x3 += (w3 * lambda) * q3;

        q2 = tri.dv2 * wv - tri.du2 * wu;
        q3 = -tri.dv1 * wv + tri.du1 * wu;
        q1 = -q2 - q3;
        diag = tri.invDet * (dot(w1 * q1, q1) + dot(w2 * q2, q2) + dot(w3 * q3, q3));
        err = dot(wu, wv);
        float s = 1.f / (1.f + tri.lu0 * tri.lv0 * epsUV / (diag * h2 * tri.area));
        lambda = -s * err / diag;
        x1 += (w1 * lambda) * q1; x2 += (w2 * lambda) * q2; x3 += (w3 * lambda) * q3;
    }

    /* SolveBends + EvaluateAngle + EvaluateGradient for one bend
       (Physics/ClothPBD.cpp:110-224); returns |error| or -1 when skipped */
    float solve_bend(const Bend& bc)
    {
        V3 x1 = pos[bc.i1], x2 = pos[bc.i2], x3 = pos[bc.i3], x4 = pos[bc.i4];
        float m1 = invMass[bc.i1], m2 = invMass[bc.i2], m3 = invMass[bc.i3], m4 = invMass[bc.i4];
        if (m1 + m2 + m3 + m4 == 0) return -1;
        /* EvaluateAngle */
        V3 x12 = x2 - x1;
        float l = len(x12);
        V3 x13 = x3 - x1;
        V3 n1 = cross(x12, x13);
        float l1 = len(n1);
        V3 x14 = x4 - x1;
        V3 n2 = cross(x14, x12);
        float l2 = len(n2);
        float cosine, theta;
        if (l1 == 0 || l2 == 0) { cosine = 1; theta = 0; }
        else
        {
            float il1 = 1.f / l1, il2 = 1.f / l2;
            cosine = dot(il1 * n1, il2 * n2);
            cosine = std::min(1.f, std::max(-1.f, cosine));
            theta = step_acos(cosine);
        }
        if (std::fabs(cosine) >= 1 - 0.001f) return -1;
        /* EvaluateGradient (recomputes the same quantities) */
        float h1 = l1 / l, h2 = l2 / l;
        float he = 0.5f * (h1 + h2);
        float il1 = 1.f / l1, il2 = 1.f / l2;
        V3 n1n = il1 * n1, n2n = il2 * n2;
        V3 n1p = n1n - n2n * cosine;
        V3 n2p = n2n - n1n * cosine;
        float sine = std::sqrt(1 - cosine * cosine);
        V3 q3 = (il1 / sine / he) * cross(x12, n2p);
        V3 q4 = (-il2 / sine / he) * cross(x12, n1p);
        V3 q2 = (-il1 / sine / he) * cross(x13, n2p) + (il2 / sine / he) * cross(x14, n1p);
        V3 q1 = -q2 - q3 - q4;
        float diag = m1 * lensq(q1) + m2 * lensq(q2) + m3 * lensq(q3) + m4 * lensq(q4);
        if (diag == 0) return -1;
        float s = 0.0005f * bendStiff;
        float e = s * theta;
        float lambda = -s * theta / he / diag;
        pos[bc.i1] += (lambda * m1) * q1;
        pos[bc.i2] += (lambda * m2) * q2;
        pos[bc.i3] += (lambda * m3) * q3;
        pos[bc.i4] += (lambda * m4) * q4;
        return std::fabs(e);
    }

    /* ComputeTriangleNormal(mesh, tri, coords, usePseudoNormal = false)
       (Geometry/ClosestPointOnMesh.cpp:37-97) */
    V3 interpolated_normal(const Topo& m, int tri, V3 c) const
    {
        V3 n0 = m.normals[m.idx[tri * 3]], n1 = m.normals[m.idx[tri * 3 + 1]], n2 = m.normals[m.idx[tri * 3 + 2]];
        return normalized(c.x * n0 + c.y * n1 + c.z * n2);
    }

    /* ClothCollisionHandler::SolveContactsPosition for one contact
       (Physics/ClothCollisionHandler.cpp:134-202) */
    float solve_vertex_contact(VContact& c, float invH, float mu)
    {
        V3& p = pos[c.idx];
        if (c.mesh >= 0)
        {
            const Topo& m = meshes[c.mesh]->m;
            int t = c.feature;
            V3 coords, cp;
            closest_pt_point_triangle(p, m.verts[m.idx[t * 3]], m.verts[m.idx[t * 3 + 1]], m.verts[m.idx[t * 3 + 2]], cp, coords);
            c.point = cp;
            c.normal = interpolated_normal(m, t, coords);
        }
        V3 delta = p - c.point;
        float l = dot(delta, c.normal);
        V3 disp = c.normal;
        if (l > thickness) return -1;
        float depth = thickness - l;
        float dLambda = depth;
        c.lambda += dLambda;
        disp = disp * dLambda;
        V3 v12 = p - prev[c.idx] - v3(0, 0, 0);
        float vnrel = dot(c.normal, v12);
        V3 vt = v12 - vnrel * c.normal;
        float vtrel = len(vt);
        const float limit = mu * c.lambda;
        if (vtrel > 0.001f)
        {
            float dLambdaF = vtrel;
            float l0 = c.lambdaF;
            c.lambdaF = l0 + dLambdaF;
            if (c.lambdaF >= limit) c.lambdaF = limit;
            dLambdaF = c.lambdaF - l0;
            vt = vt * (1.0f / vtrel);
            disp += -dLambdaF * vt;
        }
        p += disp;
        vel[c.idx] += invH * disp;
        return std::fabs(depth);
    }

    /* SolveTriContacts for one contact (Physics/ClothCollisionHandler.cpp:204-287) */
    float solve_tri_contact(TContact& c, float mu)
    {
        V3& x1 = pos[c.i1]; V3& x2 = pos[c.i2]; V3& x3 = pos[c.i3];
        float m1 = invMass[c.i1], m2 = invMass[c.i2], m3 = invMass[c.i3];
        V3 coords, p;
        closest_pt_point_triangle(c.point, x1, x2, x3, p, coords);
        c.w1 = coords.x; c.w2 = coords.y; c.w3 = coords.z;
        V3 n = normalized(-cross(x2 - x1, x3 - x1));
        c.normal = n;
        if (c.mesh >= 0 && c.feature >= 0)
        {
            V3 mn = meshes[c.mesh]->m.normals[c.feature];
            if (dot(n, mn) < 0) c.normal = -n;
        }
        float len0 = thickness;
        float l = dot(c.normal, p - c.point - v3(0, 0, 0));
        if (l > len0) return -1;
        float s = 1.f / (c.w1 * c.w1 / m1 + c.w2 * c.w2 / m2 + c.w3 * c.w3 / m3);
        float depth = len0 - l;
        float dLambda = s * depth;
        c.lambda += dLambda;
        V3 disp = dLambda * c.normal;
        if (mu != 0)
        {
            V3 p0 = c.w1 * prev[c.i1] + c.w2 * prev[c.i2] + c.w3 * prev[c.i3];
            V3 v12 = p - p0 - v3(0, 0, 0);
            float vnrel = dot(c.normal, v12);
            V3 vt = v12 - vnrel * c.normal;
            float vtrel = len(vt);
            const float limit = mu * c.lambda;
            if (vtrel > 0.001f)
            {
                float l0 = c.lambdaF;
                c.lambdaF = l0 + vtrel;
                if (c.lambdaF >= limit) c.lambdaF = limit;
                dLambda = c.lambdaF - l0;
                vt = vt * (1.f / vtrel);
                V3 pp = -s * dLambda * vt;
                x1 += pp * (c.w1 * m1); x2 += pp * (c.w2 * m2); x3 += pp * (c.w3 * m3);
            }
        }
        x1 += disp * (c.w1 * m1); x2 += disp * (c.w2 * m2); x3 += disp * (c.w3 * m3);
        return depth;
    }

    /* SolveEdgeContacts for one contact (Physics/ClothCollisionHandler.cpp:289-362) */
    float solve_edge_contact(EContact& c, float mu)
    {
        V3& x1 = pos[c.i1]; V3& x2 = pos[c.i2];
        float m1 = invMass[c.i1], m2 = invMass[c.i2];
        V3 p = c.w1 * x1 + c.w2 * x2;
        if (c.mesh >= 0)
        {
            const Topo& m = meshes[c.mesh]->m;
            float s1, t;
            V3 a = m.verts[m.edges[c.feature].i1], b = m.verts[m.edges[c.feature].i2];
            closest_pt_segm_segm(a, b, x1, x2, s1, t, c.point, p);
            c.w1 = 1.0f - t;
            c.w2 = t;
        }
        float len0 = thickness;
        float l = dot(c.normal, p - c.point - v3(0, 0, 0));
        if (l > len0) return -1;
        float s = 1.f / (c.w1 * c.w1 / m1 + c.w2 * c.w2 / m2);
        float depth = len0 - l;
        float dLambda = s * depth;
        c.lambda += dLambda;
        V3 disp = dLambda * c.normal;
        if (mu != 0)
        {
            V3 p0 = c.w1 * prev[c.i1] + c.w2 * prev[c.i2];
            V3 v12 = p - p0 - v3(0, 0, 0);
            float vnrel = dot(c.normal, v12);
            V3 vt = v12 - vnrel * c.normal;
            float vtrel = len(vt);
            const float limit = mu * c.lambda;
            if (vtrel > 0.001f)
            {
                float l0 = c.lambdaF;
                c.lambdaF = l0 + vtrel;
                if (c.lambdaF >= limit) c.lambdaF = limit;
                dLambda = c.lambdaF - l0;
                vt = vt * (1.f / vtrel);
                V3 pp = -s * dLambda * vt;
                x1 += pp * (c.w1 * m1); x2 += pp * (c.w2 * m2);
            }
        }
        x1 += disp * (c.w1 * m1); x2 += disp * (c.w2 * m2);
        return depth;
    }

    /* SolveSelfTrisPosition for one contact (Physics/ClothCollisionHandler.cpp:364-450) */
    float solve_self_tri(SContact& c, float h)
    {
        const float soften = .9f;
        float len0 = thickness * selfShrink;
        V3& x1 = pos[c.i1]; V3& x2 = pos[c.i2]; V3& x3 = pos[c.i3]; V3& x4 = pos[c.i4];
        float m1 = invMass[c.i1], m2 = invMass[c.i2], m3 = invMass[c.i3], m4 = invMass[c.i4];
        V3 p, coords;
        closest_pt_point_triangle(x4, x1, x2, x3, p, coords);
        c.w1 = coords.x; c.w2 = coords.y; c.w3 = coords.z;
        V3 delta = x4 - p;
        V3 n = normalized(cross(x2 - x1, x3 - x1));
        float side = signed_volume(x4, x1, x2, x3);
        if (c.side * side <= 0) len0 = thickness * 0.1f;
        if (dot(n, c.normal) < 0) n = -n;
        float l = dot(n, delta);
        if (l > len0) return -1;
        float im = c.w1 * c.w1 * m1 + c.w2 * c.w2 * m2 + c.w3 * c.w3 * m3 + m4;
        float s = 1.f / im;
        float err = l - len0;
        c.error = err;
        float absErr = std::max(0.f, -err);
        float dLambda = soften * s * err;
        V3 disp = dLambda * n;
        c.lambda += -dLambda / h;
        x1 += disp * (c.w1 * m1);
        x2 += disp * (c.w2 * m2);
        x3 += disp * (c.w3 * m3);
        x4 -= disp * m4;
        return absErr;
    }

    /* SolveSelfEdgesPosition for one contact (Physics/ClothCollisionHandler.cpp:453-542) */
    float solve_self_edge(SContact& c, float h)
    {
        float thick = thickness * selfShrink;
        const float soften = 0.9f;
        V3& x1 = pos[c.i1]; V3& x2 = pos[c.i2]; V3& x3 = pos[c.i3]; V3& x4 = pos[c.i4];
        float m1 = invMass[c.i1], m2 = invMass[c.i2], m3 = invMass[c.i3], m4 = invMass[c.i4];
        float side = signed_volume(x1, x2, x3, x4);
        V3 p, q;
        float t1, t2;
        closest_pt_segm_segm(x1, x2, x3, x4, t1, t2, p, q);
        c.w1 = 1 - t1;
        c.w2 = 1 - t2;
        float omw1 = 1.f - c.w1, omw2 = 1.f - c.w2;
        V3 delta = q - p;
        V3 n = normalized(delta);
        if (dot(n, c.normal) < 0.0f) n = -n;
        if (side * c.side < 0) thick = thickness * 0.1f;
        float l = dot(n, delta);
        if (l > thick) return -1;
        float im = c.w1 * c.w1 * m1 + omw1 * omw1 * m2 + c.w2 * c.w2 * m3 + omw2 * omw2 * m4;
        float s = 1.f / im;
        float err = l - thick;
        c.error = err;
        float absErr = std::max(0.f, -err);
        float dLambda = -soften * s * err;
        c.lambda += dLambda / h;
        V3 disp = dLambda * n;
        x1 -= disp * (omw1 * m1);
        x2 -= disp * (c.w1 * m2);
        x3 += disp * (omw2 * m3);
        x4 += disp * (c.w2 * m4);
        return absErr;
    }

    /* Deterministic independent-set colouring used by the GPU for contacts that
       touch several particles: a contact joins the current colour when its key
       (a hash of its particle indices, then its list index) is the smallest among
       the still uncoloured contacts on each of its particles. Returns the solve
       order (colour, then list index). */
    template <typename C, typename F>
    std::vector<int> colour_order(const std::vector<C>& list, F verts, std::vector<int>* colOut = nullptr) const
    {
        const int n = (int)list.size();
        std::vector<int> colour(n, -1);
        std::vector<uint64_t> key(n), minKey(N);
        for (int i = 0; i < n; i++)
        {
            u32 vs[4]; int nv = verts(list[i], vs);
            u32 hsh = 0x9e3779b9U;
            for (int k = 0; k < nv; k++) hsh = contact_hash(hsh ^ vs[k]);
            key[i] = ((uint64_t)hsh << 32) | (u32)i;
        }
        /* at most MAX_ROUNDS rounds; what is left takes the last colour and is
           solved in list order (as the GPU's single-thread fallback does) */
        const int MAX_ROUNDS = 127;
        int remaining = n, round = 0;
        while (remaining > 0 && round < MAX_ROUNDS)
        {
            std::fill(minKey.begin(), minKey.end(), ~0ull);
            for (int i = 0; i < n; i++)
            {
                if (colour[i] >= 0) continue;
                u32 vs[4]; int nv = verts(list[i], vs);
                for (int k = 0; k < nv; k++) minKey[vs[k]] = std::min(minKey[vs[k]], key[i]);
            }
            for (int i = 0; i < n; i++)
            {
                if (colour[i] >= 0) continue;
                u32 vs[4]; int nv = verts(list[i], vs);
                bool ok = true;
                for (int k = 0; k < nv; k++) ok = ok && minKey[vs[k]] == key[i];
                if (ok) colour[i] = round;
            }
            for (int i = 0; i < n; i++) if (colour[i] == round) remaining--;
            round++;
        }
        for (int i = 0; i < n; i++) if (colour[i] < 0) colour[i] = MAX_ROUNDS;
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return colour[a] < colour[b]; });
        if (colOut) *colOut = colour;
        return order;
    }

    /* The GPU's order of triangle / edge collider contacts: by the static colour
       of the contact's cloth triangle / edge, offset by the colour count per
       collider slot (the last colour, 127, is the serial bucket), list order within
       a colour. Without static colours (orc_set_static_colours) the independent-set
       colouring is used. */
    std::vector<int> triColour, edgeColour;
    int nTriColours = 0, nEdgeColours = 0;
    template <typename C>
    std::vector<int> static_order(const std::vector<C>& list, const std::vector<int>& colourOf, int ncol) const
    {
        const int n = (int)list.size();
        std::vector<int> colour(n);
        for (int i = 0; i < n; i++)
        {
            const int it = list[i].item;
            if (colourOf.empty() || it < 0 || it >= (int)colourOf.size()) return colour_order_any(list);
            colour[i] = std::min(colourOf[it] + ncol * list[i].slot, 127);
        }
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return colour[a] < colour[b]; });
        return order;
    }
    std::vector<int> colour_order_any(const std::vector<TContact>& l) const
    {
        return colour_order(l, [](const TContact& c, u32* v) { v[0] = c.i1; v[1] = c.i2; v[2] = c.i3; return 3; });
    }
    std::vector<int> colour_order_any(const std::vector<EContact>& l) const
    {
        return colour_order(l, [](const EContact& c, u32* v) { v[0] = c.i1; v[1] = c.i2; return 2; });
    }

    static u32 contact_hash(u32 x)
    {
        /* "lowbias32" integer finaliser (C. Wellons, public domain) */
        x ^= x >> 16; x *= 0x7feb352dU;
        x ^= x >> 15; x *= 0x846ca68bU;
        x ^= x >> 16;
        return x;
    }

    std::vector<int> seq(size_t n) const { std::vector<int> o(n); for (size_t i = 0; i < n; i++) o[i] = (int)i; return o; }

    /* ClothModelPBD::SolveGS in fixed or early-exit mode (Physics/ClothPBD.cpp:324-369) */
    void solve_gs(float h)
    {
        const float h2 = h * h;
        const float epsUV = 2 * (1 + poisson) / (std::max(shear, 0.1f) * unit * unit);
        const float invH = 1.f / h;
        std::vector<int> tOrd = triOrder.size() == tris.size() ? triOrder : seq(tris.size());
        std::vector<int> bOrd = bendOrder.size() == bends.size() ? bendOrder : seq(bends.size());
        std::vector<int> lOrd = linkOrder.size() == links.size() ? linkOrder : seq(links.size());
        const float kLink = h2 * area * unit;
        auto v3of = [](const SContact& c, u32* v) { v[0] = c.i1; v[1] = c.i2; v[2] = c.i3; v[3] = c.i4; return 4; };
        std::vector<int> stOrd = contactOrder ? colour_order(selfTris, v3of) : seq(selfTris.size());
        std::vector<int> seOrd = contactOrder ? colour_order(selfEdges, v3of) : seq(selfEdges.size());
        std::vector<int> tcOrd = contactOrder ? static_order(triContacts, triColour, nTriColours) : seq(triContacts.size());
        std::vector<int> ecOrd = contactOrder ? static_order(edgeContacts, edgeColour, nEdgeColours) : seq(edgeContacts.size());
        float cl = 0, cb = 0, cv = 0, ce = 0, ct = 0, sct = 0, see = 0;
        int k = 0;
        while (true)
        {
            if (fem)
                for (int t : tOrd) solve_triangle(tris[t], h2, epsUV);
            else
            {
                cl = 0;
                for (int li : lOrd) { float e = solve_link(links[li], kLink, 1.f); if (e > cl) cl = e; }
            }
            if (dihedral && k % bendFreq == 0)
            {
                cb = 0;
                for (int b : bOrd) { float e = solve_bend(bends[b]); if (e > cb) cb = e; }
            }
            cv = 0;
            for (VContact& c : contacts) { float e = solve_vertex_contact(c, invH, friction); if (e > cv) cv = e; }
            ce = 0;
            for (int i : ecOrd) { float e = solve_edge_contact(edgeContacts[i], friction); if (e > ce) ce = e; }
            ct = 0;
            for (int i : tcOrd) { float e = solve_tri_contact(triContacts[i], friction); if (e > ct) ct = e; }
            sct = 0;
            for (int i : stOrd) { float e = solve_self_tri(selfTris[i], h); if (e > sct) sct = e; }
            see = 0;
            for (int i : seOrd) { float e = solve_self_edge(selfEdges[i], h); if (e > see) see = e; }
            k++;
            const float eps = 0.01f;
            if (cl < 0.05f && cb < 0.005f && see < selfThreshold && sct < selfThreshold && cv < eps && ce < eps && ct < eps)
                break;
            if (k >= iterations) break;
        }
        lastIterations = k;
    }

    /* ClothModel::SolverType (Physics/ClothModel.h:23-30): 0 SOLVER_JACOBI,
       1 SOLVER_GAUSS_SEIDEL (default), otherwise SolveCR (Physics/ClothPBD.cpp:293-298) */
    int solver = 1;

    /* ClothModelPBD::SolveJacobi / SolveLinksJacobi (Physics/ClothPBD.cpp:616-661):
       every link's displacement from the same positions, omega 0.5, then applied
       in link order; links only (no FEM, bends or contacts) */
    void solve_jacobi(float h)
    {
        const float h2 = h * h;
        const float k = h2 * area * unit;
        const float omega = 0.5f;
        std::vector<V3> disp(links.size());
        for (int it = 0; it < iterations; ++it)
        {
            for (size_t i = 0; i < links.size(); i++)
            {
                const Link& lk = links[i];
                const float mu = 1.f / (invMass[lk.i1] + invMass[lk.i2]);
                V3 delta = pos[lk.i1] - pos[lk.i2];
                const float len0 = lk.len;
                const float l = len(delta);
                delta = (1 / l) * delta;
                const float err = l - len0;
                const float epsilon = len0 / (k * lk.stiffness);
                const float s = 1.f / (1.f + mu * epsilon);
                const float lambda = err * mu * s;
                disp[i] = (omega * lambda) * delta;
            }
            for (size_t i = 0; i < links.size(); i++)
            {
                const Link& l = links[i];
                pos[l.i1] = pos[l.i1] - invMass[l.i1] * disp[i];
                pos[l.i2] = pos[l.i2] + invMass[l.i2] * disp[i];
            }
        }
        lastIterations = iterations;
    }

    /* ClothModelPBD::SolveCR (Physics/ClothPBD.cpp:371-496) as compiled, with
       SKIP_ALPHA and SKIP_BETA defined: per iteration each link's error and unit
       direction, d = r + beta d with beta = (iter / (iterations - 1))^0.6, and the
       step alpha0 * d along the direction, applied in link order */
    void solve_cr(float h, float alpha0)
    {
        (void)h;
        const size_t nl = links.size();
        if (nl == 0) return;
        std::vector<float> r(nl), d(nl, 0.f);
        std::vector<V3> normal(nl);
        for (int iter = 0; iter < iterations; iter++)
        {
            for (size_t i = 0; i < nl; i++)
            {
                const Link& l = links[i];
                V3 delta = pos[l.i2] - pos[l.i1];
                const float c = (len(delta) - l.len) * l.stiffness * unit;
                const float ln = len(delta);
                delta = (1.f / ln) * delta;
                normal[i] = delta;
                r[i] = -c;
            }
            float beta = (float)iter / (float)(iterations - 1);
            beta = std::pow(beta, 0.6f);
            for (size_t i = 0; i < nl; i++) d[i] = r[i] + beta * d[i];
            const float alpha = alpha0;
            for (size_t i = 0; i < nl; i++)
            {
                const Link& l = links[i];
                const float dLambda = alpha * d[i];
                const V3 disp = dLambda * normal[i];
                pos[l.i1] = pos[l.i1] - invMass[l.i1] * disp;
                pos[l.i2] = pos[l.i2] + invMass[l.i2] * disp;
            }
        }
        lastIterations = iterations;
    }

    void velocity(float h)
    {
        const float invH = 1.f / h;
        for (int i = 0; i < N; i++)
        {
            if (invMass[i] == 0) continue;
            vel[i] = invH * (pos[i] - prev[i]);
        }
    }

    void substep(float h)
    {
        predict(h);
        detect(ccd);
        if (solver == 1) solve_gs(h);
        else if (solver == 0) solve_jacobi(h);
        else solve_cr(h, 0.1f);
        velocity(h);
    }

    /* ClothPatch::UpdateMesh (Physics/ClothPatch.cpp:266-273) */
    void update_mesh()
    {
        for (int i = 0; i < N; i++) mesh.verts[i] = pos[i] + v3(0, 0, 0);
        mesh.compute_normals();
        prevMesh.compute_normals();
    }

    /* ---- continuous self-collision (Physics/SelfCollisionDetector.cpp) ---- */
    void swept_boxes(float tol, std::vector<Box>& tb, std::vector<Box>& vb, std::vector<Box>& eb) const
    {
        /* box construction of ClothModel::ComputeTree (Physics/ClothCollision.cpp:256-321) */
        tb.resize(tris.size());
        for (size_t t = 0; t < tris.size(); t++)
        {
            Box b;
            b.add(prev[tris[t].i1]); b.add(prev[tris[t].i2]); b.add(prev[tris[t].i3]);
            b.add(pos[tris[t].i1]); b.add(pos[tris[t].i2]); b.add(pos[tris[t].i3]);
            b.extrude(tol);
            tb[t] = b;
        }
        vb.resize(N);
        for (int i = 0; i < N; i++)
        {
            Box b;
            b.add(prev[i]); b.add(pos[i]);
            b.extrude(tol);
            vb[i] = b;
        }
        const std::vector<Edge>& E = mesh.edges;
        eb.resize(E.size());
        for (size_t e = 0; e < E.size(); e++)
        {
            Box b;
            b.add(pos[E[e].i1]); b.add(pos[E[e].i2]); b.add(prev[E[e].i1]); b.add(prev[E[e].i2]);
            b.extrude(tol);
            eb[e] = b;
        }
    }

    /* All-pairs version of the Midphase filters (Physics/SelfCollisionDetector.cpp:60-135):
       VT (triangle, vertex) with the vertex not on the triangle and not pinned,
       EE (e1 < e2) sharing no vertex, in both cases with overlapping swept boxes.
       Pairs come out in ascending (triangle, vertex) / (edge, higher edge) order.
       The default is an exact sweep over the boxes sorted by min x (the same
       pair sets as the all-pairs loop, bruteforce = true, at the sizes of the
       benchmark configurations). */
    bool bruteforce = false;

    void broadphase(float tol, std::vector<std::pair<int, int>>& vt, std::vector<std::pair<int, int>>& ee) const
    {
        if (!bruteforce) { broadphase_sweep(tol, vt, ee); return; }
        std::vector<Box> tb, vb, eb;
        swept_boxes(tol, tb, vb, eb);
        vt.clear(); ee.clear();
        for (size_t t = 0; t < tris.size(); t++)
            for (int i = 0; i < N; i++)
            {
                if ((u32)i == tris[t].i1 || (u32)i == tris[t].i2 || (u32)i == tris[t].i3 || invMass[i] == 0) continue;
                if (overlap(tb[t], vb[i])) vt.push_back({(int)t, i});
            }
        const std::vector<Edge>& E = mesh.edges;
        for (size_t a = 0; a < E.size(); a++)
            for (size_t b = a + 1; b < E.size(); b++)
            {
                u32 i1 = E[a].i1, i2 = E[a].i2, i3 = E[b].i1, i4 = E[b].i2;
                if (i1 == i3 || i2 == i4 || i1 == i4 || i2 == i3) continue;
                if (overlap(eb[a], eb[b])) ee.push_back({(int)a, (int)b});
            }
    }

    /* Sweep along x: for boxes a, b with a.mn.x <= b.mn.x (and mx >= mn, which
       box construction guarantees for finite coordinates) the x part of
       overlap() reduces to b.mn.x <= a.mx.x, so scanning the sorted list
       forward from each box while that holds meets every overlapping pair once;
       overlap() itself then decides, as in the all-pairs loop. A box with a NaN
       coordinate (for which overlap() can answer true against anything) is
       tested against every box, as the all-pairs loop does. */
    static bool has_nan(const Box& b)
    {
        return b.mn.x != b.mn.x || b.mn.y != b.mn.y || b.mn.z != b.mn.z ||
               b.mx.x != b.mx.x || b.mx.y != b.mx.y || b.mx.z != b.mx.z;
    }

    template <typename F>
    static void sweep_pairs(const std::vector<Box>& A, const std::vector<Box>& B, bool same, F&& emit)
    {
        /* entries: (min x, kind, index); kind 0 = A, 1 = B (same: all from A) */
        struct Ent { float x; int kind; int idx; };
        std::vector<Ent> ent;
        std::vector<int> nanA, nanB;
        for (size_t i = 0; i < A.size(); i++)
            if (has_nan(A[i])) nanA.push_back((int)i); else ent.push_back({A[i].mn.x, 0, (int)i});
        if (!same)
            for (size_t i = 0; i < B.size(); i++)
                if (has_nan(B[i])) nanB.push_back((int)i); else ent.push_back({B[i].mn.x, 1, (int)i});
        std::sort(ent.begin(), ent.end(), [](const Ent& a, const Ent& b) { return a.x < b.x; });
        const int n = (int)ent.size();
        std::vector<std::vector<std::pair<int, int>>> part;
#pragma omp parallel
        {
#pragma omp single
            part.resize(omp_threads());
            std::vector<std::pair<int, int>>& mine = part[omp_thread()];
#pragma omp for schedule(dynamic, 256)
            for (int k = 0; k < n; k++)
            {
                const Ent& e = ent[k];
                const Box& a = e.kind == 0 ? A[e.idx] : B[e.idx];
                for (int m = k + 1; m < n && ent[m].x <= a.mx.x; m++)
                {
                    const Ent& f = ent[m];
                    if (!same && f.kind == e.kind) continue;
                    const Box& b = f.kind == 0 ? A[f.idx] : B[f.idx];
                    if (!overlap(a, b)) continue;
                    if (same) mine.push_back({std::min(e.idx, f.idx), std::max(e.idx, f.idx)});
                    else if (e.kind == 0) mine.push_back({e.idx, f.idx});
                    else mine.push_back({f.idx, e.idx});
                }
            }
        }
        std::vector<std::pair<int, int>> all;
        for (auto& v : part) all.insert(all.end(), v.begin(), v.end());
        /* NaN boxes against everything (A side and B side) */
        for (int i : nanA)
        {
            if (same) { for (size_t j = 0; j < A.size(); j++) if ((int)j != i && overlap(A[i], A[j])) all.push_back({std::min(i, (int)j), std::max(i, (int)j)}); }
            else for (size_t j = 0; j < B.size(); j++) if (overlap(A[i], B[j])) all.push_back({i, (int)j});
        }
        for (int j : nanB)
            for (size_t i = 0; i < A.size(); i++)
                if (!has_nan(A[i]) && overlap(A[i], B[j])) all.push_back({(int)i, j});
        std::sort(all.begin(), all.end());
        all.erase(std::unique(all.begin(), all.end()), all.end());
        for (auto& pr : all) emit(pr.first, pr.second);
    }

    void broadphase_sweep(float tol, std::vector<std::pair<int, int>>& vt, std::vector<std::pair<int, int>>& ee) const
    {
        std::vector<Box> tb, vb, eb;
        swept_boxes(tol, tb, vb, eb);
        vt.clear(); ee.clear();
        sweep_pairs(tb, vb, false, [&](int t, int i) {
            if ((u32)i == tris[t].i1 || (u32)i == tris[t].i2 || (u32)i == tris[t].i3 || invMass[i] == 0) return;
            vt.push_back({t, i});
        });
        const std::vector<Edge>& E = mesh.edges;
        sweep_pairs(eb, eb, true, [&](int a, int b) {
            u32 i1 = E[a].i1, i2 = E[a].i2, i3 = E[b].i1, i4 = E[b].i2;
            if (i1 == i3 || i2 == i4 || i1 == i4 || i2 == i3) return;
            ee.push_back({a, b});
        });
    }

    float coplanarity(float t, V3 x1, V3 x2, V3 x3, V3 x4, V3 v1, V3 v2, V3 v3_, V3 v4) const
    {
        /* EvaluateFun_Coplanarity (SelfCollisionDetector.cpp:279-291) */
        V3 z1 = x1 + t * v1, z2 = x2 + t * v2, z3 = x3 + t * v3_, z4 = x4 + t * v4;
        V3 n1 = cross(z2 - z1, z3 - z1);
        return dot(n1, z4 - z1);
    }

    /* CheckInterval, <= 40 bisections (SelfCollisionDetector.cpp:440-489) */
    bool check_interval(float ta, float tb, V3 x1, V3 x2, V3 x3, V3 x4, V3 v1, V3 v2, V3 v3_, V3 v4, float& tx) const
    {
        float tx0 = ta, tx1 = tb;
        float fx0 = coplanarity(tx0, x1, x2, x3, x4, v1, v2, v3_, v4);
        float fx1 = coplanarity(tx1, x1, x2, x3, x4, v1, v2, v3_, v4);
        if (fx0 * fx1 > 0) return false;
        tx = tx0;
        for (int l = 0; l < 40; l++)
        {
            float tmid = 0.5f * (tx0 + tx1);
            float fmid = coplanarity(tmid, x1, x2, x3, x4, v1, v2, v3_, v4);
            if (std::fabs(fmid) < 0.01f) { tx = tmid; break; }
            if (fx0 * fmid < 0) { tx1 = tmid; fx1 = fmid; tx = tx0; }
            else if (fmid * fx1 < 0) { tx0 = tmid; fx0 = fmid; tx = tmid; }
            else return false;
        }
        return true;
    }

    /* SolveCubic + FindInflexionPoints + CheckDegenerateCase
       (SelfCollisionDetector.cpp:293-438) */
    bool solve_cubic(V3 x1, V3 x2, V3 x3, V3 x4, V3 v1, V3 v2, V3 v3_, V3 v4, float& toi) const
    {
        float f0 = coplanarity(0.f, x1, x2, x3, x4, v1, v2, v3_, v4);
        if (std::fabs(f0) < 0.001f) return false;
        V3 v10 = v1 - v4, v20 = v2 - v4, v30 = v3_ - v4;
        V3 x10 = x1 - x4, x20 = x2 - x4, x30 = x3 - x4;
        bool coplanar = false;
        float a = triple(v10, v20, v30);
        float b = triple(x10, v20, v30) + triple(v10, x20, v30) + triple(v10, v20, x30);
        float c = triple(x10, x20, v30) + triple(x10, v20, x30) + triple(v10, x20, x30);
        if (std::fabs(a) < 0.001f)
        {
            if (std::fabs(b) < 0.001f) return false;
            float d = triple(x10, x20, x30);
            float discr = c * c - 4 * b * d;
            if (discr < 0) return false;
            if (discr == 0)
            {
                float t = -0.5f * c / b;
                if (t < 0 || t > 1) return false;
                toi = t;
                return true;
            }
            float ds = std::sqrt(discr);
            float t1 = 0.5f * (-c - ds) / b, t2 = 0.5f * (-c + ds) / b;
            float t = std::min(t1, t2);
            if (t < 0 || t > 1) return false;
            toi = t;
            return true;
        }
        float discr = b * b - 3 * a * c;
        int num;
        float ti1 = 0, ti2 = 0;
        if (discr < 0) num = 0;
        else if (discr == 0) { ti1 = ti2 = -b / (3 * a); num = 1; }
        else
        {
            float ds = std::sqrt(discr);
            ti1 = (-b - ds) / (3 * a);
            ti2 = (-b + ds) / (3 * a);
            if (ti2 < ti1) std::swap(ti1, ti2);
            num = 2;
        }
        auto CI = [&](float ta, float tb) { return check_interval(ta, tb, x1, x2, x3, x4, v1, v2, v3_, v4, toi); };
        if (num == 0) coplanar = CI(0, 1);
        else if (num == 1)
        {
            if (ti1 < 0 || ti1 > 1) coplanar = CI(0, 1);
            else coplanar = CI(0, ti1) || CI(ti1, 1);
        }
        else
        {
            if (ti1 > 1 || ti2 < 0 || (ti1 < 0 && ti2 > 1)) coplanar = CI(0, 1);
            else if (ti1 < 0 && ti2 < 1) coplanar = CI(0, ti2) || CI(ti2, 1);
            else if (ti1 < 1 && ti2 > 1) coplanar = CI(0, ti1) || CI(ti1, 1);
            else if (ti1 > 0 && ti2 < 1) coplanar = CI(0, ti1) || CI(ti1, ti2) || CI(ti2, 1);
        }
        return coplanar;
    }

    /* VertexTriangleTest + VertexTriangleCCD (SelfCollisionDetector.cpp:171-277) */
    void vt_test(int tri, int vtx)
    {
        u32 i1 = tris[tri].i1, i2 = tris[tri].i2, i3 = tris[tri].i3;
        V3 x1 = prev[i1], x2 = prev[i2], x3 = prev[i3], x4 = prev[vtx];
        V3 v1 = pos[i1] - x1, v2 = pos[i2] - x2, v3_ = pos[i3] - x3, v4 = pos[vtx] - x4;
        float toi;
        if (!solve_cubic(x1, x2, x3, x4, v1, v2, v3_, v4, toi)) return;
        V3 z1 = x1 + toi * v1, z2 = x2 + toi * v2, z3 = x3 + toi * v3_, z4 = x4 + toi * v4;
        V3 coords, p;
        closest_pt_point_triangle(z4, z1, z2, z3, p, coords);
        V3 delta = z4 - p;
        const float eps = 0.1f;
        if (!(lensq(delta) < eps * eps)) return;
        V3 triNormal = normalized(cross(x2 - x1, x3 - x1));
        float side = dot(triNormal, x4 - x1);
        V3 n = normalized(cross(z2 - z1, z3 - z1));
        if (side < 0) n = -n;
        SContact c;
        c.i1 = i1; c.i2 = i2; c.i3 = i3; c.i4 = vtx;
        c.w1 = coords.x; c.w2 = coords.y; c.w3 = coords.z;
        c.normal = n;
        c.side = signed_volume(x4, x1, x2, x3);
        c.lambda = c.lambdaF = 0; c.error = 0;
        selfTris.push_back(c);
    }

    /* EdgeEdgeTest + EdgeEdgeCCD (SelfCollisionDetector.cpp:491-606) */
    void ee_test(int ea, int eb)
    {
        const Edge& A = mesh.edges[ea];
        const Edge& B = mesh.edges[eb];
        u32 i1 = A.i1, i2 = A.i2, j1 = B.i1, j2 = B.i2;
        if (i1 == j1 || i1 == j2 || i2 == j1 || i2 == j2) return;
        V3 x1 = prev[i1], x2 = prev[i2], x3 = prev[j1], x4 = prev[j2];
        V3 v1 = pos[i1] - x1, v2 = pos[i2] - x2, v3_ = pos[j1] - x3, v4 = pos[j2] - x4;
        float toi;
        if (!solve_cubic(x1, x2, x3, x4, v1, v2, v3_, v4, toi)) return;
        V3 z1 = x1 + toi * v1, z2 = x2 + toi * v2, z3 = x3 + toi * v3_, z4 = x4 + toi * v4;
        V3 c1, c2;
        float s, t;
        closest_pt_segm_segm(z1, z2, z3, z4, s, t, c1, c2);
        float dSqr = lensq(c1 - c2);
        const float eps = 0.5f * thickness;
        if (!(dSqr <= eps * eps)) return;
        SContact c;
        c.i1 = i1; c.i2 = i2; c.i3 = j1; c.i4 = j2;
        c.w1 = s; c.w2 = t; c.w3 = 0;
        float s2, t2;
        V3 d1, d2;
        closest_pt_segm_segm(x1, x2, x3, x4, s2, t2, d1, d2);
        c.normal = normalized(d2 - d1);
        c.side = signed_volume(x1, x2, x3, x4);
        c.lambda = c.lambdaF = 0; c.error = 0;
        selfEdges.push_back(c);
    }

    void narrow(const std::vector<std::pair<int, int>>& vt, const std::vector<std::pair<int, int>>& ee)
    {
        for (auto& p : vt) vt_test(p.first, p.second);
        for (auto& p : ee) ee_test(p.first, p.second);
    }

    /* The continuous detector run inside a step. Candidate pairs are taken in
       the canonical order the GPU produces them: (vertex, triangle) ascending
       for vertex-triangle pairs, (edge, higher edge) for edge-edge pairs. */
    void ccd_detect()
    {
        std::vector<std::pair<int, int>> vt, ee;
        broadphase(thickness + tolerance * 0.5f, vt, ee);
        std::sort(vt.begin(), vt.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
            return a.second < b.second || (a.second == b.second && a.first < b.first);
        });
        narrow(vt, ee);
    }
};

} // namespace

/* ================================================================ C API */
extern "C" {

void* orc_create(void) { return new Cloth(); }
void orc_destroy(void* h) { delete (Cloth*)h; }

void orc_add_walls(void* h, const float* b)
{
    Collider c; c.type = 1;
    c.walls.mn = v3(b[0], b[1], b[2]); c.walls.mx = v3(b[3], b[4], b[5]);
    ((Cloth*)h)->colliders.push_back(c);
}

void orc_add_sphere(void* h, float cx, float cy, float cz, float r)
{
    Collider c; c.type = 3; c.center = v3(cx, cy, cz); c.radius = r;
    ((Cloth*)h)->colliders.push_back(c);
}

void orc_add_sdf(void* h, int nx, int ny, int nz, const float* b, const float* values)
{
    Cloth* cl = (Cloth*)h;
    std::unique_ptr<GridSDF> g(new GridSDF());
    Box box; box.mn = v3(b[0], b[1], b[2]); box.mx = v3(b[3], b[4], b[5]);
    g->create(nx, ny, nz, box);
    for (size_t i = 0; i < g->val.size(); i++) g->val[i] = values[i];
    g->compute_gradient();
    Collider c; c.type = 7; c.sdf = (int)cl->sdfs.size();
    cl->sdfs.push_back(std::move(g));
    cl->colliders.push_back(c);
}

void orc_add_mesh(void* h, int nv, const float* verts, int nt, const unsigned* idx)
{
    Cloth* cl = (Cloth*)h;
    std::unique_ptr<MeshCollider> mc(new MeshCollider());
    mc->m.verts.resize(nv);
    for (int i = 0; i < nv; i++) mc->m.verts[i] = v3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    mc->m.idx.assign(idx, idx + 3 * nt);
    mc->m.compute_normals();
    mc->m.construct_edges();
    mc->m.construct_rings(false, true);
    Collider c; c.type = 4; c.mesh = (int)cl->meshes.size();
    cl->meshes.push_back(std::move(mc));
    cl->colliders.push_back(c);
}

void orc_init_grid(void* h, int divX, int divY, float inc, float ox, float oy, float oz, int horizontal, int attached)
{
    ((Cloth*)h)->init_grid(divX, divY, inc, v3(ox, oy, oz), horizontal != 0, attached != 0);
}

void orc_set_params(void* h, const float* p, int n)
{
    Cloth* c = (Cloth*)h;
    if (n < 15) return;
    c->unit = p[0]; c->thickness = p[1]; c->tolerance = p[2]; c->shear = p[3]; c->bendStiff = p[4];
    c->stretch = p[5]; c->poisson = p[6]; c->friction = p[7]; c->iterations = (int)p[8];
    c->substeps = (int)p[9]; c->flags = (int)p[10]; c->fem = p[11] != 0; c->dihedral = p[12] != 0;
    c->selfThreshold = p[13] != 0 ? -1.f : 0.003f;
    c->drag = p[14];
}

void orc_set_ccd(void* h, int on) { ((Cloth*)h)->ccd = on != 0; }
void orc_set_solver(void* h, int type) { ((Cloth*)h)->solver = type; }
int orc_num_particles(void* h) { return ((Cloth*)h)->N; }
int orc_num_tris(void* h) { return (int)((Cloth*)h)->tris.size(); }
int orc_num_bends(void* h) { return (int)((Cloth*)h)->bends.size(); }
int orc_num_edges(void* h) { return (int)((Cloth*)h)->mesh.edges.size(); }

void orc_set_positions(void* h, const float* p)
{
    Cloth* c = (Cloth*)h;
    for (int i = 0; i < c->N; i++) { c->pos[i] = v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); c->prev[i] = c->pos[i]; }
}

void orc_set_state(void* h, const float* p, const float* q, const float* v)
{
    Cloth* c = (Cloth*)h;
    for (int i = 0; i < c->N; i++)
    {
        c->pos[i] = v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
        c->prev[i] = v3(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
        c->vel[i] = v3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    }
}

/* ClothModel::SetMasses (Physics/ClothModel.cpp:45-52) */
void orc_set_masses(void* h, const float* m)
{
    Cloth* c = (Cloth*)h;
    for (int i = 0; i < c->N; i++) c->invMass[i] = m[i] == 0.f ? 0.f : 1.f / m[i];
}

void orc_set_inv_mass(void* h, int i, float w) { ((Cloth*)h)->invMass[i] = w; }

/* Constraint residual: max |C| over every triangle's warp, weft and shear
   constraints at the current positions (the C values SolveTriangles computes,
   Physics/ClothPBD.cpp:66-67,76,87,99). Bends are left out: with a flat rest
   angle a draped cloth holds them away from zero at equilibrium. */
float orc_residual(void* h)
{
    Cloth* c = (Cloth*)h;
    float r = 0.f;
    for (const Tri& t : c->tris)
    {
        V3 dx1 = c->pos[t.i2] - c->pos[t.i1], dx2 = c->pos[t.i3] - c->pos[t.i1];
        V3 wu = t.invDet * (t.dv2 * dx1 - t.dv1 * dx2);
        V3 wv = t.invDet * (-t.du2 * dx1 + t.du1 * dx2);
        float cu = std::fabs(0.5f * (dot(wu, wu) - t.lu2));
        float cv = std::fabs(0.5f * (dot(wv, wv) - t.lv2));
        float cs = std::fabs(dot(wu, wv));
        r = std::max(r, std::max(cu, std::max(cv, cs)));
    }
    return r;
}

void orc_get_state(void* h, float* p, float* q, float* v, float* w)
{
    Cloth* c = (Cloth*)h;
    for (int i = 0; i < c->N; i++)
    {
        if (p) { p[3 * i] = c->pos[i].x; p[3 * i + 1] = c->pos[i].y; p[3 * i + 2] = c->pos[i].z; }
        if (q) { q[3 * i] = c->prev[i].x; q[3 * i + 1] = c->prev[i].y; q[3 * i + 2] = c->prev[i].z; }
        if (v) { v[3 * i] = c->vel[i].x; v[3 * i + 1] = c->vel[i].y; v[3 * i + 2] = c->vel[i].z; }
        if (w) w[i] = c->invMass[i];
    }
}

void orc_get_tris(void* h, unsigned* idx, float* r10)
{
    Cloth* c = (Cloth*)h;
    for (size_t i = 0; i < c->tris.size(); i++)
    {
        const Tri& t = c->tris[i];
        idx[3 * i] = t.i1; idx[3 * i + 1] = t.i2; idx[3 * i + 2] = t.i3;
        if (r10)
        {
            float* r = r10 + 10 * i;
            r[0] = t.du1; r[1] = t.du2; r[2] = t.dv1; r[3] = t.dv2; r[4] = t.invDet;
            r[5] = t.lu0; r[6] = t.lv0; r[7] = t.lu2; r[8] = t.lv2; r[9] = t.area;
        }
    }
}

void orc_get_bends(void* h, unsigned* idx)
{
    Cloth* c = (Cloth*)h;
    for (size_t i = 0; i < c->bends.size(); i++)
    { idx[4 * i] = c->bends[i].i1; idx[4 * i + 1] = c->bends[i].i2; idx[4 * i + 2] = c->bends[i].i3; idx[4 * i + 3] = c->bends[i].i4; }
}

void orc_get_edges(void* h, int* e4)
{
    Cloth* c = (Cloth*)h;
    for (size_t i = 0; i < c->mesh.edges.size(); i++)
    {
        const Edge& e = c->mesh.edges[i];
        e4[4 * i] = (int)e.i1; e4[4 * i + 1] = (int)e.i2; e4[4 * i + 2] = e.t1; e4[4 * i + 3] = e.t2;
    }
}

void orc_set_tri_order(void* h, const int* o, int n)
{
    Cloth* c = (Cloth*)h;
    if (!o) c->triOrder.clear(); else c->triOrder.assign(o, o + n);
}

void orc_set_bend_order(void* h, const int* o, int n)
{
    Cloth* c = (Cloth*)h;
    if (!o) c->bendOrder.clear(); else c->bendOrder.assign(o, o + n);
}

void orc_set_contact_order(void* h, int mode) { ((Cloth*)h)->contactOrder = mode; }

void orc_set_static_colours(void* h, const int* triColour, int nt, int nTriColours, const int* edgeColour, int ne,
                            int nEdgeColours)
{
    Cloth* c = (Cloth*)h;
    c->triColour.assign(triColour, triColour + nt);
    c->edgeColour.assign(edgeColour, edgeColour + ne);
    c->nTriColours = nTriColours;
    c->nEdgeColours = nEdgeColours;
}

/* Replace the cloth's model by an explicit topology (particles, FEM triangles
   with their rest data du1 du2 dv1 dv2 invDet lu0 lv0 lu2 lv2 area, bends, links
   with rest length and stiffness), e.g. the one ClothPatch::Init(mesh) built in
   the reference; the collision mesh is rebuilt from the triangles. */
void orc_load_topology(void* h, int n, const float* pos, const float* invMass, int nt, const unsigned* tri,
                       const float* rest10, int nb, const unsigned* bend4, int nl, const unsigned* link2,
                       const float* linkRest2)
{
    Cloth* c = (Cloth*)h;
    c->N = n;
    c->pos.assign(n, v3(0, 0, 0)); c->prev.assign(n, v3(0, 0, 0)); c->vel.assign(n, v3(0, 0, 0));
    c->invMass.assign(invMass, invMass + n); c->uv.assign(n, v3(0, 0, 0));
    for (int i = 0; i < n; i++) { c->pos[i] = v3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]); c->prev[i] = c->pos[i]; }
    c->tris.clear(); c->bends.clear(); c->links.clear();
    c->triOrder.clear(); c->bendOrder.clear(); c->linkOrder.clear();
    std::vector<u32> idxs;
    for (int t = 0; t < nt; t++)
    {
        Tri r;
        r.i1 = tri[3 * t]; r.i2 = tri[3 * t + 1]; r.i3 = tri[3 * t + 2];
        const float* q = rest10 + 10 * t;
        r.du1 = q[0]; r.du2 = q[1]; r.dv1 = q[2]; r.dv2 = q[3]; r.invDet = q[4];
        r.lu0 = q[5]; r.lv0 = q[6]; r.lu2 = q[7]; r.lv2 = q[8]; r.area = q[9];
        r.det = r.du1 * r.dv2 - r.du2 * r.dv1;
        c->tris.push_back(r);
        idxs.push_back(r.i1); idxs.push_back(r.i2); idxs.push_back(r.i3);
    }
    for (int b = 0; b < nb; b++)
    {
        Bend x; x.i1 = bend4[4 * b]; x.i2 = bend4[4 * b + 1]; x.i3 = bend4[4 * b + 2]; x.i4 = bend4[4 * b + 3];
        c->bends.push_back(x);
    }
    for (int l = 0; l < nl; l++)
    {
        Cloth::Link x; x.i1 = link2[2 * l]; x.i2 = link2[2 * l + 1]; x.len = linkRest2[2 * l]; x.stiffness = linkRest2[2 * l + 1];
        c->links.push_back(x);
    }
    c->mesh = Topo();
    c->mesh.verts = c->pos;
    c->mesh.idx = idxs;
    c->mesh.compute_normals();
    c->mesh.construct_edges();
    c->mesh.construct_rings(true, true);
    c->prevMesh = c->mesh;
}

void orc_set_link_order(void* h, const int* o, int n)
{
    Cloth* c = (Cloth*)h;
    if (!o) c->linkOrder.clear(); else c->linkOrder.assign(o, o + n);
}

int orc_num_links(void* h) { return (int)((Cloth*)h)->links.size(); }

void orc_get_links(void* h, unsigned* idx2, float* lenStiff)
{
    Cloth* c = (Cloth*)h;
    for (size_t k = 0; k < c->links.size(); k++)
    {
        if (idx2) { idx2[2 * k] = c->links[k].i1; idx2[2 * k + 1] = c->links[k].i2; }
        if (lenStiff) { lenStiff[2 * k] = c->links[k].len; lenStiff[2 * k + 1] = c->links[k].stiffness; }
    }
}

/* 0: libm acosf as the reference; 1: the library's portable arc cosine (check mode).
   Process-wide, since the initial normals are computed when a grid is built. */
void orc_set_portable_math(int on) { g_portable_math = on != 0; }
float orc_portable_acos(float x) { return portable_acos(x); }

/* ClothPatch::Step (Physics/ClothPatch.cpp:323-335) */
void orc_step(void* h, float dt)
{
    Cloth* c = (Cloth*)h;
    const float hh = dt / c->substeps;
    for (int i = 0; i < c->substeps; i++) c->substep(hh);
}

void orc_update_mesh(void* h) { ((Cloth*)h)->update_mesh(); }

void orc_predict_detect(void* h, float hh, int runCCD)
{
    Cloth* c = (Cloth*)h;
    c->predict(hh);
    c->detect(runCCD != 0);
}

int orc_num_contacts(void* h, int kind)
{
    Cloth* c = (Cloth*)h;
    switch (kind)
    {
    case 0: return (int)c->contacts.size();
    case 1: return (int)c->triContacts.size();
    case 2: return (int)c->edgeContacts.size();
    case 3: return (int)c->selfTris.size();
    case 4: return (int)c->selfEdges.size();
    }
    return 0;
}

void orc_get_vertex_contacts(void* h, int* idx2, float* f7)
{
    Cloth* c = (Cloth*)h;
    for (size_t i = 0; i < c->contacts.size(); i++)
    {
        const VContact& k = c->contacts[i];
        idx2[2 * i] = k.idx; idx2[2 * i + 1] = k.feature;
        f7[7 * i] = k.point.x; f7[7 * i + 1] = k.point.y; f7[7 * i + 2] = k.point.z;
        f7[7 * i + 3] = k.normal.x; f7[7 * i + 4] = k.normal.y; f7[7 * i + 5] = k.normal.z;
        f7[7 * i + 6] = k.depth;
    }
}

void orc_get_tri_contacts(void* h, int* idx4, float* f9)
{
    Cloth* c = (Cloth*)h;
    for (size_t i = 0; i < c->triContacts.size(); i++)
    {
        const TContact& k = c->triContacts[i];
        idx4[4 * i] = k.i1; idx4[4 * i + 1] = k.i2; idx4[4 * i + 2] = k.i3; idx4[4 * i + 3] = k.feature;
        f9[9 * i] = k.point.x; f9[9 * i + 1] = k.point.y; f9[9 * i + 2] = k.point.z;
        f9[9 * i + 3] = k.normal.x; f9[9 * i + 4] = k.normal.y; f9[9 * i + 5] = k.normal.z;
        f9[9 * i + 6] = k.w1; f9[9 * i + 7] = k.w2; f9[9 * i + 8] = k.w3;
    }
}

void orc_get_edge_contacts(void* h, int* idx3, float* f8)
{
    Cloth* c = (Cloth*)h;
    for (size_t i = 0; i < c->edgeContacts.size(); i++)
    {
        const EContact& k = c->edgeContacts[i];
        idx3[3 * i] = k.i1; idx3[3 * i + 1] = k.i2; idx3[3 * i + 2] = k.feature;
        f8[8 * i] = k.point.x; f8[8 * i + 1] = k.point.y; f8[8 * i + 2] = k.point.z;
        f8[8 * i + 3] = k.normal.x; f8[8 * i + 4] = k.normal.y; f8[8 * i + 5] = k.normal.z;
        f8[8 * i + 6] = k.w1; f8[8 * i + 7] = k.w2;
    }
}

void orc_get_self_contacts(void* h, int kind, int* idx4, float* f7)
{
    Cloth* c = (Cloth*)h;
    const std::vector<SContact>& v = kind == 3 ? c->selfTris : c->selfEdges;
    for (size_t i = 0; i < v.size(); i++)
    {
        const SContact& k = v[i];
        idx4[4 * i] = k.i1; idx4[4 * i + 1] = k.i2; idx4[4 * i + 2] = k.i3; idx4[4 * i + 3] = k.i4;
        f7[7 * i] = k.normal.x; f7[7 * i + 1] = k.normal.y; f7[7 * i + 2] = k.normal.z;
        f7[7 * i + 3] = k.w1; f7[7 * i + 4] = k.w2; f7[7 * i + 5] = k.w3; f7[7 * i + 6] = k.side;
    }
}

void orc_get_mesh_normals(void* h, int prev, float* n)
{
    Cloth* c = (Cloth*)h;
    const Topo& m = prev ? c->prevMesh : c->mesh;
    for (size_t i = 0; i < m.normals.size(); i++) { n[3 * i] = m.normals[i].x; n[3 * i + 1] = m.normals[i].y; n[3 * i + 2] = m.normals[i].z; }
}

void orc_get_mesh_tri_normals(void* h, int prev, float* n)
{
    Cloth* c = (Cloth*)h;
    const Topo& m = prev ? c->prevMesh : c->mesh;
    for (size_t i = 0; i < m.triN.size(); i++) { n[3 * i] = m.triN[i].x; n[3 * i + 1] = m.triN[i].y; n[3 * i + 2] = m.triN[i].z; }
}

void orc_self_contact_colours(void* h, int kind, int* colours)
{
    Cloth* c = (Cloth*)h;
    auto vf = [](const SContact& s, u32* v) { v[0] = s.i1; v[1] = s.i2; v[2] = s.i3; v[3] = s.i4; return 4; };
    std::vector<int> col;
    c->colour_order(kind == 3 ? c->selfTris : c->selfEdges, vf, &col);
    for (size_t i = 0; i < col.size(); i++) colours[i] = col[i];
}

void orc_set_bruteforce_broadphase(void* h, int on) { ((Cloth*)h)->bruteforce = on != 0; }

int orc_ccd_broadphase(void* h, float tol, int kind, int* pairs, int cap)
{
    Cloth* c = (Cloth*)h;
    std::vector<std::pair<int, int>> vt, ee;
    c->broadphase(tol, vt, ee);
    const auto& v = kind == 0 ? vt : ee;
    int n = (int)v.size();
    for (int i = 0; i < n && i < cap; i++) { pairs[2 * i] = v[i].first; pairs[2 * i + 1] = v[i].second; }
    return n;
}

void orc_ccd_narrow_on(void* h, int nvt, const int* vt, int nee, const int* ee)
{
    Cloth* c = (Cloth*)h;
    std::vector<std::pair<int, int>> a(nvt), b(nee);
    for (int i = 0; i < nvt; i++) a[i] = {vt[2 * i], vt[2 * i + 1]};
    for (int i = 0; i < nee; i++) b[i] = {ee[2 * i], ee[2 * i + 1]};
    c->selfTris.clear();
    c->selfEdges.clear();
    c->narrow(a, b);
}

void orc_swept_boxes(void* h, int kind, float tol, float* out)
{
    Cloth* c = (Cloth*)h;
    std::vector<Box> tb, vb, eb;
    c->swept_boxes(tol, tb, vb, eb);
    const std::vector<Box>& v = kind == 0 ? tb : (kind == 1 ? vb : eb);
    for (size_t i = 0; i < v.size(); i++)
    {
        out[6 * i] = v[i].mn.x; out[6 * i + 1] = v[i].mn.y; out[6 * i + 2] = v[i].mn.z;
        out[6 * i + 3] = v[i].mx.x; out[6 * i + 4] = v[i].mx.y; out[6 * i + 5] = v[i].mx.z;
    }
}

}
