// step_kernels.cu — sm_100a kernels of the per-substep PBD cloth step.
//
// One substep (ClothModelPBD::Step, Physics/ClothPBD.cpp:255-322) is, on the GPU:
//   predict -> [collision mesh refit, detection into fixed slots, block-scan
//   compaction, independent-set colouring of multi-particle contacts]
//   -> iterations x (FEM colours, bend colours every 2nd iteration, vertex
//   contacts, multi-particle contacts) -> velocity,
// all captured once into a CUDA graph by the host (cloth.cu).
//
// Bit-exactness: compiled with -fmad=false and IEEE division/square root; the
// arithmetic follows the reference's operation order (see scmath.cuh), so box
// overlaps, contact regions, candidate pairs and CCD hits are decided exactly as
// the reference decides them. acosf/atan2f are CUDA's and may differ from glibc's
// by a few ulp (bend angles, angle-weighted normals).
#include "step_common.cuh"
#include <cooperative_groups.h>
#include <cuda/atomic>
#include <cstdio>
#include <mutex>
#include <climits>
#include <algorithm>

namespace cg = cooperative_groups;

namespace sc {
// --------------------------------------------------------------- predict
// ClothModelPBD::Step, symplectic Euler part (Physics/ClothPBD.cpp:257-266);
// also the max |pos - prev| used by the collision thresholds
// (Physics/ClothCollision.cpp:91-100).
__global__ void k_predict(DevCloth c, SolverParams P)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    float4 p = c.pos[i];
    c.prev[i] = make_float4(p.x, p.y, p.z, 0.f);
    if (p.w == 0.f) return;
    float4 v = c.vel[i];
    const float hgx = P.h * 0.f, hgy = P.h * -9.8f, hgz = P.h * 0.f;
    v.x += P.unit * hgx; v.y += P.unit * hgy; v.z += P.unit * hgz;
    v.x = P.drag * v.x; v.y = P.drag * v.y; v.z = P.drag * v.z;
    c.vel[i] = v;
    V3 np = mk(p.x, p.y, p.z) + P.h * mk(v.x, v.y, v.z);
    c.pos[i] = make_float4(np.x, np.y, np.z, p.w);
    float tv = len(np - mk(p.x, p.y, p.z));
    atomic_max_pos(&c.scal[0], tv);
}

// ClothModelPBD::Step, velocity update (Physics/ClothPBD.cpp:314-321)
__global__ void k_velocity(DevCloth c, SolverParams P)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    float4 p = c.pos[i];
    if (p.w == 0.f) return;
    float4 q = c.prev[i];
    V3 v = P.invH * (mk(p.x, p.y, p.z) - mk(q.x, q.y, q.z));
    c.vel[i] = make_float4(v.x, v.y, v.z, 0.f);
}

// ------------------------------------------ Jacobi and conjugate-residual link solves
// ClothModelPBD::SolveLinksJacobi, first loop (Physics/ClothPBD.cpp:616-639): every
// link's displacement from the same positions (no guard against two pinned ends,
// as the reference)
__global__ void k_jacobi_disp(DevCloth c, LinkSolve ls, float k, float omega)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ls.L) return;
    const float4 r = ls.link[i];
    const float4 a = c.pos[__float_as_uint(r.x)], b = c.pos[__float_as_uint(r.y)];
    const float mu = 1.f / (a.w + b.w);
    V3 delta = mk(a.x, a.y, a.z) - mk(b.x, b.y, b.z);
    const float len0 = r.z;
    const float l = len(delta);
    delta = (1.f / l) * delta;
    const float err = l - len0;
    const float epsilon = len0 / (k * r.w);
    const float s = 1.f / (1.f + mu * epsilon);
    const float lambda = err * mu * s;
    const V3 d = (omega * lambda) * delta;
    ls.disp[i] = make_float4(d.x, d.y, d.z, 0.f);
}

// SolveCR per link as compiled (SKIP_ALPHA, SKIP_BETA; Physics/ClothPBD.cpp:371-379,
// 405-411, 440-447, 486-494): error and unit direction from the same positions,
// d = r + beta d, displacement alpha d along the direction
__global__ void k_cr_disp(DevCloth c, LinkSolve ls, float unit, float beta, float alpha)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ls.L) return;
    const float4 r = ls.link[i];
    const float4 a = c.pos[__float_as_uint(r.x)], b = c.pos[__float_as_uint(r.y)];
    V3 delta = mk(b.x, b.y, b.z) - mk(a.x, a.y, a.z);
    const float cc = (len(delta) - r.z) * r.w * unit;
    const float ln = len(delta);
    delta = (1.f / ln) * delta;
    const float res = -cc;
    const float d = res + beta * ls.d[i];
    ls.d[i] = d;
    const float dLambda = alpha * d;
    const V3 disp = dLambda * delta;
    ls.disp[i] = make_float4(disp.x, disp.y, disp.z, 0.f);
}

// the apply loop of both (Physics/ClothPBD.cpp:641-650, 486-494): particle i1 of a
// link moves by -invMass disp, i2 by +invMass disp, in link order; each particle
// takes its incident links in increasing index, which is the sequential loop's
// order of updates to it
__global__ void k_link_apply(DevCloth c, LinkSolve ls, int iterationsDone)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && iterationsDone > 0) c.scal[9] = (float)iterationsDone;
    if (p >= c.N) return;
    const float4 x = c.pos[p];
    V3 q = mk(x.x, x.y, x.z);
    const float w = x.w;
    const int e0 = ls.incStart[p], e1 = ls.incStart[p + 1];
    if (e0 == e1) return;
    for (int j = e0; j < e1; j++)
    {
        const int e = ls.inc[j];
        const float4 d = ls.disp[e >> 1];
        const V3 t = w * mk(d.x, d.y, d.z);
        q = (e & 1) ? q + t : q - t;
    }
    c.pos[p] = make_float4(q.x, q.y, q.z, w);
}

void launch_solve_jacobi(cudaStream_t s, const DevCloth& c, const SolverParams& P, const LinkSolve& ls)
{
    const float k = P.h2 * P.area * P.unit;
    for (int it = 0; it < P.iterations; it++)
    {
        if (ls.L > 0) k_jacobi_disp<<<blocks_for(ls.L), 256, 0, s>>>(c, ls, k, 0.5f);
        k_link_apply<<<blocks_for(c.N), 256, 0, s>>>(c, ls, it + 1 == P.iterations ? P.iterations : 0);
    }
}

void launch_solve_cr(cudaStream_t s, const DevCloth& c, const SolverParams& P, const LinkSolve& ls, const float* beta)
{
    if (ls.L == 0) return;
    cudaMemsetAsync(ls.d, 0, sizeof(float) * (size_t)ls.L, s);
    for (int it = 0; it < P.iterations; it++)
    {
        k_cr_disp<<<blocks_for(ls.L), 256, 0, s>>>(c, ls, P.unit, beta[it], 0.1f);
        k_link_apply<<<blocks_for(c.N), 256, 0, s>>>(c, ls, it + 1 == P.iterations ? P.iterations : 0);
    }
}

#include "solver.cuh"     // projections, contact solves and the solver kernels (IEEE build)

// ----------------------------------------------------------- normals
// Mesh::ComputeNormals (Geometry/Mesh.cpp:10-63): per-triangle unit normal and
// corner angles, then a per-vertex gather in triangle order (the reference's
// accumulation order), then normalisation.
__global__ void k_tri_normals(const float4* verts, const uint32_t* tri, int T, float4* triN, float4* ang)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    V3 a = ld3(verts, tri[3 * t]), b = ld3(verts, tri[3 * t + 1]), cc = ld3(verts, tri[3 * t + 2]);
    V3 nt = normalized(cross(b - a, cc - a));
    triN[t] = f4(nt, 0.f);
    V3 e1 = normalized(b - a), e2 = normalized(cc - b), e3 = normalized(a - cc);
    float c1 = -dot(e1, e3), c2 = -dot(e1, e2), c3 = -dot(e2, e3);
    float s1 = len(cross(e1, -e3)), s2 = len(cross(e2, -e1)), s3 = len(cross(e3, -e1));
    float t1 = fabsf(c1) > 1 ? fabsf((float)atan2((double)s1, (double)c1)) : portable_acos(c1);
    float t2 = fabsf(c2) > 1 ? fabsf((float)atan2((double)s2, (double)c2)) : portable_acos(c2);
    float t3 = fabsf(c3) > 1 ? fabsf((float)atan2((double)s3, (double)c3)) : portable_acos(c3);
    ang[t] = make_float4(t1, t2, t3, 0.f);
}

__global__ void k_vertex_normals(int N, const int* start, const int2* vt, const float4* triN, const float4* ang, float4* out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    V3 n = mk(0.f, 0.f, 0.f);
    for (int k = start[i]; k < start[i + 1]; k++)
    {
        int2 tc = vt[k];
        float4 a = ang[tc.x];
        float w = tc.y == 0 ? a.x : (tc.y == 1 ? a.y : a.z);
        n += w * ld3(triN, tc.x);
    }
    if (len(n) != 0) n = normalized(n);
    out[i] = f4(n, 0.f);
}

// ------------------------------------------------------------ SDF grid
// SDF::GetGridCoords / GetValue / GetGrad (Geometry/SDF.h:105-155): point
// fetches from 3-D textures (border mode returns the reference's 0 outside the
// grid) and the trilinear blend in FP32 registers in the reference's order.
struct GridCoord { int x, y, z; float fx, fy, fz; };

__device__ __forceinline__ GridCoord grid_coords(const VColl& g, V3 p)
{
    GridCoord r;
    float rx = (p.x - g.sdfLo.x) / g.sdfSteps.x;
    float ry = (p.y - g.sdfLo.y) / g.sdfSteps.y;
    float rz = (p.z - g.sdfLo.z) / g.sdfSteps.z;
    r.x = (int)floorf(rx); r.y = (int)floorf(ry); r.z = (int)floorf(rz);
    r.fx = fabsf(rx - r.x); r.fy = fabsf(ry - r.y); r.fz = fabsf(rz - r.z);
    return r;
}

__device__ __forceinline__ bool grid_out(const VColl& g, int x, int y, int z)
{
    return x > g.sdfCells.x || y > g.sdfCells.y || z > g.sdfCells.z || x < 0 || y < 0 || z < 0;
}

__device__ __forceinline__ float tv(const VColl& g, int x, int y, int z)
{
    return tex3D<float>(g.val, x + 0.5f, y + 0.5f, z + 0.5f);
}
__device__ __forceinline__ V3 tg(const VColl& g, int x, int y, int z)
{
    float4 a = tex3D<float4>(g.grad, x + 0.5f, y + 0.5f, z + 0.5f);
    return mk(a.x, a.y, a.z);
}

__device__ float sdf_value(const VColl& g, V3 p)
{
    GridCoord q = grid_coords(g, p);
    if (grid_out(g, q.x, q.y, q.z)) return FLT_MAX;
    const float fx = q.fx, fy = q.fy, fz = q.fz;
    const int x = q.x, y = q.y, z = q.z;
    return (1.f - fx) * (1.f - fy) * (1.f - fz) * tv(g, x, y, z) +
           (1.f - fx) * (1.f - fy) * fz * tv(g, x, y, z + 1) +
           (1.f - fx) * fy * (1.f - fz) * tv(g, x, y + 1, z) +
           (1.f - fx) * fy * fz * tv(g, x, y + 1, z + 1) +
           fx * (1.f - fy) * (1.f - fz) * tv(g, x + 1, y, z) +
           fx * (1.f - fy) * fz * tv(g, x + 1, y, z + 1) +
           fx * fy * (1.f - fz) * tv(g, x + 1, y + 1, z) +
           fx * fy * fz * tv(g, x + 1, y + 1, z + 1);
}

__device__ V3 sdf_grad(const VColl& g, V3 p)
{
    GridCoord q = grid_coords(g, p);
    if (grid_out(g, q.x, q.y, q.z)) return mk(0.f, 0.f, 0.f);
    const float fx = q.fx, fy = q.fy, fz = q.fz;
    const int x = q.x, y = q.y, z = q.z;
    return (1.f - fx) * (1.f - fy) * (1.f - fz) * tg(g, x, y, z) +
           (1.f - fx) * (1.f - fy) * fz * tg(g, x, y, z + 1) +
           (1.f - fx) * fy * (1.f - fz) * tg(g, x, y + 1, z) +
           (1.f - fx) * fy * fz * tg(g, x, y + 1, z + 1) +
           fx * (1.f - fy) * (1.f - fz) * tg(g, x + 1, y, z) +
           fx * (1.f - fy) * fz * tg(g, x + 1, y, z + 1) +
           fx * fy * (1.f - fz) * tg(g, x + 1, y + 1, z) +
           fx * fy * fz * tg(g, x + 1, y + 1, z + 1);
}

// SphereSDF::QueryPoint / GridSDF::QueryPoint (Physics/ClothCollisionSDF.h:14-24,130-139)
__device__ float query_point(const VColl& g, V3 p, V3& cp, V3& n, int& feature)
{
    if (g.type == 7)
    {
        float v = sdf_value(g, p);
        V3 gr = normalized(sdf_grad(g, p));
        n = gr;
        cp = p - v * gr;
        feature = -3;
        return v;
    }
    V3 ctr = mk(g.a.x, g.a.y, g.a.z);
    V3 delta = p - ctr;
    float l = len(delta);
    delta = (1.f / l) * delta;
    n = delta;
    cp = ctr + g.a.w * delta;
    feature = -1;
    return l - g.a.w;
}

// --------------------------------------------------- static mesh tree
// ClosestPointOnMeshToPointRec / ToTriangleRec / ToSegmentEdgeRec
// (Geometry/ClosestPointOnMesh.cpp:262-302,393-452,589-659) as an explicit-stack
// depth-first search that visits nodes in exactly the recursion's order:
// the nearer child first; the farther child is tested against the distance
// found once the nearer subtree is done.
constexpr int MESH_STACK = 48;

struct PointHit { float dist; int tri; V3 cp, bary, normal; int region; };

// The three nearest-feature searches take `bound`, the contact threshold of
// their caller: a result at or beyond it is discarded there, and starting the
// search's best distance at the bound prunes exactly the subtrees that could
// only produce such results — every node nearer than the bound is visited in the
// same order as by the unbounded search, so results below the bound (and ties
// among them) are unchanged.
// Leaf pre-filter of the nearest-feature searches: a primitive can change a
// search's result only if its distance is below the best so far (minDist), and
// its distance is at least the distance between the query and the primitive's
// bounding box. Primitives whose box distance exceeds minDist by more than the
// rounding of the exact computation (slack: 1e-4 of the coordinates' magnitude,
// orders of magnitude above it) are skipped without the exact closest-point
// computation; the searches return exactly what they return without it.
__device__ __forceinline__ float skip_slack(V3 p)
{
    return 1e-4f * (1.f + fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z))));
}
__device__ __forceinline__ bool cannot_improve(float boxDist, float minDist, float slack)
{
    return boxDist > minDist + slack;
}
__device__ __forceinline__ Box prim_box(V3 a, V3 b, V3 c)
{
    Box x = Box::empty(); x.add(a); x.add(b); x.add(c);
    return x;
}

__device__ PointHit mesh_point_query(const DevMesh& m, V3 p, int* status, float bound)
{
    PointHit r; r.dist = FLT_MAX; r.tri = -1; r.region = -1;
    r.cp = r.bary = r.normal = mk(0.f, 0.f, 0.f);
    float minDist = bound;
    const float slack = skip_slack(p);
    int stNode[MESH_STACK]; float stDist[MESH_STACK];
    int sp = 0;
    int node = 0;
    while (true)
    {
        if (node >= 0)
        {
            int4 pr = m.tree.primRange[node];
            for (int k = 0; k < pr.y; k++)
            {
                uint32_t t = m.tree.tris[pr.x + k];
                V3 a = ld3(m.v, m.tri[3 * t]), b = ld3(m.v, m.tri[3 * t + 1]), cc = ld3(m.v, m.tri[3 * t + 2]);
                if (cannot_improve(prim_box(a, b, cc).dist(p), minDist, slack)) continue;
                V3 coords, pt;
                int region = closest_point_triangle(p, a, b, cc, pt, coords);
                V3 delta = p - pt;
                float dist = len(delta);
                if (dist == 0) continue;
                if (dist < minDist)
                {
                    minDist = dist;
                    r.dist = dist; r.tri = (int)t; r.cp = pt; r.bary = coords;
                    r.normal = (1.f / dist) * delta; r.region = region;
                }
            }
            int2 ch = m.tree.children[node];
            if (ch.x >= 0 || ch.y >= 0)
            {
                Box bl, br;
                float dl = FLT_MAX, dr = FLT_MAX;
                if (ch.x >= 0) { bl.lo = ld3(m.tree.lo, ch.x); bl.hi = ld3(m.tree.hi, ch.x); dl = bl.dist(p); }
                if (ch.y >= 0) { br.lo = ld3(m.tree.lo, ch.y); br.hi = ld3(m.tree.hi, ch.y); dr = br.dist(p); }
                int nearN = ch.x, farN = ch.y; float nearD = dl, farD = dr;
                if (!(dl < dr)) { nearN = ch.y; farN = ch.x; nearD = dr; farD = dl; }
                if (sp < MESH_STACK) { stNode[sp] = farN; stDist[sp] = farD; sp++; }
                else atomicOr(status, ST_MESH_STACK_OVERFLOW);
                node = (nearD < minDist) ? nearN : -1;
                continue;
            }
        }
        // pop the next pending far child whose box is still within reach
        node = -1;
        while (sp > 0 && node < 0)
        {
            sp--;
            if (stDist[sp] < minDist) node = stNode[sp];
        }
        if (node < 0) break;
    }
    return r;
}

struct VtxHit { float dist; int vertex; V3 cpMesh, cpTri, bary, normal; int region; };

__device__ VtxHit mesh_triangle_query(const DevMesh& m, V3 a, V3 b, V3 cc, int* status, float bound)
{
    VtxHit r; r.dist = -FLT_MAX; r.vertex = -1; r.region = 0;
    r.cpMesh = r.cpTri = r.bary = r.normal = mk(0.f, 0.f, 0.f);
    float minDist = bound;
    Box tb = Box::empty(); tb.add(a); tb.add(b); tb.add(cc);
    const float slack = skip_slack(a);
    int stNode[MESH_STACK]; float stDist[MESH_STACK];
    int sp = 0, node = 0;
    while (true)
    {
        if (node >= 0)
        {
            int4 pr = m.tree.primRange[node];
            for (int k = 0; k < pr.w; k++)
            {
                uint32_t v = m.tree.verts[pr.z + k];
                V3 pv = ld3(m.v, v);
                if (cannot_improve(tb.dist(pv), minDist, slack)) continue;
                V3 bary, cp;
                int region = closest_point_triangle(pv, a, b, cc, cp, bary);
                V3 delta = cp - pv;
                float dist = len(delta);
                if (dist == 0) continue;
                if (dist < minDist)
                {
                    minDist = dist;
                    r.vertex = (int)v; r.cpMesh = pv; r.cpTri = cp; r.bary = bary;
                    r.normal = (1.f / dist) * delta; r.dist = dist; r.region = region;
                }
            }
            int2 ch = m.tree.children[node];
            if (ch.x >= 0 || ch.y >= 0)
            {
                Box bl, br;
                float dl = FLT_MAX, dr = FLT_MAX;
                if (ch.x >= 0) { bl.lo = ld3(m.tree.lo, ch.x); bl.hi = ld3(m.tree.hi, ch.x); dl = bl.dist(tb); }
                if (ch.y >= 0) { br.lo = ld3(m.tree.lo, ch.y); br.hi = ld3(m.tree.hi, ch.y); dr = br.dist(tb); }
                int nearN = ch.x, farN = ch.y; float nearD = dl, farD = dr;
                if (!(dl < dr)) { nearN = ch.y; farN = ch.x; nearD = dr; farD = dl; }
                if (sp < MESH_STACK) { stNode[sp] = farN; stDist[sp] = farD; sp++; }
                else atomicOr(status, ST_MESH_STACK_OVERFLOW);
                node = (nearD < minDist) ? nearN : -1;
                continue;
            }
        }
        node = -1;
        while (sp > 0 && node < 0) { sp--; if (stDist[sp] < minDist) node = stNode[sp]; }
        if (node < 0) break;
    }
    return r;
}

struct SegHit { float dist; int edge; V3 cpMesh, cpSegm, normal; float cs0, cs1, cm0, cm1; int region; };

// ComputeEdgeNormal (Geometry/ClosestPointOnMesh.cpp:483-497)
__device__ __forceinline__ V3 mesh_edge_normal(const DevMesh& m, int e, float param)
{
    V3 n = ld3(m.en, e);
    int4 ed = m.edge[e];
    if (param == 0.f) n = ld3(m.n, ed.x);
    if (param == 1.f) n = ld3(m.n, ed.y);
    return n;
}

__device__ SegHit mesh_segment_query(const DevMesh& m, V3 p, V3 q, int* status, float bound)
{
    SegHit r; r.dist = -FLT_MAX; r.edge = -1; r.region = -1;
    r.cpMesh = r.cpSegm = r.normal = mk(0.f, 0.f, 0.f);
    r.cs0 = r.cs1 = r.cm0 = r.cm1 = 0.f;
    float minDist = bound;
    Box eb = Box::empty(); eb.add(p); eb.add(q);
    const float slack = skip_slack(p);
    int stNode[MESH_STACK]; float stDist[MESH_STACK];
    int sp = 0, node = 0;
    while (true)
    {
        if (node >= 0)
        {
            int2 er = m.tree.edgeRange[node];
            for (int k = 0; k < er.y; k++)
            {
                uint32_t e = m.tree.edges[er.x + k];
                int4 ed = m.edge[e];
                V3 a = ld3(m.v, ed.x), b = ld3(m.v, ed.y);
                Box pb = Box::empty(); pb.add(a); pb.add(b);
                if (cannot_improve(pb.dist(eb), minDist, slack)) continue;
                float ps, pm;
                V3 cs, cm;
                int region = closest_segm_segm(p, q, a, b, ps, pm, cs, cm);
                V3 delta = cm - cs;
                float dist = len(delta);
                if (dist == 0) continue;
                if (dist < minDist)
                {
                    minDist = dist;
                    r.dist = dist; r.edge = (int)e; r.cpMesh = cm; r.cpSegm = cs;
                    r.cs0 = 1.0f - ps; r.cs1 = ps; r.cm0 = 1.0f - pm; r.cm1 = pm;
                    r.normal = mesh_edge_normal(m, (int)e, pm);
                    r.region = region;
                }
            }
            int2 ch = m.tree.children[node];
            if (ch.x >= 0 || ch.y >= 0)
            {
                Box bl, br;
                float dl = FLT_MAX, dr = FLT_MAX;
                if (ch.x >= 0) { bl.lo = ld3(m.tree.lo, ch.x); bl.hi = ld3(m.tree.hi, ch.x); dl = bl.dist(eb); }
                if (ch.y >= 0) { br.lo = ld3(m.tree.lo, ch.y); br.hi = ld3(m.tree.hi, ch.y); dr = br.dist(eb); }
                int nearN = ch.x, farN = ch.y; float nearD = dl, farD = dr;
                if (!(dl < dr)) { nearN = ch.y; farN = ch.x; nearD = dr; farD = dl; }
                if (sp < MESH_STACK) { stNode[sp] = farN; stDist[sp] = farD; sp++; }
                else atomicOr(status, ST_MESH_STACK_OVERFLOW);
                node = (nearD < minDist) ? nearN : -1;
                continue;
            }
        }
        node = -1;
        while (sp > 0 && node < 0) { sp--; if (stDist[sp] < minDist) node = stNode[sp]; }
        if (node < 0) break;
    }
    return r;
}

// ------------------------------------------------- vertex contact detection
// One thread per cloth vertex walks the world's colliders in order and writes
// its vertex contacts into per-(collider, vertex) slots, reproducing
// WallCollisions, SDFCollisions<Sphere/Grid> (vertex part) and the vertex part
// of MeshCollisions (Physics/ClothCollision.cpp:89-135,199-220,438-470).
__global__ void k_vertex_colliders(DevCloth c, SolverParams P, Buffers b)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const V3 pos = ld3(c.pos, i), prev = ld3(c.prev, i);
    const float maxTv = c.scal[0];
    const float radTolMesh = P.thickness + mx(P.tolerance, maxTv * 1.5f);
    const int2 cr = colliders_of(c, b, i);
    for (int ci = cr.x; ci < cr.x + cr.y; ci++)
    {
        const VColl& g = b.vcoll[ci];
        VC* slot = b.vc + g.slotBase + (size_t)(i - g.vBegin) * g.kmax;
        int n = 0;
        auto add = [&](V3 p, V3 nn, int feature, int mesh) {
            VC v;
            v.point = f4(p, 0.f); v.normal = f4(nn, 0.f);
            v.lam = make_float2(0.f, 0.f); v.feature = feature; v.mesh = mesh;
            slot[n++] = v;
        };
        if (g.type == 1)
        {
            if (P.flags & CF_WALLS)
            {
                const float r = P.thickness + P.tolerance;
                if (pos.y - r <= g.a.y) add(mk(pos.x, g.a.y, pos.z), mk(0, 1, 0), -1, -1);
                if (pos.x - r <= g.a.x) add(mk(g.a.x, pos.y, pos.z), mk(1, 0, 0), -1, -1);
                if (pos.x + r >= g.b.x) add(mk(g.b.x, pos.y, pos.z), mk(-1, 0, 0), -1, -1);
                if (pos.z - r <= g.a.z) add(mk(pos.x, pos.y, g.a.z), mk(0, 0, 1), -1, -1);
                if (pos.z + r >= g.b.z) add(mk(pos.x, pos.y, g.b.z), mk(0, 0, -1), -1, -1);
            }
        }
        else if (g.type == 3 || g.type == 7)
        {
            if (P.flags & CF_VERTICES)
            {
                V3 p, nn; int feature;
                float dist = query_point(g, prev, p, nn, feature);
                float tvv = len(prev - pos);
                float radTol = P.thickness + mx(P.tolerance, tvv * 1.1f);
                if (dist < radTol && dist >= 0) add(p, nn, feature, -1);
            }
        }
        else if (g.type == 4)
        {
            if (P.flags & CF_VERTICES)
            {
                PointHit h = mesh_point_query(b.meshes[g.mesh], prev, c.status, radTolMesh);
                if (h.dist < radTolMesh && h.dist >= 0) add(h.cp, h.normal, h.tri, g.mesh);
            }
        }
        b.vcCount[(size_t)g.countBase + (i - g.vBegin)] = (uint8_t)n;
    }
}

// GridSDF::QueryTriangle, Frank-Wolfe (Physics/ClothCollisionSDF.h:148-205)
__device__ float sdf_query_triangle(const VColl& g, V3 a, V3 bb, V3 cc, V3& cpOut, V3& n, V3& coords)
{
    V3 cp = 0.33f * (a + bb + cc);
    float distOld = 0;
    for (int i = 1; i < 100; i++)
    {
        float dist = sdf_value(g, cp);
        if (dist == FLT_MAX) return FLT_MAX;
        V3 gr = sdf_grad(g, cp);
        float dA = dot(a, gr), dB = dot(bb, gr), dC = dot(cc, gr);
        float d = dA; V3 s = a;
        if (dB < d) { d = dB; s = bb; }
        if (dC < d) { d = dC; s = cc; }
        if (distOld > 0)
        {
            float rel = fabsf(distOld - dist) / distOld;
            if (rel < 0.0001f) break;
        }
        distOld = dist;
        float alpha = 2.f / (i + 2.f);
        cp += alpha * (s - cp);
    }
    float v = sdf_value(g, cp);
    V3 gr = normalized(sdf_grad(g, cp));
    n = gr;
    cpOut = cp - v * gr;
    V3 v0 = bb - a, v1 = cc - a, v2 = cp - a;
    float d00 = lensq(v0), d01 = dot(v0, v1), d11 = lensq(v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    float denom = d00 * d11 - d01 * d01;
    coords.y = (d11 * d20 - d01 * d21) / denom;
    coords.z = (d00 * d21 - d01 * d20) / denom;
    coords.x = 1.f - coords.y - coords.z;
    return v;
}

// Triangle and edge contacts against sphere / SDF / mesh colliders
// (SDFCollisions edge + triangle parts, Physics/ClothCollision.cpp:472-579;
// MeshCollisions triangle + edge parts, :137-196). One thread per cloth
// triangle or edge per collider; results go to per-item slots.
__global__ void k_tri_colliders(DevCloth c, SolverParams P, Buffers b, VColl g, int slotColl)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= c.T) return;
    const uint32_t i1 = c.tri[3 * t], i2 = c.tri[3 * t + 1], i3 = c.tri[3 * t + 2];
    const size_t slot = (size_t)slotColl * c.T + t;
    b.tcFlag[slot] = 0;
    V3 a = ld3(c.prev, i1), bb = ld3(c.prev, i2), cc = ld3(c.prev, i3);
    float tv1 = len(ld3(c.prev, i1) - ld3(c.pos, i1));
    float tv2 = len(ld3(c.prev, i2) - ld3(c.pos, i2));
    float tv3 = len(ld3(c.prev, i3) - ld3(c.pos, i3));
    float tvm = mx(tv1, mx(tv2, tv3));
    TC rec;
    rec.idx = make_uint4(i1, i2, i3, (uint32_t)t | ((uint32_t)min(slotColl, 255) << 24));   // .w: triangle, collider slot
    rec.lam = make_float2(0.f, 0.f);
    if (g.type == 4)
    {
        // MeshCollisions: per-triangle threshold with 1.2 x travel (ClothCollision.cpp:137-160)
        float rt = P.thickness + mx(P.tolerance, tvm * 1.2f);
        VtxHit h = mesh_triangle_query(b.meshes[g.mesh], a, bb, cc, c.status, rt);
        if (h.dist < rt && h.dist >= 0)
        {
            rec.point = f4(h.cpMesh, 0.f); rec.normal = f4(h.normal, 0.f);
            rec.w = make_float4(h.bary.x, h.bary.y, h.bary.z, 0.f);
            rec.feature = h.vertex; rec.mesh = g.mesh;
            b.tcSlot[slot] = rec; b.tcFlag[slot] = 1;
        }
        return;
    }
    const bool handleBorder = ((P.flags & CF_VERTICES) == 0) || ((P.flags & CF_EDGES) == 0);
    const float eps = 0.001f;
    V3 cp, n, coords;
    float dist;
    if (g.type == 7) dist = sdf_query_triangle(g, a, bb, cc, cp, n, coords);
    else
    {
        V3 ctr = mk(g.a.x, g.a.y, g.a.z), pt;
        closest_point_triangle(ctr, a, bb, cc, pt, coords);
        V3 delta = pt - ctr;
        float l = len(delta);
        delta = (1.f / l) * delta;
        n = delta;
        cp = ctr + g.a.w * delta;
        dist = l - g.a.w;
    }
    float radTol = P.thickness + mx(P.tolerance, tvm * 1.1f);
    if (dist < radTol && dist >= 0 && ((coords.x > eps && coords.y > eps && coords.z > eps) || handleBorder))
    {
        rec.point = f4(cp, 0.f); rec.normal = f4(n, 0.f);
        rec.w = make_float4(coords.x, coords.y, coords.z, 0.f);
        rec.feature = -1; rec.mesh = -1;
        b.tcSlot[slot] = rec; b.tcFlag[slot] = 1;
    }
}

__global__ void k_edge_colliders(DevCloth c, SolverParams P, Buffers b, VColl g, int slotColl)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= c.E) return;
    const int4 ed = c.edge[e];
    const size_t slot = (size_t)slotColl * c.E + e;
    b.ecFlag[slot] = 0;
    V3 p = ld3(c.prev, ed.x), q = ld3(c.prev, ed.y);
    EC rec;
    rec.idx = make_uint4(ed.x, ed.y, (uint32_t)e, (uint32_t)slotColl);   // .z: edge, .w: collider slot
    rec.lam = make_float2(0.f, 0.f);
    if (g.type == 4)
    {
        const float radTol = P.thickness + mx(P.tolerance, c.scal[0] * 1.5f);
        SegHit h = mesh_segment_query(b.meshes[g.mesh], p, q, c.status, radTol);
        if (h.dist < radTol && h.dist >= 0)
        {
            rec.point = f4(h.cpMesh, 0.f); rec.normal = f4(h.normal, 0.f);
            rec.w = make_float4(h.cs0, h.cs1, 0.f, 0.f);
            rec.feature = h.edge; rec.mesh = g.mesh;
            b.ecSlot[slot] = rec; b.ecFlag[slot] = 1;
        }
        return;
    }
    const bool handleBorder = (P.flags & CF_VERTICES) == 0;
    const float eps = 0.02f;
    float c0 = 0.f, c1 = 0.f, dist;
    V3 cp = mk(0.f, 0.f, 0.f), n = mk(0.f, 0.f, 0.f);
    if (g.type == 7) dist = 0.f; // GridSDF::QuerySegment is a stub returning 0
    else
    {
        float t;
        V3 ctr = mk(g.a.x, g.a.y, g.a.z);
        V3 ps = closest_point_segment(ctr, p, q, t);
        V3 delta = ps - ctr;
        float l = len(delta);
        delta = (1.f / l) * delta;
        n = delta;
        cp = ctr + g.a.w * delta;
        c0 = 1.0f - t; c1 = t;
        dist = l - g.a.w;
    }
    float tv1 = len(ld3(c.prev, ed.x) - ld3(c.pos, ed.x));
    float tv2 = len(ld3(c.prev, ed.y) - ld3(c.pos, ed.y));
    float radTol = P.thickness + mx(P.tolerance, mx(tv1, tv2) * 1.1f);
    if (dist < radTol && dist >= 0 && ((c0 > eps && c0 < 1.f - eps && c1 > eps && c1 < 1.f - eps) || handleBorder))
    {
        rec.point = f4(cp, 0.f); rec.normal = f4(n, 0.f);
        rec.w = make_float4(c0, c1, 0.f, 0.f);
        rec.feature = -1; rec.mesh = -1;
        b.ecSlot[slot] = rec; b.ecFlag[slot] = 1;
    }
}

// ------------------------------------------ colouring of multi-particle contacts
// Deterministic independent-set colouring (Jones-Plassmann with hashed
// priorities): in each round a contact whose key is the smallest among the
// still-uncoloured contacts on every particle it touches takes the round's
// colour. Contacts of one colour share no particle, so a colour is one
// parallel sweep and the result equals the sequential sweep in
// (colour, index) order, which is what the oracle's check mode runs.

__device__ __forceinline__ int contact_verts(const Buffers& b, int kind, int i, uint32_t* v)
{
    if (kind == 0) { uint4 x = b.ecList[i].idx; v[0] = x.x; v[1] = x.y; return 2; }
    if (kind == 1) { uint4 x = b.tcList[i].idx; v[0] = x.x; v[1] = x.y; v[2] = x.z; return 3; }
    uint4 x = (kind == 2 ? b.stList[i].idx : b.seList[i].idx);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w; return 4;
}

// colouring priority of contact i: a hash of its particle indices (relative to
// its instance's first particle in a batch), then the list index — so an
// instance's contacts get the same colours in a batch as alone (a batch list
// keeps each instance's contacts in their own relative order)
__device__ __forceinline__ unsigned long long contact_key(const DevCloth& c, const uint32_t* v, int nv, int i)
{
    const uint32_t base = c.vInst ? (uint32_t)c.instStart[c.vInst[v[0]]] : 0u;
    uint32_t h = 0x9e3779b9u;
    for (int k = 0; k < nv; k++) h = mix32(h ^ (v[k] - base));
    return ((unsigned long long)h << 32) | (uint32_t)i;
}

__device__ void place_by_colour(const ClassView& cv, int n);

__device__ void colour_class(const DevCloth& c, const Buffers& b, const ClassView& cv, int* status)
{
    __shared__ int sRemaining;
    const int n = *cv.count;
    for (int i = threadIdx.x; i < n; i += blockDim.x) cv.colour[i] = -1;
    if (threadIdx.x == 0) sRemaining = n;
    __syncthreads();
    int round = 0;
    while (sRemaining > 0 && round < MAX_COLOURS - 1)
    {
        for (int i = threadIdx.x; i < n; i += blockDim.x)
        {
            if (cv.colour[i] >= 0) continue;
            uint32_t v[4]; int nv = contact_verts(b, cv.kind, i, v);
            const unsigned long long key = contact_key(c, v, nv, i);
            for (int k = 0; k < nv; k++) atomicMin(&b.vmin[v[k]], key);
        }
        __syncthreads();
        int mine = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x)
        {
            if (cv.colour[i] >= 0) continue;
            uint32_t v[4]; int nv = contact_verts(b, cv.kind, i, v);
            const unsigned long long key = contact_key(c, v, nv, i);
            bool ok = true;
            for (int k = 0; k < nv; k++) ok = ok && (b.vmin[v[k]] == key);
            if (ok) { cv.colour[i] = MAX_COLOURS + round; mine++; }   // tentative mark
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x)
        {
            int col = cv.colour[i];
            if (col >= 0 && col != MAX_COLOURS + round) continue;
            uint32_t v[4]; int nv = contact_verts(b, cv.kind, i, v);
            for (int k = 0; k < nv; k++) b.vmin[v[k]] = ~0ull;
            if (col == MAX_COLOURS + round) cv.colour[i] = round;
        }
        __shared__ int sCount;
        if (threadIdx.x == 0) sCount = 0;
        __syncthreads();
        if (mine) atomicAdd(&sCount, mine);
        __syncthreads();
        if (threadIdx.x == 0) sRemaining -= sCount;
        __syncthreads();
        round++;
    }
    if (sRemaining > 0)
    {
        // not expected for contact graphs of bounded degree: the rest go to the
        // last colour, which the solver runs on a single thread in list order
        if (threadIdx.x == 0) atomicOr(status, ST_COLOUR_OVERFLOW);
    }
    place_by_colour(cv, n);
}

// Triangle (class 1) and edge (class 0) collider contacts: the static colour of
// their cloth triangle / edge, offset by nColours per collider slot (two
// colliders can both touch one triangle); the last colour (MAX_COLOURS - 1) is
// the serial bucket. Contacts of one colour share no particle.
__device__ void static_colour_class(const DevCloth& c, const Buffers& b, const ClassView& cv)
{
    const int n = *cv.count;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
    {
        int col;
        if (cv.kind == 1)
        {
            const uint32_t w = b.tcList[i].idx.w;
            col = c.triColour[w & 0xffffffu] + c.nTriColours * (int)(w >> 24);
        }
        else
        {
            const uint4 x = b.ecList[i].idx;
            col = c.edgeColour[x.z] + c.nEdgeColours * (int)x.w;
        }
        cv.colour[i] = min(col, MAX_COLOURS - 1);
    }
    __syncthreads();
    place_by_colour(cv, n);
}

// histogram of the colours + exclusive scan + placement: order[] lists each
// colour's contacts contiguously, start[] gives the colour ranges
__device__ void place_by_colour(const ClassView& cv, int n)
{
    __shared__ int sHist[MAX_COLOURS + 1];
    __shared__ int sCursor[MAX_COLOURS + 1];
    for (int k = threadIdx.x; k <= MAX_COLOURS; k += blockDim.x) sHist[k] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
    {
        int col = cv.colour[i];
        if (col < 0) { col = MAX_COLOURS - 1; cv.colour[i] = col; }
        atomicAdd(&sHist[col], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int acc = 0;
        for (int k = 0; k < MAX_COLOURS; k++) { cv.start[k] = acc; sCursor[k] = acc; acc += sHist[k]; }
        cv.start[MAX_COLOURS] = acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
    {
        int pos = atomicAdd(&sCursor[cv.colour[i]], 1);
        cv.order[pos] = i;
    }
    __syncthreads();
}


__global__ void __launch_bounds__(1024) k_colour(DevCloth c, Buffers b, ColourArgs a)
{
    for (int k = 0; k < 4; k++)
    {
        if (a.cls[k].kind <= 1) static_colour_class(c, b, a.cls[k]);
        else colour_class(c, b, a.cls[k], c.status);
    }
}

// residual-target mode, per-colour path: after iteration `iter` the residual
// word (float bits in scal[11]) decides whether the loop is done
__global__ void k_residual_exit(DevCloth c, SolverParams P, int iter)
{
    unsigned* word = reinterpret_cast<unsigned*>(c.scal + 11);
    const float res = __uint_as_float(*word);
    *word = 0u;
    if (!gs_done(c) && res <= P.resTol) c.scal[8] = 1.f;
}

// total iterations of the substeps since the last read (scal[10])
__global__ void k_iteration_total(DevCloth c)
{
    c.scal[10] += c.scal[9];
}

// ----------------------------------------------------------------- scans
constexpr int SCAN_T = 256, SCAN_ITEMS = 4, SCAN_TILE = SCAN_T * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sWarp, int& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) sWarp[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        int nw = blockDim.x >> 5;
        int w = lane < nw ? sWarp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
        if (lane < nw) sWarp[lane] = w;
    }
    __syncthreads();
    int warpPrefix = warp ? sWarp[warp - 1] : 0;
    total = sWarp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warpPrefix + x - v;
}

__global__ void k_scan_reduce(const int* in, int n, int* blockSums)
{
    __shared__ int sWarp[32];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) if (base + k < n) s += in[base + k];
    int total;
    block_exclusive_scan(s, sWarp, total);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

__global__ void k_scan_top(int* blockSums, int nb, int* total)
{
    __shared__ int sWarp[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += blockDim.x)
    {
        int i = base + threadIdx.x;
        int v = i < nb ? blockSums[i] : 0;
        int t;
        int ex = block_exclusive_scan(v, sWarp, t);
        if (i < nb) blockSums[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += t;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_down(const int* in, int* out, int n, const int* blockSums)
{
    __shared__ int sWarp[32];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int vals[SCAN_ITEMS];
    int s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) { vals[k] = (base + k < n) ? in[base + k] : 0; s += vals[k]; }
    int total;
    int ex = block_exclusive_scan(s, sWarp, total) + blockSums[blockIdx.x];
    for (int k = 0; k < SCAN_ITEMS; k++) { if (base + k < n) out[base + k] = ex; ex += vals[k]; }
}

void scan_ints(cudaStream_t s, const int* in, int* out, int n, int* total, int* tmp)
{
    int nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb < 1) nb = 1;
    k_scan_reduce<<<nb, SCAN_T, 0, s>>>(in, n, tmp);
    k_scan_top<<<1, 1024, 0, s>>>(tmp, nb, total);
    k_scan_down<<<nb, SCAN_T, 0, s>>>(in, out, n, tmp);
}

// gather items with count[i] records from slots[i*K + k] to dense[base + off[i] + k]
template <typename R>
__global__ void k_compact(const int* cnt, const int* off, const R* slots, int K, R* dense, int n, const int* base, int cap, int* status, int ovfBit)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int m = cnt[i];
    if (m == 0) return;
    int o = off[i] + (base ? *base : 0);
    for (int k = 0; k < m; k++)
    {
        if (o + k < cap) dense[o + k] = slots[(size_t)i * K + k];
        else atomicOr(status, ovfBit);
    }
}

__global__ void k_add_counts(int* dst, const int* a, const int* b, int cap)
{
    if (threadIdx.x == 0) { int v = *a + (b ? *b : 0); *dst = v < cap ? v : cap; }
}

// ----------------------------------------------------------- LBVH refit
// Leaf boxes: kind 0 = triangle over prev positions, 1 = edge over prev
// positions, 2 = swept triangle (prev and pos, extruded by tol), 3 = swept edge.
// The swept constructions are those of ClothModel::ComputeTree
// (Physics/ClothCollision.cpp:256-321).
__device__ __forceinline__ Box leaf_box(const DevCloth& c, int kind, int prim, float tol)
{
    Box b = Box::empty();
    if (kind == 0 || kind == 2)
    {
        uint32_t i1 = c.tri[3 * prim], i2 = c.tri[3 * prim + 1], i3 = c.tri[3 * prim + 2];
        b.add(ld3(c.prev, i1)); b.add(ld3(c.prev, i2)); b.add(ld3(c.prev, i3));
        if (kind == 2) { b.add(ld3(c.pos, i1)); b.add(ld3(c.pos, i2)); b.add(ld3(c.pos, i3)); b.extrude(tol); }
    }
    else
    {
        int4 e = c.edge[prim];
        if (kind == 1) { b.add(ld3(c.prev, e.x)); b.add(ld3(c.prev, e.y)); }
        else { b.add(ld3(c.pos, e.x)); b.add(ld3(c.pos, e.y)); b.add(ld3(c.prev, e.x)); b.add(ld3(c.prev, e.y)); b.extrude(tol); }
    }
    return b;
}

// Bottom-up refit with one atomic per internal node: the second child to
// arrive builds the parent's box and continues upwards (no waiting). The
// atomic is acquire-release (it publishes this thread's box and makes the
// sibling's visible), the arriving thread keeps its own box in registers and
// loads only the sibling's, and it puts the counter back to zero for the next
// refit (counters start at zero when the tree is allocated).
// a child's box into its half of the parent's record (the link and maximum
// words after it are static)
__device__ __forceinline__ void store_child_box(float4* rec, int parent, int node, const Box& b)
{
    float4* h = rec + 4 * (size_t)parent + (node == parent + 1 ? 0 : 2);
    h[0] = make_float4(b.lo.x, b.lo.y, b.lo.z, b.hi.x);
    *reinterpret_cast<float2*>(h + 1) = make_float2(b.hi.y, b.hi.z);
}

__global__ void k_bvh_refit(DevBVH t, DevCloth c, int kind, float tol)
{
    int prim = blockIdx.x * blockDim.x + threadIdx.x;
    if (prim >= t.numLeaves) return;
    int node = t.leafNode[prim];
    Box b = leaf_box(c, kind, prim, tol);
    t.lo[node] = f4(b.lo, __int_as_float(~prim));
    t.hi[node] = f4(b.hi, __int_as_float(node + 1));
    int p = t.parent[node];
    if (p >= 0) store_child_box(t.rec, p, node, b);
    while (p >= 0)
    {
        cuda::atomic_ref<int, cuda::thread_scope_device> visit(t.visit[p]);
        if (visit.fetch_add(1, cuda::memory_order_acq_rel) == 0) return;
        visit.store(0, cuda::memory_order_relaxed);
        const int l = p + 1, r = t.child[p];
        const int sib = node == l ? r : l;
        const float4 sl = __ldcg(&t.lo[sib]), sh = __ldcg(&t.hi[sib]);
        const Box o = {mk(sl.x, sl.y, sl.z), mk(sh.x, sh.y, sh.z)};
        const Box& L = node == l ? b : o;
        const Box& R = node == l ? o : b;
        Box m;
        m.lo = vmin(L.lo, R.lo);
        m.hi = vmax(L.hi, R.hi);
        b = m;
        t.lo[p] = f4(b.lo, __int_as_float(r));
        t.hi[p] = f4(b.hi, __int_as_float(t.escape[p]));
        const int gp = t.parent[p];
        if (gp >= 0) store_child_box(t.rec, gp, p, b);
        node = p;
        p = gp;
    }
}


// Stackless preorder traversal with escape indices; calls f(prim) for every
// leaf whose box overlaps q (AabbOverlap3D on the leaf box itself). A node is
// one round trip: two 16-byte loads carry its box and its links. With above >= 0
// subtrees holding only primitives <= above are skipped (the callers reject them).
template <typename F>
__device__ __forceinline__ void bvh_query(const DevBVH& t, const Box& q, F&& f, int above = -1, int root = 0)
{
    int node = root;
    const int end = t.instRoot ? __float_as_int(__ldg(&t.hi[root]).w) : t.numNodes;   // the root's escape
    while (node < end)
    {
        const float4 lo = __ldg(&t.lo[node]), hi = __ldg(&t.hi[node]);
        const int ch = __float_as_int(lo.w), esc = __float_as_int(hi.w);
        bool hit = !(hi.x < q.lo.x || hi.y < q.lo.y || hi.z < q.lo.z || q.hi.x < lo.x || q.hi.y < lo.y || q.hi.z < lo.z);
        if (above >= 0 && hit) hit = __ldg(&t.maxPrim[node]) > above;
        if (hit)
        {
            if (ch < 0) { f(~ch); node = esc; }
            else node = node + 1;
        }
        else node = esc;
    }
}

// Child records: every internal node keeps, for each of its two children, one
// 32-byte half with the child's box, its link (node index, or ~primitive for a
// leaf) and the largest primitive index below it, so one step of a walk is two
// 256-bit loads from one 64-byte record (the refit writes the boxes, the links
// and maxima are static).
struct ChildRec { float lx, ly, lz, hx, hy, hz; int link, maxPrim; };

__device__ __forceinline__ ChildRec ld_child(const float4* rec, int node, int side)
{
    const float* a = reinterpret_cast<const float*>(rec + 4 * (size_t)node + 2 * side);
    float v[8];
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
        : "l"(a));
    ChildRec r;
    r.lx = v[0]; r.ly = v[1]; r.lz = v[2]; r.hx = v[3]; r.hy = v[4]; r.hz = v[5];
    r.link = __float_as_int(v[6]); r.maxPrim = __float_as_int(v[7]);
    return r;
}

__device__ __forceinline__ bool overlaps(const ChildRec& c, const Box& q)
{
    return !(c.hx < q.lo.x || c.hy < q.lo.y || c.hz < q.lo.z || q.hi.x < c.lx || q.hi.y < c.ly || q.hi.z < c.lz);
}

// Per-thread traversal that tests both children of an entered node in one round
// trip (the node's two child records) and keeps the second one on a short stack:
// the dependent-load chain is the number of entered internal nodes, about a
// third of the stackless walk's. Reports the same leaf set as bvh_query, in a
// different order. A median-split tree over n < 2^31 leaves is at most 31 deep,
// so the 32-entry stack cannot overflow. A walk ends early once *stop is set
// (by f).
template <typename F>
__device__ __forceinline__ void bvh_query2(const DevBVH& t, const Box& q, bool active, F&& f, int above = -1, int root = 0,
                                           const bool* stop = nullptr)
{
    if (!active || t.numNodes == 0) return;
    const float4 rlo = __ldg(&t.lo[root]), rhi = __ldg(&t.hi[root]);
    const bool rootHit = !(rhi.x < q.lo.x || rhi.y < q.lo.y || rhi.z < q.lo.z || q.hi.x < rlo.x || q.hi.y < rlo.y ||
                           q.hi.z < rlo.z);
    if (!rootHit || (above >= 0 && __ldg(&t.maxPrim[root]) <= above)) return;
    if (__float_as_int(rlo.w) < 0) { f(~__float_as_int(rlo.w)); return; }
    int stack[32];
    int sp = 0;
    int node = root;
    while (!(stop && *stop))
    {
        const ChildRec cl = ld_child(t.rec, node, 0), cr = ld_child(t.rec, node, 1);
        bool oL = overlaps(cl, q) && (above < 0 || cl.maxPrim > above);
        bool oR = overlaps(cr, q) && (above < 0 || cr.maxPrim > above);
        if (oL && cl.link < 0) { f(~cl.link); oL = false; }
        if (oR && cr.link < 0) { f(~cr.link); oR = false; }
        if (oL)
        {
            if (oR && sp < 32) stack[sp++] = cr.link;
            node = cl.link;
        }
        else if (oR) node = cr.link;
        else
        {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
}

// Warp-packet form of bvh_query2: the 32 lanes (spatially adjacent queries in
// the same tree) walk it together, testing both children of an entered node per
// step; a child is entered when any lane's box overlaps it (ballot), so every
// record load is one broadcast request instead of up to 32 scattered ones, at
// the price of visiting the union of the lanes' nodes. Each lane reports exactly
// its own leaves. All 32 lanes must call it; a warp whose lanes start in
// different trees (a batch instance boundary) takes the per-lane walk. A lane
// whose *stop is set (by f) stops reporting and no longer steers the walk.
template <typename F>
__device__ __forceinline__ void bvh_query2_warp(const DevBVH& t, const Box& q, bool active, F&& f, int above, int root,
                                                const bool* stop = nullptr)
{
    const unsigned full = 0xffffffffu;
    const unsigned act = __ballot_sync(full, active);
    if (!act) return;
    const int r0 = __shfl_sync(full, root, __ffs(act) - 1);
    if (!__all_sync(full, !active || root == r0)) { bvh_query2(t, q, active, f, above, root, stop); return; }
    const float4 rlo = __ldg(&t.lo[r0]), rhi = __ldg(&t.hi[r0]);
    const bool rootHit = active &&
                         !(rhi.x < q.lo.x || rhi.y < q.lo.y || rhi.z < q.lo.z || q.hi.x < rlo.x || q.hi.y < rlo.y ||
                           q.hi.z < rlo.z) &&
                         (above < 0 || __ldg(&t.maxPrim[r0]) > above);
    if (__float_as_int(rlo.w) < 0) { if (rootHit) f(~__float_as_int(rlo.w)); return; }
    if (!__any_sync(full, rootHit)) return;
    int stack[32];
    int sp = 0;
    int node = r0;
    while (true)
    {
        const ChildRec cl = ld_child(t.rec, node, 0), cr = ld_child(t.rec, node, 1);
        const bool live = active && !(stop && *stop);
        bool oL = live && overlaps(cl, q) && (above < 0 || cl.maxPrim > above);
        bool oR = live && overlaps(cr, q) && (above < 0 || cr.maxPrim > above);
        if (cl.link < 0) { if (oL) f(~cl.link); oL = false; }
        if (cr.link < 0) { if (oR) f(~cr.link); oR = false; }
        const bool anyL = __any_sync(full, oL), anyR = __any_sync(full, oR);
        if (anyL)
        {
            if (anyR && sp < 32) stack[sp++] = cr.link;
            node = cl.link;
        }
        else if (anyR) node = cr.link;
        else
        {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
}

// Cooperative walk of ONE query box by a group of W lanes (W a power of two up
// to 32; every lane of the group holds the same box), for queries with long
// candidate lists: each step the group takes up to W entered nodes from its
// stack, each lane tests both children of its node (one round trip), and the
// entered internal children are pushed as a new group. Only the top group is
// ever popped, so group g holds nodes of depth g exactly: at most depth groups
// of at most 2W entries, the bound the caller sizes the stack (node indices)
// by. f(a, b) is called by all lanes of the group once per step with the lane's
// overlapping leaves (-1 for none) and returns false to end the walk (uniformly
// across the group). The leaf set is bvh_query2's.
template <int W, typename F>
__device__ __forceinline__ void bvh_query_coop(const DevBVH& t, const Box& q, int above, int root, int* stack, int cap,
                                               int* groups, int gcap, int* status, F&& f)
{
    const int lane = threadIdx.x & 31, sl = lane & (W - 1);
    const unsigned mask = W == 32 ? 0xffffffffu : (((1u << W) - 1u) << (lane & ~(W - 1)));
    const unsigned lt = (1u << lane) - 1u;
    const float4 rlo = __ldg(&t.lo[root]), rhi = __ldg(&t.hi[root]);
    const bool rootHit = !(rhi.x < q.lo.x || rhi.y < q.lo.y || rhi.z < q.lo.z || q.hi.x < rlo.x || q.hi.y < rlo.y ||
                           q.hi.z < rlo.z);
    if (!rootHit || (above >= 0 && __ldg(&t.maxPrim[root]) <= above)) return;
    const int rch = __float_as_int(rlo.w);
    if (rch < 0) { f(sl == 0 ? ~rch : -1, -1); return; }
    if (sl == 0) { stack[0] = root; groups[0] = 1; }
    int sp = 1, m = 1;
    __syncwarp(mask);
    while (m > 0)
    {
        const int g = groups[m - 1];
        const int take = min(g, W);
        const int node = sl < take ? stack[sp - 1 - sl] : -1;
        __syncwarp(mask);
        sp -= take;
        int leafA = -1, leafB = -1, linkL = 0, linkR = 0;
        bool pushL = false, pushR = false;
        if (node >= 0)
        {
            const ChildRec cl = ld_child(t.rec, node, 0), cr = ld_child(t.rec, node, 1);
            const bool oL = overlaps(cl, q) && (above < 0 || cl.maxPrim > above);
            const bool oR = overlaps(cr, q) && (above < 0 || cr.maxPrim > above);
            linkL = cl.link;
            linkR = cr.link;
            if (oL) { if (linkL < 0) leafA = ~linkL; else pushL = true; }
            if (oR) { if (linkR < 0) leafB = ~linkR; else pushR = true; }
        }
        if (!f(leafA, leafB)) break;
        const unsigned bl = __ballot_sync(mask, pushL), br = __ballot_sync(mask, pushR);
        const int nl = __popc(bl), cnt = nl + __popc(br);
        if (g == take) m--;
        else if (sl == 0) groups[m - 1] = g - take;
        if (cnt > 0)
        {
            if (sp + cnt > cap || m >= gcap)
            {
                // unreachable for a tree of the stated depth; recorded, never written out of bounds
                if (sl == 0) atomicOr(status, ST_CCD_OVERFLOW);
                break;
            }
            if (pushL) stack[sp + __popc(bl & lt)] = linkL;
            if (pushR) stack[sp + nl + __popc(br & lt)] = linkR;
            if (sl == 0) groups[m] = cnt;
            sp += cnt;
            m++;
        }
        __syncwarp(mask);
    }
    __syncwarp(mask);
}

// tree root for a query on particle v: its instance's tree in a batch
__device__ __forceinline__ int tree_root(const DevCloth& c, const DevBVH& t, int v)
{
    return t.instRoot ? t.instRoot[c.vInst[v]] : 0;
}

// ------------------------------------------------------ self proximity
// Voronoi-region filters of the live self-collision query
// (Geometry/VoronoiRegions.cpp:11-113) on the collision mesh (prev positions,
// normals as of the last mesh update).
__device__ bool in_vertex_vr(const DevCloth& c, V3 p, int vid)
{
    V3 v = ld3(c.prev, vid);
    float side = 1;
    if (dot(ld3(c.prevN, vid), p - v) < 0) side = -1;
    const float eps = 0.1f;
    for (int k = c.eRingStart[vid]; k < c.eRingStart[vid + 1]; k++)
    {
        int4 ed = c.edge[c.eRing[k]];
        V3 e = normalized(ld3(c.prev, ed.x) - ld3(c.prev, ed.y));
        if (ed.y != vid) e = -e;
        float d = dot(e, p - v);
        if (side > 0 && d < -eps) return false;
        if (side < 0 && d > eps) return false;
    }
    return true;
}

__device__ bool in_triangle_vr(const DevCloth& c, V3 p, int t)
{
    V3 v1 = ld3(c.prev, c.tri[3 * t]), v2 = ld3(c.prev, c.tri[3 * t + 1]), v3 = ld3(c.prev, c.tri[3 * t + 2]);
    V3 e1 = v2 - v1, e2 = v3 - v2, e3 = v1 - v3;
    V3 n = ld3(c.prevTriN, t);
    V3 h1 = cross(e1, n), h2 = cross(e2, n), h3 = cross(e3, n);
    float d1 = dot(h1, p - v1), d2 = dot(h2, p - v2), d3 = dot(h3, p - v3);
    bool s1 = signbit(d1), s2 = signbit(d2), s3 = signbit(d3);
    return (s1 == s2) == s3;   // the reference's chained comparison
}

__device__ bool in_edge_vr(const DevCloth& c, V3 p, int eid)
{
    const float eps = 0.002f;
    int4 ed = c.edge[eid];
    V3 a = ld3(c.prev, ed.x), b = ld3(c.prev, ed.y);
    V3 e = normalized(b - a);
    float d3 = dot(e, p - a), d4 = dot(e, p - b);
    if (d3 < 0 || d4 > 0) return false;
    if (c.edgeSwapped[eid]) e = -e;
    if (ed.w >= 0)
    {
        V3 h1 = normalized(cross(e, ld3(c.prevTriN, ed.z)));
        V3 h2 = normalized(-cross(e, ld3(c.prevTriN, ed.w)));
        float d1 = dot(h1, p - a), d2 = dot(h2, p - a);
        if (d1 < -eps || d2 < -eps) return false;
    }
    else
    {
        V3 h1 = normalized(cross(e, ld3(c.prevTriN, ed.z)));
        if (dot(h1, p - a) < -eps) return false;
    }
    return true;
}

__device__ bool adjacent(const DevCloth& c, int a, int b)
{
    for (int k = c.vRingStart[a]; k < c.vRingStart[a + 1]; k++) if (c.vRing[k] == b) return true;
    return false;
}

// CheckAdjacency (Geometry/ClosestPointsBetweenMeshes.cpp:441-461)
__device__ bool check_adjacency(const DevCloth& c, int vtx, int t, int region)
{
    int i1 = c.tri[3 * t], i2 = c.tri[3 * t + 1], i3 = c.tri[3 * t + 2];
    if (i1 == vtx || i2 == vtx || i3 == vtx) return true;
    if (region == TR_VERTEX_A && adjacent(c, vtx, i1)) return true;
    if (region == TR_VERTEX_B && adjacent(c, vtx, i2)) return true;
    if (region == TR_VERTEX_C && adjacent(c, vtx, i3)) return true;
    if (region == TR_EDGE_AB && (adjacent(c, vtx, i1) && adjacent(c, vtx, i2))) return true;
    if (region == TR_EDGE_BC && (adjacent(c, vtx, i2) && adjacent(c, vtx, i3))) return true;
    if (region == TR_EDGE_AC && (adjacent(c, vtx, i1) && adjacent(c, vtx, i3))) return true;
    return false;
}

// Self vertex-triangle proximity for one vertex: the triangles within radTol
// come from the BVH (a superset: every triangle at distance <= radTol has a
// box overlapping the query cube); they are then visited in increasing
// triangle index, which is the brute-force loop order of
// ClosestPointsOnMeshToPoint (Geometry/ClosestPointOnMesh.cpp:142-246), so the
// Voronoi filters and the first-feature dedup decide exactly as there.
__global__ void __launch_bounds__(128) k_self_vt(DevCloth c, SolverParams P, Buffers b, DevBVH tb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const float radTol = P.thickness + mx(P.tolerance, c.scal[0] * 1.5f);
    const V3 p = ld3(c.prev, i);
    const float r = radTol * 1.0001f + 1e-6f;
    Box q; q.lo = p - mk(r, r, r); q.hi = p + mk(r, r, r);
    int cand[KCAND];
    int nc = 0;
    bool ovf = false;
    bvh_query(tb, q, [&](int t) { if (nc < KCAND) cand[nc++] = t; else ovf = true; }, -1, tree_root(c, tb, i));
    if (ovf) atomicOr(c.status, ST_SELF_VT_OVERFLOW);
    for (int a = 1; a < nc; a++)   // insertion sort: small lists
    {
        int v = cand[a], j = a - 1;
        while (j >= 0 && cand[j] > v) { cand[j + 1] = cand[j]; j--; }
        cand[j + 1] = v;
    }
    const bool isBorder = c.vBorder[i] != 0;
    int resType[KRES], resFeat[KRES];
    int nres = 0, nout = 0;
    SCt* out = b.stSlot + (size_t)i * KVT;
    for (int a = 0; a < nc; a++)
    {
        const int t = cand[a];
        const int i0 = c.tri[3 * t], i1 = c.tri[3 * t + 1], i2 = c.tri[3 * t + 2];
        V3 va = ld3(c.prev, i0), vb = ld3(c.prev, i1), vc = ld3(c.prev, i2);
        V3 coords, pt;
        int region = closest_point_triangle(p, va, vb, vc, pt, coords);
        V3 delta = p - pt;
        float dist = len(delta);
        if (dist > radTol) continue;
        if (dist == 0) continue;
        bool inVR = in_vertex_vr(c, pt, i);
        int rtype = -1, feature = -1;
        if (region == TR_FACE_INTERIOR)
        {
            if (!(inVR || in_triangle_vr(c, p, t))) continue;
            rtype = 0;
        }
        if (region == TR_EDGE_AB || region == TR_EDGE_BC || region == TR_EDGE_AC)
        {
            int e = c.triE[3 * t + (region == TR_EDGE_AB ? 0 : (region == TR_EDGE_BC ? 1 : 2))];
            if (!(c.edge[e].w < 0) && !(inVR || in_edge_vr(c, p, e))) continue;
            rtype = 1; feature = e;
        }
        if (region == TR_VERTEX_A || region == TR_VERTEX_B || region == TR_VERTEX_C)
        {
            int vv = region == TR_VERTEX_A ? i0 : (region == TR_VERTEX_B ? i1 : i2);
            if (!isBorder && !(inVR || in_vertex_vr(c, p, vv))) continue;
            rtype = 2; feature = vv;
        }
        if (feature >= 0)
        {
            bool found = false;
            for (int k = 0; k < nres; k++) if (resType[k] == rtype && resFeat[k] == feature) { found = true; break; }
            if (found) continue;
        }
        // only edge and vertex features take part in the dedup (faces carry -1)
        if (feature >= 0)
        {
            if (nres < KRES) { resType[nres] = rtype; resFeat[nres] = feature; nres++; }
            else { atomicOr(c.status, ST_SELF_VT_OVERFLOW); continue; }
        }
        // ClosestPoints(self) then MeshCollisions: drop adjacent features,
        // keep 0 <= dist < radTol (ClosestPointsBetweenMeshes.cpp:553-563,
        // ClothCollision.cpp:113-131)
        if (check_adjacency(c, i, t, region)) continue;
        if (!(dist < radTol && dist >= 0)) continue;
        SCt rec;
        rec.idx = make_uint4(i0, i1, i2, i);
        V3 nrm = (1.f / dist) * delta;
        rec.normal = f4(nrm, 0.f);
        rec.side = signed_volume(p, va, vb, vc);
        rec.w = make_float4(coords.x, coords.y, coords.z, 0.f);
        rec.lam = make_float2(0.f, 0.f);
        rec.error = 0.f;
        if (nout < KVT) out[nout++] = rec;
        else atomicOr(c.status, ST_SELF_VT_OVERFLOW);
    }
    b.stCnt[i] = nout;
}

__device__ __forceinline__ bool same_triangle(const DevCloth& c, int v, int t)
{
    if (t < 0) return false;
    return v == (int)c.tri[3 * t] || v == (int)c.tri[3 * t + 1] || v == (int)c.tri[3 * t + 2];
}

// Self edge-edge proximity for one edge: nearest non-adjacent edge of higher
// index (ties -> lower index, as the strict < of the reference loop), then
// CheckEdgeAdjacency (Geometry/ClosestPointOnMesh.cpp:499-542,
// ClosestPointsBetweenMeshes.cpp:474-536,568-591).
__global__ void __launch_bounds__(128) k_self_ee(DevCloth c, SolverParams P, Buffers b, DevBVH eb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.E) return;
    b.seFlag[i] = 0;
    const float radTol = P.thickness + mx(P.tolerance, c.scal[0] * 1.5f);
    const int4 e1 = c.edge[i];
    const V3 p = ld3(c.prev, e1.x), q = ld3(c.prev, e1.y);
    const float r = radTol * 1.0001f + 1e-6f;
    Box qb = Box::empty(); qb.add(p); qb.add(q);
    qb.lo = qb.lo - mk(r, r, r); qb.hi = qb.hi + mk(r, r, r);
    float best = FLT_MAX;
    int bestE = -1;
    bvh_query(eb, qb, [&](int e) {
        if (e <= i) return;
        int4 e2 = c.edge[e];
        if (e2.x == e1.x || e2.x == e1.y || e2.y == e1.x || e2.y == e1.y) return;
        float ps, pm; V3 cs, cm;
        closest_segm_segm(p, q, ld3(c.prev, e2.x), ld3(c.prev, e2.y), ps, pm, cs, cm);
        float dist = len(cs - cm);
        if (dist != 0 && (dist < best || (dist == best && e < bestE))) { best = dist; bestE = e; }
    }, i, tree_root(c, eb, e1.x));
    if (bestE < 0) return;
    const int4 e2 = c.edge[bestE];
    const V3 a = ld3(c.prev, e2.x), bb = ld3(c.prev, e2.y);
    float ps, pm; V3 cs, cm;
    int region = closest_segm_segm(p, q, a, bb, ps, pm, cs, cm);
    float dist = len(cs - cm);
    const float cs0 = 1.0f - ps, cs1 = ps, cm0 = 1.0f - pm, cm1 = pm;
    const float eps = 1e-5f;
    if ((region & ER_VERTEX_P1) != 0 || cs0 < eps)
        if (same_triangle(c, e1.x, e2.z) || same_triangle(c, e1.x, e2.w)) return;
    if ((region & ER_VERTEX_Q1) != 0 || cs1 < eps)
        if (same_triangle(c, e1.y, e2.z) || same_triangle(c, e1.y, e2.w)) return;
    if ((region & ER_VERTEX_P2) != 0 || cm0 < eps)
        if (same_triangle(c, e2.x, e1.z) || same_triangle(c, e2.x, e1.w)) return;
    if ((region & ER_VERTEX_Q2) != 0 || cm1 < eps)
        if (same_triangle(c, e2.y, e1.z) || same_triangle(c, e2.y, e1.w)) return;
    if (!(dist < radTol && dist >= 0)) return;
    SCt rec;
    rec.idx = make_uint4(e1.x, e1.y, e2.x, e2.y);
    V3 nrm = normalized(cm - cs);
    rec.normal = f4(nrm, 0.f);
    rec.side = signed_volume(p, q, a, bb);
    rec.w = make_float4(cs1, cm1, 0.f, 0.f);
    rec.lam = make_float2(0.f, 0.f);
    rec.error = 0.f;
    b.seSlot[i] = rec;
    b.seFlag[i] = 1;
}

// ---------------------------------------------------- continuous collision
// Broad phase: every (triangle, vertex) and (edge, edge) pair whose swept boxes
// overlap, with the Midphase's filters (vertex not on the triangle and not
// pinned; edges sharing no vertex), Physics/SelfCollisionDetector.cpp:60-135,
// but over all pairs rather than same-leaf pairs only. Pairs are listed per
// query: (vertex, triangle) and (edge, higher edge).
// Two passes: the first walks one query per thread and keeps up to KCCD
// candidates in the query's own slots; the queries that find more go to a list
// that the second pass walks one query per warp, storing the full lists in a
// shared pool. Lists stay in traversal order: only the (rare) hits are put in
// candidate order.
// A vertex query: its swept box and the triangles incident to it (held in
// registers, so a reported leaf costs no load).
struct VtQuery
{
    int i, nInc;
    bool pinned;
    Box box;
    int inc[KADJ];
    __device__ __forceinline__ void init(const DevCloth& c, int v, float tol)
    {
        i = v;
        const float4 p4 = c.pos[v];
        pinned = p4.w == 0.f;
        box = Box::empty(); box.add(ld3(c.prev, v)); box.add(mk(p4.x, p4.y, p4.z)); box.extrude(tol);
        const int r0 = c.vTriStart[v];
        nInc = c.vTriStart[v + 1] - r0;
#pragma unroll
        for (int k = 0; k < KADJ; k++) inc[k] = k < nInc ? c.vTri[r0 + k].x : -1;
    }
    __device__ __forceinline__ bool accept(const DevCloth& c, int t) const
    {
        if (nInc <= KADJ)
        {
            bool adj = false;
#pragma unroll
            for (int k = 0; k < KADJ; k++) adj |= inc[k] == t;
            return !adj;
        }
        return !((int)c.tri[3 * t] == i || (int)c.tri[3 * t + 1] == i || (int)c.tri[3 * t + 2] == i);
    }
};

// An edge query: its swept box and the edges sharing one of its vertices (both
// vertices' edge rings, in registers when they fit).
struct EeQuery
{
    int i;
    int4 e1;
    bool inRegs;
    Box box;
    int adjE[KADJ];
    __device__ __forceinline__ void init(const DevCloth& c, int e, float tol)
    {
        i = e;
        e1 = c.edge[e];
        box = Box::empty();
        box.add(ld3(c.pos, e1.x)); box.add(ld3(c.pos, e1.y)); box.add(ld3(c.prev, e1.x)); box.add(ld3(c.prev, e1.y));
        box.extrude(tol);
        const int a0 = c.eRingStart[e1.x], na = c.eRingStart[e1.x + 1] - a0;
        const int b0 = c.eRingStart[e1.y], nb = c.eRingStart[e1.y + 1] - b0;
        inRegs = na + nb <= KADJ;
#pragma unroll
        for (int k = 0; k < KADJ; k++)
            adjE[k] = !inRegs ? -1 : k < na ? c.eRing[a0 + k] : k < na + nb ? c.eRing[b0 + k - na] : -1;
    }
    __device__ __forceinline__ bool accept(const DevCloth& c, int e) const
    {
        if (e <= i) return false;
        if (inRegs)
        {
            bool adj = false;
#pragma unroll
            for (int k = 0; k < KADJ; k++) adj |= adjE[k] == e;
            return !adj;
        }
        const int4 e2 = c.edge[e];
        return !(e1.x == e2.x || e1.y == e2.y || e1.x == e2.y || e1.y == e2.x);
    }
};

// First pass: one query per thread (or per lane of a warp packet), at most KCCD
// candidates into the query's own slots. A query that finds more stops walking,
// keeps a count above KCCD and joins the overflow list for the second pass.
__global__ void __launch_bounds__(128) k_ccd_broad_vt(DevCloth c, SolverParams P, Buffers b, DevBVH tb, float tol)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g - (int)(threadIdx.x & 31) >= c.N) return;          // whole warp past the end
    const int i = g < c.N ? c.vQuery[g] : 0;
    bool active = g < c.N;
    if (active) b.ccdVtCnt[i] = 0;
    VtQuery Q;
    Q.init(c, i, tol);
    if (Q.pinned) active = false;
    int* out = b.ccdVtCand + (size_t)i * KCCD;
    int n = 0;
    bool stop = false;
    auto emitT = [&](int t) {
        if (!Q.accept(c, t)) return;
        if (n < KCCD) out[n] = t;
        if (++n > KCCD) stop = true;
    };
    if (b.broadWalk == BROAD_PACKET) bvh_query2_warp(tb, Q.box, active, emitT, -1, tree_root(c, tb, i), &stop);
    else bvh_query2(tb, Q.box, active, emitT, -1, tree_root(c, tb, i), &stop);
    if (!active) return;
    b.ccdVtCnt[i] = n;
    if (n > KCCD) b.ccdVtOvf[atomicAdd(b.ccdOvfN, 1)] = i;
}

__global__ void __launch_bounds__(128) k_ccd_broad_ee(DevCloth c, SolverParams P, Buffers b, DevBVH eb, float tol)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g - (int)(threadIdx.x & 31) >= c.E) return;
    const int i = g < c.E ? c.eQuery[g] : 0;
    const bool active = g < c.E;
    EeQuery Q;
    Q.init(c, i, tol);
    int* out = b.ccdEeCand + (size_t)i * KCCD;
    int n = 0;
    bool stop = false;
    auto emitE = [&](int e) {
        if (!Q.accept(c, e)) return;
        if (n < KCCD) out[n] = e;
        if (++n > KCCD) stop = true;
    };
    if (b.broadWalk == BROAD_PACKET) bvh_query2_warp(eb, Q.box, active, emitE, i, tree_root(c, eb, Q.e1.x), &stop);
    else bvh_query2(eb, Q.box, active, emitE, i, tree_root(c, eb, Q.e1.x), &stop);
    if (!active) return;
    b.ccdEeCnt[i] = n;
    if (n > KCCD) b.ccdEeOvf[atomicAdd(b.ccdOvfN + 1, 1)] = i;
}

// Second pass over the overflow list: one warp per query walks the tree
// cooperatively (bvh_query_coop) twice, counting its candidates, then writing
// them into a pool block of exactly that size. The lane order of a step and the
// step order are fixed, so each list (and the pair list) is deterministic.
template <bool VT>
__global__ void __launch_bounds__(CCD_COOP_THREADS) k_ccd_broad_coop(DevCloth c, SolverParams P, Buffers b, DevBVH t, float tol)
{
    extern __shared__ int sCoop[];
    const unsigned full = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int cap = CCD_COOP_GROUP * (t.depth + 1), gcap = t.depth + 2;
    int* stack = sCoop + warp * (cap + gcap);
    int* groups = stack + cap;
    const int nOvf = b.ccdOvfN[VT ? 0 : 1];
    const int* ovf = VT ? b.ccdVtOvf : b.ccdEeOvf;
    int* cnt = VT ? b.ccdVtCnt : b.ccdEeCnt;
    int* poolOff = VT ? b.ccdVtPoolOff : b.ccdEePoolOff;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int w = blockIdx.x * (blockDim.x >> 5) + warp; w < nOvf; w += warps)
    {
        const int i = ovf[w];
        VtQuery qv;
        EeQuery qe;
        int root, above;
        Box box;
        if (VT) { qv.init(c, i, tol); box = qv.box; root = tree_root(c, t, i); above = -1; }
        else { qe.init(c, i, tol); box = qe.box; root = tree_root(c, t, qe.e1.x); above = i; }
        auto ok = [&](int leaf) { return leaf >= 0 && (VT ? qv.accept(c, leaf) : qe.accept(c, leaf)); };
        int total = 0;
        bvh_query_coop<32>(t, box, above, root, stack, cap, groups, gcap, c.status, [&](int la, int lb) {
            total += __popc(__ballot_sync(full, ok(la))) + __popc(__ballot_sync(full, ok(lb)));
            return true;
        });
        int base = 0;
        if (lane == 0)
        {
            base = atomicAdd(b.ccdPoolUsed, total);
            if (base + total > b.ccdPoolCap) { atomicOr(c.status, ST_CCD_OVERFLOW); base = -1; }
        }
        base = __shfl_sync(full, base, 0);
        if (base < 0)
        {
            if (lane == 0) cnt[i] = 0;
            continue;
        }
        int* out = b.ccdPool + base;
        int pos = 0;
        bvh_query_coop<32>(t, box, above, root, stack, cap, groups, gcap, c.status, [&](int la, int lb) {
            const bool ka = ok(la), kb = ok(lb);
            const unsigned ba = __ballot_sync(full, ka), bb = __ballot_sync(full, kb);
            if (ka) out[pos + __popc(ba & lt)] = la;
            if (kb) out[pos + __popc(ba) + __popc(bb & lt)] = lb;
            pos += __popc(ba) + __popc(bb);
            return true;
        });
        if (lane == 0) { cnt[i] = total; poolOff[i] = base; }
        __syncwarp();
    }
}

size_t ccd_coop_smem(int depth)
{
    const int cap = CCD_COOP_GROUP * (depth + 1), gcap = depth + 2;
    return sizeof(int) * (size_t)(cap + gcap) * (CCD_COOP_THREADS / 32);
}

void ccd_kernel_setup()
{
    cudaFuncSetAttribute(k_ccd_broad_coop<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ccd_coop_smem(40));
    cudaFuncSetAttribute(k_ccd_broad_coop<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ccd_coop_smem(40));
}

// first pass in the walk the model uses (BROAD_* in launch.h)
static void launch_broad_pass1(cudaStream_t s, bool vt, const DevCloth& c, const SolverParams& P, const Buffers& b,
                               const DevBVH& t, float tol)
{
    const int n = vt ? c.N : c.E;
    if (vt) k_ccd_broad_vt<<<blocks_for(n, 128), 128, 0, s>>>(c, P, b, t, tol);
    else k_ccd_broad_ee<<<blocks_for(n, 128), 128, 0, s>>>(c, P, b, t, tol);
}

// expand per-query candidate lists (own slots, or the pool for long lists)
// into the dense pair list; one warp per query, coalesced copies
__global__ void k_ccd_pairs(const int* cnt, const int* off, const int* cand, const int* pool, const int* poolOff,
                            int n, int2* pairs, int cap, int* status, int* hitCnt)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    if (lane == 0) hitCnt[i] = 0;                 // counted by the narrow phase
    const int m = cnt[i], o = off[i];
    const int* src = m > KCCD ? pool + poolOff[i] : cand + (size_t)i * KCCD;
    for (int k = lane; k < m; k += 32)
    {
        if (o + k < cap) pairs[o + k] = make_int2(i, src[k]);
        else atomicOr(status, ST_CCD_OVERFLOW);
    }
}

// EvaluateFun_Coplanarity (Physics/SelfCollisionDetector.cpp:279-291)
__device__ __forceinline__ float coplanarity(float t, V3 x1, V3 x2, V3 x3, V3 x4, V3 v1, V3 v2, V3 v3, V3 v4)
{
    V3 z1 = x1 + t * v1, z2 = x2 + t * v2, z3 = x3 + t * v3, z4 = x4 + t * v4;
    V3 n1 = cross(z2 - z1, z3 - z1);
    return dot(n1, z4 - z1);
}

// CheckInterval, at most 40 bisections (SelfCollisionDetector.cpp:440-489)
__device__ bool check_interval(float ta, float tb, V3 x1, V3 x2, V3 x3, V3 x4, V3 v1, V3 v2, V3 v3, V3 v4, float& tx)
{
    float tx0 = ta, tx1 = tb;
    float fx0 = coplanarity(tx0, x1, x2, x3, x4, v1, v2, v3, v4);
    float fx1 = coplanarity(tx1, x1, x2, x3, x4, v1, v2, v3, v4);
    if (fx0 * fx1 > 0) return false;
    tx = tx0;
    for (int l = 0; l < 40; l++)
    {
        float tmid = 0.5f * (tx0 + tx1);
        float fmid = coplanarity(tmid, x1, x2, x3, x4, v1, v2, v3, v4);
        if (fabsf(fmid) < 0.01f) { tx = tmid; break; }
        if (fx0 * fmid < 0) { tx1 = tmid; fx1 = fmid; tx = tx0; }
        else if (fmid * fx1 < 0) { tx0 = tmid; fx0 = fmid; tx = tmid; }
        else return false;
    }
    return true;
}

// SolveCubic + FindInflexionPoints + CheckDegenerateCase (SelfCollisionDetector.cpp:293-438)
__device__ bool solve_cubic(V3 x1, V3 x2, V3 x3, V3 x4, V3 v1, V3 v2, V3 v3, V3 v4, float& toi)
{
    float f0 = coplanarity(0.f, x1, x2, x3, x4, v1, v2, v3, v4);
    if (fabsf(f0) < 0.001f) return false;
    V3 v10 = v1 - v4, v20 = v2 - v4, v30 = v3 - v4;
    V3 x10 = x1 - x4, x20 = x2 - x4, x30 = x3 - x4;
    float a = triple(v10, v20, v30);
    float b = triple(x10, v20, v30) + triple(v10, x20, v30) + triple(v10, v20, x30);
    float cc = triple(x10, x20, v30) + triple(x10, v20, x30) + triple(v10, x20, x30);
    if (fabsf(a) < 0.001f)
    {
        if (fabsf(b) < 0.001f) return false;
        float d = triple(x10, x20, x30);
        float discr = cc * cc - 4 * b * d;
        if (discr < 0) return false;
        if (discr == 0)
        {
            float t = -0.5f * cc / b;
            if (t < 0 || t > 1) return false;
            toi = t;
            return true;
        }
        float ds = sqrtf(discr);
        float t1 = 0.5f * (-cc - ds) / b, t2 = 0.5f * (-cc + ds) / b;
        float t = mn(t1, t2);
        if (t < 0 || t > 1) return false;
        toi = t;
        return true;
    }
    float discr = b * b - 3 * a * cc;
    int num;
    float ti1 = 0.f, ti2 = 0.f;
    if (discr < 0) num = 0;
    else if (discr == 0) { ti1 = ti2 = -b / (3 * a); num = 1; }
    else
    {
        float ds = sqrtf(discr);
        ti1 = (-b - ds) / (3 * a);
        ti2 = (-b + ds) / (3 * a);
        if (ti2 < ti1) { float tmp = ti1; ti1 = ti2; ti2 = tmp; }
        num = 2;
    }
#define CI(ta, tb) check_interval((ta), (tb), x1, x2, x3, x4, v1, v2, v3, v4, toi)
    bool coplanar = false;
    if (num == 0) coplanar = CI(0.f, 1.f);
    else if (num == 1)
    {
        if (ti1 < 0 || ti1 > 1) coplanar = CI(0.f, 1.f);
        else coplanar = CI(0.f, ti1) || CI(ti1, 1.f);
    }
    else
    {
        if (ti1 > 1 || ti2 < 0 || (ti1 < 0 && ti2 > 1)) coplanar = CI(0.f, 1.f);
        else if (ti1 < 0 && ti2 < 1) coplanar = CI(0.f, ti2) || CI(ti2, 1.f);
        else if (ti1 < 1 && ti2 > 1) coplanar = CI(0.f, ti1) || CI(ti1, 1.f);
        else if (ti1 > 0 && ti2 < 1) coplanar = CI(0.f, ti1) || CI(ti1, ti2) || CI(ti2, 1.f);
    }
#undef CI
    return coplanar;
}

// VertexTriangleTest + VertexTriangleCCD (SelfCollisionDetector.cpp:171-277) for
// pair k: 1 and the contact record on a hit, else 0
__device__ int ccd_vt_test(const DevCloth& c, const SolverParams& P, const Buffers& b, int k, SCt& rec)
{
    int2 pr = b.ccdVtPairs[k];
    const int vtx = pr.x, t = pr.y;
    const uint32_t i1 = c.tri[3 * t], i2 = c.tri[3 * t + 1], i3 = c.tri[3 * t + 2];
    V3 x1 = ld3(c.prev, i1), x2 = ld3(c.prev, i2), x3 = ld3(c.prev, i3), x4 = ld3(c.prev, vtx);
    V3 v1 = ld3(c.pos, i1) - x1, v2 = ld3(c.pos, i2) - x2, v3 = ld3(c.pos, i3) - x3, v4 = ld3(c.pos, vtx) - x4;
    float toi;
    if (!solve_cubic(x1, x2, x3, x4, v1, v2, v3, v4, toi)) return 0;
    V3 z1 = x1 + toi * v1, z2 = x2 + toi * v2, z3 = x3 + toi * v3, z4 = x4 + toi * v4;
    V3 coords, p;
    closest_point_triangle(z4, z1, z2, z3, p, coords);
    V3 delta = z4 - p;
    const float eps = 0.1f;
    if (!(lensq(delta) < eps * eps)) return 0;
    V3 triNormal = normalized(cross(x2 - x1, x3 - x1));
    float side = dot(triNormal, x4 - x1);
    V3 nn = normalized(cross(z2 - z1, z3 - z1));
    if (side < 0) nn = -nn;
    rec.idx = make_uint4(i1, i2, i3, vtx);
    rec.normal = f4(nn, 0.f);
    rec.w = make_float4(coords.x, coords.y, coords.z, 0.f);
    rec.side = signed_volume(x4, x1, x2, x3);
    rec.lam = make_float2(0.f, 0.f);
    rec.error = 0.f;
    return 1;
}

// EdgeEdgeTest + EdgeEdgeCCD (SelfCollisionDetector.cpp:491-606) for pair k
__device__ int ccd_ee_test(const DevCloth& c, const SolverParams& P, const Buffers& b, int k, SCt& rec)
{
    int2 pr = b.ccdEePairs[k];
    const int4 A = c.edge[pr.x], B = c.edge[pr.y];
    const int i1 = A.x, i2 = A.y, j1 = B.x, j2 = B.y;
    if (i1 == j1 || i1 == j2 || i2 == j1 || i2 == j2) return 0;
    V3 x1 = ld3(c.prev, i1), x2 = ld3(c.prev, i2), x3 = ld3(c.prev, j1), x4 = ld3(c.prev, j2);
    V3 v1 = ld3(c.pos, i1) - x1, v2 = ld3(c.pos, i2) - x2, v3 = ld3(c.pos, j1) - x3, v4 = ld3(c.pos, j2) - x4;
    float toi;
    if (!solve_cubic(x1, x2, x3, x4, v1, v2, v3, v4, toi)) return 0;
    V3 z1 = x1 + toi * v1, z2 = x2 + toi * v2, z3 = x3 + toi * v3, z4 = x4 + toi * v4;
    V3 c1, c2;
    float s, t;
    closest_segm_segm(z1, z2, z3, z4, s, t, c1, c2);
    float dSqr = lensq(c1 - c2);
    const float eps = 0.5f * P.thickness;
    if (!(dSqr <= eps * eps)) return 0;
    float s2, t2; V3 d1, d2;
    closest_segm_segm(x1, x2, x3, x4, s2, t2, d1, d2);
    rec.idx = make_uint4(i1, i2, j1, j2);
    rec.normal = f4(normalized(d2 - d1), 0.f);
    rec.w = make_float4(s, t, 0.f, 0.f);
    rec.side = signed_volume(x1, x2, x3, x4);
    rec.lam = make_float2(0.f, 0.f);
    rec.error = 0.f;
    return 1;
}

// narrow phase over the device-counted pair lists (grid-stride; every pair
// gets its hit flag, so no clearing is needed)
// per pair: hit flag, and the query's hit count (zeroed by k_ccd_pairs; hits
// are rare, so the atomics are too)
__global__ void k_ccd_narrow_vt(DevCloth c, SolverParams P, Buffers b)
{
    int n = *b.ccdVtPairCount;
    if (n > b.ccdVtCap) n = b.ccdVtCap;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    {
        SCt rec;
        const bool hit = ccd_vt_test(c, P, b, k, rec);
        b.ccdVtHit[k] = (uint8_t)hit;
        if (hit) atomicAdd(&b.ccdVtHitCnt[b.ccdVtPairs[k].x], 1);
    }
}

__global__ void k_ccd_narrow_ee(DevCloth c, SolverParams P, Buffers b)
{
    int n = *b.ccdEePairCount;
    if (n > b.ccdEeCap) n = b.ccdEeCap;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    {
        SCt rec;
        const bool hit = ccd_ee_test(c, P, b, k, rec);
        b.ccdEeHit[k] = (uint8_t)hit;
        if (hit) atomicAdd(&b.ccdEeHitCnt[b.ccdEePairs[k].x], 1);
    }
}

// append the hit records after the list's current count, per query in ascending
// candidate order (the order of an all-pairs sweep); one warp per query picks its
// hits smallest candidate first. A hit's record is recomputed by the same
// deterministic test rather than stored per pair.
template <bool VT>
__global__ void k_ccd_gather(DevCloth c, SolverParams P, Buffers b, const int* hoff, SCt* list, const int* listCount, int listCap)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int n = VT ? c.N : c.E;
    if (i >= n) return;
    const int h = (VT ? b.ccdVtHitCnt : b.ccdEeHitCnt)[i];
    if (h == 0) return;
    const int* cnt = VT ? b.ccdVtCnt : b.ccdEeCnt;
    const int* off = VT ? b.ccdVtOff : b.ccdEeOff;
    const uint8_t* hit = VT ? b.ccdVtHit : b.ccdEeHit;
    const int2* pairs = VT ? b.ccdVtPairs : b.ccdEePairs;
    const int cap = VT ? b.ccdVtCap : b.ccdEeCap;
    const int o = off[i], e = min(cap, o + cnt[i]);
    const int d0 = *listCount + hoff[i];
    int last = -1;
    for (int r = 0; r < h; r++)
    {
        int best = INT_MAX, bestK = -1;
        for (int k = o + lane; k < e; k += 32)
            if (hit[k])
            {
                const int id = pairs[k].y;
                if (id > last && id < best) { best = id; bestK = k; }
            }
        const int m = __reduce_min_sync(0xffffffffu, best);
        if (best == m && bestK >= 0)
        {
            SCt rec;
            if (VT) ccd_vt_test(c, P, b, bestK, rec); else ccd_ee_test(c, P, b, bestK, rec);
            if (d0 + r < listCap) list[d0 + r] = rec;
            else atomicOr(c.status, ST_CCD_OVERFLOW);
        }
        last = m;
    }
}

// Constraint residual: max |C| over the warp, weft and shear constraints of every
// triangle (the C values of SolveTriangles, Physics/ClothPBD.cpp:66-67,76,87,99)
// at the current positions; same operation order as the oracle's, so bit-equal.
template <typename PA>
__device__ __forceinline__ float fem_residual(const PA& pa, float4 r0, float4 r1, float4 r2)
{
    const uint32_t i1 = __float_as_uint(r0.x), i2 = __float_as_uint(r0.y), i3 = __float_as_uint(r0.z);
    const float du1 = r0.w, du2 = r1.x, dv1 = r1.y, dv2 = r1.z, invDet = r1.w;
    const float4 a = pa.ld(i1), b = pa.ld(i2), d = pa.ld(i3);
    const V3 x1 = mk(a.x, a.y, a.z), x2 = mk(b.x, b.y, b.z), x3 = mk(d.x, d.y, d.z);
    const V3 dx1 = x2 - x1, dx2 = x3 - x1;
    const V3 wu = invDet * (dv2 * dx1 - dv1 * dx2);
    const V3 wv = invDet * (-du2 * dx1 + du1 * dx2);
    const float cu = fabsf(0.5f * (dot(wu, wu) - r2.x));
    const float cv = fabsf(0.5f * (dot(wv, wv) - r2.y));
    const float cs = fabsf(dot(wu, wv));
    return fmaxf(cu, fmaxf(cv, cs));
}

// max over the triangles into *out (float bits; |C| >= 0 orders like its bits)
__global__ void k_residual(DevCloth c, unsigned* out)
{
    const GlobalPos pa{c.pos};
    float r = 0.f;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < c.T; j += gridDim.x * blockDim.x)
        r = fmaxf(r, fem_residual(pa, c.fem[3 * j], c.fem[3 * j + 1], c.fem[3 * j + 2]));
    const unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(r));
    if ((threadIdx.x & 31) == 0) atomicMax(out, u);
}

// ------------------------------------------------- cluster-resident solver
// The whole Gauss-Seidel loop of one substep (SolveGS, Physics/ClothPBD.cpp:324-369)
// plus the velocity update in ONE launch of ONE thread-block cluster. Every CTA
// owns a power-of-two block of particles and keeps their positions in its shared
// memory for the whole solve; a projection reaches any particle through the
// cluster's distributed shared memory (mapa + ld/st.shared::cluster). Colours
// are separated by hardware cluster barriers instead of kernel boundaries.
// Constraint records stream from global memory (L2-resident at these sizes).
// The phase structure is identical to the per-colour kernels, so results are
// bit-identical to them.
// Latency probe of the cluster solver's phase structure: `phases` phases of one
// cluster of the solver's size and block shape, separated by cluster barriers,
// with nothing in a phase (kind 0) or one distributed-shared-memory read and
// write per thread (kind 1: every CTA updates its neighbour's block, a
// permutation, so no two CTAs write one word in a phase). Its time per phase is
// what a colour phase costs before any projection arithmetic.
__device__ int g_phaseProbeSink;

__global__ void __launch_bounds__(GS_THREADS) k_phase_probe(int phases, int kind)
{
    __shared__ int cell[GS_THREADS];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank(), n = cl.num_blocks();
    cell[threadIdx.x] = (int)threadIdx.x;
    cl.sync();
    int acc = 0;
    for (int k = 0; k < phases; k++)
    {
        if (kind == 1)
        {
            int* peer = cl.map_shared_rank(cell, (rank + 1 + (unsigned)k) % n);
            const int v = peer[threadIdx.x];
            peer[threadIdx.x] = v + 1;
            acc += v;
        }
        cl.sync();                                   // also keeps every block alive until the last access
    }
    if (acc == 0x7fffffff) g_phaseProbeSink = acc;   // keeps the loads; never true
}

float probe_cluster_phase(int kind, int phases)
{
    int shift = 0;
    size_t smem = 0;
    const int cs = gs_cluster_size(1, shift, smem);
    if (cs == 0 || phases < 1) return -1.f;
    cudaFuncSetAttribute(k_phase_probe, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(GS_THREADS);
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = cs; at.val.clusterDim.y = 1; at.val.clusterDim.z = 1;
    cfg.attrs = &at; cfg.numAttrs = 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    float ms = -1.f;
    if (cudaLaunchKernelEx(&cfg, k_phase_probe, 1000, kind) == cudaSuccess)       // warm-up
    {
        cudaEventRecord(e0, 0);
        cudaLaunchKernelEx(&cfg, k_phase_probe, phases, kind);
        cudaEventRecord(e1, 0);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = -1.f;
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaGetLastError();
    return ms < 0.f ? -1.f : 1000.f * ms / (float)phases;
}


// ------------------------------------------------------------- launchers
// particle state <-> the packed host layout of the state transfers: positions,
// velocities and previous positions as xyz triples, then inverse masses (one
// copy each way instead of three of float4 arrays)
__global__ void k_pack_state(DevCloth c, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const size_t n = c.N;
    const float4 p = c.pos[i], v = c.vel[i], q = c.prev[i];
    float* a = out + 3 * (size_t)i;
    a[0] = p.x; a[1] = p.y; a[2] = p.z;
    a[3 * n] = v.x; a[3 * n + 1] = v.y; a[3 * n + 2] = v.z;
    a[6 * n] = q.x; a[6 * n + 1] = q.y; a[6 * n + 2] = q.z;
    out[9 * n + i] = p.w;
}

__global__ void k_unpack_state(DevCloth c, const float* in)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const size_t n = c.N;
    const float* a = in + 3 * (size_t)i;
    c.pos[i] = make_float4(a[0], a[1], a[2], in[9 * n + i]);
    c.vel[i] = make_float4(a[3 * n], a[3 * n + 1], a[3 * n + 2], 0.f);
    c.prev[i] = make_float4(a[6 * n], a[6 * n + 1], a[6 * n + 2], 0.f);
}

void launch_pack_state(cudaStream_t s, const DevCloth& c, float* out)
{
    k_pack_state<<<blocks_for(c.N), 256, 0, s>>>(c, out);
}

void launch_unpack_state(cudaStream_t s, const DevCloth& c, const float* in)
{
    k_unpack_state<<<blocks_for(c.N), 256, 0, s>>>(c, in);
}

void launch_predict(cudaStream_t s, const DevCloth& c, const SolverParams& P)
{
    cudaMemsetAsync(c.scal, 0, sizeof(float), s);
    k_predict<<<blocks_for(c.N), 256, 0, s>>>(c, P);
}

void launch_velocity(cudaStream_t s, const DevCloth& c, const SolverParams& P)
{
    k_velocity<<<blocks_for(c.N), 256, 0, s>>>(c, P);
}





void launch_normals(cudaStream_t s, const DevCloth& c, bool prevMesh, const float4* verts)
{
    float4* triN = prevMesh ? c.prevTriN : c.meshTriN;
    float4* vn = prevMesh ? c.prevN : c.meshN;
    k_tri_normals<<<blocks_for(c.T), 256, 0, s>>>(verts, c.tri, c.T, triN, c.triAngles);
    k_vertex_normals<<<blocks_for(c.N), 256, 0, s>>>(c.N, c.vTriStart, c.vTri, triN, c.triAngles, vn);
}

void launch_vertex_colliders(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, const VColl*)
{
    if (b.numVColl > 0) k_vertex_colliders<<<blocks_for(c.N, 128), 128, 0, s>>>(c, P, b);
}

void launch_tri_edge_colliders(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b,
                               const VColl* hostColl, int numColl, int flags)
{
    // per-collider triangle / edge slots: collider slot index = order among
    // colliders that produce such contacts (world order)
    int ti = 0, ei = 0;
    for (int k = 0; k < numColl; k++)
    {
        const VColl& g = hostColl[k];
        if (g.type != 3 && g.type != 4 && g.type != 7) continue;
        if (flags & CF_EDGES) { k_edge_colliders<<<blocks_for(c.E, 128), 128, 0, s>>>(c, P, b, g, ei); ei++; }
        if (flags & CF_TRIANGLES) { k_tri_colliders<<<blocks_for(c.T, 128), 128, 0, s>>>(c, P, b, g, ti); ti++; }
    }
    // compaction in (collider, item) order
    if (ti > 0)
    {
        int n = ti * c.T;
        scan_ints(s, b.tcFlag, b.scanOff, n, b.tcCount, b.scanBlock);
        k_compact<TC><<<blocks_for(n), 256, 0, s>>>(b.tcFlag, b.scanOff, b.tcSlot, 1, b.tcList, n, nullptr, b.tcCap, c.status, ST_CONTACT_OVERFLOW);
        k_add_counts<<<1, 32, 0, s>>>(b.tcCount, b.tcCount, nullptr, b.tcCap);
    }
    else cudaMemsetAsync(b.tcCount, 0, sizeof(int), s);
    if (ei > 0)
    {
        int n = ei * c.E;
        scan_ints(s, b.ecFlag, b.scanOff, n, b.ecCount, b.scanBlock);
        k_compact<EC><<<blocks_for(n), 256, 0, s>>>(b.ecFlag, b.scanOff, b.ecSlot, 1, b.ecList, n, nullptr, b.ecCap, c.status, ST_CONTACT_OVERFLOW);
        k_add_counts<<<1, 32, 0, s>>>(b.ecCount, b.ecCount, nullptr, b.ecCap);
    }
    else cudaMemsetAsync(b.ecCount, 0, sizeof(int), s);
}



void launch_colour_contacts(cudaStream_t s, const DevCloth& c, const Buffers& b)
{
    k_colour<<<1, 1024, 0, s>>>(c, b, colour_args(b));
}


void launch_bvh_refit(cudaStream_t s, const DevBVH& t, const DevCloth& c, int kind, float tol)
{
    k_bvh_refit<<<blocks_for(t.numLeaves), 256, 0, s>>>(t, c, kind, tol);
}

void launch_self_proximity(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b,
                           const DevBVH& triBvh, const DevBVH& edgeBvh)
{
    k_self_vt<<<blocks_for(c.N, 128), 128, 0, s>>>(c, P, b, triBvh);
    k_self_ee<<<blocks_for(c.E, 128), 128, 0, s>>>(c, P, b, edgeBvh);
}

void launch_compact_self(cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, const DevCloth& c,
                         const SolverParams& P, const Buffers& b, bool self, bool ccd)
{
    if (self)
    {
        int* off = b.scanOff;
        scan_ints(s, b.stCnt, off, c.N, b.stCount, b.scanBlock);
        k_compact<SCt><<<blocks_for(c.N), 256, 0, s>>>(b.stCnt, off, b.stSlot, KVT, b.stList, c.N, nullptr, b.stCap, c.status, ST_SELF_VT_OVERFLOW);
        scan_ints(s, b.seFlag, off, c.E, b.seCount, b.scanBlock);
        k_compact<SCt><<<blocks_for(c.E), 256, 0, s>>>(b.seFlag, off, b.seSlot, 1, b.seList, c.E, nullptr, b.seCap, c.status, ST_SELF_EE_OVERFLOW);
    }
    else cudaMemsetAsync(b.stCount, 0, 2 * sizeof(int), s);     // no proximity contacts (stCount, seCount)
    if (ccd)
    {
        // continuous hits go after the proximity contacts, as the detector's
        // AddSelfTriangle / AddSelfEdge would append them (in pair order); the
        // vertex-triangle list is assembled on the side stream beside the
        // edge-edge one (own offsets, block sums and total)
        cudaEventRecord(fork, s);
        cudaStreamWaitEvent(side, fork, 0);
        scan_ints(side, b.ccdVtHitCnt, b.scanOff2, c.N, b.scanTot + 1, b.scanBlock2);
        k_ccd_gather<true><<<blocks_for(32 * c.N), 256, 0, side>>>(c, P, b, b.scanOff2, b.stList, b.stCount, b.stCap);
        k_add_counts<<<1, 32, 0, side>>>(b.stCount, b.stCount, b.scanTot + 1, b.stCap);
        cudaEventRecord(join, side);
        scan_ints(s, b.ccdEeHitCnt, b.scanOff, c.E, b.scanTot, b.scanBlock);
        k_ccd_gather<false><<<blocks_for(32 * c.E), 256, 0, s>>>(c, P, b, b.scanOff, b.seList, b.seCount, b.seCap);
        k_add_counts<<<1, 32, 0, s>>>(b.seCount, b.seCount, b.scanTot, b.seCap);
        cudaStreamWaitEvent(s, join, 0);
    }
    if (self)
    {
        k_add_counts<<<1, 32, 0, s>>>(b.stCount, b.stCount, nullptr, b.stCap);
        k_add_counts<<<1, 32, 0, s>>>(b.seCount, b.seCount, nullptr, b.seCap);
    }
}

void launch_ccd(cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, const DevCloth& c,
                const SolverParams& P, const Buffers& b, const DevBVH& triBvh, const DevBVH& edgeBvh,
                const cudaEvent_t* marks)
{
    auto mark = [&](int k, cudaStream_t st) {
        if (marks && marks[k]) cudaEventRecordWithFlags(marks[k], st, cudaEventRecordExternal);
    };
    // The vertex-triangle chain (refit, broad phase, pairs, narrow phase) runs on
    // the side stream beside the edge-edge chain; each is latency bound and fills
    // only part of the GPU. They share nothing but the pool counter (atomic).
    const float tol = P.thickness + P.tolerance * 0.5f;
    cudaMemsetAsync(b.ccdPoolUsed, 0, sizeof(int), s);
    cudaMemsetAsync(b.ccdOvfN, 0, 2 * sizeof(int), s);
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(side, fork, 0);
    launch_bvh_refit(side, triBvh, c, 2, tol);
    mark(2, side);
    launch_broad_pass1(side, true, c, P, b, triBvh, tol);
    k_ccd_broad_coop<true><<<CCD_COOP_BLOCKS, CCD_COOP_THREADS, ccd_coop_smem(triBvh.depth), side>>>(c, P, b, triBvh, tol);
    mark(3, side);
    scan_ints(side, b.ccdVtCnt, b.ccdVtOff, c.N, b.ccdVtPairCount, b.scanBlock2);
    k_ccd_pairs<<<blocks_for(32 * c.N), 256, 0, side>>>(b.ccdVtCnt, b.ccdVtOff, b.ccdVtCand, b.ccdPool, b.ccdVtPoolOff, c.N,
                                                   b.ccdVtPairs, b.ccdVtCap, c.status, b.ccdVtHitCnt);
    k_ccd_narrow_vt<<<4 * 148, 128, 0, side>>>(c, P, b);
    cudaEventRecord(join, side);

    launch_bvh_refit(s, edgeBvh, c, 3, tol);
    mark(0, s);
    launch_broad_pass1(s, false, c, P, b, edgeBvh, tol);
    k_ccd_broad_coop<false><<<CCD_COOP_BLOCKS, CCD_COOP_THREADS, ccd_coop_smem(edgeBvh.depth), s>>>(c, P, b, edgeBvh, tol);
    mark(1, s);
    scan_ints(s, b.ccdEeCnt, b.ccdEeOff, c.E, b.ccdEePairCount, b.scanBlock);
    k_ccd_pairs<<<blocks_for(32 * c.E), 256, 0, s>>>(b.ccdEeCnt, b.ccdEeOff, b.ccdEeCand, b.ccdPool, b.ccdEePoolOff, c.E,
                                                b.ccdEePairs, b.ccdEeCap, c.status, b.ccdEeHitCnt);
    // narrow phase: a fixed grid strides over the device-side pair counts
    k_ccd_narrow_ee<<<8 * 148, 128, 0, s>>>(c, P, b);
    cudaStreamWaitEvent(s, join, 0);
}

// largest displacement since the snapshot (scaled), into scal[11]; new snapshot
__global__ void k_update_residual(DevCloth c, SolverParams P, bool measure)
{
    float r = 0.f;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < c.N; g += gridDim.x * blockDim.x)
    {
        const float4 x = c.pos[g];
        if (measure)
        {
            const float4 x0 = c.xsnap[g];
            const float dx = x.x - x0.x, dy = x.y - x0.y, dz = x.z - x0.z;
            r = fmaxf(r, sqrtf(dx * dx + dy * dy + dz * dz) * P.resScale);
        }
        c.xsnap[g] = x;
    }
    const unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(r));
    if (measure && (threadIdx.x & 31) == 0 && u) atomicMax(reinterpret_cast<unsigned*>(c.scal + 11), u);
}

void launch_residual_exit(cudaStream_t s, const DevCloth& c, const SolverParams& P, int iter)
{
    if (iter < 0)
    {
        k_update_residual<<<2 * 148, 256, 0, s>>>(c, P, false);     // the first snapshot
        return;
    }
    k_update_residual<<<2 * 148, 256, 0, s>>>(c, P, true);
    k_residual_exit<<<1, 1, 0, s>>>(c, P, iter);
}

void launch_iteration_total(cudaStream_t s, const DevCloth& c)
{
    k_iteration_total<<<1, 1, 0, s>>>(c);
}

void launch_residual(cudaStream_t s, const DevCloth& c, unsigned* out)
{
    cudaMemsetAsync(out, 0, sizeof(unsigned), s);
    k_residual<<<2 * 148, 256, 0, s>>>(c, out);
}

void launch_reset_gs(cudaStream_t s, const DevCloth& c)
{
    cudaMemsetAsync(c.scal + 1, 0, sizeof(float) * 9, s);
}

void launch_gs_exit_test(cudaStream_t s, const DevCloth& c, const SolverParams& P, int iter)
{
    k_gs_exit<<<1, 32, 0, s>>>(c, P, iter);
}

} // namespace sc

namespace sc {

// ------------------------------------------------------- SDF from a mesh
// SDF::CreateFromMesh (Geometry/SDF.cpp:58-76): at every grid node the distance
// to the nearest mesh triangle (ClosestPointOnMeshToPointAcc with its default
// delta normal), negated when the offset points against that normal — which,
// with the delta normal, never happens: the reference's field is unsigned.
__global__ void k_sdf_from_mesh(DevMesh m, int4 vals, float4 lo, float4 steps, float* out, int* status)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int count = vals.x * vals.y * vals.z;
    if (idx >= count) return;
    const int x = idx % vals.x, w = idx / vals.x, y = w % vals.y, z = w / vals.y;
    V3 org = mk((float)x * steps.x, (float)y * steps.y, (float)z * steps.z);
    org = org + mk(lo.x, lo.y, lo.z);
    PointHit h = mesh_point_query(m, org, status, FLT_MAX);
    float val = h.dist;
    const V3 delta = org - h.cp;
    if (dot(delta, h.normal) < 0) val = -val;
    out[idx] = val;
}

bool launch_sdf_from_mesh(const DevMesh& m, int nx, int ny, int nz, float4 lo, float4 steps, float* out, int* status)
{
    const int count = (nx + 1) * (ny + 1) * (nz + 1);
    k_sdf_from_mesh<<<blocks_for(count, 128), 128>>>(m, make_int4(nx + 1, ny + 1, nz + 1, 0), lo, steps, out, status);
    return cudaGetLastError() == cudaSuccess;
}

} // namespace sc

// ----------------------------------------------------- learned warm start
#include "mlp_kernels.cuh"

namespace sc {

static_assert(MLP_NPARAM == ML_NPARAM && MLP_NNORM == ML_NNORM, "MLP layout");

static int mlp_sm_count()
{
    static int sms = 0;
    if (sms == 0)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms < 1) sms = 1;
    }
    return sms;
}

// inference CTAs hold 128 tensor-memory columns (four fit an SM), persistent over tiles
static int mlp_infer_grid(int rows) { return std::max(1, std::min((rows + ML_ROWS - 1) / ML_ROWS, 4 * mlp_sm_count())); }

void launch_mlp_warm(cudaStream_t s, const DevCloth& c, const Buffers& b, const float* prm, const float* norm)
{
    k_mlp_warm<<<mlp_infer_grid(c.N), 128, 0, s>>>(c, b, MlpArgs{prm, norm});
}

void launch_mlp_features(cudaStream_t s, const DevCloth& c, const Buffers& b, float* feat)
{
    k_mlp_features<<<blocks_for(c.N), 256, 0, s>>>(c, b, feat);
}

void launch_mlp_targets(cudaStream_t s, const DevCloth& c, float* target)
{
    k_mlp_targets<<<blocks_for(c.N), 256, 0, s>>>(c, target);
}

void launch_mlp_forward(cudaStream_t s, const float* X, int S, const float* prm, const float* norm, float* Y)
{
    k_mlp_forward<<<mlp_infer_grid(S), 128, 0, s>>>(X, S, MlpArgs{prm, norm}, Y, nullptr);
}

size_t mlp_grad_smem() { return sizeof(MlpTcTrainSmem); }

bool launch_mlp_grad(cudaStream_t s, const float* X, const float* T, int S, const float* prm, const float* norm,
                     float* grad, float* loss)
{
    static bool attr = false;
    const size_t smem = mlp_grad_smem();
    if (!attr)
    {
        if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
        attr = true;
    }
    cudaMemsetAsync(grad, 0, sizeof(float) * ML_NPARAM, s);
    cudaMemsetAsync(loss, 0, sizeof(float), s);
    // training CTAs hold all 512 tensor-memory columns of their SM: one per SM
    const int grid = std::max(1, std::min((S + ML_ROWS - 1) / ML_ROWS, mlp_sm_count()));
    k_mlp_grad<<<grid, 128, smem, s>>>(X, T, S, MlpArgs{prm, norm}, grad, loss, nullptr);
    return cudaGetLastError() == cudaSuccess;
}

void launch_adam(cudaStream_t s, float* prm, const float* grad, float* m, float* v, int step, float lr)
{
    k_adam<<<(ML_NPARAM + 255) / 256, 256, 0, s>>>(prm, grad, m, v, step, lr, 0.9f, 0.999f, 1e-8f);
}

} // namespace sc

namespace sc {

const SolverOps& solver_ops_fast();   // solver_fast.cu

const SolverOps& solver_ops(bool fast) { return fast ? solver_ops_fast() : kSolverOps; }

} // namespace sc
