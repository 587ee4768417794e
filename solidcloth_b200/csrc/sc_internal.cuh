// sc_internal.cuh — device data layout and kernel entry points of the cloth step.
//
// HBM layout (one cloth patch):
//   pos[N]   float4 (x, y, z, inverse mass)   — SoA particle state, 16 B aligned
//   prev[N]  float4 (x, y, z, 0)               — start-of-substep positions; also
//                                               the vertex buffer of the collision mesh
//   vel[N]   float4 (x, y, z, 0)
//   fem[3T]  float4 x3 per triangle in colour order:
//            {i1, i2, i3 (as bits), du1} {du2, dv1, dv2, invDet} {lu2, lv2, lu0*lv0, area}
//   bend[B]  uint4 (i1, i2, i3, i4) in colour order
// Contacts live in fixed per-item slots (no device allocation in the step) and
// are compacted with block scans.
#pragma once
#include "scmath.cuh"

namespace sc {

enum CollFlags { CF_VERTICES = 1, CF_TRIANGLES = 2, CF_SELF = 4, CF_WALLS = 8, CF_EDGES = 16 };

// status bits reported through scGetLastError / scGetStatus
enum StatusBits {
    ST_SELF_VT_OVERFLOW = 1,     // more self vertex-triangle candidates/contacts than slots
    ST_SELF_EE_OVERFLOW = 2,
    ST_CCD_OVERFLOW = 4,
    ST_CONTACT_OVERFLOW = 8,
    ST_COLOUR_OVERFLOW = 16,     // contact colouring needed more rounds than supported
    ST_MESH_STACK_OVERFLOW = 32,
    ST_BVH_STACK_OVERFLOW = 64,
    ST_TC_TIMEOUT = 128,         // a tensor-core completion wait of the warm-start network gave up
};

struct SolverParams
{
    float unit, thickness, tolerance, shear, bend, poisson, friction, drag;
    float selfShrink;
    float h, h2, invH, epsUV;
    int iterations, flags, fem, dihedral, fixedIterations, bendFreq;
    float selfThreshold;
    float area;              // ClothModel::mArea (link compliance: k = h^2 area unit)
    float resTol;            // > 0: iterate until the update residual <= resTol
    float resScale;          // 1 / mean rest edge length (the update residual's unit)
};

// Device view of one cloth patch (plain pointers, passed by value).
struct DevCloth
{
    int N, T, E, B;
    float4* pos;
    float4* prev;
    float4* vel;
    const float4* fem;          // 3*T, colour order
    const float4* link;         // L, colour order: i1, i2 (bits), rest length, stiffness
    int L;
    const uint4* bend;          // B, colour order
    const uint32_t* tri;        // 3*T original (mesh) order
    const uint32_t* triE;       // 3*T triangle -> edge ids (Mesh::Triangle::e)
    const int4* edge;           // E: i1, i2, t1, t2
    const uint8_t* edgeSwapped; // E
    const int* vRingStart;      // N+1, vertex one-ring CSR (ConstructVertexOneRings order)
    const int* vRing;
    const int* eRingStart;      // N+1, edge one-ring CSR (ConstructEdgeOneRings order)
    const int* eRing;
    const int* vTriStart;       // N+1, incident (triangle, corner) sorted by triangle
    const int2* vTri;
    const uint8_t* vBorder;     // N, Mesh::IsBorderVertex
    const int* vInst;           // N: instance of each particle in a batch (null: one cloth)
    const int* instStart;       // batch: first particle of each instance (+ end)
    const float* edgeRest;      // E: rest length of each edge (from the uv layout)
    float4* xsnap;              // N: positions at the start of the current iteration (update residual)
    float4* xpred;              // N: positions after the substep's prediction (warm start / samples)
    float* lastCorr;            // N: last substep's solver correction along the collision normal
    const int* vQuery;          // N: vertices in spatial (Morton, rest shape) order: neighbouring
    const int* eQuery;          // E: edges likewise; queries of one warp walk the same subtrees
    float4* prevN;              // collision mesh vertex normals (refreshed per frame)
    float4* prevTriN;           // collision mesh triangle normals
    float4* meshN;              // render mesh normals
    float4* meshTriN;
    float4* triAngles;          // scratch: per-triangle angle weights
    // static colours of the cloth's triangles and edges (proper colourings: one
    // colour's triangles / edges share no particle); triangle and edge collider
    // contacts take their triangle's / edge's colour, so they need no colouring pass
    const uint8_t* triColour;   // T
    const uint8_t* edgeColour;  // E
    int nTriColours, nEdgeColours;
    float* scal;                // [0] max |pos - prev| (as float bits), [1..7] GS errors, [8] done flag
    int* status;
};

// Linear BVH with fixed topology, nodes in depth-first preorder.
struct DevBVH
{
    int numLeaves, numNodes;
    int depth;              // largest number of edges from a root to a leaf
    const int* child;       // numNodes: internal -> right child index; leaf -> ~primitive
    const int* escape;      // numNodes: preorder index after the subtree
    const int* parent;      // numNodes (root -1)
    const int* leafNode;    // numLeaves: primitive -> node index
    const int* maxPrim;     // numNodes: largest primitive index in the subtree
    const int* instRoot;    // batch: root node of each instance's tree (a forest); null: one tree at 0
    float4* lo;             // numNodes: box min; w = child[] as int bits
    float4* hi;             // numNodes: box max; w = escape[] as int bits
    float4* rec;            // numNodes x 4: an internal node's two child records (box, link, max primitive)
    int* visit;             // numNodes refit counters
};

// Static collider tree, identical to Geometry::ComputeMeshTree's, flattened.
struct DevMeshTree
{
    int numNodes;
    const float4* lo;
    const float4* hi;
    const int2* children;    // left, right (-1 if absent)
    const int4* primRange;   // tris start, tris count, verts start, verts count
    const int2* edgeRange;   // edges start, edges count
    const uint32_t* tris;
    const uint32_t* verts;
    const uint32_t* edges;
};

struct DevMesh
{
    int V, T, E;
    const float4* v;        // vertices
    const float4* n;        // angle-weighted vertex normals
    const float4* en;       // edge pseudo-normals
    const uint32_t* tri;    // 3T
    const int4* edge;       // i1 i2 t1 t2
    DevMeshTree tree;
};

} // namespace sc
