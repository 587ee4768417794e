// cloth.cu — host side of the cloth step: set-up (grid, FEM rest data, edges,
// bends, colouring, BVH topology, collider trees), device buffers, and the CUDA
// graph that runs one frame (ClothPatch::Step) on a private stream.
#include "cloth.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <numeric>
#include <array>
#include <functional>
#include <map>
#include <mutex>

namespace sc {

static inline float bits_f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

// ------------------------------------------------------------------ errors
static thread_local int g_err = SC_OK;
static thread_local std::string g_errMsg;

void set_error(int code, const std::string& msg)
{
    g_err = code;
    g_errMsg = msg;
}
int last_error() { return g_err; }
const char* last_error_string() { return g_errMsg.c_str(); }

#define SC_CUDA(x)                                                                     \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            set_error(SC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));   \
            return false;                                                              \
        }                                                                              \
    } while (0)

// the same for functions without a result
#define SC_CUDA_V(x)                                                                   \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            set_error(SC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));   \
            return;                                                                    \
        }                                                                              \
    } while (0)

// -------------------------------------------------------------------- mesh
// Mesh::ComputeNormals, angle weighted (Geometry/Mesh.cpp:10-63)
void HMesh::compute_normals()
{
    normals.assign(verts.size(), mk(0, 0, 0));
    triN.resize(idx.size() / 3);
    for (size_t i = 0; i < idx.size(); i += 3)
    {
        const int i1 = idx[i], i2 = idx[i + 1], i3 = idx[i + 2];
        V3 a = verts[i1], b = verts[i2], c = verts[i3];
        V3 nt = normalized(cross(b - a, c - a));
        triN[i / 3] = nt;
        V3 e1 = normalized(b - a), e2 = normalized(c - b), e3 = normalized(a - c);
        float c1 = -dot(e1, e3), c2 = -dot(e1, e2), c3 = -dot(e2, e3);
        float s1 = len(cross(e1, -e3)), s2 = len(cross(e2, -e1)), s3 = len(cross(e3, -e1));
        float t1 = std::fabs(c1) > 1 ? (float)std::fabs(std::atan2((double)s1, (double)c1)) : portable_acos(c1);
        float t2 = std::fabs(c2) > 1 ? (float)std::fabs(std::atan2((double)s2, (double)c2)) : portable_acos(c2);
        float t3 = std::fabs(c3) > 1 ? (float)std::fabs(std::atan2((double)s3, (double)c3)) : portable_acos(c3);
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

// Mesh::ConstructEdges (Geometry/Mesh.cpp:65-147). The half-edge array is sorted
// with std::sort and the same (i1, i2) comparator as the reference, so the two
// half-edges of each interior edge come out in the same (unstable) order and
// t1/t2 — hence bend vertex order and edge normals — match it.
void HMesh::construct_edges()
{
    edges.clear();
    const int numEdges = (int)idx.size();
    if (numEdges == 0) return;
    std::vector<HEdge> dup(numEdges);
    triE.assign(idx.size(), 0);
    for (int i = 0; i < numEdges; i++)
    {
        int i1 = idx[i], i2;
        if ((i + 1) % 3 == 0)
        {
            i2 = idx[i - 2];
            triE[i / 3 * 3 + 2] = (uint32_t)i;
            triE[i / 3 * 3 + 1] = (uint32_t)(i - 1);
            triE[i / 3 * 3 + 0] = (uint32_t)(i - 2);
        }
        else
            i2 = idx[i + 1];
        bool swapped = false;
        if (i1 > i2) { std::swap(i1, i2); swapped = true; }
        HEdge e;
        e.i1 = i1; e.i2 = i2; e.swapped = swapped; e.t1 = i / 3; e.t2 = -1;
        e.n = triN[i / 3];
        e.origIdx = i;
        dup[i] = e;
    }
    std::sort(dup.begin(), dup.end(), [](const HEdge& a, const HEdge& b) {
        return a.i1 < b.i1 || (a.i1 == b.i1 && a.i2 < b.i2);
    });
    HEdge cur = dup[0];
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
    for (size_t k = 0; k < triE.size(); k++) triE[k] = map[triE[k]];
}

void HMesh::construct_rings(bool vtx, bool edge)
{
    if (vtx) vtxRing.assign(verts.size(), {});
    if (edge) edgeRing.assign(verts.size(), {});
    for (size_t i = 0; i < edges.size(); i++)
    {
        if (vtx) { vtxRing[edges[i].i1].push_back(edges[i].i2); vtxRing[edges[i].i2].push_back(edges[i].i1); }
        if (edge) { edgeRing[edges[i].i1].push_back((int)i); edgeRing[edges[i].i2].push_back((int)i); }
    }
}

// --------------------------------------------------------------- SDF grid
SDFC::~SDFC()
{
    if (valTex) cudaDestroyTextureObject(valTex);
    if (gradTex) cudaDestroyTextureObject(gradTex);
    if (valArr) cudaFreeArray(valArr);
    if (gradArr) cudaFreeArray(gradArr);
}

// SDF::ComputeGradient, forward differences with the last layer copied
// (Geometry/SDF.cpp:210-256)
void SDFC::compute_gradient()
{
    const int nv0 = nc[0] + 1, nv1 = nc[1] + 1;
    auto index = [&](int x, int y, int z) { return x + y * nv0 + z * nv0 * nv1; };
    auto out = [&](int x, int y, int z) { return x > nc[0] || y > nc[1] || z > nc[2] || x < 0 || y < 0 || z < 0; };
    auto val = [&](int x, int y, int z) { return out(x, y, z) ? 0.f : values[index(x, y, z)]; };
    auto gat = [&](int x, int y, int z) { return out(x, y, z) ? mk(0, 0, 0) : grad[index(x, y, z)]; };
    auto set = [&](int x, int y, int z, V3 g) { if (!out(x, y, z)) grad[index(x, y, z)] = g; };
    grad.assign(values.size(), mk(0, 0, 0));
    for (int x = 0; x < nc[0]; x++)
    {
        for (int y = 0; y < nc[1]; y++)
        {
            for (int z = 0; z < nc[2]; z++)
            {
                float v = val(x, y, z);
                float dfdx = (val(x + 1, y, z) - v) / steps.x;
                float dfdy = (val(x, y + 1, z) - v) / steps.y;
                float dfdz = (val(x, y, z + 1) - v) / steps.z;
                set(x, y, z, mk(dfdx, dfdy, dfdz));
            }
            set(x, y, nc[2], gat(x, y, nc[2] - 1));
        }
        for (int z = 0; z <= nc[2]; z++) set(x, nc[1], z, gat(x, nc[1] - 1, z));
    }
    for (int y = 0; y <= nc[1]; y++)
        for (int z = 0; z <= nc[2]; z++) set(nc[0], y, z, gat(nc[0] - 1, y, z));
}

bool SDFC::upload(int dev)
{
    if (device == dev && valTex) return true;
    const int nx = nc[0] + 1, ny = nc[1] + 1, nz = nc[2] + 1;
    cudaExtent ext = make_cudaExtent(nx, ny, nz);
    cudaChannelFormatDesc cdv = cudaCreateChannelDesc<float>();
    cudaChannelFormatDesc cdg = cudaCreateChannelDesc<float4>();
    SC_CUDA(cudaMalloc3DArray(&valArr, &cdv, ext));
    SC_CUDA(cudaMalloc3DArray(&gradArr, &cdg, ext));
    std::vector<float4> g4(grad.size());
    for (size_t i = 0; i < grad.size(); i++) g4[i] = make_float4(grad[i].x, grad[i].y, grad[i].z, 0.f);
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr((void*)values.data(), nx * sizeof(float), nx, ny);
    p.dstArray = valArr; p.extent = ext; p.kind = cudaMemcpyHostToDevice;
    SC_CUDA(cudaMemcpy3D(&p));
    cudaMemcpy3DParms q = {};
    q.srcPtr = make_cudaPitchedPtr((void*)g4.data(), nx * sizeof(float4), nx, ny);
    q.dstArray = gradArr; q.extent = ext; q.kind = cudaMemcpyHostToDevice;
    SC_CUDA(cudaMemcpy3D(&q));
    cudaTextureDesc td = {};
    for (int k = 0; k < 3; k++) td.addressMode[k] = cudaAddressModeBorder;   // 0 outside, as SDF::GetValue(int)
    td.filterMode = cudaFilterModePoint;                                      // exact samples; blend in FP32
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = valArr;
    SC_CUDA(cudaCreateTextureObject(&valTex, &rd, &td, nullptr));
    rd.res.array.array = gradArr;
    SC_CUDA(cudaCreateTextureObject(&gradTex, &rd, &td, nullptr));
    device = dev;
    return true;
}

// ----------------------------------------------------------- mesh collider
MeshC::~MeshC() { if (dmem) cudaFree(dmem); }

// Geometry::ComputeMeshTree + SplitNode, exclusive child assignment,
// maxPrims 40 (Geometry/AabbTree.cpp:9-178)
void MeshC::build_tree(float tol, int maxLevel, int flags)
{
    tree.clear();
    MeshTreeNode root;
    root.box = Box::empty();
    for (V3 v : mesh.verts) { root.box.lo = vmin(root.box.lo, v); root.box.hi = vmax(root.box.hi, v); }
    if (flags & 1) for (uint32_t i = 0; i < (uint32_t)mesh.ntris(); i++) root.tris.push_back(i);
    if (flags & 2) for (uint32_t i = 0; i < (uint32_t)mesh.verts.size(); i++) root.verts.push_back(i);
    if (flags & 4) for (uint32_t i = 0; i < (uint32_t)mesh.edges.size(); i++) root.edges.push_back(i);
    tree.push_back(root);
    built = true;
    if (maxLevel <= 0) return;
    struct Item { int node, level; };
    // recursion order of SplitNode: node, then left subtree, then right subtree
    std::vector<Item> stack{{0, 1}};
    while (!stack.empty())
    {
        Item it = stack.back();
        stack.pop_back();
        const int ni = it.node;
        const size_t maxPrims = 40;
        if (tree[ni].tris.size() < maxPrims && tree[ni].verts.size() < maxPrims && tree[ni].edges.size() < maxPrims) continue;
        V3 ext = tree[ni].box.hi - tree[ni].box.lo;
        int dir = 0;
        float m = ext.x;
        if (ext.y > m) { m = ext.y; dir = 1; }
        if (ext.z > m) { m = ext.z; dir = 2; }
        const float center = 0.5f * (comp(tree[ni].box.lo, dir) + comp(tree[ni].box.hi, dir));
        MeshTreeNode L, R;
        L.box = Box::empty(); R.box = Box::empty();
        for (uint32_t t : tree[ni].tris)
        {
            Box b = Box::empty();
            b.add(mesh.verts[mesh.idx[3 * t]]); b.add(mesh.verts[mesh.idx[3 * t + 1]]); b.add(mesh.verts[mesh.idx[3 * t + 2]]);
            b.extrude(tol);
            if (comp(b.lo, dir) <= center) { L.tris.push_back(t); L.box.add(b); }
            else { R.tris.push_back(t); R.box.add(b); }
        }
        for (uint32_t e : tree[ni].edges)
        {
            Box b = Box::empty();
            b.add(mesh.verts[mesh.edges[e].i1]); b.add(mesh.verts[mesh.edges[e].i2]);
            b.extrude(tol);
            if (comp(b.lo, dir) <= center) { L.edges.push_back(e); L.box.add(b); }
            else { R.edges.push_back(e); R.box.add(b); }
        }
        for (uint32_t v : tree[ni].verts)
        {
            Box b = Box::empty();
            b.add(mesh.verts[v]);
            b.extrude(tol);
            if (comp(mesh.verts[v], dir) <= center) { L.verts.push_back(v); L.box.add(b); }
            else { R.verts.push_back(v); R.box.add(b); }
        }
        tree[ni].tris.clear(); tree[ni].edges.clear(); tree[ni].verts.clear();
        int l = -1, r = -1;
        if (!(L.tris.empty() && L.verts.empty() && L.edges.empty())) { tree.push_back(L); l = (int)tree.size() - 1; }
        if (!(R.tris.empty() && R.verts.empty() && R.edges.empty())) { tree.push_back(R); r = (int)tree.size() - 1; }
        tree[ni].left = l; tree[ni].right = r;
        if (it.level < maxLevel)
        {
            if (r >= 0) stack.push_back({r, it.level + 1});
            if (l >= 0) stack.push_back({l, it.level + 1});
        }
    }
    built = true;
}

bool MeshC::upload(int devId)
{
    if (device == devId && dmem) return true;
    const int V = (int)mesh.verts.size(), T = mesh.ntris(), E = (int)mesh.edges.size();
    const int M = (int)tree.size();
    std::vector<float4> v(V), n(V), en(E), lo(M), hi(M);
    std::vector<int4> edge(E), pr(M);
    std::vector<int2> ch(M), er(M);
    std::vector<uint32_t> tris, verts, edges;
    for (int i = 0; i < V; i++) { v[i] = f4(mesh.verts[i], 0); n[i] = f4(mesh.normals[i], 0); }
    for (int e = 0; e < E; e++)
    {
        const HEdge& h = mesh.edges[e];
        edge[e] = make_int4((int)h.i1, (int)h.i2, h.t1, h.t2);
        en[e] = f4(h.n, 0);
    }
    for (int k = 0; k < M; k++)
    {
        const MeshTreeNode& t = tree[k];
        lo[k] = f4(t.box.lo, 0); hi[k] = f4(t.box.hi, 0);
        ch[k] = make_int2(t.left, t.right);
        pr[k] = make_int4((int)tris.size(), (int)t.tris.size(), (int)verts.size(), (int)t.verts.size());
        er[k] = make_int2((int)edges.size(), (int)t.edges.size());
        tris.insert(tris.end(), t.tris.begin(), t.tris.end());
        verts.insert(verts.end(), t.verts.begin(), t.verts.end());
        edges.insert(edges.end(), t.edges.begin(), t.edges.end());
    }
    // one allocation, 256-byte aligned sub-buffers
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    size_t oV = take(V * 16), oN = take(V * 16), oEN = take(E * 16), oT = take(T * 12), oE = take(E * 16);
    size_t oLo = take(M * 16), oHi = take(M * 16), oCh = take(M * 8), oPr = take(M * 16), oEr = take(M * 8);
    size_t oTr = take(tris.size() * 4 + 4), oVe = take(verts.size() * 4 + 4), oEd = take(edges.size() * 4 + 4);
    SC_CUDA(cudaMalloc(&dmem, off));
    char* d = (char*)dmem;
    SC_CUDA(cudaMemcpy(d + oV, v.data(), V * 16, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oN, n.data(), V * 16, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oEN, en.data(), E * 16, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oT, mesh.idx.data(), T * 12, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oE, edge.data(), E * 16, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oLo, lo.data(), M * 16, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oHi, hi.data(), M * 16, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oCh, ch.data(), M * 8, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oPr, pr.data(), M * 16, cudaMemcpyHostToDevice));
    SC_CUDA(cudaMemcpy(d + oEr, er.data(), M * 8, cudaMemcpyHostToDevice));
    if (!tris.empty()) SC_CUDA(cudaMemcpy(d + oTr, tris.data(), tris.size() * 4, cudaMemcpyHostToDevice));
    if (!verts.empty()) SC_CUDA(cudaMemcpy(d + oVe, verts.data(), verts.size() * 4, cudaMemcpyHostToDevice));
    if (!edges.empty()) SC_CUDA(cudaMemcpy(d + oEd, edges.data(), edges.size() * 4, cudaMemcpyHostToDevice));
    dev.V = V; dev.T = T; dev.E = E;
    dev.v = (const float4*)(d + oV); dev.n = (const float4*)(d + oN); dev.en = (const float4*)(d + oEN);
    dev.tri = (const uint32_t*)(d + oT); dev.edge = (const int4*)(d + oE);
    dev.tree.numNodes = M;
    dev.tree.lo = (const float4*)(d + oLo); dev.tree.hi = (const float4*)(d + oHi);
    dev.tree.children = (const int2*)(d + oCh); dev.tree.primRange = (const int4*)(d + oPr);
    dev.tree.edgeRange = (const int2*)(d + oEr);
    dev.tree.tris = (const uint32_t*)(d + oTr); dev.tree.verts = (const uint32_t*)(d + oVe);
    dev.tree.edges = (const uint32_t*)(d + oEd);
    device = devId;
    return true;
}

// --------------------------------------------------------------- LBVH host
static uint32_t expand_bits(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// Linear BVH over primitive centroids: Morton-ordered primitives, median
// splits (balanced), nodes emitted in depth-first preorder so traversal needs
// no stack (escape index = first node after the subtree). The topology is
// built once from the rest shape; every substep only refits the boxes.
// primitives sorted by the 30-bit Morton code of their centroid in the set's bounds
static std::vector<int> morton_order(const std::vector<V3>& cen)
{
    const int n = (int)cen.size();
    std::vector<int> out(n);
    if (n == 0) return out;
    V3 lo = cen[0], hi = cen[0];
    for (const V3& c : cen) { lo = vmin(lo, c); hi = vmax(hi, c); }
    std::vector<std::pair<uint32_t, int>> key(n);
    for (int i = 0; i < n; i++)
    {
        auto q = [](float v, float a, float b) {
            float t = (b > a) ? (v - a) / (b - a) : 0.5f;
            int x = (int)(t * 1023.f);
            return (uint32_t)std::max(0, std::min(1023, x));
        };
        uint32_t m = (expand_bits(q(cen[i].x, lo.x, hi.x)) << 2) | (expand_bits(q(cen[i].y, lo.y, hi.y)) << 1) |
                     expand_bits(q(cen[i].z, lo.z, hi.z));
        key[i] = {m, i};
    }
    std::sort(key.begin(), key.end());
    for (int i = 0; i < n; i++) out[i] = key[i].second;
    return out;
}

void LBVHHost::build(const std::vector<V3>& cen)
{
    const int n = (int)cen.size();
    numLeaves = n;
    numNodes = n > 0 ? 2 * n - 1 : 0;
    child.assign(numNodes, 0); escape.assign(numNodes, 0); parent.assign(numNodes, -1); leafNode.assign(n, 0);
    if (n == 0) return;
    const std::vector<int> order = morton_order(cen);
    std::vector<std::pair<uint32_t, int>> key(n);
    for (int i = 0; i < n; i++) key[i] = {0u, order[i]};
    int next = 0;
    // iterative preorder build over (range, parent, is-right-child) jobs
    struct Job { int lo, hi, par; bool right; int depth; };
    std::vector<Job> jobs{{0, n, -1, false, 0}};
    depth = 0;
    while (!jobs.empty())
    {
        Job j = jobs.back();
        jobs.pop_back();
        int node = next++;
        depth = std::max(depth, j.depth);
        parent[node] = j.par;
        if (j.right && j.par >= 0) child[j.par] = node;
        if (j.hi - j.lo == 1)
        {
            child[node] = ~key[j.lo].second;
            leafNode[key[j.lo].second] = node;
            escape[node] = node + 1;
            continue;
        }
        int mid = (j.lo + j.hi) / 2;
        escape[node] = node + 2 * (j.hi - j.lo) - 1;     // subtree of k leaves has 2k-1 nodes
        jobs.push_back({mid, j.hi, node, true, j.depth + 1});
        jobs.push_back({j.lo, mid, node, false, j.depth + 1});
    }
    // children follow their parent in preorder, so a reverse sweep sees them first
    maxPrim.assign(numNodes, -1);
    for (int k = numNodes - 1; k >= 0; k--)
        maxPrim[k] = child[k] < 0 ? ~child[k] : std::max(maxPrim[k + 1], maxPrim[child[k]]);
}

// ------------------------------------------------------------------ model
ClothModel::~ClothModel()
{
    release_device();
    if (mlpPrm) cudaFree(mlpPrm);
}

void* ClothModel::dalloc(size_t bytes, bool contact)
{
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(&p, bytes) != cudaSuccess)
    {
        set_error(SC_ERR_CUDA, "cudaMalloc failed");
        return nullptr;
    }
    cudaMemset(p, 0, bytes);
    (contact ? bufAllocs : allocs).push_back(p);
    return p;
}

void ClothModel::release_buffers()
{
    for (void* p : bufAllocs) cudaFree(p);
    bufAllocs.clear();
    buf = Buffers{};
    bufWorldVersion = ~0ull;
}

void ClothModel::release_device()
{
    release_buffers();
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    dc = DevCloth{};
    if (stageHost) cudaFreeHost(stageHost);
    stageHost = nullptr;
    stageDev = nullptr;          // one of allocs
}

bool ClothModel::ensure_stage()
{
    if (stageHost && stageDev) return true;
    if (N == 0) return false;
    if (cudaHostAlloc((void**)&stageHost, sizeof(float) * 10 * (size_t)N, cudaHostAllocDefault) != cudaSuccess)
    {
        cudaGetLastError();
        stageHost = nullptr;
        return false;
    }
    stageDev = (float*)dalloc(sizeof(float) * 10 * (size_t)N);
    return stageDev != nullptr;
}

SolverParams ClothModel::solver_params(float h) const
{
    SolverParams P;
    P.unit = prm.unit; P.thickness = prm.thickness; P.tolerance = prm.tolerance; P.shear = prm.shear;
    P.bend = prm.bend; P.poisson = prm.poisson; P.friction = prm.friction; P.drag = prm.drag;
    P.selfShrink = prm.selfShrink;
    P.h = h; P.h2 = h * h; P.invH = 1.f / h;
    // epsilonUV = 1 / shear modulus (Physics/ClothPBD.cpp:56)
    P.epsUV = 2 * (1 + prm.poisson) / (std::max(prm.shear, 0.1f) * prm.unit * prm.unit);
    P.iterations = prm.iterations; P.flags = prm.flags; P.fem = prm.fem; P.dihedral = prm.dihedral;
    P.fixedIterations = prm.fixedIterations; P.bendFreq = prm.bendFreq;
    P.resTol = prm.resTol;
    P.area = prm.area;
    P.resScale = prm.resMetres ? 1.f : resScale;
    P.selfThreshold = prm.selfThreshold;
    return P;
}

// Greedy colouring in index order on the particle-sharing graph: each
// constraint takes the lowest colour unused by earlier constraints on its
// particles. Solve order = (colour, index).
template <int K, typename Get>
static void greedy_colour(int n, int N, Get verts, std::vector<int>& order, std::vector<int>& start)
{
    std::vector<uint64_t> used(N, 0);
    std::vector<int> col(n, 0);
    int maxc = 0;
    for (int i = 0; i < n; i++)
    {
        uint32_t v[K];
        verts(i, v);
        uint64_t u = 0;
        for (int k = 0; k < K; k++) u |= used[v[k]];
        int c = 0;
        while (c < 64 && (u >> c & 1ull)) c++;
        if (c >= 64) c = 63;
        col[i] = c;
        maxc = std::max(maxc, c + 1);
        for (int k = 0; k < K; k++) used[v[k]] |= 1ull << c;
    }
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return col[a] < col[b]; });
    start.assign(maxc + 1, 0);
    for (int i = 0; i < n; i++) start[col[i] + 1]++;
    for (int c = 0; c < maxc; c++) start[c + 1] += start[c];
}

// Exact colouring of a small conflict graph (items sharing a vertex conflict)
// with at most K colours: DSatur order with backtracking, bounded. Empty if none
// is found within the budget.
static std::vector<int> exact_colouring(const std::vector<std::vector<int>>& verts, int K)
{
    const int m = (int)verts.size();
    std::vector<std::vector<int>> nb(m);
    for (int a = 0; a < m; a++)
        for (int b = 0; b < m; b++)
        {
            if (a == b) continue;
            bool share = false;
            for (int x : verts[a]) for (int y : verts[b]) share |= x == y;
            if (share) nb[a].push_back(b);
        }
    std::vector<int> tc(m, -1);
    long budget = 5000000;
    std::function<bool()> search = [&]() -> bool {
        int best = -1, bs = -1, bd = -1;
        for (int a = 0; a < m; a++)
        {
            if (tc[a] >= 0) continue;
            uint32_t used = 0;
            for (int b : nb[a]) if (tc[b] >= 0) used |= 1u << tc[b];
            const int s = __builtin_popcount(used), d = (int)nb[a].size();
            if (s > bs || (s == bs && d > bd)) { best = a; bs = s; bd = d; }
        }
        if (best < 0) return true;
        if (--budget < 0) return false;
        uint32_t used = 0;
        int top = -1;
        for (int a = 0; a < m; a++) top = std::max(top, tc[a]);
        for (int b : nb[best]) if (tc[b] >= 0) used |= 1u << tc[b];
        for (int k = 0; k < K && k <= top + 1; k++)
        {
            if (used >> k & 1u) continue;
            tc[best] = k;
            if (search()) return true;
            tc[best] = -1;
        }
        return false;
    };
    if (K > 32 || !search()) return {};
    return tc;
}

// true if no particle is in two constraints of one colour
template <int V, typename Get>
static bool proper_colouring(int n, int N, Get verts, const std::vector<int>& col)
{
    std::vector<uint64_t> seen(N, 0);
    for (int k = 0; k < n; k++)
    {
        uint32_t v[V];
        verts(k, v);
        for (uint32_t x : v)
        {
            if (col[k] < 0 || col[k] >= 64 || (seen[x] >> col[k] & 1ull)) return false;
            seen[x] |= 1ull << col[k];
        }
    }
    return true;
}

// Bends of grid clothes, coloured with a pattern of period 4 in both grid
// directions: the 48 bends of the 4 x 4 torus triangulated like the grid
// (alternating diagonals by cell parity) are coloured once by an exact search
// with 16 colours — the most bends that share one particle, so the fewest
// possible — and every bend takes the colour of its edge's image on the torus.
// Two bends sharing a particle have images sharing a vertex, and distinct bends
// within reach of each other have distinct images, so the colouring is proper;
// it is checked anyway, and false means "use the greedy colouring".
static bool periodic_bend_colours(const std::vector<uint4>& bends, const std::vector<int2>& ij, int N, std::vector<int>& col)
{
    const int P = 4, K = 16;
    auto T = [&](int j, int i) { return ((j % P + P) % P) * P + ((i % P + P) % P); };
    // torus triangles, the cell rule of ClothPatch::Init(grid)
    std::vector<std::array<int, 3>> tri;
    for (int j = 0; j < P; j++)
        for (int i = 0; i < P; i++)
        {
            const int a = T(j - 1, i - 1), b = T(j - 1, i), c = T(j, i), d = T(j, i - 1);
            if ((i & 1) == (j & 1)) { tri.push_back({a, c, b}); tri.push_back({a, d, c}); }
            else { tri.push_back({b, d, c}); tri.push_back({d, b, a}); }
        }
    std::map<std::pair<int, int>, std::vector<int>> opp;
    for (auto& t : tri)
        for (int k = 0; k < 3; k++)
        {
            const int x = t[k], y = t[(k + 1) % 3], z = t[(k + 2) % 3];
            opp[{std::min(x, y), std::max(x, y)}].push_back(z);
        }
    std::vector<std::pair<int, int>> key;
    std::vector<std::vector<int>> tv;
    for (auto& e : opp)
    {
        if (e.second.size() != 2) return false;
        key.push_back(e.first);
        tv.push_back({e.first.first, e.first.second, e.second[0], e.second[1]});
    }
    const std::vector<int> tc = exact_colouring(tv, K);
    if (tc.empty()) return false;
    std::map<std::pair<int, int>, int> colourOf;
    for (size_t a = 0; a < key.size(); a++) colourOf[key[a]] = tc[a];
    col.assign(bends.size(), 0);
    for (size_t k = 0; k < bends.size(); k++)
    {
        const int2 p = ij[bends[k].x], q = ij[bends[k].y];
        const int u = T(p.x, p.y), v = T(q.x, q.y);
        auto it = colourOf.find({std::min(u, v), std::max(u, v)});
        if (it == colourOf.end()) return false;
        col[k] = it->second;
    }
    return proper_colouring<4>((int)bends.size(), N, [&](int k, uint32_t* v) {
        v[0] = bends[k].x; v[1] = bends[k].y; v[2] = bends[k].z; v[3] = bends[k].w; }, col);
}

// Links of grid clothes (stretch (0,1), (1,0); shear (1,1), (1,-1); bend (0,2),
// (2,0) in grid steps, ClothPatch::Init(grid)), coloured with a pattern of
// period 6: the 216 links of the 6 x 6 torus are coloured once by an exact
// search with 12 colours — the links at one particle, so the fewest possible —
// and every link takes its image's colour. Period 6 is the smallest that keeps
// the images of two links at one particle apart (the bend links span two steps)
// and admits 12 colours. Checked proper; false means "use the greedy colouring".
static bool periodic_link_colours(const std::vector<uint2>& links, const std::vector<int2>& ij, int N, std::vector<int>& col)
{
    const int P = 6, K = 12;
    auto T = [&](int j, int i) { return ((j % P + P) % P) * P + ((i % P + P) % P); };
    const int off[6][2] = {{0, 1}, {1, 0}, {1, 1}, {1, -1}, {0, 2}, {2, 0}};
    std::map<std::pair<int, int>, int> index;
    std::vector<std::vector<int>> tv;
    for (int j = 0; j < P; j++)
        for (int i = 0; i < P; i++)
            for (auto& o : off)
            {
                const int u = T(j, i), v = T(j + o[0], i + o[1]);
                const std::pair<int, int> k{std::min(u, v), std::max(u, v)};
                if (index.count(k)) return false;            // two links with one image
                index[k] = (int)tv.size();
                tv.push_back({u, v});
            }
    const std::vector<int> tc = exact_colouring(tv, K);
    if (tc.empty()) return false;
    col.assign(links.size(), 0);
    for (size_t k = 0; k < links.size(); k++)
    {
        const int2 p = ij[links[k].x], q = ij[links[k].y];
        const int u = T(p.x, p.y), v = T(q.x, q.y);
        auto it = index.find({std::min(u, v), std::max(u, v)});
        if (it == index.end()) return false;
        col[k] = tc[it->second];
    }
    return proper_colouring<2>((int)links.size(), N, [&](int k, uint32_t* v) { v[0] = links[k].x; v[1] = links[k].y; },
                               col);
}

// Edges of a grid cloth (any particle pairs with grid coordinates), coloured with a
// pattern of period P: the distinct images of the edges on the P x P torus are
// coloured by an exact search with K colours and every edge takes its image's
// colour. Checked proper; false means "keep the greedy colouring".
static bool periodic_pair_colours(const std::vector<uint2>& pairs, const std::vector<int2>& ij, int N, int P, int K,
                                  std::vector<int>& col)
{
    auto T = [&](int j, int i) { return ((j % P + P) % P) * P + ((i % P + P) % P); };
    std::map<std::pair<int, int>, int> index;
    std::vector<std::vector<int>> tv;
    for (const uint2& e : pairs)
    {
        const int2 p = ij[e.x], q = ij[e.y];
        const int u = T(p.x, p.y), v = T(q.x, q.y);
        if (u == v) return false;
        const std::pair<int, int> k{std::min(u, v), std::max(u, v)};
        if (!index.count(k)) { index[k] = (int)tv.size(); tv.push_back({u, v}); }
    }
    if (tv.size() > 4096) return false;
    const std::vector<int> tc = exact_colouring(tv, K);
    if (tc.empty()) return false;
    col.assign(pairs.size(), 0);
    for (size_t k = 0; k < pairs.size(); k++)
    {
        const int2 p = ij[pairs[k].x], q = ij[pairs[k].y];
        const int u = T(p.x, p.y), v = T(q.x, q.y);
        col[k] = tc[index[{std::min(u, v), std::max(u, v)}]];
    }
    return proper_colouring<2>((int)pairs.size(), N, [&](int k, uint32_t* v) { v[0] = pairs[k].x; v[1] = pairs[k].y; }, col);
}

// replace a greedy (colour, index) order by the one of `col` when it needs fewer colours
static void adopt_colours(const std::vector<int>& col, std::vector<int>& order, std::vector<int>& start)
{
    if (col.empty()) return;
    const int K = *std::max_element(col.begin(), col.end()) + 1;
    if (K >= (int)start.size() - 1) return;
    order.resize(col.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return col[a] < col[b]; });
    start.assign(K + 1, 0);
    for (int c : col) start[c + 1]++;
    for (int c = 0; c < K; c++) start[c + 1] += start[c];
}

void ClothModel::colour_constraints()
{
    greedy_colour<3>((int)tris.size(), N, [&](int i, uint32_t* v) { v[0] = tris[i].i1; v[1] = tris[i].i2; v[2] = tris[i].i3; },
                     triOrder, triColourStart);
    greedy_colour<4>((int)bends.size(), N, [&](int i, uint32_t* v) { v[0] = bends[i].x; v[1] = bends[i].y; v[2] = bends[i].z; v[3] = bends[i].w; },
                     bendOrder, bendColourStart);
    greedy_colour<2>((int)links.size(), N, [&](int i, uint32_t* v) { v[0] = links[i].x; v[1] = links[i].y; },
                     linkOrder, linkColourStart);
    // grid clothes: the periodic colourings, where they need fewer colours
    if ((int)gridIJ.size() == N)
    {
        std::vector<int> col;
        if (!bends.empty() && periodic_bend_colours(bends, gridIJ, N, col)) adopt_colours(col, bendOrder, bendColourStart);
        col.clear();
        if (!links.empty() && periodic_link_colours(links, gridIJ, N, col)) adopt_colours(col, linkOrder, linkColourStart);
    }
}

// Band plan of the band-parallel solver (k_gs_band): the largest cluster (16, 8,
// 4 or 2 CTAs) whose bands of 2^shift consecutive particles admit every FEM
// triangle, bend and link either as an interior record of the band of its lowest
// particle or as a boundary record reaching only the first `halo` particles of
// the next band, where every band's boundary records touch their own band at
// offsets >= halo. Grid clothes (particles row by row) satisfy it once a band
// holds a few rows; batches never use it.
void ClothModel::build_band_plan()
{
    bandPlan = BandPlan{};
    if (!instV.empty() || N < 64) return;
    // the kernel keeps a band's record offsets in shared memory: at most 64 colours a class
    if (triColourStart.size() > 65 || bendColourStart.size() > 65 || linkColourStart.size() > 65) return;
    struct Cls
    {
        int arity;
        const std::vector<int>* order;
        const std::vector<int>* start;
        std::function<void(int, uint32_t*)> get;
    };
    const Cls cls[3] = {
        {3, &triOrder, &triColourStart, [&](int i, uint32_t* v) { v[0] = tris[i].i1; v[1] = tris[i].i2; v[2] = tris[i].i3; }},
        {4, &bendOrder, &bendColourStart, [&](int i, uint32_t* v) { v[0] = bends[i].x; v[1] = bends[i].y; v[2] = bends[i].z; v[3] = bends[i].w; }},
        {2, &linkOrder, &linkColourStart, [&](int i, uint32_t* v) { v[0] = links[i].x; v[1] = links[i].y; }}};
    for (int cs : {16, 8, 4, 2})
    {
        int shift = 0;
        while (((size_t)1 << shift) * cs < (size_t)N) shift++;
        const int vpc = 1 << shift;
        if ((size_t)vpc * (cs - 1) >= (size_t)N) continue;            // a band would be empty
        if ((size_t)vpc * sizeof(float4) > 128 * 1024) continue;
        // part (0 interior, 1 boundary) of every record, the halo, and per band the
        // smallest own-band offset its boundary records touch
        int halo = 0;
        bool ok = true;
        std::vector<int> minOwn(cs, vpc);
        std::vector<std::vector<uint8_t>> part(3);
        for (int k = 0; k < 3 && ok; k++)
        {
            const Cls& q = cls[k];
            const int n = (int)q.order->size();
            part[k].assign(n, 0);
            for (int r = 0; r < n && ok; r++)
            {
                uint32_t v[4];
                q.get(r, v);
                uint32_t lo = v[0], hi = v[0];
                for (int a = 1; a < q.arity; a++) { lo = std::min(lo, v[a]); hi = std::max(hi, v[a]); }
                const int b = (int)(lo >> shift), hb = (int)(hi >> shift);
                if (hb == b) continue;
                if (hb != b + 1) { ok = false; break; }
                part[k][r] = 1;
                for (int a = 0; a < q.arity; a++)
                {
                    const int o = (int)(v[a] & (uint32_t)(vpc - 1));
                    if ((int)(v[a] >> shift) == b + 1) halo = std::max(halo, o + 1);
                    else minOwn[b] = std::min(minOwn[b], o);
                }
            }
        }
        for (int b = 0; b < cs && ok; b++) ok = minOwn[b] >= halo;
        if (!ok || halo > vpc) continue;
        const int haloPad = (halo + 15) & ~15;
        if (!gs_band_fits(cs, (size_t)(vpc + haloPad) * sizeof(float4))) continue;
        // records in (band, part, colour, colour order) order with their offsets,
        // and the reported order (part, colour, band, colour order)
        BandPlan& bp = bandPlan;
        bp.clusterSize = cs; bp.shift = shift; bp.halo = halo;
        std::vector<int>* outOrder[3] = {&bp.triOrder, &bp.bendOrder, &bp.linkOrder};
        std::vector<int>* outStart[3] = {&bp.triStart, &bp.bendStart, &bp.linkStart};
        int* most[3] = {&bp.femMax, &bp.bendMax, &bp.linkMax};
        std::vector<int> offs[3];
        std::vector<int> devOrder[3];
        for (int k = 0; k < 3; k++)
        {
            const Cls& q = cls[k];
            const int nCol = std::max(1, (int)q.start->size() - 1), n = (int)q.order->size();
            std::vector<int> colOf(n, 0), bandOf(n, 0);
            for (int c = 0; c + 1 < (int)q.start->size(); c++)
                for (int j = (*q.start)[c]; j < (*q.start)[c + 1]; j++) colOf[(*q.order)[j]] = c;
            for (int r = 0; r < n; r++)
            {
                uint32_t v[4];
                q.get(r, v);
                uint32_t lo = v[0];
                for (int a = 1; a < q.arity; a++) lo = std::min(lo, v[a]);
                bandOf[r] = (int)(lo >> shift);
            }
            // position of each record in the colour order: ties keep it
            std::vector<int> rank(n, 0);
            for (int j = 0; j < n; j++) rank[(*q.order)[j]] = j;
            std::vector<int> idx(n);
            std::iota(idx.begin(), idx.end(), 0);
            auto key = [&](int r) { return ((int64_t)(bandOf[r] * 2 + part[k][r]) * nCol + colOf[r]) * (int64_t)(n + 1) + rank[r]; };
            std::sort(idx.begin(), idx.end(), [&](int x, int y) { return key(x) < key(y); });
            devOrder[k] = idx;
            offs[k].assign((size_t)cs * 2 * nCol + 1, 0);
            for (int r = 0; r < n; r++) offs[k][(size_t)(bandOf[r] * 2 + part[k][r]) * nCol + colOf[r] + 1]++;
            for (size_t g = 1; g < offs[k].size(); g++) offs[k][g] += offs[k][g - 1];
            *most[k] = 0;
            for (int b = 0; b < cs; b++) *most[k] = std::max(*most[k], offs[k][(size_t)(b + 1) * 2 * nCol] - offs[k][(size_t)b * 2 * nCol]);
            auto key2 = [&](int r) { return ((int64_t)(part[k][r] * nCol + colOf[r]) * cs + bandOf[r]) * (int64_t)(n + 1) + rank[r]; };
            std::vector<int> rep(n);
            std::iota(rep.begin(), rep.end(), 0);
            std::sort(rep.begin(), rep.end(), [&](int x, int y) { return key2(x) < key2(y); });
            *outOrder[k] = rep;
            outStart[k]->assign(1, 0);
            for (int g = 0; g < 2 * nCol; g++)
            {
                int cnt = 0;
                for (int b = 0; b < cs; b++)
                    cnt += offs[k][(size_t)(b * 2 + g / nCol) * nCol + g % nCol + 1] - offs[k][(size_t)(b * 2 + g / nCol) * nCol + g % nCol];
                if (cnt) outStart[k]->push_back(outStart[k]->back() + cnt);
            }
        }
        // device arrays
        BandView& v = bp.view;
        v.shift = shift; v.halo = halo;
        v.nFemCol = std::max(1, (int)triColourStart.size() - 1);
        v.nBendCol = std::max(1, (int)bendColourStart.size() - 1);
        v.nLinkCol = std::max(1, (int)linkColourStart.size() - 1);
        int* doff[3];
        for (int k = 0; k < 3; k++)
        {
            doff[k] = (int*)dalloc(sizeof(int) * offs[k].size());
            SC_CUDA_V(cudaMemcpy(doff[k], offs[k].data(), sizeof(int) * offs[k].size(), cudaMemcpyHostToDevice));
        }
        v.femOff = doff[0]; v.bendOff = doff[1]; v.linkOff = doff[2];
        const int T = (int)tris.size(), B = (int)bends.size(), L = (int)links.size();
        std::vector<float4> fem(3 * (size_t)std::max(1, T));
        for (int j = 0; j < T; j++)
        {
            const FemHost& t = tris[devOrder[0][j]];
            fem[3 * j] = make_float4(bits_f(t.i1), bits_f(t.i2), bits_f(t.i3), t.du1);
            fem[3 * j + 1] = make_float4(t.du2, t.dv1, t.dv2, t.invDet);
            fem[3 * j + 2] = make_float4(t.lu2, t.lv2, t.lu0 * t.lv0, t.area);
        }
        std::vector<uint4> bd(std::max(1, B));
        for (int j = 0; j < B; j++) bd[j] = bends[devOrder[1][j]];
        std::vector<float4> lk(std::max(1, L));
        for (int j = 0; j < L; j++)
        {
            const int li = devOrder[2][j];
            lk[j] = make_float4(bits_f(links[li].x), bits_f(links[li].y), linkRest[li].x, linkRest[li].y);
        }
        float4* dfem = (float4*)dalloc(sizeof(float4) * fem.size());
        uint4* dbend = (uint4*)dalloc(sizeof(uint4) * bd.size());
        float4* dlink = (float4*)dalloc(sizeof(float4) * lk.size());
        SC_CUDA_V(cudaMemcpy(dfem, fem.data(), sizeof(float4) * fem.size(), cudaMemcpyHostToDevice));
        SC_CUDA_V(cudaMemcpy(dbend, bd.data(), sizeof(uint4) * bd.size(), cudaMemcpyHostToDevice));
        SC_CUDA_V(cudaMemcpy(dlink, lk.data(), sizeof(float4) * lk.size(), cudaMemcpyHostToDevice));
        v.fem = dfem; v.bend = dbend; v.link = dlink;
        v.femMax = bp.femMax; v.bendMax = bp.bendMax; v.linkMax = bp.linkMax;
        bp.valid = true;
        return;
    }
}

// dynamic shared memory of the band solver: own band, halo and the staged
// records; chooses what to stage (FEM, then bends, then links) within the limit
size_t ClothModel::band_smem()
{
    BandView& v = bandPlan.view;
    size_t bytes = ((size_t)(1 << bandPlan.shift) + (size_t)((bandPlan.halo + 15) & ~15)) * sizeof(float4);
    v.stageFem = v.stageBend = v.stageLink = 0;
    if (!prm.stageRecords) return bytes;
    const size_t fem = (size_t)3 * bandPlan.femMax * sizeof(float4), bend = (size_t)bandPlan.bendMax * sizeof(uint4),
                 link = (size_t)bandPlan.linkMax * sizeof(float4);
    auto fits = [&](size_t extra) { return bytes + extra <= (size_t)BAND_SMEM_MAX && gs_band_fits(bandPlan.clusterSize, bytes + extra); };
    if (prm.fem && fits(fem)) { bytes += fem; v.stageFem = 1; }
    if (prm.dihedral && fits(bend)) { bytes += bend; v.stageBend = 1; }
    if (!prm.fem && fits(link)) { bytes += link; v.stageLink = 1; }
    return bytes;
}

bool ClothModel::upload_topology(const HMesh& mesh)
{
    release_device();
    SC_CUDA(cudaGetDevice(&device));
    const int T = (int)tris.size(), E = (int)mesh.edges.size(), B = (int)bends.size();
    if (T >= (1 << 24))
    {
        // triangle contacts carry the triangle index in 24 bits
        set_error(SC_ERR_UNSUPPORTED, "cloth has more than 16,777,215 triangles");
        return false;
    }
    dc.N = N; dc.T = T; dc.E = E; dc.B = B;
    colour_constraints();
    // particle state
    dc.pos = (float4*)dalloc(sizeof(float4) * N);
    dc.prev = (float4*)dalloc(sizeof(float4) * N);
    dc.vel = (float4*)dalloc(sizeof(float4) * N);
    // FEM records in colour order
    std::vector<float4> fem(3 * (size_t)T);
    for (int k = 0; k < T; k++)
    {
        const FemHost& t = tris[triOrder[k]];
        fem[3 * k] = make_float4(bits_f(t.i1), bits_f(t.i2), bits_f(t.i3), t.du1);
        fem[3 * k + 1] = make_float4(t.du2, t.dv1, t.dv2, t.invDet);
        fem[3 * k + 2] = make_float4(t.lu2, t.lv2, t.lu0 * t.lv0, t.area);
    }
    float4* dfem = (float4*)dalloc(sizeof(float4) * 3 * (size_t)T);
    SC_CUDA(cudaMemcpy(dfem, fem.data(), sizeof(float4) * 3 * (size_t)T, cudaMemcpyHostToDevice));
    dc.fem = dfem;
    // link records in colour order (mass-spring path)
    const int L = (int)links.size();
    std::vector<float4> lk(std::max(1, L));
    for (int k = 0; k < L; k++)
    {
        const int li = linkOrder[k];
        lk[k] = make_float4(bits_f(links[li].x), bits_f(links[li].y), linkRest[li].x, linkRest[li].y);
    }
    float4* dlink = (float4*)dalloc(sizeof(float4) * lk.size());
    SC_CUDA(cudaMemcpy(dlink, lk.data(), sizeof(float4) * lk.size(), cudaMemcpyHostToDevice));
    dc.link = dlink;
    dc.L = L;
    // the Jacobi and conjugate-residual solves: links in index order, each
    // particle's incident links in increasing index
    {
        std::vector<float4> lo(std::max(1, L));
        std::vector<int> start(N + 1, 0), inc(std::max(1, 2 * L));
        for (int k = 0; k < L; k++)
        {
            lo[k] = make_float4(bits_f(links[k].x), bits_f(links[k].y), linkRest[k].x, linkRest[k].y);
            start[links[k].x + 1]++;
            start[links[k].y + 1]++;
        }
        for (int i = 0; i < N; i++) start[i + 1] += start[i];
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int k = 0; k < L; k++)
        {
            inc[fill[links[k].x]++] = k << 1;
            inc[fill[links[k].y]++] = (k << 1) | 1;
        }
        LinkSolve& ls = linkSolve;
        ls.L = L;
        float4* a = (float4*)dalloc(sizeof(float4) * lo.size());
        SC_CUDA(cudaMemcpy(a, lo.data(), sizeof(float4) * lo.size(), cudaMemcpyHostToDevice));
        ls.link = a;
        ls.disp = (float4*)dalloc(sizeof(float4) * lo.size());
        ls.d = (float*)dalloc(sizeof(float) * lo.size());
        int* st = (int*)dalloc(sizeof(int) * start.size());
        int* ic = (int*)dalloc(sizeof(int) * inc.size());
        SC_CUDA(cudaMemcpy(st, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(ic, inc.data(), sizeof(int) * inc.size(), cudaMemcpyHostToDevice));
        ls.incStart = st;
        ls.inc = ic;
    }
    std::vector<uint4> bd(B);
    for (int k = 0; k < B; k++) bd[k] = bends[bendOrder[k]];
    uint4* dbend = (uint4*)dalloc(sizeof(uint4) * B);
    if (B) SC_CUDA(cudaMemcpy(dbend, bd.data(), sizeof(uint4) * B, cudaMemcpyHostToDevice));
    dc.bend = dbend;
    build_band_plan();
    // static colours of triangles (their FEM colours) and of collision-mesh edges
    // (greedy in index order; grids: a period-4 pattern when it needs fewer) for
    // the triangle and edge collider contacts
    {
        std::vector<uint8_t> tcol(std::max(1, T), 0), ecol(std::max(1, E), 0);
        dc.nTriColours = std::max(1, (int)triColourStart.size() - 1);
        for (int c = 0; c + 1 < (int)triColourStart.size(); c++)
            for (int k = triColourStart[c]; k < triColourStart[c + 1]; k++) tcol[triOrder[k]] = (uint8_t)std::min(c, 255);
        std::vector<uint2> ep(E);
        for (int e = 0; e < E; e++) ep[e] = make_uint2(mesh.edges[e].i1, mesh.edges[e].i2);
        std::vector<int> eord, estart;
        greedy_colour<2>(E, N, [&](int i, uint32_t* v) { v[0] = ep[i].x; v[1] = ep[i].y; }, eord, estart);
        std::vector<int> col(E, 0);
        for (int c = 0; c + 1 < (int)estart.size(); c++)
            for (int k = estart[c]; k < estart[c + 1]; k++) col[eord[k]] = c;
        int ncol = std::max(1, (int)estart.size() - 1);
        if ((int)gridIJ.size() == N && E > 0)
        {
            std::vector<int> deg(N, 0);
            for (const uint2& e : ep) { deg[e.x]++; deg[e.y]++; }
            const int K = *std::max_element(deg.begin(), deg.end());
            std::vector<int> pc;
            if (K < ncol && periodic_pair_colours(ep, gridIJ, N, 4, K, pc)) { col = pc; ncol = K; }
        }
        for (int e = 0; e < E; e++) ecol[e] = (uint8_t)std::min(col[e], 255);
        dc.nEdgeColours = ncol;
        edgeColourHost = col;
        uint8_t* dt = (uint8_t*)dalloc(tcol.size());
        uint8_t* de = (uint8_t*)dalloc(ecol.size());
        SC_CUDA(cudaMemcpy(dt, tcol.data(), tcol.size(), cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(de, ecol.data(), ecol.size(), cudaMemcpyHostToDevice));
        dc.triColour = dt;
        dc.edgeColour = de;
    }
    // collision-mesh topology
    uint32_t* dtri = (uint32_t*)dalloc(sizeof(uint32_t) * 3 * (size_t)T);
    SC_CUDA(cudaMemcpy(dtri, mesh.idx.data(), sizeof(uint32_t) * 3 * (size_t)T, cudaMemcpyHostToDevice));
    dc.tri = dtri;
    uint32_t* dtriE = (uint32_t*)dalloc(sizeof(uint32_t) * 3 * (size_t)T);
    SC_CUDA(cudaMemcpy(dtriE, mesh.triE.data(), sizeof(uint32_t) * 3 * (size_t)T, cudaMemcpyHostToDevice));
    dc.triE = dtriE;
    std::vector<int4> ed(E);
    std::vector<uint8_t> sw(E);
    for (int e = 0; e < E; e++)
    {
        ed[e] = make_int4((int)mesh.edges[e].i1, (int)mesh.edges[e].i2, mesh.edges[e].t1, mesh.edges[e].t2);
        sw[e] = mesh.edges[e].swapped ? 1 : 0;
    }
    int4* dedge = (int4*)dalloc(sizeof(int4) * E);
    SC_CUDA(cudaMemcpy(dedge, ed.data(), sizeof(int4) * E, cudaMemcpyHostToDevice));
    dc.edge = dedge;
    uint8_t* dsw = (uint8_t*)dalloc(E);
    SC_CUDA(cudaMemcpy(dsw, sw.data(), E, cudaMemcpyHostToDevice));
    dc.edgeSwapped = dsw;
    auto csr = [&](const std::vector<std::vector<int>>& lists, const int*& startOut, const int*& dataOut) -> bool {
        std::vector<int> st(N + 1, 0), data;
        for (int i = 0; i < N; i++) { st[i + 1] = st[i] + (int)lists[i].size(); data.insert(data.end(), lists[i].begin(), lists[i].end()); }
        int* ds = (int*)dalloc(sizeof(int) * (N + 1));
        int* dd = (int*)dalloc(sizeof(int) * (data.size() + 1));
        SC_CUDA(cudaMemcpy(ds, st.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice));
        if (!data.empty()) SC_CUDA(cudaMemcpy(dd, data.data(), sizeof(int) * data.size(), cudaMemcpyHostToDevice));
        startOut = ds; dataOut = dd;
        return true;
    };
    if (!csr(mesh.vtxRing, dc.vRingStart, dc.vRing)) return false;
    if (!csr(mesh.edgeRing, dc.eRingStart, dc.eRing)) return false;
    {
        std::vector<int> st(N + 1, 0);
        std::vector<int2> vt(3 * (size_t)T);
        for (int t = 0; t < T; t++) for (int k = 0; k < 3; k++) st[mesh.idx[3 * t + k] + 1]++;
        for (int i = 0; i < N; i++) st[i + 1] += st[i];
        std::vector<int> cur(st.begin(), st.end() - 1);
        for (int t = 0; t < T; t++) for (int k = 0; k < 3; k++) vt[cur[mesh.idx[3 * t + k]]++] = make_int2(t, k);
        int* ds = (int*)dalloc(sizeof(int) * (N + 1));
        int2* dv = (int2*)dalloc(sizeof(int2) * 3 * (size_t)T);
        SC_CUDA(cudaMemcpy(ds, st.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(dv, vt.data(), sizeof(int2) * 3 * (size_t)T, cudaMemcpyHostToDevice));
        dc.vTriStart = ds; dc.vTri = dv;
    }
    std::vector<uint8_t> border(N, 0);
    for (int i = 0; i < N; i++) for (int e : mesh.edgeRing[i]) if (mesh.edges[e].t2 < 0) border[i] = 1;
    uint8_t* dborder = (uint8_t*)dalloc(N);
    SC_CUDA(cudaMemcpy(dborder, border.data(), N, cudaMemcpyHostToDevice));
    dc.vBorder = dborder;
    {
        // query orders for the tree traversals: spatially adjacent queries share a
        // warp, so its lanes walk the same subtrees (vertices and edge centroids by
        // Morton code of the rest shape)
        std::vector<V3> ec(E);
        for (int e = 0; e < E; e++) ec[e] = 0.5f * (hpos[mesh.edges[e].i1] + hpos[mesh.edges[e].i2]);
        std::vector<int> vq, eq;
        if (instV.empty()) { vq = morton_order(hpos); eq = morton_order(ec); }
        else
        {
            // a batch: instance after instance, Morton order inside each
            for (size_t k = 0; k + 1 < instV.size(); k++)
            {
                for (int v : morton_order(std::vector<V3>(hpos.begin() + instV[k], hpos.begin() + instV[k + 1])))
                    vq.push_back(v + instV[k]);
                for (int e : morton_order(std::vector<V3>(ec.begin() + instE[k], ec.begin() + instE[k + 1])))
                    eq.push_back(e + instE[k]);
            }
            std::vector<int> vi(N);
            for (size_t k = 0; k + 1 < instV.size(); k++)
                for (int v = instV[k]; v < instV[k + 1]; v++) vi[v] = (int)k;
            int* dv = (int*)dalloc(sizeof(int) * ((size_t)N + instV.size()));
            SC_CUDA(cudaMemcpy(dv, vi.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
            SC_CUDA(cudaMemcpy(dv + N, instV.data(), sizeof(int) * instV.size(), cudaMemcpyHostToDevice));
            dc.vInst = dv;
            dc.instStart = dv + N;
        }
        int* d = (int*)dalloc(sizeof(int) * ((size_t)N + E + 2));
        SC_CUDA(cudaMemcpy(d, vq.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
        if (E) SC_CUDA(cudaMemcpy(d + N, eq.data(), sizeof(int) * E, cudaMemcpyHostToDevice));
        dc.vQuery = d; dc.eQuery = d + N;
    }
    {
        // rest length of every edge from the uv layout (warm-start strain feature)
        std::vector<float> rest(std::max(1, E), 1.f);
        for (int e = 0; e < E; e++)
        {
            const int a = mesh.edges[e].i1, b2 = mesh.edges[e].i2;
            const float du = uvx[b2] - uvx[a], dv = uvy[b2] - uvy[a];
            const float l = std::sqrt(du * du + dv * dv);
            rest[e] = l > 0.f ? l : 1.f;
        }
        float* dr = (float*)dalloc(sizeof(float) * rest.size());
        SC_CUDA(cudaMemcpy(dr, rest.data(), sizeof(float) * rest.size(), cudaMemcpyHostToDevice));
        dc.edgeRest = dr;
        double sum = 0;
        for (int e = 0; e < E; e++) sum += rest[e];
        resScale = E > 0 ? (float)(E / sum) : 1.f;
        dc.xsnap = (float4*)dalloc(sizeof(float4) * (size_t)N);
        dc.xpred = (float4*)dalloc(sizeof(float4) * (size_t)N);
        dc.lastCorr = (float*)dalloc(sizeof(float) * (size_t)N);
    }
    dc.prevN = (float4*)dalloc(sizeof(float4) * N);
    dc.prevTriN = (float4*)dalloc(sizeof(float4) * T);
    dc.meshN = (float4*)dalloc(sizeof(float4) * N);
    dc.meshTriN = (float4*)dalloc(sizeof(float4) * T);
    dc.triAngles = (float4*)dalloc(sizeof(float4) * T);
    dc.scal = (float*)dalloc(sizeof(float) * 16);
    dc.status = (int*)dalloc(sizeof(int) * 4);
    {
        // collision-mesh normals as of the initial mesh (ClothPatch::Init copies
        // mMesh, normals included, into mPrevMesh)
        std::vector<float4> n4(N), t4(T);
        for (int i = 0; i < N; i++) n4[i] = f4(mesh.normals[i], 0);
        for (int t = 0; t < T; t++) t4[t] = f4(mesh.triN[t], 0);
        SC_CUDA(cudaMemcpy(dc.prevN, n4.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(dc.prevTriN, t4.data(), sizeof(float4) * T, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(dc.meshN, n4.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(dc.meshTriN, t4.data(), sizeof(float4) * T, cudaMemcpyHostToDevice));
    }
    // BVH topologies from the rest shape
    // upload a built topology (h) with its node boxes' link words
    auto upload_bvh = [&](LBVHHost& h, DevBVH& out, const std::vector<int>* roots) -> bool {
        out.numLeaves = h.numLeaves; out.numNodes = h.numNodes; out.depth = h.depth;
        int* d = (int*)dalloc(sizeof(int) * (4 * (size_t)h.numNodes + h.numLeaves + 4));
        SC_CUDA(cudaMemcpy(d, h.child.data(), sizeof(int) * h.numNodes, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(d + h.numNodes, h.escape.data(), sizeof(int) * h.numNodes, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(d + 2 * h.numNodes, h.parent.data(), sizeof(int) * h.numNodes, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(d + 3 * h.numNodes, h.maxPrim.data(), sizeof(int) * h.numNodes, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(d + 4 * h.numNodes, h.leafNode.data(), sizeof(int) * h.numLeaves, cudaMemcpyHostToDevice));
        out.child = d; out.escape = d + h.numNodes; out.parent = d + 2 * h.numNodes;
        out.maxPrim = d + 3 * h.numNodes; out.leafNode = d + 4 * h.numNodes;
        out.instRoot = nullptr;
        if (roots)
        {
            int* r = (int*)dalloc(sizeof(int) * roots->size());
            SC_CUDA(cudaMemcpy(r, roots->data(), sizeof(int) * roots->size(), cudaMemcpyHostToDevice));
            out.instRoot = r;
        }
        std::vector<float4> lo(h.numNodes), hi(h.numNodes);
        for (int k = 0; k < h.numNodes; k++)
        {
            lo[k] = make_float4(0.f, 0.f, 0.f, bits_f((uint32_t)h.child[k]));
            hi[k] = make_float4(0.f, 0.f, 0.f, bits_f((uint32_t)h.escape[k]));
        }
        out.lo = (float4*)dalloc(sizeof(float4) * h.numNodes);
        out.hi = (float4*)dalloc(sizeof(float4) * h.numNodes);
        SC_CUDA(cudaMemcpy(out.lo, lo.data(), sizeof(float4) * h.numNodes, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(out.hi, hi.data(), sizeof(float4) * h.numNodes, cudaMemcpyHostToDevice));
        out.visit = (int*)dalloc(sizeof(int) * h.numNodes);
        // child records: static link and maximum words (the refit fills the boxes)
        std::vector<float4> rec(4 * (size_t)h.numNodes, make_float4(0.f, 0.f, 0.f, 0.f));
        for (int k = 0; k < h.numNodes; k++)
        {
            if (h.child[k] < 0) continue;
            const int side[2] = {k + 1, h.child[k]};
            for (int j = 0; j < 2; j++)
            {
                const int ch = side[j];
                const int link = h.child[ch] < 0 ? h.child[ch] : ch;
                rec[4 * (size_t)k + 2 * j + 1].z = bits_f((uint32_t)link);
                rec[4 * (size_t)k + 2 * j + 1].w = bits_f((uint32_t)h.maxPrim[ch]);
            }
        }
        out.rec = (float4*)dalloc(sizeof(float4) * rec.size());
        SC_CUDA(cudaMemcpy(out.rec, rec.data(), sizeof(float4) * rec.size(), cudaMemcpyHostToDevice));
        return true;
    };
    // batch: one tree per instance over its own primitives [start[k], start[k+1]),
    // concatenated (node and primitive indices offset); queries start at their
    // instance's root, so instances never see each other
    auto mkforest = [&](const std::vector<V3>& cen, const std::vector<int>& start, DevBVH& out) -> bool {
        LBVHHost all;
        std::vector<int> roots;
        for (size_t k = 0; k + 1 < start.size(); k++)
        {
            const int p0 = start[k], np = start[k + 1] - start[k];
            const int o = all.numNodes;
            roots.push_back(o);
            if (np == 0) continue;
            LBVHHost h;
            h.build(std::vector<V3>(cen.begin() + p0, cen.begin() + p0 + np));
            for (int j = 0; j < h.numNodes; j++)
            {
                all.child.push_back(h.child[j] < 0 ? ~(~h.child[j] + p0) : h.child[j] + o);
                all.escape.push_back(h.escape[j] + o);
                all.parent.push_back(h.parent[j] < 0 ? -1 : h.parent[j] + o);
                all.maxPrim.push_back(h.maxPrim[j] + p0);
            }
            for (int j = 0; j < np; j++) all.leafNode.push_back(h.leafNode[j] + o);
            all.numNodes += h.numNodes;
            all.numLeaves += h.numLeaves;
            all.depth = std::max(all.depth, h.depth);
        }
        return upload_bvh(all, out, &roots);
    };
    // a tree over cen, or (shareTopo) a second set of boxes over another tree's topology
    auto mkbvh = [&](const std::vector<V3>& cen, DevBVH& out, DevBVH* shareTopo) -> bool {
        if (!shareTopo)
        {
            LBVHHost h;
            h.build(cen);
            return upload_bvh(h, out, nullptr);
        }
        out = *shareTopo;
        std::vector<float4> lo(out.numNodes), hi(out.numNodes);
        SC_CUDA(cudaMemcpy(lo.data(), shareTopo->lo, sizeof(float4) * out.numNodes, cudaMemcpyDeviceToHost));
        SC_CUDA(cudaMemcpy(hi.data(), shareTopo->hi, sizeof(float4) * out.numNodes, cudaMemcpyDeviceToHost));
        out.lo = (float4*)dalloc(sizeof(float4) * out.numNodes);
        out.hi = (float4*)dalloc(sizeof(float4) * out.numNodes);
        SC_CUDA(cudaMemcpy(out.lo, lo.data(), sizeof(float4) * out.numNodes, cudaMemcpyHostToDevice));
        SC_CUDA(cudaMemcpy(out.hi, hi.data(), sizeof(float4) * out.numNodes, cudaMemcpyHostToDevice));
        out.visit = (int*)dalloc(sizeof(int) * out.numNodes);
        out.rec = (float4*)dalloc(sizeof(float4) * 4 * (size_t)out.numNodes);
        SC_CUDA(cudaMemcpy(out.rec, shareTopo->rec, sizeof(float4) * 4 * (size_t)out.numNodes, cudaMemcpyDeviceToDevice));
        return true;
    };
    std::vector<V3> tc(T), ec(E);
    for (int t = 0; t < T; t++)
        tc[t] = (1.f / 3.f) * (hpos[mesh.idx[3 * t]] + hpos[mesh.idx[3 * t + 1]] + hpos[mesh.idx[3 * t + 2]]);
    for (int e = 0; e < E; e++) ec[e] = 0.5f * (hpos[mesh.edges[e].i1] + hpos[mesh.edges[e].i2]);
    if (instV.empty())
    {
        if (!mkbvh(tc, triBvh, nullptr)) return false;
        if (!mkbvh(ec, edgeBvh, nullptr)) return false;
    }
    else
    {
        if (!mkforest(tc, instT, triBvh)) return false;
        if (!mkforest(ec, instE, edgeBvh)) return false;
    }
    if (!mkbvh(tc, sweptTriBvh, &triBvh)) return false;
    if (!mkbvh(ec, sweptEdgeBvh, &edgeBvh)) return false;
    bufWorldVersion = ~0ull;
    return true;
}

void ClothModel::upload_state(cudaStream_t s)
{
    std::vector<float4> p(N), q(N), v(N);
    for (int i = 0; i < N; i++)
    {
        p[i] = f4(hpos[i], invMass[i]);
        q[i] = f4(hprev[i], 0.f);
        v[i] = f4(hvel[i], 0.f);
    }
    cudaMemcpyAsync(dc.pos, p.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dc.prev, q.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dc.vel, v.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
}

void ClothModel::download_state(cudaStream_t s)
{
    static_assert(sizeof(V3) == 3 * sizeof(float), "packed xyz");
    if (ensure_stage())
    {
        const size_t n = N;
        launch_pack_state(s, dc, stageDev);
        cudaMemcpyAsync(stageHost, stageDev, sizeof(float) * 10 * n, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        memcpy(hpos.data(), stageHost, sizeof(float) * 3 * n);
        memcpy(hvel.data(), stageHost + 3 * n, sizeof(float) * 3 * n);
        memcpy(hprev.data(), stageHost + 6 * n, sizeof(float) * 3 * n);
        memcpy(invMass.data(), stageHost + 9 * n, sizeof(float) * n);
        return;
    }
    std::vector<float4> p(N), q(N), v(N);
    cudaMemcpyAsync(p.data(), dc.pos, sizeof(float4) * N, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(q.data(), dc.prev, sizeof(float4) * N, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(v.data(), dc.vel, sizeof(float4) * N, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    for (int i = 0; i < N; i++)
    {
        hpos[i] = mk(p[i]); invMass[i] = p[i].w;
        hprev[i] = mk(q[i]);
        hvel[i] = mk(v[i]);
    }
}

void ClothModel::set_state(const float* pos, const float* prev, const float* vel, cudaStream_t s)
{
    const size_t n = N;
    memcpy(hpos.data(), pos, sizeof(float) * 3 * n);
    memcpy(hprev.data(), prev, sizeof(float) * 3 * n);
    memcpy(hvel.data(), vel, sizeof(float) * 3 * n);
    if (!ensure_stage()) { upload_state(s); return; }
    memcpy(stageHost, pos, sizeof(float) * 3 * n);
    memcpy(stageHost + 3 * n, vel, sizeof(float) * 3 * n);
    memcpy(stageHost + 6 * n, prev, sizeof(float) * 3 * n);
    memcpy(stageHost + 9 * n, invMass.data(), sizeof(float) * n);
    cudaMemcpyAsync(stageDev, stageHost, sizeof(float) * 10 * n, cudaMemcpyHostToDevice, s);
    launch_unpack_state(s, dc, stageDev);
    cudaStreamSynchronize(s);            // the staging buffer is reused by the next transfer
}

// Contact buffers depend on the world's colliders, the collision flags and the
// continuous-collision switch; they are (re)allocated before a graph capture.
bool ClothModel::ensure_buffers(const CollisionWorld& world, cudaStream_t s)
{
    const bool ccd = prm.ccd;
    if (bufWorldVersion == world.version && bufFlags == prm.flags && bufCcd == ccd && buf.vc) return true;
    release_buffers();
    const int T = dc.T, E = dc.E;
    vcollHost.clear();
    std::vector<DevMesh> meshes;
    int slotBase = 0, countBase = 0;
    // (collider, first particle, particles): the world's colliders act on the whole
    // cloth; a batch's on their own instance
    std::vector<BatchColl> entries = batchColl;
    if (instV.empty())
        for (auto& cp : world.list) entries.push_back({cp, 0, N, 0});
    std::vector<int2> instColl(instV.empty() ? 0 : instV.size() - 1, make_int2(0, 0));
    for (auto& en : entries)
    {
        Collidable* c = en.coll.get();
        VColl g = {};
        g.type = c->type;
        g.vBegin = en.vBegin;
        g.vCount = en.vCount;
        if (c->type == CT_WALLS)
        {
            WallsC* w = (WallsC*)c;
            g.kmax = WALL_SLOTS;
            g.a = f4(w->box.lo, 0); g.b = f4(w->box.hi, 0);
        }
        else if (c->type == CT_SPHERE)
        {
            SphereC* sp = (SphereC*)c;
            g.kmax = 1;
            g.a = f4(sp->center, sp->radius);
        }
        else if (c->type == CT_SDF)
        {
            SDFC* sd = (SDFC*)c;
            if (!sd->upload(device)) return false;
            g.kmax = 1;
            g.val = sd->valTex; g.grad = sd->gradTex;
            g.sdfLo = f4(sd->box.lo, 0); g.sdfSteps = f4(sd->steps, 0);
            g.sdfCells = make_int4(sd->nc[0], sd->nc[1], sd->nc[2], 0);
        }
        else if (c->type == CT_MESH)
        {
            MeshC* m = (MeshC*)c;
            // CollisionMesh::Update builds the tree once with the current
            // thickness (Physics/Common.h:124-137)
            if (!m->built) m->build_tree(prm.thickness);
            if (!m->upload(device)) return false;
            g.kmax = 1;
            g.mesh = (int)meshes.size();
            meshes.push_back(m->dev);
        }
        else
        {
            set_error(SC_ERR_UNSUPPORTED, "collidable type not supported by the GPU step (capsule/box/slab); it is ignored");
            continue;
        }
        g.slotBase = slotBase;
        slotBase += g.kmax * g.vCount;
        g.countBase = countBase;
        countBase += g.vCount;
        if (!instColl.empty())
        {
            int2& r = instColl[en.inst];
            if (r.y == 0) r.x = (int)vcollHost.size();
            r.y++;
        }
        vcollHost.push_back(g);
    }
    const int nv = (int)vcollHost.size();
    buf.instColl = nullptr;
    if (!instColl.empty())
    {
        int2* d = (int2*)dalloc(sizeof(int2) * instColl.size(), true);
        SC_CUDA(cudaMemcpy(d, instColl.data(), sizeof(int2) * instColl.size(), cudaMemcpyHostToDevice));
        buf.instColl = d;
    }
    int nTE = 0;
    for (auto& g : vcollHost) if (g.type == CT_SPHERE || g.type == CT_SDF || g.type == CT_MESH) nTE++;
    buf.numVColl = nv;
    buf.vcCount = (uint8_t*)dalloc((size_t)std::max(1, countBase), true);
    buf.vc = (VC*)dalloc(sizeof(VC) * (size_t)std::max(1, slotBase), true);
    VColl* dcoll = (VColl*)dalloc(sizeof(VColl) * std::max(1, nv), true);
    if (nv) SC_CUDA(cudaMemcpy(dcoll, vcollHost.data(), sizeof(VColl) * nv, cudaMemcpyHostToDevice));
    buf.vcoll = dcoll;
    DevMesh* dmeshes = (DevMesh*)dalloc(sizeof(DevMesh) * std::max<size_t>(1, meshes.size()), true);
    if (!meshes.empty()) SC_CUDA(cudaMemcpy(dmeshes, meshes.data(), sizeof(DevMesh) * meshes.size(), cudaMemcpyHostToDevice));
    buf.meshes = dmeshes;
    buf.numMeshes = (int)meshes.size();
    // triangle / edge contacts
    const int nTc = (prm.flags & CF_TRIANGLES) ? nTE : 0, nEc = (prm.flags & CF_EDGES) ? nTE : 0;
    buf.tcCap = std::max(1, nTc * T);
    buf.ecCap = std::max(1, nEc * E);
    buf.tcSlot = (TC*)dalloc(sizeof(TC) * (size_t)buf.tcCap, true);
    buf.tcFlag = (int*)dalloc(sizeof(int) * (size_t)buf.tcCap, true);
    buf.tcList = (TC*)dalloc(sizeof(TC) * (size_t)buf.tcCap, true);
    buf.ecSlot = (EC*)dalloc(sizeof(EC) * (size_t)buf.ecCap, true);
    buf.ecFlag = (int*)dalloc(sizeof(int) * (size_t)buf.ecCap, true);
    buf.ecList = (EC*)dalloc(sizeof(EC) * (size_t)buf.ecCap, true);
    int* counts = (int*)dalloc(sizeof(int) * 16, true);
    buf.tcCount = counts; buf.ecCount = counts + 1; buf.stCount = counts + 2; buf.seCount = counts + 3;
    buf.ccdVtPairCount = counts + 4; buf.ccdEePairCount = counts + 5; buf.scanTot = counts + 8;
    // self contacts
    const bool self = (prm.flags & CF_SELF) != 0;
    // Candidate pairs grow with (swept-box width / edge length)^2: a box of half
    // width r = thickness + tolerance / 2 around a primitive meets about
    // (2 r / l + 1)^2 primitives per layer of cloth; the stores hold four layers'
    // worth, and at least the per-query constants.
    const float r = prm.thickness + 0.5f * prm.tolerance, l = resScale > 0.f ? 1.f / resScale : 1.f;
    const double per = 4.0 * 3.0 * (2.0 * r / l + 1.0) * (2.0 * r / l + 1.0);
    const size_t vtPer = (size_t)std::max<double>(CCD_VT_PAIRS, per), eePer = (size_t)std::max<double>(CCD_EE_PAIRS, per);
    const size_t cap32 = (size_t)1 << 30;
    buf.ccdVtCap = ccd ? (int)std::max<size_t>(1, std::min(cap32, (size_t)N * vtPer)) : 1;
    buf.ccdEeCap = ccd ? (int)std::max<size_t>(1, std::min(cap32, (size_t)E * eePer)) : 1;
    buf.stCap = (self ? N * KVT : 1) + (ccd ? N * CCD_VT_HITS : 0);
    buf.seCap = (self ? E : 1) + (ccd ? E * CCD_EE_HITS : 0);
    buf.stCnt = (int*)dalloc(sizeof(int) * N, true);
    buf.stSlot = (SCt*)dalloc(sizeof(SCt) * (size_t)(self ? N * KVT : 1), true);
    buf.stList = (SCt*)dalloc(sizeof(SCt) * (size_t)buf.stCap, true);
    buf.seFlag = (int*)dalloc(sizeof(int) * E, true);
    buf.seSlot = (SCt*)dalloc(sizeof(SCt) * (size_t)E, true);
    buf.seList = (SCt*)dalloc(sizeof(SCt) * (size_t)buf.seCap, true);
    buf.ccdVtCnt = (int*)dalloc(sizeof(int) * N, true);
    buf.ccdEeCnt = (int*)dalloc(sizeof(int) * E, true);
    buf.ccdVtCand = (int*)dalloc(sizeof(int) * (size_t)(ccd ? N * KCCD : 1), true);
    buf.ccdEeCand = (int*)dalloc(sizeof(int) * (size_t)(ccd ? E * KCCD : 1), true);
    buf.ccdVtPairs = (int2*)dalloc(sizeof(int2) * (size_t)buf.ccdVtCap, true);
    buf.ccdEePairs = (int2*)dalloc(sizeof(int2) * (size_t)buf.ccdEeCap, true);
    buf.ccdVtHit = (uint8_t*)dalloc((size_t)buf.ccdVtCap, true);
    buf.ccdEeHit = (uint8_t*)dalloc((size_t)buf.ccdEeCap, true);
    buf.ccdVtOff = (int*)dalloc(sizeof(int) * N, true);
    buf.ccdEeOff = (int*)dalloc(sizeof(int) * E, true);
    buf.ccdVtHitCnt = (int*)dalloc(sizeof(int) * N, true);
    buf.ccdEeHitCnt = (int*)dalloc(sizeof(int) * E, true);
    buf.ccdVtPoolOff = (int*)dalloc(sizeof(int) * N, true);
    buf.ccdEePoolOff = (int*)dalloc(sizeof(int) * E, true);
    buf.ccdPoolCap = ccd ? std::max(buf.ccdEeCap, std::max(N, E) * KCCD / 2) : 1;
    buf.ccdPool = (int*)dalloc(sizeof(int) * (size_t)buf.ccdPoolCap, true);
    buf.ccdPoolUsed = counts + 6;
    buf.ccdVtOvf = (int*)dalloc(sizeof(int) * (size_t)(ccd ? N : 1), true);
    buf.ccdEeOvf = (int*)dalloc(sizeof(int) * (size_t)(ccd ? E : 1), true);
    buf.ccdOvfN = (int*)dalloc(sizeof(int) * 2, true);
    if (ccd) ccd_kernel_setup();
    // colouring
    buf.vmin = (unsigned long long*)dalloc(sizeof(unsigned long long) * N, true);
    SC_CUDA(cudaMemset(buf.vmin, 0xff, sizeof(unsigned long long) * N));
    buf.colourCap = buf.ecCap + buf.tcCap + buf.stCap + buf.seCap;
    buf.colour = (int*)dalloc(sizeof(int) * (size_t)buf.colourCap, true);
    buf.order = (int*)dalloc(sizeof(int) * (size_t)buf.colourCap, true);
    buf.colourStart = (int*)dalloc(sizeof(int) * 4 * (MAX_COLOURS + 1), true);
    // scans
    size_t maxScan = std::max<size_t>({(size_t)N, (size_t)E, (size_t)buf.tcCap, (size_t)buf.ecCap});
    buf.scanOff = (int*)dalloc(sizeof(int) * (maxScan + 1), true);
    buf.scanBlock = (int*)dalloc(sizeof(int) * (maxScan / 1024 + 8), true);
    buf.scanBlock2 = (int*)dalloc(sizeof(int) * (maxScan / 1024 + 8), true);
    buf.scanOff2 = (int*)dalloc(sizeof(int) * (maxScan + 1), true);
    buf.broadWalk = broadWalk;
    bufWorldVersion = world.version;
    bufFlags = prm.flags;
    bufCcd = ccd;
    (void)s;
    return true;
}

// ------------------------------------------------------------------ patch
ClothPatch::ClothPatch(CollisionWorld& w) : world(w), model(this)
{
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&evFork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&evJoin, cudaEventDisableTiming);
}

ClothPatch::~ClothPatch()
{
    if (graph) cudaGraphExecDestroy(graph);
    if (graphDef) cudaGraphDestroy(graphDef);
    if (stream) { cudaStreamSynchronize(stream); cudaStreamDestroy(stream); }
    if (side) { cudaStreamSynchronize(side); cudaStreamDestroy(side); }
    if (evFork) cudaEventDestroy(evFork);
    if (evJoin) cudaEventDestroy(evJoin);
}

// ClothModel::AddTriangle: FEM rest data from the uv parameterisation
// (Physics/ClothModel.cpp:54-92)
static FemHost make_triangle(const ClothModel& m, uint32_t i1, uint32_t i2, uint32_t i3)
{
    FemHost t = {};
    t.i1 = i1; t.i2 = i2; t.i3 = i3;
    float d1x = m.uvx[i2] - m.uvx[i1], d1y = m.uvy[i2] - m.uvy[i1];
    float d2x = m.uvx[i3] - m.uvx[i1], d2y = m.uvy[i3] - m.uvy[i1];
    t.du1 = d1x; t.du2 = d2x; t.dv1 = d1y; t.dv2 = d2y;
    t.det = t.du1 * t.dv2 - t.du2 * t.dv1;
    t.invDet = 0.f;
    if (t.det != 0) t.invDet = 1.f / t.det;
    V3 dx1 = m.hpos[i2] - m.hpos[i1], dx2 = m.hpos[i3] - m.hpos[i1];
    V3 wu = t.invDet * (t.dv2 * dx1 - t.dv1 * dx2);
    V3 wv = t.invDet * (-t.du2 * dx1 + t.du1 * dx2);
    t.lu0 = len(wu);
    t.lv0 = len(wv);
    if (t.lu0 != 0) t.su = 1.f / t.lu0;
    if (t.lv0 != 0) t.sv = 1.f / t.lv0;
    t.area = 0.5f * t.det;
    t.lu2 = t.lu0 * t.lu0;
    t.lv2 = t.lv0 * t.lv0;
    return t;
}

// ClothPatch::Init(divX, divY, inc, offset, horizontal, attached)
// (Physics/ClothPatch.cpp:135-246). The vertical layout's random incline is
// not reproduced (horizontal = false lays the grid in the XY plane with z = 0).
bool ClothPatch::init_grid(int divX, int divY, float inc, V3 offset, bool horizontal, bool attached)
{
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    if (divX < 2 || divY < 2) { set_error(SC_ERR_ARG, "grid needs at least 2x2 vertices"); return false; }
    ClothModel& m = model;
    const int N = divX * divY;
    m.N = N;
    m.hpos.assign(N, mk(0, 0, 0)); m.hprev.assign(N, mk(0, 0, 0)); m.hvel.assign(N, mk(0, 0, 0));
    m.invMass.assign(N, 1.f); m.uvx.assign(N, 0.f); m.uvy.assign(N, 0.f);
    m.gridIJ.resize(N);
    for (int j = 0; j < divX; j++)
        for (int i = 0; i < divY; i++) m.gridIJ[j * divY + i] = make_int2(j, i);
    m.tris.clear(); m.bends.clear(); m.links.clear(); m.linkRest.clear(); m.quads.clear();
    mesh = HMesh();
    isQuadMesh = true;
    const bool dihedral = m.prm.dihedral;
    const float stretch = m.prm.stretch, shear = m.prm.shear, bend = m.prm.bend;
    auto addLink = [&](uint32_t a, uint32_t b, float stiff) {
        // ClothModel::AddLink (Physics/ClothModel.inl:12-31): skipped when both
        // ends are pinned or the stiffness is zero; rest length from the positions
        if (m.invMass[a] == 0 && m.invMass[b] == 0) return;
        if (stiff == 0) return;
        m.links.push_back(make_uint2(a, b));
        m.linkRest.push_back(make_float2(len(m.hpos[a] - m.hpos[b]), stiff));
    };
    float x = -0.5f * divX * inc;
    const float startY = x;
    for (int j = 0, base = 0; j < divX; j++, base += divY)
    {
        m.hpos[base] = horizontal ? mk(x, 0, startY) + offset : mk(x, startY, 0) + offset;
        m.hprev[base] = m.hpos[base];
        m.uvx[base] = x; m.uvy[base] = 0;
        if (base >= divY)
        {
            addLink(base - divY, base, stretch);
            addLink(base - divY + 1, base, shear);
            if (base >= 2 * divY && !dihedral) addLink(base - 2 * divY, base, bend);
        }
        for (int i = 1; i < divY; i++)
        {
            const int idx = base + i;
            m.hpos[idx] = horizontal ? mk(x, 0, startY + inc * i) + offset : mk(x, startY + inc * i, 0) + offset;
            m.hprev[idx] = m.hpos[idx];
            m.uvx[idx] = x; m.uvy[idx] = inc * i;
            addLink(idx - 1, idx, stretch);
            if (idx > base + 1 && !dihedral) addLink(idx - 2, idx, bend);
            if (idx >= divY)
            {
                addLink(idx - divY, idx, stretch);
                if (i < divY - 1) addLink(idx - divY + 1, idx, shear);
                if (j > 1 && !dihedral) addLink(idx - 2 * divY, idx, bend);
            }
            if (idx > divY)
            {
                addLink(idx - divY - 1, idx, shear);
                const uint32_t a = idx - divY - 1, b = idx - divY, c = idx, d = idx - 1;
                m.quads.push_back(make_uint4(a, b, c, d));
                uint32_t t[6];
                if ((i & 1) == (j & 1)) { uint32_t u[6] = {a, c, b, a, d, c}; memcpy(t, u, sizeof(t)); }
                else { uint32_t u[6] = {b, d, c, d, b, a}; memcpy(t, u, sizeof(t)); }
                for (int k = 0; k < 2; k++)
                {
                    m.tris.push_back(make_triangle(m, t[3 * k], t[3 * k + 1], t[3 * k + 2]));
                    mesh.idx.push_back(t[3 * k]); mesh.idx.push_back(t[3 * k + 1]); mesh.idx.push_back(t[3 * k + 2]);
                }
            }
        }
        if (attached && (j == 0 || j == divX - 1)) m.invMass[base + divY - 1] = 0.f;
        x += inc;
    }
    mesh.verts = m.hpos;
    mesh.compute_normals();
    mesh.construct_edges();
    mesh.construct_rings(true, true);
    // ClothModel::AddBendConstraint for every interior edge (Physics/ClothModel.cpp:94-126)
    for (const HEdge& e : mesh.edges)
    {
        if (e.t2 < 0) continue;
        auto opp = [&](int t) -> uint32_t {
            const FemHost& tr = m.tris[t];
            if (tr.i1 != e.i1 && tr.i1 != e.i2) return tr.i1;
            if (tr.i2 != e.i1 && tr.i2 != e.i2) return tr.i2;
            return tr.i3;
        };
        m.bends.push_back(make_uint4(e.i1, e.i2, opp(e.t1), opp(e.t2)));
    }
    prevMesh = mesh;
    if (!m.upload_topology(mesh)) return false;
    m.upload_state(stream);
    hostStateDirty = false;
    return true;
}

// A batch: independent clothes stepped as one model. The parts' particles,
// triangles (with their rest data), bends, edges and rings are concatenated with
// index offsets, each part keeps the colliders of its own world, and every
// spatial query is confined to its instance (one tree per instance). Per-part
// colouring is the greedy colouring of the part alone, so a colour of the batch
// is the union of the parts' colours: each instance runs the same projections in
// the same order as it would alone.
bool ClothPatch::init_batch(const std::vector<ClothPatch*>& parts)
{
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    if (parts.empty()) { set_error(SC_ERR_ARG, "empty batch"); return false; }
    ClothModel& m = model;
    const ClothModel& m0 = parts[0]->model;
    for (ClothPatch* q : parts)
    {
        if (!q || q->model.N == 0) { set_error(SC_ERR_ARG, "batch part not initialised"); return false; }
        if (!q->model.instV.empty()) { set_error(SC_ERR_ARG, "a batch cannot contain a batch"); return false; }
        q->sync();
        const HostParams& a = q->model.prm;
        const HostParams& b = m0.prm;
        const bool same = a.unit == b.unit && a.thickness == b.thickness && a.tolerance == b.tolerance && a.shear == b.shear &&
                          a.bend == b.bend && a.stretch == b.stretch && a.poisson == b.poisson && a.friction == b.friction &&
                          a.drag == b.drag && a.iterations == b.iterations && a.flags == b.flags && a.fem == b.fem &&
                          a.dihedral == b.dihedral && a.fixedIterations == b.fixedIterations && a.ccd == b.ccd &&
                          a.bendFreq == b.bendFreq && a.area == b.area && q->numSteps == parts[0]->numSteps;
        if (!same) { set_error(SC_ERR_ARG, "batch parts must share every solver parameter and the substep count"); return false; }
    }
    if (m0.prm.flags & (CF_TRIANGLES | CF_EDGES))
    {
        set_error(SC_ERR_UNSUPPORTED, "batches support vertex, wall and self collisions (not triangle / edge collider contacts)");
        return false;
    }
    m.prm = m0.prm;
    numSteps = parts[0]->numSteps;
    m.N = 0;
    m.hpos.clear(); m.hprev.clear(); m.hvel.clear(); m.invMass.clear(); m.uvx.clear(); m.uvy.clear();
    m.tris.clear(); m.bends.clear(); m.links.clear(); m.linkRest.clear(); m.quads.clear();
    m.instV = {0}; m.instT = {0}; m.instE = {0}; m.instB = {0};
    m.gridIJ.clear();
    bool allGrids = true;
    for (ClothPatch* q : parts) allGrids = allGrids && (int)q->model.gridIJ.size() == q->model.N;
    m.batchColl.clear();
    mesh = HMesh();
    for (size_t k = 0; k < parts.size(); k++)
    {
        const ClothModel& q = parts[k]->model;
        const HMesh& qm = parts[k]->mesh;
        const uint32_t vo = (uint32_t)m.N, to = (uint32_t)m.tris.size(), eo = (uint32_t)mesh.edges.size();
        m.hpos.insert(m.hpos.end(), q.hpos.begin(), q.hpos.end());
        m.hprev.insert(m.hprev.end(), q.hprev.begin(), q.hprev.end());
        m.hvel.insert(m.hvel.end(), q.hvel.begin(), q.hvel.end());
        m.invMass.insert(m.invMass.end(), q.invMass.begin(), q.invMass.end());
        m.uvx.insert(m.uvx.end(), q.uvx.begin(), q.uvx.end());
        m.uvy.insert(m.uvy.end(), q.uvy.begin(), q.uvy.end());
        if (allGrids) m.gridIJ.insert(m.gridIJ.end(), q.gridIJ.begin(), q.gridIJ.end());
        for (FemHost t : q.tris) { t.i1 += vo; t.i2 += vo; t.i3 += vo; m.tris.push_back(t); }
        for (uint4 b : q.bends) m.bends.push_back(make_uint4(b.x + vo, b.y + vo, b.z + vo, b.w + vo));
        for (uint2 l : q.links) m.links.push_back(make_uint2(l.x + vo, l.y + vo));
        m.linkRest.insert(m.linkRest.end(), q.linkRest.begin(), q.linkRest.end());
        for (uint4 d : q.quads) m.quads.push_back(make_uint4(d.x + vo, d.y + vo, d.z + vo, d.w + vo));
        mesh.verts.insert(mesh.verts.end(), qm.verts.begin(), qm.verts.end());
        mesh.normals.insert(mesh.normals.end(), qm.normals.begin(), qm.normals.end());
        mesh.triN.insert(mesh.triN.end(), qm.triN.begin(), qm.triN.end());
        for (uint32_t i : qm.idx) mesh.idx.push_back(i + vo);
        for (uint32_t e : qm.triE) mesh.triE.push_back(e + eo);
        for (HEdge e : qm.edges)
        {
            e.i1 += vo; e.i2 += vo;
            if (e.t1 >= 0) e.t1 += (int)to;
            if (e.t2 >= 0) e.t2 += (int)to;
            mesh.edges.push_back(e);
        }
        for (const auto& r : qm.vtxRing)
        {
            mesh.vtxRing.emplace_back();
            for (int v : r) mesh.vtxRing.back().push_back(v + (int)vo);
        }
        for (const auto& r : qm.edgeRing)
        {
            mesh.edgeRing.emplace_back();
            for (int e : r) mesh.edgeRing.back().push_back(e + (int)eo);
        }
        for (auto& cp : parts[k]->world.list) m.batchColl.push_back({cp, (int)vo, q.N, (int)k});
        m.N += q.N;
        m.instV.push_back(m.N);
        m.instT.push_back((int)m.tris.size());
        m.instE.push_back((int)mesh.edges.size());
        m.instB.push_back((int)m.bends.size());
    }
    isQuadMesh = true;
    prevMesh = mesh;
    m.tuned = false;
    m.touch();
    if (!m.upload_topology(mesh)) return false;
    m.bufWorldVersion = ~0ull;
    m.upload_state(stream);
    hostStateDirty = false;
    return true;
}

// ClothPatch::Init(mesh, offset, attached) (Physics/ClothPatch.cpp:42-133): the
// cloth from a triangle mesh. Vertices at exactly the same place become one
// particle (the reference's O(V^2) merge, kept); a particle is pinned when
// `attached` and its vertex colour's red channel is non-zero; triangles take
// their rest shape from the per-corner uvs when given (else the particles' uvs);
// edges come from the first n-1 half-edges of the index buffer, sorted, as the
// reference builds them (so the last triangle's closing edge is missing, as
// there); every unique edge becomes a stretch link, an edge and a bend.
bool ClothPatch::init_mesh(const std::vector<V3>& verts, const std::vector<uint32_t>& idx, const float* uvs,
                           const float* colors, V3 offset, bool attached)
{
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    if (verts.empty() || idx.size() < 3 || idx.size() % 3) { set_error(SC_ERR_ARG, "mesh needs vertices and triangles"); return false; }
    for (uint32_t i : idx) if (i >= verts.size()) { set_error(SC_ERR_ARG, "mesh index out of range"); return false; }
    ClothModel& m = model;
    const size_t nv = verts.size();
    std::vector<int> map(nv, -1);
    m.N = 0;
    m.hpos.clear(); m.hprev.clear(); m.hvel.clear(); m.invMass.clear(); m.uvx.clear(); m.uvy.clear();
    m.tris.clear(); m.bends.clear(); m.links.clear(); m.linkRest.clear(); m.quads.clear();
    m.instV.clear(); m.instT.clear(); m.instE.clear(); m.instB.clear(); m.batchColl.clear();
    m.gridIJ.clear();
    for (size_t i = 0; i < nv; i++)
    {
        if (map[i] >= 0) continue;
        for (size_t j = i + 1; j < nv; j++)
        {
            const V3 d = verts[i] - verts[j];
            if (dot(d, d) == 0) map[j] = m.N;
        }
        map[i] = m.N;
        m.hpos.push_back(verts[i] + offset);
        m.hprev.push_back(mk(0, 0, 0));
        m.hvel.push_back(mk(0, 0, 0));
        m.invMass.push_back((attached && colors && colors[3 * i] != 0) ? 0.f : 1.f);
        m.uvx.push_back(uvs ? uvs[2 * i] : 0.f);
        m.uvy.push_back(uvs ? uvs[2 * i + 1] : 0.f);
        m.N++;
    }
    // ClothModel::AddTriangle with explicit uvs (Physics/ClothModel.cpp:54-92)
    auto addTri = [&](uint32_t a, uint32_t b, uint32_t c, uint32_t ua, uint32_t ub, uint32_t uc) {
        if (uvs)
        {
            // the particle uvs stand in for the corners' own: swap them in for make_triangle
            const float sa[3] = {m.uvx[a], m.uvx[b], m.uvx[c]}, sb[3] = {m.uvy[a], m.uvy[b], m.uvy[c]};
            m.uvx[a] = uvs[2 * ua]; m.uvy[a] = uvs[2 * ua + 1];
            m.uvx[b] = uvs[2 * ub]; m.uvy[b] = uvs[2 * ub + 1];
            m.uvx[c] = uvs[2 * uc]; m.uvy[c] = uvs[2 * uc + 1];
            m.tris.push_back(make_triangle(m, a, b, c));
            m.uvx[c] = sa[2]; m.uvy[c] = sb[2];
            m.uvx[b] = sa[1]; m.uvy[b] = sb[1];
            m.uvx[a] = sa[0]; m.uvy[a] = sb[0];
        }
        else m.tris.push_back(make_triangle(m, a, b, c));
    };
    const size_t n = idx.size();
    struct HE { uint32_t i1, i2; int t1, t2; };
    std::vector<HE> dup(n - 1);
    for (size_t i = 0; i + 1 < n; i++)
    {
        uint32_t i1 = map[idx[i]], i2 = map[idx[i + 1]];
        if ((i + 1) % 3 == 0)
        {
            i2 = map[idx[i - 2]];
            addTri(i2, map[idx[i - 1]], i1, idx[i - 2], idx[i - 1], idx[i]);
        }
        if (i1 > i2) std::swap(i1, i2);
        dup[i] = {i1, i2, (int)(i / 3), -1};
    }
    addTri(map[idx[n - 3]], map[idx[n - 2]], map[idx[n - 1]], idx[n - 3], idx[n - 2], idx[n - 1]);
    std::sort(dup.begin(), dup.end(), [](const HE& a, const HE& b) { return a.i1 < b.i1 || (a.i1 == b.i1 && a.i2 < b.i2); });
    const float stretch = m.prm.stretch;
    auto addLink = [&](uint32_t a, uint32_t b) {
        if (m.invMass[a] == 0 && m.invMass[b] == 0) return;
        if (stretch == 0) return;
        m.links.push_back(make_uint2(a, b));
        m.linkRest.push_back(make_float2(len(m.hpos[a] - m.hpos[b]), stretch));
    };
    std::vector<HE> edges;
    addLink(dup[0].i1, dup[0].i2);
    HE cur = dup[0];
    for (size_t i = 1; i < dup.size(); i++)
    {
        if (dup[i].i1 == dup[i - 1].i1 && dup[i].i2 == dup[i - 1].i2) { cur.t2 = dup[i].t1; continue; }
        addLink(dup[i].i1, dup[i].i2);
        edges.push_back(cur);
        cur = dup[i];
    }
    edges.push_back(cur);
    // the collision / render mesh over the particles, with the reference's edge list
    mesh = HMesh();
    mesh.verts = m.hpos;
    for (const FemHost& t : m.tris) { mesh.idx.push_back(t.i1); mesh.idx.push_back(t.i2); mesh.idx.push_back(t.i3); }
    mesh.compute_normals();
    std::vector<int> slot(3 * m.tris.size(), -1);
    for (size_t e = 0; e < edges.size(); e++)
    {
        HEdge h;
        h.i1 = edges[e].i1; h.i2 = edges[e].i2; h.t1 = edges[e].t1; h.t2 = edges[e].t2;
        h.n = h.t2 >= 0 ? normalized(mesh.triN[h.t1] + mesh.triN[h.t2]) : mesh.triN[h.t1];
        h.origIdx = (int)e;
        mesh.edges.push_back(h);
        // triangle -> edge ids: the triangle side with these end points
        for (int t : {h.t1, h.t2})
        {
            if (t < 0) continue;
            for (int k = 0; k < 3; k++)
            {
                const uint32_t a = mesh.idx[3 * t + k], b = mesh.idx[3 * t + (k + 1) % 3];
                if ((a == h.i1 && b == h.i2) || (a == h.i2 && b == h.i1)) slot[3 * t + k] = (int)e;
            }
        }
    }
    mesh.triE.resize(slot.size());
    for (size_t k = 0; k < slot.size(); k++) mesh.triE[k] = slot[k] < 0 ? 0u : (uint32_t)slot[k];
    mesh.construct_rings(true, true);
    // ClothModel::AddBendConstraint for every edge with two triangles (Physics/ClothModel.cpp:94-126)
    for (const HEdge& e : mesh.edges)
    {
        if (e.t2 < 0) continue;
        auto opp = [&](int t) -> uint32_t {
            const FemHost& tr = m.tris[t];
            if (tr.i1 != e.i1 && tr.i1 != e.i2) return tr.i1;
            if (tr.i2 != e.i1 && tr.i2 != e.i2) return tr.i2;
            return tr.i3;
        };
        m.bends.push_back(make_uint4(e.i1, e.i2, opp(e.t1), opp(e.t2)));
    }
    meshMap = map;
    isQuadMesh = false;
    for (int i = 0; i < m.N; i++) m.hprev[i] = m.hpos[i];
    prevMesh = mesh;
    m.tuned = false;
    m.touch();
    if (!m.upload_topology(mesh)) return false;
    m.bufWorldVersion = ~0ull;
    m.upload_state(stream);
    hostStateDirty = false;
    return true;
}

void ClothPatch::sync()
{
    cudaStreamSynchronize(stream);
    if (hostStateDirty)
    {
        model.download_state(stream);
        hostStateDirty = false;
    }
}

// One substep (ClothModelPBD::Step) recorded into the capture stream.
void ClothPatch::record_substep(float h)
{
    ClothModel& m = model;
    const SolverParams P = m.solver_params(h);
    const DevCloth& c = m.dc;
    Buffers& b = m.buf;
    cudaStream_t s = stream;
    launch_predict(s, c, P);
    const bool self = (m.prm.flags & CF_SELF) != 0, ccd = m.prm.ccd;
    // ClothModel::DetectCollisions (Physics/ClothCollision.cpp:17-48)
    if (ccd)
    {
        // the vertex contacts only read the predicted positions: they run on the
        // side stream ahead of its continuous-collision branch, which the main
        // stream joins before anything reads them
        cudaEventRecord(evFork, s);
        cudaStreamWaitEvent(side, evFork, 0);
        timing_mark(SEC_COLLIDERS, false, side);
        launch_vertex_colliders(side, c, P, b, m.vcollHost.data());
        timing_mark(SEC_COLLIDERS, true, side);
        launch_tri_edge_colliders(s, c, P, b, m.vcollHost.data(), (int)m.vcollHost.size(), m.prm.flags);
    }
    else
    {
        timing_mark(SEC_COLLIDERS, false, s);
        launch_vertex_colliders(s, c, P, b, m.vcollHost.data());
        launch_tri_edge_colliders(s, c, P, b, m.vcollHost.data(), (int)m.vcollHost.size(), m.prm.flags);
        timing_mark(SEC_COLLIDERS, true, s);
    }
    if (self)
    {
        launch_bvh_refit(s, m.triBvh, c, 0, 0.f);
        launch_bvh_refit(s, m.edgeBvh, c, 1, 0.f);
        launch_self_proximity(s, c, P, b, m.triBvh, m.edgeBvh);
    }
    if (ccd)
    {
        cudaEvent_t marks[4] = {nullptr, nullptr, nullptr, nullptr};
        if (timingFrames)
        {
            const size_t k = (size_t)recordingSubstep * NSEC * 2;
            if (k + 2 * NSEC <= timingCapture.size())
            {
                marks[0] = timingCapture[k + 2 * SEC_BROAD_EE]; marks[1] = timingCapture[k + 2 * SEC_BROAD_EE + 1];
                marks[2] = timingCapture[k + 2 * SEC_BROAD_VT]; marks[3] = timingCapture[k + 2 * SEC_BROAD_VT + 1];
            }
        }
        launch_ccd(s, side, evFork, evJoin, c, P, b, m.sweptTriBvh, m.sweptEdgeBvh, marks);
    }
    if (self || ccd) launch_compact_self(s, side, evFork, evJoin, c, P, b, self, ccd);
    else cudaMemsetAsync(b.stCount, 0, 2 * sizeof(int), s);
    launch_colour_contacts(s, c, b);
    // learned warm start (no reference counterpart): record the features and the
    // predicted positions, and / or move the particles by the network's correction
    const size_t sub = (size_t)recordingSubstep;
    const bool learn = (m.warmStart && m.mlpPrm) || m.sampleFeat;
    if (learn) launch_mlp_features(s, c, b, m.sampleFeat ? m.sampleFeat + sub * m.N * MLP_IN : nullptr);
    if (m.warmStart && m.mlpPrm) launch_mlp_warm(s, c, b, m.mlpPrm, m.mlpPrm + MLP_NPARAM);
    // ClothModelPBD::SolveGS (Physics/ClothPBD.cpp:324-369)
    launch_reset_gs(s, c);
    timing_mark(SEC_GS, false, s);
    record_solve(s, P, m.choice);
    timing_mark(SEC_GS, true, s);
    if (learn) launch_mlp_targets(s, c, m.sampleTarget ? m.sampleTarget + sub * m.N * MLP_OUT : nullptr);
    recordingSubstep++;
}


// One substep's Gauss-Seidel loop and velocity update, by the chosen solver:
// the cluster-resident kernel, the grid-resident cooperative kernel (a tuned
// variant), or one kernel per colour. The three are the same algorithm in the
// same order (bit-identical results).
bool ClothPatch::record_solve(cudaStream_t s, const SolverParams& P, const SolverChoice& ch)
{
    ClothModel& m = model;
    const DevCloth& c = m.dc;
    Buffers& b = m.buf;
    const SolverOps& ops = solver_ops(m.prm.fastMath);
    if (m.prm.solverType != 1)
    {
        // ClothModelPBD::Step with SOLVER_JACOBI or another non-Gauss-Seidel type
        // (Physics/ClothPBD.cpp:293-298): links only, fixed iterations; always the
        // IEEE kernels
        if (m.prm.solverType == 0) launch_solve_jacobi(s, c, P, m.linkSolve);
        else
        {
            std::vector<float> beta(std::max(1, P.iterations));
            for (int k = 0; k < P.iterations; k++)
            {
                const float t = (float)k / (float)(P.iterations - 1);
                beta[k] = std::pow(t, 0.6f);
            }
            launch_solve_cr(s, c, P, m.linkSolve, beta.data());
        }
        launch_iteration_total(s, c);
        launch_velocity(s, c, P);
        return true;
    }
    // the reference's loop tests its exit conditions after the body, so it always
    // runs at least one iteration (Physics/ClothPBD.cpp:335-362)
    const int iterations = m.prm.iterations > 1 ? m.prm.iterations : 1;
    const bool planFits = m.triColourStart.size() <= 65 && m.bendColourStart.size() <= 65 && m.linkColourStart.size() <= 65;
    GsPlan plan = {};
    plan.iterations = iterations;
    plan.nFemCol = (int)m.triColourStart.size() - 1;
    plan.nBendCol = (int)m.bendColourStart.size() - 1;
    if (planFits)
    {
        for (size_t k = 0; k < m.triColourStart.size(); k++) plan.femStart[k] = m.triColourStart[k];
        for (size_t k = 0; k < m.bendColourStart.size(); k++) plan.bendStart[k] = m.bendColourStart[k];
        plan.nLinkCol = (int)m.linkColourStart.size() - 1;
        for (size_t k = 0; k < m.linkColourStart.size(); k++) plan.linkStart[k] = m.linkColourStart[k];
    }
    if (ch.kind == SOLVE_BAND && m.band_active() &&
        ops.band(s, c, P, b, plan, m.bandPlan.view, m.bandPlan.clusterSize, m.band_smem(), ch.variant))
        return true;                                                 // includes the velocity update
    int shift = 0;
    size_t smem = 0;
    const int cluster = (ch.kind == SOLVE_CLUSTER && planFits) ? ops.cluster_size(m.N, shift, smem) : 0;
    if (cluster > 0)
    {
        plan.shift = shift;
        // records each CTA handles: per colour a contiguous chunk of ceil(count / cluster)
        auto perCta = [&](const std::vector<int>& start) {
            int most = 0;
            for (int r = 0; r < cluster; r++)
            {
                int sum = 0;
                for (size_t k = 0; k + 1 < start.size(); k++)
                {
                    const int cnt = start[k + 1] - start[k], chunk = (cnt + cluster - 1) / cluster;
                    sum += std::max(0, std::min(chunk, cnt - r * chunk));
                }
                most = std::max(most, sum);
            }
            return most;
        };
        plan.femStage = perCta(m.triColourStart);
        plan.bendStage = perCta(m.bendColourStart);
        const size_t staged = smem + (size_t)plan.femStage * 3 * sizeof(float4) + (size_t)plan.bendStage * sizeof(uint4);
        if (m.prm.stageRecords && staged <= (size_t)GS_SMEM_MAX)
        {
            plan.stage = 1;
            smem = staged;
        }
        ops.cluster(s, c, P, b, plan, cluster, smem, ch.variant);   // includes the velocity update
        return true;
    }
    if (ch.kind == SOLVE_GRID && planFits && ops.grid(s, c, P, b, plan, ch.variant, ch.blocksPerSm))
        return true;
    if (P.resTol > 0.f) launch_residual_exit(s, c, P, -1);
    for (int k = 0; k < iterations; k++)
    {
        if (m.prm.fem)
            for (size_t col = 0; col + 1 < m.triColourStart.size(); col++)
                ops.fem(s, c, P, m.triColourStart[col], m.triColourStart[col + 1] - m.triColourStart[col]);
        else
        {
            ops.reset_link_error(s, c);
            for (size_t col = 0; col + 1 < m.linkColourStart.size(); col++)
                ops.links(s, c, P, m.linkColourStart[col], m.linkColourStart[col + 1] - m.linkColourStart[col]);
        }
        if (m.prm.dihedral && k % m.prm.bendFreq == 0)
            for (size_t col = 0; col + 1 < m.bendColourStart.size(); col++)
                ops.bends(s, c, P, m.bendColourStart[col], m.bendColourStart[col + 1] - m.bendColourStart[col], col == 0);
        ops.vertex_contacts(s, c, P, b);
        ops.multi_contacts(s, c, P, b, k);
        if (P.resTol > 0.f) launch_residual_exit(s, c, P, k);
    }
    launch_iteration_total(s, c);
    launch_velocity(s, c, P);
    return true;
}

// Autotuner: time one substep's solve (reset + Gauss-Seidel + velocity) for
// every candidate — the cluster kernel when the cloth fits, each grid variant
// (threads per CTA x constraints per thread) at 1, 2 and the most resident CTAs
// per SM, and the per-colour kernels — each captured as a graph and replayed
// with CUDA events; positions and velocities are restored after each. The
// fastest is kept per problem shape for the process.
static std::mutex g_tuneMutex;
static std::vector<std::pair<std::vector<int>, SolverChoice>> g_tuneCache;

bool ClothPatch::autotune(float h)
{
    ClothModel& m = model;
    if (m.prm.solverType != 1) { m.tuned = true; return true; }   // the Jacobi / CR solves have no variants
    const SolverParams P = m.solver_params(h);
    std::vector<int> key = {m.N, m.dc.T, m.dc.B, m.prm.iterations, m.prm.dihedral, m.prm.fem, m.prm.fixedIterations,
                            (int)m.buf.numVColl, m.prm.bendFreq, (int)m.prm.stageRecords, m.solverMode,
                            (int)m.prm.ccd, m.broadMode, (int)m.prm.fastMath, (int)m.band_active(),
                            m.bandPlan.clusterSize, m.bandPlan.halo};
    key.insert(key.end(), m.triColourStart.begin(), m.triColourStart.end());
    key.insert(key.end(), m.bendColourStart.begin(), m.bendColourStart.end());
    {
        std::lock_guard<std::mutex> lk(g_tuneMutex);
        for (auto& kv : g_tuneCache)
            if (kv.first == key)
            {
                m.choice = kv.second;
                m.broadWalk = m.broadMode >= 0 ? m.broadMode : kv.second.broad;
                m.buf.broadWalk = m.broadWalk;
                m.tuned = true;
                return true;
            }
    }
    std::vector<SolverChoice> cand;
    int shift = 0; size_t smem = 0;
    const bool fits = m.triColourStart.size() <= 65 && m.bendColourStart.size() <= 65 && m.linkColourStart.size() <= 65;
    const SolverOps& ops = solver_ops(m.prm.fastMath);
    // the band solver (mode 4) sweeps in its own order: only its thread counts are timed
    const bool band = m.band_active();
    if (band)
        for (int v = 0; v < gs_band_variants(); v++) cand.push_back({SOLVE_BAND, v, 0, 0.f});
    if (!band && fits && (m.solverMode == SOLVE_AUTO || m.solverMode == SOLVE_CLUSTER) && ops.cluster_size(m.N, shift, smem) > 0)
        for (int v = 0; v < gs_cluster_variants(); v++) cand.push_back({SOLVE_CLUSTER, v, 0, 0.f});
    if (!band && fits && (m.solverMode == SOLVE_AUTO || m.solverMode == SOLVE_GRID))
        for (int v = 0; v < gs_grid_variants(); v++)
        {
            const int mb = ops.grid_max_blocks_per_sm(v);
            for (int bps : {1, 2, mb})
                if (bps >= 1 && bps <= mb)
                {
                    bool dup = false;
                    for (auto& c : cand) dup |= c.kind == SOLVE_GRID && c.variant == v && c.blocksPerSm == bps;
                    if (!dup) cand.push_back({SOLVE_GRID, v, bps, 0.f});
                }
        }
    if (!band && m.solverMode == SOLVE_AUTO) cand.push_back({SOLVE_KERNELS, 0, 0, 0.f});
    if (cand.empty()) cand.push_back({SOLVE_KERNELS, 0, 0, 0.f});
    const size_t bytes = sizeof(float4) * (size_t)m.N;
    float4* backup = nullptr;
    SC_CUDA(cudaMalloc(&backup, 2 * bytes));
    SC_CUDA(cudaMemcpyAsync(backup, m.dc.pos, bytes, cudaMemcpyDeviceToDevice, stream));
    SC_CUDA(cudaMemcpyAsync(backup + m.N, m.dc.vel, bytes, cudaMemcpyDeviceToDevice, stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    SolverChoice best = cand.back();
    best.ms = 1e30f;
    for (SolverChoice& ch : cand)
    {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) continue;
        launch_reset_gs(stream, m.dc);
        record_solve(stream, P, ch);
        if (cudaStreamEndCapture(stream, &g) != cudaSuccess || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
        {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            continue;
        }
        cudaGraphDestroy(g);
        const int reps = 3;
        cudaGraphLaunch(ge, stream);                  // warm-up
        cudaEventRecord(e0, stream);
        for (int r = 0; r < reps; r++) cudaGraphLaunch(ge, stream);
        cudaEventRecord(e1, stream);
        cudaError_t err = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (err == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
        {
            ch.ms = ms / reps;
            if (ch.ms < best.ms) best = ch;
        }
        cudaGetLastError();
        cudaGraphExecDestroy(ge);
        cudaMemcpyAsync(m.dc.pos, backup, bytes, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(m.dc.vel, backup + m.N, bytes, cudaMemcpyDeviceToDevice, stream);
    }
    cudaStreamSynchronize(stream);
    cudaFree(backup);
    m.tuneLog = cand;
    m.choice = best;
    // continuous broad phase: the first-pass walks (BROAD_*; same pair sets), timed
    // on this cloth's current state (the detection changes no particle)
    if (m.prm.ccd && m.buf.ccdVtCnt)
    {
        for (int mode = 0; mode < BROAD_WALKS; mode++)
        {
            m.buf.broadWalk = mode;
            m.broadMs[mode] = 1e30f;
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ge = nullptr;
            if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) continue;
            launch_ccd(stream, side, evFork, evJoin, m.dc, P, m.buf, m.sweptTriBvh, m.sweptEdgeBvh);
            if (cudaStreamEndCapture(stream, &g) != cudaSuccess || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
            {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                continue;
            }
            cudaGraphDestroy(g);
            cudaGraphLaunch(ge, stream);
            cudaEventRecord(e0, stream);
            for (int r = 0; r < 3; r++) cudaGraphLaunch(ge, stream);
            cudaEventRecord(e1, stream);
            float ms = 0.f;
            if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
                m.broadMs[mode] = ms / 3;
            cudaGetLastError();
            cudaGraphExecDestroy(ge);
        }
        m.broadWalk = 0;
        for (int mode = 1; mode < BROAD_WALKS; mode++)
            if (m.broadMs[mode] < m.broadMs[m.broadWalk]) m.broadWalk = mode;
    }
    if (m.broadMode >= 0) m.broadWalk = m.broadMode;
    m.buf.broadWalk = m.broadWalk;
    best.broad = m.broadWalk;
    m.choice = best;
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    m.tuned = true;
    std::lock_guard<std::mutex> lk(g_tuneMutex);
    g_tuneCache.push_back({key, best});
    return true;
}

void ClothPatch::timing_mark(int section, bool end, cudaStream_t s)
{
    if (!timingFrames) return;
    const size_t k = ((size_t)recordingSubstep * NSEC + section) * 2 + (end ? 1 : 0);
    // external: captured as an event-record node (a plain record only orders streams)
    if (k < timingCapture.size()) cudaEventRecordWithFlags(timingCapture[k], s, cudaEventRecordExternal);
}

bool ClothPatch::set_timing(int frames)
{
    sync();
    for (cudaEvent_t e : timingCapture) cudaEventDestroy(e);
    for (cudaEvent_t e : timingPool) cudaEventDestroy(e);
    timingCapture.clear(); timingPool.clear(); timingNodes.clear();
    timingFrames = std::max(0, frames);
    timingUsed = 0;
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }   // re-capture with (or without) the marks
    if (!timingFrames) return true;
    const size_t per = (size_t)std::max(1, numSteps) * NSEC * 2;
    timingCapture.resize(per);
    timingPool.resize(per * timingFrames);
    for (auto& e : timingCapture) SC_CUDA(cudaEventCreate(&e));
    for (auto& e : timingPool) SC_CUDA(cudaEventCreate(&e));
    return true;
}

int ClothPatch::read_timing(float* ms, int* count)
{
    sync();
    const size_t per = timingCapture.size();
    for (int sct = 0; sct < NSEC; sct++) { if (ms) ms[sct] = 0.f; if (count) count[sct] = 0; }
    for (int f = 0; f < timingUsed; f++)
        for (size_t k = 0; k + 1 < per; k += 2)
        {
            const size_t i = (size_t)f * per + k;
            float t = 0.f;
            if (timingNodes[k] && timingNodes[k + 1] && cudaEventElapsedTime(&t, timingPool[i], timingPool[i + 1]) == cudaSuccess)
            {
                const int sct = (int)((k / 2) % NSEC);
                if (ms) ms[sct] += t;
                if (count) count[sct]++;
            }
        }
    cudaGetLastError();
    const int used = timingUsed;
    timingUsed = 0;
    return used;
}

// ClothPatch::Step (Physics/ClothPatch.cpp:323-335): numSteps substeps of dt/n,
// launched as one CUDA graph (captured on first use and whenever a parameter,
// the collision world or dt changes). Asynchronous: readers synchronise.
bool ClothPatch::step(float dt)
{
    ClothModel& m = model;
    if (m.N == 0) { set_error(SC_ERR_STATE, "cloth not initialised"); return false; }
    if (!m.ensure_buffers(world, stream)) return false;
    const int n = numSteps;
    const float h = dt / n;
    if (directLaunch)
    {
        // the same substeps, launched one kernel at a time (no graph, no section timing)
        if (m.solverMode == SOLVE_KERNELS) m.choice = {SOLVE_KERNELS, 0, 0, 0.f};
        else if (!m.tuned || m.tunedVersion != m.paramVersion)
        {
            if (!autotune(h)) return false;
            m.tunedVersion = m.paramVersion;
        }
        const int frames = timingFrames;
        timingFrames = 0;
        recordingSubstep = 0;
        for (int i = 0; i < n; i++) record_substep(h);
        timingFrames = frames;
        SC_CUDA(cudaGetLastError());
        hostStateDirty = true;
        return true;
    }
    if (!graph || graphDt != dt || graphSteps != n || graphParamVersion != m.paramVersion || graphWorldVersion != world.version)
    {
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        if (m.solverMode == SOLVE_KERNELS) m.choice = {SOLVE_KERNELS, 0, 0, 0.f};
        else if (!m.tuned || m.tunedVersion != m.paramVersion)
        {
            if (!autotune(h)) return false;
            m.tunedVersion = m.paramVersion;
        }
        cudaGraph_t g;
        if (timingFrames && timingCapture.size() != (size_t)n * NSEC * 2) set_timing(timingFrames);
        recordingSubstep = 0;
        SC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < n; i++) record_substep(h);
        SC_CUDA(cudaStreamEndCapture(stream, &g));
        size_t numNodes = 0;
        cudaGraphGetNodes(g, nullptr, &numNodes);
        std::vector<cudaGraphNode_t> nodes(numNodes);
        if (numNodes) cudaGraphGetNodes(g, nodes.data(), &numNodes);
        graphKernelCount = 0;
        timingNodes.assign(timingCapture.size(), nullptr);
        for (size_t k = 0; k < numNodes; k++)
        {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(nodes[k], &t) != cudaSuccess) continue;
            if (t == cudaGraphNodeTypeKernel) graphKernelCount++;
            if (t == cudaGraphNodeTypeEventRecord && !timingCapture.empty())
            {
                cudaEvent_t ev;
                if (cudaGraphEventRecordNodeGetEvent(nodes[k], &ev) != cudaSuccess) continue;
                for (size_t j = 0; j < timingCapture.size(); j++)
                    if (timingCapture[j] == ev) { timingNodes[j] = nodes[k]; break; }
            }
        }
        cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
        // the definition outlives the instantiation: the timing nodes' handles
        // (used to retarget their events per replay) belong to it
        if (graphDef) cudaGraphDestroy(graphDef);
        graphDef = g;
        if (e != cudaSuccess) { set_error(SC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); graph = nullptr; return false; }
        graphDt = dt; graphSteps = n; graphParamVersion = m.paramVersion; graphWorldVersion = world.version;
    }
    if (timingFrames && timingUsed < timingFrames)
    {
        const size_t per = timingCapture.size();
        for (size_t k = 0; k < per; k++)
            if (timingNodes[k]) SC_CUDA(cudaGraphExecEventRecordNodeSetEvent(graph, timingNodes[k], timingPool[(size_t)timingUsed * per + k]));
        timingUsed++;
    }
    SC_CUDA(cudaGraphLaunch(graph, stream));
    hostStateDirty = true;
    return true;
}

// ClothPatch::UpdateMesh (Physics/ClothPatch.cpp:266-273): render mesh from the
// current positions, both meshes' normals recomputed; the collision mesh's
// normals feed the next substeps' Voronoi tests.
void ClothPatch::update_mesh()
{
    ClothModel& m = model;
    if (m.N == 0) return;
    launch_normals(stream, m.dc, false, m.dc.pos);
    launch_normals(stream, m.dc, true, m.dc.prev);
    sync();
    std::vector<float4> n(m.N);
    cudaMemcpy(n.data(), m.dc.meshN, sizeof(float4) * m.N, cudaMemcpyDeviceToHost);
    mesh.verts = m.hpos;
    mesh.normals.resize(m.N);
    for (int i = 0; i < m.N; i++) mesh.normals[i] = mk(n[i]);
}

} // namespace sc
