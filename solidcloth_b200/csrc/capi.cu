// capi.cu — the extern "C" sc* entry points (include/solidcloth_b200.h), each a
// thin shim over the host objects in cloth.h, mirroring Demo/ClothAPI.cpp.
#include "cloth.h"
#include "../../include/solidcloth_b200.h"
#include <cstring>
#include <cstdio>
#include <string>
#include <algorithm>
#include <cmath>

using namespace sc;

namespace {

ClothPatch* P(scClothPatch p) { return (ClothPatch*)p.ptr; }
ClothModel* M(scModel m) { return (ClothModel*)m.ptr; }
CollisionWorld* W(scCollisionWorld w) { return (CollisionWorld*)w.ptr; }
V3 v3(scVector3 a) { return mk(a.x, a.y, a.z); }
scVector3 sv(V3 a) { scVector3 r = {a.x, a.y, a.z}; return r; }

bool check_model(ClothModel* m, int i = -1)
{
    if (!m) { set_error(SC_ERR_ARG, "null model handle"); return false; }
    if (i >= 0 && i >= m->N) { set_error(SC_ERR_ARG, "particle index out of range"); return false; }
    return true;
}

void host_sync(ClothModel* m) { if (m && m->owner) m->owner->sync(); }

template <typename T>
std::vector<T> dl(const T* d, size_t n)
{
    std::vector<T> h(n);
    if (n) cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost);
    return h;
}

int dcount(const int* d)
{
    int v = 0;
    if (d) cudaMemcpy(&v, d, sizeof(int), cudaMemcpyDeviceToHost);
    return v;
}

} // namespace

extern "C" {

// ------------------------------------------------------------------ world
scCollisionWorld scCreateCollisionWorld(void) { scCollisionWorld w; w.ptr = new CollisionWorld(); return w; }
void scFreeCollisionWorld(scCollisionWorld w) { delete W(w); }
void scClearCollidables(scCollisionWorld w) { if (W(w)) { W(w)->list.clear(); W(w)->version++; } }
int scGetNumCollidables(scCollisionWorld w) { return W(w) ? (int)W(w)->list.size() : 0; }
void scAddCollidable(scCollisionWorld w, scHandle c)
{
    if (!W(w) || !c) { set_error(SC_ERR_ARG, "null handle"); return; }
    W(w)->list.push_back(std::shared_ptr<Collidable>((Collidable*)c));
    W(w)->version++;
}
scHandle scGetCollidable(scCollisionWorld w, int i)
{
    if (!W(w) || i < 0 || i >= (int)W(w)->list.size()) { set_error(SC_ERR_ARG, "collidable index out of range"); return nullptr; }
    return W(w)->list[i].get();
}

// -------------------------------------------------------------- collidables
scHandle scCreateWalls(scAabb3 box)
{
    WallsC* w = new WallsC();
    w->type = CT_WALLS;
    w->box.lo = v3(box.min); w->box.hi = v3(box.max);
    return w;
}

scHandle scCreateSphere(scVector3 center, float radius)
{
    SphereC* s = new SphereC();
    s->type = CT_SPHERE;
    s->center = v3(center);
    s->radius = radius;
    return s;
}

scHandle scCreateCapsule(scVector3 c, float rad, float halfHeight, scQuaternion q)
{
    CapsuleC* k = new CapsuleC();
    k->type = CT_CAPSULE;
    k->center = v3(c); k->r = rad; k->hh = halfHeight;
    k->rot[0] = q.s; k->rot[1] = q.v.x; k->rot[2] = q.v.y; k->rot[3] = q.v.z;
    return k;
}

// SDF::Create + CacheData + ComputeGradient (Geometry/SDF.cpp:10-40,210-256)
scHandle scCreateSDFGrid(int nx, int ny, int nz, scAabb3 box, const float* values)
{
    if (nx < 1 || ny < 1 || nz < 1 || !values) { set_error(SC_ERR_ARG, "bad SDF grid"); return nullptr; }
    SDFC* s = new SDFC();
    s->type = CT_SDF;
    s->nc[0] = nx; s->nc[1] = ny; s->nc[2] = nz;
    s->box.lo = v3(box.min); s->box.hi = v3(box.max);
    V3 ext = s->box.hi - s->box.lo;
    V3 inv = mk(1.f / nx, 1.f / ny, 1.f / nz);
    s->steps = mk(ext.x * inv.x, ext.y * inv.y, ext.z * inv.z);
    size_t n = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    s->values.assign(values, values + n);
    s->compute_gradient();
    return s;
}

static SDFC* new_sdf(int nx, int ny, int nz, scAabb3 box)
{
    SDFC* s = new SDFC();
    s->type = CT_SDF;
    s->nc[0] = nx; s->nc[1] = ny; s->nc[2] = nz;
    s->box.lo = v3(box.min); s->box.hi = v3(box.max);
    V3 ext = s->box.hi - s->box.lo;
    V3 inv = mk(1.f / nx, 1.f / ny, 1.f / nz);
    s->steps = mk(ext.x * inv.x, ext.y * inv.y, ext.z * inv.z);
    return s;
}

scHandle scCreateSDFFromMesh(const float* vertices, int nv, const unsigned* indices, int ni, int nx, int ny, int nz,
                             scAabb3 box)
{
    if (!vertices || !indices || nv <= 0 || ni <= 0 || ni % 3 || nx < 1 || ny < 1 || nz < 1)
    {
        set_error(SC_ERR_ARG, "bad mesh or SDF grid");
        return nullptr;
    }
    // the mesh and its triangle tree as SDF::CreateFromMesh builds them
    // (ComputeMeshTree(mesh, ATF_TRIANGLES, 10, 0.1f), Geometry/SDF.cpp:60-61)
    MeshC m;
    m.mesh.verts.resize(nv);
    for (int i = 0; i < nv; i++) m.mesh.verts[i] = mk(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    m.mesh.idx.assign(indices, indices + ni);
    m.mesh.compute_normals();
    m.mesh.construct_edges();
    m.build_tree(0.1f, 10, 1);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!m.upload(dev)) return nullptr;
    SDFC* s = new_sdf(nx, ny, nz, box);
    const size_t n = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    float* d = nullptr;
    int* st = nullptr;
    if (cudaMalloc(&d, sizeof(float) * n) != cudaSuccess || cudaMalloc(&st, sizeof(int)) != cudaSuccess)
    {
        if (d) cudaFree(d);
        delete s;
        set_error(SC_ERR_CUDA, "cudaMalloc failed");
        return nullptr;
    }
    cudaMemset(st, 0, sizeof(int));
    bool ok = launch_sdf_from_mesh(m.dev, nx, ny, nz, f4(s->box.lo, 0.f), f4(s->steps, 0.f), d, st);
    s->values.resize(n);
    int status = 0;
    ok = ok && cudaMemcpy(s->values.data(), d, sizeof(float) * n, cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaMemcpy(&status, st, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    cudaFree(st);
    if (!ok) { delete s; set_error(SC_ERR_CUDA, "SDF from mesh failed"); return nullptr; }
    if (status) set_error(SC_ERR_DEVICE_STATUS, "mesh tree search stack overflow");
    s->compute_gradient();
    return s;
}

int scGetSDFGrid(scHandle sdf, int* cells3, float* box6, float* values, int cap)
{
    SDFC* s = (SDFC*)sdf;
    if (!s || s->type != CT_SDF) { set_error(SC_ERR_ARG, "not an SDF"); return 0; }
    if (cells3) { cells3[0] = s->nc[0]; cells3[1] = s->nc[1]; cells3[2] = s->nc[2]; }
    if (box6)
    {
        box6[0] = s->box.lo.x; box6[1] = s->box.lo.y; box6[2] = s->box.lo.z;
        box6[3] = s->box.hi.x; box6[4] = s->box.hi.y; box6[5] = s->box.hi.z;
    }
    for (size_t i = 0; values && i < s->values.size() && (int)i < cap; i++) values[i] = s->values[i];
    return (int)s->values.size();
}

void scFreeCollidable(scHandle c) { delete (Collidable*)c; }

// SDF::WriteToFile (Geometry/SDF.cpp:78-114): 3 ints (cells per side), the box as
// doubles (min.x, max.x, min.y, max.y, min.z, max.z), the values as doubles, x fastest
bool scSaveSDF(scHandle sdf, const char* path)
{
    SDFC* s = (SDFC*)sdf;
    if (!s || s->type != CT_SDF || !path) { set_error(SC_ERR_ARG, "not an SDF"); return false; }
    FILE* f = fopen(path, "wb");
    if (!f) { set_error(SC_ERR_ARG, std::string("cannot write ") + path); return false; }
    bool ok = fwrite(s->nc, sizeof(int), 3, f) == 3;
    const double b[6] = {s->box.lo.x, s->box.hi.x, s->box.lo.y, s->box.hi.y, s->box.lo.z, s->box.hi.z};
    ok = ok && fwrite(b, sizeof(double), 6, f) == 6;
    for (size_t i = 0; ok && i < s->values.size(); i++)
    {
        const double v = s->values[i];
        ok = fwrite(&v, sizeof(double), 1, f) == 1;
    }
    fclose(f);
    if (!ok) set_error(SC_ERR_ARG, std::string("short write to ") + path);
    return ok;
}

// SDF::LoadFromFile (Geometry/SDF.cpp:116-151) into a new SDF collidable (gradient computed)
scHandle scLoadSDF(const char* path)
{
    if (!path) { set_error(SC_ERR_ARG, "null path"); return nullptr; }
    FILE* f = fopen(path, "rb");
    if (!f) { set_error(SC_ERR_ARG, std::string("cannot read ") + path); return nullptr; }
    int nc[3] = {0, 0, 0};
    double b[6];
    bool ok = fread(nc, sizeof(int), 3, f) == 3 && fread(b, sizeof(double), 6, f) == 6 &&
              nc[0] > 0 && nc[1] > 0 && nc[2] > 0 && nc[0] < 65536 && nc[1] < 65536 && nc[2] < 65536;
    if (!ok) { fclose(f); set_error(SC_ERR_ARG, std::string("not an SDF file: ") + path); return nullptr; }
    scAabb3 box;
    box.min.x = (float)b[0]; box.max.x = (float)b[1]; box.min.y = (float)b[2];
    box.max.y = (float)b[3]; box.min.z = (float)b[4]; box.max.z = (float)b[5];
    SDFC* s = new_sdf(nc[0], nc[1], nc[2], box);
    const size_t n = (size_t)(nc[0] + 1) * (nc[1] + 1) * (nc[2] + 1);
    s->values.resize(n);
    for (size_t i = 0; ok && i < n; i++)
    {
        double v;
        ok = fread(&v, sizeof(double), 1, f) == 1;
        s->values[i] = (float)v;
    }
    fclose(f);
    if (!ok) { delete s; set_error(SC_ERR_ARG, std::string("truncated SDF file: ") + path); return nullptr; }
    s->compute_gradient();
    return s;
}

scHandle scCreateMeshCollider(const float* vertices, int nv, const unsigned* indices, int ni)
{
    if (!vertices || !indices || nv <= 0 || ni <= 0 || ni % 3) { set_error(SC_ERR_ARG, "bad mesh"); return nullptr; }
    MeshC* m = new MeshC();
    m->type = CT_MESH;
    m->mesh.verts.resize(nv);
    for (int i = 0; i < nv; i++) m->mesh.verts[i] = mk(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    m->mesh.idx.assign(indices, indices + ni);
    m->mesh.compute_normals();
    m->mesh.construct_edges();
    m->mesh.construct_rings(false, true);
    return m;
}

int scGetCollidableType(scHandle c) { return c ? ((Collidable*)c)->type : CT_INVALID; }
void* scGetMeshTree(scHandle c)
{
    Collidable* k = (Collidable*)c;
    if (!k || k->type != CT_MESH) return nullptr;
    MeshC* m = (MeshC*)k;
    return m->built ? (void*)&m->tree : nullptr;
}
void scGetWallsInfo(scHandle c, scAabb3* box)
{
    Collidable* k = (Collidable*)c;
    if (!k || k->type != CT_WALLS || !box) return;
    box->min = sv(((WallsC*)k)->box.lo); box->max = sv(((WallsC*)k)->box.hi);
}
void scGetSphereInfo(scHandle c, float* radius, scVector3* center)
{
    Collidable* k = (Collidable*)c;
    if (!k || k->type != CT_SPHERE) return;
    if (radius) *radius = ((SphereC*)k)->radius;
    if (center) *center = sv(k->center);
}
void scGetCapsuleInfo(scHandle c, float* radius, float* halfHeight, scVector3* center, scQuaternion* rot)
{
    Collidable* k = (Collidable*)c;
    if (!k || k->type != CT_CAPSULE) return;
    CapsuleC* cap = (CapsuleC*)k;
    if (radius) *radius = cap->r;
    if (halfHeight) *halfHeight = cap->hh;
    if (center) *center = sv(cap->center);
    if (rot) { rot->s = cap->rot[0]; rot->v.x = cap->rot[1]; rot->v.y = cap->rot[2]; rot->v.z = cap->rot[3]; }
}

// ------------------------------------------------------------------ patch
scClothPatch scCreateClothPatch(scCollisionWorld w)
{
    scClothPatch p; p.ptr = nullptr;
    if (!W(w)) { set_error(SC_ERR_ARG, "null world"); return p; }
    p.ptr = new ClothPatch(*W(w));
    return p;
}
void scFreeClothPatch(scClothPatch p) { delete P(p); }

scClothPatch scCreateClothBatch(scCollisionWorld w, const scClothPatch* parts, int count)
{
    scClothPatch p; p.ptr = nullptr;
    if (!W(w) || !parts || count < 1) { set_error(SC_ERR_ARG, "batch needs a world and at least one patch"); return p; }
    std::vector<ClothPatch*> v;
    for (int k = 0; k < count; k++) v.push_back(P(parts[k]));
    ClothPatch* b = new ClothPatch(*W(w));
    if (!b->init_batch(v)) { delete b; return p; }
    p.ptr = b;
    return p;
}

int scGetBatchSize(scClothPatch p)
{
    if (!P(p)) return 0;
    const auto& iv = P(p)->model.instV;
    return iv.empty() ? 1 : (int)iv.size() - 1;
}

void scGetBatchInstance(scClothPatch p, int k, int* firstParticle, int* numParticles)
{
    if (!P(p)) return;
    const auto& iv = P(p)->model.instV;
    int a = 0, n = P(p)->model.N;
    if (!iv.empty())
    {
        if (k < 0 || k + 1 >= (int)iv.size()) { set_error(SC_ERR_ARG, "instance out of range"); return; }
        a = iv[k]; n = iv[k + 1] - iv[k];
    }
    if (firstParticle) *firstParticle = a;
    if (numParticles) *numParticles = n;
}
scModel scGetClothModel(scClothPatch p) { scModel m; m.ptr = P(p) ? &P(p)->model : nullptr; return m; }
scMesh scGetClothMesh(scClothPatch p) { scMesh m; m.ptr = P(p) ? &P(p)->mesh : nullptr; return m; }

void scInitCloth(scClothPatch p, int divX, int divY, float inc, scVector3 offset, bool horizontal, bool attached)
{
    if (!P(p)) { set_error(SC_ERR_ARG, "null patch"); return; }
    P(p)->init_grid(divX, divY, inc, v3(offset), horizontal, attached);
}

void scInitClothMesh(scClothPatch p, const float* vertices, int nv, const unsigned* indices, int ni, const float* uvs,
                     const float* colors, scVector3 offset, bool attached)
{
    if (!P(p) || !vertices || !indices || nv < 3 || ni < 3 || ni % 3) { set_error(SC_ERR_ARG, "bad cloth mesh"); return; }
    std::vector<V3> v(nv);
    for (int i = 0; i < nv; i++) v[i] = mk(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    std::vector<uint32_t> idx(indices, indices + ni);
    P(p)->init_mesh(v, idx, uvs, colors, v3(offset), attached);
}

// Wavefront OBJ (v, vt, f; polygons fanned into triangles) as a triangle soup:
// one vertex per face corner with its uv, as a mesh importer delivers it; the
// cloth initialisation then merges coincident corners. Returns false when the
// file cannot be read or names an index out of range.
static bool read_obj(const char* path, std::vector<V3>& verts, std::vector<uint32_t>& idx, std::vector<float>& uvs)
{
    FILE* f = fopen(path, "r");
    if (!f) return false;
    std::vector<V3> v;
    std::vector<float> vt;
    char line[4096];
    bool ok = true;
    while (ok && fgets(line, sizeof(line), f))
    {
        if (line[0] == 'v' && line[1] == ' ')
        {
            float x, y, z;
            if (sscanf(line + 2, "%f %f %f", &x, &y, &z) == 3) v.push_back(mk(x, y, z));
        }
        else if (line[0] == 'v' && line[1] == 't' && line[2] == ' ')
        {
            float a = 0, b = 0;
            if (sscanf(line + 3, "%f %f", &a, &b) >= 1) { vt.push_back(a); vt.push_back(b); }
        }
        else if (line[0] == 'f' && line[1] == ' ')
        {
            std::vector<std::pair<int, int>> corners;
            char* q = line + 2;
            while (*q)
            {
                while (*q == ' ' || *q == '\t') q++;
                if (!*q || *q == '\n' || *q == '\r') break;
                int vi = 0, ti = 0;
                int nread = 0;
                if (sscanf(q, "%d/%d%n", &vi, &ti, &nread) == 2) {}
                else if (sscanf(q, "%d%n", &vi, &nread) == 1) ti = 0;
                else { ok = false; break; }
                q += nread;
                while (*q && *q != ' ' && *q != '\t' && *q != '\n' && *q != '\r') q++;   // skip "/normal"
                if (vi < 0) vi = (int)v.size() + 1 + vi;
                if (ti < 0) ti = (int)(vt.size() / 2) + 1 + ti;
                corners.push_back({vi - 1, ti - 1});
            }
            for (size_t k = 2; ok && k < corners.size(); k++)
                for (size_t c : {(size_t)0, k - 1, k})
                {
                    const int vi = corners[c].first, ti = corners[c].second;
                    if (vi < 0 || vi >= (int)v.size() || ti >= (int)(vt.size() / 2)) { ok = false; break; }
                    idx.push_back((uint32_t)verts.size());
                    verts.push_back(v[vi]);
                    uvs.push_back(ti >= 0 ? vt[2 * ti] : 0.f);
                    uvs.push_back(ti >= 0 ? vt[2 * ti + 1] : 0.f);
                }
        }
    }
    fclose(f);
    return ok && !idx.empty();
}

bool scInitClothObj(scClothPatch p, const char* path, scVector3 offset, bool attached)
{
    if (!P(p) || !path) { set_error(SC_ERR_ARG, "null patch or path"); return false; }
    std::vector<V3> v;
    std::vector<uint32_t> idx;
    std::vector<float> uv;
    if (!read_obj(path, v, idx, uv)) { set_error(SC_ERR_ARG, std::string("cannot read OBJ mesh ") + path); return false; }
    return P(p)->init_mesh(v, idx, uv.data(), nullptr, v3(offset), attached);
}

int scGetMeshParticleMap(scClothPatch p, int* map, int cap)
{
    if (!P(p)) return 0;
    const auto& mm = P(p)->meshMap;
    for (int i = 0; map && i < cap && i < (int)mm.size(); i++) map[i] = mm[i];
    return (int)mm.size();
}

void scStepCloth(scClothPatch p, float dt)
{
    if (!P(p)) { set_error(SC_ERR_ARG, "null patch"); return; }
    P(p)->step(dt);
}

void scUpdateClothMesh(scClothPatch p) { if (P(p)) P(p)->update_mesh(); }

// ClothPatch::ComputeStrainMap (Physics/ClothPatch.cpp:337-381)
void scComputeStrainMap(scClothPatch p, scVector3* colors)
{
    if (!P(p) || !colors) return;
    ClothModel& m = P(p)->model;
    host_sync(&m);
    std::vector<V3> col(m.N, mk(0, 0, 0));
    const float PI = 3.1415926535897932384626433832795f;
    for (const FemHost& t : m.tris)
    {
        V3 dx1 = m.hpos[t.i2] - m.hpos[t.i1], dx2 = m.hpos[t.i3] - m.hpos[t.i1];
        V3 wu = t.invDet * (t.dv2 * dx1 - t.dv1 * dx2);
        V3 wv = t.invDet * (-t.du2 * dx1 + t.du1 * dx2);
        float euu = 0.5f * (dot(wu, wu) - 1), evv = 0.5f * (dot(wv, wv) - 1), euv = dot(wu, wv);
        float s = sqrtf(euu * euu + evv * evv + euv * euv);
        V3 e1 = normalized(dx1), e2 = normalized(m.hpos[t.i3] - m.hpos[t.i2]), e3 = normalized(-dx2);
        float t1 = (float)acos(-dot(e1, e3)), t2 = (float)acos(-dot(e1, e2)), t3 = (float)acos(-dot(e2, e3));
        s *= 10.f;
        V3 c = mk(s, 0, s);
        col[t.i1] += (t1 / PI) * c; col[t.i2] += (t2 / PI) * c; col[t.i3] += (t3 / PI) * c;
    }
    for (int i = 0; i < m.N; i++) colors[i] = sv(col[i]);
}

// ------------------------------------------------------------------ model
int scGetNumParticles(scModel m) { return M(m) ? M(m)->N : 0; }
void scGetParticlePos(scModel m, int i, scVector3* pos)
{
    if (!check_model(M(m), i) || !pos) return;
    host_sync(M(m));
    *pos = sv(M(m)->hpos[i]);
}
float scGetParticleInvMass(scModel m, int i)
{
    if (!check_model(M(m), i)) return 0.f;
    host_sync(M(m));
    return M(m)->invMass[i];
}
int scGetNumTris(scModel m) { return M(m) ? (int)M(m)->tris.size() : 0; }
void scGetTriangle(scModel m, int i, int* i1, int* i2, int* i3)
{
    if (!M(m) || i < 0 || i >= (int)M(m)->tris.size()) { set_error(SC_ERR_ARG, "triangle index out of range"); return; }
    const FemHost& t = M(m)->tris[i];
    if (i1) *i1 = t.i1; if (i2) *i2 = t.i2; if (i3) *i3 = t.i3;
}
void scGetTriangleInfo(scModel m, int i, float* invDet, scVector2* du, scVector2* dv, scVector2* s)
{
    if (!M(m) || i < 0 || i >= (int)M(m)->tris.size()) { set_error(SC_ERR_ARG, "triangle index out of range"); return; }
    const FemHost& t = M(m)->tris[i];
    if (invDet) *invDet = t.invDet;
    if (du) { du->x = t.du1; du->y = t.du2; }
    if (dv) { dv->x = t.dv1; dv->y = t.dv2; }
    if (s) { s->x = t.su; s->y = t.sv; }
}
int scGetNumQuads(scModel m) { return M(m) ? (int)M(m)->quads.size() : 0; }
void scGetQuad(scModel m, int i, int* i1, int* i2, int* i3, int* i4)
{
    if (!M(m) || i < 0 || i >= (int)M(m)->quads.size()) { set_error(SC_ERR_ARG, "quad index out of range"); return; }
    uint4 q = M(m)->quads[i];
    if (i1) *i1 = q.x; if (i2) *i2 = q.y; if (i3) *i3 = q.z; if (i4) *i4 = q.w;
}
int scGetNumLinks(scModel m) { return M(m) ? (int)M(m)->links.size() : 0; }
void scGetLink(scModel m, int i, int* i1, int* i2)
{
    if (!M(m) || i < 0 || i >= (int)M(m)->links.size()) { set_error(SC_ERR_ARG, "link index out of range"); return; }
    if (i1) *i1 = M(m)->links[i].x; if (i2) *i2 = M(m)->links[i].y;
}

// vertex contacts in list order: collider, then particle, then slot
static std::vector<VC> vertex_contacts(ClothModel* m, std::vector<int>* owner)
{
    std::vector<VC> out;
    if (!m->buf.vc || m->buf.numVColl == 0) return out;
    host_sync(m);
    size_t total = 0, counts = 0;
    for (auto& g : m->vcollHost)
    {
        total = std::max(total, (size_t)g.slotBase + (size_t)g.kmax * g.vCount);
        counts = std::max(counts, (size_t)g.countBase + g.vCount);
    }
    std::vector<uint8_t> cnt = dl(m->buf.vcCount, counts);
    std::vector<VC> slots = dl(m->buf.vc, total);
    for (int ci = 0; ci < m->buf.numVColl; ci++)
    {
        const VColl& g = m->vcollHost[ci];
        for (int i = g.vBegin; i < g.vBegin + g.vCount; i++)
            for (int k = 0; k < cnt[(size_t)g.countBase + (i - g.vBegin)]; k++)
            {
                out.push_back(slots[g.slotBase + (size_t)(i - g.vBegin) * g.kmax + k]);
                if (owner) owner->push_back(i);
            }
    }
    return out;
}

int scGetNumContacts(scModel m) { return M(m) ? (int)vertex_contacts(M(m), nullptr).size() : 0; }
void scGetContact(scModel m, int i, scVector3* point, scVector3* normal)
{
    if (!M(m)) return;
    std::vector<VC> v = vertex_contacts(M(m), nullptr);
    if (i < 0 || i >= (int)v.size()) { set_error(SC_ERR_ARG, "contact index out of range"); return; }
    if (point) *point = {v[i].point.x, v[i].point.y, v[i].point.z};
    if (normal) *normal = {v[i].normal.x, v[i].normal.y, v[i].normal.z};
}
int scGetNumTriContacts(scModel m)
{
    if (!M(m) || !M(m)->buf.tcCount) return 0;
    host_sync(M(m));
    return dcount(M(m)->buf.tcCount);
}
void scGetTriContact(scModel m, int i, scVector3* point, scVector3* normal)
{
    int n = scGetNumTriContacts(m);
    if (i < 0 || i >= n) { set_error(SC_ERR_ARG, "contact index out of range"); return; }
    TC t;
    cudaMemcpy(&t, M(m)->buf.tcList + i, sizeof(TC), cudaMemcpyDeviceToHost);
    if (point) *point = {t.point.x, t.point.y, t.point.z};
    if (normal) *normal = {t.normal.x, t.normal.y, t.normal.z};
}

#define SC_GETSET(Name, field, type)                                             \
    type scGet##Name(scModel m) { return M(m) ? (type)M(m)->prm.field : (type)0; } \
    void scSet##Name(scModel m, type v) { if (M(m)) { M(m)->prm.field = v; M(m)->touch(); } }

SC_GETSET(CollisionFlags, flags, int)
SC_GETSET(Thickness, thickness, float)
SC_GETSET(Tolerance, tolerance, float)
SC_GETSET(Friction, friction, float)
SC_GETSET(NumIterations, iterations, int)
SC_GETSET(UseFEM, fem, bool)
SC_GETSET(Unit, unit, float)

void* scGetClothTree(scModel m) { return M(m) ? (void*)&M(m)->triBvh : nullptr; }

void scAddMouseSpring(scModel m, int i1, int i2, int i3, scVector3 coords, scVector3 p)
{
    if (!check_model(M(m))) return;
    (void)i1; (void)i2; (void)i3; (void)coords; (void)p;
    set_error(SC_ERR_UNSUPPORTED, "mouse spring is interactive-only and not part of the GPU step");
}
void scUpdateMouseSpring(scModel m, scVector3 p) { (void)m; (void)p; }
void scRemoveMouseSpring(scModel m) { (void)m; }

// ------------------------------------------------------------------- mesh
int scGetMeshVertexCount(scMesh mesh) { return mesh.ptr ? (int)((HMesh*)mesh.ptr)->verts.size() : 0; }
int scGetMeshIndexCount(scMesh mesh) { return mesh.ptr ? (int)((HMesh*)mesh.ptr)->idx.size() : 0; }
scVector3* scGetMeshNormalBuffer(scMesh mesh)
{
    HMesh* h = (HMesh*)mesh.ptr;
    return (h && !h->normals.empty()) ? (scVector3*)h->normals.data() : nullptr;
}
scVector3* scGetMeshVertexBuffer(scMesh mesh)
{
    HMesh* h = (HMesh*)mesh.ptr;
    return (h && !h->verts.empty()) ? (scVector3*)h->verts.data() : nullptr;
}
unsigned int* scGetMeshIndexBuffer(scMesh mesh)
{
    HMesh* h = (HMesh*)mesh.ptr;
    return (h && !h->idx.empty()) ? (unsigned int*)h->idx.data() : nullptr;
}

// --------------------------------------------------------------- additions
void scSetShearStiffness(scModel m, float v) { if (M(m)) { M(m)->prm.shear = v; M(m)->touch(); } }
void scSetBendStiffness(scModel m, float v) { if (M(m)) { M(m)->prm.bend = v; M(m)->touch(); } }
void scSetStretchStiffness(scModel m, float v) { if (M(m)) { M(m)->prm.stretch = v; M(m)->touch(); } }
void scSetPoisson(scModel m, float v) { if (M(m)) { M(m)->prm.poisson = v; M(m)->touch(); } }
void scSetDragCoeff(scModel m, float v) { if (M(m)) { M(m)->prm.drag = v; M(m)->touch(); } }
void scSetDihedral(scModel m, bool v) { if (M(m)) { M(m)->prm.dihedral = v; M(m)->touch(); } }
void scSetSolverType(scModel m, int type)
{
    if (!M(m) || type < 0 || type > 4) { set_error(SC_ERR_ARG, "solver type must be 0..4"); return; }
    M(m)->prm.solverType = type;
    M(m)->touch();
}
int scGetSolverType(scModel m) { return M(m) ? M(m)->prm.solverType : 1; }
void scSetSelfShrink(scModel m, float v) { if (M(m)) { M(m)->prm.selfShrink = v; M(m)->touch(); } }
void scSetNumSteps(scClothPatch p, int v)
{
    if (!P(p) || v < 1) { set_error(SC_ERR_ARG, "substeps must be >= 1"); return; }
    P(p)->numSteps = v;
}
int scGetNumSteps(scClothPatch p) { return P(p) ? P(p)->numSteps : 0; }

void scSetMasses(scModel m, const float* masses)
{
    if (!check_model(M(m)) || !masses) return;
    host_sync(M(m));
    for (int i = 0; i < M(m)->N; i++) M(m)->invMass[i] = masses[i] == 0.f ? 0.f : 1.f / masses[i];
    M(m)->upload_state(M(m)->owner->stream);
}
void scSetParticleInvMass(scModel m, int i, float w)
{
    if (!check_model(M(m), i)) return;
    host_sync(M(m));
    M(m)->invMass[i] = w;
    M(m)->upload_state(M(m)->owner->stream);
}
void scSetParticlePositions(scModel m, const float* xyz)
{
    if (!check_model(M(m)) || !xyz) return;
    host_sync(M(m));
    for (int i = 0; i < M(m)->N; i++)
    {
        M(m)->hpos[i] = mk(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        M(m)->hprev[i] = M(m)->hpos[i];
    }
    M(m)->upload_state(M(m)->owner->stream);
}
void scSetParticleState(scModel m, const float* pos, const float* prev, const float* vel)
{
    if (!check_model(M(m)) || !pos || !prev || !vel) return;
    host_sync(M(m));
    M(m)->set_state(pos, prev, vel, M(m)->owner->stream);
}
static void get3(scModel m, float* xyz, int which)
{
    if (!check_model(M(m)) || !xyz) return;
    host_sync(M(m));
    const std::vector<V3>& v = which == 0 ? M(m)->hpos : (which == 1 ? M(m)->hvel : M(m)->hprev);
    memcpy(xyz, v.data(), sizeof(float) * 3 * M(m)->N);
}
void scGetParticlePositions(scModel m, float* xyz) { get3(m, xyz, 0); }
void scGetParticleVelocities(scModel m, float* xyz) { get3(m, xyz, 1); }
void scGetParticlePrevPositions(scModel m, float* xyz) { get3(m, xyz, 2); }
void scSetFixedIterations(scModel m, bool v) { if (M(m)) { M(m)->prm.fixedIterations = v; M(m)->touch(); } }
void scSetSelfCCD(scModel m, bool v) { if (M(m)) { M(m)->prm.ccd = v; M(m)->touch(); } }
void scSetClusterSolver(scModel m, bool v) { scSetSolverMode(m, v ? SOLVE_CLUSTER : SOLVE_KERNELS); }
void scSetSolverMode(scModel m, int mode)
{
    if (!M(m) || mode < SOLVE_AUTO || mode > SOLVE_BAND) { set_error(SC_ERR_ARG, "solver mode must be 0..4"); return; }
    M(m)->solverMode = mode;
    M(m)->tuned = false;
    M(m)->touch();
}
void scSetGridSolver(scModel m, int variant, int blocksPerSm)
{
    if (!M(m) || variant < 0 || variant >= gs_grid_variants() || blocksPerSm < 1) { set_error(SC_ERR_ARG, "bad grid solver variant"); return; }
    M(m)->solverMode = SOLVE_GRID;
    M(m)->choice = {SOLVE_GRID, variant, blocksPerSm, 0.f};
    M(m)->tuned = true;
    M(m)->touch();
    M(m)->tunedVersion = M(m)->paramVersion;
}
void scSetClusterVariant(scModel m, int variant)
{
    if (!M(m) || variant < 0 || variant >= gs_cluster_variants()) { set_error(SC_ERR_ARG, "bad cluster solver variant"); return; }
    M(m)->solverMode = SOLVE_CLUSTER;
    M(m)->choice = {SOLVE_CLUSTER, variant, 0, 0.f};
    M(m)->tuned = true;
    M(m)->touch();
    M(m)->tunedVersion = M(m)->paramVersion;
}
void scSetBandVariant(scModel m, int variant)
{
    if (!M(m) || variant < 0 || variant >= gs_band_variants()) { set_error(SC_ERR_ARG, "bad band solver variant"); return; }
    if (!M(m)->bandPlan.valid) { set_error(SC_ERR_UNSUPPORTED, "the cloth has no band plan"); return; }
    M(m)->solverMode = SOLVE_BAND;
    M(m)->choice = {SOLVE_BAND, variant, 0, 0.f};
    M(m)->tuned = true;
    M(m)->touch();
    M(m)->tunedVersion = M(m)->paramVersion;
}
int scGetSolverChoice(scModel m, int* out4, float* tuneMs, int cap)
{
    if (!M(m)) return 0;
    const SolverChoice& ch = M(m)->choice;
    if (out4)
    {
        int th = 0, ft = 0, bt = 0;
        if (ch.kind == SOLVE_GRID) gs_grid_variant_info(ch.variant, th, ft, bt);
        if (ch.kind == SOLVE_BAND) th = gs_band_threads(ch.variant);
        if (ch.kind == SOLVE_CLUSTER) th = GS_THREADS;
        out4[0] = ch.kind; out4[1] = ch.variant; out4[2] = ch.blocksPerSm; out4[3] = th;
    }
    const auto& log = M(m)->tuneLog;
    if (tuneMs)
        for (int k = 0; k < cap && k < (int)log.size(); k++)
        {
            tuneMs[4 * k] = (float)log[k].kind; tuneMs[4 * k + 1] = (float)log[k].variant;
            tuneMs[4 * k + 2] = (float)log[k].blocksPerSm; tuneMs[4 * k + 3] = log[k].ms;
        }
    return (int)log.size();
}
int scGetBandPlan(scModel m, int* out4)
{
    if (!M(m)) return 0;
    const auto& bp = M(m)->bandPlan;
    if (out4)
    {
        out4[0] = bp.valid ? bp.clusterSize : 0;
        out4[1] = bp.valid ? (1 << bp.shift) : 0;
        out4[2] = bp.valid ? bp.halo : 0;
        out4[3] = M(m)->band_active() ? 1 : 0;
    }
    return bp.valid ? 1 : 0;
}
void scSetBroadPhaseMode(scModel m, int mode)
{
    if (!M(m) || mode < -1 || mode >= BROAD_WALKS) { set_error(SC_ERR_ARG, "broad-phase mode must be -1, 0 or 1"); return; }
    M(m)->broadMode = mode;
    if (mode >= 0) { M(m)->broadWalk = mode; M(m)->buf.broadWalk = mode; }
    M(m)->tuned = false;
    M(m)->touch();
}

int scGetBroadPhaseMode(scModel m, float* ms2)
{
    if (!M(m)) return -1;
    if (ms2) for (int k = 0; k < BROAD_WALKS; k++) ms2[k] = M(m)->broadMs[k];
    return M(m)->broadWalk;
}

int scGetGridVariants(int* info3, int cap)
{
    const int n = gs_grid_variants();
    for (int v = 0; info3 && v < n && v < cap; v++) gs_grid_variant_info(v, info3[3 * v], info3[3 * v + 1], info3[3 * v + 2]);
    return n;
}
void scSetClusterStaging(scModel m, bool v) { if (M(m)) { M(m)->prm.stageRecords = v; M(m)->touch(); } }
void scSetSolverPrecision(scModel m, int mode)
{
    ClothModel* c = M(m);
    if (!c || (mode != 0 && mode != 1)) { set_error(SC_ERR_ARG, "scSetSolverPrecision: mode must be 0 (IEEE) or 1 (fast)"); return; }
    if (c->prm.fastMath != (mode == 1)) { c->prm.fastMath = mode == 1; c->touch(); }
}
int scGetSolverPrecision(scModel m) { return M(m) ? (int)M(m)->prm.fastMath : -1; }
void scSetResidualTarget(scModel m, float tol, int maxIterations)
{
    ClothModel* c = M(m);
    if (!c || tol < 0.f || maxIterations < 1) { set_error(SC_ERR_ARG, "residual target needs tol >= 0 and maxIterations >= 1"); return; }
    c->prm.resTol = tol;
    if (tol > 0.f)
    {
        c->prm.iterations = maxIterations;
        c->prm.fixedIterations = true;     // the residual decides, not the reference's exit test
    }
    c->tuned = false;
    c->touch();
}

int scGetStaticColours(scModel m, int* triColour, int* edgeColour, int* counts2)
{
    ClothModel* c = M(m);
    if (!c) { set_error(SC_ERR_ARG, "scGetStaticColours: null model"); return -1; }
    if (triColour)
        for (int col = 0; col + 1 < (int)c->triColourStart.size(); col++)
            for (int k = c->triColourStart[col]; k < c->triColourStart[col + 1]; k++) triColour[c->triOrder[k]] = col;
    if (edgeColour)
        for (size_t e = 0; e < c->edgeColourHost.size(); e++) edgeColour[e] = c->edgeColourHost[e];
    if (counts2) { counts2[0] = c->dc.nTriColours; counts2[1] = c->dc.nEdgeColours; }
    return (int)c->edgeColourHost.size();
}

void scSetResidualUnit(scModel m, int unit)
{
    ClothModel* c = M(m);
    if (!c || (unit != 0 && unit != 1)) { set_error(SC_ERR_ARG, "scSetResidualUnit: unit must be 0 (mean rest edge) or 1 (metres)"); return; }
    if (c->prm.resMetres != (unit == 1)) { c->prm.resMetres = unit == 1; c->touch(); }
}

int scGetIterationTotal(scModel m)
{
    ClothModel* c = M(m);
    if (!c || !c->dc.scal) return 0;
    host_sync(c);
    float v = 0.f;
    cudaMemcpy(&v, c->dc.scal + 10, sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemset(c->dc.scal + 10, 0, sizeof(float));
    return (int)v;
}

bool scSetWarmStart(scModel m, const float* params, const float* norm)
{
    ClothModel* c = M(m);
    if (!c) { set_error(SC_ERR_ARG, "null model"); return false; }
    host_sync(c);
    if (!params) { c->warmStart = false; c->touch(); return true; }
    if (!norm) { set_error(SC_ERR_ARG, "warm start needs its 27 normalisation values"); return false; }
    if (!c->mlpPrm && cudaMalloc(&c->mlpPrm, sizeof(float) * (MLP_NPARAM + MLP_NNORM)) != cudaSuccess)
    {
        c->mlpPrm = nullptr;
        set_error(SC_ERR_CUDA, "cudaMalloc failed");
        return false;
    }
    cudaMemcpy(c->mlpPrm, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice);
    cudaMemcpy(c->mlpPrm + MLP_NPARAM, norm, sizeof(float) * MLP_NNORM, cudaMemcpyHostToDevice);
    c->warmStart = true;
    c->tuned = false;
    c->touch();
    return true;
}

bool scSetSampleBuffers(scModel m, float* features, float* targets)
{
    ClothModel* c = M(m);
    if (!c || c->N == 0) { set_error(SC_ERR_ARG, "model not initialised"); return false; }
    host_sync(c);
    if (!features || !targets) { c->sampleFeat = c->sampleTarget = nullptr; c->touch(); return true; }
    c->sampleFeat = features;
    c->sampleTarget = targets;
    c->touch();
    return true;
}

int scMlpParamCount(void) { return MLP_NPARAM; }

int scMlpForward(const float* X, int S, const float* params, const float* norm, float* Y, void* stream)
{
    if (!X || !params || !norm || !Y || S < 0) return SC_ERR_ARG;
    launch_mlp_forward((cudaStream_t)stream, X, S, params, norm, Y);
    return cudaGetLastError() == cudaSuccess ? SC_OK : SC_ERR_CUDA;
}

int scMlpGradients(const float* X, const float* T, int S, const float* params, const float* norm, float* grad,
                   float* loss, void* stream)
{
    if (!X || !T || !params || !norm || !grad || !loss || S < 1) return SC_ERR_ARG;
    return launch_mlp_grad((cudaStream_t)stream, X, T, S, params, norm, grad, loss) ? SC_OK : SC_ERR_CUDA;
}

int scMlpAdamStep(float* params, const float* grad, float* m, float* v, int step, float lr, void* stream)
{
    if (!params || !grad || !m || !v || step < 1) return SC_ERR_ARG;
    launch_adam((cudaStream_t)stream, params, grad, m, v, step, lr);
    return cudaGetLastError() == cudaSuccess ? SC_OK : SC_ERR_CUDA;
}

float scGetResidual(scModel m)
{
    ClothModel* c = M(m);
    if (!c || !c->dc.scal || !c->dc.fem) return -1.f;
    host_sync(c);
    unsigned* word = reinterpret_cast<unsigned*>(c->dc.scal + 12);
    launch_residual(c->owner->stream, c->dc, word);
    unsigned u = 0;
    cudaMemcpyAsync(&u, word, sizeof(unsigned), cudaMemcpyDeviceToHost, c->owner->stream);
    cudaStreamSynchronize(c->owner->stream);
    float r;
    memcpy(&r, &u, sizeof(r));
    return r;
}

int scGetSolverIterations(scModel m)
{
    if (!M(m) || !M(m)->dc.scal) return 0;
    host_sync(M(m));
    float v = 0;
    cudaMemcpy(&v, M(m)->dc.scal + 9, sizeof(float), cudaMemcpyDeviceToHost);
    return (int)v;
}

int scGetConstraintOrder(scModel m, int kind, int* order, int* colourStart)
{
    if (!M(m)) return 0;
    // the band solver's order while it is the one in use (solver mode 4 on a
    // cloth with a band plan), else the colour order of the other solvers
    const bool band = M(m)->band_active();
    const auto& bp = M(m)->bandPlan;
    const std::vector<int>& o = band ? (kind == 0 ? bp.triOrder : kind == 1 ? bp.bendOrder : bp.linkOrder)
                                     : (kind == 0 ? M(m)->triOrder : kind == 1 ? M(m)->bendOrder : M(m)->linkOrder);
    const std::vector<int>& s = band ? (kind == 0 ? bp.triStart : kind == 1 ? bp.bendStart : bp.linkStart)
                                     : (kind == 0 ? M(m)->triColourStart : kind == 1 ? M(m)->bendColourStart : M(m)->linkColourStart);
    if (s.empty()) return 0;
    if (order) memcpy(order, o.data(), sizeof(int) * o.size());
    if (colourStart) memcpy(colourStart, s.data(), sizeof(int) * s.size());
    return (int)s.size() - 1;
}
void scGetTriangleRest(scModel m, float* rest10)
{
    if (!M(m) || !rest10) return;
    const auto& tr = M(m)->tris;
    for (size_t i = 0; i < tr.size(); i++)
    {
        float* r = rest10 + 10 * i;
        r[0] = tr[i].du1; r[1] = tr[i].du2; r[2] = tr[i].dv1; r[3] = tr[i].dv2; r[4] = tr[i].invDet;
        r[5] = tr[i].lu0; r[6] = tr[i].lv0; r[7] = tr[i].lu2; r[8] = tr[i].lv2; r[9] = tr[i].area;
    }
}

void scGetLinkRest(scModel m, float* rest2)
{
    if (!M(m) || !rest2) return;
    const auto& lr = M(m)->linkRest;
    for (size_t i = 0; i < lr.size(); i++) { rest2[2 * i] = lr[i].x; rest2[2 * i + 1] = lr[i].y; }
}

int scGetNumBends(scModel m) { return M(m) ? (int)M(m)->bends.size() : 0; }
void scGetBends(scModel m, unsigned* idx4)
{
    if (!M(m) || !idx4) return;
    memcpy(idx4, M(m)->bends.data(), sizeof(uint4) * M(m)->bends.size());
}
int scGetNumEdges(scModel m) { return (M(m) && M(m)->owner) ? (int)M(m)->owner->mesh.edges.size() : 0; }
void scGetEdges(scModel m, int* e4)
{
    if (!M(m) || !e4) return;
    const auto& E = M(m)->owner->mesh.edges;
    for (size_t i = 0; i < E.size(); i++) { e4[4 * i] = E[i].i1; e4[4 * i + 1] = E[i].i2; e4[4 * i + 2] = E[i].t1; e4[4 * i + 3] = E[i].t2; }
}

int scGetNumContactsOfKind(scModel m, int kind)
{
    ClothModel* c = M(m);
    if (!c || !c->buf.tcCount) return 0;
    host_sync(c);
    switch (kind)
    {
    case 0: return (int)vertex_contacts(c, nullptr).size();
    case 1: return dcount(c->buf.tcCount);
    case 2: return dcount(c->buf.ecCount);
    case 3: return dcount(c->buf.stCount);
    case 4: return dcount(c->buf.seCount);
    }
    return 0;
}

void scGetSelfContacts(scModel m, int kind, int* idx4, float* f7)
{
    ClothModel* c = M(m);
    if (!c || !c->buf.stCount) return;
    int n = scGetNumContactsOfKind(m, kind);
    std::vector<SCt> v = dl(kind == 3 ? c->buf.stList : c->buf.seList, n);
    for (int i = 0; i < n; i++)
    {
        if (idx4) { idx4[4 * i] = v[i].idx.x; idx4[4 * i + 1] = v[i].idx.y; idx4[4 * i + 2] = v[i].idx.z; idx4[4 * i + 3] = v[i].idx.w; }
        if (f7)
        {
            float* f = f7 + 7 * i;
            f[0] = v[i].normal.x; f[1] = v[i].normal.y; f[2] = v[i].normal.z;
            f[3] = v[i].w.x; f[4] = v[i].w.y; f[5] = v[i].w.z; f[6] = v[i].side;
        }
    }
}

void scGetVertexContacts(scModel m, int* idx2, float* f6)
{
    if (!M(m)) return;
    std::vector<int> owner;
    std::vector<VC> v = vertex_contacts(M(m), &owner);
    for (size_t i = 0; i < v.size(); i++)
    {
        if (idx2) { idx2[2 * i] = owner[i]; idx2[2 * i + 1] = v[i].feature; }
        if (f6)
        {
            float* f = f6 + 6 * i;
            f[0] = v[i].point.x; f[1] = v[i].point.y; f[2] = v[i].point.z;
            f[3] = v[i].normal.x; f[4] = v[i].normal.y; f[5] = v[i].normal.z;
        }
    }
}

void scGetTriContacts(scModel m, int* idx4, float* f9)
{
    ClothModel* c = M(m);
    if (!c || !c->buf.tcCount) return;
    int n = scGetNumContactsOfKind(m, 1);
    std::vector<TC> v = dl(c->buf.tcList, n);
    for (int i = 0; i < n; i++)
    {
        if (idx4) { idx4[4 * i] = v[i].idx.x; idx4[4 * i + 1] = v[i].idx.y; idx4[4 * i + 2] = v[i].idx.z; idx4[4 * i + 3] = v[i].feature; }
        if (f9)
        {
            float* f = f9 + 9 * i;
            f[0] = v[i].point.x; f[1] = v[i].point.y; f[2] = v[i].point.z;
            f[3] = v[i].normal.x; f[4] = v[i].normal.y; f[5] = v[i].normal.z;
            f[6] = v[i].w.x; f[7] = v[i].w.y; f[8] = v[i].w.z;
        }
    }
}

void scGetEdgeContacts(scModel m, int* idx3, float* f8)
{
    ClothModel* c = M(m);
    if (!c || !c->buf.ecCount) return;
    int n = scGetNumContactsOfKind(m, 2);
    std::vector<EC> v = dl(c->buf.ecList, n);
    for (int i = 0; i < n; i++)
    {
        if (idx3) { idx3[3 * i] = v[i].idx.x; idx3[3 * i + 1] = v[i].idx.y; idx3[3 * i + 2] = v[i].feature; }
        if (f8)
        {
            float* f = f8 + 8 * i;
            f[0] = v[i].point.x; f[1] = v[i].point.y; f[2] = v[i].point.z;
            f[3] = v[i].normal.x; f[4] = v[i].normal.y; f[5] = v[i].normal.z;
            f[6] = v[i].w.x; f[7] = v[i].w.y;
        }
    }
}

int scGetCCDCandidates(scModel m, int kind, int* pairs, int cap)
{
    ClothModel* c = M(m);
    if (!c || !c->buf.ccdVtPairCount || !c->prm.ccd) return 0;
    host_sync(c);
    int n = dcount(kind == 0 ? c->buf.ccdVtPairCount : c->buf.ccdEePairCount);
    int lim = kind == 0 ? c->buf.ccdVtCap : c->buf.ccdEeCap;
    n = std::min(n, lim);
    if (pairs && n > 0 && cap > 0)
    {
        // the device keeps each query's candidates in traversal order; report them sorted
        std::vector<int2> all = dl(kind == 0 ? c->buf.ccdVtPairs : c->buf.ccdEePairs, n);
        std::sort(all.begin(), all.end(), [](int2 a, int2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
        memcpy(pairs, all.data(), sizeof(int2) * std::min(n, cap));
    }
    return n;
}

int scGetContactColours(scModel m, int cls, int* counts)
{
    ClothModel* c = M(m);
    if (!c || !c->buf.colourStart || cls < 0 || cls > 3) return 0;
    host_sync(c);
    std::vector<int> st = dl(c->buf.colourStart + cls * (MAX_COLOURS + 1), MAX_COLOURS + 1);
    int used = 0;
    for (int k = 0; k < MAX_COLOURS; k++)
    {
        int n = st[k + 1] - st[k];
        if (counts) counts[k] = n;
        if (n > 0) used = k + 1;
    }
    return used;
}

void scGetCollisionMeshNormals(scModel m, float* xyz)
{
    ClothModel* c = M(m);
    if (!c || !xyz || !c->dc.prevN) return;
    host_sync(c);
    std::vector<float4> n = dl(c->dc.prevN, c->N);
    for (int i = 0; i < c->N; i++) { xyz[3 * i] = n[i].x; xyz[3 * i + 1] = n[i].y; xyz[3 * i + 2] = n[i].z; }
}

int scGetLastError(void)
{
    int e = last_error();
    set_error(SC_OK, "");
    return e;
}
const char* scGetLastErrorString(void) { return last_error_string(); }

int scGetStatus(scClothPatch p)
{
    if (!P(p) || !P(p)->model.dc.status) return 0;
    P(p)->sync();
    int s = 0;
    cudaMemcpy(&s, P(p)->model.dc.status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemset(P(p)->model.dc.status, 0, sizeof(int));
    return s;
}

void scSynchronize(scClothPatch p) { if (P(p)) P(p)->sync(); }

void* scGetCudaStream(scClothPatch p) { return P(p) ? (void*)P(p)->stream : nullptr; }

void scSetDirectLaunch(scClothPatch p, int on)
{
    if (!P(p)) { set_error(SC_ERR_ARG, "null patch"); return; }
    P(p)->sync();
    P(p)->directLaunch = on != 0;
}
int scGetGraphKernelCount(scClothPatch p)
{
    if (!P(p) || !P(p)->graph) return 0;
    return P(p)->graphKernelCount;
}

bool scSetKernelTiming(scClothPatch p, int frames)
{
    ClothPatch* cp = P(p);
    if (!cp || frames < 0) { set_error(SC_ERR_ARG, "bad timing request"); return false; }
    return cp->set_timing(frames);
}

int scGetKernelTiming(scClothPatch p, float* ms, int* counts)
{
    ClothPatch* cp = P(p);
    if (!cp) return 0;
    return cp->read_timing(ms, counts);
}

float scProbeClusterPhase(int kind, int phases)
{
    if ((kind != 0 && kind != 1) || phases < 1 || phases > 10000000)
    {
        set_error(SC_ERR_ARG, "probe kind must be 0 or 1, phases 1 .. 1e7");
        return -1.f;
    }
    const float us = probe_cluster_phase(kind, phases);
    if (us < 0.f) set_error(SC_ERR_UNSUPPORTED, "no thread-block cluster of the solver's size fits on this device");
    return us;
}

float scProfileSweep(scClothPatch p, int kind, int reps)
{
    ClothPatch* cp = P(p);
    if (!cp || cp->model.N == 0 || reps < 1) { set_error(SC_ERR_ARG, "bad profile request"); return -1.f; }
    ClothModel& m = cp->model;
    cp->sync();
    const SolverParams P0 = m.solver_params(1.f / 480.f);
    cudaStream_t s = cp->stream;
    cudaGraph_t g;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1.f;
    for (int r = 0; r < reps; r++)
    {
        if (kind == 0)
            for (size_t c = 0; c + 1 < m.triColourStart.size(); c++)
                launch_fem(s, m.dc, P0, m.triColourStart[c], m.triColourStart[c + 1] - m.triColourStart[c]);
        else
            for (size_t c = 0; c + 1 < m.bendColourStart.size(); c++)
                launch_bends(s, m.dc, P0, m.bendColourStart[c], m.bendColourStart[c + 1] - m.bendColourStart[c], 0);
    }
    if (cudaStreamEndCapture(s, &g) != cudaSuccess) return -1.f;
    cudaGraphExec_t ge;
    if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) { cudaGraphDestroy(g); return -1.f; }
    cudaGraphDestroy(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaGraphLaunch(ge, s);                 // warm-up
    cudaEventRecord(e0, s);
    cudaGraphLaunch(ge, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaGraphExecDestroy(ge);
    cp->hostStateDirty = true;
    return ms / reps;
}

} // extern "C"
