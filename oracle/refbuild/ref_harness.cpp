/*
 * ref_harness.cpp — C entry points over the UNMODIFIED SolidCloth reference
 * classes (Physics/ClothPatch, Physics/ClothModel, Physics/SelfCollisionDetector),
 * compiled from the reference's own sources into oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY. Used by tests/ (to pin the CPU restatement in
 * oracle/cloth_oracle.cpp and to produce golden vectors) and by bench.py's
 * reference arm (to time the reference's own CPU step). Never linked into the
 * shipped library.
 *
 * The reference ships a C ABI (Demo/ClothAPI.cpp) that does not compile with g++
 * (it binds an rvalue shared_ptr to a non-const reference, Demo/ClothAPI.cpp:42
 * -> Physics/CollisionWorld.h:18), so this harness calls the C++ classes the
 * same way Demo/ClothAPI.cpp does. Member access is opened in this translation
 * unit only so that the harness can read contact lists and set the one knob
 * that has no setter (mSelfCollThreshold, Physics/ClothModel.h:196).
 */
#define private public
#define protected public
#include "Physics/ClothPatch.h"
#include "Physics/ClothPBD.h"
#include "Physics/ClothModel.h"
#include "Physics/CollisionWorld.h"
#include "Physics/Common.h"
#include "Physics/SelfCollisionDetector.h"
#include "Geometry/SDF.h"
#include "Geometry/Mesh.h"
#undef private
#undef protected

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace Physics;
using namespace Geometry;
using namespace Math;

struct RefScene
{
    CollisionWorld world;
    ClothPatch* patch = nullptr;
    std::vector<SDF*> sdfs;
    std::vector<Mesh*> meshes;
    SelfCollisionsDetector ccd;
    bool ccdInStep = false;
    ~RefScene()
    {
        delete patch;
        world.ClearCollidables();
        for (SDF* s : sdfs) delete s;
        for (Mesh* m : meshes) delete m;
    }
};

static ClothModelPBD& Model(RefScene* s) { return *(ClothModelPBD*)s->patch->GetModelPtr(); }

extern "C" {

void* ref_create()
{
    RefScene* s = new RefScene();
    s->patch = new ClothPatch(s->world);
    s->ccd.SetClothModel(s->patch->GetModelPtr());
    return s;
}

void ref_destroy(void* h) { delete (RefScene*)h; }

#ifdef _OPENMP
void ref_set_threads(int n) { omp_set_num_threads(n); }
int ref_max_threads() { return omp_get_max_threads(); }
#else
// the single-threaded build (no -fopenmp), like the reference's C-ABI library
void ref_set_threads(int) {}
int ref_max_threads() { return 1; }
#endif

/* ---- colliders (Physics/Common.h:32-149) ---- */
void ref_add_walls(void* h, const float* box6)
{
    RefScene* s = (RefScene*)h;
    std::shared_ptr<Collidable> c(new Walls(Aabb3(Vector3(box6[0], box6[1], box6[2]), Vector3(box6[3], box6[4], box6[5]))));
    s->world.AddCollidable(c);
}

void ref_add_sphere(void* h, float cx, float cy, float cz, float r)
{
    RefScene* s = (RefScene*)h;
    std::shared_ptr<Collidable> c(new Sphere(Vector3(cx, cy, cz), r));
    s->world.AddCollidable(c);
}

/* values: (nx+1)(ny+1)(nz+1) floats, x fastest (Geometry/SDF.h:49-52). */
void ref_add_sdf(void* h, int nx, int ny, int nz, const float* box6, const float* values)
{
    RefScene* s = (RefScene*)h;
    SDF* sdf = new SDF();
    sdf->Create(nx, ny, nz, Aabb3(Vector3(box6[0], box6[1], box6[2]), Vector3(box6[3], box6[4], box6[5])));
    std::vector<float>& d = sdf->GetData();
    for (size_t i = 0; i < d.size(); i++) d[i] = values[i];
    sdf->ComputeGradient();
    s->sdfs.push_back(sdf);
    std::shared_ptr<Collidable> c(new CollisionSDF(sdf));
    s->world.AddCollidable(c);
}

/* Triangle-mesh collider, prepared as in Demo/ClothDemo.cpp:100-103. */
void ref_add_mesh(void* h, int nv, const float* verts, int nt, const unsigned* idx)
{
    RefScene* s = (RefScene*)h;
    Mesh* m = new Mesh();
    m->vertices.resize(nv);
    for (int i = 0; i < nv; i++) m->vertices[i] = Vector3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    m->indices.assign(idx, idx + 3 * nt);
    m->ComputeNormals();
    m->ConstructEdges();
    m->ConstructEdgeOneRings();
    s->meshes.push_back(m);
    std::shared_ptr<Collidable> c(new CollisionMesh(m));
    s->world.AddCollidable(c);
}

/* SDF::Create + SDF::CreateFromMesh (Geometry/SDF.cpp:10-18,58-76) over a triangle
   mesh; out gets (nx+1)(ny+1)(nz+1) values, x fastest. */
void ref_sdf_from_mesh(int nv, const float* verts, int nt, const unsigned* idx, int nx, int ny, int nz,
                       const float* box6, float* out)
{
    Mesh m;
    m.vertices.resize(nv);
    for (int i = 0; i < nv; i++) m.vertices[i] = Vector3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    m.indices.assign(idx, idx + 3 * nt);
    SDF sdf;
    sdf.Create(nx, ny, nz, Aabb3(Vector3(box6[0], box6[1], box6[2]), Vector3(box6[3], box6[4], box6[5])));
    sdf.CreateFromMesh(m);
    const std::vector<float>& d = sdf.GetData();
    for (size_t i = 0; i < d.size(); i++) out[i] = d[i];
}

/* SDF::WriteToFile / SDF::LoadFromFile (Geometry/SDF.cpp:78-151) */
void ref_sdf_write(int nx, int ny, int nz, const float* box6, const float* values, const char* path)
{
    SDF sdf;
    sdf.Create(nx, ny, nz, Aabb3(Vector3(box6[0], box6[1], box6[2]), Vector3(box6[3], box6[4], box6[5])));
    std::vector<float>& d = sdf.GetData();
    for (size_t i = 0; i < d.size(); i++) d[i] = values[i];
    sdf.WriteToFile(path);
}

int ref_sdf_read(const char* path, int* cells3, float* box6, float* values, int cap)
{
    SDF sdf;
    sdf.LoadFromFile(path);
    const std::vector<float>& d = sdf.GetData();
    Aabb3 b = sdf.GetBox();
    if (box6) { box6[0] = b.min.x; box6[1] = b.min.y; box6[2] = b.min.z; box6[3] = b.max.x; box6[4] = b.max.y; box6[5] = b.max.z; }
    if (cells3) sdf.GetNumCellsPerSide(cells3);
    for (size_t i = 0; values && i < d.size() && (int)i < cap; i++) values[i] = d[i];
    return (int)d.size();
}

/* ClothPatch::Init(mesh, offset, attached) (Physics/ClothPatch.cpp:42-133): the
   cloth from a triangle mesh; uvs (nv x 2) and colors (nv x 3) may be null. */
void ref_init_mesh(void* h, int nv, const float* verts, int ni, const unsigned* idx, const float* uvs,
                   const float* colors, float ox, float oy, float oz, int attached)
{
    RefScene* s = (RefScene*)h;
    Mesh m;
    m.vertices.resize(nv);
    for (int i = 0; i < nv; i++) m.vertices[i] = Vector3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    m.indices.assign(idx, idx + ni);
    if (uvs) { m.uvs.resize(nv); for (int i = 0; i < nv; i++) m.uvs[i] = Vector2(uvs[2 * i], uvs[2 * i + 1]); }
    if (colors) { m.colors.resize(nv); for (int i = 0; i < nv; i++) m.colors[i] = Vector3(colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]); }
    s->patch->Init(m, Vector3(ox, oy, oz), attached != 0);
}

void ref_get_links(void* h, unsigned* idx2, float* lenStiff)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.GetNumLinks(); i++)
    {
        const Physics::Link& l = m.GetLink(i);
        if (idx2) { idx2[2 * i] = l.i1; idx2[2 * i + 1] = l.i2; }
        if (lenStiff) { lenStiff[2 * i] = l.len; lenStiff[2 * i + 1] = l.stiffness; }
    }
}

/* ---- cloth ---- */
void ref_init_grid(void* h, int divX, int divY, float inc, float ox, float oy, float oz, int horizontal, int attached)
{
    RefScene* s = (RefScene*)h;
    s->patch->Init(divX, divY, inc, Vector3(ox, oy, oz), horizontal != 0, attached != 0);
}

void ref_set_params(void* h, const float* p, int n)
{
    /* p: unit, thickness, tolerance, shear, bend, stretch, poisson, friction,
          iterations, substeps, collFlags, fem, dihedral, fixedIterations, drag */
    RefScene* s = (RefScene*)h;
    ClothModel& m = Model(s);
    if (n < 15) return;
    m.SetUnit(p[0]);
    m.SetThickness(p[1]);
    m.SetTolerance(p[2]);
    m.SetShearStiffness(p[3]);
    m.SetBendStiffness(p[4]);
    m.SetStretchStiffness(p[5]);
    m.SetPoisson(p[6]);
    m.SetFriction(p[7]);
    m.SetNumIterations((int)p[8]);
    s->patch->SetNumSteps((int)p[9]);
    m.SetCollisionFlags((int)p[10]);
    m.SetFEM(p[11] != 0);
    m.SetDihedral(p[12] != 0);
    /* Fixed-iteration mode: the GS exit test (Physics/ClothPBD.cpp:357) requires
       selfEE < mSelfCollThreshold; errors are >= 0, so a negative threshold means
       the loop always runs mNumIterations times. */
    m.mSelfCollThreshold = p[13] != 0 ? -1.f : 0.003f;
    m.SetDragCoeff(p[14]);
}

void ref_set_ccd(void* h, int on) { ((RefScene*)h)->ccdInStep = on != 0; }

int ref_num_particles(void* h) { return (int)Model((RefScene*)h).GetNumParticles(); }
int ref_num_tris(void* h) { return (int)Model((RefScene*)h).GetNumTris(); }
int ref_num_bends(void* h) { return (int)Model((RefScene*)h).mBends.size(); }
int ref_num_edges(void* h) { return (int)Model((RefScene*)h).mEdges.size(); }
int ref_num_links(void* h) { return (int)Model((RefScene*)h).GetNumLinks(); }

/* pos and prev are set together (a freshly initialised patch has prev == pos). */
void ref_set_positions(void* h, const float* pos)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.GetNumParticles(); i++)
    {
        Particle& p = m.GetParticle(i);
        p.pos = Vector3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        p.prev = p.pos;
    }
}

void ref_set_state(void* h, const float* pos, const float* prev, const float* vel)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.GetNumParticles(); i++)
    {
        Particle& p = m.GetParticle(i);
        p.pos = Vector3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        p.prev = Vector3(prev[3 * i], prev[3 * i + 1], prev[3 * i + 2]);
        p.vel = Vector3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
}

void ref_set_masses(void* h, const float* masses) { Model((RefScene*)h).SetMasses(masses); }

void ref_set_inv_mass(void* h, int i, float w) { Model((RefScene*)h).GetParticle(i).invMass = w; }

void ref_get_state(void* h, float* pos, float* prev, float* vel, float* invMass)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.GetNumParticles(); i++)
    {
        const Particle& p = m.GetParticle(i);
        for (int k = 0; k < 3; k++)
        {
            if (pos) pos[3 * i + k] = p.pos[k];
            if (prev) prev[3 * i + k] = p.prev[k];
            if (vel) vel[3 * i + k] = p.vel[k];
        }
        if (invMass) invMass[i] = p.invMass;
    }
}

/* Topology and FEM rest data: tris 3 u32 each; rest 9 floats each
   (du1, du2, dv1, dv2, invDet, lu0, lv0, lu2, lv2) plus area. */
void ref_get_tris(void* h, unsigned* idx, float* rest10)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.GetNumTris(); i++)
    {
        const Physics::Triangle& t = m.GetTriangle(i);
        idx[3 * i] = t.i1; idx[3 * i + 1] = t.i2; idx[3 * i + 2] = t.i3;
        if (rest10)
        {
            float* r = rest10 + 10 * i;
            r[0] = t.du1; r[1] = t.du2; r[2] = t.dv1; r[3] = t.dv2; r[4] = t.invDet;
            r[5] = t.lu0; r[6] = t.lv0; r[7] = t.lu2; r[8] = t.lv2; r[9] = t.area;
        }
    }
}

void ref_get_bends(void* h, unsigned* idx)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.mBends.size(); i++)
    {
        idx[4 * i] = m.mBends[i].i1; idx[4 * i + 1] = m.mBends[i].i2;
        idx[4 * i + 2] = m.mBends[i].i3; idx[4 * i + 3] = m.mBends[i].i4;
    }
}

/* edges: i1, i2, t1, t2 per edge (Geometry/Mesh.h:15-25) */
void ref_get_edges(void* h, int* e4)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.mEdges.size(); i++)
    {
        e4[4 * i] = (int)m.mEdges[i].i1; e4[4 * i + 1] = (int)m.mEdges[i].i2;
        e4[4 * i + 2] = m.mEdges[i].t1; e4[4 * i + 3] = m.mEdges[i].t2;
    }
}

/* The render mesh index buffer (grid meshes share vertex numbering with particles). */
int ref_mesh_index_count(void* h) { return (int)((RefScene*)h)->patch->GetMesh().indices.size(); }
void ref_get_mesh_indices(void* h, unsigned* idx)
{
    const Mesh& mesh = ((RefScene*)h)->patch->GetMesh();
    for (size_t i = 0; i < mesh.indices.size(); i++) idx[i] = mesh.indices[i];
}
void ref_get_mesh_normals(void* h, int prev, float* n)
{
    RefScene* s = (RefScene*)h;
    const Mesh& mesh = prev ? *s->patch->GetPrevMesh() : s->patch->GetMesh();
    for (size_t i = 0; i < mesh.normals.size(); i++)
        for (int k = 0; k < 3; k++) n[3 * i + k] = mesh.normals[i][k];
}
void ref_get_mesh_tri_normals(void* h, int prev, float* n)
{
    RefScene* s = (RefScene*)h;
    const Mesh& mesh = prev ? *s->patch->GetPrevMesh() : s->patch->GetMesh();
    for (size_t i = 0; i < mesh.triangles.size(); i++)
        for (int k = 0; k < 3; k++) n[3 * i + k] = mesh.triangles[i].n[k];
}

/* ---- stepping ---- */
void ref_step(void* h, float dt)
{
    RefScene* s = (RefScene*)h;
    if (!s->ccdInStep)
    {
        s->patch->Step(dt);
        return;
    }
    /* Same substep as ClothPatch::Step -> ClothModelPBD::Step
       (Physics/ClothPatch.cpp:323-335, Physics/ClothPBD.cpp:255-322) with the
       dead continuous detector run right after DetectCollisions, appending its
       contacts to mSelfTris/mSelfEdges as its Detect() was written to do. */
    ClothModelPBD& m = Model(s);
    const int n = s->patch->GetNumSteps();
    const float hh = dt / n;
    for (int k = 0; k < n; k++)
    {
        for (size_t i = 0; i < m.mParticles.size(); i++)
        {
            m.mParticles[i].prev = m.mParticles[i].pos;
            if (m.mParticles[i].invMass == 0)
                continue;
            m.mParticles[i].vel += hh * gravity * m.mUnit;
            m.mParticles[i].vel *= m.mDragCoeff;
            m.mParticles[i].pos += hh * m.mParticles[i].vel;
        }
        m.DetectCollisions();
        s->ccd.Detect();
        m.ResetConstraints();
        m.SolveGS(hh);
        const float invH = 1.f / hh;
        for (size_t i = 0; i < m.mParticles.size(); i++)
        {
            if (m.mParticles[i].invMass == 0)
                continue;
            m.mParticles[i].vel = invH * (m.mParticles[i].pos - m.mParticles[i].prev);
        }
    }
}

void ref_update_mesh(void* h) { ((RefScene*)h)->patch->UpdateMesh(); }

/* Predict (Physics/ClothPBD.cpp:257-266) followed by DetectCollisions only, so
   that detection outputs can be read before the solver rewrites them. */
void ref_predict_detect(void* h, float hh, int runCCD)
{
    RefScene* s = (RefScene*)h;
    ClothModelPBD& m = Model(s);
    for (size_t i = 0; i < m.mParticles.size(); i++)
    {
        m.mParticles[i].prev = m.mParticles[i].pos;
        if (m.mParticles[i].invMass == 0)
            continue;
        m.mParticles[i].vel += hh * gravity * m.mUnit;
        m.mParticles[i].vel *= m.mDragCoeff;
        m.mParticles[i].pos += hh * m.mParticles[i].vel;
    }
    m.DetectCollisions();
    if (runCCD)
        s->ccd.Detect();
}

/* ClothModel::SetSolver (Physics/ClothModel.h:138): the SolverType of ClothModelPBD::Step */
void ref_set_solver(void* h, int type) { Model((RefScene*)h).SetSolver((SolverType)type); }
int ref_solver_iterations(void* h) { return Model((RefScene*)h).mStats.iterations; }

/* ---- contact lists ---- */
int ref_num_contacts(void* h, int kind)
{
    ClothModel& m = Model((RefScene*)h);
    switch (kind)
    {
    case 0: return (int)m.mContacts.size();
    case 1: return (int)m.mTriContacts.size();
    case 2: return (int)m.mEdgeContacts.size();
    case 3: return (int)m.mSelfTris.size();
    case 4: return (int)m.mSelfEdges.size();
    }
    return 0;
}

/* Vertex contacts: idx, feature; point(3), normal(3), depth */
void ref_get_vertex_contacts(void* h, int* idx2, float* f7)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.mContacts.size(); i++)
    {
        const Contact& c = m.mContacts[i];
        idx2[2 * i] = (int)c.idx; idx2[2 * i + 1] = c.feature;
        for (int k = 0; k < 3; k++) { f7[7 * i + k] = c.point[k]; f7[7 * i + 3 + k] = c.normal[k]; }
        f7[7 * i + 6] = c.depth;
    }
}

/* Tri contacts: i1 i2 i3 feature; point(3) normal(3) w(3) */
void ref_get_tri_contacts(void* h, int* idx4, float* f9)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.mTriContacts.size(); i++)
    {
        const TriContact& c = m.mTriContacts[i];
        idx4[4 * i] = c.i1; idx4[4 * i + 1] = c.i2; idx4[4 * i + 2] = c.i3; idx4[4 * i + 3] = c.feature;
        for (int k = 0; k < 3; k++) { f9[9 * i + k] = c.point[k]; f9[9 * i + 3 + k] = c.normal[k]; }
        f9[9 * i + 6] = c.w1; f9[9 * i + 7] = c.w2; f9[9 * i + 8] = c.w3;
    }
}

/* Edge contacts: i1 i2 feature; point(3) normal(3) w(2) */
void ref_get_edge_contacts(void* h, int* idx3, float* f8)
{
    ClothModel& m = Model((RefScene*)h);
    for (size_t i = 0; i < m.mEdgeContacts.size(); i++)
    {
        const EdgeContact& c = m.mEdgeContacts[i];
        idx3[3 * i] = c.i1; idx3[3 * i + 1] = c.i2; idx3[3 * i + 2] = c.feature;
        for (int k = 0; k < 3; k++) { f8[8 * i + k] = c.point[k]; f8[8 * i + 3 + k] = c.normal[k]; }
        f8[8 * i + 6] = c.w1; f8[8 * i + 7] = c.w2;
    }
}

/* Self contacts (kind 3 = VT, 4 = EE): i1..i4; normal(3) w1 w2 w3 side */
void ref_get_self_contacts(void* h, int kind, int* idx4, float* f7)
{
    ClothModel& m = Model((RefScene*)h);
    const std::vector<SelfContact>& v = kind == 3 ? m.mSelfTris : m.mSelfEdges;
    for (size_t i = 0; i < v.size(); i++)
    {
        const SelfContact& c = v[i];
        idx4[4 * i] = c.i1; idx4[4 * i + 1] = c.i2; idx4[4 * i + 2] = c.i3; idx4[4 * i + 3] = c.i4;
        for (int k = 0; k < 3; k++) f7[7 * i + k] = c.normal[k];
        f7[7 * i + 3] = c.w1; f7[7 * i + 4] = c.w2; f7[7 * i + 5] = c.w3; f7[7 * i + 6] = c.side;
    }
}

/* ---- continuous self-collision detector (dead in the reference build) ---- */
void ref_ccd_midphase(void* h) { ((RefScene*)h)->ccd.Midphase(); }
int ref_ccd_num_candidates(void* h, int kind)
{
    RefScene* s = (RefScene*)h;
    return (int)(kind == 0 ? s->ccd.mVertexTriangleCandidates.size() : s->ccd.mEdgeEdgeCandidates.size());
}
void ref_ccd_get_candidates(void* h, int kind, int* pairs)
{
    RefScene* s = (RefScene*)h;
    const auto& v = kind == 0 ? s->ccd.mVertexTriangleCandidates : s->ccd.mEdgeEdgeCandidates;
    for (size_t i = 0; i < v.size(); i++) { pairs[2 * i] = v[i].idx1; pairs[2 * i + 1] = v[i].idx2; }
}
/* Replace the candidate lists, clear the self lists and run the narrow phase
   (Physics/SelfCollisionDetector.cpp:137-169) on exactly these pairs. */
void ref_ccd_narrow_on(void* h, int nvt, const int* vt, int nee, const int* ee)
{
    RefScene* s = (RefScene*)h;
    ClothModel& m = Model(s);
    s->ccd.mVertexTriangleCandidates.resize(nvt);
    for (int i = 0; i < nvt; i++) { s->ccd.mVertexTriangleCandidates[i].idx1 = vt[2 * i]; s->ccd.mVertexTriangleCandidates[i].idx2 = vt[2 * i + 1]; }
    s->ccd.mEdgeEdgeCandidates.resize(nee);
    for (int i = 0; i < nee; i++) { s->ccd.mEdgeEdgeCandidates[i].idx1 = ee[2 * i]; s->ccd.mEdgeEdgeCandidates[i].idx2 = ee[2 * i + 1]; }
    m.mSelfTris.clear();
    m.mSelfEdges.clear();
    s->ccd.Narrowphase();
}

/* Swept boxes of the cloth tree root lists (Physics/ClothCollision.cpp:240-321)
   before splitting is not retained by the reference; this rebuilds the tree with
   maxLevel 0 and reads the root's box lists. kind 0 = triangles, 1 = vertices,
   2 = edges; out: 6 floats per primitive (min, max). */
void ref_swept_boxes(void* h, int kind, float tol, float* out)
{
    ClothModel& m = Model((RefScene*)h);
    m.ComputeTree(ATF_VERTICES | ATF_TRIANGLES | ATF_EDGES, 0, tol);
    const std::vector<BoxInfo>& v = kind == 0 ? m.mTree->triangles : (kind == 1 ? m.mTree->vertices : m.mTree->edges);
    for (size_t i = 0; i < v.size(); i++)
        for (int k = 0; k < 3; k++) { out[6 * i + k] = v[i].box.min[k]; out[6 * i + 3 + k] = v[i].box.max[k]; }
}

}
