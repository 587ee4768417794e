// solver.cuh — the Gauss-Seidel loop of one substep: the constraint
// projections (FEM triangles, dihedral bends, links), the contact solves, the
// one-kernel-per-colour path and the two persistent solvers (cluster-resident
// and grid-resident), with their host launchers.
//
// This file is included twice, each time inside a namespace:
//   * step_kernels.cu, namespace sc — compiled with -fmad=false and IEEE
//     division and square root, so every projection follows the reference's
//     operation order bit for bit (the check-mode build);
//   * solver_fast.cu, namespace sc::fast — the same source compiled with FMA
//     contraction and approximate division / square root (div.full,
//     sqrt.approx): shorter dependent chains per projection, results within
//     a few ulp of the IEEE build per operation.
// The detection kernels (boxes, pairs, continuous-collision hits, contact
// lists) exist only in the IEEE build, so candidate pairs and contacts are
// bit-exact whichever solver runs.
// (no include guard: one copy per namespace)

// ------------------------------------------------------------ FEM sweep
// ClothModelPBD::SolveTriangles for the triangles of one colour
// (Physics/ClothPBD.cpp:52-108): warp and weft hard, shear compliant.
template <class PA>
__device__ __forceinline__ void fem_project(const PA& pa, float4 r0, float4 r1, float4 r2, const SolverParams& P)
{
    const uint32_t i1 = __float_as_uint(r0.x), i2 = __float_as_uint(r0.y), i3 = __float_as_uint(r0.z);
    const float du1 = r0.w, du2 = r1.x, dv1 = r1.y, dv2 = r1.z, invDet = r1.w;
    const float lu2 = r2.x, lv2 = r2.y, lu0lv0 = r2.z, area = r2.w;
    float4 a = pa.ld(i1), b = pa.ld(i2), d = pa.ld(i3);
    V3 x1 = mk(a.x, a.y, a.z), x2 = mk(b.x, b.y, b.z), x3 = mk(d.x, d.y, d.z);
    const float w1 = a.w, w2 = b.w, w3 = d.w;
    V3 dx1 = x2 - x1, dx2 = x3 - x1;
    V3 wu = invDet * (dv2 * dx1 - dv1 * dx2);
    V3 wv = invDet * (-du2 * dx1 + du1 * dx2);
    float err, diag, lambda;
    V3 q1, q2, q3;
    // warp
    q2 = (invDet * dv2) * wu;
    q3 = (-invDet * dv1) * wu;
    q1 = -q2 - q3;
    diag = dot(w1 * q1, q1) + dot(w2 * q2, q2) + dot(w3 * q3, q3);
    err = 0.5f * (dot(wu, wu) - lu2);
    lambda = -err / diag;
    x1 += (w1 * lambda) * q1; x2 += (w2 * lambda) * q2; x3 += (w3 * lambda) * q3;
    // weft
    q2 = (-invDet * du2) * wv;
    q3 = (invDet * du1) * wv;
    q1 = -q2 - q3;
    diag = dot(w1 * q1, q1) + dot(w2 * q2, q2) + dot(w3 * q3, q3);
    err = 0.5f * (dot(wv, wv) - lv2);
    lambda = -err / diag;
    x1 += (w1 * lambda) * q1; x2 += (w2 * lambda) * q2; x3 += (w3 * lambda) * q3;
    // shear
    q2 = dv2 * wv - du2 * wu;
    q3 = -dv1 * wv + du1 * wu;
    q1 = -q2 - q3;
    diag = invDet * (dot(w1 * q1, q1) + dot(w2 * q2, q2) + dot(w3 * q3, q3));
    err = dot(wu, wv);
    float s = 1.f / (1.f + lu0lv0 * P.epsUV / (diag * P.h2 * area));
    lambda = -s * err / diag;
    x1 += (w1 * lambda) * q1; x2 += (w2 * lambda) * q2; x3 += (w3 * lambda) * q3;
    pa.st(i1, make_float4(x1.x, x1.y, x1.z, w1));
    pa.st(i2, make_float4(x2.x, x2.y, x2.z, w2));
    pa.st(i3, make_float4(x3.x, x3.y, x3.z, w3));
}

// SolveLinks (Physics/ClothPBD.cpp:9-50), omega = 1, for one link record
// {i1, i2 (bits), rest length, stiffness}; returns |s err| or -1 when skipped
template <class PA>
__device__ __forceinline__ float link_project(const PA& pa, float4 rec, const SolverParams& P)
{
    const uint32_t i1 = __float_as_uint(rec.x), i2 = __float_as_uint(rec.y);
    float4 a = pa.ld(i1), b = pa.ld(i2);
    const float w1 = a.w, w2 = b.w;
    if (w1 + w2 == 0) return -1.f;
    const float mu = 1.f / (w1 + w2);
    V3 delta = mk(a.x, a.y, a.z) - mk(b.x, b.y, b.z);
    const float len0 = rec.z;
    const float l = len(delta);
    if (l == 0 || isnan(l) || isinf(l)) return -1.f;
    const float err = l - len0;
    delta = (1 / l) * delta;
    const float k = P.h2 * P.area * P.unit;
    const float epsilon = len0 / (k * rec.w);
    const float s = 1.f / (1.f + mu * epsilon);
    const float lambda = err * mu * s;
    const float omega = 1.f;
    const V3 fc = omega * lambda * delta;
    const V3 x1 = mk(a.x, a.y, a.z) - w1 * fc, x2 = mk(b.x, b.y, b.z) + w2 * fc;
    pa.st(i1, make_float4(x1.x, x1.y, x1.z, w1));
    pa.st(i2, make_float4(x2.x, x2.y, x2.z, w2));
    return fabsf(s * err);
}

__global__ void __launch_bounds__(256) k_links(DevCloth c, SolverParams P, int first, int count)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count || gs_done(c)) return;
    const float e = link_project(GlobalPos{c.pos}, c.link[first + k], P);
    if (!P.fixedIterations && e > 0.f) atomic_max_pos(&c.scal[1], e);
}

__global__ void __launch_bounds__(256) k_fem(DevCloth c, SolverParams P, int first, int count)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count || gs_done(c)) return;
    k += first;
    fem_project(GlobalPos{c.pos}, c.fem[3 * k], c.fem[3 * k + 1], c.fem[3 * k + 2], P);
}

// ---------------------------------------------------------- bend sweep
// SolveBends + EvaluateAngle + EvaluateGradient for one colour
// (Physics/ClothPBD.cpp:110-224).
// returns |error| of the projection, or -1 when the bend is skipped
template <class PA>
__device__ __forceinline__ float bend_project(const PA& pa, uint4 bc, const SolverParams& P)
{
    float4 a = pa.ld(bc.x), b = pa.ld(bc.y), d = pa.ld(bc.z), e = pa.ld(bc.w);
    const float m1 = a.w, m2 = b.w, m3 = d.w, m4 = e.w;
    if (m1 + m2 + m3 + m4 == 0) return -1.f;
    V3 x1 = mk(a.x, a.y, a.z), x2 = mk(b.x, b.y, b.z), x3 = mk(d.x, d.y, d.z), x4 = mk(e.x, e.y, e.z);
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
        cosine = mn(1.f, mx(-1.f, cosine));
        theta = portable_acos(cosine);
    }
    if (fabsf(cosine) >= 1 - 0.001f) return -1.f;
    float h1 = l1 / l, h2 = l2 / l;
    float he = 0.5f * (h1 + h2);
    float il1 = 1.f / l1, il2 = 1.f / l2;
    V3 n1n = il1 * n1, n2n = il2 * n2;
    V3 n1p = n1n - n2n * cosine;
    V3 n2p = n2n - n1n * cosine;
    float sine = sqrtf(1 - cosine * cosine);
    V3 q3 = (il1 / sine / he) * cross(x12, n2p);
    V3 q4 = (-il2 / sine / he) * cross(x12, n1p);
    V3 q2 = (-il1 / sine / he) * cross(x13, n2p) + (il2 / sine / he) * cross(x14, n1p);
    V3 q1 = -q2 - q3 - q4;
    float diag = m1 * lensq(q1) + m2 * lensq(q2) + m3 * lensq(q3) + m4 * lensq(q4);
    if (diag == 0) return -1.f;
    float s = 0.0005f * P.bend;
    float errv = fabsf(s * theta);
    float lambda = -s * theta / he / diag;
    x1 += (lambda * m1) * q1; x2 += (lambda * m2) * q2; x3 += (lambda * m3) * q3; x4 += (lambda * m4) * q4;
    pa.st(bc.x, make_float4(x1.x, x1.y, x1.z, m1));
    pa.st(bc.y, make_float4(x2.x, x2.y, x2.z, m2));
    pa.st(bc.z, make_float4(x3.x, x3.y, x3.z, m3));
    pa.st(bc.w, make_float4(x4.x, x4.y, x4.z, m4));
    return errv;
}

__global__ void __launch_bounds__(256) k_bends(DevCloth c, SolverParams P, int first, int count)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count || gs_done(c)) return;
    float errv = bend_project(GlobalPos{c.pos}, c.bend[first + k], P);
    if (!P.fixedIterations && errv >= 0.f) atomic_max_pos(&c.scal[2], errv);
}

// --------------------------------------------------------- contact solves
// Data that no solver kernel writes (the collider meshes, the contact slots'
// collider ranges and counts, the colour orders, the start-of-substep
// positions) is read through the non-coherent path, so that it stays in L1
// across the colour phases and iterations: in a contact phase only the contact
// record and the particles then pay the L2 latency.
__device__ __forceinline__ V3 ldg3(const float4* p, uint32_t i) { const float4 a = __ldg(&p[i]); return mk(a.x, a.y, a.z); }
template <typename T>
__device__ __forceinline__ const T* ldg_ptr(const T* const* p)
{
    return reinterpret_cast<const T*>(__ldg(reinterpret_cast<const unsigned long long*>(p)));
}
// the fields of collider mesh k the contact solves read
struct MeshView { const float4* v; const float4* n; const uint32_t* tri; const int4* edge; };
__device__ __forceinline__ MeshView mesh_view(const Buffers& b, int k)
{
    const DevMesh* m = b.meshes + k;
    return MeshView{ldg_ptr(&m->v), ldg_ptr(&m->n), ldg_ptr(&m->tri), ldg_ptr(&m->edge)};
}

// ComputeTriangleNormal(mesh, tri, coords, false): vertex normals blended by the
// barycentric coordinates (Geometry/ClosestPointOnMesh.cpp:37-60).
__device__ __forceinline__ V3 blended_normal(const MeshView& m, int t, V3 w)
{
    V3 n0 = ldg3(m.n, __ldg(&m.tri[3 * t])), n1 = ldg3(m.n, __ldg(&m.tri[3 * t + 1])), n2 = ldg3(m.n, __ldg(&m.tri[3 * t + 2]));
    return normalized(w.x * n0 + w.y * n1 + w.z * n2);
}

// SolveContactsPosition (Physics/ClothCollisionHandler.cpp:134-202): one thread
// per particle processes that particle's contacts in list order (collider, slot),
// which equals the reference's sequential order because every vertex contact
// moves a single particle.
template <class PA>
__device__ __forceinline__ float vertex_contacts_one(const PA& pa, const DevCloth& c, const SolverParams& P, const Buffers& b, int i)
{
    float err = 0.f;
    float4 p4 = pa.ld(i);
    V3 p = mk(p4.x, p4.y, p4.z);
    const V3 q = ldg3(c.prev, i);
    bool touched = false;
    const int2 cr = colliders_of(c, b, i);
    for (int ci = cr.x; ci < cr.x + cr.y; ci++)
    {
        const VColl& g = b.vcoll[ci];
        const int n = __ldg(&b.vcCount[(size_t)__ldg(&g.countBase) + (i - __ldg(&g.vBegin))]);
        VC* slot = b.vc + g.slotBase + (size_t)(i - g.vBegin) * g.kmax;
        for (int k = 0; k < n; k++)
        {
            VC v = slot[k];
            V3 point = mk(v.point.x, v.point.y, v.point.z), normal = mk(v.normal.x, v.normal.y, v.normal.z);
            if (v.mesh >= 0)
            {
                const MeshView m = mesh_view(b, v.mesh);
                int t = v.feature;
                V3 coords, cp;
                closest_point_triangle(p, ldg3(m.v, __ldg(&m.tri[3 * t])), ldg3(m.v, __ldg(&m.tri[3 * t + 1])),
                                       ldg3(m.v, __ldg(&m.tri[3 * t + 2])), cp, coords);
                point = cp;
                normal = blended_normal(m, t, coords);
                v.point = f4(point, 0.f); v.normal = f4(normal, 0.f);
            }
            V3 delta = p - point;
            float l = dot(delta, normal);
            V3 disp = normal;
            if (l > P.thickness) { slot[k] = v; continue; }
            float depth = P.thickness - l;
            err = mx(err, fabsf(depth));
            float dLambda = depth;
            v.lam.x += dLambda;
            disp = disp * dLambda;
            V3 v12 = p - q - mk(0.f, 0.f, 0.f);
            float vnrel = dot(normal, v12);
            V3 vt = v12 - vnrel * normal;
            float vtrel = len(vt);
            const float limit = P.friction * v.lam.x;
            if (vtrel > 0.001f)
            {
                float dLF = vtrel;
                float l0 = v.lam.y;
                v.lam.y = l0 + dLF;
                if (v.lam.y >= limit) v.lam.y = limit;
                dLF = v.lam.y - l0;
                vt = vt * (1.0f / vtrel);
                disp += -dLF * vt;
            }
            p += disp;
            float4 vv = c.vel[i];
            V3 nv = mk(vv.x, vv.y, vv.z) + P.invH * disp;
            c.vel[i] = make_float4(nv.x, nv.y, nv.z, 0.f);
            touched = true;
            slot[k] = v;
        }
    }
    if (touched) pa.st(i, make_float4(p.x, p.y, p.z, p4.w));
    return err;
}

__global__ void k_solve_vertex_contacts(DevCloth c, SolverParams P, Buffers b)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N || gs_done(c)) return;
    float err = vertex_contacts_one(GlobalPos{c.pos}, c, P, b, i);
    if (!P.fixedIterations && err > 0.f) atomic_max_pos(&c.scal[3], err);
}

// SolveEdgeContacts for one contact (Physics/ClothCollisionHandler.cpp:289-362)
template <class PA>
__device__ float solve_edge_contact(const PA& pa, const DevCloth& c, const SolverParams& P, const Buffers& b, EC& k)
{
    float4 a4 = pa.ld(k.idx.x), b4 = pa.ld(k.idx.y);
    V3 x1 = mk(a4.x, a4.y, a4.z), x2 = mk(b4.x, b4.y, b4.z);
    const float m1 = a4.w, m2 = b4.w;
    float w1 = k.w.x, w2 = k.w.y;
    V3 point = mk(k.point.x, k.point.y, k.point.z), normal = mk(k.normal.x, k.normal.y, k.normal.z);
    V3 p = w1 * x1 + w2 * x2;
    if (k.mesh >= 0)
    {
        const MeshView m = mesh_view(b, k.mesh);
        const int4 ed = __ldg(&m.edge[k.feature]);
        float s1, t;
        closest_segm_segm(ldg3(m.v, ed.x), ldg3(m.v, ed.y), x1, x2, s1, t, point, p);
        w1 = 1.0f - t; w2 = t;
        k.point = f4(point, 0.f);
    }
    k.w.x = w1; k.w.y = w2;
    const float len0 = P.thickness;
    float l = dot(normal, p - point - mk(0.f, 0.f, 0.f));
    if (l > len0) return -1.f;
    float s = 1.f / (w1 * w1 / m1 + w2 * w2 / m2);
    float depth = len0 - l;
    float dLambda = s * depth;
    k.lam.x += dLambda;
    V3 disp = dLambda * normal;
    if (P.friction != 0)
    {
        V3 p0 = w1 * ldg3(c.prev, k.idx.x) + w2 * ldg3(c.prev, k.idx.y);
        V3 v12 = p - p0 - mk(0.f, 0.f, 0.f);
        float vnrel = dot(normal, v12);
        V3 vt = v12 - vnrel * normal;
        float vtrel = len(vt);
        const float limit = P.friction * k.lam.x;
        if (vtrel > 0.001f)
        {
            float l0 = k.lam.y;
            k.lam.y = l0 + vtrel;
            if (k.lam.y >= limit) k.lam.y = limit;
            dLambda = k.lam.y - l0;
            vt = vt * (1.f / vtrel);
            V3 pp = -s * dLambda * vt;
            x1 += pp * (w1 * m1); x2 += pp * (w2 * m2);
        }
    }
    x1 += disp * (w1 * m1); x2 += disp * (w2 * m2);
    pa.st(k.idx.x, make_float4(x1.x, x1.y, x1.z, m1));
    pa.st(k.idx.y, make_float4(x2.x, x2.y, x2.z, m2));
    return depth;
}

// SolveTriContacts for one contact (Physics/ClothCollisionHandler.cpp:204-287)
template <class PA>
__device__ float solve_tri_contact(const PA& pa, const DevCloth& c, const SolverParams& P, const Buffers& b, TC& k)
{
    float4 a4 = pa.ld(k.idx.x), b4 = pa.ld(k.idx.y), c4 = pa.ld(k.idx.z);
    V3 x1 = mk(a4.x, a4.y, a4.z), x2 = mk(b4.x, b4.y, b4.z), x3 = mk(c4.x, c4.y, c4.z);
    const float m1 = a4.w, m2 = b4.w, m3 = c4.w;
    V3 point = mk(k.point.x, k.point.y, k.point.z);
    V3 coords, p;
    closest_point_triangle(point, x1, x2, x3, p, coords);
    const float w1 = coords.x, w2 = coords.y, w3 = coords.z;
    k.w = make_float4(w1, w2, w3, 0.f);
    V3 n = normalized(-cross(x2 - x1, x3 - x1));
    V3 normal = n;
    if (k.mesh >= 0 && k.feature >= 0)
    {
        V3 mnrm = ldg3(mesh_view(b, k.mesh).n, k.feature);
        if (dot(n, mnrm) < 0) normal = -n;
    }
    k.normal = f4(normal, 0.f);
    const float len0 = P.thickness;
    float l = dot(normal, p - point - mk(0.f, 0.f, 0.f));
    if (l > len0) return -1.f;
    float s = 1.f / (w1 * w1 / m1 + w2 * w2 / m2 + w3 * w3 / m3);
    float depth = len0 - l;
    float dLambda = s * depth;
    k.lam.x += dLambda;
    V3 disp = dLambda * normal;
    if (P.friction != 0)
    {
        V3 p0 = w1 * ldg3(c.prev, k.idx.x) + w2 * ldg3(c.prev, k.idx.y) + w3 * ldg3(c.prev, k.idx.z);
        V3 v12 = p - p0 - mk(0.f, 0.f, 0.f);
        float vnrel = dot(normal, v12);
        V3 vt = v12 - vnrel * normal;
        float vtrel = len(vt);
        const float limit = P.friction * k.lam.x;
        if (vtrel > 0.001f)
        {
            float l0 = k.lam.y;
            k.lam.y = l0 + vtrel;
            if (k.lam.y >= limit) k.lam.y = limit;
            dLambda = k.lam.y - l0;
            vt = vt * (1.f / vtrel);
            V3 pp = -s * dLambda * vt;
            x1 += pp * (w1 * m1); x2 += pp * (w2 * m2); x3 += pp * (w3 * m3);
        }
    }
    x1 += disp * (w1 * m1); x2 += disp * (w2 * m2); x3 += disp * (w3 * m3);
    pa.st(k.idx.x, make_float4(x1.x, x1.y, x1.z, m1));
    pa.st(k.idx.y, make_float4(x2.x, x2.y, x2.z, m2));
    pa.st(k.idx.z, make_float4(x3.x, x3.y, x3.z, m3));
    return depth;
}

// SolveSelfTrisPosition for one contact (Physics/ClothCollisionHandler.cpp:364-450)
template <class PA>
__device__ float solve_self_tri(const PA& pa, const DevCloth& c, const SolverParams& P, SCt& k)
{
    const float soften = .9f;
    float len0 = P.thickness * P.selfShrink;
    float4 a4 = pa.ld(k.idx.x), b4 = pa.ld(k.idx.y), c4 = pa.ld(k.idx.z), d4 = pa.ld(k.idx.w);
    V3 x1 = mk(a4.x, a4.y, a4.z), x2 = mk(b4.x, b4.y, b4.z), x3 = mk(c4.x, c4.y, c4.z), x4 = mk(d4.x, d4.y, d4.z);
    const float m1 = a4.w, m2 = b4.w, m3 = c4.w, m4 = d4.w;
    V3 p, coords;
    closest_point_triangle(x4, x1, x2, x3, p, coords);
    const float w1 = coords.x, w2 = coords.y, w3 = coords.z;
    k.w.x = w1; k.w.y = w2; k.w.z = w3;
    V3 delta = x4 - p;
    V3 n = normalized(cross(x2 - x1, x3 - x1));
    float side = signed_volume(x4, x1, x2, x3);
    if (k.side * side <= 0) len0 = P.thickness * 0.1f;
    if (dot(n, mk(k.normal.x, k.normal.y, k.normal.z)) < 0) n = -n;
    float l = dot(n, delta);
    if (l > len0) return -1.f;
    float im = w1 * w1 * m1 + w2 * w2 * m2 + w3 * w3 * m3 + m4;
    float s = 1.f / im;
    float err = l - len0;
    k.error = err;
    float absErr = mx(0.f, -err);
    float dLambda = soften * s * err;
    V3 disp = dLambda * n;
    k.lam.x += -dLambda / P.h;
    x1 += disp * (w1 * m1);
    x2 += disp * (w2 * m2);
    x3 += disp * (w3 * m3);
    x4 -= disp * m4;
    pa.st(k.idx.x, make_float4(x1.x, x1.y, x1.z, m1));
    pa.st(k.idx.y, make_float4(x2.x, x2.y, x2.z, m2));
    pa.st(k.idx.z, make_float4(x3.x, x3.y, x3.z, m3));
    pa.st(k.idx.w, make_float4(x4.x, x4.y, x4.z, m4));
    return absErr;
}

// SolveSelfEdgesPosition for one contact (Physics/ClothCollisionHandler.cpp:453-542)
template <class PA>
__device__ float solve_self_edge(const PA& pa, const DevCloth& c, const SolverParams& P, SCt& k)
{
    float thick = P.thickness * P.selfShrink;
    const float soften = 0.9f;
    float4 a4 = pa.ld(k.idx.x), b4 = pa.ld(k.idx.y), c4 = pa.ld(k.idx.z), d4 = pa.ld(k.idx.w);
    V3 x1 = mk(a4.x, a4.y, a4.z), x2 = mk(b4.x, b4.y, b4.z), x3 = mk(c4.x, c4.y, c4.z), x4 = mk(d4.x, d4.y, d4.z);
    const float m1 = a4.w, m2 = b4.w, m3 = c4.w, m4 = d4.w;
    float side = signed_volume(x1, x2, x3, x4);
    V3 p, q;
    float t1, t2;
    closest_segm_segm(x1, x2, x3, x4, t1, t2, p, q);
    const float w1 = 1 - t1, w2 = 1 - t2;
    k.w.x = w1; k.w.y = w2;
    const float omw1 = 1.f - w1, omw2 = 1.f - w2;
    V3 delta = q - p;
    V3 n = normalized(delta);
    if (dot(n, mk(k.normal.x, k.normal.y, k.normal.z)) < 0.0f) n = -n;
    if (side * k.side < 0) thick = P.thickness * 0.1f;
    float l = dot(n, delta);
    if (l > thick) return -1.f;
    float im = w1 * w1 * m1 + omw1 * omw1 * m2 + w2 * w2 * m3 + omw2 * omw2 * m4;
    float s = 1.f / im;
    float err = l - thick;
    k.error = err;
    float absErr = mx(0.f, -err);
    float dLambda = -soften * s * err;
    k.lam.x += dLambda / P.h;
    V3 disp = dLambda * n;
    x1 -= disp * (omw1 * m1);
    x2 -= disp * (w1 * m2);
    x3 += disp * (omw2 * m3);
    x4 += disp * (w2 * m4);
    pa.st(k.idx.x, make_float4(x1.x, x1.y, x1.z, m1));
    pa.st(k.idx.y, make_float4(x2.x, x2.y, x2.z, m2));
    pa.st(k.idx.z, make_float4(x3.x, x3.y, x3.z, m3));
    pa.st(k.idx.w, make_float4(x4.x, x4.y, x4.z, m4));
    return absErr;
}

// one contact of class cls (0 edge, 1 triangle, 2 self VT, 3 self EE)
template <class PA>
__device__ __forceinline__ float solve_contact(const PA& pa, const DevCloth& c, const SolverParams& P, const Buffers& b, int cls, int i)
{
    float e;
    if (cls == 0) { EC k = b.ecList[i]; e = solve_edge_contact(pa, c, P, b, k); b.ecList[i] = k; }
    else if (cls == 1) { TC k = b.tcList[i]; e = solve_tri_contact(pa, c, P, b, k); b.tcList[i] = k; }
    else if (cls == 2) { SCt k = b.stList[i]; e = solve_self_tri(pa, c, P, k); b.stList[i] = k; }
    else { SCt k = b.seList[i]; e = solve_self_edge(pa, c, P, k); b.seList[i] = k; }
    return e;
}

// The multi-particle contact classes in the reference's order within one GS
// iteration: edge, triangle, self vertex-triangle, self edge-edge
// (Physics/ClothPBD.cpp:349-352). One CTA; one __syncthreads per colour.
__global__ void __launch_bounds__(1024) k_solve_multi(DevCloth c, SolverParams P, Buffers b, ColourArgs a)
{
    if (gs_done(c)) return;
    __shared__ float sErr[4];
    if (threadIdx.x < 4) sErr[threadIdx.x] = 0.f;
    __syncthreads();
    for (int cls = 0; cls < 4; cls++)
    {
        const ClassView& cv = a.cls[cls];
        const int n = *cv.count;
        if (n == 0) continue;
        for (int col = 0; col < MAX_COLOURS; col++)
        {
            const int s0 = cv.start[col], s1 = cv.start[col + 1];
            if (s0 == s1) continue;
            // the last colour holds contacts left after the colouring rounds; one
            // thread solves them in list order (deterministic, as the oracle does)
            const bool serial = (col == MAX_COLOURS - 1);
            const int jEnd = serial ? n : s1;
            for (int j = serial ? 0 : s0 + threadIdx.x; j < jEnd; j += (serial ? 1 : blockDim.x))
            {
                if (serial && threadIdx.x != 0) break;
                if (serial && cv.colour[j] != MAX_COLOURS - 1) continue;
                int i = serial ? j : cv.order[j];
                float e = solve_contact(GlobalPos{c.pos}, c, P, b, cls, i);
                if (e > 0.f) atomicMax((int*)&sErr[cls], __float_as_int(e));
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0 && !P.fixedIterations)
    {
        c.scal[4] = sErr[0]; c.scal[5] = sErr[1]; c.scal[6] = sErr[2]; c.scal[7] = sErr[3];
    }
}

// SolveGS exit test (Physics/ClothPBD.cpp:354-361); FEM mode has no link error.
__global__ void k_gs_exit(DevCloth c, SolverParams P, int iter)
{
    if (gs_done(c)) return;
    c.scal[9] = (float)(iter + 1);
    if (P.fixedIterations) return;
    const float eps = 0.01f;
    float cb = c.scal[2], cv = c.scal[3], ce = c.scal[4], ct = c.scal[5], sct = c.scal[6], see = c.scal[7];
    const float cl = P.fem ? 0.f : c.scal[1];
    if (cl < 0.05f && cb < 0.005f && see < P.selfThreshold && sct < P.selfThreshold && cv < eps && ce < eps && ct < eps)
        c.scal[8] = 1.f;
}

__global__ void k_reset_iter_errors(DevCloth c)
{
    // cv is a per-iteration maximum written with atomics; cb persists between
    // bend iterations (it is only recomputed when bends run)
    if (threadIdx.x == 0) c.scal[3] = 0.f;
}

// cl (the links' error) is a per-iteration maximum: cleared before the link sweep
__global__ void k_reset_link_error(DevCloth c)
{
    if (threadIdx.x == 0 && !gs_done(c)) c.scal[1] = 0.f;
}

__global__ void k_reset_bend_error(DevCloth c)
{
    if (threadIdx.x == 0 && !gs_done(c)) c.scal[2] = 0.f;
}


struct ClusterPos
{
    float4* local;
    uint32_t shift, mask;
    __device__ __forceinline__ float4* addr(uint32_t v) const
    {
        return cg::this_cluster().map_shared_rank(local + (v & mask), v >> shift);
    }
    __device__ __forceinline__ float4 ld(uint32_t v) const { return *addr(v); }
    __device__ __forceinline__ void st(uint32_t v, float4 x) const { *addr(v) = x; }
};

// particle accessor over a tile entry's own registers (the projection functions
// load their particles first and store them last)
struct RegPos
{
    uint32_t id[4];
    mutable float4 v[4];
    __device__ __forceinline__ float4 ld(uint32_t q) const
    {
        return q == id[0] ? v[0] : q == id[1] ? v[1] : q == id[2] ? v[2] : v[3];
    }
    __device__ __forceinline__ void st(uint32_t q, float4 x) const
    {
        if (q == id[0]) v[0] = x;
        else if (q == id[1]) v[1] = x;
        else if (q == id[2]) v[2] = x;
        else v[3] = x;
    }
};

// A thread of the cluster solver takes TILE consecutive constraints of its CTA's
// chunk of a colour and issues all their particle loads (distributed shared
// memory) before any projection, so their latencies overlap; the constraints of
// a colour share no particle, so the result is unchanged.
template <int TILE, class PA>
__device__ __forceinline__ void cluster_fem(const PA& pa, const DevCloth& c, const SolverParams& P, const float4* staged,
                                            int a, int e)
{
    if constexpr (TILE == 1)
    {
        // one constraint a thread: project straight through the accessor
        for (int j = a + (int)threadIdx.x; j < e; j += (int)blockDim.x)
        {
            if (staged)
            {
                const float4* r = staged + 3 * (j - a);
                fem_project(pa, r[0], r[1], r[2], P);
            }
            else
                fem_project(pa, __ldg(&c.fem[3 * j]), __ldg(&c.fem[3 * j + 1]), __ldg(&c.fem[3 * j + 2]), P);
        }
        return;
    }
    for (int j0 = a + (int)threadIdx.x * TILE; j0 < e; j0 += (int)blockDim.x * TILE)
    {
        float4 r0[TILE], r1[TILE], r2[TILE];
        RegPos rp[TILE];
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            const int j = min(j0 + u, e - 1);
            if (staged)
            {
                const float4* r = staged + 3 * (j - a);
                r0[u] = r[0]; r1[u] = r[1]; r2[u] = r[2];
            }
            else
            {
                r0[u] = __ldg(&c.fem[3 * j]); r1[u] = __ldg(&c.fem[3 * j + 1]); r2[u] = __ldg(&c.fem[3 * j + 2]);
            }
        }
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            rp[u].id[0] = __float_as_uint(r0[u].x); rp[u].id[1] = __float_as_uint(r0[u].y);
            rp[u].id[2] = __float_as_uint(r0[u].z); rp[u].id[3] = 0xffffffffu;
            rp[u].v[0] = pa.ld(rp[u].id[0]); rp[u].v[1] = pa.ld(rp[u].id[1]); rp[u].v[2] = pa.ld(rp[u].id[2]);
        }
#pragma unroll
        for (int u = 0; u < TILE; u++)
            if (j0 + u < e) fem_project(rp[u], r0[u], r1[u], r2[u], P);
#pragma unroll
        for (int u = 0; u < TILE; u++)
            if (j0 + u < e)
            {
                pa.st(rp[u].id[0], rp[u].v[0]); pa.st(rp[u].id[1], rp[u].v[1]); pa.st(rp[u].id[2], rp[u].v[2]);
            }
    }
}

template <int TILE, class PA>
__device__ __forceinline__ float cluster_bends(const PA& pa, const DevCloth& c, const SolverParams& P, const uint4* staged,
                                               int a, int e)
{
    float err = 0.f;
    if constexpr (TILE == 1)
    {
        for (int j = a + (int)threadIdx.x; j < e; j += (int)blockDim.x)
            err = fmaxf(err, bend_project(pa, staged ? staged[j - a] : __ldg(&c.bend[j]), P));
        return err;
    }
    for (int j0 = a + (int)threadIdx.x * TILE; j0 < e; j0 += (int)blockDim.x * TILE)
    {
        uint4 bc[TILE];
        RegPos rp[TILE];
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            const int j = min(j0 + u, e - 1);
            bc[u] = staged ? staged[j - a] : __ldg(&c.bend[j]);
        }
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            rp[u].id[0] = bc[u].x; rp[u].id[1] = bc[u].y; rp[u].id[2] = bc[u].z; rp[u].id[3] = bc[u].w;
            rp[u].v[0] = pa.ld(bc[u].x); rp[u].v[1] = pa.ld(bc[u].y); rp[u].v[2] = pa.ld(bc[u].z); rp[u].v[3] = pa.ld(bc[u].w);
        }
        bool moved[TILE];
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            moved[u] = false;
            if (j0 + u < e)
            {
                const float ev = bend_project(rp[u], bc[u], P);
                moved[u] = ev >= 0.f;
                err = fmaxf(err, ev);
            }
        }
#pragma unroll
        for (int u = 0; u < TILE; u++)
            if (moved[u])
            {
                pa.st(bc[u].x, rp[u].v[0]); pa.st(bc[u].y, rp[u].v[1]); pa.st(bc[u].z, rp[u].v[2]); pa.st(bc[u].w, rp[u].v[3]);
            }
    }
    return err;
}

// The multi-particle contact classes inside a cluster-resident solver (edge,
// triangle, self vertex-triangle, self edge-edge; Physics/ClothPBD.cpp:349-352):
// each colour split into one contiguous chunk per CTA, particles through
// distributed shared memory, a cluster barrier after every colour.
template <class PA>
__device__ __forceinline__ void cluster_contact_classes(const PA& pa, const DevCloth& c, const SolverParams& P,
                                                        const Buffers& b, const ColourArgs& ca, int rank, int nRank,
                                                        bool track, float* sErr)
{
    cg::cluster_group cl = cg::this_cluster();
    for (int cls = 0; cls < 4; cls++)
    {
        const ClassView& cv = ca.cls[cls];
        const int n = *cv.count;
        if (n == 0) continue;
        for (int col = 0; col < MAX_COLOURS; col++)
        {
            const int s0 = cv.start[col], s1 = cv.start[col + 1];
            if (s0 == s1) continue;
            if (col == MAX_COLOURS - 1)
            {
                // colours exhausted: one thread, list order (as the oracle)
                if (rank == 0 && threadIdx.x == 0)
                    for (int i = 0; i < n; i++)
                        if (cv.colour[i] == MAX_COLOURS - 1)
                        {
                            float e = solve_contact(pa, c, P, b, cls, i);
                            if (track && e > 0.f) atomicMax((int*)&sErr[4 + cls], __float_as_int(e));
                        }
            }
            else
            {
                const int chunk = (s1 - s0 + nRank - 1) / nRank;
                const int a = s0 + rank * chunk, e = min(s1, a + chunk);
                for (int j = a + threadIdx.x; j < e; j += blockDim.x)
                {
                    float err = solve_contact(pa, c, P, b, cls, __ldg(&cv.order[j]));
                    if (track && err > 0.f) atomicMax((int*)&sErr[4 + cls], __float_as_int(err));
                }
            }
            cl.sync();
        }
    }
}

// End of one Gauss-Seidel iteration of a cluster-resident solver whose CTA holds
// the particles [v0, v0 + vpc) in sPos: the iteration count, the update residual
// test (residual-target mode) and the reference's exit test
// (Physics/ClothPBD.cpp:354-361). True when the loop ends.
__device__ __forceinline__ bool cluster_iteration_end(const DevCloth& c, const SolverParams& P, const float4* sPos,
                                                      int v0, uint32_t vpc, int rank, int k, bool track, float* sErr)
{
    cg::cluster_group cl = cg::this_cluster();
    if (threadIdx.x == 0 && rank == 0) c.scal[9] = (float)(k + 1);
    if (P.resTol > 0.f)
    {
        // residual-target mode: the largest displacement of this iteration (own
        // particles, against the snapshot), cluster-wide; then the next snapshot
        float r = 0.f;
        for (uint32_t v = threadIdx.x; v < vpc; v += blockDim.x)
        {
            const int g = v0 + (int)v;
            if (g >= c.N) continue;
            const float4 x = sPos[v], x0 = c.xsnap[g];
            const float dx = x.x - x0.x, dy = x.y - x0.y, dz = x.z - x0.z;
            r = fmaxf(r, sqrtf(dx * dx + dy * dy + dz * dz) * P.resScale);
            c.xsnap[g] = x;
        }
        const unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(r));
        unsigned* word = reinterpret_cast<unsigned*>(c.scal + 11);
        if ((threadIdx.x & 31) == 0 && u) atomicMax(word, u);
        cl.sync();
        const float res = __uint_as_float(__ldcg(word));
        cl.sync();
        if (rank == 0 && threadIdx.x == 0) *word = 0u;
        if (res <= P.resTol) return true;
    }
    if (track)
    {
        // SolveGS exit test (Physics/ClothPBD.cpp:354-361) on cluster-wide maxima
        if (threadIdx.x < 8 && threadIdx.x >= 1 && sErr[threadIdx.x] > 0.f)
            atomic_max_pos(&c.scal[threadIdx.x], sErr[threadIdx.x]);
        cl.sync();
        if (rank == 0 && threadIdx.x == 0)
        {
            const float eps = 0.01f;
            float cb = c.scal[2], cv = c.scal[3], ce = c.scal[4], ct = c.scal[5], sct = c.scal[6], see = c.scal[7];
            const float clk = P.fem ? 0.f : c.scal[1];
            if (clk < 0.05f && cb < 0.005f && see < P.selfThreshold && sct < P.selfThreshold && cv < eps && ce < eps && ct < eps)
                c.scal[8] = 1.f;
            c.scal[1] = 0.f;
            for (int s = 3; s < 8; s++) c.scal[s] = 0.f;          // per-iteration maxima
            if ((k + 1) % P.bendFreq == 0) c.scal[2] = 0.f;       // recomputed by the next bend sweep
        }
        if (threadIdx.x < 8) sErr[threadIdx.x] = 0.f;
        cl.sync();
        if (__ldcg(&c.scal[8]) != 0.f) return true;
    }
    return false;
}

template <int TILE>
__global__ void __launch_bounds__(GS_THREADS) k_gs_cluster(DevCloth c, SolverParams P, Buffers b, ColourArgs ca, GsPlan plan)
{
    extern __shared__ float4 sPos[];
    __shared__ float sErr[8];
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int nRank = (int)cl.num_blocks();
    const uint32_t vpc = 1u << plan.shift;
    const int v0 = rank * (int)vpc;
    for (uint32_t v = threadIdx.x; v < vpc; v += blockDim.x)
    {
        int g = v0 + (int)v;
        if (g < c.N) sPos[v] = c.pos[g];
    }
    if (threadIdx.x < 8) sErr[threadIdx.x] = 0.f;
    // split [s0, s1) into nRank contiguous chunks (contiguous constraints are
    // spatially close, so most particle accesses stay in the CTA's own block)
    auto range = [&](int s0, int s1, int& a, int& e) {
        const int chunk = (s1 - s0 + nRank - 1) / nRank;
        a = s0 + rank * chunk;
        e = min(s1, a + chunk);
    };
    // staged records: this CTA's chunks of every colour, copied once per substep
    // (layout after the particle block: FEM records, then bends)
    __shared__ int sFemOff[65], sBendOff[65];
    float4* sFem = sPos + vpc;
    uint4* sBend = reinterpret_cast<uint4*>(sFem + 3 * plan.femStage);
    if (threadIdx.x == 0)
    {
        int acc = 0;
        for (int col = 0; col < plan.nFemCol; col++)
        {
            int a, e;
            range(plan.femStart[col], plan.femStart[col + 1], a, e);
            sFemOff[col] = acc;
            acc += max(0, e - a);
        }
        acc = 0;
        for (int col = 0; col < plan.nBendCol; col++)
        {
            int a, e;
            range(plan.bendStart[col], plan.bendStart[col + 1], a, e);
            sBendOff[col] = acc;
            acc += max(0, e - a);
        }
    }
    __syncthreads();
    if (plan.stage)
    {
        for (int col = 0; col < plan.nFemCol; col++)
        {
            int a, e;
            range(plan.femStart[col], plan.femStart[col + 1], a, e);
            for (int j = a * 3 + threadIdx.x; j < e * 3; j += blockDim.x) sFem[3 * sFemOff[col] + (j - 3 * a)] = c.fem[j];
        }
        for (int col = 0; col < plan.nBendCol; col++)
        {
            int a, e;
            range(plan.bendStart[col], plan.bendStart[col + 1], a, e);
            for (int j = a + threadIdx.x; j < e; j += blockDim.x) sBend[sBendOff[col] + (j - a)] = c.bend[j];
        }
    }
    cl.sync();
    const ClusterPos pa{sPos, (uint32_t)plan.shift, vpc - 1};
    const bool track = !P.fixedIterations;
    if (P.resTol > 0.f)
    {
        for (uint32_t v = threadIdx.x; v < vpc; v += blockDim.x)
            if (v0 + (int)v < c.N) c.xsnap[v0 + v] = sPos[v];
        cl.sync();     // no CTA writes a particle before its snapshot is taken
    }
    for (int k = 0; k < plan.iterations; k++)
    {
        if (P.fem)
            for (int col = 0; col < plan.nFemCol; col++)
            {
                int a, e;
                range(plan.femStart[col], plan.femStart[col + 1], a, e);
                cluster_fem<TILE>(pa, c, P, plan.stage ? sFem + 3 * sFemOff[col] : nullptr, a, e);
                cl.sync();
            }
        else
            for (int col = 0; col < plan.nLinkCol; col++)
            {
                int a, e;
                range(plan.linkStart[col], plan.linkStart[col + 1], a, e);
                for (int j = a + threadIdx.x; j < e; j += blockDim.x)
                {
                    const float err = link_project(pa, __ldg(&c.link[j]), P);
                    if (track && err > 0.f) atomicMax((int*)&sErr[1], __float_as_int(err));
                }
                cl.sync();
            }
        if (P.dihedral && k % P.bendFreq == 0)
            for (int col = 0; col < plan.nBendCol; col++)
            {
                int a, e;
                range(plan.bendStart[col], plan.bendStart[col + 1], a, e);
                const float errv = cluster_bends<TILE>(pa, c, P, plan.stage ? sBend + sBendOff[col] : nullptr, a, e);
                if (track && errv > 0.f) atomicMax((int*)&sErr[2], __float_as_int(errv));
                cl.sync();
            }
        if (b.numVColl > 0)
        {
            // each CTA solves the vertex contacts of its own particles
            for (uint32_t v = threadIdx.x; v < vpc; v += blockDim.x)
            {
                const int g = v0 + (int)v;
                if (g >= c.N) continue;
                float err = vertex_contacts_one(pa, c, P, b, g);
                if (track && err > 0.f) atomicMax((int*)&sErr[3], __float_as_int(err));
            }
            cl.sync();
        }
        cluster_contact_classes(pa, c, P, b, ca, rank, nRank, track, sErr);
        if (cluster_iteration_end(c, P, sPos, v0, vpc, rank, k, track, sErr)) break;
    }
    if (rank == 0 && threadIdx.x == 0) c.scal[10] += c.scal[9];
    // write back own particles and update their velocities (ClothPBD.cpp:314-321)
    for (uint32_t v = threadIdx.x; v < vpc; v += blockDim.x)
    {
        const int g = v0 + (int)v;
        if (g >= c.N) continue;
        const float4 p = sPos[v];
        c.pos[g] = p;
        if (p.w == 0.f) continue;
        const float4 q = c.prev[g];
        V3 vel = P.invH * (mk(p.x, p.y, p.z) - mk(q.x, q.y, q.z));
        c.vel[g] = make_float4(vel.x, vel.y, vel.z, 0.f);
    }
}

// ---------------------------------------------------- band-parallel solver
// One cluster per cloth; CTA r owns the particles [r 2^shift, (r + 1) 2^shift)
// (a band), resident in its shared memory for the whole substep. Each class's
// records (FEM triangles, bends, links) are split per band into interior
// records (all particles in the band) and boundary records (lowest particle in
// the band, the others in it or among the first `halo` particles of the next
// band). A sweep runs, in every CTA at once, the band's interior records colour
// by colour on its own shared memory with CTA barriers between colours; then,
// after a cluster barrier, each CTA copies the next band's first `halo`
// particles into a local buffer, runs its boundary records colour by colour on
// its band and that buffer, and copies the buffer back before a second cluster
// barrier. Interior record sets of different bands share no particle; neither
// do boundary sets, because the host admits a plan only if the boundary records
// of every band touch their own band at offsets >= halo (beyond the part the
// previous band copies). The launch therefore computes the sequential
// Gauss-Seidel sweep in the order (part, band, colour, record), which equals
// (part, colour, band, record): two colour phases per class sweep end in a
// cluster barrier instead of every colour. The contact classes run as in the
// cluster solver (chunks, distributed shared memory, a cluster barrier per
// colour); vertex contacts touch one particle each and run on the owner CTA.

// particle accessor of a band CTA: its own band, then the copied head of the next
struct BandPos
{
    float4* own;
    float4* halo;
    uint32_t v0, v1;
    __device__ __forceinline__ float4* addr(uint32_t g) const { return g < v1 ? own + (g - v0) : halo + (g - v1); }
    __device__ __forceinline__ float4 ld(uint32_t g) const { return *addr(g); }
    __device__ __forceinline__ void st(uint32_t g, float4 x) const { *addr(g) = x; }
};

// one record of class KIND (0 FEM: three float4; 1 bend: a uint4; 2 link: a
// float4), from shared memory (staged: index relative to the band's first
// record) or through the non-coherent path
template <int KIND>
struct BandRec { float4 r[KIND == 0 ? 3 : 1]; };

template <int KIND>
__device__ __forceinline__ BandRec<KIND> band_load(const BandView& bv, const float4* staged, int base, int j)
{
    BandRec<KIND> q;
    if constexpr (KIND == 0)
    {
        if (staged)
        {
            const float4* r = staged + 3 * (j - base);
            q.r[0] = r[0]; q.r[1] = r[1]; q.r[2] = r[2];
        }
        else
        {
            q.r[0] = __ldg(&bv.fem[3 * j]); q.r[1] = __ldg(&bv.fem[3 * j + 1]); q.r[2] = __ldg(&bv.fem[3 * j + 2]);
        }
    }
    else if constexpr (KIND == 1)
        q.r[0] = staged ? staged[j - base] : __ldg(reinterpret_cast<const float4*>(bv.bend) + j);
    else
        q.r[0] = staged ? staged[j - base] : __ldg(&bv.link[j]);
    return q;
}

template <int KIND>
__device__ __forceinline__ float band_apply(const BandPos& pa, const SolverParams& P, const BandRec<KIND>& q)
{
    if constexpr (KIND == 0)
    {
        fem_project(pa, q.r[0], q.r[1], q.r[2], P);
        return 0.f;
    }
    else if constexpr (KIND == 1)
    {
        const float4 f = q.r[0];
        return bend_project(pa, make_uint4(__float_as_uint(f.x), __float_as_uint(f.y), __float_as_uint(f.z),
                                           __float_as_uint(f.w)), P);
    }
    else
        return link_project(pa, q.r[0], P);
}

// one sweep of a class over the cluster: 2 nCol steps (interior colours, then
// boundary colours); each thread's first record of the next step is loaded
// before the current step's projections, so its latency overlaps them. Returns
// this thread's largest projection error.
template <int KIND, int NT>
__device__ __forceinline__ float band_sweep(const BandPos& pa, const SolverParams& P, const BandView& bv,
                                            const float4* staged, int band, int nb, float4* nextHead, const int* off)
{
    // off: this band's 2 nCol + 1 record offsets of the class, in shared memory
    cg::cluster_group cl = cg::this_cluster();
    const int nCol = KIND == 0 ? bv.nFemCol : KIND == 1 ? bv.nBendCol : bv.nLinkCol;
    const int base = off[0];
    const int tid = (int)threadIdx.x;
    const bool hasNext = band + 1 < nb;
    float err = 0.f;
    int a = off[0], e = off[1];
    BandRec<KIND> cur;
    if (a + tid < e) cur = band_load<KIND>(bv, staged, base, a + tid);
    for (int step = 0; step < 2 * nCol; step++)
    {
        // off[step] .. off[step + 1] is this band's step: (part, colour) = (step / nCol, step % nCol)
        int a2 = 0, e2 = 0;
        BandRec<KIND> nxt;
        if (step + 1 < 2 * nCol)
        {
            a2 = off[step + 1]; e2 = off[step + 2];
            if (a2 + tid < e2) nxt = band_load<KIND>(bv, staged, base, a2 + tid);
        }
        if (step == nCol)
        {
            cl.sync();                 // every band's interior records are done
            if (hasNext)
                for (int i = tid; i < bv.halo; i += NT) pa.halo[i] = nextHead[i];
            __syncthreads();
        }
        if (a + tid < e) err = fmaxf(err, band_apply<KIND>(pa, P, cur));
        for (int j = a + tid + NT; j < e; j += NT) err = fmaxf(err, band_apply<KIND>(pa, P, band_load<KIND>(bv, staged, base, j)));
        if (step + 1 != nCol) __syncthreads();
        cur = nxt;
        a = a2; e = e2;
    }
    if (hasNext)
        for (int i = tid; i < bv.halo; i += NT) nextHead[i] = pa.halo[i];
    cl.sync();                         // the heads are back with their owners
    return err;
}

template <int NT>
__global__ void __launch_bounds__(NT) k_gs_band(DevCloth c, SolverParams P, Buffers b, ColourArgs ca, GsPlan plan,
                                                BandView bv)
{
    extern __shared__ float4 sPos[];
    __shared__ float sErr[8];
    cg::cluster_group cl = cg::this_cluster();
    const int band = (int)cl.block_rank(), nb = (int)cl.num_blocks();
    const uint32_t vpc = 1u << bv.shift;
    const int v0 = band * (int)vpc;
    // shared memory: own band | halo (rounded to 16 particles) | staged FEM | bends | links
    float4* sHalo = sPos + vpc;
    float4* sFem = sHalo + ((bv.halo + 15) & ~15);
    float4* sBend = sFem + (bv.stageFem ? 3 * bv.femMax : 0);
    float4* sLink = sBend + (bv.stageBend ? bv.bendMax : 0);
    float4* nextHead = band + 1 < nb ? cl.map_shared_rank(sPos, band + 1) : nullptr;
    for (uint32_t v = threadIdx.x; v < vpc; v += NT)
    {
        const int g = v0 + (int)v;
        if (g < c.N) sPos[v] = c.pos[g];
    }
    auto stage = [&](int nCol, const int* off, const float4* src, int perRec, float4* dst) {
        const int a = __ldg(&off[band * 2 * nCol]), e = __ldg(&off[(band + 1) * 2 * nCol]);
        for (int j = a * perRec + (int)threadIdx.x; j < e * perRec; j += NT) dst[j - a * perRec] = __ldg(&src[j]);
    };
    if (bv.stageFem) stage(bv.nFemCol, bv.femOff, bv.fem, 3, sFem);
    if (bv.stageBend) stage(bv.nBendCol, bv.bendOff, reinterpret_cast<const float4*>(bv.bend), 1, sBend);
    if (bv.stageLink) stage(bv.nLinkCol, bv.linkOff, bv.link, 1, sLink);
    // this band's record offsets of each class (at most 64 colours a class)
    __shared__ int sOff[3][129];
    {
        const int nc[3] = {bv.nFemCol, bv.nBendCol, bv.nLinkCol};
        const int* src[3] = {bv.femOff, bv.bendOff, bv.linkOff};
        for (int k = 0; k < 3; k++)
            for (int j = (int)threadIdx.x; j <= 2 * nc[k] && j < 129; j += NT) sOff[k][j] = __ldg(&src[k][band * 2 * nc[k] + j]);
    }
    if (threadIdx.x < 8) sErr[threadIdx.x] = 0.f;
    cl.sync();
    const BandPos pa{sPos, sHalo, (uint32_t)v0, (uint32_t)v0 + vpc};
    const ClusterPos cpa{sPos, (uint32_t)bv.shift, vpc - 1};
    const bool track = !P.fixedIterations;
    if (P.resTol > 0.f)
    {
        for (uint32_t v = threadIdx.x; v < vpc; v += NT)
            if (v0 + (int)v < c.N) c.xsnap[v0 + v] = sPos[v];
        __syncthreads();
    }
    for (int k = 0; k < plan.iterations; k++)
    {
        if (P.fem)
            band_sweep<0, NT>(pa, P, bv, bv.stageFem ? sFem : nullptr, band, nb, nextHead, sOff[0]);
        else
        {
            const float e = band_sweep<2, NT>(pa, P, bv, bv.stageLink ? sLink : nullptr, band, nb, nextHead, sOff[2]);
            if (track && e > 0.f) atomicMax((int*)&sErr[1], __float_as_int(e));
        }
        if (P.dihedral && k % P.bendFreq == 0)
        {
            const float e = band_sweep<1, NT>(pa, P, bv, bv.stageBend ? sBend : nullptr, band, nb, nextHead, sOff[1]);
            if (track && e > 0.f) atomicMax((int*)&sErr[2], __float_as_int(e));
        }
        if (b.numVColl > 0)
        {
            // each CTA solves the vertex contacts of its own particles
            for (uint32_t v = threadIdx.x; v < vpc; v += NT)
            {
                const int g = v0 + (int)v;
                if (g >= c.N) continue;
                const float err = vertex_contacts_one(pa, c, P, b, g);
                if (track && err > 0.f) atomicMax((int*)&sErr[3], __float_as_int(err));
            }
        }
        // the contact classes reach any particle: all vertex contacts first
        bool contacts = false;
        for (int cls = 0; cls < 4; cls++) contacts |= *ca.cls[cls].count > 0;
        if (contacts) cl.sync();
        else __syncthreads();
        cluster_contact_classes(cpa, c, P, b, ca, band, nb, track, sErr);
        if (cluster_iteration_end(c, P, sPos, v0, vpc, band, k, track, sErr)) break;
    }
    if (band == 0 && threadIdx.x == 0) c.scal[10] += c.scal[9];
    // write back own particles and update their velocities (ClothPBD.cpp:314-321)
    for (uint32_t v = threadIdx.x; v < vpc; v += NT)
    {
        const int g = v0 + (int)v;
        if (g >= c.N) continue;
        const float4 p = sPos[v];
        c.pos[g] = p;
        if (p.w == 0.f) continue;
        const float4 q = c.prev[g];
        V3 vel = P.invH * (mk(p.x, p.y, p.z) - mk(q.x, q.y, q.z));
        c.vel[g] = make_float4(vel.x, vel.y, vel.z, 0.f);
    }
}

// ---------------------------------------------------- grid-resident solver
// The same Gauss-Seidel loop as k_gs_cluster for clothes (and batches of
// clothes) too large for one cluster: one cooperative launch per substep, every
// CTA of the grid resident, particles in global memory (L2-resident: 16 B per
// particle), grid-wide barriers between colours. Each thread takes TILE
// consecutive constraints of a colour and issues all their loads before any
// projection (the constraints of a colour share no particle), so TILE
// projections' memory latencies overlap. Same phases and order as the
// per-colour kernels: bit-identical results.


// Constraint records are constant for the whole launch: they are read through the
// non-coherent path (ld.global.nc), which keeps them in the SM's L1 from one
// iteration to the next (each thread sweeps the same records every iteration),
// so only the particle loads pay the L2 latency in a colour phase.
template <int TILE>
__device__ __forceinline__ void fem_tiles(const DevCloth& c, const SolverParams& P, const float4* fem, int s0, int s1,
                                          int tid, int nth)
{
    for (int base = s0 + tid * TILE; base < s1; base += nth * TILE)
    {
        float4 r0[TILE], r1[TILE], r2[TILE];
        RegPos rp[TILE];
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            const int j = min(base + u, s1 - 1);
            r0[u] = __ldg(&fem[3 * j]); r1[u] = __ldg(&fem[3 * j + 1]); r2[u] = __ldg(&fem[3 * j + 2]);
        }
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            rp[u].id[0] = __float_as_uint(r0[u].x); rp[u].id[1] = __float_as_uint(r0[u].y);
            rp[u].id[2] = __float_as_uint(r0[u].z); rp[u].id[3] = 0xffffffffu;
            rp[u].v[0] = c.pos[rp[u].id[0]]; rp[u].v[1] = c.pos[rp[u].id[1]]; rp[u].v[2] = c.pos[rp[u].id[2]];
        }
#pragma unroll
        for (int u = 0; u < TILE; u++)
            if (base + u < s1) fem_project(rp[u], r0[u], r1[u], r2[u], P);
#pragma unroll
        for (int u = 0; u < TILE; u++)
            if (base + u < s1)
            {
                c.pos[rp[u].id[0]] = rp[u].v[0]; c.pos[rp[u].id[1]] = rp[u].v[1]; c.pos[rp[u].id[2]] = rp[u].v[2];
            }
    }
}

template <int TILE>
__device__ __forceinline__ float bend_tiles(const DevCloth& c, const SolverParams& P, const uint4* bend, int s0, int s1,
                                           int tid, int nth)
{
    float err = 0.f;
    for (int base = s0 + tid * TILE; base < s1; base += nth * TILE)
    {
        uint4 bc[TILE];
        RegPos rp[TILE];
#pragma unroll
        for (int u = 0; u < TILE; u++) bc[u] = __ldg(&bend[min(base + u, s1 - 1)]);
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            rp[u].id[0] = bc[u].x; rp[u].id[1] = bc[u].y; rp[u].id[2] = bc[u].z; rp[u].id[3] = bc[u].w;
            rp[u].v[0] = c.pos[bc[u].x]; rp[u].v[1] = c.pos[bc[u].y]; rp[u].v[2] = c.pos[bc[u].z]; rp[u].v[3] = c.pos[bc[u].w];
        }
        bool moved[TILE];
#pragma unroll
        for (int u = 0; u < TILE; u++)
        {
            moved[u] = false;
            if (base + u < s1)
            {
                const float e = bend_project(rp[u], bc[u], P);
                moved[u] = e >= 0.f;
                err = fmaxf(err, e);
            }
        }
#pragma unroll
        for (int u = 0; u < TILE; u++)
            if (moved[u])
            {
                c.pos[bc[u].x] = rp[u].v[0]; c.pos[bc[u].y] = rp[u].v[1]; c.pos[bc[u].z] = rp[u].v[2]; c.pos[bc[u].w] = rp[u].v[3];
            }
    }
    return err;
}

template <int NT, int FT, int BT>
__global__ void __launch_bounds__(NT) k_gs_grid(DevCloth c, SolverParams P, Buffers b, ColourArgs ca, GsPlan plan)
{
    cg::grid_group grid = cg::this_grid();
    __shared__ float sErr[8];
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const GlobalPos pa{c.pos};
    const bool track = !P.fixedIterations;
    if (threadIdx.x < 8) sErr[threadIdx.x] = 0.f;
    if (P.resTol > 0.f)
    {
        for (int g = tid; g < c.N; g += nth) c.xsnap[g] = c.pos[g];
        grid.sync();
    }
    __syncthreads();
    for (int k = 0; k < plan.iterations; k++)
    {
        if (P.fem)
            for (int col = 0; col < plan.nFemCol; col++)
            {
                fem_tiles<FT>(c, P, c.fem, plan.femStart[col], plan.femStart[col + 1], tid, nth);
                grid.sync();
            }
        else
            for (int col = 0; col < plan.nLinkCol; col++)
            {
                for (int j = plan.linkStart[col] + tid; j < plan.linkStart[col + 1]; j += nth)
                {
                    const float err = link_project(pa, __ldg(&c.link[j]), P);
                    if (track && err > 0.f) atomicMax((int*)&sErr[1], __float_as_int(err));
                }
                grid.sync();
            }
        if (P.dihedral && k % P.bendFreq == 0)
            for (int col = 0; col < plan.nBendCol; col++)
            {
                const float e = bend_tiles<BT>(c, P, c.bend, plan.bendStart[col], plan.bendStart[col + 1], tid, nth);
                if (track && e > 0.f) atomicMax((int*)&sErr[2], __float_as_int(e));
                grid.sync();
            }
        if (b.numVColl > 0)
        {
            for (int i = tid; i < c.N; i += nth)
            {
                const float e = vertex_contacts_one(pa, c, P, b, i);
                if (track && e > 0.f) atomicMax((int*)&sErr[3], __float_as_int(e));
            }
            grid.sync();
        }
        for (int cls = 0; cls < 4; cls++)
        {
            const ClassView& cv = ca.cls[cls];
            const int n = *cv.count;
            if (n == 0) continue;
            for (int col = 0; col < MAX_COLOURS; col++)
            {
                const int s0 = cv.start[col], s1 = cv.start[col + 1];
                if (s0 == s1) continue;
                if (col == MAX_COLOURS - 1)
                {
                    // colours exhausted: one thread, list order (as the oracle)
                    if (tid == 0)
                        for (int i = 0; i < n; i++)
                            if (cv.colour[i] == MAX_COLOURS - 1)
                            {
                                const float e = solve_contact(pa, c, P, b, cls, i);
                                if (track && e > 0.f) atomicMax((int*)&sErr[4 + cls], __float_as_int(e));
                            }
                }
                else
                    for (int j = s0 + tid; j < s1; j += nth)
                    {
                        const float e = solve_contact(pa, c, P, b, cls, __ldg(&cv.order[j]));
                        if (track && e > 0.f) atomicMax((int*)&sErr[4 + cls], __float_as_int(e));
                    }
                grid.sync();
            }
        }
        if (tid == 0) c.scal[9] = (float)(k + 1);
        if (P.resTol > 0.f)
        {
            // residual-target mode: the largest displacement of this iteration,
            // grid-wide; then the next snapshot (each thread its own particles)
            float r = 0.f;
            for (int g = tid; g < c.N; g += nth)
            {
                const float4 x = c.pos[g], x0 = c.xsnap[g];
                const float dx = x.x - x0.x, dy = x.y - x0.y, dz = x.z - x0.z;
                r = fmaxf(r, sqrtf(dx * dx + dy * dy + dz * dz) * P.resScale);
                c.xsnap[g] = x;
            }
            const unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(r));
            unsigned* word = reinterpret_cast<unsigned*>(c.scal + 11);
            if ((threadIdx.x & 31) == 0 && u) atomicMax(word, u);
            grid.sync();
            const float res = __uint_as_float(__ldcg(word));
            grid.sync();
            if (tid == 0) *word = 0u;
            if (res <= P.resTol) break;
        }
        if (track)
        {
            // SolveGS exit test (Physics/ClothPBD.cpp:354-361) on grid-wide maxima
            __syncthreads();
            if (threadIdx.x < 8 && threadIdx.x >= 1 && sErr[threadIdx.x] > 0.f)
                atomic_max_pos(&c.scal[threadIdx.x], sErr[threadIdx.x]);
            grid.sync();
            if (tid == 0)
            {
                const float eps = 0.01f;
                float cb = c.scal[2], cv = c.scal[3], ce = c.scal[4], ct = c.scal[5], sct = c.scal[6], see = c.scal[7];
                const float clk = P.fem ? 0.f : c.scal[1];
                if (clk < 0.05f && cb < 0.005f && see < P.selfThreshold && sct < P.selfThreshold && cv < eps && ce < eps && ct < eps)
                    c.scal[8] = 1.f;
                c.scal[1] = 0.f;
                for (int s2 = 3; s2 < 8; s2++) c.scal[s2] = 0.f;
                if ((k + 1) % P.bendFreq == 0) c.scal[2] = 0.f;
            }
            if (threadIdx.x < 8) sErr[threadIdx.x] = 0.f;
            grid.sync();
            if (__ldcg(&c.scal[8]) != 0.f) break;
        }
    }
    if (tid == 0) c.scal[10] += c.scal[9];
    // velocity update (ClothPBD.cpp:314-321)
    for (int g = tid; g < c.N; g += nth)
    {
        const float4 p = c.pos[g];
        if (p.w == 0.f) continue;
        const float4 q = c.prev[g];
        V3 vel = P.invH * (mk(p.x, p.y, p.z) - mk(q.x, q.y, q.z));
        c.vel[g] = make_float4(vel.x, vel.y, vel.z, 0.f);
    }
}

// variants the tuner chooses among: (threads per CTA, FEM tile, bend tile)
using GridKernel = void (*)(DevCloth, SolverParams, Buffers, ColourArgs, GsPlan);
static const GridKernel kGridVariants[] = {
    k_gs_grid<256, 1, 1>, k_gs_grid<256, 2, 1>, k_gs_grid<256, 2, 2>, k_gs_grid<256, 4, 2>,
    k_gs_grid<512, 1, 1>, k_gs_grid<512, 2, 1>, k_gs_grid<512, 2, 2>, k_gs_grid<512, 4, 2>,
};
static const int kGridThreads[] = {256, 256, 256, 256, 512, 512, 512, 512};
static const int kGridFemTile[] = {1, 2, 2, 4, 1, 2, 2, 4};
static const int kGridBendTile[] = {1, 1, 2, 2, 1, 1, 2, 2};

int gs_grid_variants() { return (int)(sizeof(kGridThreads) / sizeof(int)); }

void gs_grid_variant_info(int v, int& threads, int& femTile, int& bendTile)
{
    threads = kGridThreads[v]; femTile = kGridFemTile[v]; bendTile = kGridBendTile[v];
}

// resident CTAs per SM for variant v (0 if it cannot launch cooperatively)
int gs_grid_max_blocks_per_sm(int v)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kGridVariants[v], kGridThreads[v], 0) != cudaSuccess) n = 0;
    cudaGetLastError();
    return n;
}

bool launch_gs_grid(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, GsPlan plan,
                    int variant, int blocksPerSm)
{
    int dev = 0, sms = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    const int maxB = gs_grid_max_blocks_per_sm(variant);
    if (!coop || maxB < 1) return false;
    const int bps = blocksPerSm < 1 ? 1 : (blocksPerSm > maxB ? maxB : blocksPerSm);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(sms * bps);
    cfg.blockDim = dim3(kGridThreads[variant]);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeCooperative;
    at.val.cooperative = 1;
    cfg.attrs = &at; cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kGridVariants[variant], c, P, b, colour_args(b), plan) == cudaSuccess;
}

// cluster solver variants: constraints per thread 1 or 2
static const GridKernel kClusterVariants[] = {k_gs_cluster<1>, k_gs_cluster<2>};
int gs_cluster_variants() { return 2; }

int gs_cluster_size(int N, int& shift, size_t& smem)
{
    static int supported = -1;
    if (supported < 0)
    {
        supported = 0;
        for (auto k : kClusterVariants)
        {
            cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, GS_SMEM_MAX);
        }
        for (int cs : {16, 8})
        {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cs);
            cfg.blockDim = dim3(GS_THREADS);
            cfg.dynamicSmemBytes = GS_SMEM_MAX;
            cudaLaunchAttribute at;
            at.id = cudaLaunchAttributeClusterDimension;
            at.val.clusterDim.x = cs; at.val.clusterDim.y = 1; at.val.clusterDim.z = 1;
            cfg.attrs = &at; cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, kClusterVariants[1], &cfg) == cudaSuccess && clusters > 0)
            {
                supported = cs;
                break;
            }
        }
        cudaGetLastError();
    }
    if (supported == 0) return 0;
    const int cs = supported;
    int vpc = 1, sh = 0;
    while (vpc * cs < N) { vpc <<= 1; sh++; }
    if ((size_t)vpc * sizeof(float4) > 128 * 1024) return 0;
    shift = sh;
    smem = (size_t)vpc * sizeof(float4);
    return cs;
}

void launch_gs_cluster(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, GsPlan plan,
                       int clusterSize, size_t smem, int variant)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(clusterSize);
    cfg.blockDim = dim3(GS_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = clusterSize; at.val.clusterDim.y = 1; at.val.clusterDim.z = 1;
    cfg.attrs = &at; cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kClusterVariants[variant == 1 ? 1 : 0], c, P, b, colour_args(b), plan);
}

// ---------------------------------------------- band solver launchers
using BandKernel = void (*)(DevCloth, SolverParams, Buffers, ColourArgs, GsPlan, BandView);
static const BandKernel kBandVariants[] = {k_gs_band<256>, k_gs_band<512>, k_gs_band<1024>};
static const int kBandThreads[] = {256, 512, 1024};

int gs_band_variants() { return 3; }
int gs_band_threads(int variant) { return (variant >= 0 && variant < 3) ? kBandThreads[variant] : 0; }

// kernel attributes (once per process): non-portable cluster sizes, the shared memory limit
static void band_attributes()
{
    static std::once_flag once;
    std::call_once(once, [] {
        for (auto k : kBandVariants)
        {
            cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, BAND_SMEM_MAX);
        }
        cudaGetLastError();
    });
}

static cudaLaunchConfig_t band_config(int clusterSize, int threads, size_t smem, cudaStream_t s, cudaLaunchAttribute* at)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(clusterSize);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at->id = cudaLaunchAttributeClusterDimension;
    at->val.clusterDim.x = clusterSize; at->val.clusterDim.y = 1; at->val.clusterDim.z = 1;
    cfg.attrs = at; cfg.numAttrs = 1;
    return cfg;
}

// a cluster of clusterSize CTAs with smem bytes each fits for some variant
bool gs_band_fits(int clusterSize, size_t smem)
{
    if (smem > (size_t)BAND_SMEM_MAX) return false;
    band_attributes();
    bool ok = false;
    for (int v = 0; v < 3 && !ok; v++)
    {
        cudaLaunchAttribute at;
        cudaLaunchConfig_t cfg = band_config(clusterSize, kBandThreads[v], smem, nullptr, &at);
        int clusters = 0;
        ok = cudaOccupancyMaxActiveClusters(&clusters, kBandVariants[v], &cfg) == cudaSuccess && clusters > 0;
    }
    cudaGetLastError();
    return ok;
}

bool launch_gs_band(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, GsPlan plan,
                    const BandView& bv, int clusterSize, size_t smem, int variant)
{
    if (variant < 0 || variant >= 3) return false;
    band_attributes();
    cudaLaunchAttribute at;
    cudaLaunchConfig_t cfg = band_config(clusterSize, kBandThreads[variant], smem, s, &at);
    return cudaLaunchKernelEx(&cfg, kBandVariants[variant], c, P, b, colour_args(b), plan, bv) == cudaSuccess;
}

// ---------------------------------------------- per-colour path launchers
void launch_reset_link_error(cudaStream_t s, const DevCloth& c)
{
    k_reset_link_error<<<1, 32, 0, s>>>(c);
}
void launch_links(cudaStream_t s, const DevCloth& c, const SolverParams& P, int first, int count)
{
    if (count > 0) k_links<<<blocks_for(count), 256, 0, s>>>(c, P, first, count);
}
void launch_fem(cudaStream_t s, const DevCloth& c, const SolverParams& P, int first, int count)
{
    if (count > 0) k_fem<<<blocks_for(count), 256, 0, s>>>(c, P, first, count);
}
void launch_bends(cudaStream_t s, const DevCloth& c, const SolverParams& P, int first, int count, int resetErr)
{
    if (resetErr) k_reset_bend_error<<<1, 32, 0, s>>>(c);
    if (count > 0) k_bends<<<blocks_for(count), 256, 0, s>>>(c, P, first, count);
}
void launch_solve_vertex_contacts(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b)
{
    k_reset_iter_errors<<<1, 32, 0, s>>>(c);
    if (b.numVColl > 0) k_solve_vertex_contacts<<<blocks_for(c.N, 128), 128, 0, s>>>(c, P, b);
}
void launch_solve_multi_contacts(cudaStream_t s, const DevCloth& c, const SolverParams& P, const Buffers& b, int iter)
{
    k_solve_multi<<<1, 1024, 0, s>>>(c, P, b, colour_args(b));
    k_gs_exit<<<1, 32, 0, s>>>(c, P, iter);
}

// this build's entry points
static const SolverOps kSolverOps = {launch_fem, launch_links, launch_reset_link_error, launch_bends,
                                     launch_solve_vertex_contacts, launch_solve_multi_contacts, gs_cluster_size,
                                     launch_gs_cluster, gs_grid_max_blocks_per_sm, launch_gs_grid, launch_gs_band};
