/*
 * oracle_math.h — float3 arithmetic and geometric primitives for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product). Each primitive is
 * a restatement of the SolidCloth reference function cited beside it, written
 * so that every floating-point operation happens in the same order as there:
 * compiled with -ffp-contract=off it reproduces the reference bit for bit.
 *
 * Operation-order conventions of the reference (Math/Vector3.h):
 *   s * v        -> (s*v.x, s*v.y, s*v.z)                      (Vector3.h:238-247)
 *   u * v, dot   -> (u.x*v.x + u.y*v.y) + u.z*v.z              (Vector3.h:104-107,263-266)
 *   Normalize    -> v * (1.f / |v|)  (multiply by reciprocal)  (Vector3.h:136-141)
 *   v /= s       -> v * (1 / s)                                 (Vector3.h:96-100)
 *   vmin / vmax  -> std::min / std::max per component           (Vector3.h:295-305)
 */
#pragma once
#include <cmath>
#include <cfloat>
#include <algorithm>

namespace orc {

struct V3 { float x, y, z; };

static inline V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3 operator*(float s, V3 v) { return v3(s * v.x, s * v.y, s * v.z); }
static inline V3 operator*(V3 v, float s) { return v3(s * v.x, s * v.y, s * v.z); }
static inline V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
static inline V3& operator-=(V3& a, V3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b)
{
    /* Vector3T::Cross (Math/Vector3.h:149-152) */
    return v3(a.y * b.z - b.y * a.z, -a.x * b.z + a.z * b.x, a.x * b.y - b.x * a.y);
}
static inline float lensq(V3 a) { return dot(a, a); }
static inline float len(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 normalized(V3 a) { float l = len(a); return (1.f / l) * a; }
static inline float fmin_ref(float a, float b) { return std::min(a, b); }
static inline float fmax_ref(float a, float b) { return std::max(a, b); }
static inline V3 vmin(V3 a, V3 b) { return v3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)); }
static inline V3 vmax(V3 a, V3 b) { return v3(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)); }
static inline float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

/* triple(v1, v2, v3) = v3 . (v1 x v2)  (Math/Vector3.h:289-292) */
static inline float triple(V3 a, V3 b, V3 c) { return dot(c, cross(a, b)); }

/* Geometry::SignedVolume (Geometry/Collision3D.cpp:298-301) */
static inline float signed_volume(V3 a0, V3 a1, V3 a2, V3 a3) { return triple(a1 - a0, a2 - a0, a3 - a0); }

/* Region codes of Geometry/Collision3D.h:21-39 */
enum { TR_VERTEX_A, TR_VERTEX_B, TR_VERTEX_C, TR_EDGE_AB, TR_EDGE_AC, TR_EDGE_BC, TR_FACE_INTERIOR };
enum { ER_EDGE_INTERIOR = 0, ER_VERTEX_P1 = 1, ER_VERTEX_Q1 = 2, ER_VERTEX_P2 = 4, ER_VERTEX_Q2 = 8 };

static inline float clamp01(float v) { return std::max(0.f, std::min(1.f, v)); }

/* Geometry::ClosestPtSegmSegm (Geometry/Collision3D.cpp:10-58), Ericson's
   segment-segment closest points; returns the ER_* region bits. */
static inline int closest_pt_segm_segm(V3 p1, V3 q1, V3 p2, V3 q2, float& s, float& t, V3& c1, V3& c2)
{
    V3 d1 = q1 - p1;
    V3 d2 = q2 - p2;
    V3 r = p1 - p2;
    float a = lensq(d1);
    float e = lensq(d2);
    float f = dot(d2, r);
    float c = dot(d1, r);
    float b = dot(d1, d2);
    float denom = a * e - b * b;
    if (denom != 0.f)
        s = clamp01((b * f - c * e) / denom);
    else
        s = 0.f;
    int region = ER_EDGE_INTERIOR;
    t = (b * s + f) / e;
    if (t < 0.f)
    {
        region |= ER_VERTEX_P2;
        t = 0.f;
        s = clamp01(-c / a);
    }
    else if (t > 1.f)
    {
        region |= ER_VERTEX_Q2;
        t = 1.f;
        s = clamp01((b - c) / a);
    }
    if (s == 0.f) region |= ER_VERTEX_P1;
    if (s == 1.f) region |= ER_VERTEX_Q1;
    c1 = p1 + s * d1;
    c2 = p2 + t * d2;
    return region;
}

/* Geometry::ClosestPtPointTriangle (Geometry/Collision3D.cpp:62-141), Ericson's
   Voronoi-region walk; returns the TR_* region and barycentric coordinates. */
static inline int closest_pt_point_triangle(V3 p, V3 a, V3 b, V3 c, V3& cp, V3& bar)
{
    bar = v3(0.f, 0.f, 0.f);
    V3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) { bar.x = 1.f; cp = a; return TR_VERTEX_A; }
    V3 bp = p - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.f && d4 <= d3) { bar.y = 1.f; cp = b; return TR_VERTEX_B; }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f)
    {
        bar.y = d1 / (d1 - d3);
        bar.x = 1 - bar.y;
        cp = a + bar.y * ab;
        return TR_EDGE_AB;
    }
    V3 cpp = p - c;
    float d5 = dot(ab, cpp), d6 = dot(ac, cpp);
    if (d6 >= 0.f && d5 <= d6) { bar.z = 1.f; cp = c; return TR_VERTEX_C; }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f)
    {
        bar.z = d2 / (d2 - d6);
        bar.x = 1 - bar.z;
        cp = a + bar.z * ac;
        return TR_EDGE_AC;
    }
    float va = d3 * d6 - d5 * d4;
    float d43 = d4 - d3, d56 = d5 - d6;
    if (va <= 0.f && d43 >= 0.f && d56 >= 0.f)
    {
        bar.z = d43 / (d43 + d56);
        bar.y = 1 - bar.z;
        cp = b + bar.z * (c - b);
        return TR_EDGE_BC;
    }
    float denom = 1.f / (va + vb + vc);
    bar.y = vb * denom;
    bar.z = vc * denom;
    bar.x = 1.f - bar.y - bar.z;
    cp = a + ab * bar.y + ac * bar.z;
    return TR_FACE_INTERIOR;
}

/* Geometry::ClosestPtSegm (Geometry/Collision3D.h:125-141) */
static inline V3 closest_pt_segm(V3 p, V3 a, V3 b, float& t)
{
    V3 u = b - a, v = p - a;
    t = dot(u, v) / lensq(u);
    if (t <= 0.f) { t = 0.f; return a; }
    if (t >= 1.f) { t = 1.f; return b; }
    return a + t * u;
}

/* Geometry::Barycentric (Geometry/Collision3D.h:42-58) */
static inline V3 barycentric(V3 a, V3 b, V3 c, V3 p)
{
    V3 v0 = b - a, v1 = c - a, v2 = p - a;
    float d00 = lensq(v0), d01 = dot(v0, v1), d11 = lensq(v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    float denom = d00 * d11 - d01 * d01;
    V3 r;
    r.y = (d11 * d20 - d01 * d21) / denom;
    r.z = (d00 * d21 - d01 * d20) / denom;
    r.x = 1.f - r.y - r.z;
    return r;
}

/* Axis-aligned box with the reference's empty-box convention (Geometry/Aabb3.h:8-70). */
struct Box
{
    V3 mn, mx;
    Box() { mn = v3(1e7f, 1e7f, 1e7f); mx = v3(-1e7f, -1e7f, -1e7f); }
    void add(V3 v) { mn = vmin(mn, v); mx = vmax(mx, v); }
    void add(const Box& b) { mn = vmin(mn, b.mn); mx = vmax(mx, b.mx); }
    void extrude(float e) { V3 ext = v3(e, e, e); mn -= ext; mx += ext; }
    /* Aabb3::DistanceSquared(Vector3) / Distance (Geometry/Aabb3.h:34-45) */
    float dist(V3 v) const
    {
        float dx = (v.x < mn.x) ? mn.x - v.x : (v.x > mx.x ? v.x - mx.x : 0);
        float dy = (v.y < mn.y) ? mn.y - v.y : (v.y > mx.y ? v.y - mx.y : 0);
        float dz = (v.z < mn.z) ? mn.z - v.z : (v.z > mx.z ? v.z - mx.z : 0);
        return std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    /* Aabb3::DistanceSquared(Aabb3) / Distance (Geometry/Aabb3.h:47-68) */
    float dist(const Box& b2) const
    {
        float dxx = std::fabs((b2.mn.x + b2.mx.x) - (mn.x + mx.x)) - ((mx.x - mn.x) + (b2.mx.x - b2.mn.x));
        if (dxx < 0) dxx = 0;
        float dyy = std::fabs((b2.mn.y + b2.mx.y) - (mn.y + mx.y)) - ((mx.y - mn.y) + (b2.mx.y - b2.mn.y));
        if (dyy < 0) dyy = 0;
        float dzz = std::fabs((b2.mn.z + b2.mx.z) - (mn.z + mx.z)) - ((mx.z - mn.z) + (b2.mx.z - b2.mn.z));
        if (dzz < 0) dzz = 0;
        return std::sqrt(0.25f * (dxx * dxx + dyy * dyy + dzz * dzz));
    }
};

/* Geometry::AabbOverlap3D (Geometry/Aabb3.h:72-87) */
static inline bool overlap(const Box& a, const Box& b)
{
    if (a.mx.x < b.mn.x) return false;
    if (a.mx.y < b.mn.y) return false;
    if (a.mx.z < b.mn.z) return false;
    if (b.mx.x < a.mn.x) return false;
    if (b.mx.y < a.mn.y) return false;
    if (b.mx.z < a.mn.z) return false;
    return true;
}

} // namespace orc

namespace orc {
/* The library's portable arc cosine (same algorithm and operation order as
   solidcloth_b200/csrc/scmath.cuh: Moshier's Cephes asinf polynomial), used by
   the oracle's check mode so bends and normal weights match the GPU bit for bit. */
static inline float asin_core(float a)
{
    const float z = a * a;
    float p = 4.2163199048E-2f;
    p = p * z + 2.4181311049E-2f;
    p = p * z + 4.5470025998E-2f;
    p = p * z + 7.4953002686E-2f;
    p = p * z + 1.6666752422E-1f;
    return p * z * a + a;
}

static inline float portable_acos(float x)
{
    const float PIO2 = 1.5707963267948966192f, PI_F = 3.14159265358979323846f;
    if (x < -0.5f) return PI_F - 2.0f * asin_core(std::sqrt(0.5f * (1.0f + x)));
    if (x > 0.5f) return 2.0f * asin_core(std::sqrt(0.5f * (1.0f - x)));
    return PIO2 - asin_core(x);
}

/* acos used by the step: libm's acosf (as the reference) or the portable one */
extern bool g_portable_math;
static inline float step_acos(float x) { return g_portable_math ? portable_acos(x) : acosf(x); }
} // namespace orc
