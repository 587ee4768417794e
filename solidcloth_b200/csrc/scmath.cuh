// scmath.cuh — float3 arithmetic and geometric primitives shared by the host
// set-up code and the sm_100a kernels.
//
// Floating-point contract: every expression keeps the operation order of the
// SolidCloth reference (Math/Vector3.h conventions: s*v scales each component,
// a.b = (ax*bx + ay*by) + az*bz, Normalize multiplies by the reciprocal length,
// min/max are the std:: ternaries). The library is compiled with -fmad=false and
// IEEE division / square root, so integer-valued decisions (contact regions,
// box overlaps, CCD hits) and most projections are reproduced bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>

#ifdef __CUDACC__
#define SC_HD __host__ __device__ __forceinline__
#else
#define SC_HD inline
#endif

namespace sc {

struct V3 { float x, y, z; };

SC_HD V3 mk(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
SC_HD V3 mk(float4 a) { return mk(a.x, a.y, a.z); }
SC_HD float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
SC_HD V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
SC_HD V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
SC_HD V3 operator-(V3 a) { return mk(-a.x, -a.y, -a.z); }
SC_HD V3 operator*(float s, V3 v) { return mk(s * v.x, s * v.y, s * v.z); }
SC_HD V3 operator*(V3 v, float s) { return mk(s * v.x, s * v.y, s * v.z); }
SC_HD V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
SC_HD V3& operator-=(V3& a, V3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
SC_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SC_HD V3 cross(V3 a, V3 b) { return mk(a.y * b.z - b.y * a.z, -a.x * b.z + a.z * b.x, a.x * b.y - b.x * a.y); }
SC_HD float lensq(V3 a) { return dot(a, a); }
SC_HD float len(V3 a) { return sqrtf(dot(a, a)); }
SC_HD V3 normalized(V3 a) { float l = len(a); return (1.f / l) * a; }
SC_HD float mn(float a, float b) { return (b < a) ? b : a; }   // std::min
SC_HD float mx(float a, float b) { return (a < b) ? b : a; }   // std::max
SC_HD V3 vmin(V3 a, V3 b) { return mk(mn(a.x, b.x), mn(a.y, b.y), mn(a.z, b.z)); }
SC_HD V3 vmax(V3 a, V3 b) { return mk(mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)); }
SC_HD float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
SC_HD float triple(V3 a, V3 b, V3 c) { return dot(c, cross(a, b)); }
SC_HD float signed_volume(V3 a0, V3 a1, V3 a2, V3 a3) { return triple(a1 - a0, a2 - a0, a3 - a0); }
SC_HD float clamp01(float v) { return mx(0.f, mn(1.f, v)); }

enum { TR_VERTEX_A, TR_VERTEX_B, TR_VERTEX_C, TR_EDGE_AB, TR_EDGE_AC, TR_EDGE_BC, TR_FACE_INTERIOR };
enum { ER_EDGE_INTERIOR = 0, ER_VERTEX_P1 = 1, ER_VERTEX_Q1 = 2, ER_VERTEX_P2 = 4, ER_VERTEX_Q2 = 8 };

// Segment-segment closest points (Ericson), same branch structure and operation
// order as Geometry::ClosestPtSegmSegm (Geometry/Collision3D.cpp:10-58).
SC_HD int closest_segm_segm(V3 p1, V3 q1, V3 p2, V3 q2, float& s, float& t, V3& c1, V3& c2)
{
    V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    float a = lensq(d1), e = lensq(d2), f = dot(d2, r);
    float c = dot(d1, r), b = dot(d1, d2);
    float denom = a * e - b * b;
    s = (denom != 0.f) ? clamp01((b * f - c * e) / denom) : 0.f;
    int region = ER_EDGE_INTERIOR;
    t = (b * s + f) / e;
    if (t < 0.f) { region |= ER_VERTEX_P2; t = 0.f; s = clamp01(-c / a); }
    else if (t > 1.f) { region |= ER_VERTEX_Q2; t = 1.f; s = clamp01((b - c) / a); }
    if (s == 0.f) region |= ER_VERTEX_P1;
    if (s == 1.f) region |= ER_VERTEX_Q1;
    c1 = p1 + s * d1;
    c2 = p2 + t * d2;
    return region;
}

// Point-triangle closest point by Voronoi-region walk (Ericson), as
// Geometry::ClosestPtPointTriangle (Geometry/Collision3D.cpp:62-141).
SC_HD int closest_point_triangle(V3 p, V3 a, V3 b, V3 c, V3& cp, V3& bar)
{
    bar = mk(0.f, 0.f, 0.f);
    V3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) { bar.x = 1.f; cp = a; return TR_VERTEX_A; }
    V3 bp = p - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.f && d4 <= d3) { bar.y = 1.f; cp = b; return TR_VERTEX_B; }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f)
    {
        bar.y = d1 / (d1 - d3); bar.x = 1.f - bar.y; cp = a + bar.y * ab; return TR_EDGE_AB;
    }
    V3 cpp = p - c;
    float d5 = dot(ab, cpp), d6 = dot(ac, cpp);
    if (d6 >= 0.f && d5 <= d6) { bar.z = 1.f; cp = c; return TR_VERTEX_C; }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f)
    {
        bar.z = d2 / (d2 - d6); bar.x = 1.f - bar.z; cp = a + bar.z * ac; return TR_EDGE_AC;
    }
    float va = d3 * d6 - d5 * d4;
    float d43 = d4 - d3, d56 = d5 - d6;
    if (va <= 0.f && d43 >= 0.f && d56 >= 0.f)
    {
        bar.z = d43 / (d43 + d56); bar.y = 1.f - bar.z; cp = b + bar.z * (c - b); return TR_EDGE_BC;
    }
    float denom = 1.f / (va + vb + vc);
    bar.y = vb * denom;
    bar.z = vc * denom;
    bar.x = 1.f - bar.y - bar.z;
    cp = a + ab * bar.y + ac * bar.z;
    return TR_FACE_INTERIOR;
}

// Point-segment closest point (Geometry/Collision3D.h:125-141).
SC_HD V3 closest_point_segment(V3 p, V3 a, V3 b, float& t)
{
    V3 u = b - a, v = p - a;
    t = dot(u, v) / lensq(u);
    if (t <= 0.f) { t = 0.f; return a; }
    if (t >= 1.f) { t = 1.f; return b; }
    return a + t * u;
}

// Axis-aligned box with the reference's empty-box convention (min 1e7, max -1e7,
// Geometry/Aabb3.h:11), grown with the std::min/max ternaries so that boxes are
// bit-identical to the reference's.
struct Box
{
    V3 lo, hi;
    SC_HD static Box empty() { Box b; b.lo = mk(1e7f, 1e7f, 1e7f); b.hi = mk(-1e7f, -1e7f, -1e7f); return b; }
    SC_HD void add(V3 v) { lo = vmin(lo, v); hi = vmax(hi, v); }
    SC_HD void add(const Box& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    SC_HD void extrude(float e) { V3 x = mk(e, e, e); lo -= x; hi += x; }
    // Aabb3::Distance(Vector3) (Geometry/Aabb3.h:34-45)
    SC_HD float dist(V3 v) const
    {
        float dx = (v.x < lo.x) ? lo.x - v.x : (v.x > hi.x ? v.x - hi.x : 0.f);
        float dy = (v.y < lo.y) ? lo.y - v.y : (v.y > hi.y ? v.y - hi.y : 0.f);
        float dz = (v.z < lo.z) ? lo.z - v.z : (v.z > hi.z ? v.z - hi.z : 0.f);
        return sqrtf(dx * dx + dy * dy + dz * dz);
    }
    // Aabb3::Distance(Aabb3) (Geometry/Aabb3.h:47-68)
    SC_HD float dist(const Box& b) const
    {
        float x = fabsf((b.lo.x + b.hi.x) - (lo.x + hi.x)) - ((hi.x - lo.x) + (b.hi.x - b.lo.x));
        if (x < 0) x = 0;
        float y = fabsf((b.lo.y + b.hi.y) - (lo.y + hi.y)) - ((hi.y - lo.y) + (b.hi.y - b.lo.y));
        if (y < 0) y = 0;
        float z = fabsf((b.lo.z + b.hi.z) - (lo.z + hi.z)) - ((hi.z - lo.z) + (b.hi.z - b.lo.z));
        if (z < 0) z = 0;
        return sqrtf(0.25f * (x * x + y * y + z * z));
    }
};

// Geometry::AabbOverlap3D (Geometry/Aabb3.h:72-87)
SC_HD bool overlap(const Box& a, const Box& b)
{
    if (a.hi.x < b.lo.x) return false;
    if (a.hi.y < b.lo.y) return false;
    if (a.hi.z < b.lo.z) return false;
    if (b.hi.x < a.lo.x) return false;
    if (b.hi.y < a.lo.y) return false;
    if (b.hi.z < a.lo.z) return false;
    return true;
}

// Arc cosine evaluated identically on the host and the GPU (plain float
// operations, no fused multiply-add), after Moshier's Cephes single-precision
// asinf/acosf: acos(x) = pi/2 - asin(x) for |x| <= 0.5 and
// acos(x) = 2 asin(sqrt((1 - |x|)/2)) (reflected for x < 0) otherwise, with
// asin(a) = a + a z P(z), z = a^2, P the Cephes degree-4 polynomial. About one
// ulp from the correctly rounded value; used for bend angles and normal
// weights so the library and the oracle's check mode agree bit for bit.
SC_HD float asin_core(float a)
{
    const float z = a * a;
    float p = 4.2163199048E-2f;
    p = p * z + 2.4181311049E-2f;
    p = p * z + 4.5470025998E-2f;
    p = p * z + 7.4953002686E-2f;
    p = p * z + 1.6666752422E-1f;
    return p * z * a + a;
}

SC_HD float portable_acos(float x)
{
    const float PIO2 = 1.5707963267948966192f, PI_F = 3.14159265358979323846f;
    if (x < -0.5f)
    {
        const float s = sqrtf(0.5f * (1.0f + x));
        return PI_F - 2.0f * asin_core(s);
    }
    if (x > 0.5f)
    {
        const float s = sqrtf(0.5f * (1.0f - x));
        return 2.0f * asin_core(s);
    }
    return PIO2 - asin_core(x);
}

// Integer finaliser used to give contacts pseudo-random colouring priorities
// ("lowbias32", C. Wellons, public domain).
SC_HD uint32_t mix32(uint32_t x)
{
    x ^= x >> 16; x *= 0x7feb352dU;
    x ^= x >> 15; x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

} // namespace sc
