// step_common.cuh — device helpers and contact-class views shared by the
// detection kernels (step_kernels.cu) and the two builds of the solver
// (solver.cuh, compiled in step_kernels.cu and in solver_fast.cu).
#pragma once
#include "launch.h"

namespace sc {

__device__ __forceinline__ V3 ld3(const float4* p, uint32_t i) { float4 a = p[i]; return mk(a.x, a.y, a.z); }
__device__ __forceinline__ void st3(float4* p, uint32_t i, V3 v)
{
    float4 a = p[i]; a.x = v.x; a.y = v.y; a.z = v.z; p[i] = a;
}
__device__ __forceinline__ void atomic_max_pos(float* addr, float v)
{
    // non-negative floats order like their bit patterns
    atomicMax((int*)addr, __float_as_int(v));
}
__device__ __forceinline__ bool gs_done(const DevCloth& c) { return c.scal[8] != 0.f; }

// Particle positions as the projections see them: plain global memory here;
// the cluster solver (gs_cluster.cu) substitutes distributed shared memory.
// the vertex colliders acting on particle i: all of them for one cloth, the
// instance's own for a batch
__device__ __forceinline__ int2 colliders_of(const DevCloth& c, const Buffers& b, int i)
{
    return b.instColl ? b.instColl[c.vInst[i]] : make_int2(0, b.numVColl);
}

struct GlobalPos
{
    float4* p;
    __device__ __forceinline__ float4 ld(uint32_t v) const { return p[v]; }
    __device__ __forceinline__ void st(uint32_t v, float4 x) const { p[v] = x; }
};

static inline int blocks_for(int n, int t = 256) { int b = (n + t - 1) / t; return b < 1 ? 1 : b; }


// one multi-particle contact class as the colouring and the solvers see it
struct ClassView
{
    int kind;          // 0 edge, 1 tri, 2 self VT, 3 self EE
    const int* count;
    int* colour;
    int* order;
    int* start;        // MAX_COLOURS + 1
};

struct ColourArgs { ClassView cls[4]; };

static inline ColourArgs colour_args(const Buffers& b)
{
    ColourArgs a;
    a.cls[0] = {0, b.ecCount, b.colour, b.order, b.colourStart};
    a.cls[1] = {1, b.tcCount, b.colour + b.ecCap, b.order + b.ecCap, b.colourStart + (MAX_COLOURS + 1)};
    a.cls[2] = {2, b.stCount, b.colour + b.ecCap + b.tcCap, b.order + b.ecCap + b.tcCap, b.colourStart + 2 * (MAX_COLOURS + 1)};
    a.cls[3] = {3, b.seCount, b.colour + b.ecCap + b.tcCap + b.stCap, b.order + b.ecCap + b.tcCap + b.stCap,
                b.colourStart + 3 * (MAX_COLOURS + 1)};
    return a;
}

} // namespace sc
