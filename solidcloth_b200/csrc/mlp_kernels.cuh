// mlp_kernels.cuh — the learned warm start: a per-particle MLP
// 12 -> 64 -> 64 -> 64 -> 3 (GELU) that predicts the Gauss-Seidel correction of a
// substep from 1-ring features, so that plain iterations start closer to the
// solution. It has no counterpart in the reference; the plain iterations still
// run after it, and the residual target decides when a substep is done.
//
// Every contraction runs on the fifth-generation tensor cores (tc05.cuh): tiles
// of 128 particles (rows) per CTA, BF16 operands staged in shared memory, FP32
// accumulators in tensor memory, one thread issuing tcgen05.mma and the CTA
// waiting on an mbarrier that tcgen05.commit arrives on; the four warps read
// their 32 rows back with tcgen05.ld for the bias / GELU epilogue, which writes
// the next layer's BF16 operand tile. Training runs the same forward, then the
// backward on the tensor cores too: dH = dZ W (K-major operands, transposed
// weights in shared memory) and dW = dZ^T H (the activation tiles read
// MN-major, summed over the CTA's tiles in tensor memory before one atomic
// pass). Adam updates the FP32 master weights. Included by step_kernels.cu (the
// features use the collider queries defined there).
#pragma once
#include <cuda_bf16.h>
#include "tc05.cuh"

namespace sc {

constexpr int ML_IN = 12, ML_H = 64, ML_OUT = 3;
// FP32 parameter vector: W[out][in] row-major per layer, then the biases
constexpr int ML_W1 = 0, ML_B1 = ML_W1 + ML_H * ML_IN;
constexpr int ML_W2 = ML_B1 + ML_H, ML_B2 = ML_W2 + ML_H * ML_H;
constexpr int ML_W3 = ML_B2 + ML_H, ML_B3 = ML_W3 + ML_H * ML_H;
constexpr int ML_W4 = ML_B3 + ML_H, ML_B4 = ML_W4 + ML_OUT * ML_H;
constexpr int ML_NPARAM = ML_B4 + ML_OUT;     // 9347
constexpr int ML_NNORM = 2 * ML_IN + ML_OUT;  // feature mean, feature 1/std, output scale
constexpr int ML_ROWS = 128;                  // rows (particles / samples) per tile = MMA M

// instruction descriptors: M = 128 rows, N = 64 hidden units or 16 (padded outputs
// / padded inputs); forward and dH operands K-major, weight-gradient operands MN-major
constexpr uint32_t IDESC_N64 = umma_idesc(128, 64, 0, 0);
constexpr uint32_t IDESC_N16 = umma_idesc(128, 16, 0, 0);
constexpr uint32_t IDESC_GRAD_N64 = umma_idesc(128, 64, 1, 1);
constexpr uint32_t IDESC_GRAD_N16 = umma_idesc(128, 16, 1, 1);

// BF16 weights in core layout: forward operands W[out][in] (layer 1 inputs padded
// to 16, layer 4 outputs padded to 16) and, for training, the transposes
// W^T[in][out] of layers 2-4 (layer 4's outputs padded to 16)
struct __align__(128) MlpTcWeights
{
    unsigned char w1[64 * 16 * 2];
    unsigned char w2[64 * 64 * 2];
    unsigned char w3[64 * 64 * 2];
    unsigned char w4[16 * 64 * 2];
    float b1[ML_H], b2[ML_H], b3[ML_H], b4[16];
    float mean[ML_IN], istd[ML_IN], oscale[ML_OUT];
};
struct __align__(128) MlpTcTrans
{
    unsigned char w2t[64 * 64 * 2];
    unsigned char w3t[64 * 64 * 2];
    unsigned char w4t[64 * 16 * 2];
};

__device__ __forceinline__ void put_bf16(unsigned char* tile, int r, int k, int K, float v)
{
    *reinterpret_cast<__nv_bfloat16*>(tile + core_off(r, k, K)) = __float2bfloat16_rn(v);
}

__device__ __forceinline__ void mlp_tc_load(MlpTcWeights& s, MlpTcTrans* t, const float* prm, const float* norm)
{
    for (int k = threadIdx.x; k < 64 * 16; k += blockDim.x)
    {
        const int o = k / 16, i = k % 16;
        put_bf16(s.w1, o, i, 16, i < ML_IN ? prm[ML_W1 + o * ML_IN + i] : 0.f);
    }
    for (int k = threadIdx.x; k < 64 * 64; k += blockDim.x)
    {
        const int o = k / 64, i = k % 64;
        put_bf16(s.w2, o, i, 64, prm[ML_W2 + k]);
        put_bf16(s.w3, o, i, 64, prm[ML_W3 + k]);
        if (t)
        {
            put_bf16(t->w2t, i, o, 64, prm[ML_W2 + k]);
            put_bf16(t->w3t, i, o, 64, prm[ML_W3 + k]);
        }
    }
    for (int k = threadIdx.x; k < 16 * 64; k += blockDim.x)
    {
        const int o = k / 64, i = k % 64;
        const float w = o < ML_OUT ? prm[ML_W4 + o * ML_H + i] : 0.f;
        put_bf16(s.w4, o, i, 64, w);
        if (t) put_bf16(t->w4t, i, o, 16, w);
    }
    for (int k = threadIdx.x; k < ML_H; k += blockDim.x)
    {
        s.b1[k] = prm[ML_B1 + k]; s.b2[k] = prm[ML_B2 + k]; s.b3[k] = prm[ML_B3 + k];
    }
    if (threadIdx.x < 16) s.b4[threadIdx.x] = threadIdx.x < ML_OUT ? prm[ML_B4 + threadIdx.x] : 0.f;
    if (threadIdx.x < ML_IN) { s.mean[threadIdx.x] = norm[threadIdx.x]; s.istd[threadIdx.x] = norm[ML_IN + threadIdx.x]; }
    if (threadIdx.x < ML_OUT) s.oscale[threadIdx.x] = norm[2 * ML_IN + threadIdx.x];
}

// GELU, tanh form, and its derivative
__device__ __forceinline__ float gelu(float x)
{
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float x)
{
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * 0.7978845608028654f * (1.f + 3.f * 0.044715f * x * x);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x = lo (lower 16 bits)
    return *reinterpret_cast<const uint32_t*>(&v);
}


// this thread's row of a 16-column operand tile (K = 16) from 16 floats
__device__ __forceinline__ void put_row16(unsigned char* tile, int r, const float* x)
{
    uint4 q0, q1;
    q0.x = pack_bf16(x[0], x[1]); q0.y = pack_bf16(x[2], x[3]); q0.z = pack_bf16(x[4], x[5]); q0.w = pack_bf16(x[6], x[7]);
    q1.x = pack_bf16(x[8], x[9]); q1.y = pack_bf16(x[10], x[11]); q1.z = pack_bf16(x[12], x[13]); q1.w = pack_bf16(x[14], x[15]);
    *reinterpret_cast<uint4*>(tile + core_off(r, 0, 16)) = q0;
    *reinterpret_cast<uint4*>(tile + core_off(r, 8, 16)) = q1;
}

// 32 accumulator columns of this thread's row (tensor memory at taddr) plus bias,
// through GELU, into columns [c0, c0 + 32) of row r of a K-column operand tile
__device__ __forceinline__ void epilogue_gelu32(uint32_t taddr, const float* bias, unsigned char* tile, int r, int c0, int K)
{
    uint32_t v[32];
    tc_ld32(taddr, v);
    tc_wait_ld();
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
        float h[8];
#pragma unroll
        for (int j = 0; j < 8; j++) h[j] = gelu(__uint_as_float(v[8 * c + j]) + bias[c0 + 8 * c + j]);
        uint4 q;
        q.x = pack_bf16(h[0], h[1]); q.y = pack_bf16(h[2], h[3]); q.z = pack_bf16(h[4], h[5]); q.w = pack_bf16(h[6], h[7]);
        *reinterpret_cast<uint4*>(tile + core_off(r, c0 + 8 * c, K)) = q;
    }
}

// Shared state of a CTA driving the tensor cores: the mbarrier the commits arrive
// on, its next parity, and the tensor-memory base.
struct TcCtx
{
    uint32_t mbar, phase, tmem;
    bool ok;
    __device__ __forceinline__ bool wait()
    {
        const bool done = mbar_wait(mbar, phase);
        phase ^= 1u;
        tc_fence_after();
        return __syncthreads_and(done) != 0;   // every thread takes the same path
    }
};

// Forward of the CTA's 128-row tile whose normalised inputs (BF16, K = 16) are
// already in x: hidden layers into tensor-memory columns zcol[0..2] (pre-
// activations, no bias), their GELU outputs as operand tiles h[0..2] (each may be
// the same buffer when they need not survive), outputs into column ycol. Returns
// false if a wait gave up.
__device__ __forceinline__ bool mlp_tc_forward(TcCtx& t, const MlpTcWeights& s, unsigned char* x,
                                               unsigned char* const* h, const uint32_t* zcol, uint32_t ycol)
{
    const int r = threadIdx.x;
    const uint32_t lanes = tmem_lane_base(t.tmem);
    tc_sync_for_mma();
    if (r == 0)
    {
        umma_bf16(t.tmem + zcol[0], desc_kmajor(smem_addr(x), 16), desc_kmajor(smem_addr(s.w1), 16), IDESC_N64, 0);
        umma_commit(t.mbar);
    }
    if (!t.wait()) return false;
    const float* bias[3] = {s.b1, s.b2, s.b3};
    const unsigned char* w[3] = {s.w2, s.w3, s.w4};
    for (int l = 0; l < 3; l++)
    {
        epilogue_gelu32(lanes + zcol[l], bias[l], h[l], r, 0, 64);
        epilogue_gelu32(lanes + zcol[l] + 32, bias[l], h[l], r, 32, 64);
        tc_sync_for_mma();
        if (r == 0)
        {
            const uint32_t dst = l < 2 ? zcol[l + 1] : ycol;
            for (int ks = 0; ks < 4; ks++)
                umma_bf16(t.tmem + dst, desc_kmajor(smem_addr(h[l]) + 256 * ks, 64), desc_kmajor(smem_addr(w[l]) + 256 * ks, 64),
                          l < 2 ? IDESC_N64 : IDESC_N16, ks > 0);
            umma_commit(t.mbar);
        }
        if (!t.wait()) return false;
    }
    return true;
}

// the outputs (before the output scale) of this thread's row
__device__ __forceinline__ void mlp_tc_outputs(const TcCtx& t, const MlpTcWeights& s, uint32_t ycol, float* y)
{
    uint32_t v[16];
    tc_ld16(tmem_lane_base(t.tmem) + ycol, v);
    tc_wait_ld();
    for (int k = 0; k < ML_OUT; k++) y[k] = __uint_as_float(v[k]) + s.b4[k];
}

// CTA set-up of the inference kernels: weights, mbarrier, 128 tensor-memory columns
struct __align__(128) MlpTcInferSmem
{
    MlpTcWeights w;
    unsigned char x[ML_ROWS * 16 * 2];
    unsigned char h[ML_ROWS * 64 * 2];
    unsigned long long mbar;
    uint32_t tmemSlot;
};

__device__ __forceinline__ TcCtx mlp_tc_begin(MlpTcInferSmem& s, uint32_t cols)
{
    TcCtx t;
    if (threadIdx.x == 0) mbar_init(smem_addr(&s.mbar), 1);
    t.tmem = tmem_alloc(&s.tmemSlot, cols);    // includes a CTA barrier
    t.mbar = smem_addr(&s.mbar);
    t.phase = 0;
    t.ok = true;
    return t;
}

// ------------------------------------------------------------- features
// The 12 inputs of particle i after the substep's prediction: predicted minus
// previous position (3), velocity (3), mean strain of its incident edges (1),
// collision-mesh normal (3), signed distance to its first sphere / SDF collider
// (1, clamped to +-1 m), and — the twelfth, chosen here — the previous
// substep's solver correction along that normal (1): corrections are coherent
// in time, and the normal component carries the contact response.
__device__ __forceinline__ void ml_features(const DevCloth& c, const Buffers& b, int i, float* f)
{
    const float4 p = c.pos[i], q = c.prev[i], v = c.vel[i];
    f[0] = p.x - q.x; f[1] = p.y - q.y; f[2] = p.z - q.z;
    f[3] = v.x; f[4] = v.y; f[5] = v.z;
    float strain = 0.f;
    const int r0 = c.eRingStart[i], r1 = c.eRingStart[i + 1];
    for (int k = r0; k < r1; k++)
    {
        const int e = c.eRing[k];
        const int4 ed = c.edge[e];
        const int j = ed.x == i ? ed.y : ed.x;
        const float4 pj = c.pos[j];
        const float dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
        strain += sqrtf(dx * dx + dy * dy + dz * dz) / c.edgeRest[e] - 1.f;
    }
    f[6] = r1 > r0 ? strain / (float)(r1 - r0) : 0.f;
    const float4 n = c.prevN[i];
    f[7] = n.x; f[8] = n.y; f[9] = n.z;
    float dist = 1.f;
    const int2 cr = colliders_of(c, b, i);
    for (int ci = cr.x; ci < cr.x + cr.y; ci++)
    {
        const VColl& g = b.vcoll[ci];
        if (g.type != 3 && g.type != 7) continue;
        V3 cp, nn; int fe;
        dist = query_point(g, mk(p.x, p.y, p.z), cp, nn, fe);
        break;
    }
    f[10] = fminf(1.f, fmaxf(-1.f, dist));
    f[11] = c.lastCorr[i];
}

struct MlpArgs
{
    const float* prm;    // ML_NPARAM FP32 master weights
    const float* norm;   // ML_NNORM
};

// warm start: features -> MLP -> position correction, tiles of 128 particles
// (one per thread), CTAs persistent over the tiles; pinned particles are left
// alone. A wait that gives up sets ST_TC_TIMEOUT and ends the CTA's work.
__global__ void __launch_bounds__(128) k_mlp_warm(DevCloth c, Buffers b, MlpArgs ml)
{
    __shared__ MlpTcInferSmem s;
    mlp_tc_load(s.w, nullptr, ml.prm, ml.norm);
    TcCtx t = mlp_tc_begin(s, 128);
    unsigned char* hs[3] = {s.h, s.h, s.h};
    const uint32_t zc[3] = {0, 64, 0};
    const int tiles = (c.N + ML_ROWS - 1) / ML_ROWS;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x)
    {
        const int i = tile * ML_ROWS + (int)threadIdx.x;
        float f[16];
        if (i < c.N) ml_features(c, b, i, f);
#pragma unroll
        for (int k = 0; k < 16; k++) f[k] = (i < c.N && k < ML_IN) ? (f[k] - s.w.mean[k]) * s.w.istd[k] : 0.f;
        put_row16(s.x, threadIdx.x, f);
        if (!mlp_tc_forward(t, s.w, s.x, hs, zc, 64))
        {
            if (threadIdx.x == 0) atomicOr(c.status, ST_TC_TIMEOUT);
            break;
        }
        float y[ML_OUT];
        mlp_tc_outputs(t, s.w, 64, y);
        if (i < c.N)
        {
            float4 p = c.pos[i];
            if (p.w > 0.f)
            {
                p.x += y[0] * s.w.oscale[0];
                p.y += y[1] * s.w.oscale[1];
                p.z += y[2] * s.w.oscale[2];
                c.pos[i] = p;
            }
        }
    }
    tmem_free(t.tmem, 128);
}

// the predicted positions, and (sample recording) every particle's raw features
__global__ void k_mlp_features(DevCloth c, Buffers b, float* feat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    if (feat)
    {
        float f[ML_IN];
        ml_features(c, b, i, f);
        for (int k = 0; k < ML_IN; k++) feat[(size_t)i * ML_IN + k] = f[k];
    }
    c.xpred[i] = c.pos[i];
}

// the substep's correction (solved minus predicted positions): its normal
// component for the next substep's features, and (sample recording) the target
__global__ void k_mlp_targets(DevCloth c, float* target)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const float4 p = c.pos[i], q = c.xpred[i], n = c.prevN[i];
    const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
    c.lastCorr[i] = dx * n.x + dy * n.y + dz * n.z;
    if (target) { target[3 * (size_t)i] = dx; target[3 * (size_t)i + 1] = dy; target[3 * (size_t)i + 2] = dz; }
}

// forward over raw feature rows (S x 12) -> outputs (S x 3, output scale applied)
__global__ void __launch_bounds__(128) k_mlp_forward(const float* X, int S, MlpArgs ml, float* Y, int* status)
{
    __shared__ MlpTcInferSmem s;
    mlp_tc_load(s.w, nullptr, ml.prm, ml.norm);
    TcCtx t = mlp_tc_begin(s, 128);
    unsigned char* hs[3] = {s.h, s.h, s.h};
    const uint32_t zc[3] = {0, 64, 0};
    const int tiles = (S + ML_ROWS - 1) / ML_ROWS;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x)
    {
        const int r = tile * ML_ROWS + (int)threadIdx.x;
        float f[16];
#pragma unroll
        for (int k = 0; k < 16; k++) f[k] = (r < S && k < ML_IN) ? (X[(size_t)r * ML_IN + k] - s.w.mean[k]) * s.w.istd[k] : 0.f;
        put_row16(s.x, threadIdx.x, f);
        if (!mlp_tc_forward(t, s.w, s.x, hs, zc, 64))
        {
            if (threadIdx.x == 0 && status) atomicOr(status, 1);
            break;
        }
        float y[ML_OUT];
        mlp_tc_outputs(t, s.w, 64, y);
        if (r < S)
            for (int k = 0; k < ML_OUT; k++) Y[(size_t)r * ML_OUT + k] = y[k] * s.w.oscale[k];
    }
    tmem_free(t.tmem, 128);
}

// ------------------------------------------------------------ training
// Sum over a warp of 64 per-lane values: a butterfly in which each step halves
// the columns a lane keeps, so that lane l ends with the sums of columns 2l and
// 2l + 1 (62 shuffles instead of 64 x 5).
__device__ __forceinline__ float2 warp_colsum64(const float (&v)[64])
{
    const int lane = threadIdx.x & 31;
    float a[32];
    {
        const bool hi = lane & 16;
#pragma unroll
        for (int j = 0; j < 32; j++)
        {
            const float keep = hi ? v[j + 32] : v[j], send = hi ? v[j] : v[j + 32];
            a[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
    }
    float b16[16];
    {
        const bool hi = lane & 8;
#pragma unroll
        for (int j = 0; j < 16; j++)
        {
            const float keep = hi ? a[j + 16] : a[j], send = hi ? a[j] : a[j + 16];
            b16[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
    }
    float c8[8];
    {
        const bool hi = lane & 4;
#pragma unroll
        for (int j = 0; j < 8; j++)
        {
            const float keep = hi ? b16[j + 8] : b16[j], send = hi ? b16[j] : b16[j + 8];
            c8[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
        }
    }
    float d4[4];
    {
        const bool hi = lane & 2;
#pragma unroll
        for (int j = 0; j < 4; j++)
        {
            const float keep = hi ? c8[j + 4] : c8[j], send = hi ? c8[j] : c8[j + 4];
            d4[j] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
        }
    }
    float e2[2];
    {
        const bool hi = lane & 1;
#pragma unroll
        for (int j = 0; j < 2; j++)
        {
            const float keep = hi ? d4[j + 2] : d4[j], send = hi ? d4[j] : d4[j + 2];
            e2[j] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
        }
    }
    return make_float2(e2[0], e2[1]);
}

// dZ = dH * gelu'(Z + b) for this thread's row: dH and Z (no bias) from tensor
// memory, dZ as BF16 into columns 0..63 of row r of the 128-column tile d, and
// its per-column sums over the warp into bsum (lane l: columns 2l, 2l + 1)
__device__ __forceinline__ void epilogue_dz(uint32_t lanes, uint32_t dhCol, uint32_t zCol, const float* bias,
                                            unsigned char* d, int r, float2& bsum)
{
    float dz[64];
#pragma unroll
    for (int half = 0; half < 2; half++)
    {
        uint32_t vh[32], vz[32];
        tc_ld32(lanes + dhCol + 32 * half, vh);
        tc_ld32(lanes + zCol + 32 * half, vz);
        tc_wait_ld();
#pragma unroll
        for (int j = 0; j < 32; j++)
            dz[32 * half + j] = __uint_as_float(vh[j]) * gelu_grad(__uint_as_float(vz[j]) + bias[32 * half + j]);
    }
#pragma unroll
    for (int c = 0; c < 8; c++)
    {
        uint4 q;
        q.x = pack_bf16(dz[8 * c], dz[8 * c + 1]); q.y = pack_bf16(dz[8 * c + 2], dz[8 * c + 3]);
        q.z = pack_bf16(dz[8 * c + 4], dz[8 * c + 5]); q.w = pack_bf16(dz[8 * c + 6], dz[8 * c + 7]);
        *reinterpret_cast<uint4*>(d + core_off(r, 8 * c, 128)) = q;
    }
    const float2 s2 = warp_colsum64(dz);
    bsum.x += s2.x;
    bsum.y += s2.y;
}

// Tensor-memory columns of the training kernel (512 allocated)
constexpr uint32_t TM_Z1 = 0, TM_Z2 = 64, TM_Z3 = 128, TM_Y = 192, TM_DH = 208;
constexpr uint32_t TM_DW4 = 272, TM_DW3 = 336, TM_DW2 = 400, TM_DW1 = 464;

struct __align__(128) MlpTcTrainSmem
{
    MlpTcWeights w;
    MlpTcTrans t;
    unsigned char x[ML_ROWS * 16 * 2];
    unsigned char h1[ML_ROWS * 64 * 2], h2[ML_ROWS * 64 * 2], h3[ML_ROWS * 64 * 2];
    // dY / dZ tile, 128 columns: 0..63 in use, 64..127 zero (the padded rows of
    // the M = 128 weight-gradient products)
    unsigned char d[ML_ROWS * 128 * 2];
    unsigned long long mbar;
    uint32_t tmemSlot;
};

// Gradients of the mean squared error between the network's output and
// target / output scale (mean over S x 3 elements), accumulated into grad[] and
// loss[0] (both zeroed by the caller). CTAs are persistent over 128-row tiles;
// the weight gradients of all their tiles are summed in tensor memory and added
// to grad[] once per CTA. A wait that gives up sets *status (if given).
__global__ void __launch_bounds__(128) k_mlp_grad(const float* X, const float* T, int S, MlpArgs ml, float* grad,
                                                  float* loss, int* status)
{
    extern __shared__ __align__(1024) unsigned char dyn[];
    MlpTcTrainSmem& s = *reinterpret_cast<MlpTcTrainSmem*>(dyn);
    mlp_tc_load(s.w, &s.t, ml.prm, ml.norm);
    for (int k = threadIdx.x; k < ML_ROWS * 128 * 2 / 16; k += blockDim.x)
        reinterpret_cast<uint4*>(s.d)[k] = make_uint4(0u, 0u, 0u, 0u);
    TcCtx t;
    if (threadIdx.x == 0) mbar_init(smem_addr(&s.mbar), 1);
    t.tmem = tmem_alloc(&s.tmemSlot, 512);
    t.mbar = smem_addr(&s.mbar);
    t.phase = 0;
    const int r = threadIdx.x, lane = r & 31;
    const uint32_t lanes = tmem_lane_base(t.tmem);
    const float inv = 1.f / (float)(S * ML_OUT);
    float2 db1 = make_float2(0.f, 0.f), db2 = db1, db3 = db1;
    float db4[ML_OUT] = {0.f, 0.f, 0.f}, lsum = 0.f;
    unsigned char* hs[3] = {s.h1, s.h2, s.h3};
    const uint32_t zc[3] = {TM_Z1, TM_Z2, TM_Z3};
    const int tiles = (S + ML_ROWS - 1) / ML_ROWS;
    bool first = true, ok = true;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x)
    {
        const int row = tile * ML_ROWS + r;
        const bool live = row < S;
        float f[16];
#pragma unroll
        for (int k = 0; k < 16; k++) f[k] = (live && k < ML_IN) ? (X[(size_t)row * ML_IN + k] - s.w.mean[k]) * s.w.istd[k] : 0.f;
        put_row16(s.x, r, f);
        if (!(ok = mlp_tc_forward(t, s.w, s.x, hs, zc, TM_Y))) break;
        // output layer: dL/dy (zero for rows past S) into dY columns 0..2
        float y[ML_OUT], dy[16];
        mlp_tc_outputs(t, s.w, TM_Y, y);
#pragma unroll
        for (int k = 0; k < 16; k++) dy[k] = 0.f;
        for (int k = 0; k < ML_OUT; k++)
            if (live)
            {
                const float e = y[k] - T[(size_t)row * ML_OUT + k] / s.w.oscale[k];
                lsum += e * e * inv;
                dy[k] = 2.f * e * inv;
            }
        for (int k = 0; k < ML_OUT; k++)
        {
            float v = dy[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            db4[k] += v;
        }
        {
            uint4 q0, q1;
            q0.x = pack_bf16(dy[0], dy[1]); q0.y = pack_bf16(dy[2], 0.f); q0.z = 0u; q0.w = 0u;
            q1 = make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(s.d + core_off(r, 0, 128)) = q0;
            for (int c = 1; c < 8; c++) *reinterpret_cast<uint4*>(s.d + core_off(r, 8 * c, 128)) = q1;
        }
        // dH3 = dY W4 (K = 16) and dW4 += dY^T H3 (sum over the tile's rows)
        tc_sync_for_mma();
        if (r == 0)
        {
            umma_bf16(t.tmem + TM_DH, desc_kmajor(smem_addr(s.d), 128), desc_kmajor(smem_addr(s.t.w4t), 16), IDESC_N64, 0);
            for (int ks = 0; ks < ML_ROWS / 16; ks++)
                umma_bf16(t.tmem + TM_DW4, desc_mnmajor(smem_addr(s.d) + ks * 2 * 2048, 128),
                          desc_mnmajor(smem_addr(s.h3) + ks * 2 * 1024, 64), IDESC_GRAD_N64, (!first || ks > 0) ? 1u : 0u);
            umma_commit(t.mbar);
        }
        if (!(ok = t.wait())) break;
        // hidden layers 3, 2, 1: dZ, then dH of the layer below and dW += dZ^T H
        const float* bias[3] = {s.w.b1, s.w.b2, s.w.b3};
        float2* dbs[3] = {&db1, &db2, &db3};
        const unsigned char* wt[3] = {nullptr, s.t.w2t, s.t.w3t};
        const uint32_t dwc[3] = {TM_DW1, TM_DW2, TM_DW3};
        for (int l = 2; l >= 0 && ok; l--)
        {
            epilogue_dz(lanes, TM_DH, zc[l], bias[l], s.d, r, *dbs[l]);
            tc_sync_for_mma();
            if (r == 0)
            {
                if (l > 0)
                    for (int ks = 0; ks < 4; ks++)
                        umma_bf16(t.tmem + TM_DH, desc_kmajor(smem_addr(s.d) + 256 * ks, 128),
                                  desc_kmajor(smem_addr(wt[l]) + 256 * ks, 64), IDESC_N64, ks > 0);
                const unsigned char* hb = l > 0 ? hs[l - 1] : s.x;
                const int hk = l > 0 ? 64 : 16;
                for (int ks = 0; ks < ML_ROWS / 16; ks++)
                    umma_bf16(t.tmem + dwc[l], desc_mnmajor(smem_addr(s.d) + ks * 2 * 2048, 128),
                              desc_mnmajor(smem_addr(hb) + ks * 2 * hk * 16, hk), l > 0 ? IDESC_GRAD_N64 : IDESC_GRAD_N16,
                              (!first || ks > 0) ? 1u : 0u);
                umma_commit(t.mbar);
            }
            ok = t.wait();
        }
        first = false;
    }
    if (!ok && threadIdx.x == 0 && status) atomicOr(status, 1);
    // this CTA's sums: weight gradients (rows 0..63 = output units: warps 0, 1),
    // bias gradients (lane l of each warp: units 2l, 2l + 1), loss
    if (ok && !first)
    {
        // tensor-memory loads are warp-collective: every warp loads, the warps
        // holding rows 0..63 (output units) add them
        const bool mine = r < 64;
        uint32_t v[32];
        for (int half = 0; half < 2; half++)
        {
            tc_ld32(lanes + TM_DW3 + 32 * half, v);
            tc_wait_ld();
            if (mine) for (int j = 0; j < 32; j++) atomicAdd(&grad[ML_W3 + r * ML_H + 32 * half + j], __uint_as_float(v[j]));
            tc_ld32(lanes + TM_DW2 + 32 * half, v);
            tc_wait_ld();
            if (mine) for (int j = 0; j < 32; j++) atomicAdd(&grad[ML_W2 + r * ML_H + 32 * half + j], __uint_as_float(v[j]));
            tc_ld32(lanes + TM_DW4 + 32 * half, v);
            tc_wait_ld();
            if (r < ML_OUT) for (int j = 0; j < 32; j++) atomicAdd(&grad[ML_W4 + r * ML_H + 32 * half + j], __uint_as_float(v[j]));
        }
        uint32_t v16[16];
        tc_ld16(lanes + TM_DW1, v16);
        tc_wait_ld();
        if (mine) for (int j = 0; j < ML_IN; j++) atomicAdd(&grad[ML_W1 + r * ML_IN + j], __uint_as_float(v16[j]));
    }
    if (ok && !first)
    {
        atomicAdd(&grad[ML_B1 + 2 * lane], db1.x); atomicAdd(&grad[ML_B1 + 2 * lane + 1], db1.y);
        atomicAdd(&grad[ML_B2 + 2 * lane], db2.x); atomicAdd(&grad[ML_B2 + 2 * lane + 1], db2.y);
        atomicAdd(&grad[ML_B3 + 2 * lane], db3.x); atomicAdd(&grad[ML_B3 + 2 * lane + 1], db3.y);
        if (lane == 0)
            for (int k = 0; k < ML_OUT; k++) atomicAdd(&grad[ML_B4 + k], db4[k]);
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0) atomicAdd(loss, lsum);
    }
    tmem_free(t.tmem, 512);
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; m and v follow the parameters
__global__ void k_adam(float* prm, const float* grad, float* m, float* v, int step, float lr, float b1, float b2, float eps)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ML_NPARAM) return;
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.f - b1) * g;
    const float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk; v[k] = vk;
    const float mh = mk / (1.f - powf(b1, (float)step)), vh = vk / (1.f - powf(b2, (float)step));
    prm[k] -= lr * mh / (sqrtf(vh) + eps);
}

} // namespace sc
