// mlp_kernels.cuh — the learned warm start: a per-particle MLP
// 12 -> 64 -> 64 -> 64 -> 3 (GELU) that predicts the Gauss-Seidel correction of a
// substep from 1-ring features, so that plain iterations start closer to the
// solution. It has no counterpart in the reference; the plain solver stays the
// fallback and the judge (the residual decides when a substep is done).
//
// Forward on the tensor cores: BF16 weights and activations, FP32 accumulation,
// mma.sync m16n8k16 (a warp owns 16-row tiles of particles; a layer's FP32
// accumulator fragments are packed in registers into the next layer's BF16
// operand fragments, so activations never leave the warp). Backward in FP32
// from shared memory; weight gradients accumulate over the grid with atomics;
// Adam updates the FP32 master weights. Included by step_kernels.cu (it uses the
// collider queries defined there).
#pragma once
#include <cuda_bf16.h>

namespace sc {

constexpr int ML_IN = 12, ML_H = 64, ML_OUT = 3;
// FP32 parameter vector: W[out][in] row-major per layer, then the biases
constexpr int ML_W1 = 0, ML_B1 = ML_W1 + ML_H * ML_IN;
constexpr int ML_W2 = ML_B1 + ML_H, ML_B2 = ML_W2 + ML_H * ML_H;
constexpr int ML_W3 = ML_B2 + ML_H, ML_B3 = ML_W3 + ML_H * ML_H;
constexpr int ML_W4 = ML_B3 + ML_H, ML_B4 = ML_W4 + ML_OUT * ML_H;
constexpr int ML_NPARAM = ML_B4 + ML_OUT;     // 9347
constexpr int ML_NNORM = 2 * ML_IN + ML_OUT;  // feature mean, feature 1/std, output scale

// BF16 weights in shared memory, [out][in] with in padded to 16 (layer 1) and out
// padded to 8 (layer 4): the B fragment pairs (k, k+1) of one n are one 32-bit word
struct MlpSmem
{
    __nv_bfloat16 w1[ML_H * 16];
    __nv_bfloat16 w2[ML_H * ML_H];
    __nv_bfloat16 w3[ML_H * ML_H];
    __nv_bfloat16 w4[8 * ML_H];
    float b1[ML_H], b2[ML_H], b3[ML_H], b4[8];
    float mean[ML_IN], istd[ML_IN], oscale[ML_OUT];
};

__device__ __forceinline__ void mlp_load_smem(MlpSmem& s, const float* prm, const float* norm)
{
    for (int k = threadIdx.x; k < ML_H * 16; k += blockDim.x)
    {
        const int o = k / 16, i = k % 16;
        s.w1[k] = __float2bfloat16_rn(i < ML_IN ? prm[ML_W1 + o * ML_IN + i] : 0.f);
    }
    for (int k = threadIdx.x; k < ML_H * ML_H; k += blockDim.x)
    {
        s.w2[k] = __float2bfloat16_rn(prm[ML_W2 + k]);
        s.w3[k] = __float2bfloat16_rn(prm[ML_W3 + k]);
    }
    for (int k = threadIdx.x; k < 8 * ML_H; k += blockDim.x)
    {
        const int o = k / ML_H, i = k % ML_H;
        s.w4[k] = __float2bfloat16_rn(o < ML_OUT ? prm[ML_W4 + o * ML_H + i] : 0.f);
    }
    for (int k = threadIdx.x; k < ML_H; k += blockDim.x)
    {
        s.b1[k] = prm[ML_B1 + k]; s.b2[k] = prm[ML_B2 + k]; s.b3[k] = prm[ML_B3 + k];
    }
    if (threadIdx.x < 8) s.b4[threadIdx.x] = threadIdx.x < ML_OUT ? prm[ML_B4 + threadIdx.x] : 0.f;
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

// D += A (16x16 bf16, row) * B (16x8 bf16, col), FP32 accumulate
__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One dense layer for a warp's 16-row tile: acc[NT][4] = A[KT] * W^T + bias.
// Fragment coordinates (lane = 4 g + t): A a0 (g, 2t..2t+1) a1 (g+8, 2t..)
// a2 (g, 2t+8..) a3 (g+8, 2t+8..); B b0 (k = 2t.., n = g) b1 (k = 2t+8.., n = g);
// C c0,c1 (g, 2t..2t+1) c2,c3 (g+8, 2t..2t+1).
template <int KT, int NT>
__device__ __forceinline__ void mlp_layer(const uint32_t (&a)[KT][4], const __nv_bfloat16* w, const float* bias, float (&acc)[NT][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    constexpr int KP = KT * 16;
#pragma unroll
    for (int j = 0; j < NT; j++)
    {
        acc[j][0] = acc[j][2] = bias[8 * j + 2 * t];
        acc[j][1] = acc[j][3] = bias[8 * j + 2 * t + 1];
        const __nv_bfloat16* col = w + (8 * j + g) * KP + 2 * t;
#pragma unroll
        for (int kt = 0; kt < KT; kt++)
        {
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(col + 16 * kt);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(col + 16 * kt + 8);
            mma_bf16(acc[j], a[kt], b0, b1);
        }
    }
}

// accumulator fragments (after GELU) -> next layer's operand fragments
template <int NT>
__device__ __forceinline__ void acc_to_operand(const float (&acc)[NT][4], uint32_t (&a)[NT / 2][4])
{
#pragma unroll
    for (int j = 0; j < NT; j++)
    {
        const uint32_t lo = pack_bf16(gelu(acc[j][0]), gelu(acc[j][1]));
        const uint32_t hi = pack_bf16(gelu(acc[j][2]), gelu(acc[j][3]));
        if (j & 1) { a[j >> 1][2] = lo; a[j >> 1][3] = hi; }
        else { a[j >> 1][0] = lo; a[j >> 1][1] = hi; }
    }
}

// Forward for the warp's 16 rows whose normalised inputs are x[16][16] (FP32,
// shared memory, columns >= 12 zero). out[16][3] gets the output (before the
// output scale). When z is given (training), the pre-activations of the three
// hidden layers are stored to z[layer][16][64].
__device__ __forceinline__ void mlp_forward_tile(const MlpSmem& s, const float* x, float* out, float* z)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a0[1][4];
    a0[0][0] = pack_bf16(x[g * 16 + 2 * t], x[g * 16 + 2 * t + 1]);
    a0[0][1] = pack_bf16(x[(g + 8) * 16 + 2 * t], x[(g + 8) * 16 + 2 * t + 1]);
    a0[0][2] = pack_bf16(x[g * 16 + 2 * t + 8], x[g * 16 + 2 * t + 9]);
    a0[0][3] = pack_bf16(x[(g + 8) * 16 + 2 * t + 8], x[(g + 8) * 16 + 2 * t + 9]);
    float acc[8][4];
    uint32_t a[4][4];
    auto keep = [&](int layer) {
        if (!z) return;
        float* zz = z + layer * 16 * ML_H;
#pragma unroll
        for (int j = 0; j < 8; j++)
        {
            zz[g * ML_H + 8 * j + 2 * t] = acc[j][0]; zz[g * ML_H + 8 * j + 2 * t + 1] = acc[j][1];
            zz[(g + 8) * ML_H + 8 * j + 2 * t] = acc[j][2]; zz[(g + 8) * ML_H + 8 * j + 2 * t + 1] = acc[j][3];
        }
    };
    mlp_layer<1, 8>(a0, s.w1, s.b1, acc);
    keep(0);
    acc_to_operand<8>(acc, a);
    mlp_layer<4, 8>(a, s.w2, s.b2, acc);
    keep(1);
    acc_to_operand<8>(acc, a);
    mlp_layer<4, 8>(a, s.w3, s.b3, acc);
    keep(2);
    acc_to_operand<8>(acc, a);
    float o[1][4];
    mlp_layer<4, 1>(a, s.w4, s.b4, o);
    if (2 * t < ML_OUT) { out[g * 4 + 2 * t] = o[0][0]; out[(g + 8) * 4 + 2 * t] = o[0][2]; }
    if (2 * t + 1 < ML_OUT) { out[g * 4 + 2 * t + 1] = o[0][1]; out[(g + 8) * 4 + 2 * t + 1] = o[0][3]; }
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

// warm start: features -> MLP -> position correction, 128 particles per CTA
// (4 warps x 2 tiles of 16); pinned particles are left alone
__global__ void __launch_bounds__(128) k_mlp_warm(DevCloth c, Buffers b, MlpArgs ml)
{
    __shared__ MlpSmem s;
    __shared__ float sx[128 * 16];
    __shared__ float sy[128 * 4];
    mlp_load_smem(s, ml.prm, ml.norm);
    __syncthreads();
    const int i = blockIdx.x * 128 + threadIdx.x;
    float f[16];
    if (i < c.N) ml_features(c, b, i, f);
    else for (int k = 0; k < ML_IN; k++) f[k] = 0.f;
#pragma unroll
    for (int k = 0; k < ML_IN; k++) sx[threadIdx.x * 16 + k] = (f[k] - s.mean[k]) * s.istd[k];
#pragma unroll
    for (int k = ML_IN; k < 16; k++) sx[threadIdx.x * 16 + k] = 0.f;
    __syncthreads();
    const int w = threadIdx.x >> 5;
    for (int tile = 0; tile < 2; tile++)
    {
        const int row0 = w * 32 + tile * 16;
        mlp_forward_tile(s, sx + row0 * 16, sy + row0 * 4, nullptr);
    }
    __syncthreads();
    if (i < c.N)
    {
        float4 p = c.pos[i];
        if (p.w > 0.f)
        {
            p.x += sy[threadIdx.x * 4] * s.oscale[0];
            p.y += sy[threadIdx.x * 4 + 1] * s.oscale[1];
            p.z += sy[threadIdx.x * 4 + 2] * s.oscale[2];
            c.pos[i] = p;
        }
    }
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
__global__ void __launch_bounds__(128) k_mlp_forward(const float* X, int S, MlpArgs ml, float* Y)
{
    __shared__ MlpSmem s;
    __shared__ float sx[128 * 16];
    __shared__ float sy[128 * 4];
    mlp_load_smem(s, ml.prm, ml.norm);
    __syncthreads();
    const int r = blockIdx.x * 128 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 16; k++)
        sx[threadIdx.x * 16 + k] = (r < S && k < ML_IN) ? (X[(size_t)r * ML_IN + k] - s.mean[k]) * s.istd[k] : 0.f;
    __syncthreads();
    const int w = threadIdx.x >> 5;
    for (int tile = 0; tile < 2; tile++)
        mlp_forward_tile(s, sx + (w * 32 + tile * 16) * 16, sy + (w * 32 + tile * 16) * 4, nullptr);
    __syncthreads();
    if (r < S)
        for (int k = 0; k < ML_OUT; k++) Y[(size_t)r * ML_OUT + k] = sy[threadIdx.x * 4 + k] * s.oscale[k];
}

// ------------------------------------------------------------ training
// Gradients of the mean squared error between the network's output and
// target / output scale, for 64 rows per CTA (4 warps x one 16-row tile);
// accumulated into grad[ML_NPARAM] and loss[0] (both zeroed by the caller).
constexpr int ML_ROWS = 64;
struct MlpTrainSmem
{
    float x[ML_ROWS * 16];
    float z[ML_ROWS / 16][3 * 16 * ML_H];   // per warp: pre-activations of the 3 hidden layers
    float y[ML_ROWS * 4];
    float d0[ML_ROWS * ML_H], d1[ML_ROWS * ML_H];
};

__global__ void __launch_bounds__(128) k_mlp_grad(const float* X, const float* T, int S, MlpArgs ml, float* grad, float* loss)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    MlpSmem& s = *reinterpret_cast<MlpSmem*>(dyn);
    MlpTrainSmem& a = *reinterpret_cast<MlpTrainSmem*>(dyn + ((sizeof(MlpSmem) + 15) / 16) * 16);
    mlp_load_smem(s, ml.prm, ml.norm);
    const int r0 = blockIdx.x * ML_ROWS;
    for (int k = threadIdx.x; k < ML_ROWS * 16; k += blockDim.x)
    {
        const int r = r0 + k / 16, col = k % 16;
        a.x[k] = (r < S && col < ML_IN) ? (X[(size_t)r * ML_IN + col] - ml.norm[col]) * ml.norm[ML_IN + col] : 0.f;
    }
    __syncthreads();
    const int w = threadIdx.x >> 5;
    mlp_forward_tile(s, a.x + w * 16 * 16, a.y + w * 16 * 4, a.z[w]);
    __syncthreads();
    // output layer: dL/dy for rows inside the batch (mean over S x 3 elements)
    const float inv = 1.f / (float)(S * ML_OUT);
    float lsum = 0.f;
    for (int k = threadIdx.x; k < ML_ROWS * 4; k += blockDim.x)
    {
        const int rr = k / 4, col = k % 4, r = r0 + rr;
        float d = 0.f;
        if (col < ML_OUT && r < S)
        {
            const float e = a.y[k] - T[(size_t)r * ML_OUT + col] / ml.norm[2 * ML_IN + col];
            lsum += e * e;
            d = 2.f * e * inv;
        }
        a.y[k] = d;
    }
    atomicAdd(loss, lsum * inv);
    __syncthreads();
    auto zat = [&](int layer, int r, int o) { return a.z[r / 16][layer * 16 * ML_H + (r % 16) * ML_H + o]; };
    auto hat = [&](int layer, int r, int i) { return gelu(zat(layer, r, i)); };
    // layer 4: grads, and dH3 = dY W4 (into d0)
    for (int k = threadIdx.x; k < ML_OUT * ML_H; k += blockDim.x)
    {
        const int o = k / ML_H, i = k % ML_H;
        float gsum = 0.f;
        for (int r = 0; r < ML_ROWS; r++) gsum += a.y[r * 4 + o] * hat(2, r, i);
        atomicAdd(&grad[ML_W4 + k], gsum);
    }
    if (threadIdx.x < ML_OUT)
    {
        float gsum = 0.f;
        for (int r = 0; r < ML_ROWS; r++) gsum += a.y[r * 4 + threadIdx.x];
        atomicAdd(&grad[ML_B4 + threadIdx.x], gsum);
    }
    for (int k = threadIdx.x; k < ML_ROWS * ML_H; k += blockDim.x)
    {
        const int r = k / ML_H, i = k % ML_H;
        float d = 0.f;
        for (int o = 0; o < ML_OUT; o++) d += a.y[r * 4 + o] * ml.prm[ML_W4 + o * ML_H + i];
        a.d0[k] = d * gelu_grad(zat(2, r, i));      // dZ3
    }
    __syncthreads();
    // hidden layers 3, 2: dW = dZ^T H_prev, db = sum dZ, dZ_prev = (dZ W) * gelu'(Z_prev)
    float* dz = a.d0;
    float* dn = a.d1;
    for (int layer = 2; layer >= 1; layer--)
    {
        const int wo = layer == 2 ? ML_W3 : ML_W2, bo = layer == 2 ? ML_B3 : ML_B2;
        for (int k = threadIdx.x; k < ML_H * ML_H; k += blockDim.x)
        {
            const int o = k / ML_H, i = k % ML_H;
            float gsum = 0.f;
            for (int r = 0; r < ML_ROWS; r++) gsum += dz[r * ML_H + o] * hat(layer - 1, r, i);
            atomicAdd(&grad[wo + k], gsum);
        }
        if (threadIdx.x < ML_H)
        {
            float gsum = 0.f;
            for (int r = 0; r < ML_ROWS; r++) gsum += dz[r * ML_H + threadIdx.x];
            atomicAdd(&grad[bo + threadIdx.x], gsum);
        }
        for (int k = threadIdx.x; k < ML_ROWS * ML_H; k += blockDim.x)
        {
            const int r = k / ML_H, i = k % ML_H;
            float d = 0.f;
            for (int o = 0; o < ML_H; o++) d += dz[r * ML_H + o] * ml.prm[wo + o * ML_H + i];
            dn[k] = d * gelu_grad(zat(layer - 1, r, i));
        }
        __syncthreads();
        float* tmp = dz; dz = dn; dn = tmp;
    }
    // layer 1: dW1 = dZ1^T X, db1
    for (int k = threadIdx.x; k < ML_H * ML_IN; k += blockDim.x)
    {
        const int o = k / ML_IN, i = k % ML_IN;
        float gsum = 0.f;
        for (int r = 0; r < ML_ROWS; r++) gsum += dz[r * ML_H + o] * a.x[r * 16 + i];
        atomicAdd(&grad[ML_W1 + k], gsum);
    }
    if (threadIdx.x < ML_H)
    {
        float gsum = 0.f;
        for (int r = 0; r < ML_ROWS; r++) gsum += dz[r * ML_H + threadIdx.x];
        atomicAdd(&grad[ML_B1 + threadIdx.x], gsum);
    }
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
