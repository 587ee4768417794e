// render.cu — headless rasteriser of a cloth patch's mesh into a device image:
// the reference demo's Phong program (Shaders/shader_phong_vertex.glsl:21-36,
// shader_phong_geometry.glsl compute_distances(), shader_phong_fragment.glsl
// orennayar() and main()) restated as CUDA math, for pictures without a
// graphics stack. Two kernels: one thread per triangle resolves depth per pixel
// with a 64-bit atomicMin of (depth key, triangle index) — deterministic; the
// nearest wins and ties go to the lower index, as GL_LESS does in draw order —
// and one thread per pixel interpolates the world position and normal
// (perspective correct) and shades. Supported flags: OREN_NAYAR (2), MONOCHROME
// (8), WIREFRAME (16); vertex colours, textures and shadow maps are not
// restated. Triangles with a vertex behind the eye (clip w <= 0) are dropped
// instead of clipped.
#include "cloth.h"
#include "../../include/solidcloth_b200.h"

namespace sc {

struct RenderArgs
{
    float vp[16];            // view-projection, row-major, applied to (x, y, z, 1)
    float light[3], eye[3], kd[3], ks[3];
    float shininess, flip, background;
    int flags, width, height;
};

__device__ __forceinline__ float4 to_clip(const RenderArgs& r, float4 p)
{
    const float* m = r.vp;
    return make_float4(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
                       m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
                       m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11],
                       m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15]);
}

// window coordinates (x right, y down from the top row) and NDC depth
__device__ __forceinline__ bool project(const RenderArgs& r, float4 p, float& x, float& y, float& z, float& w)
{
    const float4 c = to_clip(r, p);
    if (!(c.w > 0.f)) return false;
    const float iw = 1.f / c.w;
    x = (c.x * iw + 1.f) * 0.5f * (float)r.width;
    y = (1.f - c.y * iw) * 0.5f * (float)r.height;
    z = c.z * iw;
    w = c.w;
    return true;
}

__device__ __forceinline__ float edge_fn(float ax, float ay, float bx, float by, float px, float py)
{
    return (bx - ax) * (py - ay) - (by - ay) * (px - ax);
}

// depth as an order-preserving 32-bit key (NDC z in [-1, 1])
__device__ __forceinline__ unsigned depth_key(float z)
{
    const unsigned u = __float_as_uint(z);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_raster(const float4* pos, const uint32_t* tri, int T, RenderArgs r, unsigned long long* zbuf)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    float x[3], y[3], z[3], w[3];
    for (int k = 0; k < 3; k++)
        if (!project(r, pos[tri[3 * t + k]], x[k], y[k], z[k], w[k])) return;   // no near-plane clipping
    const float area = edge_fn(x[0], y[0], x[1], y[1], x[2], y[2]);
    if (area == 0.f) return;
    const int x0 = max(0, (int)floorf(fminf(x[0], fminf(x[1], x[2])))), x1 = min(r.width - 1, (int)ceilf(fmaxf(x[0], fmaxf(x[1], x[2]))));
    const int y0 = max(0, (int)floorf(fminf(y[0], fminf(y[1], y[2])))), y1 = min(r.height - 1, (int)ceilf(fmaxf(y[0], fmaxf(y[1], y[2]))));
    const float ia = 1.f / area;
    for (int py = y0; py <= y1; py++)
        for (int px = x0; px <= x1; px++)
        {
            const float cx = (float)px + 0.5f, cy = (float)py + 0.5f;
            const float b0 = edge_fn(x[1], y[1], x[2], y[2], cx, cy) * ia;
            const float b1 = edge_fn(x[2], y[2], x[0], y[0], cx, cy) * ia;
            const float b2 = edge_fn(x[0], y[0], x[1], y[1], cx, cy) * ia;
            // both windings are drawn (the cloth has two sides); NaN tests fail
            if (!(b0 >= 0.f && b1 >= 0.f && b2 >= 0.f)) continue;
            const float zz = b0 * z[0] + b1 * z[1] + b2 * z[2];
            if (!(zz >= -1.f && zz <= 1.f)) continue;
            const unsigned long long key = ((unsigned long long)depth_key(zz) << 32) | (unsigned)t;
            atomicMin(&zbuf[(size_t)py * r.width + px], key);
        }
}

enum { RF_OREN_NAYAR = 2, RF_MONOCHROME = 8, RF_WIREFRAME = 16, RF_SUPPORTED = 2 | 8 | 16 };

// shader_phong_fragment.glsl orennayar(): uses the unflipped normal
__device__ float oren_nayar(V3 p, V3 n, V3 light, V3 eye, float roughness)
{
    const V3 L = normalized(light - p), N = normalized(n), V = normalized(eye - p);
    const float acosVN = acosf(dot(V, N)), acosLN = acosf(dot(L, N));
    const float alpha = fmaxf(acosVN, acosLN), beta = fminf(acosVN, acosLN);
    const float gamma = dot(V - dot(V, N) * N, L - dot(L, N) * N);
    const float r2 = roughness * roughness;
    const float C1 = 1.f - 0.5f * (r2 / (r2 + 0.33f));
    float C2 = 0.45f * (r2 / (r2 + 0.09f));
    if (gamma >= 0.f) C2 *= sinf(alpha);
    else C2 *= sinf(alpha) - powf((2.f * beta) / 3.14167f, 3.f);
    float C3 = 1.f / 8.f;
    C3 *= r2 / (r2 + 0.09f);
    C3 *= powf((4.f * alpha * beta) / (3.14167f * 3.14167f), 2.f);
    const float A = gamma * C2 * tanf(beta);
    const float B = (1.f - fabsf(gamma)) * C3 * tanf((alpha + beta) / 2.f);
    return fminf(fmaxf(0.f, dot(N, L)) * (C1 + A + B), 0.99f);
}

__global__ void k_shade(const float4* pos, const float4* nrm, const uint32_t* tri, RenderArgs r,
                        const unsigned long long* zbuf, float4* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r.width * r.height) return;
    const unsigned long long key = zbuf[i];
    if (key == ~0ull) { out[i] = make_float4(r.background, r.background, r.background, 1.f); return; }
    const int t = (int)(key & 0xffffffffu);
    const int px = i % r.width, py = i / r.width;
    float x[3], y[3], z[3], w[3];
    for (int k = 0; k < 3; k++) project(r, pos[tri[3 * t + k]], x[k], y[k], z[k], w[k]);
    const float cx = (float)px + 0.5f, cy = (float)py + 0.5f;
    const float ia = 1.f / edge_fn(x[0], y[0], x[1], y[1], x[2], y[2]);
    float b[3] = {edge_fn(x[1], y[1], x[2], y[2], cx, cy) * ia, edge_fn(x[2], y[2], x[0], y[0], cx, cy) * ia,
                  edge_fn(x[0], y[0], x[1], y[1], cx, cy) * ia};
    const V3 kd = mk(r.kd[0], r.kd[1], r.kd[2]), ks = mk(r.ks[0], r.ks[1], r.ks[2]);
    V3 light;
    if (r.flags & RF_MONOCHROME)
        light = kd;
    else
    {
        // perspective-correct weights of the vertex shader's outputs
        float wb[3], s = 0.f;
        for (int k = 0; k < 3; k++) { wb[k] = b[k] / w[k]; s += wb[k]; }
        V3 p = mk(0, 0, 0), n = mk(0, 0, 0);
        for (int k = 0; k < 3; k++)
        {
            const float4 q = pos[tri[3 * t + k]], m = nrm[tri[3 * t + k]];
            const float wk = wb[k] / s;
            p = p + wk * mk(q.x, q.y, q.z);
            n = n + wk * normalized(mk(m.x, m.y, m.z));     // the vertex shader normalises
        }
        const V3 lp = mk(r.light[0], r.light[1], r.light[2]), ep = mk(r.eye[0], r.eye[1], r.eye[2]);
        const V3 N = r.flip * normalized(n);
        const V3 L = normalized(lp - p);
        const V3 V = normalized(ep - p);
        const float ambient = 0.2f;
        const float diffuse = fmaxf(dot(L, N), 0.f);
        float spec = 0.f;
        if (diffuse > 0.f && len(ks) > 0.f)
        {
            const V3 R = -L - (2.f * dot(N, -L)) * N;          // reflect(-L, N)
            spec = powf(fmaxf(dot(V, R), 0.f), r.shininess);
        }
        const float shade = (r.flags & RF_OREN_NAYAR) ? oren_nayar(p, n, lp, ep, 1.4f) : (ambient + diffuse) / (1.f + ambient);
        light = shade * kd + spec * ks;
    }
    if (r.flags & RF_WIREFRAME)
    {
        // geometry shader: window-space height of each vertex over the opposite
        // edge, interpolated linearly in window space
        float d = FLT_MAX;
        for (int k = 0; k < 3; k++)
        {
            const int a = (k + 1) % 3, c = (k + 2) % 3;
            const float ux = x[a] - x[k], uy = y[a] - y[k], vx = x[c] - x[k], vy = y[c] - y[k];
            const float area = fabsf(ux * vy - uy * vx);
            const float h = area / sqrtf((ux - vx) * (ux - vx) + (uy - vy) * (uy - vy));
            d = fminf(d, b[k] * h);
        }
        const float lineWidth = 1.f;
        if (d > 0.5f * lineWidth + 1.f) d = 2.f;
        d = fminf(fmaxf(d - (0.5f * lineWidth - 1.f), 0.f), 2.f);
        const float I = exp2f(-2.f * d * d);
        light = (1.f - I) * light;                           // line colour black
    }
    out[i] = make_float4(light.x, light.y, light.z, 1.f);
}

} // namespace sc

using namespace sc;

extern "C" {

int scRenderCloth(scClothPatch patch, const float* viewProj16, const float* params16, int width, int height,
                  float* rgba, void* zscratch)
{
    ClothPatch* p = (ClothPatch*)patch.ptr;
    if (!p || !viewProj16 || !params16 || !rgba || !zscratch || width < 1 || height < 1 || p->model.N == 0 ||
        (long long)width * height > (1ll << 28))
    {
        set_error(SC_ERR_ARG, "bad render request");
        return SC_ERR_ARG;
    }
    const int flags = (int)params16[15];
    if (flags & ~RF_SUPPORTED)
    {
        set_error(SC_ERR_UNSUPPORTED, "render flags: only OREN_NAYAR, MONOCHROME and WIREFRAME are restated");
        return SC_ERR_UNSUPPORTED;
    }
    ClothModel& m = p->model;
    p->sync();
    RenderArgs r;
    for (int k = 0; k < 16; k++) r.vp[k] = viewProj16[k];
    for (int k = 0; k < 3; k++)
    {
        r.light[k] = params16[k]; r.eye[k] = params16[3 + k]; r.kd[k] = params16[6 + k]; r.ks[k] = params16[9 + k];
    }
    r.shininess = params16[12]; r.flip = params16[13]; r.background = params16[14];
    r.flags = flags; r.width = width; r.height = height;
    cudaStream_t s = p->stream;
    launch_normals(s, m.dc, false, m.dc.pos);      // the render mesh's normals (Mesh::ComputeNormals)
    unsigned long long* z = (unsigned long long*)zscratch;
    cudaMemsetAsync(z, 0xff, sizeof(unsigned long long) * (size_t)width * height, s);
    k_raster<<<(m.dc.T + 127) / 128, 128, 0, s>>>(m.dc.pos, m.dc.tri, m.dc.T, r, z);
    k_shade<<<(width * height + 255) / 256, 256, 0, s>>>(m.dc.pos, m.dc.meshN, m.dc.tri, r, z, (float4*)rgba);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(SC_ERR_CUDA, cudaGetErrorString(e)); return SC_ERR_CUDA; }
    return SC_OK;
}

} // extern "C"
