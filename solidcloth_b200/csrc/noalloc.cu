// noalloc.cu — angle-weighted vertex normals without any device allocation.
//
// Some callers cannot call cudaMalloc: engines that reserve all GPU memory up
// front and forbid allocation once their frame loop runs, code executing inside
// another library's memory pool, or real-time threads where an allocation (an
// implicit device synchronisation) would stall the frame. For them this entry
// point computes the same normals as scUpdateClothMesh (Mesh::ComputeNormals,
// Geometry/Mesh.cpp:10-63) on caller-owned device buffers, with its only scratch
// — one float4 accumulator per vertex — in a fixed file-scope device array.
//
// Properties a caller must know:
//   * capacity: at most SC_NOALLOC_MAX_VERTICES vertices (65,536: a 256 x 256
//     grid); larger meshes are rejected with SC_ERR_ARG;
//   * every triangle index is checked against numVertices on the device: a
//     triangle with an index out of range is skipped (nothing is written for it)
//     and the call returns SC_ERR_ARG. To report that, the call waits for its
//     work on the stream to finish before it returns;
//   * the scratch array (1 MiB) is resident on every GPU that loads this library
//     until the process exits;
//   * every call shares that array and it keeps the last call's contents; a call
//     clears what it needs first. Calls that overlap on the GPU (different
//     streams, or another thread) race on it and must be serialised by the caller;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture that would include later calls. Later calls
//     look it up again (it is cheap) unless the stream is capturing, so a
//     context reset between calls does not leave a stale address behind;
//   * the per-vertex sums use atomic adds, so the order of additions (and the
//     last bits of the result) can differ from scUpdateClothMesh's ordered sum.
#include "cloth.h"
#include "../../include/solidcloth_b200.h"
#include <mutex>

namespace sc {

static __device__ __align__(256) float4 g_noalloc_normal_acc[SC_NOALLOC_MAX_VERTICES];
// number of triangles of the last call that had an index >= numVertices
static __device__ int g_noalloc_bad_triangles;

__global__ void k_noalloc_clear(float4* acc, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) g_noalloc_bad_triangles = 0;
    if (i < n) acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// per triangle: unit normal and corner angles as k_tri_normals computes them,
// accumulated into the three corner vertices; a triangle with an index outside
// [0, n) is counted and skipped, so no write leaves acc[0, n)
__global__ void k_noalloc_tri(const float* v, const unsigned* idx, int T, int n, float4* acc)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const size_t o = 3 * (size_t)t;
    const unsigned i1 = idx[o], i2 = idx[o + 1], i3 = idx[o + 2];
    if (i1 >= (unsigned)n || i2 >= (unsigned)n || i3 >= (unsigned)n)
    {
        atomicAdd(&g_noalloc_bad_triangles, 1);
        return;
    }
    V3 a = mk(v[3 * i1], v[3 * i1 + 1], v[3 * i1 + 2]);
    V3 b = mk(v[3 * i2], v[3 * i2 + 1], v[3 * i2 + 2]);
    V3 c = mk(v[3 * i3], v[3 * i3 + 1], v[3 * i3 + 2]);
    V3 nt = normalized(cross(b - a, c - a));
    V3 e1 = normalized(b - a), e2 = normalized(c - b), e3 = normalized(a - c);
    float c1 = -dot(e1, e3), c2 = -dot(e1, e2), c3 = -dot(e2, e3);
    float s1 = len(cross(e1, -e3)), s2 = len(cross(e2, -e1)), s3 = len(cross(e3, -e1));
    float t1 = fabsf(c1) > 1 ? fabsf((float)atan2((double)s1, (double)c1)) : portable_acos(c1);
    float t2 = fabsf(c2) > 1 ? fabsf((float)atan2((double)s2, (double)c2)) : portable_acos(c2);
    float t3 = fabsf(c3) > 1 ? fabsf((float)atan2((double)s3, (double)c3)) : portable_acos(c3);
    const unsigned ids[3] = {i1, i2, i3};
    const float w[3] = {t1, t2, t3};
    for (int k = 0; k < 3; k++)
    {
        V3 d = w[k] * nt;
        atomicAdd(&acc[ids[k]].x, d.x);
        atomicAdd(&acc[ids[k]].y, d.y);
        atomicAdd(&acc[ids[k]].z, d.z);
    }
}

__global__ void k_noalloc_normalise(const float4* acc, int n, float* out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = acc[i];
    V3 s = mk(a.x, a.y, a.z);
    if (len(s) != 0) s = normalized(s);
    out[3 * i] = s.x; out[3 * i + 1] = s.y; out[3 * i + 2] = s.z;
}

// device address of the scratch array, looked up once per device
static std::mutex g_noalloc_mutex;
static float4* g_noalloc_ptr[64] = {nullptr};

static float4* noalloc_scratch(int dev, bool capturing)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!g_noalloc_ptr[dev] || !capturing)
    {
        float4* p = nullptr;
        // host code must not take the array's address directly: that is a host
        // stand-in, not a device address
        cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_normal_acc);
        if (e != cudaSuccess)
        {
            set_error(SC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return nullptr;
        }
        g_noalloc_ptr[dev] = p;
    }
    return g_noalloc_ptr[dev];
}

} // namespace sc

using namespace sc;

extern "C" int scComputeVertexNormalsNoAlloc(const float* vertices, int numVertices, const unsigned* indices,
                                             int numTriangles, float* normals, void* stream)
{
    if (!vertices || !normals || (numTriangles > 0 && !indices))
    {
        set_error(SC_ERR_ARG, "scComputeVertexNormalsNoAlloc: null buffer");
        return SC_ERR_ARG;
    }
    if (numVertices <= 0 || numVertices > SC_NOALLOC_MAX_VERTICES || numTriangles < 0 ||
        numTriangles > SC_NOALLOC_MAX_TRIANGLES)
    {
        set_error(SC_ERR_ARG, "scComputeVertexNormalsNoAlloc: numVertices must be in [1, " +
                                  std::to_string(SC_NOALLOC_MAX_VERTICES) + "] and numTriangles in [0, " +
                                  std::to_string(SC_NOALLOC_MAX_TRIANGLES) + "], got " +
                                  std::to_string(numVertices) + " / " + std::to_string(numTriangles));
        return SC_ERR_ARG;
    }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { set_error(SC_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e)); return SC_ERR_CUDA; }
    cudaStream_t s = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) { set_error(SC_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e)); return SC_ERR_CUDA; }
    float4* acc = noalloc_scratch(dev, cap != cudaStreamCaptureStatusNone);
    if (!acc) return SC_ERR_CUDA;
    const int nb = (numVertices + 255) / 256;
    k_noalloc_clear<<<nb, 256, 0, s>>>(acc, numVertices);
    if (numTriangles > 0)
        k_noalloc_tri<<<(numTriangles + 255) / 256, 256, 0, s>>>(vertices, indices, numTriangles, numVertices, acc);
    k_noalloc_normalise<<<nb, 256, 0, s>>>(acc, numVertices, normals);
    e = cudaGetLastError();
    if (e != cudaSuccess) { set_error(SC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e)); return SC_ERR_CUDA; }
    // the index check's outcome: read the device counter once the work is done
    int bad = 0;
    e = cudaMemcpyFromSymbolAsync(&bad, g_noalloc_bad_triangles, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(SC_ERR_CUDA, std::string("status read: ") + cudaGetErrorString(e)); return SC_ERR_CUDA; }
    if (bad > 0)
    {
        set_error(SC_ERR_ARG, "scComputeVertexNormalsNoAlloc: " + std::to_string(bad) +
                                  " triangle(s) have an index >= numVertices (" + std::to_string(numVertices) +
                                  "); they were skipped");
        return SC_ERR_ARG;
    }
    return SC_OK;
}
