// Linear BVH topology built on the GPU, for large meshes without a prebuilt tree.
//
// The reference builds its BVH on the host with a binned SAH (GenerateBVHTree,
// mcml_intersection.cpp:88-344), which for a 2 x 130,050-triangle height field takes a large part of
// a second. Here the topology comes from the parallel construction of Karras (2012, "Maximizing
// parallelism in the construction of BVHs, octrees, and k-d trees"):
//   1. each triangle gets a 64-bit key: the 30-bit Morton code of its centroid (10 bits per axis,
//      one cubic grid over the centroid bounds) above its index, so keys are unique;
//   2. the keys are sorted (CUB radix sort);
//   3. internal node i of the n - 1 derives, from the longest common key prefixes around position
//      i, the key range it covers and the split inside it, and so its two children (internal nodes
//      or single-triangle leaves), all nodes in parallel.
// The host (bvh.cpp) turns the topology into the kernel's threaded layout: subtrees of a few
// triangles become leaves (the sorted order keeps them contiguous), boxes are computed from the FP32
// vertices, and nodes are renumbered, exactly as for a tree built on the host.
#include <cub/cub.cuh>

#include <string>
#include <vector>

#include "xmc_internal.h"

namespace xmc {
namespace {

// 10-bit value -> its bits spread to every third position (bit i -> bit 3i)
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void morton_kernel(const float* __restrict__ cen, int n, float3 lo, float3 inv_ext,
                              unsigned long long* __restrict__ keys) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float c[3] = {cen[3 * (size_t)t], cen[3 * (size_t)t + 1], cen[3 * (size_t)t + 2]};
    const float l[3] = {lo.x, lo.y, lo.z}, s[3] = {inv_ext.x, inv_ext.y, inv_ext.z};
    uint32_t q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float u = (c[k] - l[k]) * s[k];  // [0, 1] (0 on a flat axis)
        q[k] = (uint32_t)fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f);
    }
    const uint32_t m = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    keys[t] = ((unsigned long long)m << 32) | (uint32_t)t;
}

// Length of the common prefix of sorted keys i and j; -1 when j is outside [0, n).
__device__ __forceinline__ int delta(const unsigned long long* __restrict__ k, int n, int i, long long j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(k[i] ^ k[j]);
}

// Karras (2012), section 4: children of internal node i; a child c >= 0 is internal node c, a child
// c < 0 is the leaf holding sorted triangle -1 - c. range[i] = first and last sorted position.
__global__ void karras_kernel(const unsigned long long* __restrict__ k, int n, int2* __restrict__ child,
                              int2* __restrict__ range) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = delta(k, n, i, (long long)i + 1) - delta(k, n, i, (long long)i - 1) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, (long long)i - d);
    long long lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    long long l = 0;
    for (long long t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const long long j = i + l * d;
    const int dnode = delta(k, n, i, j);
    long long s = 0;
    long long t = l;
    do {
        t = (t + 1) / 2;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const long long g = i + s * d + (d < 0 ? -1 : 0);
    const long long lo = i < j ? i : j, hi = i < j ? j : i;
    child[i] = make_int2(lo == g ? (int)(-1 - g) : (int)g, hi == g + 1 ? (int)(-1 - (g + 1)) : (int)(g + 1));
    range[i] = make_int2((int)lo, (int)hi);
}

}  // namespace

// Topology of a linear BVH over `n` (>= 2) triangles with centroids `cen` (3 floats each) on
// device `device`: the sorted triangle order, and per internal node (root 0) its children and its
// range of sorted positions. Returns false with *err set on a CUDA failure.
bool gpu_lbvh_topology(const std::vector<float>& cen, int n, int device, std::vector<int>* order,
                       std::vector<int2>* child, std::vector<int2>* range, std::string* err) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int t = 0; t < n; ++t)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], cen[3 * (size_t)t + k]);
            hi[k] = std::max(hi[k], cen[3 * (size_t)t + k]);
        }
    // one scale for the three axes (cubic Morton cells): a thin axis (the depth of a layer stack)
    // is then split only where its cells are as small as the others, not at every third level
    const float ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    const float s = ext > 0.0f ? 1.0f / ext : 0.0f;
    const float inv[3] = {s, s, s};

    float* d_cen = nullptr;
    unsigned long long *d_keys = nullptr, *d_sorted = nullptr;
    int2 *d_child = nullptr, *d_range = nullptr;
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaSetDevice(device);
    auto ok = [&](cudaError_t r, const char* what) {
        if (r != cudaSuccess && e == cudaSuccess) {
            e = r;
            *err = std::string("GPU BVH build, ") + what + ": " + cudaGetErrorString(r);
        }
        return e == cudaSuccess;
    };
    if (!ok(e, "cudaSetDevice")) return false;
    if (ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream") &&
        ok(cudaMalloc(&d_cen, sizeof(float) * 3 * (size_t)n), "alloc") &&
        ok(cudaMalloc(&d_keys, sizeof(unsigned long long) * (size_t)n), "alloc") &&
        ok(cudaMalloc(&d_sorted, sizeof(unsigned long long) * (size_t)n), "alloc") &&
        ok(cudaMalloc(&d_child, sizeof(int2) * (size_t)(n - 1)), "alloc") &&
        ok(cudaMalloc(&d_range, sizeof(int2) * (size_t)(n - 1)), "alloc") &&
        ok(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, d_keys, d_sorted, n, 0, 64, st), "sort size") &&
        ok(cudaMalloc(&d_tmp, tmp_bytes ? tmp_bytes : 16), "alloc") &&
        ok(cudaMemcpyAsync(d_cen, cen.data(), sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, st), "upload")) {
        morton_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_cen, n, make_float3(lo[0], lo[1], lo[2]),
                                                        make_float3(inv[0], inv[1], inv[2]), d_keys);
        if (ok(cudaGetLastError(), "morton") &&
            ok(cub::DeviceRadixSort::SortKeys(d_tmp, tmp_bytes, d_keys, d_sorted, n, 0, 64, st), "sort")) {
            karras_kernel<<<(n - 1 + 255) / 256, 256, 0, st>>>(d_sorted, n, d_child, d_range);
            std::vector<unsigned long long> keys(n);
            child->resize(n - 1);
            range->resize(n - 1);
            if (ok(cudaGetLastError(), "hierarchy") &&
                ok(cudaMemcpyAsync(keys.data(), d_sorted, sizeof(unsigned long long) * (size_t)n, cudaMemcpyDeviceToHost,
                                   st), "download") &&
                ok(cudaMemcpyAsync(child->data(), d_child, sizeof(int2) * (size_t)(n - 1), cudaMemcpyDeviceToHost, st),
                   "download") &&
                ok(cudaMemcpyAsync(range->data(), d_range, sizeof(int2) * (size_t)(n - 1), cudaMemcpyDeviceToHost, st),
                   "download") &&
                ok(cudaStreamSynchronize(st), "synchronize")) {
                order->resize(n);
                for (int i = 0; i < n; ++i) (*order)[i] = (int)(uint32_t)keys[i];
            }
        }
    }
    for (void* p : {(void*)d_cen, (void*)d_keys, (void*)d_sorted, (void*)d_child, (void*)d_range, d_tmp})
        if (p) cudaFree(p);
    if (st) cudaStreamDestroy(st);
    return e == cudaSuccess;
}

}  // namespace xmc
