// Ray queries of the walk, compiled for the device (the transport kernel) and for the host (the
// geometry self-test entry point xmc_debug_nearest), so the CPU test suite exercises the exact
// traversal and triangle arithmetic the kernel runs.
#pragma once

#include <cstdint>
#include <cstring>

#include "xmc_internal.h"

#ifdef __CUDA_ARCH__
#define XMC_LDG(p) __ldg(p)
#else
#define XMC_LDG(p) (*(p))
#endif

namespace xmc {

__host__ __device__ __forceinline__ int f2i(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_int(f);
#else
    int i;
    std::memcpy(&i, &f, sizeof(i));
    return i;
#endif
}

struct Hit {
    float t;
    int tri;  // index into the triangle array, -1 if none
};

// FP64 re-test of a ray-triangle pair near an edge (rare; kept out of line to spare registers).
__host__ __device__ __noinline__ float tri_distance_fp64(float4 a, float4 b, float4 c, float ox, float oy, float oz,
                                                        float dx, float dy, float dz) {
    const double E1x = (double)b.x - a.x, E1y = (double)b.y - a.y, E1z = (double)b.z - a.z;
    const double E2x = (double)c.x - a.x, E2y = (double)c.y - a.y, E2z = (double)c.z - a.z;
    const double Dx = dx, Dy = dy, Dz = dz;
    const double Px = Dy * E2z - Dz * E2y, Py = Dz * E2x - Dx * E2z, Pz = Dx * E2y - Dy * E2x;
    const double Det = E1x * Px + E1y * Py + E1z * Pz;
    if (Det < 1e-6 && Det > -1e-6) return INFINITY;
    const double Inv = 1.0 / Det;
    const double Sx = (double)ox - a.x, Sy = (double)oy - a.y, Sz = (double)oz - a.z;
    const double U = (Sx * Px + Sy * Py + Sz * Pz) * Inv;
    if (U < 0.0 || U > 1.0) return INFINITY;
    const double Qx = Sy * E1z - Sz * E1y, Qy = Sz * E1x - Sx * E1z, Qz = Sx * E1y - Sy * E1x;
    const double V = (Dx * Qx + Dy * Qy + Dz * Qz) * Inv;
    if (V < 0.0 || U + V > 1.0) return INFINITY;
    return (float)((E2x * Qx + E2y * Qy + E2z * Qz) * Inv);
}

// Moller-Trumbore in FP32 with the reference's determinant cut (mcml_intersection.cpp:44-86).
// Inside a barycentric band around the edges (width stored per triangle in c.w: kEdgeBandLength
// divided by the triangle's shortest edge, at least kEdgeBandMin) the test is redone in FP64 on the
// same FP32 inputs so neighbouring triangles agree on which of them a ray crosses.
__host__ __device__ __forceinline__ float tri_distance(float4 a, float4 b, float4 c, float ox, float oy, float oz,
                                                       float dx, float dy, float dz, unsigned& retests) {
    const float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
    const float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
    const float px = dy * e2z - dz * e2y, py = dz * e2x - dx * e2z, pz = dx * e2y - dy * e2x;
    const float det = e1x * px + e1y * py + e1z * pz;
    if (fabsf(det) < 1e-6f) return INFINITY;
    const float inv = 1.0f / det;
    const float sx = ox - a.x, sy = oy - a.y, sz = oz - a.z;
    const float u = (sx * px + sy * py + sz * pz) * inv;
    const float qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const float v = (dx * qx + dy * qy + dz * qz) * inv;
    const float w = 1.0f - u - v;
    const float band = c.w;  // per-triangle barycentric width of the FP64 re-test band
    if (u < -band || v < -band || w < -band) return INFINITY;
    if (u > band && v > band && w > band) return (e2x * qx + e2y * qy + e2z * qz) * inv;
    ++retests;
    return tri_distance_fp64(a, b, c, ox, oy, oz, dx, dy, dz);
}
// Nearest hit with tmin <= t <= tmax over the threaded BVH (no stack): the reference's
// ComputeBVHIntersection / ComputeBVHIntersectionWithoutStep contract (mcml_intersection.cpp:354-584).
// Nodes below n_smem_nodes and triangles below n_smem_tris are read from the staged copies.
__host__ __device__ __forceinline__ Hit bvh_nearest(const float4* __restrict__ g_nodes, const float4* __restrict__ g_tris,
                                                    int n_nodes, const float4* __restrict__ s_nodes, int n_smem_nodes,
                                                    const float4* __restrict__ s_tris, int n_smem_tris,
                                                    float ox, float oy, float oz, float dx, float dy, float dz,
                                                    float tmin, float tmax, int excl, unsigned& retests,
                                                    unsigned& n_visit, unsigned& n_tri) {
    Hit h;
    h.t = tmax;
    h.tri = -1;
    if (n_nodes == 0) return h;
    const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dz;
    int node = 0;
    while (node >= 0) {
        float4 lo, hi;
        if (node < n_smem_nodes) {
            lo = s_nodes[2 * node];
            hi = s_nodes[2 * node + 1];
        } else {
            lo = XMC_LDG(&g_nodes[2 * node]);
            hi = XMC_LDG(&g_nodes[2 * node + 1]);
        }
        const float t0x = (lo.x - ox) * ix, t1x = (hi.x - ox) * ix;
        const float t0y = (lo.y - oy) * iy, t1y = (hi.y - oy) * iy;
        const float t0z = (lo.z - oz) * iz, t1z = (hi.z - oz) * iz;
        const float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.0f));
        const float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), h.t));
        const int child = f2i(lo.w);
        const int miss = f2i(hi.w);
        ++n_visit;
        if (tn <= tf) {
            if (child >= 0) {
                node = child;
                continue;
            }
            const int code = -1 - child;
            const int first = code >> 3, end = first + (code & 7) + 1;
            n_tri += end - first;
            for (int i = first; i < end; ++i) {
                if (i == excl) continue;
                float4 a, b, c;
                if (i < n_smem_tris) {
                    a = s_tris[3 * i]; b = s_tris[3 * i + 1]; c = s_tris[3 * i + 2];
                } else {
                    a = XMC_LDG(&g_tris[3 * i]); b = XMC_LDG(&g_tris[3 * i + 1]); c = XMC_LDG(&g_tris[3 * i + 2]);
                }
                const float t = tri_distance(a, b, c, ox, oy, oz, dx, dy, dz, retests);
                // nearest wins; on equal distances the first triangle found keeps the hit; a
                // distance equal to tmax still counts (the reference accepts distance <= step)
                if (t >= tmin && t < INFINITY && (t < h.t || (t == h.t && h.tri < 0))) {
                    h.t = t;
                    h.tri = i;
                }
            }
        }
        node = miss;
    }
    return h;
}

}  // namespace xmc
