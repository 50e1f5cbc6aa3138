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
                // nearest wins; equal distances keep the lower triangle index (as the grid search
                // does, so both find the same hit); a distance equal to tmax still counts (the
                // reference accepts distance <= step)
                if (t >= tmin && t < INFINITY && (t < h.t || (t == h.t && (h.tri < 0 || i < h.tri)))) {
                    h.t = t;
                    h.tri = i;
                }
            }
        }
        node = miss;
    }
    return h;
}

// One ray-triangle candidate of the grid search: nearest wins, equal distances keep the lower index.
__host__ __device__ __forceinline__ void grid_candidate(float4 a, float4 b, float4 c, int t, float ox, float oy, float oz,
                                                        float dx, float dy, float dz, float tmin, unsigned& retests,
                                                        Hit& h) {
    const float d = tri_distance(a, b, c, ox, oy, oz, dx, dy, dz, retests);
    if (d >= tmin && d < INFINITY && (d < h.t || (d == h.t && (h.tri < 0 || t < h.tri)))) {
        h.t = d;
        h.tri = t;
    }
}

// Nearest hit with tmin <= t <= tmax for a bounded segment: the big triangles (shared memory) and
// the cells under the segment's xy bounding box, entries culled by z-range, loaded four at a time so
// their fetches overlap. Returns false when the box covers more than kGridMaxCells cells; the caller
// then uses the BVH.
__host__ __device__ __forceinline__ bool grid_nearest(const uint2* __restrict__ cells, const float4* __restrict__ cell_z,
                                                      const float4* __restrict__ entries,
                                                      const float4* __restrict__ big, int n_big, float gx0, float gy0,
                                                      float icx, float icy, int nx, int ny,
                                                      const float4* __restrict__ g_tris, const float4* __restrict__ s_tris,
                                                      int n_smem_tris, float ox, float oy, float oz, float dx, float dy,
                                                      float dz, float tmin, float tmax, int excl, unsigned& retests,
                                                      unsigned& n_visit, unsigned& n_tri, Hit& h) {
    const float ex = fmaf(dx, tmax, ox), ey = fmaf(dy, tmax, oy), ez = fmaf(dz, tmax, oz);
    const float fx0 = fminf(fmaxf((fminf(ox, ex) - gx0) * icx, -1.0f), (float)nx);
    const float fx1 = fminf(fmaxf((fmaxf(ox, ex) - gx0) * icx, -1.0f), (float)nx);
    const float fy0 = fminf(fmaxf((fminf(oy, ey) - gy0) * icy, -1.0f), (float)ny);
    const float fy1 = fminf(fmaxf((fmaxf(oy, ey) - gy0) * icy, -1.0f), (float)ny);
    h.t = tmax;
    h.tri = -1;
    const bool inside = fx1 >= 0.0f && fy1 >= 0.0f && fx0 < (float)nx && fy0 < (float)ny;
    const int i0 = max(0, (int)floorf(fx0)), i1 = min(nx - 1, (int)floorf(fx1));
    const int j0 = max(0, (int)floorf(fy0)), j1 = min(ny - 1, (int)floorf(fy1));
    if (inside && (i1 - i0 + 1) * (j1 - j0 + 1) > kGridMaxCells) return false;
    const float zl = fminf(oz, ez), zh = fmaxf(oz, ez);
    // the large triangles (they may extend beyond the grid's bounds), then the cells
    for (int k = 0; k < n_big; ++k) {
        const float4 en = big[4 * k];
        if (en.y < zl || en.x > zh) continue;
        const int t = f2i(en.z);
        if (t == excl) continue;
        ++n_tri;
        grid_candidate(big[4 * k + 1], big[4 * k + 2], big[4 * k + 3], t, ox, oy, oz, dx, dy, dz, tmin, retests, h);
    }
    if (!inside) return true;  // every other triangle lies inside the grid's bounds
    for (int j = j0; j <= j1; ++j) {
        for (int i = i0; i <= i1; ++i) {
            const unsigned int ci = (unsigned int)j * (unsigned int)nx + (unsigned int)i;
            const uint2 cell = XMC_LDG(&cells[ci]);
            const float4 za = XMC_LDG(&cell_z[2 * ci]), zb = XMC_LDG(&cell_z[2 * ci + 1]);
            n_visit += 1;
            // the cell's occupied z-intervals: skip it when the step's z-range misses all of them
            if ((za.y < zl || za.x > zh) && (za.w < zl || za.z > zh) && (zb.y < zl || zb.x > zh) && (zb.w < zl || zb.z > zh))
                continue;
            for (unsigned int k = 0; k < cell.y; k += 4) {
                float4 en[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    en[q] = k + q < cell.y ? XMC_LDG(&entries[cell.x + k + q]) : make_float4(INFINITY, -INFINITY, 0.0f, 0.0f);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (en[q].y < zl || en[q].x > zh) continue;
                    const int t = f2i(en[q].z);
                    if (t == excl) continue;
                    float4 a, b, c;
                    if (t < n_smem_tris) {
                        a = s_tris[3 * t]; b = s_tris[3 * t + 1]; c = s_tris[3 * t + 2];
                    } else {
                        a = XMC_LDG(&g_tris[3 * t]); b = XMC_LDG(&g_tris[3 * t + 1]); c = XMC_LDG(&g_tris[3 * t + 2]);
                    }
                    ++n_tri;
                    grid_candidate(a, b, c, t, ox, oy, oz, dx, dy, dz, tmin, retests, h);
                }
            }
        }
    }
    return true;
}

}  // namespace xmc
