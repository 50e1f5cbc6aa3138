// Persistent photon-transport kernel for sm_100a: the GPU counterpart of the reference's
// ComputePhoton walk (base/xmcml/xmcml/mcml_kernel.cpp:39-126) driven by LaunchOMP's photon loop
// (base/xmcml/xmcmlLauncher/launcher_omp.cpp:138-144).
//
// One thread walks one photon at a time; a warp claims photon ids in chunks from a global
// dispenser and refills lanes whose photon died before the next iteration (warp-level compaction
// of live photons), so lanes stay busy until the dispenser runs dry. Every random number comes
// from Philox4x32-10 keyed by the seed with counter (photon id, iteration, 0): one block of four
// 24-bit uniforms per walk iteration, with fixed slots, so a photon's path does not depend on
// which thread runs it and the tallies (64-bit fixed-point integer sums) are bit-identical for
// every launch shape.
//
// Per iteration (tissue layer): slot 0 step length; on a boundary hit slot 1 Fresnel test and
// slot 2 roulette; on an interaction slot 1 HG cos(theta), slot 2 azimuth, slot 3 roulette.
// Glass layer: slot 0 Fresnel test, slot 1 roulette. The photon-weight arithmetic is integer
// (weight 1.0 == 2^31): every deposit is subtracted from the photon's integer weight, so the
// ledger terms add up to launched weight exactly.
#include <cstdint>
#include <type_traits>

#include "geom.cuh"
#include "photon.cuh"
#include "xmc_internal.h"

namespace xmc {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// Photon weight in 2^31 fixed point: 32 bits (weight <= 1 always holds without biasing) or 64 bits
// (the biasing factor W / p can raise a weight above 1).
template <typename WT>
struct Photon {
    float px, py, pz, dx, dy, dz;
    float time, trange, orange;
    WT w;
    int layer;
    uint32_t visited;
    uint32_t iter;
    int excl;
    float tmin;
    float gap_lo, gap_hi;  // triangle-free z-gap containing the photon (empty if none)
    int rdet;              // replay pass: the detector this photon reached in the run pass
    unsigned long long pid;
};

__device__ __forceinline__ float w2f(uint32_t w) { return __uint2float_rn(w); }
__device__ __forceinline__ float w2f(unsigned long long w) { return __ull2float_rn(w); }
template <typename WT> __device__ __forceinline__ WT f2w(float f);
template <> __device__ __forceinline__ uint32_t f2w<uint32_t>(float f) { return __float2uint_rn(f); }
template <> __device__ __forceinline__ unsigned long long f2w<unsigned long long>(float f) { return __float2ull_rn(f); }
// w^2 in fixed point ((w w) >> 31), exact for weights below 2^32 in weight units
__device__ __forceinline__ unsigned long long wsq(uint32_t w) { return ((unsigned long long)w * w) >> 31; }
__device__ __forceinline__ unsigned long long wsq(unsigned long long w) { return (__umul64hi(w, w) << 33) | ((w * w) >> 31); }

// The triangle-free z-gap around z: (highest occupied top below z, lowest occupied bottom above
// z), or an empty interval when z lies inside an occupied slab.
__device__ __forceinline__ void find_gap(const float* __restrict__ zlo, const float* __restrict__ zhi, int n, float z,
                                         float& glo, float& ghi) {
    glo = -INFINITY;
    ghi = INFINITY;
    for (int i = 0; i < n; ++i) {
        if (z >= zlo[i] && z <= zhi[i]) {
            glo = INFINITY;
            ghi = -INFINITY;
            return;
        }
        if (zhi[i] < z) glo = fmaxf(glo, zhi[i]);
        if (zlo[i] > z) ghi = fminf(ghi, zlo[i]);
    }
}

// GetAreaIndex (mcml_kernel.cpp:190-227): voxel of a point, -1 outside Area. `tol` (voxel units)
// widens the box for points on a surface: the reference stops 1e-10 mm in front of a surface
// (mcml_kernel.cpp:60,87), so a surface lying on an Area face counts as inside; the FP32 hit point
// sits on the surface within rounding and is accepted within tol, clamped to the edge voxel.
__device__ __forceinline__ int area_index(const KParams& P, float x, float y, float z, float tol) {
    float fx = (x - P.ax) * P.asx, fy = (y - P.ay) * P.asy, fz = (z - P.az) * P.asz;
    if (!(fx >= -tol && fy >= -tol && fz >= -tol)) return -1;
    if (!(fx < (float)P.nx + tol && fy < (float)P.ny + tol && fz < (float)P.nz + tol)) return -1;
    const int ix = min(max((int)fx, 0), P.nx - 1), iy = min(max((int)fy, 0), P.ny - 1), iz = min(max((int)fz, 0), P.nz - 1);
    if (P.byte_sentinel && ix == 255 && iy == 255 && iz == 255) return -1;
    return (ix * P.ny + iy) * P.nz + iz;
}

// Block-private tallies in shared memory.
struct SmemTally {
    unsigned long long* ledger;  // [kLedgerSlots]
    unsigned long long* det;     // [n_dets * 4]
};

__device__ __forceinline__ void lat(unsigned long long* p, unsigned long long v) {
    if (v) atomicAdd(p, v);
}

// mcml_kernel.cpp:663-742 (first matching cube, then ring; layer filter; angle test) and the
// detector tallies of :744-858. Weight arithmetic in fixed point.
template <class Ph>
__device__ int find_detector(const KParams& P, const DevDetector* __restrict__ s_det, const Ph& ph) {
    int det = -1;
    const float l2 = ph.dx * ph.dx + ph.dy * ph.dy + ph.dz * ph.dz;
    const float ac = -ph.dz / l2;
    const int n_scan = P.rings_sorted ? P.n_cubes : P.n_dets;
    for (int i = 0; i < n_scan; ++i) {
        const DevDetector D = s_det[i];
        bool inside;
        if (i < P.n_cubes) {
            inside = ph.px >= D.cx - D.hx && ph.px < D.cx + D.hx && ph.py >= D.cy - D.hy && ph.py < D.cy + D.hy &&
                     ph.pz >= D.cz - D.hz && ph.pz < D.cz + D.hz;
        } else {
            const float ex = ph.px - D.cx, ey = ph.py - D.cy;
            const float r = sqrtf(ex * ex + ey * ey);
            inside = r >= D.hx && r < D.hy;
        }
        if (inside && (D.filter & ph.visited) && ac > D.cos_angle) {
            det = i;
            break;
        }
    }
    if (det < 0 && P.rings_sorted) {
        // concentric, sorted, non-overlapping rings: the only ring that can contain the radius is
        // the last one whose small radius is <= r, so the first match of the scan is this one
        const DevDetector* R = s_det + P.n_cubes;
        const float ex = ph.px - R[0].cx, ey = ph.py - R[0].cy;
        const float r = sqrtf(ex * ex + ey * ey);
        int lo = 0, hi = P.n_rings - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (R[mid].hx <= r) lo = mid;
            else hi = mid - 1;
        }
        const DevDetector D = R[lo];
        if (r >= D.hx && r < D.hy && (D.filter & ph.visited) && ac > D.cos_angle) det = P.n_cubes + lo;
    }
    return det;
}

template <class Ph>
__device__ void tally_detection(const KParams& P, const SmemTally& S, const Ph& ph, int det) {
    using WT = decltype(ph.w);
    const WT w = ph.w;
    const float total = ph.trange + ph.orange;
    const WT tw = total > 0.0f ? f2w<WT>(w2f(w) * (ph.trange / total)) : (WT)0;
    const unsigned long long w2 = wsq(w);
    atomicAdd(&S.det[4 * det + 0], (unsigned long long)w);
    atomicAdd(&S.det[4 * det + 1], 1ull);
    lat(&S.det[4 * det + 2], tw);
    lat(&S.det[4 * det + 3], w2);
    atomicAdd(&S.ledger[L_N_DETECTED], 1ull);
    // time bins (mcml_kernel.cpp:812-849): [t0 + i dt, t0 + (i+1) dt), last bin open-ended
    if (ph.time >= P.t0) {
        int bin = P.n_time - 1;
        if (P.dt > 0.0f) {
            const float f = (ph.time - P.t0) / P.dt;
            if (f < (float)(P.n_time - 1)) bin = (int)f;
        }
        unsigned long long* tb = P.tbin + 4 * ((size_t)det * P.n_time + bin);
        atomicAdd(tb + 0, (unsigned long long)w);
        atomicAdd(tb + 1, 1ull);
        lat(tb + 2, tw);
        lat(tb + 3, w2);
    }
}

// UpdatePhotonTrajectory (mcml_kernel.cpp:750-792): for a move from p0 to p1, every z-plane through
// voxel centres between them (inside Area) is crossed at one voxel. The run pass adds the photon's
// weight to the scattering map there and appends the voxel to the thread's crossing log (`xl`, `xn`
// entries so far, counted past the capacity so that an overflow shows); at detection the log is
// counted in the detector's trajectory map (UpdateDetectorTrajectory, :794-810, which walks the
// reference's per-photon PhotonTrajectory the same way). The replay pass, for photons whose log
// overflowed, counts each crossing in the map of the detector the photon reached.
// Row of the crossing log of thread `thread` of this block.
__device__ __forceinline__ unsigned* xlog_row(const KParams& P, unsigned thread) {
    return P.xlog + ((size_t)blockIdx.x * blockDim.x + thread) * P.xlog_cap;
}

__device__ void cross_planes(const KParams& P, float x0, float y0, float z0, float x1, float y1, float z1,
                             unsigned long long w, int rdet, unsigned* __restrict__ xl, unsigned& xn,
                             unsigned& n_cross) {
    if (z1 == z0) return;
    // first plane at or above the lower end of the move; most moves cross none and stop here
    const float step = P.plane_dz;
    const int k = (int)fmaf(fminf(z0, z1) - P.az, P.asz, 0.5f);
    float plane = P.az + k * step + 0.5f * step;
    if (plane > fmaxf(z0, z1) || plane >= P.area_zend) return;
    float sx = x0, sy = y0, sz = z0, fz = z1, ex = x1 - x0, ey = y1 - y0, ez = z1 - z0;
    if (z1 < z0) {
        sx = x1; sy = y1; sz = z1; fz = z0;
        ex = -ex; ey = -ey; ez = -ez;
    }
    const float inv = 1.0f / ez;
    for (int guard = 0; plane <= fz && plane < P.area_zend && guard < 65536; ++guard) {
        const float t = (plane - sz) * inv;
        const int idx = area_index(P, fmaf(ex, t, sx), fmaf(ey, t, sy), plane, 0.0f);
        if (idx < 0) break;
        ++n_cross;
        if (P.mode == 0) {
            if (w && P.scatter) atomicAdd(&P.scatter[idx], (unsigned long long)w);
            if (xl) {
                if (xn < P.xlog_cap) xl[xn] = (unsigned)idx;
                xn += xn <= P.xlog_cap;  // saturates at capacity + 1: overflowed
            }
        } else {
            atomicAdd(&P.traj[(size_t)rdet * P.grid + idx], 1ull);
        }
        plane += step;
    }
}

// Nearest hit with tmin <= t <= tmax of every querying lane's short segment, by the whole warp at once
// (all 32 lanes call it; `need` marks the lanes with a query). The same candidates and the same
// choice as grid_nearest (geom.cuh): the big triangles, then the triangles listed in the xy cells
// under the segment, culled by the cells' and entries' z-ranges; the nearest distance wins and equal
// distances keep the lower triangle index. Instead of each lane walking its own cells and entries
// (serial loops whose trip counts differ from lane to lane), the warp flattens the work:
//   1. each querying lane's cell rectangle (at most kGridMaxCells cells; more: `fallback`, the lane
//      uses the BVH) and its big-triangle candidates;
//   2. all (lane, cell) pairs of the warp, 32 per round: cell header and z-intervals loaded by one
//      lane each, cells whose intervals miss the segment dropped, the rest compacted into a list;
//   3. all (lane, entry) pairs of the kept cells, 32 per round: entry z-cull, the triangle test by
//      one lane each, the packed (distance, triangle) minimum per querying lane in shared memory.
// Each stage costs one dependent load round trip per 32 pairs instead of one per cell (or per four
// entries) and lane, and every lane of the warp does useful tests.
__device__ __forceinline__ unsigned long long pack_hit(float d, unsigned tri) {
    return ((unsigned long long)__float_as_uint(d) << 32) | tri;
}

__device__ __forceinline__ void warp_grid_query(const KParams& P, WarpQuery& W, const float4* __restrict__ s_big,
                                             const float4* __restrict__ s_tris, bool need, float ox, float oy, float oz,
                                             float dx, float dy, float dz, float tmin, float tmax, int excl, Hit& hit,
                                             bool& fallback, unsigned& retests, unsigned& n_visit, unsigned& n_tri) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    fallback = false;
    int ncell = 0;
    unsigned long long best = pack_hit(tmax, 0xffffffffu);
    if (need) {
        const float ex = fmaf(dx, tmax, ox), ey = fmaf(dy, tmax, oy), ez = fmaf(dz, tmax, oz);
        const float fx0 = fminf(fmaxf((fminf(ox, ex) - P.grid_x0) * P.grid_icx, -1.0f), (float)P.grid_nx);
        const float fx1 = fminf(fmaxf((fmaxf(ox, ex) - P.grid_x0) * P.grid_icx, -1.0f), (float)P.grid_nx);
        const float fy0 = fminf(fmaxf((fminf(oy, ey) - P.grid_y0) * P.grid_icy, -1.0f), (float)P.grid_ny);
        const float fy1 = fminf(fmaxf((fmaxf(oy, ey) - P.grid_y0) * P.grid_icy, -1.0f), (float)P.grid_ny);
        const bool inside = fx1 >= 0.0f && fy1 >= 0.0f && fx0 < (float)P.grid_nx && fy0 < (float)P.grid_ny;
        const int i0 = max(0, (int)floorf(fx0)), i1 = min(P.grid_nx - 1, (int)floorf(fx1));
        const int j0 = max(0, (int)floorf(fy0)), j1 = min(P.grid_ny - 1, (int)floorf(fy1));
        const float zl = fminf(oz, ez), zh = fmaxf(oz, ez);
        if (inside && (i1 - i0 + 1) * (j1 - j0 + 1) > kGridMaxCells) {
            fallback = true;
        } else {
            for (int k = 0; k < P.n_big; ++k) {
                const float4 en = s_big[4 * k];
                if (en.y < zl || en.x > zh) continue;
                const int t = f2i(en.z);
                if (t == excl) continue;
                ++n_tri;
                const float d = tri_distance(s_big[4 * k + 1], s_big[4 * k + 2], s_big[4 * k + 3], ox, oy, oz, dx, dy, dz,
                                             retests);
                if (d >= tmin && d <= tmax) best = min(best, pack_hit(__fadd_rn(d, 0.0f), (unsigned)t));
            }
            if (inside) {
                ncell = (i1 - i0 + 1) * (j1 - j0 + 1);
                W.ij0[lane] = i0 | (j0 << 16);
                W.w[lane] = i1 - i0 + 1;
            }
            W.o[lane] = make_float4(ox, oy, oz, tmin);
            W.d[lane] = make_float4(dx, dy, dz, tmax);
            W.z[lane] = make_float2(zl, zh);
            W.excl[lane] = excl;
        }
    }
    W.best[lane] = best;
    // (lane, cell) pairs: exclusive scan of the cell counts
    int incl = ncell;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
    }
    const int n_pairs = __shfl_sync(FULL, incl, 31);
    W.coff[lane] = incl - ncell;
    __syncwarp();
    int nk = 0;
    for (int base = 0; base < n_pairs; base += 32) {
        const int k = base + lane;
        bool keep = false;
        uint2 cell = make_uint2(0u, 0u);
        int own = 0;
        if (k < n_pairs) {
            // the pair's lane: the last lane whose offset is <= k (it has cells: the next offset is > k)
            int lo = 0, hi = 31;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (W.coff[mid] <= k) lo = mid;
                else hi = mid - 1;
            }
            own = lo;
            const int loc = k - W.coff[own], ww = W.w[own], ij = W.ij0[own];
            const unsigned ci = (unsigned)((ij >> 16) + loc / ww) * (unsigned)P.grid_nx + (unsigned)((ij & 0xffff) + loc % ww);
            cell = __ldg(&P.cells[ci]);
            const float4 za = __ldg(&P.cell_z[2 * ci]), zb = __ldg(&P.cell_z[2 * ci + 1]);
            const uint32_t runs = __ldg(&P.cell_runs[ci]);
            const float2 z = W.z[own];
            ++n_visit;
            // the z-intervals the segment overlaps are consecutive; keep only their entries (the others
            // lie inside intervals the segment misses and would fail the entry z-cull)
            const bool ov[4] = {!(za.y < z.x || za.x > z.y), !(za.w < z.x || za.z > z.y), !(zb.y < z.x || zb.x > z.y),
                                !(zb.w < z.x || zb.z > z.y)};
            keep = cell.y > 0 && (ov[0] || ov[1] || ov[2] || ov[3]);
            if (keep && runs != 0xffffffffu) {
                unsigned skip = 0, take = 0;
                bool seen = false;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const unsigned cq = (runs >> (8 * q)) & 0xffu;
                    if (ov[q]) {
                        seen = true;
                        take += cq;
                    } else if (!seen) {
                        skip += cq;
                    }
                }
                cell.x += skip;
                cell.y = take;
                keep = take > 0;
            }
        }
        const unsigned km = __ballot_sync(FULL, keep);
        if (keep) {
            const int pos = nk + __popc(km & lt);
            W.cell[pos] = cell;
            W.owner[pos] = (unsigned char)own;
        }
        nk += __popc(km);
    }
    __syncwarp();
    // (lane, entry) pairs over the kept cells: exclusive scan of their entry counts
    int n_ent = 0;
    for (int base = 0; base < nk; base += 32) {
        const int c = base + lane;
        const int cnt = c < nk ? (int)W.cell[c].y : 0;
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(FULL, inc, o);
            if (lane >= o) inc += v;
        }
        if (c < nk) W.eoff[c] = n_ent + inc - cnt;
        n_ent += __shfl_sync(FULL, inc, 31);
    }
    __syncwarp();
    for (int base = 0; base < n_ent; base += 32) {
        const int k = base + lane;
        if (k < n_ent) {
            int lo = 0, hi = nk - 1;  // the entry's cell: the last kept cell whose offset is <= k
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (W.eoff[mid] <= k) lo = mid;
                else hi = mid - 1;
            }
            const int own = W.owner[lo];
            const float4 en = __ldg(&P.cell_entries[W.cell[lo].x + (unsigned)(k - W.eoff[lo])]);
            const float2 z = W.z[own];
            const int t = f2i(en.z);
            if (!(en.y < z.x || en.x > z.y) && t != W.excl[own]) {
                float4 a, b, c;
                if (t < P.smem_tris) {
                    a = s_tris[3 * t]; b = s_tris[3 * t + 1]; c = s_tris[3 * t + 2];
                } else {
                    a = __ldg(&P.tris[3 * t]); b = __ldg(&P.tris[3 * t + 1]); c = __ldg(&P.tris[3 * t + 2]);
                }
                ++n_tri;
                const float4 o = W.o[own], dd = W.d[own];
                const float d = tri_distance(a, b, c, o.x, o.y, o.z, dd.x, dd.y, dd.z, retests);
                if (d >= o.w && d <= dd.w) atomicMin(&W.best[own], pack_hit(__fadd_rn(d, 0.0f), (unsigned)t));
            }
        }
    }
    __syncwarp();
    if (need && !fallback) {
        const unsigned long long b = W.best[lane];
        const unsigned t = (unsigned)(b & 0xffffffffu);
        hit.tri = t == 0xffffffffu ? -1 : (int)t;
        hit.t = t == 0xffffffffu ? tmax : __uint_as_float((unsigned)(b >> 32));
    }
    __syncwarp();  // W is reused by the next query round
}

template <class Ph>
__device__ __forceinline__ void kill(const SmemTally& S, Ph& ph, bool& alive, int count_slot, int weight_slot) {
    atomicAdd(&S.ledger[count_slot], 1ull);
    lat(&S.ledger[weight_slot], ph.w);
    atomicAdd(&S.ledger[L_TERMINATED], 1ull);
    alive = false;
}

template <class Ph>
__device__ __forceinline__ void launch_photon(const KParams& P, Ph& ph, unsigned long long pid) {
    ph.pid = pid;
    ph.px = P.sx;
    ph.py = P.sy;
    ph.pz = P.sz;
    if (P.beam_radius > 0.0f) {
        const uint4 r = philox4x32_10(make_uint4((uint32_t)pid, (uint32_t)(pid >> 32), 0u, 1u), P.key0, P.key1);
        const float rad = P.beam_radius * sqrtf(u24(r.x));
        float a = u24(r.y);
        a = a > 0.5f ? a - 1.0f : a;
        float sp, cp;
        __sincosf(6.283185307179586f * a, &sp, &cp);
        ph.px += rad * cp;
        ph.py += rad * sp;
    }
    ph.dx = P.dx;
    ph.dy = P.dy;
    ph.dz = P.dz;
    ph.time = 0.0f;
    ph.trange = 0.0f;
    ph.orange = 0.0f;
    ph.w = P.w0;
    ph.layer = 1;
    ph.visited = 1u << 1;
    ph.iter = 0;
    ph.excl = -1;
    ph.tmin = kTminAfter;
}

constexpr uint32_t kBiasMaxTrials = 65536;

// ComputePhotonDirectionWithBiasing (mcml_kernel.cpp:398-428): the local attractive direction v
// (GetLocalAttractiveVector, :325-364: normalised difference of the fields of two point sources on
// the vertical through the target point, l_tr above it and l_tr + 2 delta below it), a new direction
// by rejection from HG with acceptance p = (0.1 + 0.45 (1 + d.v))^attractiveFactor (trial k draws the
// Philox block (id, iteration, 2 + k): slot 0 cos theta, slot 1 azimuth, slot 2 acceptance), and
// the weight factor W(d_old.v) / p from the layer's weight-integral table (nearest node).
template <class Ph>
__device__ __forceinline__ void biased_spin(const KParams& P, const DevLayer& L, int layer, Ph& ph,
                                            unsigned long long& gained, unsigned long long& lost) {
    using WT = decltype(ph.w);
    const float ltr = 3.0f * (1.0f / (3.0f * ((1.0f - L.g) * L.mus + L.mua)));
    const float delta = 0.74f * ltr;
    const float rx = ph.px - P.bias_ox, ry = ph.py - P.bias_oy, rz = ph.pz - P.bias_oz;
    const float ex = rx - P.bias_rx, ey = ry - P.bias_ry;
    const float az = rz - (P.bias_rz + ltr), bz = rz - (P.bias_rz - ltr - 2.0f * delta);
    const float ia = rsqrtf(ex * ex + ey * ey + az * az), ib = rsqrtf(ex * ex + ey * ey + bz * bz);
    const float ca = ia * ia * ia, cb = ib * ib * ib;
    float vx = ex * (cb - ca), vy = ey * (cb - ca), vz = bz * cb - az * ca;
    const float vn = rsqrtf(vx * vx + vy * vy + vz * vz);
    vx *= vn; vy *= vn; vz *= vn;
    const float dot0 = ph.dx * vx + ph.dy * vy + ph.dz * vz;
    float nx = ph.dx, ny = ph.dy, nz = ph.dz, p = 1.0f;
    for (uint32_t k = 0; k < kBiasMaxTrials; ++k) {
        const uint4 r = philox4x32_10(make_uint4((uint32_t)ph.pid, (uint32_t)(ph.pid >> 32), ph.iter - 1u, 2u + k),
                                      P.key0, P.key1);
        nx = ph.dx; ny = ph.dy; nz = ph.dz;
        hg_spin(L.hg_a, L.hg_b, L.hg_c, L.hg_d, L.hg_e, u24(r.x), u24(r.y), nx, ny, nz);
        p = powf(fmaf(0.45f, 1.0f + (nx * vx + ny * vy + nz * vz), 0.1f), P.bias_eps);
        if (p > u24(r.z)) break;
    }
    const int t = P.layer_wtab[layer];
    if (t >= 0) {
        const float step = 2.0f / (float)(P.wtab_n - 1);
        int e = (int)floorf((dot0 + 1.0f) / step + 0.5f);
        e = min(max(e, 0), P.wtab_n - 1);
        const float W = __ldg(&P.wtab[(size_t)t * P.wtab_n + e]);
        const WT nw = f2w<WT>(w2f(ph.w) * (W / p));
        if (nw > ph.w) gained += nw - ph.w;
        else lost += ph.w - nw;
        ph.w = nw;
    }
    ph.dx = nx; ph.dy = ny; ph.dz = nz;
}

}  // namespace

// kBias: biased spin with 64-bit weights; kLog: run pass that logs crossings for the trajectory maps
template <bool kBias, bool kLog>
__global__ void __launch_bounds__(512, 1) transport_kernel(const KParams P) {
    using WT = typename std::conditional<kBias, unsigned long long, uint32_t>::type;
    extern __shared__ __align__(16) unsigned char smem[];
    // --- shared memory carve-up (must match smem_layout on the host) ---
    unsigned long long* s_ledger = reinterpret_cast<unsigned long long*>(smem);
    unsigned long long* s_dettal = s_ledger + kLedgerSlots;
    float4* s_nodes = reinterpret_cast<float4*>(s_dettal + 4 * P.n_dets);
    float4* s_tris = s_nodes + 2 * P.smem_nodes;
    DevLayer* s_layer = reinterpret_cast<DevLayer*>(s_tris + 3 * P.smem_tris);
    DevDetector* s_det = reinterpret_cast<DevDetector*>(s_layer + MAX_LAYERS);
    int8_t* s_next = reinterpret_cast<int8_t*>(s_det + P.n_dets);
    const size_t fixed = (size_t)(reinterpret_cast<unsigned char*>(s_next + P.smem_next) - smem);
    WarpQuery* s_wq = reinterpret_cast<WarpQuery*>(smem + ((fixed + 15) & ~(size_t)15)) + (threadIdx.x >> 5);
    __shared__ float s_zlo[kMaxZSlabs], s_zhi[kMaxZSlabs];
    __shared__ float4 s_big[4 * kMaxBigTriangles];
    for (int i = threadIdx.x; i < 4 * P.n_big; i += blockDim.x) s_big[i] = P.big[i];
    for (int i = threadIdx.x; i < P.n_zocc; i += blockDim.x) {
        s_zlo[i] = P.zocc_lo[i];
        s_zhi[i] = P.zocc_hi[i];
    }

    for (int i = threadIdx.x; i < kLedgerSlots + 4 * P.n_dets; i += blockDim.x) s_ledger[i] = 0ull;
    for (int i = threadIdx.x; i < 2 * P.smem_nodes; i += blockDim.x) s_nodes[i] = __ldg(&P.nodes[i]);
    for (int i = threadIdx.x; i < 3 * P.smem_tris; i += blockDim.x) s_tris[i] = __ldg(&P.tris[i]);
    for (int i = threadIdx.x; i < MAX_LAYERS; i += blockDim.x) s_layer[i] = P.layer[i];
    for (int i = threadIdx.x; i < P.n_dets; i += blockDim.x) s_det[i] = P.dets[i];
    for (int i = threadIdx.x; i < P.smem_next; i += blockDim.x) s_next[i] = P.next_layer[i];
    __syncthreads();
    const SmemTally S{s_ledger, s_dettal};

    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const bool area_kill = !(P.flags & XMC_NO_AREA_KILL);
    const bool roulette = (P.flags & XMC_ROULETTE) != 0;
    // trajectory maps from the crossing log: each thread's log holds its current photon's crossings
    const bool log_traj = kLog;
    const bool record_planes = P.mode == 1 || (P.flags & XMC_SCATTERING_MAP) != 0 || log_traj;
    unsigned xn = 0;  // crossings of the current photon (capacity + 1: the log overflowed)
    // cooperative queries: a lane whose step needs the warp's query round waits (parked) until the
    // round runs (query_batch lanes waiting, or every live lane); the step's draws and length are
    // taken again when the round comes, exactly as the lane took them
    bool parked = false;

    unsigned long long cbeg = 0, cend = 0;  // warp-uniform chunk of photon indices
    bool exhausted = false;                 // warp-uniform
    bool alive = false;
    Photon<WT> ph;
    ph.rdet = -1;
    unsigned steps = 0, retests = 0, n_visit = 0, n_tri = 0, n_cross = 0;
    unsigned long long bias_gained = 0, bias_lost = 0;
    unsigned long long absorbed = 0, absorbed_out = 0, absorbed_tgt = 0;  // per-thread sums, flushed at the end
    unsigned budget_hit = 0;

    for (;;) {
        // ---- trajectory maps of the photons detected in the last iteration: the whole warp reads
        // each detected photon's log (coalesced) and counts it in its detector's map ----
        // (in the run pass a dead photon's rdet holds the detector its log goes to, -1 if none)
        if (log_traj) {
            unsigned fl = __ballot_sync(FULL, ph.rdet >= 0);
            if (fl) {
                __syncwarp();  // orders each lane's log stores before the other lanes' loads
                do {
                    const int src = __ffs(fl) - 1;
                    fl &= fl - 1u;
                    const int d = __shfl_sync(FULL, ph.rdet, src);
                    const unsigned n = __shfl_sync(FULL, xn, src);
                    const unsigned* xs = xlog_row(P, (threadIdx.x & ~31u) + src);
                    unsigned long long* tm = P.traj + (size_t)d * P.grid;
                    // four loads in flight per lane before their adds: the row was written over the
                    // photon's whole walk and is usually back in DRAM
                    for (unsigned j0 = lane; j0 < n; j0 += 128) {
                        unsigned v[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) v[u] = j0 + 32u * u < n ? xs[j0 + 32u * u] : 0xffffffffu;
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            if (v[u] != 0xffffffffu) atomicAdd(&tm[v[u]], 1ull);
                    }
                } while (fl);
                ph.rdet = -1;
            }
        }
        // ---- refill dead lanes with new photons (warp-level compaction) ----
        unsigned need = __ballot_sync(FULL, !alive && !exhausted);
        while (need) {
            if (cbeg == cend) {
                unsigned long long b = 0;
                int cancelled = 0;
                if (lane == 0) {
                    if (P.cancel && *P.cancel) cancelled = 1;  // device memory, written by xmc_cancel
                    b = cancelled ? P.n_photons : atomicAdd(P.counter, (unsigned long long)P.chunk);
                }
                b = __shfl_sync(FULL, b, 0);
                cancelled = __shfl_sync(FULL, cancelled, 0);
                if (cancelled && lane == 0) atomicOr(P.status, 2);
                if (b >= P.n_photons) {
                    exhausted = true;
                    break;
                }
                cbeg = b;
                cend = min(b + (unsigned long long)P.chunk, P.n_photons);
            }
            const unsigned long long avail = cend - cbeg;
            const int rank = __popc(need & lt_mask);
            const int cnt = __popc(need);
            const int take = (int)min((unsigned long long)cnt, avail);
            if (((need >> lane) & 1u) && rank < take) {
                unsigned long long idx = cbeg + rank;
                ph.rdet = -1;
                xn = 0;
                if (P.mode == 1) {
                    const unsigned long long e = P.replay_list[idx];
                    idx = e >> 16;
                    ph.rdet = (int)(e & 0xffffu);
                }
                launch_photon(P, ph, P.first_id + idx);
                find_gap(s_zlo, s_zhi, P.n_zocc, ph.pz, ph.gap_lo, ph.gap_hi);
                alive = true;
                atomicAdd(&S.ledger[L_LAUNCHED], 1ull);
            }
            cbeg += take;
            need = __ballot_sync(FULL, !alive && !exhausted);
        }
        if (__ballot_sync(FULL, alive) == 0u) break;

        // ---- one walk iteration (mcml_kernel.cpp:47-125) ----
        // Up to the ray query no lane leaves the iteration, so that every lane reaches the query
        // converged (the warp-cooperative query needs all 32); lanes with no photon or a photon that
        // ends before it only skip the work.
        bool act = alive && !parked;  // takes a new step this iteration
        const bool fresh = act;
        bool resumed = false;         // a waiting lane whose query round runs this iteration
        bool needq = false;
        float u_roulette = 0.0f;
        bool boundary = false;
        Hit hit;
        hit.t = 0.0f;
        hit.tri = -1;
        float step = 0.0f;
        uint4 r = make_uint4(0u, 0u, 0u, 0u);
        const DevLayer* Lp = &s_layer[0];
        if (act) {
            if (ph.iter >= P.max_steps) {
                budget_hit = 1;
                kill(S, ph, alive, L_N_BUDGET, L_BUDGET);
                act = false;
            } else {
                r = philox4x32_10(make_uint4((uint32_t)ph.pid, (uint32_t)(ph.pid >> 32), ph.iter, 0u), P.key0, P.key1);
                ph.iter++;
                steps++;
                Lp = &s_layer[ph.layer];
                if (Lp->glass) {
                    hit = bvh_nearest(P.nodes, P.tris, P.n_nodes, s_nodes, P.smem_nodes, s_tris, P.smem_tris, ph.px, ph.py,
                                      ph.pz, ph.dx, ph.dy, ph.dz, ph.tmin, INFINITY, ph.excl, retests, n_visit, n_tri);
                    boundary = true;
                    u_roulette = u24(r.y);
                    if (hit.tri < 0) {
                        kill(S, ph, alive, L_N_GLASS, L_GLASS);
                        act = false;
                    } else {
                        step = hit.t;
                    }
                } else {
                    step = -__logf(u24(r.x)) * Lp->inv_mut;  // mcml_kernel.cpp:618-631
                    const float zend = fmaf(step + kStepExtend, ph.dz, ph.pz);
                    if (fminf(ph.pz, zend) > ph.gap_lo && fmaxf(ph.pz, zend) < ph.gap_hi) {
                        hit.tri = -1;  // the step stays inside a triangle-free z-gap: no surface to cross
                        hit.t = step;
                    } else {
                        needq = true;
                    }
                }
            }
        }
        if (P.grid_nx > 0 && P.coop_query) {
            parked = parked || needq;
            const unsigned pm = __ballot_sync(FULL, parked);
            if (pm && (__popc(pm) >= P.query_batch || pm == __ballot_sync(FULL, alive))) {
                if (parked && !fresh) {
                    Lp = &s_layer[ph.layer];
                    r = philox4x32_10(make_uint4((uint32_t)ph.pid, (uint32_t)(ph.pid >> 32), ph.iter - 1u, 0u), P.key0,
                                      P.key1);
                    step = -__logf(u24(r.x)) * Lp->inv_mut;
                }
                bool fb = false;
                warp_grid_query(P, *s_wq, s_big, s_tris, parked, ph.px, ph.py, ph.pz, ph.dx, ph.dy, ph.dz, ph.tmin,
                                step + kStepExtend, ph.excl, hit, fb, retests, n_visit, n_tri);
                if (parked && fb)
                    hit = bvh_nearest(P.nodes, P.tris, P.n_nodes, s_nodes, P.smem_nodes, s_tris, P.smem_tris, ph.px,
                                      ph.py, ph.pz, ph.dx, ph.dy, ph.dz, ph.tmin, step + kStepExtend, ph.excl, retests,
                                      n_visit, n_tri);
                resumed = parked;
                parked = false;
            }
        } else if (needq) {
            if (!(P.grid_nx > 0 &&
                  grid_nearest(P.cells, P.cell_z, P.cell_entries, s_big, P.n_big, P.grid_x0, P.grid_y0, P.grid_icx,
                               P.grid_icy, P.grid_nx, P.grid_ny, P.tris, s_tris, P.smem_tris, ph.px, ph.py, ph.pz, ph.dx,
                               ph.dy, ph.dz, ph.tmin, step + kStepExtend, ph.excl, retests, n_visit, n_tri, hit))) {
                hit = bvh_nearest(P.nodes, P.tris, P.n_nodes, s_nodes, P.smem_nodes, s_tris, P.smem_tris, ph.px, ph.py,
                                  ph.pz, ph.dx, ph.dy, ph.dz, ph.tmin, step + kStepExtend, ph.excl, retests, n_visit, n_tri);
            }
        }
        if (!(act || resumed) || parked) continue;  // no photon, ended before its step, or waiting for its round
        const DevLayer& L = *Lp;
        if (!L.glass) {
            boundary = hit.tri >= 0;
            if (boundary) step = hit.t;
            u_roulette = boundary ? u24(r.z) : u24(r.w);
        }
        // move (mcml_kernel.cpp:151-174): optical path length, target/other range
        const float ox = ph.px, oy = ph.py, oz = ph.pz;
        ph.px = fmaf(step, ph.dx, ph.px);
        ph.py = fmaf(step, ph.dy, ph.py);
        ph.pz = fmaf(step, ph.dz, ph.pz);
        if (record_planes) cross_planes(P, ox, oy, oz, ph.px, ph.py, ph.pz, ph.w, ph.rdet,
                                        log_traj ? xlog_row(P, threadIdx.x) : nullptr, xn, n_cross);
        ph.time = fmaf(step, L.n, ph.time);
        if (!(ph.pz > ph.gap_lo && ph.pz < ph.gap_hi)) find_gap(s_zlo, s_zhi, P.n_zocc, ph.pz, ph.gap_lo, ph.gap_hi);
        if ((P.target_mask >> ph.layer) & 1u) ph.trange += step;
        else ph.orange += step;
        const int idx = area_index(P, ph.px, ph.py, ph.pz, boundary ? 1e-4f : 0.0f);
        if (idx < 0 && area_kill) {  // outside Area: the reference kills the photon (:63-76, :90-117)
            kill(S, ph, alive, L_N_AREA, L_AREA);
            continue;
        }
        if (boundary) {
            // ---- CrossBoundary (mcml_kernel.cpp:229-284) ----
            const float4 a = hit.tri < P.smem_tris ? s_tris[3 * hit.tri] : __ldg(&P.tris[3 * hit.tri]);
            const float4 b = hit.tri < P.smem_tris ? s_tris[3 * hit.tri + 1] : __ldg(&P.tris[3 * hit.tri + 1]);
            const float4 c = hit.tri < P.smem_tris ? s_tris[3 * hit.tri + 2] : __ldg(&P.tris[3 * hit.tri + 2]);
            // GetPlaneNormal (mcml_math.cpp:45-50), normalised
            const float e1x = a.x - b.x, e1y = a.y - b.y, e1z = a.z - b.z;
            const float e2x = a.x - c.x, e2y = a.y - c.y, e2z = a.z - c.z;
            float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
            const float nr = rsqrtf(nx * nx + ny * ny + nz * nz);
            nx *= nr; ny *= nr; nz *= nr;
            const int surf = __float_as_int(a.w);
            const int next = surf * MAX_LAYERS + ph.layer < P.smem_next ? (int)s_next[surf * MAX_LAYERS + ph.layer]
                                                                         : (int)__ldg(&P.next_layer[surf * MAX_LAYERS + ph.layer]);
            if (next < 0) {
                kill(S, ph, alive, L_N_INVALID, L_INVALID);
                continue;
            }
            const float ni = L.n, nt = s_layer[next].n;
            const float dn = ph.dx * nx + ph.dy * ny + ph.dz * nz;
            const float R = fresnel_reflectance(ni, nt, fabsf(dn));
            const float u_fresnel = L.glass ? u24(r.x) : u24(r.y);
            if (u_fresnel > R) {
                if (next == 0) {
                    // leaves the tissue: detectors (mcml_kernel.cpp:257-268)
                    const int det = find_detector(P, s_det, ph);
                    if (P.mode == 0) {
                        if (det >= 0) {
                            tally_detection(P, S, ph, det);
                            if (log_traj && xn <= P.xlog_cap) {
                                ph.rdet = det;  // the warp counts the log at the top of the next iteration
                            } else if (P.flags & XMC_DETECTOR_TRAJ) {
                                const unsigned long long slot = atomicAdd(P.replay_count, 1ull);
                                if (slot < P.replay_cap)
                                    P.replay_list[slot] = ((ph.pid - P.first_id) << 16) | (unsigned long long)det;
                            }
                        }
                    } else if (det != ph.rdet) {
                        atomicAdd(&S.ledger[L_N_REPLAY_MISMATCH], 1ull);
                    }
                    if (ph.dz < 0.0f) kill(S, ph, alive, L_N_TOP, L_TOP);
                    else kill(S, ph, alive, L_N_BOTTOM, L_BOTTOM);
                    continue;
                }
                // RefractVector (mcml_kernel.cpp:595-616)
                const float six = ni * ph.dx, siy = ni * ph.dy, siz = ni * ph.dz;
                const float t1 = six * nx + siy * ny + siz * nz;
                float t2 = sqrtf((nt * nt - ni * ni) / (t1 * t1) + 1.0f);
                t2 = (t2 - 1.0f) * t1;
                float ox = six + t2 * nx, oy = siy + t2 * ny, oz = siz + t2 * nz;
                const float on = rsqrtf(ox * ox + oy * oy + oz * oz);
                ph.dx = ox * on; ph.dy = oy * on; ph.dz = oz * on;
                ph.layer = next;
                ph.visited |= 1u << next;
            } else {
                // ReflectVector (mcml_kernel.cpp:582-593)
                const float t = 2.0f * dn;
                float ox = ph.dx - t * nx, oy = ph.dy - t * ny, oz = ph.dz - t * nz;
                const float on = rsqrtf(ox * ox + oy * oy + oz * oz);
                ph.dx = ox * on; ph.dy = oy * on; ph.dz = oz * on;
            }
            ph.excl = hit.tri;
            ph.tmin = kTminAfter;
        } else {
            // ---- drop (mcml_kernel.cpp:633-642) ----
            WT dw = f2w<WT>(w2f(ph.w) * L.absorb);
            dw = min(dw, ph.w);
            ph.w -= dw;
            if (idx >= 0) {
                if (dw && P.mode == 0) atomicAdd(&P.absorb[idx], (unsigned long long)dw);
                absorbed += dw;
            } else {
                absorbed_out += dw;
            }
            if ((P.target_mask >> ph.layer) & 1u) absorbed_tgt += dw;
            // ---- spin (mcml_kernel.cpp:442-495) ----
            if constexpr (kBias) {  // mcml_kernel.cpp:108-109
                biased_spin(P, L, ph.layer, ph, bias_gained, bias_lost);
            } else {
                hg_spin(L.hg_a, L.hg_b, L.hg_c, L.hg_d, L.hg_e, u24(r.y), u24(r.z), ph.dx, ph.dy, ph.dz);
            }
            ph.excl = -1;
            ph.tmin = 0.0f;
        }
        // ---- weight cut / roulette (mcml_kernel.cpp:121-124; planar GPU kernel.cu:214-222) ----
        if (ph.w < P.w_min) {
            if (roulette) {
                if (ph.w == 0u) {
                    kill(S, ph, alive, L_N_ROULETTE, L_RKILLED);
                } else if (u_roulette < P.chance) {
                    const WT nw = min(f2w<WT>(w2f(ph.w) * P.inv_chance), (WT)kWeightOne);
                    lat(&S.ledger[L_RGAINED], nw - ph.w);
                    ph.w = nw;
                } else {
                    kill(S, ph, alive, L_N_ROULETTE, L_RKILLED);
                }
            } else {
                kill(S, ph, alive, L_N_CUT, L_CUT);
            }
        }
    }

    // ---- flush block-private tallies ----
    atomicAdd(&S.ledger[L_STEPS], (unsigned long long)steps);
    lat(&S.ledger[L_ABSORBED], absorbed);
    lat(&S.ledger[L_ABSORBED_OUT], absorbed_out);
    lat(&S.ledger[L_ABSORBED_TGT], absorbed_tgt);
    if (kBias) {
        lat(&S.ledger[L_BIAS_GAINED], bias_gained);
        lat(&S.ledger[L_BIAS_LOST], bias_lost);
    }
    if (retests) atomicAdd(&S.ledger[L_N_RETEST], (unsigned long long)retests);
    atomicAdd(&S.ledger[L_N_NODES], (unsigned long long)n_visit);
    atomicAdd(&S.ledger[L_N_TRIS], (unsigned long long)n_tri);
    if (n_cross) atomicAdd(&S.ledger[L_N_CROSSINGS], (unsigned long long)n_cross);
    if (budget_hit) atomicOr(P.status, 1);
    __syncthreads();
    for (int i = threadIdx.x; i < kLedgerSlots; i += blockDim.x) lat(&P.ledger[i], s_ledger[i]);
    for (int i = threadIdx.x; i < 4 * P.n_dets; i += blockDim.x) lat(&P.det[i], s_dettal[i]);
}

__global__ void philox_probe_kernel(uint32_t k0, uint32_t k1, unsigned long long pid, uint32_t n, uint4* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = philox4x32_10(make_uint4((uint32_t)pid, (uint32_t)(pid >> 32), i, 0u), k0, k1);
}

// Throughput of 64-bit atomic adds to scattered addresses of an L2-resident array (the tally
// pattern of the walk: absorption voxels and map cells): each thread adds to `per_thread` slots
// picked by a multiplicative hash of (thread, iteration).
__global__ void atomic_probe_kernel(unsigned long long* slots, unsigned long long mask, unsigned per_thread) {
    const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long h = t * 0x9E3779B97F4A7C15ull;
    for (unsigned i = 0; i < per_thread; ++i) {
        h = (h ^ (h >> 29)) * 0xBF58476D1CE4E5B9ull + i;
        atomicAdd(&slots[(h >> 17) & mask], 1ull);
    }
}

cudaError_t atomic_throughput(int device, unsigned log2_slots, unsigned per_thread, double* atomics_per_s, double* ms_out) {
    DeviceGuard guard;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    const size_t n = (size_t)1 << log2_slots;
    unsigned long long* d = nullptr;
    e = cudaMalloc(&d, n * sizeof(unsigned long long));
    if (e != cudaSuccess) return e;
    cudaEvent_t a = nullptr, b = nullptr;
    const dim3 grid(sms * 8), block(256);
    float ms = 0.0f;
    e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) e = cudaMemset(d, 0, n * sizeof(unsigned long long));
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // the first launch warms up
        cudaEventRecord(a);
        atomic_probe_kernel<<<grid, block>>>(d, n - 1, per_thread);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    }
    if (e == cudaSuccess) {
        *atomics_per_s = (double)grid.x * block.x * per_thread / (ms * 1e-3);
        *ms_out = ms;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(d);
    return e;
}

cudaError_t enqueue_transport(Context* ctx) {
    const KParams& kp = ctx->kp;
    const bool log = kp.mode == 0 && (kp.flags & XMC_DETECTOR_TRAJ) && kp.xlog && kp.xlog_cap > 0;
    const dim3 g(ctx->grid), b(ctx->block);
    if (kp.use_bias) {
        if (log) transport_kernel<true, true><<<g, b, ctx->smem_bytes, ctx->stream>>>(kp);
        else transport_kernel<true, false><<<g, b, ctx->smem_bytes, ctx->stream>>>(kp);
    } else {
        if (log) transport_kernel<false, true><<<g, b, ctx->smem_bytes, ctx->stream>>>(kp);
        else transport_kernel<false, false><<<g, b, ctx->smem_bytes, ctx->stream>>>(kp);
    }
    return cudaGetLastError();
}

template <bool kBias, bool kLog>
static cudaError_t occupancy_of(int block, size_t smem, int* blocks_per_sm) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, transport_kernel<kBias, kLog>);
    if (e != cudaSuccess) return e;
    if (block > fa.maxThreadsPerBlock) {
        *blocks_per_sm = 0;
        return cudaSuccess;
    }
    e = cudaFuncSetAttribute(transport_kernel<kBias, kLog>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, transport_kernel<kBias, kLog>, block, smem);
}

// Resident blocks per SM of both variants (with and without the crossing log) of the kernel; sets
// their dynamic shared-memory limit.
cudaError_t transport_occupancy(int block, size_t smem, int* blocks_per_sm, bool bias) {
    int a = 0, b = 0;
    cudaError_t e = bias ? occupancy_of<true, false>(block, smem, &a) : occupancy_of<false, false>(block, smem, &a);
    if (e == cudaSuccess) e = bias ? occupancy_of<true, true>(block, smem, &b) : occupancy_of<false, true>(block, smem, &b);
    *blocks_per_sm = a < b ? a : b;
    return e;
}

cudaError_t device_philox(uint32_t key0, uint32_t key1, uint64_t pid, uint32_t n, uint32_t* host_out) {
    uint4* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(uint4) * (size_t)(n ? n : 1));
    if (e != cudaSuccess) return e;
    philox_probe_kernel<<<(n + 127) / 128, 128>>>(key0, key1, pid, n, d);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(host_out, d, sizeof(uint4) * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e;
}

}  // namespace xmc

// L2 atomic-add throughput of this GPU (roofline of the walk's tallies); allocates its own array.
extern "C" int xmc_atomic_throughput(int device, unsigned log2_slots, unsigned adds_per_thread, double* atomics_per_s,
                                     double* ms) {
    if (!atomics_per_s || !ms || log2_slots < 10 || log2_slots > 30 || adds_per_thread == 0) {
        xmc::set_error("xmc_atomic_throughput: bad arguments");
        return XMC_ERR_INVALID_INPUT;
    }
    cudaError_t e = xmc::atomic_throughput(device, log2_slots, adds_per_thread, atomics_per_s, ms);
    if (e != cudaSuccess) {
        xmc::set_error(std::string("xmc_atomic_throughput: ") + cudaGetErrorString(e));
        return XMC_ERR_DEVICE;
    }
    return XMC_OK;
}

// Host run of the kernel's ray query on the geometry image of `in` (self-test of the traversal).
extern "C" int xmc_debug_nearest(const InputInfo* in, int n_rays, const float* rays, float tmin, float tmax,
                                 float* t_out, int* surf_out, float* normal_out, int flags) {
    xmc::GeomImage g;
    std::string err;
    const bool use_grid = (flags & 1) != 0;
    if (!xmc::build_geometry(in, &g, &err, (flags & 2) ? 0 : -1)) {
        xmc::set_error(err);
        return (flags & 2) ? XMC_ERR_DEVICE : XMC_ERR_INVALID_INPUT;
    }
    xmc::GridImage grid;
    if (use_grid) xmc::build_xy_grid(g, &grid);
    for (int r = 0; r < n_rays; ++r) {
        const float* q = rays + 6 * (size_t)r;
        unsigned retests = 0, nv = 0, nt = 0;
        xmc::Hit h;
        if (!(use_grid && grid.nx > 0 && tmax < INFINITY &&
              xmc::grid_nearest(grid.cells.data(), grid.cell_z.data(), grid.entries.data(), grid.big.data(), (int)(grid.big.size() / 4), grid.x0,
                                grid.y0, grid.icx, grid.icy, grid.nx, grid.ny, g.tris.data(), nullptr, 0, q[0], q[1], q[2],
                                q[3], q[4], q[5], tmin, tmax, -1, retests, nv, nt, h)))
            h = xmc::bvh_nearest(g.nodes.data(), g.tris.data(), g.n_nodes, nullptr, 0, nullptr, 0, q[0], q[1], q[2],
                                 q[3], q[4], q[5], tmin, tmax, -1, retests, nv, nt);
        t_out[r] = h.tri >= 0 ? h.t : INFINITY;
        surf_out[r] = h.tri >= 0 ? xmc::f2i(g.tris[3 * (size_t)h.tri].w) : -1;
        if (normal_out && h.tri >= 0) {
            const float4 a = g.tris[3 * (size_t)h.tri], b = g.tris[3 * (size_t)h.tri + 1], c = g.tris[3 * (size_t)h.tri + 2];
            const float e1x = a.x - b.x, e1y = a.y - b.y, e1z = a.z - b.z, e2x = a.x - c.x, e2y = a.y - c.y, e2z = a.z - c.z;
            float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
            const float nr = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
            normal_out[3 * (size_t)r] = nx * nr; normal_out[3 * (size_t)r + 1] = ny * nr; normal_out[3 * (size_t)r + 2] = nz * nr;
        }
    }
    return XMC_OK;
}
