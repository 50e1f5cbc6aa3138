/*
 * ORACLE — TEST INFRASTRUCTURE ONLY. Nothing in the product (the xmcml_b200 package, its CUDA
 * kernels, its C-ABI library) links, loads or calls this file; only tests/, the smoke check and
 * the CPU-baseline leg of bench.py use it, as the checker.
 *
 * FP64 CPU restatement of xMCML's photon walk (the hot path behind LaunchOMP), written from the
 * reference's source, one function per reference function, each citing the reference file:line
 * it follows (paths are relative to the reference project root):
 *   base/xmcml/xmcml/mcml_kernel.cpp        ComputePhoton walk, optics, detectors, tallies
 *   base/xmcml/xmcml/mcml_intersection.cpp  ray-triangle distance, nearest hit
 *   base/xmcml/xmcml/mcml_mcg59.cpp         MCG59 generator
 *   base/xmcml/xmcmlLauncher/launcher_omp.cpp  the photon loop and output accumulation
 *
 * Parity pins: with rng_kind = ORACLE_RNG_MCG59, one thread, roulette off and all tallies on, the
 * walk reproduces the reference compiled here (oracle/_ref) bit for bit (tests/test_oracle_vs_ref.py);
 * the function-level known-answer vectors of the reference's own unit tests
 * (stable/1.2/xmcml/xmcml_tests/*.cpp) are checked in tests/test_oracle_kat.py.
 *
 * Extensions beyond the reference (used to check the GPU path, each off by default):
 *   - counter RNG: Philox4x32-10 keyed by (seed, photon id), one block of 4 uniforms per walk
 *     iteration with fixed slots, identical to the GPU kernel's, so both draw the same numbers;
 *   - Russian roulette at minWeight (stable/plane_parallel/1.0/McmlGpu/kernel/kernel.cu:214-222);
 *   - an energy ledger: escaped top/bottom, absorbed outside Area, lost to the Area kill, the
 *     weight cut, glass misses and the step budget, roulette killed/gained weight;
 *   - no Area kill (photons leaving Area keep walking), a uniform-disk beam radius;
 *   - sums of squared detector and time-bin weights for per-bin Monte Carlo variances.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/xmcml_b200.h"

#define O_PI 3.14159265358979323846
#define O_COSINE_OF_ZERO (1.0 - 1.0E-12)  /* mcml_kernel.cpp:11 */
#define O_COSINE_OF_90D 1.0E-12           /* mcml_kernel.cpp:12 */
#define O_MIN_DISTANCE 1.0E-8             /* mcml_kernel.cpp:13 */
#define O_EPSILON 1E-6                    /* mcml_intersection.h:6 */
#define O_MAX_DISTANCE 1.0E+256           /* mcml_intersection.h:7 */

#define ORACLE_RNG_MCG59 0
#define ORACLE_RNG_PHILOX 1

#define OFLAG_ROULETTE (1u << 0)
#define OFLAG_NO_AREA_KILL (1u << 1)
#define OFLAG_SCATTERING (1u << 2)
#define OFLAG_TRAJECTORY (1u << 3)

typedef struct oracle_opts {
    uint32_t flags;
    int32_t rng_kind;
    double roulette_chance;
    double beam_radius;
    uint64_t max_steps;
    int32_t nthreads;
    int32_t pad;
} oracle_opts;

typedef struct oracle_ledger {
    uint64_t launched, terminated, steps;
    uint64_t n_escaped_top, n_escaped_bottom, n_area, n_cut, n_roulette, n_glass, n_budget,
        n_invalid, n_detected;
    double specular, absorbed, absorbed_outside, escaped_top, escaped_bottom, lost_area, lost_cut,
        lost_glass, lost_budget, lost_invalid, roulette_killed, roulette_gained;
    double absorbed_target; /* weight dropped in layers flagged in targetRangeLayers (inside or outside Area) */
    double bias_gained, bias_lost; /* weight added / removed by the biasing weight factor */
} oracle_ledger;

/* ------------------------------------------------------------------------ RNG: MCG59 */

/* mcml_mcg59.cpp:3-5 */
#define MCG59_C 302875106592253ULL
#define MCG59_M 576460752303423488ULL
#define MCG59_DEC_M 576460752303423487ULL

/* mcml_mcg59.cpp:7-22 (square-and-multiply power mod 2^64) */
static uint64_t o_raise(uint64_t a, uint32_t p) {
    uint64_t r = 1;
    while (p > 0) {
        if ((p & 1) == 0) { a *= a; p >>= 1; }
        else { r *= a; --p; }
    }
    return r;
}

/* mcml_mcg59.cpp:24-32 */
void oracle_mcg59_init(MCG59* g, uint64_t seed, uint32_t id, uint32_t step) {
    uint64_t v = 2 * seed + 1;
    v = (v * o_raise(MCG59_C, id)) & MCG59_DEC_M;
    g->value = v;
    g->offset = o_raise(MCG59_C, step);
}

/* mcml_mcg59.cpp:34-38 */
double oracle_mcg59_next(MCG59* g) {
    g->value = (g->value * g->offset) & MCG59_DEC_M;
    return (double)(g->value) / MCG59_M;
}

/* ------------------------------------------------------------------------ RNG: Philox4x32-10 */

/* Philox4x32 with 10 rounds, as published by Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3" (SC'11): two 32x32->64 multiplications per round, Weyl key schedule. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 24-bit uniform in (0,1): ((x >> 8) + 0.5) * 2^-24, exact in float and double. */
static double o_u24(uint32_t x) { return ((double)(x >> 8) + 0.5) * (1.0 / 16777216.0); }

typedef struct o_rng {
    int kind;
    MCG59* mcg;           /* MCG59: the reference's sequential stream */
    uint32_t key[2];      /* Philox key = seed */
    uint64_t pid;         /* Philox photon id */
    uint32_t iter;        /* walk iteration (Philox counter word 2) */
    double u[4];          /* current block */
} o_rng;

static void o_rng_block(o_rng* r) {
    if (r->kind != ORACLE_RNG_PHILOX) return;
    uint32_t ctr[4] = {(uint32_t)r->pid, (uint32_t)(r->pid >> 32), r->iter, 0u};
    uint32_t out[4];
    oracle_philox4x32_10(ctr, r->key, out);
    for (int i = 0; i < 4; ++i) r->u[i] = o_u24(out[i]);
    r->iter++;
}

/* Draw for slot `slot` of the current iteration (Philox) or the next MCG59 value. */
static double o_draw(o_rng* r, int slot) {
    if (r->kind == ORACLE_RNG_PHILOX) return r->u[slot];
    return oracle_mcg59_next(r->mcg);
}

/* ------------------------------------------------------------------------ vector math */
/* mcml_math.cpp:6-74 */
static double3 v3(double x, double y, double z) { double3 r; r.x = x; r.y = y; r.z = z; return r; }
static double3 o_sub(double3 a, double3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static double3 o_div(double3 a, double b) { return v3(a.x / b, a.y / b, a.z / b); }
static double o_dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double o_len(double3 a) { return sqrt(o_dot(a, a)); }
static double3 o_norm(double3 a) { return o_div(a, o_len(a)); }
static double3 o_cross(double3 a, double3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* mcml_math.cpp:45-50 */
static double3 o_plane_normal(double3 a, double3 b, double3 c) { return o_cross(o_sub(a, b), o_sub(a, c)); }

/* mcml_math.cpp:52-80 */
static double3 o_plane_segment(double3 a, double3 b, double z) {
    double3 n = v3(0.0, 0.0, 1.0);
    double3 v = v3(-a.x, -a.y, z - a.z);
    double d = o_dot(n, v);
    double3 w = o_sub(b, a);
    double e = o_dot(n, w);
    double3 r;
    if (e != 0.0) {
        r.x = a.x + w.x * (d / e);
        r.y = a.y + w.y * (d / e);
        r.z = a.z + w.z * (d / e);
        if (o_dot(o_sub(a, r), o_sub(b, r)) > 0.0) r = v3(O_MAX_DISTANCE, O_MAX_DISTANCE, O_MAX_DISTANCE);
    } else {
        r = v3(O_MAX_DISTANCE, O_MAX_DISTANCE, O_MAX_DISTANCE);
    }
    return r;
}

/* ------------------------------------------------------------------------ geometry */

/* mcml_intersection.cpp:44-86 (Moller-Trumbore with the reference's det epsilon) */
double oracle_triangle_distance(double3 o, double3 d, double3 a, double3 b, double3 c) {
    double3 e1 = o_sub(b, a), e2 = o_sub(c, a);
    double3 p = o_cross(d, e2);
    double det = o_dot(e1, p);
    if (det < O_EPSILON && det > -O_EPSILON) return O_MAX_DISTANCE;
    double inv = 1.0 / det;
    double3 t = o_sub(o, a);
    double u = o_dot(t, p) * inv;
    if (u < 0.0 || u > 1.0) return O_MAX_DISTANCE;
    double3 q = o_cross(t, e1);
    double v = o_dot(d, q) * inv;
    if (v < 0.0 || u + v > 1.0) return O_MAX_DISTANCE;
    return o_dot(e2, q) * inv;
}

/* Flattened triangle list + a median-split BVH of the oracle's own (only for speed on large
 * meshes; the nearest hit it returns is the same as an exhaustive search). */
typedef struct o_tri { int surf, idx; double3 a, b, c; } o_tri;
typedef struct o_node { double lo[3], hi[3]; int left, right, first, count; } o_node;
typedef struct o_geom {
    o_tri* tris; int ntris;
    o_node* nodes; int nnodes;
    int* order;
} o_geom;

static void o_tri_bounds(const o_tri* t, double lo[3], double hi[3]) {
    for (int k = 0; k < 3; ++k) {
        double a = t->a.cell[k], b = t->b.cell[k], c = t->c.cell[k];
        lo[k] = fmin(a, fmin(b, c));
        hi[k] = fmax(a, fmax(b, c));
    }
}

static o_geom* o_geom_cmp_ctx;
static int o_geom_axis;
static int o_cmp_centroid(const void* x, const void* y) {
    const o_tri* t = o_geom_cmp_ctx->tris;
    int i = *(const int*)x, j = *(const int*)y;
    double ci = t[i].a.cell[o_geom_axis] + t[i].b.cell[o_geom_axis] + t[i].c.cell[o_geom_axis];
    double cj = t[j].a.cell[o_geom_axis] + t[j].b.cell[o_geom_axis] + t[j].c.cell[o_geom_axis];
    if (ci < cj) return -1;
    if (ci > cj) return 1;
    return i - j;
}

static int o_build(o_geom* g, int first, int count) {
    int id = g->nnodes++;
    o_node* n = &g->nodes[id];
    for (int k = 0; k < 3; ++k) { n->lo[k] = 1e300; n->hi[k] = -1e300; }
    for (int i = first; i < first + count; ++i) {
        double lo[3], hi[3];
        o_tri_bounds(&g->tris[g->order[i]], lo, hi);
        for (int k = 0; k < 3; ++k) { n->lo[k] = fmin(n->lo[k], lo[k]); n->hi[k] = fmax(n->hi[k], hi[k]); }
    }
    if (count <= 4) { n->left = n->right = -1; n->first = first; n->count = count; return id; }
    int axis = 0;
    double ext = -1;
    for (int k = 0; k < 3; ++k) if (n->hi[k] - n->lo[k] > ext) { ext = n->hi[k] - n->lo[k]; axis = k; }
    o_geom_cmp_ctx = g; o_geom_axis = axis;
    qsort(g->order + first, (size_t)count, sizeof(int), o_cmp_centroid);
    int half = count / 2;
    n->first = -1; n->count = 0;
    int l = o_build(g, first, half);
    int r = o_build(g, first + half, count - half);
    g->nodes[id].left = l; g->nodes[id].right = r;
    return id;
}

static o_geom* o_geom_create(const InputInfo* in) {
    o_geom* g = (o_geom*)calloc(1, sizeof(o_geom));
    int n = 0;
    for (int s = 0; s < in->numberOfSurfaces; ++s) n += in->surface[s].numberOfTriangles;
    g->ntris = n;
    g->tris = (o_tri*)malloc(sizeof(o_tri) * (size_t)(n > 0 ? n : 1));
    g->order = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int k = 0;
    for (int s = 0; s < in->numberOfSurfaces; ++s) {
        const Surface* S = &in->surface[s];
        for (int j = 0; j < S->numberOfTriangles; ++j, ++k) {
            int3 T = S->triangles[j];
            g->tris[k].surf = s; g->tris[k].idx = j;
            g->tris[k].a = S->vertices[T.x]; g->tris[k].b = S->vertices[T.y]; g->tris[k].c = S->vertices[T.z];
            g->order[k] = k;
        }
    }
    g->nodes = (o_node*)malloc(sizeof(o_node) * (size_t)(2 * (n > 0 ? n : 1)));
    g->nnodes = 0;
    if (n > 0) o_build(g, 0, n);
    return g;
}

static void o_geom_free(o_geom* g) {
    if (!g) return;
    free(g->tris); free(g->order); free(g->nodes); free(g);
}

/* Conservative slab test: does the box overlap the ray segment [0, tmax]? */
static int o_box_hit(const o_node* n, double3 o, double3 d, double tmax) {
    double t0 = 0.0, t1 = tmax;
    for (int k = 0; k < 3; ++k) {
        double ok = o.cell[k], dk = d.cell[k];
        double lo = n->lo[k], hi = n->hi[k];
        if (dk == 0.0) {
            if (ok < lo || ok > hi) return 0;
        } else {
            double ta = (lo - ok) / dk, tb = (hi - ok) / dk;
            if (ta > tb) { double x = ta; ta = tb; tb = x; }
            /* widen by a relative margin so boundary-touching triangles are never culled */
            double m = 1e-9 * (fabs(ta) + fabs(tb) + 1.0);
            ta -= m; tb += m;
            if (ta > t0) t0 = ta;
            if (tb < t1) t1 = tb;
            if (t0 > t1) return 0;
        }
    }
    return 1;
}

/* Nearest hit with t >= 0 (and t <= step when bounded), the reference's result contract of
 * ComputeBVHIntersection / ComputeBVHIntersectionWithoutStep (mcml_intersection.cpp:354-584):
 * the smallest distance wins; among equal distances the first in surface/triangle order. */
static IntersectionInfo o_nearest(const o_geom* g, double3 o, double3 d, double step, int bounded) {
    IntersectionInfo r;
    memset(&r, 0, sizeof(r));
    r.isFindIntersection = 0;
    r.distance = O_MAX_DISTANCE;
    int best = -1;
    double best_t = O_MAX_DISTANCE;
    if (g->ntris == 0) return r;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    double limit = bounded ? step : 1e300;
    while (sp > 0) {
        const o_node* n = &g->nodes[stack[--sp]];
        double tm = best_t < limit ? best_t : limit;
        if (!o_box_hit(n, o, d, tm)) continue;
        if (n->count > 0) {
            for (int i = n->first; i < n->first + n->count; ++i) {
                int ti = g->order[i];
                const o_tri* t = &g->tris[ti];
                double dist = oracle_triangle_distance(o, d, t->a, t->b, t->c);
                if (dist >= 0.0 && (dist < best_t || (dist == best_t && ti < best))) {
                    best_t = dist; best = ti;
                }
            }
        } else {
            if (sp + 2 > 128) continue;
            stack[sp++] = n->right;
            stack[sp++] = n->left;
        }
    }
    if (best >= 0 && (!bounded || best_t <= step)) {
        const o_tri* t = &g->tris[best];
        r.distance = best_t;
        r.surfaceId = t->surf;
        r.isFindIntersection = 1;
        r.normal = o_norm(o_plane_normal(t->a, t->b, t->c));
    }
    return r;
}

/* ------------------------------------------------------------------------ optics (mcml_kernel.cpp) */

/* mcml_kernel.cpp:16-37 */
double oracle_specular_reflectance(const LayerInfo* layer) {
    double r1, r2, t = (layer[0].refractiveIndex - layer[1].refractiveIndex) /
                       (layer[0].refractiveIndex + layer[1].refractiveIndex);
    r1 = t * t;
    if (layer[1].absorptionCoefficient == 0.0 && layer[1].scatteringCoefficient == 0.0) {
        t = (layer[1].refractiveIndex - layer[2].refractiveIndex) /
            (layer[1].refractiveIndex + layer[2].refractiveIndex);
        r2 = t * t;
        t = 1 - r1;
        r1 = r1 + t * t * r2 / (1 - r1 * r2);
    }
    return r1;
}

/* mcml_kernel.cpp:475-495 (HG inverse CDF), given the uniform */
double oracle_hg_cos(double g, double u) {
    double c;
    if (g != 0.0) {
        double t = (1 - g * g) / (1 - g + 2 * g * u);
        c = (1 + g * g - t * t) / (2 * g);
    } else {
        c = 2.0 * u - 1.0;
    }
    if (c > 1.0) c = 1.0;
    else if (c < -1.0) c = -1.0;
    return c;
}

/* mcml_kernel.cpp:442-473 (spin), given cos(theta) and the azimuth uniform */
double3 oracle_spin(double3 u, double cost, double upsi) {
    double3 r;
    double sint = sqrt(1.0 - cost * cost);
    double psi = 2.0 * O_PI * upsi;
    double cp = cos(psi), sp = sin(psi);
    if (fabs(u.z) <= O_COSINE_OF_ZERO) {
        double t = sqrt(1.0 - u.z * u.z);
        r.x = sint * (u.x * u.z * cp - u.y * sp) / t + u.x * cost;
        r.y = sint * (u.y * u.z * cp + u.x * sp) / t + u.y * cost;
        r.z = -sint * cp * t + u.z * cost;
    } else {
        double t = (u.z >= 0.0) ? 1.0 : -1.0;
        r.x = sint * cp;
        r.y = sint * sp;
        r.z = t * cost;
    }
    return r;
}

/* mcml_kernel.cpp:497-529 */
double oracle_transmit_cos(double ni, double nt, double ci) {
    if (ni == nt) return ci;
    if (ci > O_COSINE_OF_ZERO) return ci;
    if (ci < O_COSINE_OF_90D) return 0.0;
    double si = sqrt(1.0 - ci * ci);
    double st = ni * si / nt;
    if (st >= 1.0) return 0.0;
    return sqrt(1.0 - st * st);
}

/* mcml_kernel.cpp:531-564 */
double oracle_fresnel(double ni, double nt, double ci, double ct) {
    double r;
    if (ni == nt) {
        r = 0.0;
    } else if (ci > O_COSINE_OF_ZERO) {
        r = (nt - ni) / (nt + ni);
        r *= r;
    } else if (ci < O_COSINE_OF_90D) {
        r = 1.0;
    } else {
        double si = sqrt(1.0 - ci * ci);
        double st = sqrt(1.0 - ct * ct);
        double cs = ci * ct - si * st;
        double cd = ci * ct + si * st;
        double ss = si * ct + ci * st;
        double sd = si * ct - ci * st;
        r = 0.5 * sd * sd * (cd * cd + cs * cs) / (ss * ss * cd * cd);
    }
    return r;
}

/* mcml_kernel.cpp:566-580 */
int oracle_find_layer(const InputInfo* in, int surf, int cur) {
    for (int i = 0; i < in->numberOfLayers; ++i)
        for (int j = 0; j < in->layerInfo[i].numberOfSurfaces; ++j)
            if (in->layerInfo[i].surfaceId[j] == surf && i != cur) return i;
    return -1;
}

/* mcml_kernel.cpp:582-593 */
double3 oracle_reflect(double3 i, double3 n) {
    double3 sn = o_norm(n), si = o_norm(i);
    double t = 2 * o_dot(si, sn);
    sn.x *= t; sn.y *= t; sn.z *= t;
    return o_norm(o_sub(si, sn));
}

/* mcml_kernel.cpp:595-616 */
double3 oracle_refract(double ni, double nt, double3 i, double3 n) {
    double3 si = o_norm(i);
    si.x *= ni; si.y *= ni; si.z *= ni;
    double3 sn = o_norm(n);
    double t1 = o_dot(si, sn);
    double t2 = sqrt((nt * nt - ni * ni) / (t1 * t1) + 1);
    t2 = (t2 - 1) * t1;
    return o_norm(v3(si.x + t2 * sn.x, si.y + t2 * sn.y, si.z + t2 * sn.z));
}

/* mcml_kernel.cpp:644-661 */
double oracle_critical_cos(const LayerInfo* layer, int cur, int next) {
    double a = layer[cur].refractiveIndex, b = layer[next].refractiveIndex;
    if (a > b) return sqrt(1.0 - b * b / (a * a));
    return 0.0;
}

/* mcml_kernel.cpp:190-213: voxel index vector with the reference's byte casts (255 = outside) */
static byte3 o_area_vec(double3 p, const Area* a) {
    byte3 r;
    r.x = 255; r.y = 255; r.z = 255;
    double ix = a->partitionNumber.x * (p.x - a->corner.x) / a->length.x;
    double iy = a->partitionNumber.y * (p.y - a->corner.y) / a->length.y;
    double iz = a->partitionNumber.z * (p.z - a->corner.z) / a->length.z;
    int in = !((ix < 0.0 || ix >= a->partitionNumber.x) || (iy < 0.0 || iy >= a->partitionNumber.y) ||
               (iz < 0.0 || iz >= a->partitionNumber.z));
    if (in) { r.x = (byte)ix; r.y = (byte)iy; r.z = (byte)iz; }
    return r;
}

/* mcml_kernel.cpp:215-227 */
int oracle_area_index(double3 p, const Area* a) {
    byte3 v = o_area_vec(p, a);
    if (v.x == 255 && v.y == 255 && v.z == 255) return -1;
    return v.x * a->partitionNumber.y * a->partitionNumber.z + v.y * a->partitionNumber.z + v.z;
}

/* mcml_kernel.cpp:663-742 */
int oracle_detector_id(const InputInfo* in, double3 pos, double3 dir, const bool* visited) {
    for (int i = 0; i < in->numberOfCubeDetectors; ++i) {
        const CubeDetector* c = &in->cubeDetector[i];
        double3 h = v3(c->length.x / 2.0, c->length.y / 2.0, c->length.z / 2.0);
        int inside = (pos.x >= (c->center.x - h.x)) && (pos.x < (c->center.x + h.x)) &&
                     (pos.y >= (c->center.y - h.y)) && (pos.y < (c->center.y + h.y)) &&
                     (pos.z >= (c->center.z - h.z)) && (pos.z < (c->center.z + h.z));
        if (inside) {
            int hit = 0;
            for (int j = 0; j < MAX_LAYERS; ++j) if (visited[j] && c->filterLayers[j]) { hit = 1; break; }
            if (hit) {
                double l2 = dir.x * dir.x + dir.y * dir.y + dir.z * dir.z;
                if ((-dir.z) / l2 > cos(c->targetAngle * O_PI / 180.0)) return i;
            }
        }
    }
    for (int i = 0; i < in->numberOfRingDetectors; ++i) {
        const RingDetector* rd = &in->ringDetector[i];
        double dist = sqrt(((pos.x - rd->center.x) * (pos.x - rd->center.x)) +
                           ((pos.y - rd->center.y) * (pos.y - rd->center.y)));
        if (dist >= rd->smallRadius && dist < rd->bigRadius) {
            int hit = 0;
            for (int j = 0; j < MAX_LAYERS; ++j) if (visited[j] && rd->filterLayers[j]) { hit = 1; break; }
            if (hit) {
                double l2 = dir.x * dir.x + dir.y * dir.y + dir.z * dir.z;
                if ((-dir.z) / l2 > cos(rd->targetAngle * O_PI / 180.0)) return in->numberOfCubeDetectors + i;
            }
        }
    }
    return -1;
}

/* ------------------------------------------------------------------------ the walk */

typedef struct o_photon {
    double3 pos, dir;
    double step;
    int layer;
    bool visited[MAX_LAYERS];
    double weight, time, target_range, other_range;
    int dead;
    uint64_t iters;
} o_photon;

typedef struct o_traj { byte x[MAX_TRAJECTORY_SIZE], y[MAX_TRAJECTORY_SIZE], z[MAX_TRAJECTORY_SIZE]; int n; } o_traj;

typedef struct o_out {        /* per-thread partial output */
    double* absorption;
    double* scattering;
    double* det_w2;           /* [D] */
    double* time_w2;          /* [D*T] */
    oracle_ledger led;
} o_out;

typedef struct o_ctx {
    const InputInfo* in;
    OutputInfo* out;          /* shared detector tallies (updated under a lock when threaded) */
    const oracle_opts* opt;
    const o_geom* geom;
    double rsp;
} o_ctx;

/* mcml_kernel.cpp:750-792 (z-plane crossings at voxel centres: scattering map + crossing log) */
static void o_update_traj(const o_ctx* C, o_out* po, o_photon* ph, o_traj* tr, double3 prev) {
    if (!(C->opt->flags & (OFLAG_SCATTERING | OFLAG_TRAJECTORY))) return;
    const Area* a = C->in->area;
    double3 s, f;
    if (ph->pos.z > prev.z) { s = prev; f = ph->pos; }
    else if (ph->pos.z < prev.z) { s = ph->pos; f = prev; }
    else return;
    double step = a->length.z / a->partitionNumber.z;
    int pi = (int)((s.z - a->corner.z + step / 2.0) / step);
    double plane = a->corner.z + pi * step + step / 2.0;
    while ((plane <= f.z) && (plane < a->corner.z + a->length.z)) {
        double3 ip = o_plane_segment(s, f, plane);
        int si = oracle_area_index(ip, a);
        byte3 v = o_area_vec(ip, a);
        if ((v.x == 255 && v.y == 255 && v.z == 255) || si == -1) break;
        if (tr->n < MAX_TRAJECTORY_SIZE) {
            tr->x[tr->n] = v.x; tr->y[tr->n] = v.y; tr->z[tr->n] = v.z;
            ++tr->n;
        }
        if (C->opt->flags & OFLAG_SCATTERING) po->scattering[si] += ph->weight;
        plane += step;
    }
}

/* mcml_kernel.cpp:158-174 */
static void o_move(const o_ctx* C, o_out* po, o_photon* ph, o_traj* tr) {
    double3 prev = ph->pos;
    ph->time += ph->step * C->in->layerInfo[ph->layer].refractiveIndex;
    if (C->in->targetRangeLayers[ph->layer]) ph->target_range += ph->step;
    else ph->other_range += ph->step;
    ph->pos.x += ph->step * ph->dir.x;
    ph->pos.y += ph->step * ph->dir.y;
    ph->pos.z += ph->step * ph->dir.z;
    o_update_traj(C, po, ph, tr, prev);
}

/* mcml_kernel.cpp:176-188 */
static void o_move_min(const o_ctx* C, o_out* po, o_photon* ph, o_traj* tr) {
    double3 prev = ph->pos;
    ph->pos.x += O_MIN_DISTANCE * ph->dir.x;
    ph->pos.y += O_MIN_DISTANCE * ph->dir.y;
    ph->pos.z += O_MIN_DISTANCE * ph->dir.z;
    o_update_traj(C, po, ph, tr, prev);
}

/* mcml_kernel.cpp:744-858: detector weight, trajectory replay + count, time bins, ranges */
static void o_detect(const o_ctx* C, o_out* po, o_photon* ph, o_traj* tr, int det) {
    OutputInfo* out = C->out;
    DetectorInfo* D = &out->detectorInfo[det];
    double w = ph->weight;
    double total = ph->target_range + ph->other_range;
    double tw = ph->target_range * (w / total);
#ifdef _OPENMP
#pragma omp critical(oracle_detect)
#endif
    {
        D->weight += w;                                            /* :744-748 */
        if (C->opt->flags & OFLAG_TRAJECTORY) {                    /* :794-810 */
            const Area* a = C->in->area;
            for (int i = 0; i < tr->n; ++i) {
                int idx = tr->x[i] * a->partitionNumber.y * a->partitionNumber.z +
                          tr->y[i] * a->partitionNumber.z + tr->z[i];
                ++(D->trajectory[idx]);
            }
        }
        ++(D->numberOfPhotons);
        int T = D->timeScaleSize;                                  /* :812-849 */
        TimeInfo* ts = D->timeScale;
        int bin = -1;
        for (int i = 0; i < T - 1; ++i)
            if (ph->time >= ts[i].timeStart && ph->time < ts[i].timeFinish) { bin = i; break; }
        if (bin < 0 && ph->time >= ts[T - 1].timeStart) bin = T - 1;
        if (bin >= 0) {
            ts[bin].targetWeight += tw;
            ++(ts[bin].numberOfPhotons);
            ts[bin].weight += w;
            po->time_w2[det * T + bin] += w * w;
        }
        D->targetWeight += tw;                                     /* :851-858 */
    }
    po->det_w2[det] += w * w;
    po->led.n_detected++;
}

/* mcml_kernel.cpp:229-284 */
static void o_cross_boundary(const o_ctx* C, o_out* po, o_photon* ph, IntersectionInfo* hit, o_rng* rng,
                    o_traj* tr, int slot) {
    const InputInfo* in = C->in;
    double ci = o_dot(ph->dir, hit->normal);
    if (ci < 0.0) ci = -ci;
    int cur = ph->layer;
    int next = oracle_find_layer(in, hit->surfaceId, cur);
    if (next < 0) {  /* the reference indexes layerInfo[-1] here; the oracle records it instead */
        po->led.n_invalid++; po->led.lost_invalid += ph->weight; ph->dead = 1; return;
    }
    double cc = oracle_critical_cos(in->layerInfo, cur, next);
    double R;
    if (ci <= cc) {
        R = 1.0;
    } else {
        double ct = oracle_transmit_cos(in->layerInfo[cur].refractiveIndex, in->layerInfo[next].refractiveIndex, ci);
        R = oracle_fresnel(in->layerInfo[cur].refractiveIndex, in->layerInfo[next].refractiveIndex, ci, ct);
    }
    if (o_draw(rng, slot) > R) {
        if (next == 0) {
            int det = oracle_detector_id(in, ph->pos, ph->dir, ph->visited);
            if (det >= 0) o_detect(C, po, ph, tr, det);
            if (ph->dir.z < 0.0) { po->led.n_escaped_top++; po->led.escaped_top += ph->weight; }
            else { po->led.n_escaped_bottom++; po->led.escaped_bottom += ph->weight; }
            ph->dead = 1;
        } else {
            ph->dir = oracle_refract(in->layerInfo[cur].refractiveIndex, in->layerInfo[next].refractiveIndex, ph->dir, hit->normal);
            ph->layer = next;
            ph->visited[next] = true;
            o_move_min(C, po, ph, tr);
        }
    } else {
        ph->dir = oracle_reflect(ph->dir, hit->normal);
        o_move_min(C, po, ph, tr);
    }
}

/* mcml_kernel.cpp:128-149 (+ optional uniform-disk beam) */
static void o_launch(const o_ctx* C, o_photon* ph, o_rng* rng) {
    const InputInfo* in = C->in;
    memset(ph, 0, sizeof(*ph));
    ph->weight = 1.0 - C->rsp;
    ph->dead = 0;
    ph->layer = 1;
    ph->pos.x = in->startPosition.x;
    ph->pos.y = in->startPosition.y;
    ph->pos.z = in->startPosition.z + O_MIN_DISTANCE;
    if (C->opt->beam_radius > 0.0 && rng->kind == ORACLE_RNG_PHILOX) {
        uint32_t ctr[4] = {(uint32_t)rng->pid, (uint32_t)(rng->pid >> 32), 0u, 1u}, out[4];
        oracle_philox4x32_10(ctr, rng->key, out);
        double r = C->opt->beam_radius * sqrt(o_u24(out[0]));
        double phi = 2.0 * O_PI * o_u24(out[1]);
        ph->pos.x += r * cos(phi);
        ph->pos.y += r * sin(phi);
    }
    ph->dir = in->startDirection;
    for (int i = 0; i < MAX_LAYERS; ++i) ph->visited[i] = false;
    ph->visited[1] = true;
}

static void o_absorb_outside(o_out* po, o_photon* ph, const InputInfo* in) {
    const LayerInfo* L = &in->layerInfo[ph->layer];
    double dw = ph->weight * L->absorptionCoefficient / (L->absorptionCoefficient + L->scatteringCoefficient);
    ph->weight -= dw;
    po->led.absorbed_outside += dw;
    if (in->targetRangeLayers[ph->layer]) po->led.absorbed_target += dw;
}

/* ------------------------------------------------------------------------ biasing */

/* mcml_kernel.cpp:325-364: the local attractive direction at the photon, the normalised
 * difference of the fields of two point sources placed on the vertical through the target point:
 * one l_tr above it, one l_tr + 2 delta below it (l_tr = 3D, D = 1 / (3 ((1 - g) mus + mua)),
 * delta = 0.74 l_tr), positions relative to the start position. */
static double3 o_attractive(const InputInfo* in, const o_photon* ph) {
    const LayerInfo* L = &in->layerInfo[ph->layer];
    double g = L->anisotropy, mus = L->scatteringCoefficient, mua = L->absorptionCoefficient;
    double3 r = o_sub(ph->pos, in->startPosition);
    double3 rd = o_sub(in->targetPoint, in->startPosition);
    double diff = 1 / (3 * ((1 - g) * mus + mua));
    double ltr = 3 * diff;
    double delta = 0.74 * ltr;
    double3 above = rd, below = rd;
    above.z += ltr;
    below.z -= ltr + 2 * delta;
    double3 fa = o_sub(r, above);
    double la = o_len(fa);
    fa = o_div(fa, la * la * la);
    double3 fb = o_sub(r, below);
    double lb = o_len(fb);
    fb = o_div(fb, lb * lb * lb);
    return o_norm(o_sub(fb, fa));
}

/* mcml_kernel.cpp:430-440: the table of the layer's anisotropy (the last exact match) */
static int o_weight_table(const InputInfo* in, double g) {
    int found = -1;
    for (int i = 0; i < in->numberOfWeightTables; ++i)
        if (in->weightTable[i].anisotropy == g) found = i;
    return found;
}

#define O_BIAS_MAX_TRIALS 65536u

/* mcml_kernel.cpp:398-428: direction by rejection from HG with acceptance
 * p = (0.1 + 0.9 (1 + d.v) / 2)^attractiveFactor, then weight *= W(d_old.v) / p with W from the
 * weight-integral table (nearest node). MCG59: the draws are HG cos, azimuth, acceptance per trial,
 * in that order. Philox: trial k uses the block of counter (id, iteration, 2 + k), slots 0, 1, 2;
 * after O_BIAS_MAX_TRIALS trials the last candidate is taken (never reached for moderate factors). */
static void o_biased_spin(const o_ctx* C, o_out* po, o_photon* ph, o_rng* rng) {
    const InputInfo* in = C->in;
    double g = in->layerInfo[ph->layer].anisotropy;
    double3 v = o_attractive(in, ph);
    double3 nd;
    double p = 1.0;
    for (uint32_t k = 0;; ++k) {
        double u1, u2, u3;
        if (rng->kind == ORACLE_RNG_PHILOX) {
            uint32_t ctr[4] = {(uint32_t)rng->pid, (uint32_t)(rng->pid >> 32), rng->iter - 1u, 2u + k};
            uint32_t out[4];
            oracle_philox4x32_10(ctr, rng->key, out);
            u1 = o_u24(out[0]); u2 = o_u24(out[1]); u3 = o_u24(out[2]);
        } else {
            u1 = oracle_mcg59_next(rng->mcg);
            u2 = oracle_mcg59_next(rng->mcg);
            u3 = oracle_mcg59_next(rng->mcg);
        }
        nd = oracle_spin(ph->dir, oracle_hg_cos(g, u1), u2);
        p = 0.1 + 0.9 * ((1 + o_dot(nd, v)) / 2);
        p = pow(p, in->attractiveFactor);
        if (p > u3) break;
        if (rng->kind == ORACLE_RNG_PHILOX && k + 1 >= O_BIAS_MAX_TRIALS) break;
    }
    int ti = o_weight_table(in, g);
    if (ti >= 0) {
        const WeightIntegralTable* T = &in->weightTable[ti];
        double a = -1.0, b = 1.0;
        int n = T->numberOfElements - 1;
        double step = (b - a) / n;
        double dot = o_dot(ph->dir, v);
        int e = (int)floor((dot - a) / step + 0.5);
        double nw = ph->weight * T->elements[e] / p;
        if (nw > ph->weight) po->led.bias_gained += nw - ph->weight;
        else po->led.bias_lost += ph->weight - nw;
        ph->weight = nw;
    }
    ph->dir = nd;
}

/* mcml_integration.cpp:7-83: W(dot) = (1 / 2 pi) * integral over the sphere of the HG phase
 * function about a direction at cosine `dot` to the attractive direction, times the acceptance
 * (0.1 + 0.45 (1 + cos))^eps, by the product two-point Gauss-Legendre rule on n x n cells of
 * (theta, phi) in [0, pi] x [0, 2 pi]. */
double oracle_weight_integral(double dot, double g, double eps, unsigned n) {
    const double coeff = 2.0 * sqrt(3.0);  /* Gauss nodes at the midpoint +- h / (2 sqrt 3) */
    const double hx = O_PI / n, hy = 2 * O_PI / n;
    const double g2 = g * g;
    const double s = sqrt(1 - dot * dot);
    double total = 0.0;
    for (unsigned i = 0; i < n; ++i) {
        double x0 = hx * i, x1 = x0 + hx;
        double xs[2] = {0.5 * (x0 + x1) + (x1 - x0) / coeff, 0.5 * (x0 + x1) - (x1 - x0) / coeff};
        for (unsigned j = 0; j < n; ++j) {
            double y0 = hy * j, y1 = y0 + hy;
            double ys[2] = {0.5 * (y0 + y1) + (y1 - y0) / coeff, 0.5 * (y0 + y1) - (y1 - y0) / coeff};
            double cell = 0.0;
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b) {
                    double st = sin(xs[a]);
                    double along = st * cos(ys[b]);                     /* cosine to the attractive direction */
                    double c = dot * along + s * st * sin(ys[b]);       /* cosine to the photon direction */
                    double q = 1 + g2 - 2 * g * c;
                    double f = (1 - g2) / (2 * q * sqrt(q));
                    cell += f * pow(0.1 + 0.9 * 0.5 * (1 + along), eps) * st;
                }
            total += 0.25 * (x1 - x0) * (y1 - y0) * cell;
        }
    }
    return total / (2.0 * O_PI);
}

/* weight_integral.cpp:67-104 and :34-65: one table per distinct anisotropy of layers 1..L-1,
 * weightTablePrecision + 1 nodes over dot in [-1, 1], integral precision scaled up for strongly
 * forward-peaked layers. Tables are malloc'ed; free with oracle_free_weight_tables. */
int oracle_weight_tables(InputInfo* in) {
    double gs[MAX_LAYERS];
    int ng = 0;
    for (int l = 1; l < in->numberOfLayers; ++l) {
        double g = in->layerInfo[l].anisotropy;
        int seen = 0;
        for (int k = 0; k < ng; ++k) if (gs[k] == g) seen = 1;
        if (!seen) gs[ng++] = g;
    }
    in->numberOfWeightTables = ng;
    in->weightTable = (WeightIntegralTable*)calloc((size_t)(ng > 0 ? ng : 1), sizeof(WeightIntegralTable));
    for (int k = 0; k < ng; ++k) {
        unsigned prec = in->weightIntegralPrecision;
        if (gs[k] > 0.98) prec *= 16;
        else if (gs[k] > 0.97) prec *= 8;
        else if (gs[k] > 0.95) prec *= 4;
        else if (gs[k] > 0.90) prec *= 2;
        WeightIntegralTable* T = &in->weightTable[k];
        T->anisotropy = gs[k];
        T->numberOfElements = (int)in->weightTablePrecision + 1;
        T->elements = (double*)malloc(sizeof(double) * (size_t)T->numberOfElements);
        double step = 2.0 / in->weightTablePrecision;
        for (int j = 0; j < T->numberOfElements; ++j)
            T->elements[j] = oracle_weight_integral(-1.0 + j * step, gs[k], in->attractiveFactor, prec);
    }
    return ng;
}

void oracle_free_weight_tables(InputInfo* in) {
    for (int k = 0; k < in->numberOfWeightTables; ++k) free(in->weightTable[k].elements);
    free(in->weightTable);
    in->weightTable = NULL;
    in->numberOfWeightTables = 0;
}

/* mcml_kernel.cpp:39-126: one photon, start to death */
static void o_photon_walk(const o_ctx* C, o_out* po, o_rng* rng, o_traj* tr) {
    const InputInfo* in = C->in;
    const oracle_opts* opt = C->opt;
    int area_kill = !(opt->flags & OFLAG_NO_AREA_KILL);
    o_photon ph;
    tr->n = 0;
    o_launch(C, &ph, rng);
    po->led.launched++;
    po->led.specular += C->rsp;
    while (!ph.dead) {
        if (ph.iters >= opt->max_steps) {
            po->led.n_budget++; po->led.lost_budget += ph.weight; ph.dead = 1; break;
        }
        ph.iters++;
        po->led.steps++;
        o_rng_block(rng);
        int roulette_slot;
        const LayerInfo* L = &in->layerInfo[ph.layer];
        int glass = (L->absorptionCoefficient == 0.0) && (L->scatteringCoefficient == 0.0);
        if (glass) {
            IntersectionInfo hit = o_nearest(C->geom, ph.pos, ph.dir, 0.0, 0);
            roulette_slot = 1;
            if (hit.isFindIntersection) {
                ph.step = hit.distance - 0.01 * O_MIN_DISTANCE;
                o_move(C, po, &ph, tr);
                if (!area_kill || oracle_area_index(ph.pos, in->area) >= 0) o_cross_boundary(C, po, &ph, &hit, rng, tr, 0);
                else { ph.dead = 1; po->led.n_area++; po->led.lost_area += ph.weight; }
            } else {
                ph.dead = 1; po->led.n_glass++; po->led.lost_glass += ph.weight;
            }
        } else {
            /* mcml_kernel.cpp:618-631 */
            double u;
            do { u = o_draw(rng, 0); } while (u == 0.0);
            ph.step = -log(u) / (L->absorptionCoefficient + L->scatteringCoefficient);
            IntersectionInfo hit = o_nearest(C->geom, ph.pos, ph.dir, ph.step, 1);
            if (hit.isFindIntersection) {
                roulette_slot = 2;
                ph.step = hit.distance - 0.01 * O_MIN_DISTANCE;
                o_move(C, po, &ph, tr);
                if (!area_kill || oracle_area_index(ph.pos, in->area) >= 0) o_cross_boundary(C, po, &ph, &hit, rng, tr, 1);
                else { ph.dead = 1; po->led.n_area++; po->led.lost_area += ph.weight; }
            } else {
                roulette_slot = 3;
                o_move(C, po, &ph, tr);
                int idx = oracle_area_index(ph.pos, in->area);
                if (idx >= 0 || !area_kill) {
                    if (idx >= 0) {
                        /* mcml_kernel.cpp:633-642 */
                        double dw = ph.weight * L->absorptionCoefficient / (L->absorptionCoefficient + L->scatteringCoefficient);
                        ph.weight -= dw;
                        po->absorption[idx] += dw;
                        po->led.absorbed += dw;
                        if (in->targetRangeLayers[ph.layer]) po->led.absorbed_target += dw;
                    } else {
                        o_absorb_outside(po, &ph, in);
                    }
                    if (in->useBiasing) {  /* mcml_kernel.cpp:108-109 */
                        o_biased_spin(C, po, &ph, rng);
                    } else {
                        double cost = oracle_hg_cos(L->anisotropy, o_draw(rng, 1));
                        ph.dir = oracle_spin(ph.dir, cost, o_draw(rng, 2));
                    }
                } else {
                    ph.dead = 1; po->led.n_area++; po->led.lost_area += ph.weight;
                }
            }
        }
        if (!ph.dead && ph.weight < in->minWeight) {   /* mcml_kernel.cpp:121-124 */
            if (opt->flags & OFLAG_ROULETTE) {
                /* stable/plane_parallel/1.0/McmlGpu/kernel/kernel.cu:214-222 */
                if (ph.weight == 0.0) { ph.dead = 1; po->led.n_roulette++; }
                else if (o_draw(rng, roulette_slot) < opt->roulette_chance) {
                    double nw = ph.weight / opt->roulette_chance;
                    po->led.roulette_gained += nw - ph.weight;
                    ph.weight = nw;
                } else {
                    po->led.n_roulette++; po->led.roulette_killed += ph.weight; ph.dead = 1;
                }
            } else {
                po->led.n_cut++; po->led.lost_cut += ph.weight; ph.dead = 1;
            }
        }
    }
    po->led.terminated++;
}

static void o_out_alloc(o_out* po, int grid, int D, int T) {
    memset(po, 0, sizeof(*po));
    po->absorption = (double*)calloc((size_t)grid, sizeof(double));
    po->scattering = (double*)calloc((size_t)grid, sizeof(double));
    po->det_w2 = (double*)calloc((size_t)(D > 0 ? D : 1), sizeof(double));
    po->time_w2 = (double*)calloc((size_t)(D * T > 0 ? D * T : 1), sizeof(double));
}

static void o_out_free(o_out* po) {
    free(po->absorption); free(po->scattering); free(po->det_w2); free(po->time_w2);
}

static void o_led_add(oracle_ledger* a, const oracle_ledger* b) {
    a->launched += b->launched; a->terminated += b->terminated; a->steps += b->steps;
    a->n_escaped_top += b->n_escaped_top; a->n_escaped_bottom += b->n_escaped_bottom;
    a->n_area += b->n_area; a->n_cut += b->n_cut; a->n_roulette += b->n_roulette;
    a->n_glass += b->n_glass; a->n_budget += b->n_budget; a->n_invalid += b->n_invalid;
    a->n_detected += b->n_detected;
    a->specular += b->specular; a->absorbed += b->absorbed; a->absorbed_outside += b->absorbed_outside;
    a->escaped_top += b->escaped_top; a->escaped_bottom += b->escaped_bottom;
    a->lost_area += b->lost_area; a->lost_cut += b->lost_cut; a->lost_glass += b->lost_glass;
    a->lost_budget += b->lost_budget; a->lost_invalid += b->lost_invalid;
    a->roulette_killed += b->roulette_killed; a->roulette_gained += b->roulette_gained;
    a->absorbed_target += b->absorbed_target;
    a->bias_gained += b->bias_gained; a->bias_lost += b->bias_lost;
}

void oracle_default_opts(oracle_opts* o) {
    memset(o, 0, sizeof(*o));
    o->flags = OFLAG_SCATTERING | OFLAG_TRAJECTORY;
    o->rng_kind = ORACLE_RNG_MCG59;
    o->roulette_chance = 0.1;
    o->max_steps = 10000000ULL;
    o->nthreads = 1;
}

/*
 * launcher_omp.cpp:123-163 restated: photons [first_id, first_id + n) are walked and the tallies
 * are ADDED to `out` (absorption/scattering per voxel, detector weights, counts, time bins,
 * ranges); out->specularReflectance is set. With ORACLE_RNG_MCG59, `mcg` is the reference's
 * per-thread generator array (only mcg[0] is used, one thread, photons in order); with
 * ORACLE_RNG_PHILOX, photon i draws from Philox(seed, first_id + i), threads run photons in any
 * order and the result does not depend on the thread count beyond FP64 summation order.
 * det_w2[D] and time_w2[D*T] (optional) receive sums of squared detected weights.
 */
int oracle_run(const InputInfo* in, OutputInfo* out, const oracle_opts* opt_in, uint64_t seed,
               uint64_t first_id, uint64_t n, MCG59* mcg, oracle_ledger* ledger, double* det_w2,
               double* time_w2) {
    oracle_opts opt;
    if (opt_in) opt = *opt_in; else oracle_default_opts(&opt);
    if (opt.max_steps == 0) opt.max_steps = 10000000ULL;
    int grid = out->gridSize;
    int D = out->numberOfDetectors;
    int T = D > 0 ? out->detectorInfo[0].timeScaleSize : 1;
    o_geom* g = o_geom_create(in);
    o_ctx C;
    C.in = in; C.out = out; C.opt = &opt; C.geom = g;
    C.rsp = oracle_specular_reflectance(in->layerInfo);
    int nth = 1;
#ifdef _OPENMP
    if (opt.rng_kind == ORACLE_RNG_PHILOX && opt.nthreads > 1) nth = opt.nthreads;
#endif
    o_out* parts = (o_out*)calloc((size_t)nth, sizeof(o_out));
    for (int t = 0; t < nth; ++t) o_out_alloc(&parts[t], grid, D, T);
    if (opt.rng_kind == ORACLE_RNG_MCG59) {
        o_traj* tr = (o_traj*)malloc(sizeof(o_traj));
        o_rng rng;
        memset(&rng, 0, sizeof(rng));
        rng.kind = ORACLE_RNG_MCG59;
        rng.mcg = mcg;
        for (uint64_t i = 0; i < n; ++i) o_photon_walk(&C, &parts[0], &rng, tr);
        free(tr);
    } else {
#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
#endif
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            o_traj* tr = (o_traj*)malloc(sizeof(o_traj));
            o_rng rng;
            memset(&rng, 0, sizeof(rng));
            rng.kind = ORACLE_RNG_PHILOX;
            rng.key[0] = (uint32_t)seed;
            rng.key[1] = (uint32_t)(seed >> 32);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
            for (long long i = 0; i < (long long)n; ++i) {
                rng.pid = first_id + (uint64_t)i;
                rng.iter = 0;
                o_photon_walk(&C, &parts[t], &rng, tr);
            }
            free(tr);
        }
    }
    out->specularReflectance = C.rsp;
    oracle_ledger led;
    memset(&led, 0, sizeof(led));
    for (int t = 0; t < nth; ++t) {
        for (int j = 0; j < grid; ++j) {
            out->absorption[j] += parts[t].absorption[j];
            out->scattering[j] += parts[t].scattering[j];
        }
        if (det_w2) for (int d = 0; d < D; ++d) det_w2[d] += parts[t].det_w2[d];
        if (time_w2) for (int k = 0; k < D * T; ++k) time_w2[k] += parts[t].time_w2[k];
        o_led_add(&led, &parts[t].led);
        o_out_free(&parts[t]);
    }
    free(parts);
    o_geom_free(g);
    if (ledger) o_led_add(ledger, &led);
    return 0;
}

/* ------------------------------------------------------------------------ KAT entry points */

/* mcml_kernel.cpp:475-495 with the generator, as the reference's tests call it */
double oracle_kat_cosine_theta(double g, MCG59* r) { return oracle_hg_cos(g, oracle_mcg59_next(r)); }

/* mcml_kernel.cpp:442-473 with the generator (theta draw first, then psi) */
void oracle_kat_new_direction(const double* dir_in, double g, MCG59* r, double* dir_out) {
    double3 u = v3(dir_in[0], dir_in[1], dir_in[2]);
    double c = oracle_hg_cos(g, oracle_mcg59_next(r));
    double3 o = oracle_spin(u, c, oracle_mcg59_next(r));
    dir_out[0] = o.x; dir_out[1] = o.y; dir_out[2] = o.z;
}

/* mcml_kernel.cpp:618-631 */
double oracle_kat_step_size(double mua, double mus, MCG59* r) {
    double u;
    do { u = oracle_mcg59_next(r); } while (u == 0.0);
    return -log(u) / (mua + mus);
}

/* mcml_kernel.cpp:633-642: returns the new weight, *dw the dropped weight */
double oracle_kat_drop(double w, double mua, double mus, double* dw) {
    double d = w * mua / (mua + mus);
    *dw = d;
    return w - d;
}

double oracle_kat_area_index(const double* p, const Area* a) { return (double)oracle_area_index(v3(p[0], p[1], p[2]), a); }

double oracle_kat_triangle(const double* o, const double* d, const double* a, const double* b, const double* c) {
    return oracle_triangle_distance(v3(o[0], o[1], o[2]), v3(d[0], d[1], d[2]), v3(a[0], a[1], a[2]),
                                    v3(b[0], b[1], b[2]), v3(c[0], c[1], c[2]));
}

void oracle_kat_reflect(const double* i, const double* n, double* out) {
    double3 r = oracle_reflect(v3(i[0], i[1], i[2]), v3(n[0], n[1], n[2]));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

void oracle_kat_refract(double ni, double nt, const double* i, const double* n, double* out) {
    double3 r = oracle_refract(ni, nt, v3(i[0], i[1], i[2]), v3(n[0], n[1], n[2]));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

/* Nearest hit of the oracle's search over all surfaces of `in` (for geometry parity tests). */
int oracle_kat_nearest(const InputInfo* in, const double* o, const double* d, double step, int bounded,
                       double* dist, int* surf, double* normal) {
    o_geom* g = o_geom_create(in);
    IntersectionInfo h = o_nearest(g, v3(o[0], o[1], o[2]), v3(d[0], d[1], d[2]), step, bounded);
    o_geom_free(g);
    *dist = h.distance;
    *surf = h.isFindIntersection ? h.surfaceId : -1;
    if (h.isFindIntersection) { normal[0] = h.normal.x; normal[1] = h.normal.y; normal[2] = h.normal.z; }
    return h.isFindIntersection;
}

/* The same for n rays (rays[6*i]: origin, direction) over one geometry build. */
int oracle_kat_nearest_batch(const InputInfo* in, int n, const double* rays, double step, int bounded,
                             double* dist, int* surf, double* normal) {
    o_geom* g = o_geom_create(in);
    int hits = 0;
    for (int i = 0; i < n; ++i) {
        const double* q = rays + 6 * (size_t)i;
        IntersectionInfo h = o_nearest(g, v3(q[0], q[1], q[2]), v3(q[3], q[4], q[5]), step, bounded);
        dist[i] = h.distance;
        surf[i] = h.isFindIntersection ? h.surfaceId : -1;
        if (h.isFindIntersection) {
            normal[3 * (size_t)i] = h.normal.x; normal[3 * (size_t)i + 1] = h.normal.y; normal[3 * (size_t)i + 2] = h.normal.z;
            ++hits;
        }
    }
    o_geom_free(g);
    return hits;
}
