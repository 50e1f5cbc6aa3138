// Batched planar transport: many optical-property instances of one planar layer stack in one
// persistent launch (no counterpart in the reference, which runs one model per LaunchOMP call,
// base/xmcml/xmcmlLauncher/launcher_omp.cpp:123-163).
//
// An instance is the planar model of the reference's walk (ComputePhoton,
// base/xmcml/xmcml/mcml_kernel.cpp:39-126): ambient medium above and below, tissue layers between
// horizontal planes, a pencil beam (or uniform disk) at normal incidence, ring detectors around the
// beam axis and time bins in optical path length. For horizontal planes the ray query of the
// mesh kernel reduces to one division, (z_plane - z) / uz, and the surface normal is the z axis, so
// this kernel carries no BVH and keeps the current layer's constants in registers.
//
// All instances share one photon-id dispenser: instance k owns the global indices
// [first_k, first_k + photons_k), a warp claims `chunk` consecutive indices at a time and each lane
// maps its index to (instance, photon id) with a binary search over first_k (usually a hit on the
// lane's previous instance). Random numbers are Philox4x32-10 keyed by the instance seed with
// counter (photon id, iteration, 0) and the same slot use as the mesh kernel, so instance k
// reproduces photon for photon a single run of the same model with that seed.
//
// Tallies per instance: rings (weight, count, weight^2), ring x time bins (same) and a ledger of
// XMC_BATCH_LEDGER 64-bit slots; weights are 2^31 fixed point, so every sum is exact and the
// results do not depend on the launch shape. Tally scheme 0 adds each photon's ledger terms with
// global atomics when it dies; scheme 1 keeps them in registers while a thread walks photons of one
// instance and flushes when it moves on (fewer atomics on the hot ledger words).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "photon.cuh"
#include "xmc_internal.h"

namespace xmc {
namespace {

constexpr unsigned FULL = 0xffffffffu;

struct BInst {                 // 32 B per instance
    unsigned long long first;  // first global photon index of the instance
    unsigned long long count;  // photons of the instance
    uint32_t key0, key1;       // counter-RNG key: the instance seed
    uint32_t w0;               // start weight after specular reflection (2^31 fixed point)
    float beam_radius;         // mm
};

// Layers of an instance: 0 ambient above, 1..n_layers tissue, n_layers + 1 ambient below; three
// float4 each: {z_top, z_bot, 1/(mua+mus), mua/(mua+mus)}, {1-g^2, 1+g^2, 1/2g, 1-g}, {2g, n, 0, 0}.
constexpr int kLayerF4 = 3;

struct BatchParams {
    const BInst* inst;
    const float4* layers;
    const unsigned long long* hdr;  // [0] instances, [1] photons of all instances
    int stride;                     // n_layers + 2
    int n_layers;
    int n_rings, n_time;
    float ring_width, inv_ring_width, cos_angle;
    float t0, inv_dt;  // inv_dt == 0: a single bin
    uint32_t w_min;
    float chance, inv_chance;
    unsigned long long max_steps;
    int chunk;
    unsigned long long* counter;
    int* status;
    unsigned long long* ring;    // [instance][ring][3]
    unsigned long long* tbin;    // [instance][ring][time][3]
    unsigned long long* ledger;  // [instance][XMC_BATCH_LEDGER]
};

struct LayerRegs {
    float z_top, z_bot, inv_mut, absorb, hg_a, hg_b, hg_c, hg_d, hg_e, n;
};

__device__ __forceinline__ void load_layer(const float4* __restrict__ p, LayerRegs& L) {
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    L.z_top = a.x; L.z_bot = a.y; L.inv_mut = a.z; L.absorb = a.w;
    L.hg_a = b.x; L.hg_b = b.y; L.hg_c = b.z; L.hg_d = b.w;
    L.hg_e = c.x; L.n = c.y;
}

// Instance owning global photon index g: the hint when it matches, else the last instance whose
// first index is <= g (instances without photons share their successor's first index).
__device__ __forceinline__ int find_instance(const BInst* __restrict__ I, int n, unsigned long long g, int hint) {
    if (hint >= 0) {
        const unsigned long long f = __ldg(&I[hint].first), c = __ldg(&I[hint].count);
        if (g >= f && g - f < c) return hint;
    }
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&I[mid].first) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void lat(unsigned long long* p, unsigned long long v) {
    if (v) atomicAdd(p, v);
}

template <int kScheme>
__global__ void __launch_bounds__(256, 3) batch_kernel(const BatchParams P) {
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int n_inst = (int)P.hdr[0];
    const unsigned long long total = P.hdr[1];

    unsigned long long cbeg = 0, cend = 0;  // warp-uniform chunk of global photon indices
    bool exhausted = false, alive = false;
    float px = 0.0f, py = 0.0f, pz = 0.0f, dx = 0.0f, dy = 0.0f, dz = 1.0f, time = 0.0f;
    uint32_t w = 0, iter = 0, key0 = 0, key1 = 0;
    int layer = 1, inst = -1;
    unsigned long long pid = 0;  // photon id within its instance
    LayerRegs L{};
    // ledger sums: of one photon (scheme 0) or of a run of photons of instance a_inst (scheme 1)
    unsigned long long a_abs = 0, a_gain = 0, a_kill = 0, a_steps = 0;
    unsigned a_launched = 0, a_nroul = 0;
    int a_inst = -1;
    unsigned budget_hit = 0;

    auto flush = [&](int k) {
        if (k < 0) return;
        unsigned long long* led = P.ledger + (size_t)k * XMC_BATCH_LEDGER;
        lat(&led[XMC_BL_LAUNCHED], a_launched);
        lat(&led[XMC_BL_STEPS], a_steps);
        lat(&led[XMC_BL_ABSORBED_FX], a_abs);
        lat(&led[XMC_BL_RGAINED_FX], a_gain);
        lat(&led[XMC_BL_RKILLED_FX], a_kill);
        lat(&led[XMC_BL_N_ROULETTE], a_nroul);
        a_launched = 0; a_nroul = 0;
        a_abs = 0; a_gain = 0; a_kill = 0; a_steps = 0;
    };
    auto die = [&]() {
        alive = false;
        a_steps += iter;
        if (kScheme == 0) flush(inst);
    };

    for (;;) {
        // ---- refill dead lanes with new photons (warp-level compaction) ----
        unsigned need = __ballot_sync(FULL, !alive && !exhausted);
        while (need) {
            if (cbeg == cend) {
                unsigned long long b = 0;
                if (lane == 0) b = atomicAdd(P.counter, (unsigned long long)P.chunk);
                b = __shfl_sync(FULL, b, 0);
                if (b >= total) {
                    exhausted = true;
                    break;
                }
                cbeg = b;
                cend = min(b + (unsigned long long)P.chunk, total);
            }
            const unsigned long long avail = cend - cbeg;
            const int rank = __popc(need & lt_mask);
            const int take = (int)min((unsigned long long)__popc(need), avail);
            if (((need >> lane) & 1u) && rank < take) {
                const unsigned long long g = cbeg + rank;
                const int k = find_instance(P.inst, n_inst, g, inst);
                if (kScheme == 1 && k != a_inst) {
                    flush(a_inst);
                    a_inst = k;
                }
                inst = k;
                const BInst* I = P.inst + k;
                pid = g - __ldg(&I->first);
                key0 = __ldg(&I->key0);
                key1 = __ldg(&I->key1);
                w = __ldg(&I->w0);
                // LaunchPhoton (mcml_kernel.cpp:128-149) at the origin, or a uniform disk
                px = 0.0f; py = 0.0f; pz = 0.0f;
                const float br = __ldg(&I->beam_radius);
                if (br > 0.0f) {
                    const uint4 r = philox4x32_10(make_uint4((uint32_t)pid, (uint32_t)(pid >> 32), 0u, 1u), key0, key1);
                    const float rad = br * sqrtf(u24(r.x));
                    float a = u24(r.y);
                    a = a > 0.5f ? a - 1.0f : a;
                    float sp, cp;
                    __sincosf(6.283185307179586f * a, &sp, &cp);
                    px = rad * cp;
                    py = rad * sp;
                }
                dx = 0.0f; dy = 0.0f; dz = 1.0f;
                time = 0.0f;
                layer = 1;
                iter = 0;
                load_layer(P.layers + kLayerF4 * ((size_t)k * P.stride + 1), L);
                a_launched++;
                alive = true;
            }
            cbeg += take;
            need = __ballot_sync(FULL, !alive && !exhausted);
        }
        if (__ballot_sync(FULL, alive) == 0u) break;
        if (!alive) continue;

        // ---- one walk iteration (mcml_kernel.cpp:78-124) ----
        if (iter >= P.max_steps) {
            budget_hit = 1;
            unsigned long long* led = P.ledger + (size_t)inst * XMC_BATCH_LEDGER;
            atomicAdd(&led[XMC_BL_N_BUDGET], 1ull);
            lat(&led[XMC_BL_BUDGET_FX], w);
            die();
            continue;
        }
        const uint4 r = philox4x32_10(make_uint4((uint32_t)pid, (uint32_t)(pid >> 32), iter, 0u), key0, key1);
        iter++;
        float step = -__logf(u24(r.x)) * L.inv_mut;  // ComputeStepSizeInTissue (:618-631)
        // distance to the layer's plane ahead (the reference's ray query against the two planes)
        float tb = INFINITY;
        if (dz > 0.0f) tb = __fdividef(L.z_bot - pz, dz);
        else if (dz < 0.0f) tb = __fdividef(L.z_top - pz, dz);
        tb = fmaxf(tb, 0.0f);
        const bool boundary = tb <= step;
        if (boundary) step = tb;
        // MovePhoton (:151-174): position and optical path length
        px = fmaf(step, dx, px);
        py = fmaf(step, dy, py);
        pz = boundary ? (dz > 0.0f ? L.z_bot : L.z_top) : fmaf(step, dz, pz);
        time = fmaf(step, L.n, time);
        float u_roulette;
        if (boundary) {
            // CrossBoundary (:229-284) at a horizontal interface: incidence cosine |uz|
            u_roulette = u24(r.z);
            const int next = dz > 0.0f ? layer + 1 : layer - 1;
            const float nt = __ldg(&P.layers[kLayerF4 * ((size_t)inst * P.stride + next) + 2]).y;
            const float R = fresnel_reflectance(L.n, nt, fabsf(dz));
            if (u24(r.y) > R) {
                if (next == 0 || next == P.n_layers + 1) {
                    unsigned long long* led = P.ledger + (size_t)inst * XMC_BATCH_LEDGER;
                    if (next == 0) {
                        // leaves through the top: ring detectors (GetDetectorId, :663-742)
                        const float rr = sqrtf(px * px + py * py);
                        const float fr = rr * P.inv_ring_width;
                        int ring = P.n_rings;
                        if (fr < (float)P.n_rings + 1.0f) {
                            // ring i covers [i w, (i+1) w): settle the rounding of the product
                            ring = (int)fr;
                            if (ring > 0 && rr < (float)ring * P.ring_width) ring--;
                            else if (rr >= (float)(ring + 1) * P.ring_width) ring++;
                        }
                        if (ring < P.n_rings && -dz > P.cos_angle) {
                            const unsigned long long w2 = ((unsigned long long)w * w) >> 31;
                            unsigned long long* rt = P.ring + 3 * ((size_t)inst * P.n_rings + ring);
                            atomicAdd(rt + 0, (unsigned long long)w);
                            atomicAdd(rt + 1, 1ull);
                            lat(rt + 2, w2);
                            // UpdateDetectorTimeScale (:812-849): last bin open-ended
                            if (time >= P.t0) {
                                int bin = P.n_time - 1;
                                const float f = (time - P.t0) * P.inv_dt;
                                if (f < (float)(P.n_time - 1)) bin = (int)f;
                                unsigned long long* tt =
                                    P.tbin + 3 * (((size_t)inst * P.n_rings + ring) * P.n_time + bin);
                                atomicAdd(tt + 0, (unsigned long long)w);
                                atomicAdd(tt + 1, 1ull);
                                lat(tt + 2, w2);
                            }
                            atomicAdd(&led[XMC_BL_N_DETECTED], 1ull);
                        }
                        atomicAdd(&led[XMC_BL_N_TOP], 1ull);
                        lat(&led[XMC_BL_TOP_FX], w);
                    } else {
                        atomicAdd(&led[XMC_BL_N_BOTTOM], 1ull);
                        lat(&led[XMC_BL_BOTTOM_FX], w);
                    }
                    die();
                    continue;
                }
                // RefractVector (:595-616) for the normal (0, 0, 1): the tangential part scales by
                // ni / nt, |uz| becomes the transmitted cosine
                const float eta = L.n / nt;
                const float ct = sqrtf(fmaxf(0.0f, 1.0f - eta * eta * (1.0f - dz * dz)));
                dx *= eta;
                dy *= eta;
                dz = dz > 0.0f ? ct : -ct;
                layer = next;
                load_layer(P.layers + kLayerF4 * ((size_t)inst * P.stride + layer), L);
            } else {
                dz = -dz;  // ReflectVector (:582-593)
            }
        } else {
            // drop (ComputeDroppedWeightOfPhoton, :633-642) and spin (:442-495)
            u_roulette = u24(r.w);
            uint32_t dw = __float2uint_rn(__uint2float_rn(w) * L.absorb);
            dw = min(dw, w);
            w -= dw;
            a_abs += dw;
            hg_spin(L.hg_a, L.hg_b, L.hg_c, L.hg_d, L.hg_e, u24(r.y), u24(r.z), dx, dy, dz);
        }
        // roulette below min_weight (weight cut :121-124; roulette as in the planar GPU kernel.cu:214-222)
        if (w < P.w_min) {
            if (w != 0u && u_roulette < P.chance) {
                const uint32_t nw = min(__float2uint_rn(__uint2float_rn(w) * P.inv_chance), kWeightOne);
                a_gain += nw - w;
                w = nw;
            } else {
                a_kill += w;
                a_nroul++;
                die();
            }
        }
    }
    if (kScheme == 1) flush(a_inst);
    if (budget_hit) atomicOr(P.status, 1);
}

// Fixed point -> FP64 fractions of the launched weight (the only FP64 work of a batch run).
__global__ void batch_reduce_kernel(const BInst* __restrict__ inst, const unsigned long long* __restrict__ ring,
                                    const unsigned long long* __restrict__ tbin, int n, int R, int T,
                                    double* __restrict__ ring_out, double* __restrict__ tbin_out) {
    const size_t nrt = (size_t)n * R * T, nr = (size_t)n * R;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrt + nr; i += (size_t)gridDim.x * blockDim.x) {
        if (i < nrt) {
            const size_t k = i / ((size_t)R * T);
            const double s = 1.0 / (kWeightScale * (double)max(inst[k].count, 1ull));
            tbin_out[i] = (double)tbin[3 * i] * s;
        } else {
            const size_t j = i - nrt;
            const size_t k = j / (size_t)R;
            const double s = 1.0 / (kWeightScale * (double)max(inst[k].count, 1ull));
            ring_out[j] = (double)ring[3 * j] * s;
        }
    }
}

int bfail(int status, const std::string& msg) {
    set_error(msg);
    return status;
}

#define XB_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return bfail(XMC_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

bool finite_pos(double x) { return std::isfinite(x) && x > 0.0; }

void normalise_spec(const xmc_batch_spec* in, xmc_batch_spec* s) {
    std::memset(s, 0, sizeof(*s));
    if (in && in->struct_size) std::memcpy(s, in, std::min((size_t)in->struct_size, sizeof(*s)));
    s->struct_size = sizeof(*s);
    if (s->max_steps_per_photon == 0) s->max_steps_per_photon = 10000000ull;
}

int validate_spec(const xmc_batch_spec& s) {
    if (s.n_layers < 1 || s.n_layers > XMC_BATCH_MAX_LAYERS)
        return bfail(XMC_ERR_RANGE, "n_layers must be in [1, " + std::to_string(XMC_BATCH_MAX_LAYERS) + "]");
    if (s.n_rings < 1 || s.n_rings > 4096) return bfail(XMC_ERR_RANGE, "n_rings must be in [1, 4096]");
    if (s.n_time < 1 || s.n_time > 4096) return bfail(XMC_ERR_RANGE, "n_time must be in [1, 4096]");
    if (!finite_pos(s.ring_width)) return bfail(XMC_ERR_INVALID_INPUT, "ring_width must be > 0");
    if (!std::isfinite(s.time_start) || !std::isfinite(s.time_finish) || s.time_finish < s.time_start)
        return bfail(XMC_ERR_INVALID_INPUT, "time window must satisfy time_start <= time_finish");
    if (!(s.ring_angle > 0.0 && s.ring_angle <= 180.0)) return bfail(XMC_ERR_INVALID_INPUT, "ring_angle must be in (0, 180]");
    if (!(s.min_weight >= 0.0 && s.min_weight < 1.0)) return bfail(XMC_ERR_INVALID_INPUT, "min_weight must be in [0, 1)");
    if (!(s.roulette_chance > 0.0 && s.roulette_chance <= 1.0))
        return bfail(XMC_ERR_INVALID_INPUT, "roulette_chance must be in (0, 1]");
    if (s.max_instances < 1 || s.max_instances > (1 << 20)) return bfail(XMC_ERR_RANGE, "max_instances must be in [1, 2^20]");
    if ((double)s.max_instances * s.n_rings * s.n_time * 24.0 > 64e9)
        return bfail(XMC_ERR_RANGE, "ring x time tallies of max_instances exceed 64 GB");
    return XMC_OK;
}

int validate_instances(const xmc_batch_spec& s, const xmc_batch_instance* inst, int n) {
    if (n < 0 || n > s.max_instances) return bfail(XMC_ERR_RANGE, "instance count outside [0, max_instances]");
    if (n > 0 && !inst) return bfail(XMC_ERR_INVALID_INPUT, "instance table is NULL");
    unsigned long long total = 0;
    for (int k = 0; k < n; ++k) {
        const xmc_batch_instance& I = inst[k];
        const std::string who = "instance " + std::to_string(k) + ": ";
        for (int l = 0; l < s.n_layers; ++l) {
            if (!(std::isfinite(I.mua[l]) && I.mua[l] >= 0.0 && std::isfinite(I.mus[l]) && I.mus[l] >= 0.0 &&
                  I.mua[l] + I.mus[l] > 0.0))
                return bfail(XMC_ERR_INVALID_INPUT, who + "layer " + std::to_string(l) + ": need mua, mus >= 0, mua + mus > 0");
            if (!(I.g[l] > -1.0 && I.g[l] < 1.0)) return bfail(XMC_ERR_INVALID_INPUT, who + "anisotropy must be in (-1, 1)");
            if (!finite_pos(I.n[l])) return bfail(XMC_ERR_INVALID_INPUT, who + "refractive index must be > 0");
            if (!finite_pos(I.thickness[l])) return bfail(XMC_ERR_INVALID_INPUT, who + "thickness must be > 0");
        }
        if (!finite_pos(I.n_above) || !finite_pos(I.n_below))
            return bfail(XMC_ERR_INVALID_INPUT, who + "ambient refractive index must be > 0");
        if (!(std::isfinite(I.beam_radius) && I.beam_radius >= 0.0))
            return bfail(XMC_ERR_INVALID_INPUT, who + "beam_radius must be >= 0");
        if (I.photons > (1ull << 48)) return bfail(XMC_ERR_RANGE, who + "more than 2^48 photons");
        total += I.photons;
    }
    if (total > (1ull << 56)) return bfail(XMC_ERR_RANGE, "more than 2^56 photons in one batch");
    return XMC_OK;
}

}  // namespace
}  // namespace xmc

using namespace xmc;

struct xmc_batch {
    xmc_batch_spec spec{};
    int stride = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    xmc_batch_tuning tuning{256, 0, 64, 1, 0.0};
    int grid = 0, block = 0;
    // device
    unsigned char* d_misc = nullptr;  // [0,16) header, [64,72) dispenser, [72,76) status
    BInst* d_inst = nullptr;
    float4* d_layers = nullptr;
    unsigned long long *d_ring = nullptr, *d_tbin = nullptr, *d_ledger = nullptr;
    double *d_ring_f = nullptr, *d_tbin_f = nullptr;
    // pinned host
    unsigned long long* h_hdr = nullptr;
    BInst* h_inst = nullptr;
    float4* h_layers = nullptr;
    double *h_ring_f = nullptr, *h_tbin_f = nullptr;
    unsigned long long* h_ledger = nullptr;
    int* h_status = nullptr;
    std::map<int, cudaGraphExec_t> graphs;  // by instance count, for the current tuning
    int last_n = 0;
};

namespace xmc {
namespace {

void free_batch(xmc_batch* b) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!b) return;
    cudaSetDevice(b->spec.device);
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    void* d[] = {b->d_misc, b->d_inst, b->d_layers, b->d_ring, b->d_tbin, b->d_ledger, b->d_ring_f, b->d_tbin_f};
    for (void* p : d)
        if (p) cudaFree(p);
    void* h[] = {b->h_hdr, b->h_inst, b->h_layers, b->h_ring_f, b->h_tbin_f, b->h_ledger, b->h_status};
    for (void* p : h)
        if (p) cudaFreeHost(p);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

// Host image of n instances into the pinned staging buffers.
void pack(xmc_batch* b, const xmc_batch_instance* inst, int n) {
    const xmc_batch_spec& s = b->spec;
    unsigned long long first = 0;
    for (int k = 0; k < n; ++k) {
        const xmc_batch_instance& I = inst[k];
        BInst& D = b->h_inst[k];
        D.first = first;
        D.count = I.photons;
        first += I.photons;
        D.key0 = (uint32_t)I.seed;
        D.key1 = (uint32_t)(I.seed >> 32);
        // ComputeSpecularReflectance (mcml_kernel.cpp:16-37) for a tissue first layer
        const double t = (I.n_above - I.n[0]) / (I.n_above + I.n[0]);
        D.w0 = (uint32_t)std::llround((1.0 - t * t) * kWeightScale);
        D.beam_radius = (float)I.beam_radius;
        float4* L = b->h_layers + (size_t)kLayerF4 * k * b->stride;
        double z = 0.0;
        L[0] = make_float4(-INFINITY, 0.0f, 0.0f, 0.0f);
        L[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        L[2] = make_float4(0.0f, (float)I.n_above, 0.0f, 0.0f);
        for (int l = 0; l < s.n_layers; ++l) {
            float4* Q = L + kLayerF4 * (l + 1);
            const double mut = I.mua[l] + I.mus[l], g = I.g[l];
            const double z1 = z + I.thickness[l];
            Q[0] = make_float4((float)z, (float)z1, (float)(1.0 / mut), (float)(I.mua[l] / mut));
            Q[1] = make_float4((float)(1 - g * g), (float)(1 + g * g), g != 0.0 ? (float)(1.0 / (2 * g)) : 0.0f, (float)(1 - g));
            Q[2] = make_float4((float)(2 * g), (float)I.n[l], 0.0f, 0.0f);
            z = z1;
        }
        float4* Q = L + kLayerF4 * (s.n_layers + 1);
        Q[0] = make_float4((float)z, INFINITY, 0.0f, 0.0f);
        Q[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        Q[2] = make_float4(0.0f, (float)I.n_below, 0.0f, 0.0f);
    }
    b->h_hdr[0] = (unsigned long long)n;
    b->h_hdr[1] = first;
}

BatchParams params(const xmc_batch* b) {
    const xmc_batch_spec& s = b->spec;
    BatchParams P{};
    P.inst = b->d_inst;
    P.layers = b->d_layers;
    P.hdr = reinterpret_cast<const unsigned long long*>(b->d_misc);
    P.stride = b->stride;
    P.n_layers = s.n_layers;
    P.n_rings = s.n_rings;
    P.n_time = s.n_time;
    P.ring_width = (float)s.ring_width;
    P.inv_ring_width = (float)(1.0 / s.ring_width);
    P.cos_angle = (float)std::cos(s.ring_angle * 3.14159265358979323846 / 180.0);
    P.t0 = (float)s.time_start;
    const double dt = (s.time_finish - s.time_start) / s.n_time;
    P.inv_dt = dt > 0.0 ? (float)(1.0 / dt) : 0.0f;
    double wm = std::ceil(s.min_weight * kWeightScale);
    P.w_min = (uint32_t)std::min(std::max(wm, 0.0), 4294967295.0);
    P.chance = (float)s.roulette_chance;
    P.inv_chance = (float)(1.0 / s.roulette_chance);
    P.max_steps = s.max_steps_per_photon;
    P.chunk = b->tuning.photons_per_chunk;
    P.counter = reinterpret_cast<unsigned long long*>(b->d_misc + 64);
    P.status = reinterpret_cast<int*>(b->d_misc + 72);
    P.ring = b->d_ring;
    P.tbin = b->d_tbin;
    P.ledger = b->d_ledger;
    return P;
}

int occupancy(int scheme, int block, int* occ) {
    cudaError_t e = scheme == 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, batch_kernel<0>, block, 0)
                                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, batch_kernel<1>, block, 0);
    if (e != cudaSuccess) return bfail(XMC_ERR_DEVICE, std::string("occupancy: ") + cudaGetErrorString(e));
    if (*occ <= 0) return bfail(XMC_ERR_INVALID_INPUT, "batched kernel cannot run with this block size");
    return XMC_OK;
}

int apply_tuning(xmc_batch* b, const xmc_batch_tuning& t) {
    if (t.block_size < 32 || t.block_size > 256 || t.block_size % 32)
        return bfail(XMC_ERR_INVALID_INPUT, "block_size must be a multiple of 32 in [32, 256]");
    if (t.photons_per_chunk < 1 || t.photons_per_chunk > (1 << 20))
        return bfail(XMC_ERR_INVALID_INPUT, "photons_per_chunk must be in [1, 2^20]");
    if (t.tally_scheme != 0 && t.tally_scheme != 1) return bfail(XMC_ERR_INVALID_INPUT, "tally_scheme must be 0 or 1");
    if (t.blocks_per_sm < 0) return bfail(XMC_ERR_INVALID_INPUT, "blocks_per_sm must be >= 0");
    int occ = 0;
    int st = occupancy(t.tally_scheme, t.block_size, &occ);
    if (st) return st;
    const int bps = t.blocks_per_sm > 0 ? std::min(t.blocks_per_sm, occ) : occ;
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    b->tuning = t;
    b->tuning.blocks_per_sm = bps;
    b->block = t.block_size;
    b->grid = b->sms * bps;
    return XMC_OK;
}

// The stream work of one run of n instances (n >= 1): upload, zero, transport, reduce, read back.
int enqueue(xmc_batch* b, int n, bool capturing) {
    const xmc_batch_spec& s = b->spec;
    const size_t R = (size_t)s.n_rings, T = (size_t)s.n_time;
    cudaStream_t st = b->stream;
    XB_CUDA(cudaMemcpyAsync(b->d_misc, b->h_hdr, 16, cudaMemcpyHostToDevice, st));
    XB_CUDA(cudaMemcpyAsync(b->d_inst, b->h_inst, sizeof(BInst) * n, cudaMemcpyHostToDevice, st));
    XB_CUDA(cudaMemcpyAsync(b->d_layers, b->h_layers, sizeof(float4) * kLayerF4 * b->stride * (size_t)n,
                            cudaMemcpyHostToDevice, st));
    XB_CUDA(cudaMemsetAsync(b->d_misc + 64, 0, 16, st));
    XB_CUDA(cudaMemsetAsync(b->d_ring, 0, sizeof(unsigned long long) * 3 * R * n, st));
    XB_CUDA(cudaMemsetAsync(b->d_tbin, 0, sizeof(unsigned long long) * 3 * R * T * n, st));
    XB_CUDA(cudaMemsetAsync(b->d_ledger, 0, sizeof(unsigned long long) * XMC_BATCH_LEDGER * n, st));
    if (capturing) XB_CUDA(cudaEventRecordWithFlags(b->ev[0], st, cudaEventRecordExternal));
    else XB_CUDA(cudaEventRecord(b->ev[0], st));
    const BatchParams P = params(b);
    if (b->tuning.tally_scheme == 0) batch_kernel<0><<<b->grid, b->block, 0, st>>>(P);
    else batch_kernel<1><<<b->grid, b->block, 0, st>>>(P);
    XB_CUDA(cudaGetLastError());
    if (capturing) XB_CUDA(cudaEventRecordWithFlags(b->ev[1], st, cudaEventRecordExternal));
    else XB_CUDA(cudaEventRecord(b->ev[1], st));
    const size_t work = (size_t)n * R * (T + 1);
    const int rgrid = (int)std::min<size_t>((work + 255) / 256, (size_t)b->sms * 8);
    batch_reduce_kernel<<<rgrid, 256, 0, st>>>(b->d_inst, b->d_ring, b->d_tbin, n, (int)R, (int)T, b->d_ring_f, b->d_tbin_f);
    XB_CUDA(cudaGetLastError());
    XB_CUDA(cudaMemcpyAsync(b->h_ring_f, b->d_ring_f, sizeof(double) * R * n, cudaMemcpyDeviceToHost, st));
    XB_CUDA(cudaMemcpyAsync(b->h_tbin_f, b->d_tbin_f, sizeof(double) * R * T * n, cudaMemcpyDeviceToHost, st));
    XB_CUDA(cudaMemcpyAsync(b->h_ledger, b->d_ledger, sizeof(unsigned long long) * XMC_BATCH_LEDGER * n,
                            cudaMemcpyDeviceToHost, st));
    XB_CUDA(cudaMemcpyAsync(b->h_status, b->d_misc + 72, sizeof(int), cudaMemcpyDeviceToHost, st));
    return XMC_OK;
}

int graph_for(xmc_batch* b, int n, cudaGraphExec_t* out) {
    auto it = b->graphs.find(n);
    if (it != b->graphs.end()) {
        *out = it->second;
        return XMC_OK;
    }
    XB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue(b, n, true);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return bfail(XMC_ERR_DEVICE, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bfail(XMC_ERR_DEVICE, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    if (b->graphs.size() >= 16) {  // bounded cache of instance counts
        cudaGraphExecDestroy(b->graphs.begin()->second);
        b->graphs.erase(b->graphs.begin());
    }
    b->graphs[n] = ex;
    *out = ex;
    return XMC_OK;
}

// One run of n >= 1 packed instances; waits for it.
int run_packed(xmc_batch* b, int n, bool use_graph, double* kernel_ms) {
    if (use_graph) {
        cudaGraphExec_t ex = nullptr;
        int st = graph_for(b, n, &ex);
        if (st) return st;
        XB_CUDA(cudaGraphLaunch(ex, b->stream));
    } else {
        int st = enqueue(b, n, false);
        if (st) return st;
    }
    XB_CUDA(cudaStreamSynchronize(b->stream));
    float ms = 0.0f;
    XB_CUDA(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
    if (kernel_ms) *kernel_ms = ms;
    b->last_n = n;
    return XMC_OK;
}

}  // namespace
}  // namespace xmc

extern "C" int xmc_batch_validate(const xmc_batch_spec* spec, const xmc_batch_instance* inst, int n) {
    if (!spec) return bfail(XMC_ERR_INVALID_INPUT, "spec is NULL");
    xmc_batch_spec s;
    normalise_spec(spec, &s);
    int st = validate_spec(s);
    if (st) return st;
    return validate_instances(s, inst, n);
}

extern "C" int xmc_batch_create(const xmc_batch_spec* spec, xmc_batch** out) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!out) return bfail(XMC_ERR_INVALID_INPUT, "out is NULL");
    *out = nullptr;
    if (!spec) return bfail(XMC_ERR_INVALID_INPUT, "spec is NULL");
    xmc_batch* b = new (std::nothrow) xmc_batch;
    if (!b) return bfail(XMC_ERR_DEVICE, "out of host memory");
    normalise_spec(spec, &b->spec);
    int st = validate_spec(b->spec);
    if (st) {
        delete b;
        return st;
    }
    const xmc_batch_spec& s = b->spec;
    b->stride = s.n_layers + 2;
    const size_t cap = (size_t)s.max_instances, R = (size_t)s.n_rings, T = (size_t)s.n_time;
#define XB_TRY(call)                                                                             \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                      \
            free_batch(b);                                                                       \
            return XMC_ERR_DEVICE;                                                               \
        }                                                                                        \
    } while (0)
    XB_TRY(cudaSetDevice(s.device));
    XB_TRY(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, s.device));
    XB_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    XB_TRY(cudaEventCreate(&b->ev[0]));
    XB_TRY(cudaEventCreate(&b->ev[1]));
    XB_TRY(cudaMalloc(&b->d_misc, 256));
    XB_TRY(cudaMalloc(&b->d_inst, sizeof(BInst) * cap));
    XB_TRY(cudaMalloc(&b->d_layers, sizeof(float4) * kLayerF4 * b->stride * cap));
    XB_TRY(cudaMalloc(&b->d_ring, sizeof(unsigned long long) * 3 * R * cap));
    XB_TRY(cudaMalloc(&b->d_tbin, sizeof(unsigned long long) * 3 * R * T * cap));
    XB_TRY(cudaMalloc(&b->d_ledger, sizeof(unsigned long long) * XMC_BATCH_LEDGER * cap));
    XB_TRY(cudaMalloc(&b->d_ring_f, sizeof(double) * R * cap));
    XB_TRY(cudaMalloc(&b->d_tbin_f, sizeof(double) * R * T * cap));
    XB_TRY(cudaMallocHost(&b->h_hdr, 16));
    XB_TRY(cudaMallocHost(&b->h_inst, sizeof(BInst) * cap));
    XB_TRY(cudaMallocHost(&b->h_layers, sizeof(float4) * kLayerF4 * b->stride * cap));
    XB_TRY(cudaMallocHost(&b->h_ring_f, sizeof(double) * R * cap));
    XB_TRY(cudaMallocHost(&b->h_tbin_f, sizeof(double) * R * T * cap));
    XB_TRY(cudaMallocHost(&b->h_ledger, sizeof(unsigned long long) * XMC_BATCH_LEDGER * cap));
    XB_TRY(cudaMallocHost(&b->h_status, sizeof(int)));
#undef XB_TRY
    st = apply_tuning(b, b->tuning);
    if (st) {
        free_batch(b);
        return st;
    }
    *out = b;
    return XMC_OK;
}

extern "C" int xmc_batch_run(xmc_batch* b, const xmc_batch_instance* inst, int n, double* ring_time, double* ring,
                             xmc_batch_result* result, double* kernel_ms) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!b) return bfail(XMC_ERR_INVALID_INPUT, "batch is NULL");
    int st = validate_instances(b->spec, inst, n);
    if (st) return st;
    const size_t R = (size_t)b->spec.n_rings, T = (size_t)b->spec.n_time;
    if (kernel_ms) *kernel_ms = 0.0;
    if (n == 0) {
        b->last_n = 0;
        return XMC_OK;
    }
    XB_CUDA(cudaSetDevice(b->spec.device));
    pack(b, inst, n);
    st = run_packed(b, n, b->spec.use_graph != 0, kernel_ms);
    if (st) return st;
    if (ring_time) std::memcpy(ring_time, b->h_tbin_f, sizeof(double) * R * T * n);
    if (ring) std::memcpy(ring, b->h_ring_f, sizeof(double) * R * n);
    if (result) {
        for (int k = 0; k < n; ++k) {
            const unsigned long long* L = b->h_ledger + (size_t)k * XMC_BATCH_LEDGER;
            xmc_batch_result& o = result[k];
            std::memset(&o, 0, sizeof(o));
            o.photons = L[XMC_BL_LAUNCHED];
            o.steps = L[XMC_BL_STEPS];
            o.n_detected = L[XMC_BL_N_DETECTED];
            o.n_top = L[XMC_BL_N_TOP];
            o.n_bottom = L[XMC_BL_N_BOTTOM];
            o.n_roulette = L[XMC_BL_N_ROULETTE];
            o.n_budget = L[XMC_BL_N_BUDGET];
            const double s = 1.0 / (kWeightScale * (double)std::max<unsigned long long>(inst[k].photons, 1ull));
            o.specular = (double)((unsigned long long)(kWeightOne - b->h_inst[k].w0) * o.photons) * s;
            o.escaped_top = (double)L[XMC_BL_TOP_FX] * s;
            o.escaped_bottom = (double)L[XMC_BL_BOTTOM_FX] * s;
            o.absorbed = (double)L[XMC_BL_ABSORBED_FX] * s;
            o.roulette_killed = (double)L[XMC_BL_RKILLED_FX] * s;
            o.roulette_gained = (double)L[XMC_BL_RGAINED_FX] * s;
            o.lost_budget = (double)L[XMC_BL_BUDGET_FX] * s;
        }
    }
    if (*b->h_status & 1) return bfail(XMC_ERR_BUDGET, "a photon reached the step budget and was terminated");
    return XMC_OK;
}

extern "C" int xmc_batch_read_tallies(xmc_batch* b, int n, uint64_t* ring, uint64_t* ring_time, uint64_t* ledger) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!b) return bfail(XMC_ERR_INVALID_INPUT, "batch is NULL");
    if (n < 0 || n > b->last_n) return bfail(XMC_ERR_RANGE, "n exceeds the instance count of the last run");
    if (n == 0) return XMC_OK;
    const size_t R = (size_t)b->spec.n_rings, T = (size_t)b->spec.n_time;
    XB_CUDA(cudaSetDevice(b->spec.device));
    if (ring) XB_CUDA(cudaMemcpy(ring, b->d_ring, sizeof(uint64_t) * 3 * R * n, cudaMemcpyDeviceToHost));
    if (ring_time) XB_CUDA(cudaMemcpy(ring_time, b->d_tbin, sizeof(uint64_t) * 3 * R * T * n, cudaMemcpyDeviceToHost));
    if (ledger) XB_CUDA(cudaMemcpy(ledger, b->d_ledger, sizeof(uint64_t) * XMC_BATCH_LEDGER * n, cudaMemcpyDeviceToHost));
    return XMC_OK;
}

extern "C" int xmc_batch_set_tuning(xmc_batch* b, const xmc_batch_tuning* t) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!b || !t) return bfail(XMC_ERR_INVALID_INPUT, "batch or tuning is NULL");
    XB_CUDA(cudaSetDevice(b->spec.device));
    return apply_tuning(b, *t);
}

extern "C" int xmc_batch_get_tuning(const xmc_batch* b, xmc_batch_tuning* t) {
    if (!b || !t) return bfail(XMC_ERR_INVALID_INPUT, "batch or tuning is NULL");
    *t = b->tuning;
    return XMC_OK;
}

extern "C" int xmc_batch_autotune(xmc_batch* b, const xmc_batch_instance* sample, int n, uint64_t photons_cap,
                                  xmc_batch_tuning* best) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!b) return bfail(XMC_ERR_INVALID_INPUT, "batch is NULL");
    int st = validate_instances(b->spec, sample, n);
    if (st) return st;
    if (n == 0) return bfail(XMC_ERR_INVALID_INPUT, "autotune needs at least one instance");
    XB_CUDA(cudaSetDevice(b->spec.device));
    std::vector<xmc_batch_instance> capped(sample, sample + n);
    for (auto& I : capped)
        if (photons_cap > 0) I.photons = std::min<uint64_t>(I.photons, photons_cap);
    pack(b, capped.data(), n);
    const xmc_batch_tuning keep = b->tuning;
    xmc_batch_tuning win{};
    win.ms = INFINITY;
    const int blocks[] = {64, 128, 256};
    const int chunks[] = {32, 64, 128, 256};
    for (int scheme = 0; scheme < 2; ++scheme)
        for (int bs : blocks)
            for (int ch : chunks) {
                xmc_batch_tuning t{bs, 0, ch, scheme, 0.0};
                if (apply_tuning(b, t)) continue;  // shape does not fit: skip it
                double ms = INFINITY;
                for (int rep = 0; rep < 2; ++rep) {
                    double k = 0.0;
                    st = run_packed(b, n, false, &k);
                    if (st && st != XMC_ERR_BUDGET) {
                        apply_tuning(b, keep);
                        return st;
                    }
                    ms = std::min(ms, k);
                }
                if (ms < win.ms) {
                    win = b->tuning;
                    win.ms = ms;
                }
            }
    if (!std::isfinite(win.ms)) {
        apply_tuning(b, keep);
        return bfail(XMC_ERR_DEVICE, "autotune: no launch shape ran");
    }
    st = apply_tuning(b, win);
    if (st) return st;
    b->tuning.ms = win.ms;
    b->last_n = 0;  // the trial tallies are not a result
    if (best) *best = b->tuning;
    return XMC_OK;
}

extern "C" int xmc_batch_destroy(xmc_batch* b) {
    if (!b) return XMC_OK;
    free_batch(b);
    return XMC_OK;
}
