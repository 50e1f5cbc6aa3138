// C-ABI of the library: context creation (device image upload), runs, tally read-back and the
// reference-signature shims. See include/xmcml_b200.h for the contract of each entry point.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "xmc_internal.h"

namespace xmc {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

static int fail(int status, const std::string& msg) {
    set_error(msg);
    return status;
}

#define XMC_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(XMC_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

static void free_context(Context* c) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!c) return;
    int dev = -1;
    if (cudaGetDevice(&dev) == cudaSuccess && dev != c->device) cudaSetDevice(c->device);
    void* dbufs[] = {c->d_nodes, c->d_tris, c->d_next, c->d_dets, c->d_absorb, c->d_det,
                     c->d_tbin, c->d_ledger, c->d_counter, c->d_status, c->d_scatter, c->d_traj,
                     c->d_replay, c->d_replay_count, c->d_replay_ledger, c->d_cells, c->d_cell_z, c->d_cell_entries,
                     c->d_big, c->d_cancel, c->d_wtab, c->d_xlog, c->d_cell_runs, c->d_nz_counts, c->d_nz_offsets,
                     c->d_nz_tmp, c->d_nz_idx, c->d_nz_val};
    for (void* p : dbufs)
        if (p) cudaFree(p);
    void* hbufs[] = {c->h_cancel, c->h_absorb, c->h_det, c->h_tbin, c->h_ledger, c->h_status, c->h_maps,
                     c->h_nz_offsets, c->h_nz_idx, c->h_nz_val, c->h_traj};
    for (void* p : hbufs)
        if (p) cudaFreeHost(p);
    for (cudaEvent_t& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->cancel_stream) cudaStreamDestroy(c->cancel_stream);
    delete c;
}

static unsigned host_threads_for(size_t n) {
    return n < ((size_t)1 << 18) ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
}

// dst[i] += src[i] * scale, over n elements on up to 16 host threads (the caller's FP64 output
// arrays hold one value per voxel).
static void accumulate(double* dst, const unsigned long long* src, size_t n, double scale) {
    const unsigned hw = host_threads_for(n);
    const size_t per = (n + hw - 1) / hw;
    parallel_parts(hw, [&](unsigned t) {
        const size_t a = std::min(n, t * per), b = std::min(n, a + per);
        for (size_t i = a; i < b; ++i) dst[i] += (double)src[i] * scale;
    });
}

// mcml_kernel.cpp:16-37 (FP64, exactly as the reference computes it)
static double specular(const LayerInfo* layer) {
    double r1, r2, t = (layer[0].refractiveIndex - layer[1].refractiveIndex) /
                       (layer[0].refractiveIndex + layer[1].refractiveIndex);
    r1 = t * t;
    if (layer[1].absorptionCoefficient == 0.0 && layer[1].scatteringCoefficient == 0.0) {
        t = (layer[1].refractiveIndex - layer[2].refractiveIndex) / (layer[1].refractiveIndex + layer[2].refractiveIndex);
        r2 = t * t;
        t = 1 - r1;
        r1 = r1 + t * t * r2 / (1 - r1 * r2);
    }
    return r1;
}

// Dynamic shared memory of a transport block (the kernel's carve-up): block-private ledger and
// detector tallies, staged BVH nodes and triangles, layers, detectors, the transition table and,
// for warp-cooperative queries, one WarpQuery per warp.
static size_t smem_layout(int n_dets, int smem_nodes, int smem_tris, int smem_next, int coop_warps) {
    size_t b = sizeof(unsigned long long) * (size_t)(kLedgerSlots + 4 * n_dets);
    b += sizeof(float4) * (size_t)(2 * smem_nodes + 3 * smem_tris);
    b += sizeof(DevLayer) * MAX_LAYERS;
    b += sizeof(DevDetector) * (size_t)n_dets;
    b += (size_t)smem_next;
    b = (b + 15) & ~(size_t)15;
    b += sizeof(WarpQuery) * (size_t)coop_warps;
    return b;
}

static int validate(const InputInfo* in, const xmc_options& opt) {
    if (!in) return fail(XMC_ERR_INVALID_INPUT, "input is NULL");
    if (in->numberOfLayers < 2 || in->numberOfLayers > MAX_LAYERS)
        return fail(XMC_ERR_RANGE, "numberOfLayers must be in [2, " + std::to_string(MAX_LAYERS) + "]");
    if (!in->layerInfo) return fail(XMC_ERR_INVALID_INPUT, "layerInfo is NULL");
    if (!in->area) return fail(XMC_ERR_INVALID_INPUT, "area is NULL");
    const Area& a = *in->area;
    if (a.partitionNumber.x <= 0 || a.partitionNumber.y <= 0 || a.partitionNumber.z <= 0)
        return fail(XMC_ERR_INVALID_INPUT, "Area partition numbers must be positive");
    if (!(a.length.x > 0 && a.length.y > 0 && a.length.z > 0))
        return fail(XMC_ERR_INVALID_INPUT, "Area lengths must be positive");
    const int maxp = (opt.flags & XMC_LARGE_GRID) ? 4096 : 256;
    if (a.partitionNumber.x > maxp || a.partitionNumber.y > maxp || a.partitionNumber.z > maxp)
        return fail(XMC_ERR_RANGE, "Area partition number above " + std::to_string(maxp) +
                                       " (the reference indexes voxels with bytes; set XMC_LARGE_GRID for full indices)");
    if ((long long)a.partitionNumber.x * a.partitionNumber.y * a.partitionNumber.z > (1ll << 31) - 1)
        return fail(XMC_ERR_RANGE, "Area grid too large");
    if (in->numberOfSurfaces < 0 || (in->numberOfSurfaces > 0 && !in->surface))
        return fail(XMC_ERR_INVALID_INPUT, "surfaces missing");
    if (in->numberOfSurfaces > 4096) return fail(XMC_ERR_RANGE, "more than 4096 surfaces");
    if (in->numberOfCubeDetectors < 0 || in->numberOfRingDetectors < 0 ||
        (in->numberOfCubeDetectors > 0 && !in->cubeDetector) || (in->numberOfRingDetectors > 0 && !in->ringDetector))
        return fail(XMC_ERR_INVALID_INPUT, "detectors missing");
    if (in->numberOfCubeDetectors + in->numberOfRingDetectors > 1024) return fail(XMC_ERR_RANGE, "more than 1024 detectors");
    if (in->timeScaleSize < 1) return fail(XMC_ERR_INVALID_INPUT, "timeScaleSize must be >= 1");
    if ((long long)in->timeScaleSize * (in->numberOfCubeDetectors + in->numberOfRingDetectors) > (1ll << 26))
        return fail(XMC_ERR_RANGE, "time-bin tally too large");
    if (in->useBiasing && !(std::isfinite(in->attractiveFactor) && in->attractiveFactor >= 0))
        return fail(XMC_ERR_INVALID_INPUT, "attractiveFactor must be finite and >= 0");
    for (int l = 0; l < in->numberOfLayers; ++l) {
        const LayerInfo& L = in->layerInfo[l];
        if (L.numberOfSurfaces < 0 || (L.numberOfSurfaces > 0 && !L.surfaceId))
            return fail(XMC_ERR_INVALID_INPUT, "layer " + std::to_string(l) + ": surface ids missing");
        if (!(L.refractiveIndex > 0)) return fail(XMC_ERR_INVALID_INPUT, "layer " + std::to_string(l) + ": refractive index must be > 0");
        if (L.absorptionCoefficient < 0 || L.scatteringCoefficient < 0)
            return fail(XMC_ERR_INVALID_INPUT, "layer " + std::to_string(l) + ": negative coefficients");
    }
    if (!(opt.roulette_chance > 0 && opt.roulette_chance <= 1)) return fail(XMC_ERR_INVALID_INPUT, "roulette_chance must be in (0, 1]");
    if (opt.beam_radius < 0) return fail(XMC_ERR_INVALID_INPUT, "beam_radius must be >= 0");
    if (opt.query_batch < 0 || opt.query_batch > 32) return fail(XMC_ERR_RANGE, "query_batch must be in [0, 32]");
    if (opt.grid_cell_tris < 0 || opt.grid_cell_tris > 4096) return fail(XMC_ERR_RANGE, "grid_cell_tris must be in [0, 4096]");
    if (opt.trajectory_log < -1 || opt.trajectory_log > 65536)
        return fail(XMC_ERR_RANGE, "trajectory_log must be -1, 0 or at most 65536");
    return XMC_OK;
}

int prepare_image(const InputInfo* in, const xmc_options* opt_in, HostImage* img) {
    xmc_options opt;
    xmc_default_options(&opt);
    if (opt_in && opt_in->struct_size) {
        size_t n = std::min((size_t)opt_in->struct_size, sizeof(xmc_options));
        std::memcpy(&opt, opt_in, n);
        opt.struct_size = sizeof(xmc_options);
        if (opt.roulette_chance == 0) opt.roulette_chance = 0.1;
        if (opt.max_steps_per_photon == 0) opt.max_steps_per_photon = 10000000ull;
        if (opt.photons_per_chunk <= 0) opt.photons_per_chunk = 32;
    }
    int st = validate(in, opt);
    if (st) return st;
    img->opt = opt;

    std::string err;
    if (!build_geometry(in, &img->geom, &err, (opt.flags & XMC_GPU_BVH) ? opt.device : -1))
        return fail(err.rfind("GPU BVH", 0) == 0 ? XMC_ERR_DEVICE : XMC_ERR_INVALID_INPUT, err);
    const GeomImage& geom = img->geom;

    KParams& kp = img->kp;
    std::memset(&kp, 0, sizeof(kp));
    // ---- layers ----
    kp.n_layers = in->numberOfLayers;
    for (int l = 0; l < MAX_LAYERS; ++l) {
        DevLayer& D = kp.layer[l];
        std::memset(&D, 0, sizeof(D));
        if (l >= in->numberOfLayers) { D.glass = 1; D.n = 1.0f; continue; }
        const LayerInfo& L = in->layerInfo[l];
        const double mut = L.absorptionCoefficient + L.scatteringCoefficient;
        const double g = L.anisotropy;
        D.n = (float)L.refractiveIndex;
        D.mua = (float)L.absorptionCoefficient;
        D.mus = (float)L.scatteringCoefficient;
        D.g = (float)g;
        D.glass = (L.absorptionCoefficient == 0.0 && L.scatteringCoefficient == 0.0) ? 1 : 0;
        D.inv_mut = D.glass ? 0.0f : (float)(1.0 / mut);
        D.absorb = D.glass ? 0.0f : (float)(L.absorptionCoefficient / mut);
        D.hg_a = (float)(1 - g * g);
        D.hg_b = (float)(1 + g * g);
        D.hg_c = g != 0.0 ? (float)(1.0 / (2 * g)) : 0.0f;
        D.hg_d = (float)(1 - g);
        D.hg_e = (float)(2 * g);
    }
    kp.target_mask = 0;
    for (int l = 0; l < MAX_LAYERS; ++l)
        if (in->targetRangeLayers[l]) kp.target_mask |= 1u << l;
    // ---- surface -> layer transitions: FindIntersectionLayer (mcml_kernel.cpp:566-580) ----
    const int ns = in->numberOfSurfaces;
    std::vector<int8_t>& next = img->next;
    next.assign((size_t)std::max(1, ns) * MAX_LAYERS, (int8_t)-1);
    for (int s = 0; s < ns; ++s)
        for (int cur = 0; cur < MAX_LAYERS; ++cur) {
            int found = -1;
            for (int i = 0; i < in->numberOfLayers && found < 0; ++i)
                for (int j = 0; j < in->layerInfo[i].numberOfSurfaces; ++j)
                    if (in->layerInfo[i].surfaceId[j] == s && i != cur) { found = i; break; }
            next[(size_t)s * MAX_LAYERS + cur] = (int8_t)found;
        }
    kp.n_surf = ns;
    // ---- Area ----
    const Area& A = *in->area;
    kp.ax = (float)A.corner.x; kp.ay = (float)A.corner.y; kp.az = (float)A.corner.z;
    kp.asx = (float)(A.partitionNumber.x / A.length.x);
    kp.asy = (float)(A.partitionNumber.y / A.length.y);
    kp.asz = (float)(A.partitionNumber.z / A.length.z);
    kp.nx = A.partitionNumber.x; kp.ny = A.partitionNumber.y; kp.nz = A.partitionNumber.z;
    kp.byte_sentinel = (A.partitionNumber.x >= 256 && A.partitionNumber.y >= 256 && A.partitionNumber.z >= 256 &&
                        !(opt.flags & XMC_LARGE_GRID)) ? 1 : 0;
    img->grid_size = A.partitionNumber.x * A.partitionNumber.y * A.partitionNumber.z;
    kp.grid = img->grid_size;
    kp.plane_dz = (float)(A.length.z / A.partitionNumber.z);
    kp.area_zend = (float)(A.corner.z + A.length.z);
    // ---- detectors: cubes then rings (GetDetectorId order, mcml_kernel.cpp:663-742) ----
    const int nd = in->numberOfCubeDetectors + in->numberOfRingDetectors;
    std::vector<DevDetector>& dets = img->dets;
    dets.assign((size_t)std::max(1, nd), DevDetector{});
    const double kPi = 3.14159265358979323846;
    for (int i = 0; i < in->numberOfCubeDetectors; ++i) {
        const CubeDetector& D = in->cubeDetector[i];
        DevDetector& o = dets[i];
        o.cx = (float)D.center.x; o.cy = (float)D.center.y; o.cz = (float)D.center.z;
        o.hx = (float)(D.length.x / 2.0); o.hy = (float)(D.length.y / 2.0); o.hz = (float)(D.length.z / 2.0);
        o.cos_angle = (float)std::cos(D.targetAngle * kPi / 180.0);
        o.filter = 0;
        for (int j = 0; j < MAX_LAYERS; ++j) if (D.filterLayers[j]) o.filter |= 1u << j;
    }
    for (int i = 0; i < in->numberOfRingDetectors; ++i) {
        const RingDetector& D = in->ringDetector[i];
        DevDetector& o = dets[in->numberOfCubeDetectors + i];
        o.cx = (float)D.center.x; o.cy = (float)D.center.y; o.cz = (float)D.center.z;
        o.hx = (float)D.smallRadius; o.hy = (float)D.bigRadius; o.hz = 0.0f;
        o.cos_angle = (float)std::cos(D.targetAngle * kPi / 180.0);
        o.filter = 0;
        for (int j = 0; j < MAX_LAYERS; ++j) if (D.filterLayers[j]) o.filter |= 1u << j;
    }
    kp.n_cubes = in->numberOfCubeDetectors;
    kp.n_rings = in->numberOfRingDetectors;
    kp.rings_sorted = in->numberOfRingDetectors > 1 ? 1 : 0;
    for (int i = 0; i < in->numberOfRingDetectors && kp.rings_sorted; ++i) {
        const RingDetector& R = in->ringDetector[i];
        if (R.center.x != in->ringDetector[0].center.x || R.center.y != in->ringDetector[0].center.y ||
            !(R.smallRadius <= R.bigRadius))
            kp.rings_sorted = 0;
        if (i > 0 && !(in->ringDetector[i - 1].bigRadius <= R.smallRadius)) kp.rings_sorted = 0;
    }
    kp.n_dets = nd;
    img->n_dets = nd;
    // ---- time bins: InitOutput (launcher_omp.cpp:36-55) ----
    const int T = in->timeScaleSize;
    double tstep = (in->timeFinish - in->timeStart) / T;
    if (tstep < 0.0) tstep = 0.0;
    kp.t0 = (float)in->timeStart;
    kp.dt = (float)tstep;
    kp.n_time = T;
    img->n_time = T;
    // ---- launch (mcml_kernel.cpp:128-149) ----
    img->rsp = specular(in->layerInfo);
    const double w0 = 1.0 - img->rsp;
    img->w0_fx = (uint32_t)std::llround(w0 * kWeightScale);
    kp.w0 = img->w0_fx;
    {
        double wm = std::ceil(in->minWeight * kWeightScale);
        if (!(wm > 0)) wm = 0;
        if (wm > 4294967295.0) wm = 4294967295.0;
        kp.w_min = (uint32_t)wm;
    }
    kp.sx = (float)in->startPosition.x;
    kp.sy = (float)in->startPosition.y;
    kp.sz = (float)(in->startPosition.z + 1.0e-8);
    kp.dx = (float)in->startDirection.x;
    kp.dy = (float)in->startDirection.y;
    kp.dz = (float)in->startDirection.z;
    kp.beam_radius = (float)opt.beam_radius;
    kp.chance = (float)opt.roulette_chance;
    kp.inv_chance = (float)(1.0 / opt.roulette_chance);
    kp.flags = opt.flags;
    kp.max_steps = opt.max_steps_per_photon;
    kp.chunk = opt.photons_per_chunk;

    // ---- shared-memory staging plan ----
    const size_t smem_cap = 48 * 1024;  // per block, leaves room for several blocks per SM
    int smem_next = (int)std::min<size_t>((size_t)ns * MAX_LAYERS, 4096);
    int smem_tris = geom.n_tris <= 256 ? geom.n_tris : 0;
    int smem_nodes = 0;
    if (opt.smem_nodes >= 0) {
        size_t base = smem_layout(nd, 0, smem_tris, smem_next, 0);
        if (base < smem_cap) smem_nodes = (int)std::min<size_t>((smem_cap - base) / 32, (size_t)geom.n_nodes);
        if (opt.smem_nodes > 0) smem_nodes = std::min(smem_nodes, opt.smem_nodes);
    }
    kp.smem_nodes = smem_nodes;
    kp.smem_tris = smem_tris;
    kp.smem_next = smem_next;
    kp.n_nodes = geom.n_nodes;
    kp.n_tris = geom.n_tris;
    // the occupied z-slabs and the xy grid read only the geometry: built side by side
    int n_zocc = 0;
    parallel_parts(2, [&](unsigned t) {
        if (t == 1) n_zocc = occupied_z_slabs(geom, kp.zocc_lo, kp.zocc_hi);
        else build_xy_grid(geom, &img->grid, opt.grid_cell_tris > 0 ? opt.grid_cell_tris : 12);
    });
    kp.n_zocc = n_zocc;
    kp.grid_x0 = img->grid.x0;
    kp.grid_y0 = img->grid.y0;
    kp.grid_icx = img->grid.icx;
    kp.grid_icy = img->grid.icy;
    kp.grid_nx = img->grid.nx;
    kp.grid_ny = img->grid.ny;
    kp.n_big = (int)(img->grid.big.size() / 4);
    kp.coop_query = (opt.flags & XMC_LANE_QUERIES) ? 0 : 1;
    kp.query_batch = opt.query_batch > 0 ? std::min(32, (int)opt.query_batch) : 12;
    const int block = opt.block_size > 0 ? opt.block_size : 512;
    img->smem_bytes = smem_layout(nd, smem_nodes, smem_tris, smem_next, kp.coop_query ? block / 32 : 0);
    // ---- biasing (mcml_kernel.cpp:325-440) ----
    kp.use_bias = in->useBiasing ? 1 : 0;
    for (int l = 0; l < MAX_LAYERS; ++l) kp.layer_wtab[l] = -1;
    if (kp.use_bias) {
        kp.bias_eps = (float)in->attractiveFactor;
        kp.bias_ox = (float)in->startPosition.x;
        kp.bias_oy = (float)in->startPosition.y;
        kp.bias_oz = (float)in->startPosition.z;
        kp.bias_rx = (float)(in->targetPoint.x - in->startPosition.x);
        kp.bias_ry = (float)(in->targetPoint.y - in->startPosition.y);
        kp.bias_rz = (float)(in->targetPoint.z - in->startPosition.z);
        if (in->weightTable && in->numberOfWeightTables > 0) {
            // the caller's tables (the reference's launcher computes them before LaunchOMP)
            const int ne = in->weightTable[0].numberOfElements;
            std::vector<double> gs, tab;
            for (int k = 0; k < in->numberOfWeightTables; ++k) {
                const WeightIntegralTable& T = in->weightTable[k];
                if (T.numberOfElements != ne || ne < 2 || !T.elements)
                    return fail(XMC_ERR_INVALID_INPUT, "weight tables must share one element count >= 2");
                gs.push_back(T.anisotropy);
                tab.insert(tab.end(), T.elements, T.elements + ne);
            }
            st = set_weight_tables(in, gs, tab, ne, img);
            if (st) return st;
        } else {
            img->need_wtab = true;
        }
    }
    return XMC_OK;
}

// Layer -> table (GetWeightTableIndex, mcml_kernel.cpp:430-440: the last table whose anisotropy
// equals the layer's) and the FP32 copy the kernel reads.
int set_weight_tables(const InputInfo* in, const std::vector<double>& gs, const std::vector<double>& tables, int n_elem,
                      HostImage* img) {
    KParams& kp = img->kp;
    for (int l = 0; l < MAX_LAYERS; ++l) kp.layer_wtab[l] = -1;
    for (int l = 0; l < in->numberOfLayers; ++l) {
        const LayerInfo& L = in->layerInfo[l];
        int found = -1;
        for (size_t k = 0; k < gs.size(); ++k)
            if (gs[k] == L.anisotropy) found = (int)k;
        const bool tissue = !(L.absorptionCoefficient == 0.0 && L.scatteringCoefficient == 0.0);
        if (found < 0 && tissue && l > 0)
            return fail(XMC_ERR_INVALID_INPUT, "no weight table for the anisotropy of layer " + std::to_string(l));
        if (found > 127) return fail(XMC_ERR_RANGE, "too many weight tables");
        kp.layer_wtab[l] = (int8_t)found;
    }
    img->wtab.resize(tables.size());
    for (size_t i = 0; i < tables.size(); ++i) img->wtab[i] = (float)tables[i];
    kp.wtab_n = n_elem;
    img->need_wtab = false;
    return XMC_OK;
}

void fill_ledger(const unsigned long long* L, uint32_t w0_fx, uint64_t n, xmc_ledger* led) {
    std::memset(led, 0, sizeof(*led));
    led->photons_launched = L[L_LAUNCHED];
    led->photons_terminated = L[L_TERMINATED];
    led->steps = L[L_STEPS];
    led->n_escaped_top = L[L_N_TOP];
    led->n_escaped_bottom = L[L_N_BOTTOM];
    led->n_area = L[L_N_AREA];
    led->n_cut = L[L_N_CUT];
    led->n_roulette = L[L_N_ROULETTE];
    led->n_glass = L[L_N_GLASS];
    led->n_budget = L[L_N_BUDGET];
    led->n_invalid = L[L_N_INVALID];
    led->n_detected = L[L_N_DETECTED];
    led->n_fp64_retests = L[L_N_RETEST];
    led->n_node_visits = L[L_N_NODES];
    led->n_triangle_tests = L[L_N_TRIS];
    led->n_plane_crossings = L[L_N_CROSSINGS];
    led->specular_fx = (unsigned long long)(kWeightOne - w0_fx) * L[L_LAUNCHED];
    led->absorbed_fx = L[L_ABSORBED];
    led->absorbed_outside_fx = L[L_ABSORBED_OUT];
    led->escaped_top_fx = L[L_TOP];
    led->escaped_bottom_fx = L[L_BOTTOM];
    led->lost_area_fx = L[L_AREA];
    led->lost_cut_fx = L[L_CUT];
    led->lost_glass_fx = L[L_GLASS];
    led->lost_budget_fx = L[L_BUDGET];
    led->lost_invalid_fx = L[L_INVALID];
    led->roulette_killed_fx = L[L_RKILLED];
    led->roulette_gained_fx = L[L_RGAINED];
    const double np = n > 0 ? (double)n : 1.0;
    const double s = 1.0 / kWeightScale / np;
    led->specular = (double)led->specular_fx * s;
    led->absorbed = (double)led->absorbed_fx * s;
    led->absorbed_outside = (double)led->absorbed_outside_fx * s;
    led->escaped_top = (double)led->escaped_top_fx * s;
    led->escaped_bottom = (double)led->escaped_bottom_fx * s;
    led->lost_area = (double)led->lost_area_fx * s;
    led->lost_cut = (double)led->lost_cut_fx * s;
    led->lost_glass = (double)led->lost_glass_fx * s;
    led->lost_budget = (double)led->lost_budget_fx * s;
    led->lost_invalid = (double)led->lost_invalid_fx * s;
    led->roulette_killed = (double)led->roulette_killed_fx * s;
    led->roulette_gained = (double)led->roulette_gained_fx * s;
    led->absorbed_target_fx = L[L_ABSORBED_TGT];
    led->absorbed_target = (double)led->absorbed_target_fx * s;
    led->bias_gained_fx = L[L_BIAS_GAINED];
    led->bias_lost_fx = L[L_BIAS_LOST];
    led->bias_gained = (double)led->bias_gained_fx * s;
    led->bias_lost = (double)led->bias_lost_fx * s;
}

// Host image of `in` with its weight tables (computed on the GPU when biasing needs them and the
// caller gave none).
static int full_image(const InputInfo* in, const xmc_options* opt_in, HostImage* img) {
    int st = prepare_image(in, opt_in, img);
    if (st) return st;
    if (img->need_wtab) {  // biasing without the caller's tables: compute them (weight_integral.cpp:34-65) on the GPU
        std::vector<double> gs, tables;
        int ne = 0;
        st = compute_weight_tables(in, img->opt.device, &gs, &tables, &ne);
        if (st) return st;
        st = set_weight_tables(in, gs, tables, ne, img);
        if (st) return st;
    }
    return XMC_OK;
}

static int create_from_image(const HostImage& img, Context** out);

static int create(const InputInfo* in, const xmc_options* opt_in, Context** out) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    *out = nullptr;
    HostImage img;
    int st = full_image(in, opt_in, &img);
    if (st) return st;
    return create_from_image(img, out);
}

// Device context (buffers, uploads, launch shape) from a host image.
static int create_from_image(const HostImage& img, Context** out) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    *out = nullptr;
    const xmc_options& opt = img.opt;
    const GeomImage& geom = img.geom;
    const std::vector<int8_t>& next = img.next;
    const std::vector<DevDetector>& dets = img.dets;

    Context* c = new (std::nothrow) Context();
    if (!c) return fail(XMC_ERR_DEVICE, "out of host memory");
    c->opt = opt;
    c->device = opt.device;
    c->kp = img.kp;
    c->rsp = img.rsp;
    c->w0_fx = img.w0_fx;
    c->grid_size = img.grid_size;
    c->n_dets = img.n_dets;
    c->n_time = img.n_time;
    c->smem_bytes = img.smem_bytes;
    KParams& kp = c->kp;
    const int nd = img.n_dets, T = img.n_time;
    auto bail = [&](int s) { free_context(c); return s; };
    {
        cudaError_t e = cudaSetDevice(c->device);
        if (e != cudaSuccess) return bail(fail(XMC_ERR_DEVICE, std::string("cudaSetDevice: ") + cudaGetErrorString(e)));
    }
#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return bail(fail(XMC_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_))); \
    } while (0)
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, c->device));
    c->num_sms = prop.multiProcessorCount;

    // ---- device buffers ----
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : c->ev) CK(cudaEventCreate(&e));
    auto up = [&](void** d, const void* h, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(d, bytes ? bytes : 16);
        if (e != cudaSuccess) return e;
        if (bytes) e = cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, c->stream);
        return e;
    };
    c->h2d_bytes = sizeof(float4) * (geom.nodes.size() + geom.tris.size()) + next.size() + sizeof(DevDetector) * dets.size();
    CK(up(&c->d_nodes, geom.nodes.data(), sizeof(float4) * geom.nodes.size()));
    CK(up(&c->d_tris, geom.tris.data(), sizeof(float4) * geom.tris.size()));
    CK(up(&c->d_next, next.data(), next.size()));
    CK(up(&c->d_dets, dets.data(), sizeof(DevDetector) * dets.size()));
    CK(up(&c->d_cells, img.grid.cells.data(), sizeof(uint2) * img.grid.cells.size()));
    CK(up(&c->d_cell_z, img.grid.cell_z.data(), sizeof(float4) * img.grid.cell_z.size()));
    CK(up(&c->d_cell_entries, img.grid.entries.data(), sizeof(float4) * img.grid.entries.size()));
    CK(up(&c->d_big, img.grid.big.data(), sizeof(float4) * img.grid.big.size()));
    CK(up(&c->d_cell_runs, img.grid.cell_runs.data(), sizeof(uint32_t) * img.grid.cell_runs.size()));
    if (img.kp.use_bias) {
        CK(up(&c->d_wtab, img.wtab.data(), sizeof(float) * img.wtab.size()));
        c->h2d_bytes += sizeof(float) * img.wtab.size();
    }
    c->h2d_bytes += sizeof(uint2) * img.grid.cells.size() + sizeof(uint32_t) * img.grid.cell_runs.size() +
                    sizeof(float4) * (img.grid.cell_z.size() + img.grid.entries.size() + img.grid.big.size());
    const size_t absorb_b = sizeof(unsigned long long) * (size_t)c->grid_size;
    const size_t det_b = sizeof(unsigned long long) * 4 * (size_t)std::max(1, nd);
    const size_t tbin_b = sizeof(unsigned long long) * 4 * (size_t)std::max(1, nd) * T;
    const size_t led_b = sizeof(unsigned long long) * kLedgerSlots;
    CK(cudaMalloc(&c->d_absorb, absorb_b));
    CK(cudaMalloc(&c->d_det, det_b));
    CK(cudaMalloc(&c->d_tbin, tbin_b));
    CK(cudaMalloc(&c->d_ledger, led_b));
    CK(cudaMalloc(&c->d_counter, 16));
    CK(cudaMalloc(&c->d_status, 16));
    if (opt.flags & XMC_SCATTERING_MAP) CK(cudaMalloc(&c->d_scatter, absorb_b));
    if (opt.flags & XMC_DETECTOR_TRAJ) {
        CK(cudaMalloc(&c->d_traj, absorb_b * (size_t)std::max(1, nd)));
        CK(cudaMalloc(&c->d_replay_count, 16));
        CK(cudaMalloc(&c->d_replay_ledger, led_b));
    }
    CK(cudaHostAlloc((void**)&c->h_cancel, 16, cudaHostAllocDefault));
    *c->h_cancel = 1;
    CK(cudaMalloc(&c->d_cancel, 16));
    CK(cudaStreamCreateWithFlags(&c->cancel_stream, cudaStreamNonBlocking));
    CK(cudaHostAlloc((void**)&c->h_absorb, absorb_b, cudaHostAllocDefault));
    CK(cudaHostAlloc((void**)&c->h_det, det_b, cudaHostAllocDefault));
    CK(cudaHostAlloc((void**)&c->h_tbin, tbin_b, cudaHostAllocDefault));
    CK(cudaHostAlloc((void**)&c->h_ledger, 2 * led_b, cudaHostAllocDefault));  // run + replay ledgers
    CK(cudaHostAlloc((void**)&c->h_status, 16, cudaHostAllocDefault));
    kp.nodes = (const float4*)c->d_nodes;
    kp.tris = (const float4*)c->d_tris;
    kp.next_layer = (const int8_t*)c->d_next;
    kp.dets = (const DevDetector*)c->d_dets;
    kp.cells = (const uint2*)c->d_cells;
    kp.cell_z = (const float4*)c->d_cell_z;
    kp.cell_entries = (const float4*)c->d_cell_entries;
    kp.big = (const float4*)c->d_big;
    kp.cell_runs = (const uint32_t*)c->d_cell_runs;
    kp.wtab = (const float*)c->d_wtab;
    kp.absorb = (unsigned long long*)c->d_absorb;
    kp.det = (unsigned long long*)c->d_det;
    kp.tbin = (unsigned long long*)c->d_tbin;
    kp.ledger = (unsigned long long*)c->d_ledger;
    kp.counter = (unsigned long long*)c->d_counter;
    kp.cancel = (const volatile int*)c->d_cancel;
    kp.status = (int*)c->d_status;
    kp.scatter = (unsigned long long*)c->d_scatter;
    kp.traj = (unsigned long long*)c->d_traj;
    kp.replay_count = (unsigned long long*)c->d_replay_count;

    // ---- launch shape ----
    c->block = opt.block_size > 0 ? opt.block_size : 512;
    if (c->block % 32 != 0 || c->block > 1024) return bail(fail(XMC_ERR_INVALID_INPUT, "block_size must be a multiple of 32 <= 1024"));
    int occ = 0;
    CK(transport_occupancy(c->block, c->smem_bytes, &occ, c->kp.use_bias != 0));
    if (occ <= 0) return bail(fail(XMC_ERR_DEVICE, "transport kernel cannot be resident with this block size / shared memory"));
    c->blocks_per_sm = opt.blocks_per_sm > 0 ? std::min(opt.blocks_per_sm, occ) : occ;
    c->grid = c->num_sms * c->blocks_per_sm;
    if ((opt.flags & XMC_DETECTOR_TRAJ) && opt.trajectory_log >= 0) {
        // crossing log: one row per resident thread, reused photon after photon
        // 4,096 entries: on the height field no detected photon overflows it (1,024 left 0.2 % of them
        // to the replay pass, whose longest walk added ~30 ms to a 1e7-photon run)
        const unsigned cap = opt.trajectory_log > 0 ? (unsigned)opt.trajectory_log : 4096u;
        CK(cudaMalloc(&c->d_xlog, sizeof(unsigned) * (size_t)c->grid * c->block * cap));
        kp.xlog = (unsigned*)c->d_xlog;
        kp.xlog_cap = cap;
    }
    CK(cudaStreamSynchronize(c->stream));
#undef CK
    *out = c;
    return XMC_OK;
}

static int run(Context* c, uint64_t seed, uint64_t first, uint64_t n, OutputInfo* out, xmc_ledger* led) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    XMC_CUDA(cudaSetDevice(c->device));
    KParams& kp = c->kp;
    kp.key0 = (uint32_t)seed;
    kp.key1 = (uint32_t)(seed >> 32);
    kp.first_id = first;
    kp.n_photons = n;
    const size_t absorb_b = sizeof(unsigned long long) * (size_t)c->grid_size;
    const size_t det_b = sizeof(unsigned long long) * 4 * (size_t)std::max(1, c->n_dets);
    const size_t tbin_b = det_b * c->n_time;
    const size_t led_b = sizeof(unsigned long long) * kLedgerSlots;
    const bool traj = (c->opt.flags & XMC_DETECTOR_TRAJ) != 0;
    const bool scat = (c->opt.flags & XMC_SCATTERING_MAP) != 0;
    if (out) {
        if (out->gridSize != c->grid_size) return fail(XMC_ERR_INVALID_INPUT, "output gridSize does not match the input Area");
        if (out->numberOfDetectors != c->n_dets) return fail(XMC_ERR_INVALID_INPUT, "output numberOfDetectors does not match the input");
    }
    const bool want_scat = out && scat && out->scattering;
    const bool want_traj = out && traj && c->n_dets > 0;
    if (want_scat) {  // pinned staging of the scattering map, kept by the context
        const size_t need = absorb_b;
        if (c->h_maps_bytes < need) {
            if (c->h_maps) cudaFreeHost(c->h_maps);
            c->h_maps = nullptr;
            c->h_maps_bytes = 0;
            XMC_CUDA(cudaHostAlloc((void**)&c->h_maps, need, cudaHostAllocDefault));
            c->h_maps_bytes = need;
        }
    }
    XMC_CUDA(cudaEventRecord(c->ev[0], c->stream));
    XMC_CUDA(cudaMemsetAsync(c->d_absorb, 0, absorb_b, c->stream));
    XMC_CUDA(cudaMemsetAsync(c->d_det, 0, det_b, c->stream));
    XMC_CUDA(cudaMemsetAsync(c->d_tbin, 0, tbin_b, c->stream));
    XMC_CUDA(cudaMemsetAsync(c->d_ledger, 0, led_b, c->stream));
    XMC_CUDA(cudaMemsetAsync(c->d_counter, 0, 16, c->stream));
    XMC_CUDA(cudaMemsetAsync(c->d_status, 0, 16, c->stream));
    XMC_CUDA(cudaMemsetAsync(c->d_cancel, 0, 16, c->stream));
    if (scat) XMC_CUDA(cudaMemsetAsync(c->d_scatter, 0, absorb_b, c->stream));
    if (traj) {
        XMC_CUDA(cudaMemsetAsync(c->d_traj, 0, absorb_b * (size_t)std::max(1, c->n_dets), c->stream));
        XMC_CUDA(cudaMemsetAsync(c->d_replay_ledger, 0, led_b, c->stream));
    }
    XMC_CUDA(cudaEventRecord(c->ev[1], c->stream));
    if (n > 0 && !traj) XMC_CUDA(enqueue_transport(c));
    if (n > 0 && traj) {
        // Detector trajectory maps: the run pass logs each photon's z-plane crossings per thread
        // (as the reference's PhotonTrajectory, mcml_kernel_types.h:118-124) and counts the log of
        // a detected photon in its detector's map. A detected photon whose log overflowed is listed
        // as (index, detector); the replay pass walks exactly those photons again (same
        // counter-RNG draws, same code) and counts their crossings in that detector's map.
        c->last_replayed = 0;
        const uint64_t portion_max = 1ull << 26;
        const uint64_t cap = std::min<uint64_t>(n, portion_max);
        if (c->replay_cap < cap) {
            if (c->d_replay) cudaFree(c->d_replay);
            c->d_replay = nullptr;
            c->replay_cap = 0;
            XMC_CUDA(cudaMalloc(&c->d_replay, sizeof(unsigned long long) * cap));
            c->replay_cap = cap;
        }
        for (uint64_t done = 0; done < n; done += portion_max) {
            const uint64_t portion = std::min(portion_max, n - done);
            kp.mode = 0;
            kp.first_id = first + done;
            kp.n_photons = portion;
            kp.replay_list = (unsigned long long*)c->d_replay;
            kp.replay_cap = c->replay_cap;
            kp.ledger = (unsigned long long*)c->d_ledger;
            XMC_CUDA(cudaMemsetAsync(c->d_counter, 0, 16, c->stream));
            XMC_CUDA(cudaMemsetAsync(c->d_replay_count, 0, 16, c->stream));
            XMC_CUDA(enqueue_transport(c));
            unsigned long long listed = 0;
            XMC_CUDA(cudaMemcpyAsync(&listed, c->d_replay_count, sizeof(listed), cudaMemcpyDeviceToHost, c->stream));
            XMC_CUDA(cudaStreamSynchronize(c->stream));
            c->last_replayed += listed;
            kp.mode = 1;
            kp.n_photons = std::min<unsigned long long>(listed, c->replay_cap);
            kp.ledger = (unsigned long long*)c->d_replay_ledger;
            XMC_CUDA(cudaMemsetAsync(c->d_counter, 0, 16, c->stream));
            if (kp.n_photons) XMC_CUDA(enqueue_transport(c));
            kp.mode = 0;
            kp.ledger = (unsigned long long*)c->d_ledger;
        }
        kp.first_id = first;
        kp.n_photons = n;
    }
    XMC_CUDA(cudaEventRecord(c->ev[2], c->stream));
    // Read-back: every copy is enqueued and waited for before anything is added into the caller's
    // OutputInfo, so a failed copy returns with the output unchanged.
    if (out) XMC_CUDA(cudaMemcpyAsync(c->h_absorb, c->d_absorb, absorb_b, cudaMemcpyDeviceToHost, c->stream));
    XMC_CUDA(cudaMemcpyAsync(c->h_det, c->d_det, det_b, cudaMemcpyDeviceToHost, c->stream));
    if (out) XMC_CUDA(cudaMemcpyAsync(c->h_tbin, c->d_tbin, tbin_b, cudaMemcpyDeviceToHost, c->stream));
    XMC_CUDA(cudaMemcpyAsync(c->h_ledger, c->d_ledger, led_b, cudaMemcpyDeviceToHost, c->stream));
    XMC_CUDA(cudaMemcpyAsync(c->h_status, c->d_status, 16, cudaMemcpyDeviceToHost, c->stream));
    if (traj)
        XMC_CUDA(cudaMemcpyAsync(c->h_ledger + kLedgerSlots, c->d_replay_ledger, led_b, cudaMemcpyDeviceToHost, c->stream));
    XMC_CUDA(cudaEventRecord(c->ev[3], c->stream));
    // maps: the scattering map through its pinned staging; the trajectory maps as the list of their
    // non-zero cells (count pass and scan, the list's length to the host, write pass, copy), or
    // dense when the list (12 bytes per cell) would be larger than the maps (8 bytes per cell)
    unsigned long long* hs = c->h_maps;
    const size_t G = (size_t)c->grid_size;
    if (want_scat) XMC_CUDA(cudaMemcpyAsync(hs, c->d_scatter, absorb_b, cudaMemcpyDeviceToHost, c->stream));
    size_t nz_total = 0;
    bool traj_sparse = true;
    std::vector<size_t> map_start;
    if (want_traj) {
        const size_t D = (size_t)c->n_dets;
        const size_t nb = (size_t)sparse_blocks_per_map(G) * D;
        if (!c->d_nz_counts) {
            XMC_CUDA(cudaMalloc(&c->d_nz_counts, sizeof(unsigned long long) * nb));
            XMC_CUDA(cudaMalloc(&c->d_nz_offsets, sizeof(unsigned long long) * nb));
            XMC_CUDA(cudaHostAlloc((void**)&c->h_nz_offsets, sizeof(unsigned long long) * (nb + 1), cudaHostAllocDefault));
        }
        XMC_CUDA(sparse_maps_count((const unsigned long long*)c->d_traj, G, (int)D, c->d_nz_counts,
                                   c->d_nz_offsets, &c->d_nz_tmp, &c->nz_tmp_bytes, c->stream));
        XMC_CUDA(cudaMemcpyAsync(c->h_nz_offsets, c->d_nz_offsets, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost,
                                 c->stream));
        XMC_CUDA(cudaMemcpyAsync(c->h_nz_offsets + nb, c->d_nz_counts + nb - 1, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, c->stream));
        XMC_CUDA(cudaStreamSynchronize(c->stream));
        nz_total = (size_t)(c->h_nz_offsets[nb - 1] + c->h_nz_offsets[nb]);
        const size_t bpm = nb / D;
        map_start.resize(D + 1);
        for (size_t d = 0; d < D; ++d) map_start[d] = (size_t)c->h_nz_offsets[d * bpm];
        map_start[D] = nz_total;
        const size_t dense_b = absorb_b * D;
        traj_sparse = (sizeof(unsigned) + sizeof(unsigned long long)) * nz_total < dense_b;
        if (!traj_sparse) {
            if (c->h_traj_bytes < dense_b) {
                if (c->h_traj) cudaFreeHost(c->h_traj);
                c->h_traj = nullptr;
                c->h_traj_bytes = 0;
                XMC_CUDA(cudaHostAlloc((void**)&c->h_traj, dense_b, cudaHostAllocDefault));
                c->h_traj_bytes = dense_b;
            }
            XMC_CUDA(cudaMemcpyAsync(c->h_traj, c->d_traj, dense_b, cudaMemcpyDeviceToHost, c->stream));
        }
        if (traj_sparse && nz_total > c->nz_cap) {
            const size_t cap = nz_total + nz_total / 4 + 1024;
            if (c->d_nz_idx) cudaFree(c->d_nz_idx);
            if (c->d_nz_val) cudaFree(c->d_nz_val);
            c->d_nz_idx = nullptr;
            c->d_nz_val = nullptr;
            c->nz_cap = 0;
            XMC_CUDA(cudaMalloc(&c->d_nz_idx, sizeof(unsigned) * cap));
            XMC_CUDA(cudaMalloc(&c->d_nz_val, sizeof(unsigned long long) * cap));
            c->nz_cap = cap;
        }
        if (traj_sparse && nz_total > c->h_nz_cap) {
            const size_t cap = c->nz_cap;
            if (c->h_nz_idx) cudaFreeHost(c->h_nz_idx);
            if (c->h_nz_val) cudaFreeHost(c->h_nz_val);
            c->h_nz_idx = nullptr;
            c->h_nz_val = nullptr;
            c->h_nz_cap = 0;
            XMC_CUDA(cudaHostAlloc((void**)&c->h_nz_idx, sizeof(unsigned) * cap, cudaHostAllocDefault));
            XMC_CUDA(cudaHostAlloc((void**)&c->h_nz_val, sizeof(unsigned long long) * cap, cudaHostAllocDefault));
            c->h_nz_cap = cap;
        }
        if (traj_sparse)
            XMC_CUDA(sparse_maps_write((const unsigned long long*)c->d_traj, G, (int)D, c->d_nz_offsets, c->d_nz_idx,
                                       c->d_nz_val, c->stream));
        if (traj_sparse && nz_total) {
            XMC_CUDA(cudaMemcpyAsync(c->h_nz_idx, c->d_nz_idx, sizeof(unsigned) * nz_total, cudaMemcpyDeviceToHost,
                                     c->stream));
            XMC_CUDA(cudaMemcpyAsync(c->h_nz_val, c->d_nz_val, sizeof(unsigned long long) * nz_total,
                                     cudaMemcpyDeviceToHost, c->stream));
        }
    }
    XMC_CUDA(cudaStreamSynchronize(c->stream));
    float k_ms = 0, t_ms = 0;
    XMC_CUDA(cudaEventElapsedTime(&k_ms, c->ev[1], c->ev[2]));
    XMC_CUDA(cudaEventElapsedTime(&t_ms, c->ev[0], c->ev[3]));
    c->last_kernel_ms = k_ms;
    c->last_total_ms = t_ms;
    c->last_n = n;

    const unsigned long long* L = c->h_ledger;
    const double inv_scale = 1.0 / kWeightScale;
    if (out) {
        out->specularReflectance = c->rsp;
        for (int d = 0; d < c->n_dets; ++d) {
            DetectorInfo& D = out->detectorInfo[d];
            const unsigned long long* t = c->h_det + 4 * (size_t)d;
            D.weight += (double)t[0] * inv_scale;
            D.numberOfPhotons += t[1];
            D.targetWeight += (double)t[2] * inv_scale;
            if (D.timeScale && D.timeScaleSize == c->n_time) {
                for (int j = 0; j < c->n_time; ++j) {
                    const unsigned long long* b = c->h_tbin + 4 * ((size_t)d * c->n_time + j);
                    D.timeScale[j].weight += (double)b[0] * inv_scale;
                    D.timeScale[j].numberOfPhotons += b[1];
                    D.timeScale[j].targetWeight += (double)b[2] * inv_scale;
                }
            }
        }
        // voxel arrays on up to 16 host threads, each owning a slice of the grid: absorption and
        // scattering (FP64 from fixed point); then the trajectory maps' non-zero cells, each thread a
        // slice of the list (a cell appears once per map, so the slices touch disjoint cells)
        const unsigned hw = host_threads_for(G);
        const size_t per = (G + hw - 1) / hw;
        parallel_parts(hw, [&](unsigned t) {
            const size_t a = std::min(G, t * per), b = std::min(G, a + per);
            if (out->absorption)
                for (size_t i = a; i < b; ++i) out->absorption[i] += (double)c->h_absorb[i] * inv_scale;
            if (want_scat)
                for (size_t i = a; i < b; ++i) out->scattering[i] += (double)hs[i] * inv_scale;
        });
        if (want_traj && !traj_sparse) {
            // dense copy: each thread a slice of the grid in every map, non-zero cells only
            const unsigned hd = host_threads_for(G * (size_t)c->n_dets);
            const size_t pd = (G + hd - 1) / hd;
            parallel_parts(hd, [&](unsigned t) {
                const size_t a = std::min(G, t * pd), b = std::min(G, a + pd);
                for (int d = 0; d < c->n_dets; ++d) {
                    DetectorInfo& D = out->detectorInfo[d];
                    if (!D.trajectory || D.trajectorySize != c->grid_size) continue;
                    const unsigned long long* src = c->h_traj + (size_t)d * G;
                    for (size_t i = a; i < b; ++i)
                        if (src[i]) D.trajectory[i] += src[i];
                }
            });
        }
        if (want_traj && traj_sparse && nz_total) {
            const unsigned hz = host_threads_for(nz_total);
            const size_t pz = (nz_total + hz - 1) / hz;
            parallel_parts(hz, [&](unsigned t) {
                const size_t a = std::min(nz_total, t * pz), b = std::min(nz_total, a + pz);
                if (a >= b) return;
                size_t d = (size_t)(std::upper_bound(map_start.begin(), map_start.end(), a) - map_start.begin()) - 1;
                for (size_t e = a; e < b; ++e) {
                    while (e >= map_start[d + 1]) ++d;
                    DetectorInfo& D = out->detectorInfo[d];
                    if (D.trajectory && D.trajectorySize == c->grid_size) D.trajectory[c->h_nz_idx[e]] += c->h_nz_val[e];
                }
            });
        }
    }
    if (led) {
        fill_ledger(L, c->w0_fx, n, led);
        led->kernel_ms = k_ms;
        led->total_ms = t_ms;
        led->h2d_bytes = c->h2d_bytes + sizeof(KParams);
        // every device-to-host copy of this call: tallies, ledgers and status, the scattering map, and
        // the trajectory maps (block offsets, then the (cell, count) pairs or the dense maps)
        size_t maps_b = want_scat ? absorb_b : 0;
        if (want_traj)
            maps_b += sizeof(unsigned long long) * ((size_t)c->n_dets * sparse_blocks_per_map(G) + 1) +
                      (traj_sparse ? (sizeof(unsigned) + sizeof(unsigned long long)) * nz_total
                                   : absorb_b * (size_t)c->n_dets);
        led->d2h_bytes = (out ? absorb_b + tbin_b : 0) + det_b + led_b + 16 + (traj ? led_b : 0) + maps_b;
        led->n_replay_mismatch = traj ? c->h_ledger[kLedgerSlots + L_N_REPLAY_MISMATCH] : 0;
        led->n_trajectory_replayed = traj ? c->last_replayed : 0;
    }
    if (c->h_status[0] & 2) return fail(XMC_ERR_CANCELLED, "run cancelled");
    if (c->h_status[0] & 1) return fail(XMC_ERR_BUDGET, "a photon reached the step budget and was terminated");
    return XMC_OK;
}

}  // namespace xmc

using namespace xmc;

extern "C" {

int xmc_version(void) { return 10000 * 0 + 100 * 1 + 0; }

const char* xmc_last_error(void) { return g_last_error.c_str(); }

void xmc_default_options(xmc_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(xmc_options);
    o->roulette_chance = 0.1;
    o->max_steps_per_photon = 10000000ull;
    o->photons_per_chunk = 32;
}

int xmc_create(const InputInfo* input, const xmc_options* opt, xmc_context** out_ctx) {
    if (!out_ctx) return fail(XMC_ERR_INVALID_INPUT, "out_ctx is NULL");
    set_error("");
    Context* c = nullptr;
    int st = create(input, opt, &c);
    *out_ctx = reinterpret_cast<xmc_context*>(c);
    return st;
}

int xmc_run(xmc_context* ctx, uint64_t seed, uint64_t first_photon_id, uint64_t n_photons, OutputInfo* output,
            xmc_ledger* ledger) {
    if (!ctx) return fail(XMC_ERR_INVALID_INPUT, "context is NULL");
    return run(reinterpret_cast<Context*>(ctx), seed, first_photon_id, n_photons, output, ledger);
}

int xmc_read_tallies(xmc_context* ctx, uint64_t* absorption, uint64_t* det_weight, uint64_t* det_count,
                     uint64_t* det_target, uint64_t* det_weight2, uint64_t* time_weight, uint64_t* time_count,
                     uint64_t* time_target, uint64_t* time_weight2) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!ctx) return fail(XMC_ERR_INVALID_INPUT, "context is NULL");
    Context* c = reinterpret_cast<Context*>(ctx);
    XMC_CUDA(cudaSetDevice(c->device));
    const size_t absorb_b = sizeof(unsigned long long) * (size_t)c->grid_size;
    const size_t det_b = sizeof(unsigned long long) * 4 * (size_t)std::max(1, c->n_dets);
    const size_t tbin_b = det_b * c->n_time;
    XMC_CUDA(cudaMemcpyAsync(c->h_absorb, c->d_absorb, absorb_b, cudaMemcpyDeviceToHost, c->stream));
    XMC_CUDA(cudaMemcpyAsync(c->h_det, c->d_det, det_b, cudaMemcpyDeviceToHost, c->stream));
    XMC_CUDA(cudaMemcpyAsync(c->h_tbin, c->d_tbin, tbin_b, cudaMemcpyDeviceToHost, c->stream));
    XMC_CUDA(cudaStreamSynchronize(c->stream));
    if (absorption) std::memcpy(absorption, c->h_absorb, absorb_b);
    for (int d = 0; d < c->n_dets; ++d) {
        const unsigned long long* t = c->h_det + 4 * (size_t)d;
        if (det_weight) det_weight[d] = t[0];
        if (det_count) det_count[d] = t[1];
        if (det_target) det_target[d] = t[2];
        if (det_weight2) det_weight2[d] = t[3];
        for (int j = 0; j < c->n_time; ++j) {
            const unsigned long long* b = c->h_tbin + 4 * ((size_t)d * c->n_time + j);
            const size_t k = (size_t)d * c->n_time + j;
            if (time_weight) time_weight[k] = b[0];
            if (time_count) time_count[k] = b[1];
            if (time_target) time_target[k] = b[2];
            if (time_weight2) time_weight2[k] = b[3];
        }
    }
    return XMC_OK;
}

int xmc_read_maps(xmc_context* ctx, uint64_t* scattering, uint64_t* trajectory) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!ctx) return fail(XMC_ERR_INVALID_INPUT, "context is NULL");
    Context* c = reinterpret_cast<Context*>(ctx);
    XMC_CUDA(cudaSetDevice(c->device));
    const size_t b = sizeof(unsigned long long) * (size_t)c->grid_size;
    if (scattering) {
        if (!c->d_scatter) return fail(XMC_ERR_INVALID_INPUT, "context was created without XMC_SCATTERING_MAP");
        XMC_CUDA(cudaMemcpy(scattering, c->d_scatter, b, cudaMemcpyDeviceToHost));
    }
    if (trajectory) {
        if (!c->d_traj) return fail(XMC_ERR_INVALID_INPUT, "context was created without XMC_DETECTOR_TRAJ");
        XMC_CUDA(cudaMemcpy(trajectory, c->d_traj, b * (size_t)std::max(1, c->n_dets), cudaMemcpyDeviceToHost));
    }
    return XMC_OK;
}

int xmc_cancel(xmc_context* ctx) {
    if (!ctx) return fail(XMC_ERR_INVALID_INPUT, "context is NULL");
    Context* c = reinterpret_cast<Context*>(ctx);
    // the running kernel polls d_cancel; write it from a second stream so the copy does not queue
    // behind the kernel on the run stream
    XMC_CUDA(cudaMemcpyAsync(c->d_cancel, c->h_cancel, sizeof(int), cudaMemcpyHostToDevice, c->cancel_stream));
    XMC_CUDA(cudaStreamSynchronize(c->cancel_stream));
    return XMC_OK;
}

int xmc_destroy(xmc_context* ctx) {
    free_context(reinterpret_cast<Context*>(ctx));
    return XMC_OK;
}

// Kernel time of `n` photons under the options of `img` (a fresh context; the first, smaller run warms
// it up). Returns XMC_OK, or the status of a shape that cannot run (*ms untouched).
static int time_shape(const HostImage& img, uint64_t n, uint64_t seed, double* ms) {
    Context* c = nullptr;
    int st = create_from_image(img, &c);
    if (st) return st;
    xmc_ledger led;
    st = run(c, seed, 0, std::max<uint64_t>(n / 4, 1), nullptr, &led);
    if (!st || st == XMC_ERR_BUDGET) st = run(c, seed + 1, 0, n, nullptr, &led);
    free_context(c);
    if (st && st != XMC_ERR_BUDGET) return st;
    *ms = led.kernel_ms;
    return XMC_OK;
}

int xmc_autotune(const InputInfo* input, const xmc_options* base, uint64_t sample_photons, xmc_options* best,
                 double* best_ms) {
    if (!input || !best) return fail(XMC_ERR_INVALID_INPUT, "xmc_autotune: NULL argument");
    set_error("");
    DeviceGuard device_guard;
    const uint64_t n = sample_photons ? sample_photons : 1000000ull;
    const int densities[] = {2, 8, 16, 32};
    const int n_dens = (int)(sizeof(densities) / sizeof(densities[0]));
    const int blocks[] = {256, 512};
    const int chunks[] = {32, 64};
    const int batches[] = {1, 8, 12, 16};
    struct Cand {
        xmc_options opt;
        double ms;
    };
    std::vector<Cand> cands;
    std::vector<HostImage> images(n_dens);
    std::string last_err;
    for (int di = 0; di < n_dens; ++di) {
        // the xy grid's cell size is part of the device image: one image per density
        xmc_options o;
        xmc_default_options(&o);
        if (base && base->struct_size) std::memcpy(&o, base, std::min((size_t)base->struct_size, sizeof(o)));
        o.struct_size = sizeof(o);
        o.grid_cell_tris = densities[di];
        HostImage& img = images[di];
        int st = full_image(input, &o, &img);
        if (st) return st;
        for (int coop = 1; coop >= 0; --coop) {
            for (int b : blocks) {
                for (int ch : chunks) {
                    for (int qb : batches) {
                        if (!coop && qb > 1) continue;  // query batches apply to the cooperative scheme only
                        xmc_options c = img.opt;
                        c.block_size = b;
                        c.blocks_per_sm = 0;
                        c.photons_per_chunk = ch;
                        c.query_batch = qb;
                        c.flags = coop ? (c.flags & ~XMC_LANE_QUERIES) : (c.flags | XMC_LANE_QUERIES);
                        cands.push_back({c, INFINITY});
                    }
                }
            }
        }
    }
    // launch-shape fields only: the tally arithmetic stays the same
    auto shaped = [&](const xmc_options& c) {
        int di = 0;
        while (di + 1 < n_dens && densities[di] != c.grid_cell_tris) ++di;
        HostImage img = images[di];
        img.opt = c;
        img.kp.flags = c.flags;
        img.kp.chunk = c.photons_per_chunk;
        img.kp.coop_query = (c.flags & XMC_LANE_QUERIES) ? 0 : 1;
        img.kp.query_batch = c.query_batch;
        img.smem_bytes = smem_layout(img.n_dets, img.kp.smem_nodes, img.kp.smem_tris, img.kp.smem_next,
                                     img.kp.coop_query ? c.block_size / 32 : 0);
        return img;
    };
    for (Cand& c : cands) {
        if (time_shape(shaped(c.opt), n, 1, &c.ms)) {
            last_err = g_last_error;  // this shape cannot run here (shared memory, registers): skip it
            c.ms = INFINITY;
        }
    }
    // one timing each ranks them; the four fastest are timed twice more (other photons) and the best of
    // their three timings decides, so that one noisy sample does not pick the shape
    std::sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.ms < y.ms; });
    if (cands.empty() || !(cands[0].ms < INFINITY))
        return fail(XMC_ERR_DEVICE, "xmc_autotune: no launch shape could run: " + last_err);
    const size_t top = std::min<size_t>(4, cands.size());
    for (size_t k = 0; k < top && cands[k].ms < INFINITY; ++k) {
        for (uint64_t rep = 0; rep < 2; ++rep) {
            double ms = INFINITY;
            const int st = time_shape(shaped(cands[k].opt), n, 11 + 2 * rep, &ms);
            if (st) return st;
            cands[k].ms = std::min(cands[k].ms, ms);
        }
    }
    std::sort(cands.begin(), cands.begin() + top, [](const Cand& x, const Cand& y) { return x.ms < y.ms; });
    *best = cands[0].opt;
    if (best_ms) *best_ms = cands[0].ms;
    return XMC_OK;
}

}  // extern "C"

namespace {

// 64-bit fingerprint of everything a device image depends on (word-wise multiply-xorshift mix).
struct Fingerprint {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    void add(const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        if (!b) n = 0;
        size_t i = 0;
        for (; i + 8 <= n; i += 8) {
            uint64_t w;
            std::memcpy(&w, b + i, 8);
            mix(w);
        }
        uint64_t w = 0;
        std::memcpy(&w, b + i, n - i);
        mix(w ^ ((uint64_t)n << 56));
    }
    template <typename T> void val(const T& v) { add(&v, sizeof(v)); }
    void mix(uint64_t w) {
        h ^= w;
        h *= 0xff51afd7ed558ccdull;
        h ^= h >> 32;
    }
};

uint64_t input_fingerprint(const InputInfo* in, const xmc_options* opt) {
    Fingerprint f;
    f.val(in->numberOfLayers); f.val(in->numberOfSurfaces); f.val(in->numberOfCubeDetectors);
    f.val(in->numberOfRingDetectors); f.val(in->minWeight); f.val(in->timeStart); f.val(in->timeFinish);
    f.val(in->timeScaleSize); f.val(in->startPosition); f.val(in->startDirection); f.val(in->useBiasing);
    f.val(in->weightIntegralPrecision); f.val(in->weightTablePrecision); f.val(in->attractiveFactor);
    f.val(in->targetPoint); f.add(in->targetRangeLayers, sizeof(in->targetRangeLayers));
    if (in->area) f.val(*in->area);
    for (int l = 0; in->layerInfo && l < in->numberOfLayers; ++l) {
        const LayerInfo& L = in->layerInfo[l];
        f.val(L.refractiveIndex); f.val(L.absorptionCoefficient); f.val(L.scatteringCoefficient); f.val(L.anisotropy);
        f.val(L.numberOfSurfaces);
        f.add(L.surfaceId, sizeof(int) * (size_t)std::max(0, L.numberOfSurfaces));
    }
    for (int s = 0; in->surface && s < in->numberOfSurfaces; ++s) {
        const Surface& S = in->surface[s];
        f.val(S.numberOfVertices); f.val(S.numberOfTriangles);
        f.add(S.vertices, sizeof(double3) * (size_t)std::max(0, S.numberOfVertices));
        f.add(S.triangles, sizeof(int3) * (size_t)std::max(0, S.numberOfTriangles));
    }
    f.add(in->cubeDetector, sizeof(CubeDetector) * (size_t)std::max(0, in->numberOfCubeDetectors));
    f.add(in->ringDetector, sizeof(RingDetector) * (size_t)std::max(0, in->numberOfRingDetectors));
    f.val(in->numberOfWeightTables);
    for (int k = 0; in->weightTable && k < in->numberOfWeightTables; ++k) {
        const WeightIntegralTable& T = in->weightTable[k];
        f.val(T.anisotropy); f.val(T.numberOfElements);
        f.add(T.elements, sizeof(double) * (size_t)std::max(0, T.numberOfElements));
    }
    if (in->bvhTree) {
        const BVHTree& B = *in->bvhTree;
        f.val(B.numOfNodes); f.val(B.root); f.val(B.numOfTriangles);
        f.add(B.nodes, sizeof(BVHNode) * (size_t)std::max(0, B.numOfNodes));
        f.add(B.triangles, sizeof(Triangle) * (size_t)std::max(0, B.numOfTriangles));
    } else {
        f.val((uint64_t)0);
    }
    xmc_options o;
    xmc_default_options(&o);
    if (opt && opt->struct_size) std::memcpy(&o, opt, std::min((size_t)opt->struct_size, sizeof(o)));
    o.struct_size = sizeof(o);
    f.val(o);
    return f.h;
}

// Options xmc_launch_omp uses (xmc_launch_set_options; defaults until set).
std::mutex g_omp_opts_mutex;
xmc_options g_omp_opts{};
bool g_omp_opts_set = false;

// The device context of the last model run through xmc_launch, kept for the next call on the same
// model contents (the reference's launchers call LaunchOMP repeatedly on one InputInfo).
std::mutex g_launch_mutex;
xmc::Context* g_launch_ctx = nullptr;
uint64_t g_launch_fp = 0;

}  // namespace

extern "C" {

int xmc_launch(const InputInfo* input, OutputInfo* output, uint64_t seed, uint64_t first_photon_id,
               const xmc_options* opt, xmc_ledger* ledger) {
    if (!input) return fail(XMC_ERR_INVALID_INPUT, "input is NULL");
    std::lock_guard<std::mutex> lock(g_launch_mutex);
    const uint64_t fp = input_fingerprint(input, opt);
    if (!g_launch_ctx || fp != g_launch_fp) {
        if (g_launch_ctx) free_context(g_launch_ctx);
        g_launch_ctx = nullptr;
        xmc_context* c = nullptr;
        int st = xmc_create(input, opt, &c);
        if (st) return st;
        g_launch_ctx = reinterpret_cast<Context*>(c);
        g_launch_fp = fp;
    }
    int st = xmc_run(reinterpret_cast<xmc_context*>(g_launch_ctx), seed, first_photon_id, input->numberOfPhotons, output,
                     ledger);
    if (st && st != XMC_ERR_BUDGET && st != XMC_ERR_CANCELLED) {  // a failed run: do not keep its context
        std::string keep = g_last_error;
        free_context(g_launch_ctx);
        g_launch_ctx = nullptr;
        set_error(keep);
    }
    return st;
}

int xmc_launch_release(void) {
    std::lock_guard<std::mutex> lock(g_launch_mutex);
    if (g_launch_ctx) free_context(g_launch_ctx);
    g_launch_ctx = nullptr;
    return XMC_OK;
}

int xmc_launch_set_options(const xmc_options* opt) {
    std::lock_guard<std::mutex> lock(g_omp_opts_mutex);
    g_omp_opts_set = opt && opt->struct_size;
    xmc_default_options(&g_omp_opts);
    if (g_omp_opts_set) std::memcpy(&g_omp_opts, opt, std::min((size_t)opt->struct_size, sizeof(g_omp_opts)));
    g_omp_opts.struct_size = sizeof(g_omp_opts);
    return XMC_OK;
}

int xmc_launch_omp(InputInfo* input, OutputInfo* output, MCG59* rng, int numThreads) {
    (void)numThreads;
    if (!input || !output || !rng) {
        set_error("xmc_launch_omp: NULL argument");
        std::fprintf(stderr, "xmc_launch_omp: %s\n", xmc_last_error());
        return XMC_ERR_INVALID_INPUT;
    }
    xmc_options opt;
    {
        std::lock_guard<std::mutex> lock(g_omp_opts_mutex);
        if (g_omp_opts_set) opt = g_omp_opts;
        else xmc_default_options(&opt);
    }
    opt.flags |= XMC_SCATTERING_MAP | XMC_DETECTOR_TRAJ;  // every tally LaunchOMP fills
    int dev = 0;  // LaunchOMP has no device argument: the caller's current device
    if (cudaGetDevice(&dev) == cudaSuccess) opt.device = dev;
    int st = xmc_launch(input, output, rng[0].value, 0, &opt, nullptr);
    if (st && st != XMC_ERR_BUDGET) {
        std::fprintf(stderr, "xmc_launch_omp: %s\n", xmc_last_error());
        return st;
    }
    // advance the caller's generator by one MCG59 step (mcml_mcg59.cpp:34-38) so the next call
    // (the next backup portion) uses a fresh key
    rng[0].value = (rng[0].value * rng[0].offset) & 576460752303423487ULL;
    return st;
}

double xmc_specular_reflectance(const LayerInfo* layer) { return specular(layer); }

void xmc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

int xmc_device_philox(uint64_t seed, uint64_t photon_id, uint32_t n, uint32_t* out) {
    XMC_CUDA(device_philox((uint32_t)seed, (uint32_t)(seed >> 32), photon_id, n, out));
    return XMC_OK;
}

}  // extern "C"
