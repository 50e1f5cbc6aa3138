// Internal declarations shared by the host C++ files and the CUDA transport kernel.
#pragma once

#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

// CUDA's vector_types.h also defines double3 and int3; inside this library the reference's
// vertex and index types are named xmc_ref_double3 / xmc_ref_int3 (same layout, same union tags).
#define double3 xmc_ref_double3
#define int3 xmc_ref_int3
#include "../../include/xmcml_b200.h"
#undef double3
#undef int3

namespace xmc {

// Runs body(t) for t in [0, parts) on up to `parts` host threads, the calling thread included. When
// the system cannot start a thread (std::system_error), the parts that got no thread run on the
// calling thread, so no C++ exception crosses the C-ABI.
template <typename F>
inline void parallel_parts(unsigned parts, F body) {
    std::vector<std::thread> pool;
    unsigned started = 1;
    try {
        for (; started < parts; ++started) pool.emplace_back(body, started);
    } catch (...) {
    }
    body(0);
    for (unsigned t = started; t < parts; ++t) body(t);
    for (auto& th : pool) th.join();
}

// Fixed point of photon weights and tallies: weight 1.0 == 2^31.
constexpr double kWeightScale = 2147483648.0;
constexpr uint32_t kWeightOne = 0x80000000u;

// Geometric tolerances of the FP32 walk (mm). A step that ends within kStepExtend in front of a
// surface is taken to the surface; after a boundary interaction hits closer than kTminAfter are
// ignored and the triangle just hit is excluded from the next query. The reference's FP64 nudges
// of 1e-8 mm (mcml_kernel.cpp:13) are below FP32 resolution at mm scale and are replaced by these.
constexpr float kStepExtend = 2e-6f;
constexpr float kTminAfter = 2e-6f;
// Band around triangle edges inside which the FP32 ray-triangle test is redone in FP64: about
// kEdgeBandLength mm measured along the triangle, as a barycentric width clamped to
// [kEdgeBandMin, kEdgeBandMax] (FP32 barycentrics carry ~1e-7 relative error).
constexpr float kEdgeBandLength = 1e-5f;
constexpr float kEdgeBandMin = 1.0f / 262144.0f;
constexpr float kEdgeBandMax = 1.0f / 1024.0f;

// Per-layer constants of the walk (FP32).
struct DevLayer {
    float n;          // refractive index
    float mua, mus;   // mm^-1
    float g;          // anisotropy
    float inv_mut;    // 1 / (mua + mus), 0 for glass
    float absorb;     // mua / (mua + mus)
    float hg_a;       // 1 - g^2
    float hg_b;       // 1 + g^2
    float hg_c;       // 1 / (2 g)  (0 when g == 0)
    float hg_d;       // 1 - g
    float hg_e;       // 2 g
    int glass;        // 1 when mua == mus == 0
};

// Detector record: cube detectors first, then rings (the reference's GetDetectorId order).
struct DevDetector {
    float cx, cy, cz;     // centre
    float hx, hy, hz;     // cube: half lengths; ring: (small radius, big radius, unused)
    float cos_angle;      // cos(targetAngle) as computed by the reference, rounded to float
    uint32_t filter;      // bitmask of filterLayers
};

// Ledger slots of the device tally (uint64 each).
enum LedgerSlot {
    L_LAUNCHED = 0, L_TERMINATED, L_STEPS,
    L_N_TOP, L_N_BOTTOM, L_N_AREA, L_N_CUT, L_N_ROULETTE, L_N_GLASS, L_N_BUDGET, L_N_INVALID,
    L_N_DETECTED, L_N_RETEST, L_N_NODES, L_N_TRIS,
    L_ABSORBED, L_ABSORBED_OUT, L_TOP, L_BOTTOM, L_AREA, L_CUT, L_GLASS, L_BUDGET, L_INVALID,
    L_RKILLED, L_RGAINED, L_N_REPLAY_MISMATCH, L_ABSORBED_TGT, L_BIAS_GAINED, L_BIAS_LOST,
    L_N_CROSSINGS,
    L_COUNT
};
constexpr int kLedgerSlots = 32;  // padded

// xy cell grid over all triangles for short (bounded) ray queries: each cell lists the triangles
// whose xy bounding box overlaps it, with their z-range; a query whose xy footprint covers at most
// kGridMaxCells cells tests those lists, longer ones use the BVH.
constexpr int kGridMaxCells = 4;
// Triangles whose xy bounding box covers more than kBigTriangleCells cells (large planes) are kept
// out of the cells in a short list staged in shared memory (at most kMaxBigTriangles of them).
constexpr int kBigTriangleCells = 64;
constexpr int kMaxBigTriangles = 64;

// Shared-memory scratch of one warp for the warp-cooperative grid query: the rays of the lanes that
// query (origin + tmin, direction + tmax, segment z-range, excluded triangle, cell rectangle), the
// per-lane cell offsets, the cells that survive the z-cull with their entry offsets, and one packed
// (distance bits << 32 | triangle) minimum per lane.
constexpr int kWarpQueryCells = 32 * kGridMaxCells;
struct WarpQuery {
    float4 o[32];
    float4 d[32];
    float2 z[32];
    int excl[32];
    int ij0[32];                      // i0 | j0 << 16
    int w[32];                        // cells per row of the lane's rectangle
    int coff[33];                     // exclusive scan of the lanes' cell counts
    int eoff[kWarpQueryCells + 1];    // exclusive scan of the kept cells' entry counts
    unsigned long long best[32];
    uint2 cell[kWarpQueryCells];      // kept cells: first entry, entry count
    unsigned char owner[kWarpQueryCells];
};

// z-intervals occupied by triangles (merged, padded, sorted): a step whose z-range lies strictly
// inside a gap between them cannot cross any surface, so its ray query is skipped.
constexpr int kMaxZSlabs = 24;

// Everything the kernel reads, by value (kernel parameter space).
struct KParams {
    // geometry
    const float4* nodes;      // 2 float4 per node
    const float4* tris;       // 3 float4 per triangle
    const int8_t* next_layer; // [n_surf * MAX_LAYERS]: layer across surface s from layer l, -1 if none
    int n_nodes, n_tris, n_surf;
    int smem_nodes, smem_tris, smem_next;  // how many of each are staged in shared memory
    float zocc_lo[kMaxZSlabs], zocc_hi[kMaxZSlabs];
    int n_zocc;
    // xy cell grid (grid_nx == 0: none)
    const uint2* cells;               // [grid_nx * grid_ny]: {first entry, entry count}
    const float4* cell_z;             // [2 * grid_nx * grid_ny]: up to 4 merged z-intervals occupied in the cell
    const float4* cell_entries;       // {zmin, zmax, triangle index (bits), 0}, sorted by zmin within a cell
    const uint32_t* cell_runs;        // [grid_nx * grid_ny]: entries per z-interval of the cell (4 x 8 bits),
                                      // 0xffffffff when a count exceeds 255 (the cell is not split)
    const float4* big;                // [n_big * 4]: {zmin, zmax, triangle index (bits), 0}, then the 3 triangle float4s
    int n_big;
    float grid_x0, grid_y0, grid_icx, grid_icy;  // origin and 1 / cell size
    int grid_nx, grid_ny;
    int coop_query;           // 1: grid queries run warp-cooperatively (WarpQuery scratch per warp in
                              // shared memory); 0: each lane walks its own cells
    int query_batch;          // cooperative: a warp runs its query round once this many lanes wait (or
                              // every live lane waits)
    // layers
    DevLayer layer[MAX_LAYERS];
    int n_layers;
    uint32_t target_mask;     // targetRangeLayers as bitmask
    // Area
    float ax, ay, az;         // corner
    float asx, asy, asz;      // partitions / length
    int nx, ny, nz;
    int byte_sentinel;        // voxel (255,255,255) counts as outside (reference byte index semantics)
    // detectors and time bins
    const DevDetector* dets;
    int n_cubes, n_rings, n_dets;
    int rings_sorted;         // rings share one centre, are sorted and do not overlap: at most one
                              // ring contains a radius, found by binary search
    float t0, dt;             // time bins: [t0 + i dt, t0 + (i+1) dt), last bin open-ended
    int n_time;
    // launch
    float sx, sy, sz, dx, dy, dz;
    float beam_radius;
    uint32_t w0;              // start weight (fixed point)
    uint32_t w_min;           // minWeight (fixed point)
    float chance, inv_chance; // roulette
    uint32_t flags;
    uint32_t key0, key1;      // Philox key (seed)
    unsigned long long first_id, n_photons, max_steps;
    int chunk;
    // z-plane crossing tallies (UpdatePhotonTrajectory): planes at voxel centres
    float plane_dz;           // Area length.z / partitions.z
    float area_zend;          // corner.z + length.z
    int grid;                 // nx * ny * nz
    int mode;                 // 0: transport run, 1: trajectory replay of detected photons
    unsigned long long* scatter;        // [grid] scattering map (XMC_SCATTERING_MAP), weight fixed point
    unsigned long long* traj;           // [n_dets * grid] detector trajectory maps, counts
    unsigned* xlog;                     // run: [grid threads][xlog_cap] voxel of each z-plane crossing of the
    unsigned xlog_cap;                  //      thread's current photon (null / 0: no log, replay every photon)
    unsigned long long* replay_list;    // run: (index << 16 | detector) of detected photons whose log
                                        //      overflowed; replay: input
    unsigned long long* replay_count;   // run: number of entries written
    unsigned long long replay_cap;      // run: capacity of replay_list
    // tallies (device, fixed point)
    unsigned long long* absorb;   // [nx*ny*nz]
    unsigned long long* det;      // [n_dets * 4]: weight, count, target weight, weight^2
    unsigned long long* tbin;     // [n_dets * n_time * 4]
    unsigned long long* ledger;   // [kLedgerSlots]
    unsigned long long* counter;  // photon id dispenser
    const volatile int* cancel;   // device cancel flag, written by xmc_cancel from another stream (may be null)
    int* status;                  // device status word: bit0 budget hit, bit1 cancelled
    // biasing (InputInfo.useBiasing): attractive point and weight-integral tables
    int use_bias;
    float bias_eps;                       // attractiveFactor
    float bias_ox, bias_oy, bias_oz;      // startPosition
    float bias_rx, bias_ry, bias_rz;      // targetPoint - startPosition
    const float* wtab;                    // [tables x wtab_n]
    int wtab_n;                           // elements per table
    int8_t layer_wtab[MAX_LAYERS];        // table of each layer's anisotropy, -1 if none
};

// Host-side device image and buffers of one context.
struct Context {
    int device = 0;
    xmc_options opt{};
    KParams kp{};
    double rsp = 0.0;         // specular reflectance (FP64, as the reference computes it)
    uint32_t w0_fx = 0;
    int grid_size = 0, n_dets = 0, n_time = 0;
    size_t smem_bytes = 0;
    int block = 256, blocks_per_sm = 0, num_sms = 0, grid = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // device buffers
    void* d_nodes = nullptr; void* d_tris = nullptr; void* d_next = nullptr; void* d_dets = nullptr;
    void* d_absorb = nullptr; void* d_det = nullptr; void* d_tbin = nullptr; void* d_ledger = nullptr;
    void* d_counter = nullptr; void* d_status = nullptr;
    void* d_cells = nullptr; void* d_cell_z = nullptr; void* d_cell_entries = nullptr; void* d_big = nullptr; void* d_cancel = nullptr;
    void* d_cell_runs = nullptr;
    void* d_wtab = nullptr;
    cudaStream_t cancel_stream = nullptr;
    void* d_scatter = nullptr; void* d_traj = nullptr; void* d_replay = nullptr; void* d_replay_count = nullptr;
    void* d_replay_ledger = nullptr;
    void* d_xlog = nullptr;     // crossing log of the trajectory maps
    unsigned long long replay_cap = 0;
    unsigned long long last_replayed = 0;  // photons the last run walked again (crossing log overflow)
    int* h_cancel = nullptr;  // pinned source of the value xmc_cancel writes into d_cancel
    // pinned read-back buffers
    unsigned long long* h_absorb = nullptr; unsigned long long* h_det = nullptr;
    unsigned long long* h_tbin = nullptr;
    unsigned long long* h_ledger = nullptr;  // [2 x kLedgerSlots]: the run pass, then the replay pass
    unsigned long long* h_maps = nullptr;   // pinned staging of the scattering map (lazy)
    size_t h_maps_bytes = 0;
    // sparse read-back of the trajectory maps (lazy): block counts and their scan, the non-zero cells as
    // (cell, count) pairs grouped by map, and their pinned staging
    unsigned long long* d_nz_counts = nullptr; unsigned long long* d_nz_offsets = nullptr;
    void* d_nz_tmp = nullptr; size_t nz_tmp_bytes = 0;
    unsigned* d_nz_idx = nullptr; unsigned long long* d_nz_val = nullptr; size_t nz_cap = 0;
    unsigned long long* h_nz_offsets = nullptr;  // [maps x blocks per map + 1]: offsets, then the last count
    unsigned* h_nz_idx = nullptr; unsigned long long* h_nz_val = nullptr; size_t h_nz_cap = 0;
    unsigned long long* h_traj = nullptr; size_t h_traj_bytes = 0;  // dense copy, when the list would be larger
    int* h_status = nullptr;
    uint64_t last_n = 0;
    double last_kernel_ms = 0.0, last_total_ms = 0.0;
    uint64_t h2d_bytes = 0;   // bytes uploaded by xmc_create (device image)
};

// Host image of the geometry before upload.
struct GeomImage {
    std::vector<float4> nodes;   // 2 per node
    std::vector<float4> tris;    // 3 per triangle
    int n_nodes = 0, n_tris = 0;
};

// Host image of the xy cell grid.
struct GridImage {
    float x0 = 0, y0 = 0, icx = 0, icy = 0;
    int nx = 0, ny = 0;
    std::vector<uint2> cells;
    std::vector<float4> cell_z;   // 2 per cell: (lo0, hi0, lo1, hi1), (lo2, hi2, lo3, hi3); unused = (inf, -inf)
    std::vector<uint32_t> cell_runs;  // per cell: entries in each z-interval (4 x 8 bits), 0xffffffff: not split
    std::vector<float4> entries;  // per cell, sorted by z-low: the entries of each z-interval are contiguous
    std::vector<float4> big;      // 4 float4 per big triangle
};

// Everything the kernel needs, built on the host from an InputInfo (no device memory yet): kernel
// parameters with null device pointers, and the arrays they will point to.
struct HostImage {
    xmc_options opt{};
    KParams kp{};
    GeomImage geom;
    std::vector<int8_t> next;        // [n_surf * MAX_LAYERS]
    std::vector<float> wtab;         // weight-integral tables (biasing)
    bool need_wtab = false;          // biasing without caller tables: compute them on the GPU
    std::vector<DevDetector> dets;   // [max(1, n_dets)]
    GridImage grid;
    double rsp = 0.0;
    uint32_t w0_fx = 0;
    int grid_size = 0, n_dets = 0, n_time = 0;
    size_t smem_bytes = 0;
};

// weight_table.cu: weight-integral tables of the biased walk, computed on `device` in FP64
int compute_weight_tables(const InputInfo* in, int device, std::vector<double>* gs, std::vector<double>* tables,
                          int* n_elem);
std::vector<double> distinct_anisotropies(const InputInfo* in);
// capi.cpp: layer -> table mapping and float tables for the kernel from FP64 tables
int set_weight_tables(const InputInfo* in, const std::vector<double>& gs, const std::vector<double>& tables, int n_elem,
                      HostImage* img);

// capi.cpp: validate `in` and build its host image (options normalised as xmc_create does).
int prepare_image(const InputInfo* in, const xmc_options* opt, HostImage* img);
// capi.cpp: fill a ledger from the raw device ledger slots of a run of n photons.
void fill_ledger(const unsigned long long* raw, uint32_t w0_fx, uint64_t n, xmc_ledger* led);

// bvh.cpp
// gpu_device >= 0 and no usable prebuilt tree: the BVH topology is built on that GPU (bvh_gpu.cu)
bool build_geometry(const InputInfo* in, GeomImage* out, std::string* err, int gpu_device = -1);
bool gpu_lbvh_topology(const std::vector<float>& cen, int n, int device, std::vector<int>* order,
                       std::vector<int2>* child, std::vector<int2>* range, std::string* err);
// bvh.cpp: merged z-intervals occupied by the triangles of `g` (at most kMaxZSlabs, conservative)
int occupied_z_slabs(const GeomImage& g, float* lo, float* hi);

// bvh.cpp: build the xy cell grid over the triangles of `g` (empty grid when there are none)
void build_xy_grid(const GeomImage& g, GridImage* out, int tris_per_cell = 2);

// transport.cu: enqueue one transport kernel launch on ctx->stream (tallies must be zeroed).
cudaError_t enqueue_transport(Context* ctx);
// sparse_maps.cu: blocks of cells per map, and the two passes of the sparse map read-back
unsigned sparse_blocks_per_map(size_t cells);
cudaError_t sparse_maps_count(const unsigned long long* maps, size_t cells, int n_maps, unsigned long long* counts,
                              unsigned long long* offsets, void** scan_tmp, size_t* scan_tmp_bytes, cudaStream_t st);
cudaError_t sparse_maps_write(const unsigned long long* maps, size_t cells, int n_maps, const unsigned long long* offsets,
                              unsigned* idx, unsigned long long* val, cudaStream_t st);
// transport.cu: occupancy of the kernel for a block size and dynamic shared memory.
cudaError_t transport_occupancy(int block, size_t smem, int* blocks_per_sm, bool bias = false);
// transport.cu: Philox blocks computed on the device (self test).
cudaError_t device_philox(uint32_t key0, uint32_t key1, uint64_t pid, uint32_t n, uint32_t* host_out);

void set_error(const std::string& msg);

// Keeps the caller's current CUDA device across an entry point: the device current on entry is
// made current again when the guard goes out of scope (every return path), so an entry point that
// selects a context's device does not move the caller's later work (or xmc_launch_omp, which runs
// on the current device) to another GPU.
class DeviceGuard {
  public:
    DeviceGuard() { ok_ = cudaGetDevice(&prev_) == cudaSuccess; }
    ~DeviceGuard() {
        int cur = -1;
        if (ok_ && cudaGetDevice(&cur) == cudaSuccess && cur != prev_) cudaSetDevice(prev_);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

  private:
    int prev_ = 0;
    bool ok_ = false;
};

}  // namespace xmc
