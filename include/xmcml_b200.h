/*
 * xmcml_b200 — C-ABI of the B200 photon-transport library.
 *
 * The library replaces the node driver of xMCML (the OpenMP `LaunchOMP` call and the
 * `ComputePhoton` walk below it) with one persistent CUDA kernel per call on an sm_100a GPU.
 *
 * Part 1 declares the reference's own data structures with the reference's field order, types
 * and struct tags, so a caller built against the reference headers passes the same objects:
 *   base/xmcml/xmcml/mcml_types.h:1-41           (double3, int3, byte3, Area, Surface)
 *   base/xmcml/xmcml/mcml_intersection.h:12-57   (IntersectionInfo, Triangle, AABB, BVHNode, BVHTree)
 *   base/xmcml/xmcml/mcml_kernel_types.h:7-124   (TimeInfo ... PhotonTrajectory, MAX_LAYERS)
 *   base/xmcml/xmcml/mcml_mcg59.h:6-10           (MCG59)
 * The layouts are checked field by field against the reference headers by the test suite
 * (xmc_layout_offsets below).
 *
 * Part 2 declares the entry points. Every function returns an xmc_status (0 = success) unless
 * it mirrors a reference function whose return type it keeps; xmc_last_error() gives the text of
 * the last failure on the calling thread.
 */
#ifndef XMCML_B200_H
#define XMCML_B200_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- Part 1: reference layouts */

#define MAX_LAYERS 8
#define MAX_TRAJECTORY_SIZE 20480

typedef unsigned char byte;
typedef unsigned int uint;
typedef unsigned long long int uint64;

typedef union __double3 {
    struct { double x, y, z; };
    struct { double cell[3]; };
} double3;

typedef union __int3 {
    struct { int x, y, z; };
    struct { int cell[3]; };
} int3;

typedef union __byte3 {
    struct { byte x, y, z; };
    struct { byte cell[3]; };
} byte3;

typedef struct __Area {
    double3 corner;
    double3 length;
    int3 partitionNumber;
} Area;

typedef struct __Surface {
    double3* vertices;
    int numberOfVertices;
    int3* triangles;
    int numberOfTriangles;
} Surface;

typedef struct __IntersectionInfo {
    double3 normal;
    double distance;
    int surfaceId;
    int isFindIntersection;
} IntersectionInfo;

typedef struct __Triangle {
    int surfId;
    int trIndex;
} Triangle;

typedef struct __AABB {
    double3 Ver1;
    double3 Ver2;
} AABB;

/* The reference gives BVHNode and BVHTree C++ constructors; the layout is the same. */
typedef struct __BVHNode {
    AABB Box;
    int rightNode;
    int leftNode;
    int offset;
    int numOfTriangles;
} BVHNode;

typedef struct __BVHTree {
    BVHNode* nodes;
    int numOfNodes;
    int root;
    Triangle* triangles;
    int numOfTriangles;
} BVHTree;

typedef struct __TimeInfo {
    double timeStart;
    double timeFinish;
    uint64 numberOfPhotons;
    double weight;
    double targetWeight;
} TimeInfo;

typedef struct __CubeDetector {
    double3 center;
    double3 length;
    bool filterLayers[MAX_LAYERS];
    double targetAngle;
} CubeDetector;

typedef struct __RingDetector {
    double3 center;
    double smallRadius;
    double bigRadius;
    bool filterLayers[MAX_LAYERS];
    double targetAngle;
} RingDetector;

typedef struct __DetectorInfo {
    uint64 numberOfPhotons;
    uint64* trajectory;
    int trajectorySize;
    TimeInfo* timeScale;
    int timeScaleSize;
    double targetWeight;
    double weight;
} DetectorInfo;

typedef struct __WeightIntegralTable {
    double anisotropy;
    int numberOfElements;
    double* elements;
} WeightIntegralTable;

typedef struct __LayerInfo {
    double refractiveIndex;
    double absorptionCoefficient;
    double scatteringCoefficient;
    double anisotropy;
    int* surfaceId;
    int numberOfSurfaces;
} LayerInfo;

typedef struct __InputInfo {
    uint64 numberOfPhotons;
    Area* area;
    LayerInfo* layerInfo;
    int numberOfLayers;
    Surface* surface;
    int numberOfSurfaces;
    CubeDetector* cubeDetector;
    int numberOfCubeDetectors;
    RingDetector* ringDetector;
    int numberOfRingDetectors;
    double minWeight;
    BVHTree* bvhTree;
    double timeStart;
    double timeFinish;
    int timeScaleSize;
    double3 startPosition;
    double3 startDirection;
    byte useBiasing;
    uint weightIntegralPrecision;
    uint weightTablePrecision;
    double attractiveFactor;
    WeightIntegralTable* weightTable;
    int numberOfWeightTables;
    double3 targetPoint;
    unsigned char targetRangeLayers[MAX_LAYERS];
} InputInfo;

typedef struct __OutputInfo {
    uint64 numberOfPhotons;
    double specularReflectance;
    double* absorption;
    double* scattering;
    int gridSize;
    DetectorInfo* detectorInfo;
    int numberOfDetectors;
} OutputInfo;

typedef struct __MCG59 {
    uint64 value;
    uint64 offset;
} MCG59;

/* ---------------------------------------------------------------- Part 2: entry points */

typedef enum xmc_status {
    XMC_OK = 0,
    XMC_ERR_INVALID_INPUT = 1,   /* a field of InputInfo/OutputInfo is missing or inconsistent */
    XMC_ERR_RANGE = 2,           /* a size is outside what the library supports (e.g. partition > 256) */
    XMC_ERR_DEVICE = 3,          /* a CUDA call failed; the text names it */
    XMC_ERR_BUDGET = 4,          /* a photon hit the per-photon step budget (it was terminated) */
    XMC_ERR_CANCELLED = 5,       /* xmc_cancel() stopped the run; tallies hold the photons done */
    XMC_ERR_IO = 6,              /* a file could not be read or written */
    XMC_ERR_UNSUPPORTED = 7      /* a reference feature the GPU path does not provide (biasing) */
} xmc_status;

/* Option flags (xmc_options.flags). */
#define XMC_ROULETTE        (1u << 0)  /* Russian roulette at minWeight instead of killing the photon */
#define XMC_NO_AREA_KILL    (1u << 1)  /* photons leaving Area keep walking; their absorption goes to
                                          the ledger's absorbed_outside term                         */
#define XMC_SCATTERING_MAP  (1u << 2)  /* tally the z-plane crossing map OutputInfo.scattering         */
#define XMC_DETECTOR_TRAJ   (1u << 3)  /* tally per-detector trajectory maps DetectorInfo.trajectory
                                          (from a per-thread crossing log; photons whose log overflows
                                          are walked again in a replay pass)                        */
#define XMC_LARGE_GRID      (1u << 4)  /* accept Area partitions above 256 per axis (the reference wraps
                                          voxel indices at 256; this library indexes them in full)    */
#define XMC_GPU_BVH         (1u << 5)  /* without input->bvhTree, build the BVH topology on the GPU (linear
                                          BVH over Morton-sorted triangle centroids) instead of the
                                          host's binned SAH: far faster to build for large meshes, a
                                          little slower to traverse; xmc_run_noalloc ignores it      */
#define XMC_LANE_QUERIES    (1u << 6)  /* short ray queries walk the xy cell grid lane by lane instead of
                                          warp-cooperatively (same hits, same tallies bit for bit;
                                          a launch-shape choice for the autotuner)                    */

typedef struct xmc_options {
    uint32_t struct_size;          /* sizeof(xmc_options); 0 selects all defaults                */
    uint32_t flags;                /* XMC_* flags above                                           */
    double   roulette_chance;      /* survival probability of roulette (default 0.1)             */
    double   beam_radius;          /* uniform-disk beam radius in mm around startPosition (0 = pencil) */
    uint64_t max_steps_per_photon; /* step budget per photon (0 = 10,000,000)                    */
    int32_t  device;               /* CUDA device ordinal (default 0)                            */
    int32_t  block_size;           /* threads per block (0 = 512)                                  */
    int32_t  blocks_per_sm;        /* resident blocks per SM (0 = occupancy maximum)              */
    int32_t  photons_per_chunk;    /* photon ids a warp claims at a time (0 = 32)                 */
    int32_t  smem_nodes;           /* BVH nodes staged in shared memory (-1 = none, 0 = auto)      */
    int32_t  trajectory_log;       /* XMC_DETECTOR_TRAJ: z-plane crossings logged per resident thread
                                    * (0 = 4096, at most 65536; -1 = no log, every detected photon
                                    * is replayed)                                                 */
    int32_t  query_batch;          /* cooperative ray queries: rays a warp collects (the lanes that
                                    * need one wait) before it runs a query round (0 = 12; 1 = every
                                    * iteration). A scheduling choice: tallies are the same bit for bit */
    int32_t  grid_cell_tris;       /* triangles per cell the xy grid of short ray queries aims at (0 = 12;
                                    * larger: coarser cells, fewer queries fall back to the BVH). A
                                    * speed choice: tallies are the same bit for bit              */
    int32_t  reserved[4];
} xmc_options;

/* Energy ledger of one or more runs: every photon's start weight 1 is split exactly into these
 * terms. The *_fx fields are the raw 64-bit fixed-point sums (weight * 2^31); the double fields
 * are the same sums divided by the number of photons. specular + absorbed + absorbed_outside +
 * escaped_top + escaped_bottom + lost_area + lost_cut + lost_glass + lost_budget + lost_invalid
 * + roulette_killed - roulette_gained == 1 holds exactly in the fixed-point sums. */
typedef struct xmc_ledger {
    uint64_t photons_launched;
    uint64_t photons_terminated;
    uint64_t steps;                /* walk-loop iterations                                      */
    uint64_t n_escaped_top, n_escaped_bottom, n_area, n_cut, n_roulette, n_glass, n_budget, n_invalid;
    uint64_t n_detected;           /* photons that scored in a detector                        */
    uint64_t n_fp64_retests;       /* ray-triangle tests redone in FP64 in an edge band          */
    uint64_t n_node_visits;        /* BVH nodes visited by all ray queries                      */
    uint64_t n_triangle_tests;     /* ray-triangle tests                                        */
    uint64_t n_replay_mismatch;    /* trajectory replay: photons whose replayed exit differed (0) */
    uint64_t specular_fx, absorbed_fx, absorbed_outside_fx, escaped_top_fx, escaped_bottom_fx,
             lost_area_fx, lost_cut_fx, lost_glass_fx, lost_budget_fx, lost_invalid_fx,
             roulette_killed_fx, roulette_gained_fx;
    double specular, absorbed, absorbed_outside, escaped_top, escaped_bottom, lost_area, lost_cut,
           lost_glass, lost_budget, lost_invalid, roulette_killed, roulette_gained;
    double kernel_ms;              /* device time of the transport kernel(s), CUDA events       */
    double total_ms;               /* device time of the whole run incl. zeroing and read-back  */
    uint64_t h2d_bytes;            /* bytes copied host->device for the context's device image  */
    uint64_t d2h_bytes;            /* bytes copied device->host by this run                     */
    uint64_t absorbed_target_fx;   /* weight dropped while in a layer flagged in targetRangeLayers
                                    * (inside or outside Area; a part of absorbed + absorbed_outside) */
    double absorbed_target;        /* the same per launched photon                               */
    uint64_t bias_gained_fx;       /* biasing: weight added by the weight-table factor W / p > 1  */
    uint64_t bias_lost_fx;         /* biasing: weight removed by factors < 1                      */
    double bias_gained, bias_lost; /* the same per launched photon                               */
    uint64_t n_trajectory_replayed;/* XMC_DETECTOR_TRAJ: detected photons walked again because their
                                    * crossing log overflowed                                       */
    uint64_t n_plane_crossings;    /* z-plane crossings through voxel centres recorded for the
                                    * scattering / trajectory maps (run pass; 0 without maps)       */
} xmc_ledger;

typedef struct xmc_context xmc_context;

/* Library version as 10000*major + 100*minor + patch. */
int xmc_version(void);

/* Text of the last error on this thread ("" if none). */
const char* xmc_last_error(void);

/* Fill *opt with defaults (sets struct_size). */
void xmc_default_options(xmc_options* opt);

/* Build a device image of `input` (layers, triangles, BVH, detectors, time bins, Area) on the
 * GPU. Uses input->bvhTree when it is set (the reference's GenerateBVHTree output, as the
 * reference's launchers prebuild it: base/xmcml/xmcmlLauncher/launcher_mpi.cpp:396), else builds
 * a BVH itself. Does not retain any pointer into `input`. */
int xmc_create(const InputInfo* input, const xmc_options* opt, xmc_context** out_ctx);

/* Run photons [first_photon_id, first_photon_id + n_photons) with counter-RNG key `seed` and
 * ADD the tallies to `output` (reference semantics: LaunchOMP accumulates,
 * base/xmcml/xmcmlLauncher/launcher_omp.cpp:146-154), setting output->specularReflectance.
 * `output` may be NULL (tallies stay on the device, see xmc_read_tallies); `ledger` may be NULL.
 * Returns XMC_ERR_BUDGET if any photon hit the step budget (tallies are still valid). */
int xmc_run(xmc_context* ctx, uint64_t seed, uint64_t first_photon_id, uint64_t n_photons,
            OutputInfo* output, xmc_ledger* ledger);

/* Raw 64-bit fixed-point device tallies of the last xmc_run, copied to host arrays (any may be
 * NULL): absorption[gridSize], detector weight/count/targetWeight/weight^2 [numberOfDetectors],
 * time bins weight/count/targetWeight/weight^2 [numberOfDetectors * timeScaleSize]. */
int xmc_read_tallies(xmc_context* ctx, uint64_t* absorption, uint64_t* det_weight,
                     uint64_t* det_count, uint64_t* det_target, uint64_t* det_weight2,
                     uint64_t* time_weight, uint64_t* time_count, uint64_t* time_target,
                     uint64_t* time_weight2);

/* The z-plane crossing tallies of the last xmc_run (host arrays, either may be NULL): the
 * scattering map [gridSize] in weight fixed point (context created with XMC_SCATTERING_MAP) and the
 * detector trajectory maps [numberOfDetectors * gridSize] as crossing counts (XMC_DETECTOR_TRAJ). */
int xmc_read_maps(xmc_context* ctx, uint64_t* scattering, uint64_t* trajectory);

/* Ask a running xmc_run on another thread to stop after the photons in flight. */
int xmc_cancel(xmc_context* ctx);

int xmc_destroy(xmc_context* ctx);

/* No counterpart in the reference (the project's autotuner of the transport kernel's launch shape).
 * Builds the device image of `input` under `base` (its flags, device and semantics are kept) and
 * times `sample_photons` photons (0 = 1e6) under every candidate: xy-grid density grid_cell_tris
 * {2, 8, 16, 32} triangles per cell, block size {256, 512} at the occupancy maximum, photon ids a warp
 * claims from the dispenser at a time {32, 64}, and the ray-query scheme (warp-cooperative with
 * query_batch {1, 8, 12, 16}, or lane by lane with XMC_LANE_QUERIES): 80 candidates, each timed once, the
 * four fastest twice more on other photons. *best gets `base` with the fastest one, *best_ms (may be
 * NULL) its best kernel time. Every candidate gives bit-identical
 * tallies: a photon's random numbers, its candidate triangles' arithmetic and the choice among equal
 * distances (the lower triangle index) do not depend on them. */
int xmc_autotune(const InputInfo* input, const xmc_options* base, uint64_t sample_photons, xmc_options* best,
                 double* best_ms);

/* One call = create + run on a device context. The context of the last model is kept for the next
 * call when nothing its device image depends on has changed (a 64-bit fingerprint over the layers,
 * surfaces, detectors, Area, time bins, start, biasing fields, weight tables, caller BVH and options;
 * numberOfPhotons may change), as the reference's launchers call LaunchOMP repeatedly on one
 * InputInfo. Calls are serialised by a lock. xmc_launch_release() frees the kept context. */
int xmc_launch_release(void);
int xmc_launch(const InputInfo* input, OutputInfo* output, uint64_t seed,
               uint64_t first_photon_id, const xmc_options* opt, xmc_ledger* ledger);

/* No counterpart in the reference. A transport run that allocates no GPU memory, for callers that
 * cannot call cudaMalloc: code running inside a host framework that owns all device memory through
 * its own pool, or a process that must not grow its device footprint once it is running. The
 * caller passes the model (`input`, host memory, as for xmc_create) and its own device buffers for
 * the raw 64-bit fixed-point outputs (weight 1.0 == 2^31), which the call zeroes and then fills:
 *   d_absorption [gridSize]; d_detectors [4 * D] (weight, count, target weight, weight^2 per
 *   detector, D = cube + ring detectors, at least 1); d_time_bins [4 * D * timeScaleSize];
 *   d_ledger [32] (raw energy-ledger slots).
 * The device copy of the model (BVH nodes, triangles, layer transitions, detectors, xy cell grid)
 * and the photon-id dispenser live in one static device array of XMC_NOALLOC_SCRATCH_BYTES (8 MiB)
 * that every GPU loading the library holds until exit; a model that needs more is rejected with
 * XMC_ERR_RANGE (a mesh of up to roughly 50,000 triangles fits). The first call on a device is its
 * set-up: it looks up that array's device address (cudaGetSymbolAddress) and keeps it, so make that
 * first call before any stream capture starts on the device. All calls share the array and it keeps
 * the last call's contents: calls that overlap on the GPU (on different streams or threads) race and
 * must be serialised by the caller. `stream` is a cudaStream_t (NULL = the default stream); each call
 * copies the model into the array, runs, and waits for the run to finish on that stream before it
 * returns. The caller's current device is unchanged on return. No host event, pinned buffer or
 * device allocation is made; the only host memory used is ordinary heap for the model image. */
#define XMC_NOALLOC_SCRATCH_BYTES (8u << 20)
int xmc_run_noalloc(const InputInfo* input, const xmc_options* opt, uint64_t seed, uint64_t first_photon_id,
                    uint64_t n_photons, unsigned long long* d_absorption, unsigned long long* d_detectors,
                    unsigned long long* d_time_bins, unsigned long long* d_ledger, void* stream);

/* No counterpart in the reference (a measurement utility): throughput of 64-bit atomic adds to
 * scattered addresses of a device array of 2^log2_slots u64 (2^20 = 8 MB stays in L2), the access
 * pattern of the walk's absorption-grid and map tallies; adds_per_thread per thread over a grid of
 * 8 blocks of 256 threads per SM. Allocates and frees its own array on `device`. */
int xmc_atomic_throughput(int device, unsigned log2_slots, unsigned adds_per_thread, double* atomics_per_s,
                          double* ms);

/* No counterpart in the reference (LaunchOMP has no options argument). Sets the options
 * xmc_launch_omp uses for its later calls in this process, e.g. the launch shape xmc_autotune found
 * for the model (NULL: back to the defaults). xmc_launch_omp still sets XMC_SCATTERING_MAP and
 * XMC_DETECTOR_TRAJ and takes the device from the calling thread; the options are copied. */
int xmc_launch_set_options(const xmc_options* opt);

/* Replaces LaunchOMP(InputInfo*, OutputInfo*, MCG59*, int)
 * (base/xmcml/xmcmlLauncher/launcher_omp.h:10, launcher_omp.cpp:123-163): runs
 * input->numberOfPhotons photons on the GPU and adds the tallies to `output` (output->
 * numberOfPhotons is left to the caller, as the reference does). The counter-RNG key is
 * randomGenerator[0].value and the photons are ids 0..numberOfPhotons-1 (all of LaunchOMP's
 * tallies are filled, including the scattering map and the detector trajectory maps); afterwards
 * randomGenerator[0] is advanced by one MCG59 step, so consecutive calls (the reference's backup
 * portions, launcher_mpi.cpp:357-380) use fresh keys. numThreads is ignored. It runs on the
 * calling thread's current CUDA device (cudaSetDevice), so one process per GPU, each with its own
 * device selected, runs its own share. Default options otherwise (reference semantics: weight cut
 * at minWeight, photons killed outside Area). Returns 0 on success; on failure it prints
 * xmc_last_error() to stderr and returns the status. */
int xmc_launch_omp(InputInfo* input, OutputInfo* output, MCG59* randomGenerator, int numThreads);

/* Replaces InitOutput / FreeOutput (base/xmcml/xmcmlLauncher/launcher_omp.cpp:10-58, 76-104):
 * allocates and zeroes the tally arrays of `output` for `input`. */
void xmc_init_output(InputInfo* input, OutputInfo* output);
void xmc_free_output(OutputInfo* output);

/* Replaces ParseInputFile / ParseSurfaceFile (base/xmcml/xmcmlLauncher/parser.cpp:18-514,
 * 583-611): reads the reference's XML model and binary .surface file into `input`.
 * Return true on success, like the reference. */
bool xmc_parse_input_file(const char* fileName, InputInfo* input);
bool xmc_parse_surface_file(const char* fileName, InputInfo* input);
void xmc_free_input(InputInfo* input);

/* Replaces WriteOutputToFile (base/xmcml/xmcmlLauncher/writer.cpp:431-471): writes the
 * sectioned binary .mcml.out. Returns true on success, like the reference. */
bool xmc_write_output_file(InputInfo* input, OutputInfo* output, const char* fileName);

/* Replaces GenerateBVHTree (base/xmcml/xmcml/mcml_intersection.cpp:316-344): builds a binned-SAH
 * BVH over all triangles of `surfaces` in the reference's BVHTree layout (FP64 boxes, leaves as
 * (surfId, trIndex) runs), for callers that prebuild input->bvhTree once (launcher_mpi.cpp:396).
 * Returns NULL on invalid input (see xmc_last_error). Free with xmc_free_bvh_tree. */
BVHTree* xmc_generate_bvh_tree(const Surface* surfaces, int numberOfSurfaces);
void xmc_free_bvh_tree(BVHTree* tree);

/* Replaces the computing branch of GetWeightIntegralTable (base/xmcml/xmcmlLauncher/weight_integral.cpp:
 * 17-104, mcml_integration.cpp:7-83): the biased walk's weight-integral tables, one per distinct
 * anisotropy of layers 1..numberOfLayers-1, weightTablePrecision + 1 values each, computed on GPU
 * `device` in FP64 and stored in input->weightTable / numberOfWeightTables (new[]-allocated; freed
 * by xmc_free_input; a previous table is not freed). xmc_create computes them itself when
 * input->useBiasing is set and input->weightTable is NULL. */
int xmc_weight_integral_table(InputInfo* input, int device);

/* Replaces ComputeSpecularReflectance (base/xmcml/xmcml/mcml_kernel.cpp:16-37). */
double xmc_specular_reflectance(const LayerInfo* layer);

/* Counter RNG used by the kernel: Philox4x32-10 (Salmon et al., SC'11) of counter
 * (ctr[0..3]) and key (key[0..1]); host implementation for tests and tools. */
void xmc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Byte offsets of the Part 1 struct fields in a fixed order (see layout.cpp); returns count. */
int xmc_layout_offsets(int64_t* out, int max_count);

/* Self test of the kernel's ray query compiled for the host: for each ray (ox,oy,oz,dx,dy,dz in
 * rays[6*i]) the nearest hit with tmin <= t <= tmax over the device image of `input` (distance,
 * surface id or -1, unit normal or NULL), through the xy cell grid where the kernel would use it
 * (bit 0 of `flags`) or the BVH only; bit 1 builds the image's BVH on GPU 0 (XMC_GPU_BVH) instead
 * of the host. Used by the test suites. */
int xmc_debug_nearest(const InputInfo* input, int n_rays, const float* rays, float tmin, float tmax,
                      float* t_out, int* surf_out, float* normal_out, int flags);

/* Run the photon kernel's device-side self test: `n` Philox blocks for the given key written to
 * out[4*n] (device path), for comparing with xmc_philox4x32_10. */
int xmc_device_philox(uint64_t seed, uint64_t photon_id, uint32_t n, uint32_t* out);

/* ---------------------------------------------------------------- Part 3: batched instances
 *
 * Many optical-property instances of one planar layer stack in ONE persistent launch. No
 * counterpart in the reference, which runs one InputInfo per LaunchOMP call; an instance is the
 * planar model a caller would otherwise run through LaunchOMP: ambient medium above and below,
 * n_layers tissue layers (planes at the cumulative thicknesses), pencil beam at normal incidence
 * entering at the origin (or a uniform disk of beam_radius), rings of equal width around the
 * beam axis, time bins in optical path length (the reference's timeStart/timeFinish, mm), and
 * roulette below min_weight. Instance k walks photon ids 0..photons-1 with counter-RNG key
 * seed_k, so it reproduces photon for photon xmc_run(seed_k) on the equivalent planar InputInfo
 * (with XMC_ROULETTE | XMC_NO_AREA_KILL). Photon budgets may differ between instances: the
 * kernel hands out photon ids of all instances from one dispenser. */
#define XMC_BATCH_MAX_LAYERS 6
#define XMC_BATCH_LEDGER 16

typedef struct xmc_batch_spec {
    uint32_t struct_size;          /* sizeof(xmc_batch_spec)                                     */
    int32_t n_layers;              /* tissue layers, 1..XMC_BATCH_MAX_LAYERS                     */
    int32_t n_rings;               /* ring i covers radii [i, i+1) * ring_width                  */
    int32_t n_time;                /* time bins per ring, >= 1 (the last bin is open-ended)      */
    double ring_width;             /* mm                                                         */
    double time_start, time_finish;/* optical path length window of the time bins, mm            */
    double ring_angle;             /* acceptance half-angle, degrees: -uz > cos(angle) (90 = all) */
    double min_weight;             /* roulette threshold (e.g. 1e-4)                             */
    double roulette_chance;        /* survival chance (e.g. 0.1)                                 */
    uint64_t max_steps_per_photon; /* step budget per photon (0 = 1e7)                           */
    int32_t max_instances;         /* capacity of the device tables                              */
    int32_t use_graph;             /* 1: each run is a replayed CUDA graph; 0: plain stream work  */
    int32_t device;
    int32_t reserved[7];
} xmc_batch_spec;

typedef struct xmc_batch_instance {
    double mua[XMC_BATCH_MAX_LAYERS];       /* mm^-1 */
    double mus[XMC_BATCH_MAX_LAYERS];       /* mm^-1, mua + mus > 0 */
    double g[XMC_BATCH_MAX_LAYERS];         /* anisotropy, (-1, 1) */
    double n[XMC_BATCH_MAX_LAYERS];         /* refractive index */
    double thickness[XMC_BATCH_MAX_LAYERS]; /* mm; the last tissue layer ends at the sum */
    double n_above, n_below;                /* ambient refractive index */
    double beam_radius;                     /* mm, uniform disk (0 = pencil beam) */
    uint64_t photons;                       /* budget of this instance (0 allowed) */
    uint64_t seed;                          /* counter-RNG key */
} xmc_batch_instance;

/* Launch shape of the batched kernel; chosen by xmc_batch_autotune or set by the caller. */
typedef struct xmc_batch_tuning {
    int32_t block_size;         /* threads per block, multiple of 32, <= 256                   */
    int32_t blocks_per_sm;      /* resident blocks per SM (0 = as many as fit)                 */
    int32_t photons_per_chunk;  /* photon ids a warp takes from the dispenser at a time        */
    int32_t tally_scheme;       /* 0: per-photon global atomics for the instance ledger;
                                 * 1: thread-private ledger sums, flushed when the thread moves
                                 *    to another instance and at the end                      */
    double ms;                  /* autotuner: kernel time of the winning trial                 */
} xmc_batch_tuning;

/* Per-instance ledger slots (uint64 each; *_FX are weights in 2^31 fixed point). */
enum {
    XMC_BL_LAUNCHED = 0, XMC_BL_STEPS = 1, XMC_BL_TOP_FX = 2, XMC_BL_BOTTOM_FX = 3, XMC_BL_ABSORBED_FX = 4,
    XMC_BL_RKILLED_FX = 5, XMC_BL_RGAINED_FX = 6, XMC_BL_BUDGET_FX = 7, XMC_BL_N_TOP = 8, XMC_BL_N_BOTTOM = 9,
    XMC_BL_N_ROULETTE = 10, XMC_BL_N_BUDGET = 11, XMC_BL_N_DETECTED = 12
};

/* Per-instance summary in FP64, fractions of the launched weight. */
typedef struct xmc_batch_result {
    uint64_t photons, steps, n_detected, n_top, n_bottom, n_roulette, n_budget;
    double specular, escaped_top, escaped_bottom, absorbed, roulette_killed, roulette_gained, lost_budget;
} xmc_batch_result;

typedef struct xmc_batch xmc_batch;

/* Host-only check of a spec and an instance table (no GPU needed): the status xmc_batch_run
 * would return for them before touching the device. */
int xmc_batch_validate(const xmc_batch_spec* spec, const xmc_batch_instance* inst, int n);

/* Device tables for up to spec->max_instances instances on spec->device. */
int xmc_batch_create(const xmc_batch_spec* spec, xmc_batch** out);

/* Run n instances. Outputs (each may be NULL), as fractions of the instance's launched weight:
 * ring_time[n][n_rings][n_time], ring[n][n_rings], result[n]. kernel_ms (may be NULL) gets the
 * device time of the transport kernel. With use_graph the whole run (table upload, zeroing,
 * kernel, FP64 reduction, read-back) is captured once per instance count and replayed. */
int xmc_batch_run(xmc_batch* b, const xmc_batch_instance* inst, int n, double* ring_time, double* ring,
                  xmc_batch_result* result, double* kernel_ms);

/* Integer tallies of the last run: ring[n][n_rings][3] and ring_time[n][n_rings][n_time][3]
 * as (weight_fx, count, weight^2_fx), ledger[n][XMC_BATCH_LEDGER] (XMC_BL_* slots). Any may be NULL. */
int xmc_batch_read_tallies(xmc_batch* b, int n, uint64_t* ring, uint64_t* ring_time, uint64_t* ledger);

int xmc_batch_set_tuning(xmc_batch* b, const xmc_batch_tuning* t);
int xmc_batch_get_tuning(const xmc_batch* b, xmc_batch_tuning* t);

/* Times the batched kernel on `sample` (n instances, each capped at photons_cap photons) for
 * every candidate launch shape (block size {64, 128, 256} x photons per chunk {32, 64, 128, 256} x
 * tally scheme {0, 1}, as many blocks per SM as fit),
 * keeps the fastest in `b` and returns it in *best. */
int xmc_batch_autotune(xmc_batch* b, const xmc_batch_instance* sample, int n, uint64_t photons_cap,
                       xmc_batch_tuning* best);

int xmc_batch_destroy(xmc_batch* b);

/* ---------------------------------------------------------------- Part 4: surrogate network
 *
 * A fully connected network (n_hidden SiLU layers of width `hidden`, linear output) trained and
 * evaluated on the GPU's tensor cores: BF16 weights and activations, FP32 accumulation, FP32
 * master weights and Adam moments. No counterpart in the reference. It stands in for the Monte
 * Carlo inside inverse fitting: inputs are optical properties of a layered model, outputs its
 * ring- and time-resolved reflectance (the caller's normalisation on both sides). Row counts of
 * every call are multiples of 128 up to max_rows. Calls on one model are serialised. */
typedef struct xmc_mlp_spec {
    uint32_t struct_size;   /* sizeof(xmc_mlp_spec)                           */
    int32_t n_in;           /* inputs, 1..64                                  */
    int32_t hidden;         /* hidden width: 128 or 256                       */
    int32_t n_hidden;       /* hidden layers, 1..8                            */
    int32_t n_out;          /* outputs, 1..4096                               */
    int32_t max_rows;       /* row capacity of a forward or training batch    */
    int32_t device;
    int32_t forward_kernel; /* inference forward: 0 = one fused kernel for all layers when
                             * n_out % 4 == 0 (else per layer), 1 = one GEMM per layer  */
    int32_t reserved[8];
} xmc_mlp_spec;

typedef struct xmc_mlp xmc_mlp;

int xmc_mlp_create(const xmc_mlp_spec* spec, xmc_mlp** out);
/* Number of FP32 parameters in the flat layout: for each layer l, W_l [out_l][in_l] row-major
 * then b_l [out_l] (in_0 = n_in, out_last = n_out). */
int64_t xmc_mlp_param_count(const xmc_mlp* m);
/* Set / get the FP32 master parameters (set also resets the Adam moments and step count). */
int xmc_mlp_set_params(xmc_mlp* m, const float* params);
int xmc_mlp_get_params(const xmc_mlp* m, float* params);
/* y[rows][n_out] = network(x[rows][n_in]) with host buffers; *ms (may be NULL) = device time. */
int xmc_mlp_forward(xmc_mlp* m, const float* x, int rows, float* y, double* ms);
/* Mean device time of `reps` forward passes over the inputs of the last xmc_mlp_forward call
 * (device-resident, replayed CUDA graph). */
int xmc_mlp_forward_timed(xmc_mlp* m, int rows, int reps, double* ms);
/* Gradients of the mean squared error over rows (flat parameter layout), no update. */
int xmc_mlp_gradients(xmc_mlp* m, const float* x, const float* t, int rows, float* grads, float* loss);
/* Device-resident training set x[rows][n_in], t[rows][n_out]. */
int xmc_mlp_set_dataset(xmc_mlp* m, const float* x, const float* t, int rows);
/* `steps` Adam steps on minibatches of `batch` rows drawn from the training set with replacement
 * (Philox keyed by seed); losses[steps] (may be NULL) = each minibatch's mean squared error. */
int xmc_mlp_train(xmc_mlp* m, int steps, int batch, float lr, float beta1, float beta2, float eps,
                  uint64_t seed, float* losses, double* ms);
/* Per-output weights w[n_out] >= 0 of the squared error in training and xmc_mlp_gradients
 * (loss = mean over rows and outputs of w_j (y_j - t_j)^2); NULL restores all weights to 1. */
int xmc_mlp_set_output_weights(xmc_mlp* m, const float* w);
int xmc_mlp_destroy(xmc_mlp* m);

/* D[M][N] = A[M][K] . B[N][K]^T on the tensor cores (bf16 inputs as raw 16-bit patterns, FP32
 * out) through the network's GEMM kernel, tile width bn (64, 128, 256) and `splits` K-splits;
 * M % 128, N % bn and K % (64 splits) must be 0. For tests. */
int xmc_gemm_bf16(const uint16_t* a, const uint16_t* b, int M, int N, int K, int bn, int splits, float* d);

#ifdef __cplusplus
}
#endif

#endif /* XMCML_B200_H */
