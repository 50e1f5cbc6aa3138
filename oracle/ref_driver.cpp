/*
 * ORACLE — TEST INFRASTRUCTURE ONLY (not part of the product).
 *
 * Project-written driver around the reference's own sources, compiled where they lie by
 * oracle/Makefile into oracle/_ref/libxmcml_ref.so. It exposes plain C entry points so tests and
 * the CPU-baseline leg of bench.py can call the unmodified reference code through ctypes:
 * ParseInputFile / ParseSurfaceFile (base/xmcml/xmcmlLauncher/parser.cpp:18,583), InitOutput and
 * LaunchOMP (base/xmcml/xmcmlLauncher/launcher_omp.cpp:10,123), InitMCG59/NextMCG59
 * (base/xmcml/xmcml/mcml_mcg59.cpp:24,34), GenerateBVHTree (base/xmcml/xmcml/mcml_intersection.cpp:316),
 * WriteOutputToFile (base/xmcml/xmcmlLauncher/writer.cpp:431), and the per-function exports the
 * reference's unit tests call (base/xmcml/xmcml/mcml_kernel_debug.def).
 * The reference's main() and MPI launcher are not built (MPI is absent); this driver takes the
 * place of main.cpp:63-177 for a single process.
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "mcml_kernel.h"
#include "mcml_intersection.h"
#include "mcml_mcg59.h"
#include "mcml_math.h"
#include "launcher_omp.h"
#include "parser.h"
#include "writer.h"
#include "weight_integral.h"

// weight_integral.cpp:34-65 (external linkage, not declared in its header)
void ComputeWeightIntegral(InputInfo* input, CmdArguments* args);

extern "C" {

/* mcml_integration.cpp:7-83: one weight-integral value */
double ref_weight_integral(double dot, double g, double eps, unsigned n) { return ComputeWeightIntegral(dot, g, eps, n); }

/* weight_integral.cpp:34-65: the weight tables of every distinct layer anisotropy, as the
 * reference's launcher computes them before LaunchOMP when <Biasing> is on (no file written) */
void ref_weight_tables(InputInfo* in, int nthreads) {
    CmdArguments args;
    memset(&args, 0, sizeof(args));
    args.numberOfThreads = nthreads > 0 ? nthreads : 1;
    ComputeWeightIntegral(in, &args);
}

int ref_parse_input(const char* xml, InputInfo* in) {
    memset(in, 0, sizeof(*in));
    return ParseInputFile((char*)xml, in) ? 1 : 0;
}

int ref_parse_surface(const char* path, InputInfo* in) { return ParseSurfaceFile((char*)path, in) ? 1 : 0; }

/* main.cpp:146-152: the dummy weight table used when biasing is off */
void ref_dummy_weight_table(InputInfo* in) {
    in->numberOfWeightTables = 1;
    in->weightTable = new WeightIntegralTable[1];
    in->weightTable[0].numberOfElements = 1;
    in->weightTable[0].elements = new double[1];
    in->weightTable[0].elements[0] = 0.0;
    in->weightTable[0].anisotropy = 0.0;
}

void ref_init_output(InputInfo* in, OutputInfo* out) { InitOutput(in, out); }
void ref_free_output(OutputInfo* out) { FreeOutput(out); }

void ref_generate_bvh(InputInfo* in) { in->bvhTree = GenerateBVHTree(in->surface, in->numberOfSurfaces); }

void ref_init_mcg59(MCG59* g, uint64_t seed, unsigned id, unsigned step) { InitMCG59(g, seed, id, step); }
double ref_next_mcg59(MCG59* g) { return NextMCG59(g); }

/* main.cpp:105-112: one generator per thread, leapfrogged over all threads */
void ref_init_threads_mcg59(MCG59* g, uint64_t seed, int nthreads) {
    for (int i = 0; i < nthreads; ++i) InitMCG59(&g[i], seed, i, nthreads);
}

void ref_launch_omp(InputInfo* in, OutputInfo* out, MCG59* g, int nthreads) { LaunchOMP(in, out, g, nthreads); }

int ref_write_output(InputInfo* in, OutputInfo* out, const char* path) { return WriteOutputToFile(in, out, (char*)path) ? 1 : 0; }

/* ---- per-function exports (mcml_kernel_debug.def) ---- */
double ref_specular(LayerInfo* layers) { return ComputeSpecularReflectance(layers); }
double ref_cosine_theta(double g, MCG59* r) { return ComputeCosineTheta(g, r); }
void ref_new_direction(const double* in3, double g, MCG59* r, double* out3) {
    PhotonState p;
    memset(&p, 0, sizeof(p));
    p.direction.x = in3[0]; p.direction.y = in3[1]; p.direction.z = in3[2];
    double3 d = GetNewPhotonDirection(&p, g, r);
    out3[0] = d.x; out3[1] = d.y; out3[2] = d.z;
}
double ref_transmit_cos(double ni, double nt, double ci) { return ComputeTransmitCosine(ni, nt, ci); }
double ref_fresnel(double ni, double nt, double ci, double ct) { return ComputeFrenselReflectance(ni, nt, ci, ct); }
double ref_critical_cos(LayerInfo* layers, int cur, int next) { return GetCriticalCos(layers, cur, next); }
int ref_find_layer(InputInfo* in, int surf, int cur) { return FindIntersectionLayer(in, surf, cur); }
double ref_step_size(double mua, double mus, MCG59* r) {
    LayerInfo layers[2];
    memset(layers, 0, sizeof(layers));
    layers[1].absorptionCoefficient = mua;
    layers[1].scatteringCoefficient = mus;
    InputInfo in;
    memset(&in, 0, sizeof(in));
    in.layerInfo = layers;
    PhotonState p;
    memset(&p, 0, sizeof(p));
    p.layerId = 1;
    ComputeStepSizeInTissue(&p, &in, r);
    return p.step;
}
double ref_drop(double w, double mua, double mus, double* dw) {
    LayerInfo layers[2];
    memset(layers, 0, sizeof(layers));
    layers[1].absorptionCoefficient = mua;
    layers[1].scatteringCoefficient = mus;
    InputInfo in;
    memset(&in, 0, sizeof(in));
    in.layerInfo = layers;
    double cell = 0.0;
    OutputInfo out;
    memset(&out, 0, sizeof(out));
    out.absorption = &cell;
    PhotonState p;
    memset(&p, 0, sizeof(p));
    p.layerId = 1;
    p.weight = w;
    ComputeDroppedWeightOfPhoton(&p, &in, &out, 0);
    *dw = cell;
    return p.weight;
}
double ref_area_index(const double* p3, Area* a) {
    double3 p; p.x = p3[0]; p.y = p3[1]; p.z = p3[2];
    return (double)GetAreaIndex(p, a);
}
double ref_triangle(const double* o, const double* d, const double* a, const double* b, const double* c) {
    double3 O, Dd, A, B, C;
    O.x = o[0]; O.y = o[1]; O.z = o[2];
    Dd.x = d[0]; Dd.y = d[1]; Dd.z = d[2];
    A.x = a[0]; A.y = a[1]; A.z = a[2];
    B.x = b[0]; B.y = b[1]; B.z = b[2];
    C.x = c[0]; C.y = c[1]; C.z = c[2];
    return GetTriangleIntersectionDistance(O, Dd, A, B, C);
}
void ref_reflect(const double* i, const double* n, double* out) {
    double3 I, N; I.x = i[0]; I.y = i[1]; I.z = i[2]; N.x = n[0]; N.y = n[1]; N.z = n[2];
    double3 r = ReflectVector(I, N);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void ref_refract(double ni, double nt, const double* i, const double* n, double* out) {
    double3 I, N; I.x = i[0]; I.y = i[1]; I.z = i[2]; N.x = n[0]; N.y = n[1]; N.z = n[2];
    double3 r = RefractVector(ni, nt, I, N);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
int ref_detector_id(InputInfo* in, const double* pos, const double* dir, const unsigned char* visited) {
    PhotonState p;
    memset(&p, 0, sizeof(p));
    p.position.x = pos[0]; p.position.y = pos[1]; p.position.z = pos[2];
    p.direction.x = dir[0]; p.direction.y = dir[1]; p.direction.z = dir[2];
    for (int j = 0; j < MAX_LAYERS; ++j) p.visitedLayers[j] = visited[j] != 0;
    return GetDetectorId(&p, in);
}
/* BVH nearest hit of the reference (the caller prebuilt in->bvhTree). */
int ref_bvh_intersection(InputInfo* in, const double* o, const double* d, double step, int bounded,
                         double* dist, int* surf, double* normal) {
    double3 O, Dd;
    O.x = o[0]; O.y = o[1]; O.z = o[2];
    Dd.x = d[0]; Dd.y = d[1]; Dd.z = d[2];
    IntersectionInfo h = bounded ? ComputeBVHIntersection(O, Dd, step, in->bvhTree, in->surface)
                                 : ComputeBVHIntersectionWithoutStep(O, Dd, in->bvhTree, in->surface);
    *dist = h.distance;
    *surf = h.isFindIntersection ? h.surfaceId : -1;
    if (h.isFindIntersection) { normal[0] = h.normal.x; normal[1] = h.normal.y; normal[2] = h.normal.z; }
    return h.isFindIntersection;
}

/* Offsets of the reference structs' fields, in the order xmc_layout_offsets uses. */
int ref_layout_offsets(int64_t* o, int max_count) {
    int64_t v[] = {
        (int64_t)sizeof(double3), (int64_t)sizeof(int3), (int64_t)sizeof(byte3),
        (int64_t)sizeof(Area), (int64_t)offsetof(Area, length), (int64_t)offsetof(Area, partitionNumber),
        (int64_t)sizeof(Surface), (int64_t)offsetof(Surface, numberOfVertices), (int64_t)offsetof(Surface, triangles),
        (int64_t)offsetof(Surface, numberOfTriangles),
        (int64_t)sizeof(BVHNode), (int64_t)offsetof(BVHNode, rightNode), (int64_t)offsetof(BVHNode, leftNode),
        (int64_t)offsetof(BVHNode, offset), (int64_t)offsetof(BVHNode, numOfTriangles),
        (int64_t)sizeof(BVHTree), (int64_t)offsetof(BVHTree, numOfNodes), (int64_t)offsetof(BVHTree, root),
        (int64_t)offsetof(BVHTree, triangles), (int64_t)offsetof(BVHTree, numOfTriangles),
        (int64_t)sizeof(Triangle),
        (int64_t)sizeof(TimeInfo), (int64_t)offsetof(TimeInfo, numberOfPhotons), (int64_t)offsetof(TimeInfo, weight),
        (int64_t)offsetof(TimeInfo, targetWeight),
        (int64_t)sizeof(CubeDetector), (int64_t)offsetof(CubeDetector, length), (int64_t)offsetof(CubeDetector, filterLayers),
        (int64_t)offsetof(CubeDetector, targetAngle),
        (int64_t)sizeof(RingDetector), (int64_t)offsetof(RingDetector, smallRadius), (int64_t)offsetof(RingDetector, bigRadius),
        (int64_t)offsetof(RingDetector, filterLayers), (int64_t)offsetof(RingDetector, targetAngle),
        (int64_t)sizeof(DetectorInfo), (int64_t)offsetof(DetectorInfo, trajectory), (int64_t)offsetof(DetectorInfo, trajectorySize),
        (int64_t)offsetof(DetectorInfo, timeScale), (int64_t)offsetof(DetectorInfo, timeScaleSize),
        (int64_t)offsetof(DetectorInfo, targetWeight), (int64_t)offsetof(DetectorInfo, weight),
        (int64_t)sizeof(WeightIntegralTable), (int64_t)offsetof(WeightIntegralTable, numberOfElements),
        (int64_t)offsetof(WeightIntegralTable, elements),
        (int64_t)sizeof(LayerInfo), (int64_t)offsetof(LayerInfo, absorptionCoefficient),
        (int64_t)offsetof(LayerInfo, scatteringCoefficient), (int64_t)offsetof(LayerInfo, anisotropy),
        (int64_t)offsetof(LayerInfo, surfaceId), (int64_t)offsetof(LayerInfo, numberOfSurfaces),
        (int64_t)sizeof(InputInfo), (int64_t)offsetof(InputInfo, area), (int64_t)offsetof(InputInfo, layerInfo),
        (int64_t)offsetof(InputInfo, numberOfLayers), (int64_t)offsetof(InputInfo, surface),
        (int64_t)offsetof(InputInfo, numberOfSurfaces), (int64_t)offsetof(InputInfo, cubeDetector),
        (int64_t)offsetof(InputInfo, numberOfCubeDetectors), (int64_t)offsetof(InputInfo, ringDetector),
        (int64_t)offsetof(InputInfo, numberOfRingDetectors), (int64_t)offsetof(InputInfo, minWeight),
        (int64_t)offsetof(InputInfo, bvhTree), (int64_t)offsetof(InputInfo, timeStart), (int64_t)offsetof(InputInfo, timeFinish),
        (int64_t)offsetof(InputInfo, timeScaleSize), (int64_t)offsetof(InputInfo, startPosition),
        (int64_t)offsetof(InputInfo, startDirection), (int64_t)offsetof(InputInfo, useBiasing),
        (int64_t)offsetof(InputInfo, weightIntegralPrecision), (int64_t)offsetof(InputInfo, weightTablePrecision),
        (int64_t)offsetof(InputInfo, attractiveFactor), (int64_t)offsetof(InputInfo, weightTable),
        (int64_t)offsetof(InputInfo, numberOfWeightTables), (int64_t)offsetof(InputInfo, targetPoint),
        (int64_t)offsetof(InputInfo, targetRangeLayers),
        (int64_t)sizeof(OutputInfo), (int64_t)offsetof(OutputInfo, specularReflectance), (int64_t)offsetof(OutputInfo, absorption),
        (int64_t)offsetof(OutputInfo, scattering), (int64_t)offsetof(OutputInfo, gridSize),
        (int64_t)offsetof(OutputInfo, detectorInfo), (int64_t)offsetof(OutputInfo, numberOfDetectors),
        (int64_t)sizeof(MCG59), (int64_t)offsetof(MCG59, offset),
    };
    int n = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < max_count; ++i) o[i] = v[i];
    return n;
}

}  // extern "C"
