"""ctypes mirrors of the reference's data structures and of this library's option/ledger structs.

Field order, types and sizes follow include/xmcml_b200.h, which restates
base/xmcml/xmcml/mcml_types.h, mcml_intersection.h, mcml_kernel_types.h and mcml_mcg59.h of the
reference (see the header for line citations).
"""
from __future__ import annotations

import ctypes as C

MAX_LAYERS = 8
MAX_TRAJECTORY_SIZE = 20480


class double3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class int3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


class Area(C.Structure):
    _fields_ = [("corner", double3), ("length", double3), ("partitionNumber", int3)]


class Surface(C.Structure):
    _fields_ = [("vertices", C.POINTER(double3)), ("numberOfVertices", C.c_int),
                ("triangles", C.POINTER(int3)), ("numberOfTriangles", C.c_int)]


class AABB(C.Structure):
    _fields_ = [("Ver1", double3), ("Ver2", double3)]


class BVHNode(C.Structure):
    _fields_ = [("Box", AABB), ("rightNode", C.c_int), ("leftNode", C.c_int), ("offset", C.c_int),
                ("numOfTriangles", C.c_int)]


class Triangle(C.Structure):
    _fields_ = [("surfId", C.c_int), ("trIndex", C.c_int)]


class BVHTree(C.Structure):
    _fields_ = [("nodes", C.POINTER(BVHNode)), ("numOfNodes", C.c_int), ("root", C.c_int),
                ("triangles", C.POINTER(Triangle)), ("numOfTriangles", C.c_int)]


class TimeInfo(C.Structure):
    _fields_ = [("timeStart", C.c_double), ("timeFinish", C.c_double), ("numberOfPhotons", C.c_uint64),
                ("weight", C.c_double), ("targetWeight", C.c_double)]


class CubeDetector(C.Structure):
    _fields_ = [("center", double3), ("length", double3), ("filterLayers", C.c_bool * MAX_LAYERS),
                ("targetAngle", C.c_double)]


class RingDetector(C.Structure):
    _fields_ = [("center", double3), ("smallRadius", C.c_double), ("bigRadius", C.c_double),
                ("filterLayers", C.c_bool * MAX_LAYERS), ("targetAngle", C.c_double)]


class DetectorInfo(C.Structure):
    _fields_ = [("numberOfPhotons", C.c_uint64), ("trajectory", C.POINTER(C.c_uint64)),
                ("trajectorySize", C.c_int), ("timeScale", C.POINTER(TimeInfo)), ("timeScaleSize", C.c_int),
                ("targetWeight", C.c_double), ("weight", C.c_double)]


class WeightIntegralTable(C.Structure):
    _fields_ = [("anisotropy", C.c_double), ("numberOfElements", C.c_int), ("elements", C.POINTER(C.c_double))]


class LayerInfo(C.Structure):
    _fields_ = [("refractiveIndex", C.c_double), ("absorptionCoefficient", C.c_double),
                ("scatteringCoefficient", C.c_double), ("anisotropy", C.c_double),
                ("surfaceId", C.POINTER(C.c_int)), ("numberOfSurfaces", C.c_int)]


class InputInfo(C.Structure):
    _fields_ = [("numberOfPhotons", C.c_uint64), ("area", C.POINTER(Area)), ("layerInfo", C.POINTER(LayerInfo)),
                ("numberOfLayers", C.c_int), ("surface", C.POINTER(Surface)), ("numberOfSurfaces", C.c_int),
                ("cubeDetector", C.POINTER(CubeDetector)), ("numberOfCubeDetectors", C.c_int),
                ("ringDetector", C.POINTER(RingDetector)), ("numberOfRingDetectors", C.c_int),
                ("minWeight", C.c_double), ("bvhTree", C.POINTER(BVHTree)), ("timeStart", C.c_double),
                ("timeFinish", C.c_double), ("timeScaleSize", C.c_int), ("startPosition", double3),
                ("startDirection", double3), ("useBiasing", C.c_ubyte), ("weightIntegralPrecision", C.c_uint),
                ("weightTablePrecision", C.c_uint), ("attractiveFactor", C.c_double),
                ("weightTable", C.POINTER(WeightIntegralTable)), ("numberOfWeightTables", C.c_int),
                ("targetPoint", double3), ("targetRangeLayers", C.c_ubyte * MAX_LAYERS)]


class OutputInfo(C.Structure):
    _fields_ = [("numberOfPhotons", C.c_uint64), ("specularReflectance", C.c_double),
                ("absorption", C.POINTER(C.c_double)), ("scattering", C.POINTER(C.c_double)),
                ("gridSize", C.c_int), ("detectorInfo", C.POINTER(DetectorInfo)), ("numberOfDetectors", C.c_int)]


class MCG59(C.Structure):
    _fields_ = [("value", C.c_uint64), ("offset", C.c_uint64)]


# ----------------------------------------------------------------------------- library structs

XMC_OK = 0
XMC_ERR_INVALID_INPUT = 1
XMC_ERR_RANGE = 2
XMC_ERR_DEVICE = 3
XMC_ERR_BUDGET = 4
XMC_ERR_CANCELLED = 5
XMC_ERR_IO = 6
XMC_ERR_UNSUPPORTED = 7

XMC_ROULETTE = 1 << 0
XMC_NO_AREA_KILL = 1 << 1
XMC_SCATTERING_MAP = 1 << 2
XMC_DETECTOR_TRAJ = 1 << 3
XMC_LARGE_GRID = 1 << 4
XMC_GPU_BVH = 1 << 5
XMC_LANE_QUERIES = 1 << 6


class XmcOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("flags", C.c_uint32), ("roulette_chance", C.c_double),
                ("beam_radius", C.c_double), ("max_steps_per_photon", C.c_uint64), ("device", C.c_int32),
                ("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("photons_per_chunk", C.c_int32),
                ("smem_nodes", C.c_int32), ("trajectory_log", C.c_int32), ("query_batch", C.c_int32),
                ("grid_cell_tris", C.c_int32), ("reserved", C.c_int32 * 4)]


_LEDGER_COUNTS = ["photons_launched", "photons_terminated", "steps", "n_escaped_top", "n_escaped_bottom",
                  "n_area", "n_cut", "n_roulette", "n_glass", "n_budget", "n_invalid", "n_detected",
                  "n_fp64_retests", "n_node_visits", "n_triangle_tests", "n_replay_mismatch"]
LEDGER_TERMS = ["specular", "absorbed", "absorbed_outside", "escaped_top", "escaped_bottom", "lost_area",
                "lost_cut", "lost_glass", "lost_budget", "lost_invalid", "roulette_killed", "roulette_gained"]


class XmcLedger(C.Structure):
    _fields_ = ([(n, C.c_uint64) for n in _LEDGER_COUNTS]
                + [(n + "_fx", C.c_uint64) for n in LEDGER_TERMS]
                + [(n, C.c_double) for n in LEDGER_TERMS]
                + [("kernel_ms", C.c_double), ("total_ms", C.c_double), ("h2d_bytes", C.c_uint64),
                   ("d2h_bytes", C.c_uint64), ("absorbed_target_fx", C.c_uint64), ("absorbed_target", C.c_double),
                   ("bias_gained_fx", C.c_uint64), ("bias_lost_fx", C.c_uint64), ("bias_gained", C.c_double),
                   ("bias_lost", C.c_double), ("n_trajectory_replayed", C.c_uint64),
                   ("n_plane_crossings", C.c_uint64)])

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


# ----------------------------------------------------------------------------- batched instances

XMC_BATCH_MAX_LAYERS = 6
XMC_BATCH_LEDGER = 16
BATCH_LEDGER_SLOTS = ["launched", "steps", "top_fx", "bottom_fx", "absorbed_fx", "rkilled_fx", "rgained_fx",
                      "budget_fx", "n_top", "n_bottom", "n_roulette", "n_budget", "n_detected"]


class BatchSpec(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("n_layers", C.c_int32), ("n_rings", C.c_int32), ("n_time", C.c_int32),
                ("ring_width", C.c_double), ("time_start", C.c_double), ("time_finish", C.c_double),
                ("ring_angle", C.c_double), ("min_weight", C.c_double), ("roulette_chance", C.c_double),
                ("max_steps_per_photon", C.c_uint64), ("max_instances", C.c_int32), ("use_graph", C.c_int32),
                ("device", C.c_int32), ("reserved", C.c_int32 * 7)]


_L6 = C.c_double * XMC_BATCH_MAX_LAYERS


class BatchInstance(C.Structure):
    _fields_ = [("mua", _L6), ("mus", _L6), ("g", _L6), ("n", _L6), ("thickness", _L6), ("n_above", C.c_double),
                ("n_below", C.c_double), ("beam_radius", C.c_double), ("photons", C.c_uint64), ("seed", C.c_uint64)]


class BatchTuning(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("photons_per_chunk", C.c_int32),
                ("tally_scheme", C.c_int32), ("ms", C.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchResult(C.Structure):
    _fields_ = ([(n, C.c_uint64) for n in ["photons", "steps", "n_detected", "n_top", "n_bottom", "n_roulette",
                                           "n_budget"]]
                + [(n, C.c_double) for n in ["specular", "escaped_top", "escaped_bottom", "absorbed",
                                             "roulette_killed", "roulette_gained", "lost_budget"]])


# ----------------------------------------------------------------------------- surrogate network

class MlpSpec(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("n_in", C.c_int32), ("hidden", C.c_int32), ("n_hidden", C.c_int32),
                ("n_out", C.c_int32), ("max_rows", C.c_int32), ("device", C.c_int32), ("forward_kernel", C.c_int32),
                ("reserved", C.c_int32 * 8)]
