"""The drop-in boundary without a GPU: the C-ABI library loads and exports every entry point of
include/xmcml_b200.h, its structs have the reference's layout, the reference-format I/O (XML model,
.surface, .mcml.out) matches the reference's own parser and writer, and invalid input is rejected
with status codes."""
import ctypes as C
import os
import re
import struct

import numpy as np
import pytest

from oracle import bind as B
from xmcml_b200 import _lib, api, scenes
from xmcml_b200 import structs as S

from helpers import rich_planar

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "xmcml_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\**\s+\**\s*(xmc_[A-Za-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_header_function():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(_lib.EXPORTS) <= set(names)


def test_version_and_defaults():
    lib = _lib.load()
    assert lib.xmc_version() >= 100
    o = S.XmcOptions()
    lib.xmc_default_options(C.byref(o))
    assert o.struct_size == C.sizeof(S.XmcOptions)
    assert o.roulette_chance == 0.1 and o.max_steps_per_photon == 10_000_000 and o.photons_per_chunk == 32


def _ctypes_offsets():
    def off(cls, f):
        return getattr(cls, f).offset
    sz = C.sizeof
    return [sz(S.double3), sz(S.int3), 3,
            sz(S.Area), off(S.Area, "length"), off(S.Area, "partitionNumber"),
            sz(S.Surface), off(S.Surface, "numberOfVertices"), off(S.Surface, "triangles"), off(S.Surface, "numberOfTriangles"),
            sz(S.BVHNode), off(S.BVHNode, "rightNode"), off(S.BVHNode, "leftNode"), off(S.BVHNode, "offset"),
            off(S.BVHNode, "numOfTriangles"),
            sz(S.BVHTree), off(S.BVHTree, "numOfNodes"), off(S.BVHTree, "root"), off(S.BVHTree, "triangles"),
            off(S.BVHTree, "numOfTriangles"), sz(S.Triangle),
            sz(S.TimeInfo), off(S.TimeInfo, "numberOfPhotons"), off(S.TimeInfo, "weight"), off(S.TimeInfo, "targetWeight"),
            sz(S.CubeDetector), off(S.CubeDetector, "length"), off(S.CubeDetector, "filterLayers"), off(S.CubeDetector, "targetAngle"),
            sz(S.RingDetector), off(S.RingDetector, "smallRadius"), off(S.RingDetector, "bigRadius"),
            off(S.RingDetector, "filterLayers"), off(S.RingDetector, "targetAngle"),
            sz(S.DetectorInfo), off(S.DetectorInfo, "trajectory"), off(S.DetectorInfo, "trajectorySize"),
            off(S.DetectorInfo, "timeScale"), off(S.DetectorInfo, "timeScaleSize"), off(S.DetectorInfo, "targetWeight"),
            off(S.DetectorInfo, "weight"),
            sz(S.WeightIntegralTable), off(S.WeightIntegralTable, "numberOfElements"), off(S.WeightIntegralTable, "elements"),
            sz(S.LayerInfo), off(S.LayerInfo, "absorptionCoefficient"), off(S.LayerInfo, "scatteringCoefficient"),
            off(S.LayerInfo, "anisotropy"), off(S.LayerInfo, "surfaceId"), off(S.LayerInfo, "numberOfSurfaces"),
            sz(S.InputInfo)] + [off(S.InputInfo, f) for f in [
                "area", "layerInfo", "numberOfLayers", "surface", "numberOfSurfaces", "cubeDetector",
                "numberOfCubeDetectors", "ringDetector", "numberOfRingDetectors", "minWeight", "bvhTree", "timeStart",
                "timeFinish", "timeScaleSize", "startPosition", "startDirection", "useBiasing", "weightIntegralPrecision",
                "weightTablePrecision", "attractiveFactor", "weightTable", "numberOfWeightTables", "targetPoint",
                "targetRangeLayers"]] + [
            sz(S.OutputInfo)] + [off(S.OutputInfo, f) for f in [
                "specularReflectance", "absorption", "scattering", "gridSize", "detectorInfo", "numberOfDetectors"]] + [
            sz(S.MCG59), off(S.MCG59, "offset")]


def test_struct_layouts_match_reference_headers():
    lib = _lib.load()
    mine = (C.c_int64 * 200)()
    n = lib.xmc_layout_offsets(mine, 200)
    assert list(mine[:n]) == _ctypes_offsets()
    if B.ref_available():
        ref = (C.c_int64 * 200)()
        m = B.ref().ref_layout_offsets(ref, 200)
        assert m == n and list(ref[:m]) == list(mine[:n])


def test_specular_reflectance_entry_point():
    lib = _lib.load()
    lay = (S.LayerInfo * 3)()
    lay[0].refractiveIndex, lay[1].refractiveIndex, lay[2].refractiveIndex = 1.0, 2.0, 3.0
    assert lib.xmc_specular_reflectance(lay) == pytest.approx(1.0 / 7.0, abs=1e-12)  # glass double reflection


def test_host_philox_matches_oracle():
    lib = _lib.load()
    rng = np.random.default_rng(5)
    for _ in range(50):
        ctr = (C.c_uint32 * 4)(*rng.integers(0, 2 ** 32, 4, dtype=np.uint64).tolist())
        key = (C.c_uint32 * 2)(*rng.integers(0, 2 ** 32, 2, dtype=np.uint64).tolist())
        a, b = (C.c_uint32 * 4)(), (C.c_uint32 * 4)()
        lib.xmc_philox4x32_10(ctr, key, a)
        B.oracle().oracle_philox4x32_10(ctr, key, b)
        assert list(a) == list(b)


# ------------------------------------------------------------------------------ reference-format I/O

def _fields(info: S.InputInfo):
    """Comparable dump of an InputInfo (everything the walk reads)."""
    a = info.area.contents
    d = {"photons": info.numberOfPhotons, "minWeight": info.minWeight, "time": (info.timeStart, info.timeFinish, info.timeScaleSize),
         "start": (info.startPosition.x, info.startPosition.y, info.startPosition.z),
         "dir": (info.startDirection.x, info.startDirection.y, info.startDirection.z),
         "area": (a.corner.x, a.corner.y, a.corner.z, a.length.x, a.length.y, a.length.z, a.partitionNumber.x,
                  a.partitionNumber.y, a.partitionNumber.z),
         "target": list(info.targetRangeLayers), "biasing": info.useBiasing, "nsurf": info.numberOfSurfaces}
    d["layers"] = [(L.refractiveIndex, L.absorptionCoefficient, L.scatteringCoefficient, L.anisotropy,
                    [L.surfaceId[j] for j in range(L.numberOfSurfaces)])
                   for L in (info.layerInfo[i] for i in range(info.numberOfLayers))]
    d["cubes"] = [(c.center.x, c.center.y, c.center.z, c.length.x, c.length.y, c.length.z, list(c.filterLayers), c.targetAngle)
                  for c in (info.cubeDetector[i] for i in range(info.numberOfCubeDetectors))]
    d["rings"] = [(r.center.x, r.center.y, r.center.z, r.smallRadius, r.bigRadius, list(r.filterLayers), r.targetAngle)
                  for r in (info.ringDetector[i] for i in range(info.numberOfRingDetectors))]
    d["surfaces"] = []
    for s in range(info.numberOfSurfaces):
        S_ = info.surface[s]
        v = np.ctypeslib.as_array(C.cast(S_.vertices, C.POINTER(C.c_double)), shape=(S_.numberOfVertices * 3,)).copy()
        t = np.ctypeslib.as_array(C.cast(S_.triangles, C.POINTER(C.c_int)), shape=(S_.numberOfTriangles * 3,)).copy()
        d["surfaces"].append((v.tobytes(), t.tobytes()))
    return d


@pytest.mark.skipif(not B.ref_available(), reason="reference build oracle/_ref missing")
@pytest.mark.parametrize("which", ["rich", "heightfield", "ellipsoid"])
def test_parser_matches_reference_parser(tmp_path, which):
    sc = {"rich": lambda: rich_planar(100),
          "heightfield": lambda: scenes.height_field_tissue(photons=123, grid=16),
          "ellipsoid": lambda: scenes.ellipsoid_target(photons=77, subdiv=2)}[which]()
    xml, surf = sc.write(str(tmp_path), which)
    mine = api.Model(xml, surf)
    ref = B.ref_load_model(xml, surf)
    assert _fields(mine.info) == _fields(ref)


def test_detectors_reordered_by_filter_count(tmp_path):
    """parser.cpp:59-60,488,498-511: detectors are stored in a multimap keyed by their number of
    filter layers, so a ring with one filter layer comes before one with none (all 8)."""
    sc = rich_planar(10)
    xml, surf = sc.write(str(tmp_path), "order")
    m = api.Model(xml, surf)
    counts = [sum(m.info.ringDetector[i].filterLayers) for i in range(m.info.numberOfRingDetectors)]
    assert counts == sorted(counts)
    assert (m.info.ringDetector[0].smallRadius, m.info.ringDetector[1].smallRadius) == (0.3, 2.0)


@pytest.mark.skipif(not B.ref_available(), reason="reference build oracle/_ref missing")
def test_writer_matches_reference_writer_bytes(tmp_path):
    sc = rich_planar(10)
    xml, surf = sc.write(str(tmp_path), "w")
    m = api.Model(xml, surf)
    out = api.Output(m)
    rng = np.random.default_rng(0)
    out.info.specularReflectance = 0.0370
    out.absorption[:] = rng.random(out.info.gridSize)
    np.ctypeslib.as_array(out.info.scattering, shape=(out.info.gridSize,))[:] = rng.random(out.info.gridSize)
    for d in range(out.info.numberOfDetectors):
        D = out.info.detectorInfo[d]
        D.weight, D.targetWeight, D.numberOfPhotons = rng.random(), rng.random(), int(rng.integers(0, 1000))
        D.trajectory[int(rng.integers(0, out.info.gridSize))] = 7
        for j in range(D.timeScaleSize):
            D.timeScale[j].weight, D.timeScale[j].targetWeight = rng.random(), rng.random()
            D.timeScale[j].numberOfPhotons = int(rng.integers(0, 50))
    p1, p2 = str(tmp_path / "mine.mcml.out"), str(tmp_path / "ref.mcml.out")
    out.write(p1)
    assert B.ref().ref_write_output(C.byref(m.info), C.byref(out.info), p2.encode())
    assert open(p1, "rb").read() == open(p2, "rb").read()


def test_init_output_matches_reference_layout(tmp_path):
    sc = rich_planar(10)
    xml, surf = sc.write(str(tmp_path), "io")
    m = api.Model(xml, surf)
    out = api.Output(m)
    assert out.info.gridSize == 100 * 100 * 100 and out.info.numberOfDetectors == 7
    ts = out.info.detectorInfo[0].timeScale
    T = out.info.detectorInfo[0].timeScaleSize
    assert T == 12
    step = (30.0 - 1.0) / 12
    for j in range(T - 1):
        assert ts[j].timeStart == 1.0 + j * step and ts[j].timeFinish == ts[j].timeStart + step
    assert ts[T - 1].timeFinish == 30.0 and out.absorption.sum() == 0


def test_surface_file_errors(tmp_path):
    sc = scenes.planar(photons=5)
    xml, surf = sc.write(str(tmp_path), "bad")
    data = open(surf, "rb").read()
    lib = _lib.load()
    # truncated file
    open(surf, "wb").write(data[:-7])
    info = S.InputInfo()
    assert lib.xmc_parse_input_file(xml.encode(), C.byref(info))
    assert not lib.xmc_parse_surface_file(surf.encode(), C.byref(info))
    assert "truncated" in _lib.last_error()
    lib.xmc_free_input(C.byref(info))
    # wrong section id
    open(surf, "wb").write(struct.pack("<I", 0x0200) + data[4:])
    info = S.InputInfo()
    assert lib.xmc_parse_input_file(xml.encode(), C.byref(info))
    assert not lib.xmc_parse_surface_file(surf.encode(), C.byref(info))
    lib.xmc_free_input(C.byref(info))
    # missing files
    with pytest.raises(_lib.XmcError):
        api.Model(str(tmp_path / "nope.xml"), surf)


def test_xml_errors(tmp_path):
    sc = scenes.planar(photons=5)
    xml, surf = sc.write(str(tmp_path), "x")
    text = open(xml).read()
    bad = tmp_path / "bad.xml"
    bad.write_text(text.replace("<NumberOfLayers>4</NumberOfLayers>", "<NumberOfLayers>3</NumberOfLayers>"))
    with pytest.raises(_lib.XmcError, match="number of layers invalid"):
        api.Model(str(bad), surf)
    bad.write_text(text.replace("</Input>", ""))
    with pytest.raises(_lib.XmcError, match="missing"):
        api.Model(str(bad), surf)


def test_create_rejects_invalid_input_before_touching_the_device(tmp_path):
    lib = _lib.load()
    ctx = C.c_void_p()
    assert lib.xmc_create(None, None, C.byref(ctx)) == S.XMC_ERR_INVALID_INPUT
    sc = scenes.planar(photons=5, area_partitions=(300, 10, 10))
    xml, surf = sc.write(str(tmp_path), "big")
    m = api.Model(xml, surf)
    assert lib.xmc_create(C.byref(m.info), None, C.byref(ctx)) == S.XMC_ERR_RANGE
    assert "256" in _lib.last_error()
    sc = scenes.planar(photons=5)
    xml, surf = sc.write(str(tmp_path), "bias")
    m = api.Model(xml, surf)
    m.info.useBiasing = 1
    m.info.attractiveFactor = -1.0
    assert lib.xmc_create(C.byref(m.info), None, C.byref(ctx)) == S.XMC_ERR_INVALID_INPUT
    m.info.attractiveFactor = 1.0
    # caller tables without the anisotropy of a tissue layer (GetWeightTableIndex would find none)
    tab = (S.WeightIntegralTable * 1)()
    elems = (C.c_double * 3)(1.0, 1.0, 1.0)
    tab[0].anisotropy, tab[0].numberOfElements, tab[0].elements = 0.123, 3, elems
    m.info.weightTable, m.info.numberOfWeightTables = C.cast(tab, C.POINTER(S.WeightIntegralTable)), 1
    assert lib.xmc_create(C.byref(m.info), None, C.byref(ctx)) == S.XMC_ERR_INVALID_INPUT
    assert "weight table" in _lib.last_error()
    m.info.weightTable, m.info.numberOfWeightTables = None, 0
    m.info.useBiasing = 0
    m.info.numberOfLayers = 9
    assert lib.xmc_create(C.byref(m.info), None, C.byref(ctx)) == S.XMC_ERR_RANGE
    m.info.numberOfLayers = 4
    for bad in (-2, 65537):  # crossing-log entries per thread: -1 (no log), 0 (default) .. 65536
        o = api.options(trajectories=True, trajectory_log=bad)
        assert lib.xmc_create(C.byref(m.info), C.byref(o), C.byref(ctx)) == S.XMC_ERR_RANGE
        assert "trajectory_log" in _lib.last_error()
    m.info.surface[0].triangles[0].y = 99
    assert lib.xmc_create(C.byref(m.info), None, C.byref(ctx)) == S.XMC_ERR_INVALID_INPUT
    assert "vertex index" in _lib.last_error()


def test_no_cpu_fallback_without_gpu(tmp_path):
    """Without a CUDA device the library reports a device error; it never computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    sc = scenes.planar(photons=5)
    xml, surf = sc.write(str(tmp_path), "nogpu")
    m = api.Model(xml, surf)
    with pytest.raises(_lib.XmcError) as e:
        api.Transport(m)
    assert e.value.status == S.XMC_ERR_DEVICE


@pytest.mark.parametrize("grid", [16, 256])
def test_bad_vertex_index_is_reported_before_the_gpu(tmp_path, grid):
    """xmc_create checks every triangle's vertex indices while it gathers the mesh (on several host
    threads for the 2 x 130,050-triangle mesh, on one for the small one) and reports the first bad
    triangle in input order, before any device work, so this runs without a GPU."""
    sc = scenes.height_field_tissue(photons=1000, grid=grid, time_bins=4)
    xml, surf = sc.write(str(tmp_path), "bad")
    m = api.Model(xml, surf)
    s1, s0 = m.info.surface[1], m.info.surface[0]
    late = s1.numberOfTriangles - 2
    s1.triangles[late].z = -1
    s1.triangles[5].y = s1.numberOfVertices + 3
    lib = _lib.load()
    o = S.XmcOptions()
    lib.xmc_default_options(C.byref(o))
    ctx = C.c_void_p()
    assert lib.xmc_create(C.byref(m.info), C.byref(o), C.byref(ctx)) == S.XMC_ERR_INVALID_INPUT
    assert _lib.last_error() == "surface 1 triangle 5: vertex index out of range"
    s1.triangles[5].y = 0
    assert lib.xmc_create(C.byref(m.info), C.byref(o), C.byref(ctx)) == S.XMC_ERR_INVALID_INPUT
    assert _lib.last_error() == f"surface 1 triangle {late}: vertex index out of range"
    assert s0.numberOfTriangles > 0
    m.close()
