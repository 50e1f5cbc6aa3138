"""Ray queries of the transport kernel (its device code compiled for the host through
xmc_debug_nearest) against the FP64 oracle's nearest-hit search and the reference's own BVH
traversal (ComputeBVHIntersection, mcml_intersection.cpp:354-466), on planar, height-field and
ellipsoid meshes, with the library's own SAH tree and with the reference's tree converted."""
import ctypes as C

import numpy as np
import pytest

from oracle import bind as B
from xmcml_b200 import _lib, api, scenes
from xmcml_b200 import structs as S

lib = _lib.load()

SCENES = {
    "planar": lambda: scenes.planar(photons=1),
    "heightfield": lambda: scenes.height_field_tissue(photons=1, grid=48),
    "ellipsoid": lambda: scenes.ellipsoid_target(photons=1, subdiv=3),
}


def rays(n, seed, lo=(-3, -3, -0.2), hi=(3, 3, 4)):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


def kernel_query(info, r, tmax, tmin=0.0, use_grid=1):
    n = r.shape[0]
    t = np.zeros(n, np.float32)
    s = np.zeros(n, np.int32)
    nr = np.zeros((n, 3), np.float32)
    pf = C.POINTER(C.c_float)
    _lib.check(lib.xmc_debug_nearest(C.byref(info), n, r.ctypes.data_as(pf), tmin, tmax, t.ctypes.data_as(pf),
                                     s.ctypes.data_as(C.POINTER(C.c_int)), nr.ctypes.data_as(pf), use_grid))
    return t, s, nr


def oracle_query(info, r, tmax, bounded=True):
    n = r.shape[0]
    q = np.ascontiguousarray(r, dtype=np.float64)
    dist = np.zeros(n)
    surf = np.zeros(n, np.int32)
    nrm = np.zeros((n, 3))
    pd = C.POINTER(C.c_double)
    B.oracle().oracle_kat_nearest_batch(C.byref(info), n, q.ctypes.data_as(pd), tmax, 1 if bounded else 0,
                                        dist.ctypes.data_as(pd), surf.ctypes.data_as(C.POINTER(C.c_int)),
                                        nrm.ctypes.data_as(pd))
    dist = np.where(surf >= 0, dist, np.inf)
    return dist, surf, nrm


def ref_query(info, r, tmax):
    out_t, out_s = [], []
    for q in r.astype(np.float64):
        o, d = (C.c_double * 3)(*q[:3]), (C.c_double * 3)(*q[3:])
        dist, surf, nrm = C.c_double(), C.c_int(), (C.c_double * 3)()
        hit = B.ref().ref_bvh_intersection(C.byref(info), o, d, tmax, 1, C.byref(dist), C.byref(surf), nrm)
        out_t.append(dist.value if hit else np.inf)
        out_s.append(surf.value if hit else -1)
    return np.array(out_t), np.array(out_s)


def agree(t1, s1, t2, s2, tol=2e-5):
    same_surf = s1 == s2
    both = (s1 >= 0) & (s2 >= 0)
    with np.errstate(invalid="ignore"):
        dt = np.where(both, np.abs(t1 - t2) <= tol * np.maximum(1.0, np.abs(t2)), True)
    return same_surf & dt


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("tmax", [0.05, 0.3, 5.0])
@pytest.mark.parametrize("use_grid", [1, 0])
def test_kernel_query_matches_oracle(tmp_path, name, tmax, use_grid):
    xml, surf = SCENES[name]().write(str(tmp_path), name)
    m = api.Model(xml, surf)
    r = rays(1500, 11 if tmax < 1 else 12)
    if tmax < 0.1:  # short steps near the surfaces, where the cell grid answers the query
        r[:, 2] = np.random.default_rng(3).uniform(-0.08, 0.2, len(r))
    t, s, nrm = kernel_query(m.info, r, tmax, use_grid=use_grid)
    ot, os_, on = oracle_query(m.info, r, tmax)
    ok = agree(t, s, ot, os_)
    assert ok.mean() >= 0.999, f"{(~ok).sum()} disagreements"
    assert (s >= 0).sum() > (50 if tmax > 0.1 else 10)
    hit = (s >= 0) & (os_ >= 0)
    # normals: same plane up to sign (the reference's GetPlaneNormal orientation is arbitrary)
    assert np.all(np.abs(np.abs(np.sum(nrm[hit] * on[hit], 1)) - 1) < 1e-4)


@pytest.mark.parametrize("tmax", [0.3, 5.0])
def test_queries_outside_the_cell_grid(tmp_path, tmax):
    """The cell grid covers the small triangles only (here the ellipsoid, 4 x 4 mm); the layer planes
    (+-100 mm) are tested from the large-triangle list, also for segments outside the grid."""
    xml, surf = scenes.ellipsoid_target(photons=1, subdiv=4).write(str(tmp_path), "e")
    m = api.Model(xml, surf)
    r = rays(1500, 31, lo=(-40, -40, -0.2), hi=(40, 40, 4))
    r[:500, 2] = np.random.default_rng(5).uniform(-0.08, 0.2, 500)
    t, s, _ = kernel_query(m.info, r, tmax, use_grid=1)
    ot, os_, _ = oracle_query(m.info, r, tmax)
    ok = agree(t, s, ot, os_)
    assert ok.mean() >= 0.999, f"{(~ok).sum()} disagreements"
    assert (os_ >= 0).sum() > 50


@pytest.mark.skipif(not B.ref_available(), reason="reference build oracle/_ref missing")
@pytest.mark.parametrize("name", list(SCENES))
def test_kernel_query_matches_reference_bvh_and_converted_tree(tmp_path, name):
    xml, surf = SCENES[name]().write(str(tmp_path), name)
    m = api.Model(xml, surf)
    rinfo = B.ref_load_model(xml, surf)
    B.ref().ref_generate_bvh(C.byref(rinfo))
    r = rays(1200, 21)
    rt, rs = ref_query(rinfo, r, 0.5)
    t_own, s_own, _ = kernel_query(m.info, r, 0.5)
    assert agree(t_own, s_own, rt, rs).mean() >= 0.999
    # the same query on the reference's own tree, converted node for node (input->bvhTree set)
    m.info.bvhTree = rinfo.bvhTree
    t_ref, s_ref, _ = kernel_query(m.info, r, 0.5)
    assert agree(t_ref, s_ref, rt, rs).mean() >= 0.999
    assert np.array_equal(s_ref, s_own)
    m.info.bvhTree = None


def test_min_distance_and_no_geometry(tmp_path):
    xml, surf = SCENES["planar"]().write(str(tmp_path), "p")
    m = api.Model(xml, surf)
    r = np.array([[0.0, 0.0, 0.05, 0.0, 0.0, 1.0]], np.float32)  # 0.05 mm above the z = 0.1 plane
    t, s, _ = kernel_query(m.info, r, 1.0)
    assert s[0] == 1 and abs(t[0] - 0.05) < 1e-6
    t, s, _ = kernel_query(m.info, r, 0.04)  # step shorter than the distance
    assert s[0] == -1
    t, s, _ = kernel_query(m.info, r, 2.0, tmin=0.06)  # nearest hit closer than tmin is skipped
    assert s[0] == 2 and abs(t[0] - 1.05) < 1e-5
    m.info.numberOfSurfaces = 0
    t, s, _ = kernel_query(m.info, r, 100.0)
    assert s[0] == -1
    m.info.numberOfSurfaces = 4
