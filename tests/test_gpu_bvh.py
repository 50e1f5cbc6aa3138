"""The BVH topology built on the GPU (XMC_GPU_BVH: Morton-sorted centroids, Karras's parallel
hierarchy) against the host's binned-SAH tree: the nearest hit of every ray is the same triangle
set's minimum, so distances agree exactly whichever tree finds them; the walk with the GPU-built
tree keeps the exact energy ledger and matches the oracle within 3 sigma."""
import ctypes as C
import time

import numpy as np
import pytest

from oracle import bind as B
from xmcml_b200 import _lib, api, scenes

from helpers import ledger_identity_fx, oracle_opts_for, rich_planar, sum_var, zscores

pytestmark = pytest.mark.gpu

SCENES = {"heightfield": lambda: scenes.height_field_tissue(photons=10, grid=256),
          "ellipsoid": lambda: scenes.ellipsoid_target(photons=10, subdiv=5),
          "glass": lambda: rich_planar(10)}


def _rays(rng, n, lo, hi):
    o = rng.uniform(lo, hi, size=(n, 3))
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.ascontiguousarray(np.hstack([o, d]).astype(np.float32))


def _nearest(m, rays, flags, tmax=np.inf):
    lib = _lib.load()
    n = rays.shape[0]
    t = np.zeros(n, np.float32)
    s = np.zeros(n, np.int32)
    F, I = C.POINTER(C.c_float), C.POINTER(C.c_int)
    t0 = time.perf_counter()
    st = lib.xmc_debug_nearest(C.byref(m.info), n, rays.ctypes.data_as(F), C.c_float(0.0), C.c_float(tmax),
                               t.ctypes.data_as(F), s.ctypes.data_as(I), None, flags)
    assert st == 0, _lib.last_error()
    return t, s, time.perf_counter() - t0


@pytest.mark.parametrize("which", list(SCENES))
def test_gpu_built_tree_finds_the_same_hits(tmp_path, which):
    xml, surf = SCENES[which]().write(str(tmp_path), which)
    m = api.Model(xml, surf)
    rng = np.random.default_rng(5)
    rays = _rays(rng, 20000, (-6.0, -6.0, -0.5), (6.0, 6.0, 6.0))
    for tmax, grid in ((np.inf, 0), (0.3, 1)):
        th, sh, dt_h = _nearest(m, rays, grid, tmax)
        tg, sg, dt_g = _nearest(m, rays, grid | 2, tmax)
        hit = np.isfinite(th)
        print(f"{which} tmax {tmax}: {hit.mean():.3f} hit, host build+query {dt_h:.3f} s, GPU build+query {dt_g:.3f} s")
        assert hit.sum() > 1000 or tmax < np.inf
        assert np.array_equal(th, tg)
        assert np.mean(sh == sg) > 0.999


def test_gpu_bvh_build_time_large_mesh(tmp_path):
    """2 x 130,050-triangle height field: context creation with the GPU topology against the host SAH."""
    xml, surf = scenes.height_field_tissue(photons=10).write(str(tmp_path), "big")
    m = api.Model(xml, surf)
    times = {}
    for gpu in (False, True, False, True):
        t0 = time.perf_counter()
        t = api.Transport(m, roulette=True, gpu_bvh=gpu)
        times[gpu] = time.perf_counter() - t0
        led = t.run(20000, seed=3)
        assert ledger_identity_fx(led) == 20000 * 2 ** 31
        t.close()
    print(f"xmc_create: host SAH {times[False] * 1e3:.0f} ms, GPU topology {times[True] * 1e3:.0f} ms")
    assert times[True] < times[False]


def test_walk_with_gpu_bvh_matches_oracle(tmp_path):
    n = 100_000
    sc = scenes.height_field_tissue(photons=n, grid=96, time_bins=40)
    xml, surf = sc.write(str(tmp_path), "hfg")
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True, gpu_bvh=True)
    led = t.run(n, seed=9)
    tal = t.tallies()
    t.close()
    assert led["photons_launched"] == led["photons_terminated"] == n
    assert ledger_identity_fx(led) == n * 2 ** 31
    out = api.Output(m)
    _, dw2, _ = B.oracle_run(m.info, out.info, oracle_opts_for(True), seed=9, n=n)
    g = tal["det_weight"].astype(float) / 2 ** 31
    g2 = tal["det_weight2"].astype(float) / 2 ** 31
    o = out.detector_weights()
    z = zscores(g, o, sum_var(g, g2, n), sum_var(o, dw2, n))
    print("gpu bvh rings max|z|", np.abs(z).max())
    assert np.all(np.abs(z) < 3.0)
