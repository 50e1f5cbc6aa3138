"""Parity of the CUDA transport kernel (through the C-ABI) with the FP64 oracle.

Both draw the same random numbers (Philox4x32-10 keyed by seed and photon id, one block of four
uniforms per walk iteration), so most photons follow the same path in FP32 and in FP64 and the
tallies agree far inside the Monte Carlo error; the checks are
  * exact: launched == terminated == N, the per-cause counts add up, and the fixed-point energy
    ledger closes exactly (specular + absorbed + escaped + losses + roulette killed - gained == N);
  * statistical (3 sigma contract): every ring / time-bin / ledger total within 3 combined
    standard errors of the oracle (variances from per-photon sums of squares), and within 0.5
    combined standard errors for the totals (the paths are shared);
  * bit-reproducibility of the integer tallies across launch shapes.
"""
import ctypes as C
import os
import threading
import time

import numpy as np
import pytest

from oracle import bind as B
from xmcml_b200 import _lib, api, scenes
from xmcml_b200 import structs as S

from helpers import WEIGHT_SCALE, ledger_identity_fx, oracle_opts_for, rich_planar, sum_var, zscores

pytestmark = pytest.mark.gpu


def _run_pair(tmp_path, sc, n, seed=777, roulette=False, area_kill=True, beam_radius=0.0, stem="s", **kw):
    xml, surf = sc.write(str(tmp_path), stem)
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=roulette, area_kill=area_kill, beam_radius=beam_radius, **kw)
    led = t.run(n, seed=seed)
    tal = t.tallies()
    out = api.Output(m)
    oled, dw2, tw2 = B.oracle_run(m.info, out.info, oracle_opts_for(roulette, area_kill, beam_radius), seed=seed, n=n)
    t.close()
    return m, led, tal, out, oled, dw2, tw2


def _check_exact(led, n):
    assert led["photons_launched"] == n
    assert led["photons_terminated"] == n
    causes = ["n_escaped_top", "n_escaped_bottom", "n_area", "n_cut", "n_roulette", "n_glass", "n_budget", "n_invalid"]
    assert sum(led[c] for c in causes) == n
    assert ledger_identity_fx(led) == n * 2 ** 31


def _check_rings(tal, out, dw2, n, label):
    g = tal["det_weight"].astype(float) / WEIGHT_SCALE
    g2 = tal["det_weight2"].astype(float) / WEIGHT_SCALE
    o = out.detector_weights()
    z = zscores(g, o, sum_var(g, g2, n), sum_var(o, dw2, n))
    print(f"{label}: rings max|z| {np.max(np.abs(z)):.3f}, sum gpu {g.sum():.2f} oracle {o.sum():.2f}")
    assert np.all(np.abs(z) < 3.0)
    zt = zscores(g.sum(), o.sum(), sum_var(g.sum(), g2.sum(), n), sum_var(o.sum(), dw2.sum(), n))
    assert abs(zt) < 0.5
    # detected photon counts (binomial)
    c = tal["det_count"].astype(float)
    oc = out.detector_counts().astype(float)
    zc = zscores(c, oc, c * (1 - c / n), oc * (1 - oc / n))
    assert np.all(np.abs(zc) < 3.0)
    return z


def _check_ledger_terms(led, oled, n, label):
    """Totals of the energy ledger (each photon scores at most its start weight in one term)."""
    for k in ["escaped_top", "escaped_bottom", "lost_area", "lost_cut", "roulette_killed"]:
        g = led[k + "_fx"] / WEIGHT_SCALE
        o = oled[k]
        # binomial-type variance bound: a term of total T from n photons, each <= 1: var <= T
        z = (g - o) / np.sqrt(max(g + o, 1e-12))
        print(f"{label}: {k} gpu {g / n:.6f} oracle {o / n:.6f} z {z:.3f}")
        assert abs(z) < 3.0
    ga = led["absorbed_fx"] / WEIGHT_SCALE + led["absorbed_outside_fx"] / WEIGHT_SCALE
    oa = oled["absorbed"] + oled["absorbed_outside"]
    assert abs(ga - oa) / n < 5e-3


def test_c1_reference_semantics(tmp_path):
    """3-layer planar config: weight cut at minWeight, Area kill (the reference's own semantics)."""
    n = 200_000
    m, led, tal, out, oled, dw2, tw2 = _run_pair(tmp_path, scenes.planar(photons=n), n)
    _check_exact(led, n)
    assert oled["launched"] == oled["terminated"] == n
    _check_rings(tal, out, dw2, n, "c1")
    _check_ledger_terms(led, oled, n, "c1")
    # absorption per depth slab and per radial shell of voxels
    ga = tal["absorption"].astype(float).reshape(100, 100, 100) / WEIGHT_SCALE
    oa = out.absorption.reshape(100, 100, 100)
    for axis_sum in [(0, 1), (1, 2)]:
        gs, os_ = ga.sum(axis=axis_sum), oa.sum(axis=axis_sum)
        rel = np.abs(gs - os_) / np.maximum(os_, 1e-9)
        big = os_ > 0.02 * os_.max()
        print("c1 absorption profile max rel diff", rel[big].max())
        assert rel[big].max() < 0.02
    assert led["steps"] == pytest.approx(oled["steps"], rel=0.01)


def test_c1_roulette_no_area_kill(tmp_path):
    """Roulette semantics: roulette 1e-4 / 0.1 and no Area kill; R + T + A + losses == 1 exactly."""
    n = 100_000
    m, led, tal, out, oled, dw2, tw2 = _run_pair(tmp_path, scenes.planar(photons=n), n, roulette=True, area_kill=False)
    _check_exact(led, n)
    assert led["n_area"] == 0 and led["n_roulette"] > 0
    total = sum(led[k] for k in S.LEDGER_TERMS if k != "roulette_gained") - led["roulette_gained"]
    assert abs(total - 1.0) < 1e-9
    _check_rings(tal, out, dw2, n, "c1r")
    _check_ledger_terms(led, oled, n, "c1r")


def test_height_field_rings_and_time_bins(tmp_path):
    n = 100_000
    sc = scenes.height_field_tissue(photons=n, grid=96, time_bins=40)
    m, led, tal, out, oled, dw2, tw2 = _run_pair(tmp_path, sc, n, roulette=True)
    _check_exact(led, n)
    assert led["n_invalid"] == 0
    _check_rings(tal, out, dw2, n, "hf")
    _check_ledger_terms(led, oled, n, "hf")
    g = tal["time_weight"].astype(float) / WEIGHT_SCALE
    g2 = tal["time_weight2"].astype(float) / WEIGHT_SCALE
    o = out.time_weights()
    z = zscores(g, o, sum_var(g, g2, n), sum_var(o, tw2, n))
    print("hf time bins max|z|", np.max(np.abs(z)))
    assert np.all(np.abs(z) < 3.0)


def test_ellipsoid_target_region(tmp_path):
    """Large target-region scene (3 planar layers + a triangulated ellipsoid inside L3, absorption grid
    256x256x128, 100 rings x 200 time bins), at 20,480 triangles: rings, time bins, ledger and the
    weight absorbed inside the target."""
    n = 100_000
    sc = scenes.ellipsoid_target(photons=n, subdiv=5)
    m, led, tal, out, oled, dw2, tw2 = _run_pair(tmp_path, sc, n, roulette=True)
    _check_exact(led, n)
    assert led["n_invalid"] == 0
    _check_rings(tal, out, dw2, n, "ellipsoid")
    _check_ledger_terms(led, oled, n, "ellipsoid")
    g = led["absorbed_target_fx"] / WEIGHT_SCALE
    o = oled["absorbed_target"]
    print(f"ellipsoid: absorbed in target gpu {g / n:.6f} oracle {o / n:.6f}")
    assert o > 0.0 and abs(g - o) / np.sqrt(g + o) < 3.0
    g = tal["time_weight"].astype(float) / WEIGHT_SCALE
    z = zscores(g, out.time_weights(), sum_var(g, tal["time_weight2"].astype(float) / WEIGHT_SCALE, n),
                sum_var(out.time_weights(), tw2, n))
    assert np.all(np.abs(z) < 3.0)


def test_glass_cubes_filters_targets_beam(tmp_path):
    n = 100_000
    sc = rich_planar(n)
    m, led, tal, out, oled, dw2, tw2 = _run_pair(tmp_path, sc, n, roulette=True, beam_radius=0.3)
    _check_exact(led, n)
    _check_rings(tal, out, dw2, n, "rich")
    g = tal["det_target"].astype(float) / WEIGHT_SCALE
    o = out.detector_target_weights()
    gw = tal["det_weight"].astype(float) / WEIGHT_SCALE
    rel = np.abs(g - o) / np.maximum(np.abs(o), 1e-9)
    print("rich target weights", g, o)
    assert np.all((rel < 0.03) | (np.abs(g - o) < 0.01 * gw.sum() / len(gw)))
    g = tal["time_weight"].astype(float) / WEIGHT_SCALE
    z = zscores(g, out.time_weights(), sum_var(g, tal["time_weight2"].astype(float) / WEIGHT_SCALE, n),
                sum_var(out.time_weights(), tw2, n))
    assert np.all(np.abs(z) < 3.0)


def test_bit_reproducible_across_launch_shapes(tmp_path):
    n = 50_000
    xml, surf = scenes.height_field_tissue(photons=n, grid=64, time_bins=20).write(str(tmp_path), "rep")
    m = api.Model(xml, surf)
    res = []
    for kw in [dict(), dict(block_size=128, blocks_per_sm=1, photons_per_chunk=32), dict(block_size=512, smem_nodes=-1)]:
        t = api.Transport(m, roulette=True, **kw)
        led = t.run(n, seed=99)
        res.append((t.tallies(), led))
        t.close()
    for tal, led in res[1:]:
        for k in tal:
            assert np.array_equal(tal[k], res[0][0][k]), k
        for k in S.LEDGER_TERMS:
            assert led[k + "_fx"] == res[0][1][k + "_fx"]


@pytest.mark.parametrize("which", ["heightfield", "ellipsoid"])
def test_cooperative_and_lane_queries_are_identical(tmp_path, which):
    """The warp-cooperative grid query (default), the same with rays collected into rounds of 8 or 16
    (query_batch, lanes wait for their round), the lane-by-lane walk of the cells (XMC_LANE_QUERIES)
    and coarser xy grids (grid_cell_tris) keep the same nearest hit: every tally, both maps and every
    ledger term are identical bit for bit. With the same grid the counts of cells visited and
    triangles tested are the same too."""
    n = 40_000
    sc = (scenes.height_field_tissue(photons=n, grid=128, time_bins=20) if which == "heightfield"
          else scenes.ellipsoid_target(photons=n, subdiv=4))
    xml, surf = sc.write(str(tmp_path), "q" + which)
    m = api.Model(xml, surf)
    res = []
    for kw in (dict(), dict(lane_queries=True), dict(query_batch=8), dict(query_batch=16, grid_cell_tris=32),
               dict(lane_queries=True, grid_cell_tris=8), dict(query_batch=12, grid_cell_tris=16)):
        t = api.Transport(m, roulette=True, scattering=True, trajectories=which == "heightfield", **kw)
        led = t.run(n, seed=17)
        res.append((t.tallies(), t.maps(), led))
        t.close()
    ta, ma, la = res[0]
    for i, (tb, mb, lb) in enumerate(res[1:]):
        for k in ta:
            assert np.array_equal(ta[k], tb[k]), k
        for k in ma:
            assert np.array_equal(ma[k], mb[k]), k
        for k in S.LEDGER_TERMS:
            assert la[k + "_fx"] == lb[k + "_fx"], k
        same_grid = i < 2
        for k in ("steps", "n_plane_crossings", "n_detected") + (("n_node_visits", "n_triangle_tests") if same_grid else ()):
            assert la[k] == lb[k], k
    assert la["n_triangle_tests"] > 0


def test_split_runs_add_up(tmp_path):
    """Photons are identified by id: running [0, n) in two calls gives the same integer tallies."""
    n = 40_000
    xml, surf = scenes.planar(photons=n).write(str(tmp_path), "split")
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True)
    t.run(n, seed=5)
    whole = t.tallies()
    t.run(n // 4, seed=5, first_photon=0)
    a = t.tallies()
    t.run(n - n // 4, seed=5, first_photon=n // 4)
    b = t.tallies()
    for k in whole:
        assert np.array_equal(whole[k], a[k] + b[k]), k
    t.close()


@pytest.mark.parametrize("which,log", [("planar", 0), ("heightfield", 0), ("heightfield", 16), ("planar", -1)])
def test_scattering_and_trajectory_maps(tmp_path, which, log):
    """UpdatePhotonTrajectory / UpdateDetectorTrajectory (mcml_kernel.cpp:750-810): the scattering map
    (weight at every z-plane crossing through voxel centres) and, per detector, the crossing counts
    of the photons it detected. GPU: each thread's crossing log (log = 0: 4096 entries), counted at
    detection; a photon whose log overflows (log = 16: most of them) or every detected photon (log =
    -1: no log) is walked again by the replay pass."""
    n = 50_000
    sc = scenes.planar(photons=n) if which == "planar" else scenes.height_field_tissue(photons=n, grid=64, time_bins=10)
    xml, surf = sc.write(str(tmp_path), "maps_" + which)
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True, scattering=True, trajectories=True, trajectory_log=log)
    led = t.run(n, seed=31)
    maps = t.maps()
    tal = t.tallies()
    t.close()
    assert led["n_replay_mismatch"] == 0
    n_det = int(tal["det_count"].sum())
    if log == -1:
        assert led["n_trajectory_replayed"] == n_det
    elif log == 16:
        assert 0 < led["n_trajectory_replayed"] < n_det
    else:
        assert led["n_trajectory_replayed"] < 0.01 * n_det
    out = api.Output(m)
    opts = oracle_opts_for(roulette=True)
    opts.flags |= B.OFLAG_SCATTERING | B.OFLAG_TRAJECTORY
    B.oracle_run(m.info, out.info, opts, seed=31, n=n)
    G = out.info.gridSize
    osc = np.ctypeslib.as_array(out.info.scattering, shape=(G,))
    gsc = maps["scattering"].astype(float) / WEIGHT_SCALE
    shape = m.grid_shape
    gz, oz = gsc.reshape(shape).sum(axis=(0, 1)), osc.reshape(shape).sum(axis=(0, 1))
    big = oz > 0.02 * oz.max()
    print(which, "scattering total", gsc.sum() / n, osc.sum() / n, "max rel slab diff", np.max(np.abs(gz - oz)[big] / oz[big]))
    assert abs(gsc.sum() - osc.sum()) / osc.sum() < 5e-3
    assert np.max(np.abs(gz - oz)[big] / oz[big]) < 0.03
    D = m.n_detectors
    otr = np.stack([np.ctypeslib.as_array(out.info.detectorInfo[d].trajectory, shape=(G,)) for d in range(D)])
    gtr = maps["trajectory"][:D]
    gt, ot = gtr.sum(axis=1).astype(float), otr.sum(axis=1).astype(float)
    sel = ot > 1000
    print(which, "trajectory totals (first 5)", gt[:5], ot[:5])
    assert np.all(np.abs(gt - ot)[sel] / ot[sel] < 0.03)
    # the detectors that saw photons are the oracle's
    assert np.array_equal(tal["det_count"][:D] > 0, out.detector_counts() > 0)


def test_trajectory_log_equals_replay(tmp_path):
    """The crossing log and the replay pass count the same crossings of the same photons (same
    counter-RNG draws): the integer trajectory and scattering maps agree exactly whether every
    detected photon, some (a log that overflows) or almost none is replayed."""
    n = 40_000
    sc = scenes.height_field_tissue(photons=n, grid=64, time_bins=10)
    xml, surf = sc.write(str(tmp_path), "maps_log")
    m = api.Model(xml, surf)
    res = {}
    for log in (-1, 16, 0):
        t = api.Transport(m, roulette=True, scattering=True, trajectories=True, trajectory_log=log)
        led = t.run(n, seed=8)
        res[log] = (t.maps(), t.tallies()["det_count"], led["n_trajectory_replayed"])
        t.close()
    base_maps, base_det, _ = res[-1]
    assert res[16][2] > 0 and res[0][2] < res[16][2]
    for log in (16, 0):
        maps, det, _ = res[log]
        assert np.array_equal(det, base_det)
        assert np.array_equal(maps["scattering"], base_maps["scattering"])
        assert np.array_equal(maps["trajectory"], base_maps["trajectory"])


def test_launch_omp_shim_accumulates(tmp_path):
    n = 20_000
    xml, surf = scenes.planar(photons=n).write(str(tmp_path), "omp")
    m = api.Model(xml, surf)
    out = api.Output(m)
    rng = api.mcg59_init(777, 0, 1)
    v0 = rng.value
    api.launch_omp(m, out, rng, 8)
    w1 = out.detector_weights().sum()
    assert out.info.specularReflectance == pytest.approx(0.0277777777777, rel=1e-9)
    assert out.info.numberOfPhotons == 0  # left to the caller, as the reference's LaunchOMP does
    assert rng.value != v0
    api.launch_omp(m, out, rng, 8)
    w2 = out.detector_weights().sum()
    assert 1.8 * w1 < w2 < 2.2 * w1
    assert out.detector_counts().sum() > 0 and out.absorption.sum() > 0
    # LaunchOMP fills the scattering map and the detector trajectory maps too
    assert np.ctypeslib.as_array(out.info.scattering, shape=(out.info.gridSize,)).sum() > 0
    assert sum(np.ctypeslib.as_array(out.info.detectorInfo[d].trajectory, shape=(out.info.gridSize,)).sum()
               for d in range(out.info.numberOfDetectors)) > 0
    p = str(tmp_path / "r.mcml.out")
    out.write(p)
    assert os.path.getsize(p) > out.info.gridSize * 8


def test_device_philox_matches_host():
    lib = _lib.load()
    n = 1000
    dev = (C.c_uint32 * (4 * n))()
    _lib.check(lib.xmc_device_philox(0x123456789ABCDEF, 77, n, dev))
    host = (C.c_uint32 * 4)()
    for i in [0, 1, 17, 999]:
        ctr = (C.c_uint32 * 4)(77, 0, i, 0)
        key = (C.c_uint32 * 2)(0x89ABCDEF, 0x1234567)
        lib.xmc_philox4x32_10(ctr, key, host)
        assert list(host) == list(dev[4 * i:4 * i + 4])


def test_step_budget_terminates_and_reports(tmp_path):
    n = 10_000
    xml, surf = scenes.planar(photons=n).write(str(tmp_path), "budget")
    m = api.Model(xml, surf)
    t = api.Transport(m, max_steps=5)
    with pytest.raises(_lib.XmcError) as e:
        t.run(n)
    assert e.value.status == S.XMC_ERR_BUDGET
    led = t.run(n, allow_budget=True)
    assert led["n_budget"] > 0 and led["photons_terminated"] == n
    assert ledger_identity_fx(led) == n * 2 ** 31
    t.close()


def test_cancel_stops_a_run(tmp_path):
    xml, surf = scenes.planar(photons=1).write(str(tmp_path), "cancel")
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True, area_kill=False)
    n = 2_000_000_000
    result = {}

    def worker():
        try:
            result["led"] = t.run(n)
        except _lib.XmcError as e:
            result["err"] = e

    th = threading.Thread(target=worker)
    th.start()
    time.sleep(1.0)
    t.cancel()
    th.join(timeout=60)
    assert not th.is_alive()
    assert "err" in result and result["err"].status == S.XMC_ERR_CANCELLED
    t.close()


def test_zero_photons_and_no_detectors(tmp_path):
    sc = scenes.planar(photons=1, n_rings=0)
    xml, surf = sc.write(str(tmp_path), "zero")
    m = api.Model(xml, surf)
    t = api.Transport(m)
    led = t.run(0)
    assert led["photons_launched"] == 0 and ledger_identity_fx(led) == 0
    led = t.run(1000)
    assert led["photons_terminated"] == 1000 and led["n_detected"] == 0
    t.close()


def test_checkpoint_resume_bit_identical(tmp_path):
    """A run stopped after its first portion and resumed from the checkpoint file gives the same
    integer tallies and ledger as one uninterrupted run."""
    from xmcml_b200 import checkpoint as CK
    n = 60_000
    xml, surf = scenes.planar(photons=n).write(str(tmp_path), "ck")
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True)
    t.run(n, seed=31)
    whole = t.tallies()
    whole_led = t.run(n, seed=31)
    path = str(tmp_path / "run.ckpt")

    class Stop(Exception):
        pass

    def stop(st):
        if st.next_id >= 25_000:
            raise Stop()

    with pytest.raises(Stop):
        CK.run_portions(t, CK.RunState(31, n, 25_000), path, stop)
    st = CK.run_portions(t, CK.RunState.load(path), path)
    assert st.done
    for k, v in whole.items():
        assert np.array_equal(st.tallies[k], v), k
    for k in ("photons_launched", "steps", "absorbed_fx", "escaped_top_fx", "roulette_killed_fx", "roulette_gained_fx"):
        assert st.ledger[k] == whole_led[k], k
    t.close()


def _biased_scene(n, factor=1.0, target=(1, 0, 2)):
    sc = scenes.planar(photons=n, name="bias")
    sc.time_start, sc.time_finish, sc.time_bins = 0.0, 30.0, 10
    sc.bias_target, sc.bias_factor = target, factor
    sc.bias_integral_precision, sc.bias_table_precision = 12, 512
    return sc


def test_weight_integral_tables_on_gpu(tmp_path):
    """xmc_weight_integral_table (FP64 on the GPU) against the oracle's restatement of the reference's
    quadrature (itself pinned bit for bit), including a layer with g > 0.95 (4x integral precision)."""
    sc = _biased_scene(10, factor=1.7)
    sc.layers[2].g = 0.96
    xml, surf = sc.write(str(tmp_path), "wt")
    m = api.Model(xml, surf)
    _lib.check(_lib.load().xmc_weight_integral_table(C.byref(m.info), 0))
    o = S.InputInfo.from_buffer_copy(m.info)
    o.weightTable, o.numberOfWeightTables = None, 0
    B.oracle().oracle_weight_tables(C.byref(o))
    assert m.info.numberOfWeightTables == o.numberOfWeightTables == 3
    worst = 0.0
    for k in range(3):
        a, b = m.info.weightTable[k], o.weightTable[k]
        assert a.anisotropy == b.anisotropy and a.numberOfElements == b.numberOfElements == 513
        ga = np.ctypeslib.as_array(a.elements, shape=(513,))
        ob = np.ctypeslib.as_array(b.elements, shape=(513,))
        worst = max(worst, float(np.max(np.abs(ga - ob) / np.abs(ob))))
    print("weight tables max rel diff", worst)
    assert worst < 1e-11
    B.oracle().oracle_free_weight_tables(C.byref(o))


@pytest.mark.parametrize("factor", [1.0, 3.0])
def test_biasing_matches_oracle(tmp_path, factor):
    """<Biasing> on (attractive point, weight tables computed on the GPU): rings and time bins within
    3 sigma of the oracle, the fixed-point ledger (with the weight created and removed by the
    biasing factor) closes exactly, and weights above 1 (factor 3) do not overflow."""
    n = 60_000
    sc = _biased_scene(n, factor=factor)
    xml, surf = sc.write(str(tmp_path), f"b{int(factor)}")
    m = api.Model(xml, surf)
    _lib.check(_lib.load().xmc_weight_integral_table(C.byref(m.info), 0))
    t = api.Transport(m, roulette=True)
    led = t.run(n, seed=5)
    tal = t.tallies()
    out = api.Output(m)
    oled, dw2, tw2 = B.oracle_run(m.info, out.info, oracle_opts_for(True, True, 0.0), seed=5, n=n)
    t.close()
    _check_exact(led, n)
    assert led["bias_gained_fx"] > 0 and led["bias_lost_fx"] > 0
    print(f"bias x{factor}: gained {led['bias_gained']:.4f} / {oled['bias_gained'] / n:.4f}, "
          f"lost {led['bias_lost']:.4f} / {oled['bias_lost'] / n:.4f}")
    z = _check_rings(tal, out, dw2, n, f"bias{factor}")
    g = tal["time_weight"].astype(float) / WEIGHT_SCALE
    zt = zscores(g, out.time_weights(), sum_var(g, tal["time_weight2"].astype(float) / WEIGHT_SCALE, n),
                 sum_var(out.time_weights(), tw2, n))
    assert np.all(np.abs(zt) < 3.0)
    for k in ("bias_gained", "bias_lost"):
        assert led[k] == pytest.approx(oled[k] / n, rel=0.05)


def test_launch_keeps_context_only_for_unchanged_models(tmp_path):
    """xmc_launch_omp keeps the device image of the last model: a second call on the unchanged model
    repeats a fresh run bit for bit, and after a change of an optical property the result is the new
    model's (as a fresh context gives it), not the kept image's."""
    n = 20_000
    xml, surf = scenes.planar(photons=n).write(str(tmp_path), "cache")
    m = api.Model(xml, surf)

    def via_launch(key):
        out = api.Output(m)
        g = S.MCG59()
        g.value, g.offset = key, 1
        api.launch_omp(m, out, g, 0)
        return out.detector_weights(), out.absorption.copy()

    def fresh(key):
        out = api.Output(m)
        t = api.Transport(m, scattering=True, trajectories=True)
        t.run(n, seed=key, output=out)
        t.close()
        return out.detector_weights(), out.absorption.copy()

    _lib.check(_lib.load().xmc_launch_release())
    a1 = via_launch(99)
    a2 = via_launch(99)  # kept context
    assert np.array_equal(a1[0], a2[0]) and np.array_equal(a1[1], a2[1])
    f = fresh(99)
    assert np.array_equal(a1[0], f[0]) and np.array_equal(a1[1], f[1])
    m.info.layerInfo[1].scatteringCoefficient *= 1.5
    b = via_launch(99)
    fb = fresh(99)
    assert np.array_equal(b[0], fb[0]) and np.array_equal(b[1], fb[1])
    assert not np.array_equal(b[0], a1[0])
    _lib.check(_lib.load().xmc_launch_release())


@pytest.mark.parametrize("partitions", [(100, 100, 100), (40, 40, 40), (2, 2, 4)])
def test_output_maps_accumulate_the_device_maps_exactly(tmp_path, partitions):
    """xmc_run with an OutputInfo adds the run's maps into the caller's arrays (the trajectory maps read
    back as the list of their non-zero cells, or dense when that list would be larger, and added by
    host threads; 1e6 cells use several threads, 64,000 one): after two runs every detector's
    trajectory map is exactly the sum of the two runs' integer maps, and the scattering map their FP64
    value. The ledger's read-back bytes count 12 bytes per non-zero trajectory cell (8 per cell when the
    maps go dense) over a part that does not depend on the run. On the 16-cell grid about 80 % of the
    cells are non-zero (the reference's own LaunchOMP gives 81.5 % on this scene), so the maps go dense."""
    n = 30_000
    sc = scenes.height_field_tissue(photons=n, grid=64, time_bins=10, area_partitions=partitions)
    xml, surf = sc.write(str(tmp_path), "acc")
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True, scattering=True, trajectories=True)
    out = api.Output(m)
    G, D = out.info.gridSize, m.n_detectors
    traj_sum = np.zeros((D, G), dtype=np.uint64)
    scat_sum = np.zeros(G, dtype=np.float64)
    fixed = set()
    for seed in (3, 4):
        led = t.run(n, seed=seed, output=out)
        maps = t.maps()
        traj_sum += maps["trajectory"][:D]
        scat_sum += maps["scattering"].astype(np.float64) / WEIGHT_SCALE
        nz = int(np.count_nonzero(maps["trajectory"][:D]))
        assert 0 < nz <= D * G
        listed = 12 * nz if 12 * nz < 8 * G * D else 8 * G * D
        print(f"{G} cells x {D} maps: {nz / (D * G):.1%} non-zero, read back {'sparse' if listed < 8 * G * D else 'dense'}")
        fixed.add(int(led["d2h_bytes"]) - listed)
        if G == 16:
            assert listed == 8 * G * D  # the dense read-back
    t.close()
    assert len(fixed) == 1 and fixed.pop() > 8 * G
    got = np.stack([np.ctypeslib.as_array(out.info.detectorInfo[d].trajectory, shape=(G,)) for d in range(D)])
    assert traj_sum.sum() > 0
    assert np.array_equal(got, traj_sum)
    scat = np.ctypeslib.as_array(out.info.scattering, shape=(G,))
    assert np.allclose(scat, scat_sum, rtol=1e-12, atol=0.0)


def test_entry_points_keep_the_callers_device_and_launch_omp_follows_it(tmp_path):
    """Entry points that select a context's device restore the caller's current device on return, and
    xmc_launch_omp runs on the calling thread's current device: on device 1 its tallies equal a device-0
    run bit for bit, and switching back to device 0 rebuilds the kept context there. Needs 2 GPUs."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    n = 20_000
    xml, surf = scenes.planar(photons=n).write(str(tmp_path), "dev")
    m = api.Model(xml, surf)
    lib = _lib.load()

    def launch(dev):
        torch.cuda.set_device(dev)
        out = api.Output(m)
        g = S.MCG59()
        g.value, g.offset = 12345, 1
        api.launch_omp(m, out, g, 0)
        assert torch.cuda.current_device() == dev
        return out.detector_weights(), out.absorption.copy()

    _lib.check(lib.xmc_launch_release())
    a0 = launch(0)
    free1_before = torch.cuda.mem_get_info(1)[0]
    a1 = launch(1)
    assert torch.cuda.mem_get_info(1)[0] < free1_before  # the kept context now lives on device 1
    assert np.array_equal(a0[0], a1[0]) and np.array_equal(a0[1], a1[1])
    b0 = launch(0)
    assert np.array_equal(a0[0], b0[0]) and np.array_equal(a0[1], b0[1])
    # a context on device 1 used from device 0: every entry point leaves device 0 current
    torch.cuda.set_device(0)
    t = api.Transport(m, device=1)
    assert torch.cuda.current_device() == 0
    t.run(1000)
    t.tallies()
    assert torch.cuda.current_device() == 0
    t.close()
    assert torch.cuda.current_device() == 0
    _lib.check(lib.xmc_launch_release())


def test_autotune_picks_a_shape_with_identical_tallies(tmp_path):
    """xmc_autotune times the candidate launch shapes (block size, photons per warp claim, query
    scheme) on a sample and returns the fastest; a run with the tuned options gives the same tallies
    as the default shape, bit for bit."""
    n = 30_000
    xml, surf = scenes.height_field_tissue(photons=n, grid=96, time_bins=20).write(str(tmp_path), "tune")
    m = api.Model(xml, surf)
    best, ms = api.autotune(m, sample_photons=20_000, roulette=True)
    assert ms > 0 and best.block_size in (256, 512) and best.photons_per_chunk in (32, 64)
    assert best.query_batch in (1, 8, 12, 16) and best.grid_cell_tris in (2, 8, 16, 32)
    assert best.flags & S.XMC_ROULETTE
    res = []
    for opts in (api.options(roulette=True), best):
        t = api.Transport(m, opts)
        led = t.run(n, seed=3)
        res.append((t.tallies(), led))
        t.close()
    for k in res[0][0]:
        assert np.array_equal(res[0][0][k], res[1][0][k]), k
    for k in S.LEDGER_TERMS:
        assert res[0][1][k + "_fx"] == res[1][1][k + "_fx"]


def test_launch_omp_uses_the_options_set_for_it(tmp_path):
    """xmc_launch_set_options: the LaunchOMP replacement runs with a caller's launch shape (as
    xmc_autotune returns it) and gives the same OutputInfo as with the defaults, bit for bit; NULL
    restores the defaults."""
    n = 20_000
    xml, surf = scenes.height_field_tissue(photons=n, grid=64, time_bins=10).write(str(tmp_path), "setopt")
    m = api.Model(xml, surf)

    def via_launch():
        out = api.Output(m)
        g = S.MCG59()
        g.value, g.offset = 4242, 1
        api.launch_omp(m, out, g, 0)
        G = out.info.gridSize
        traj = np.stack([np.ctypeslib.as_array(out.info.detectorInfo[d].trajectory, shape=(G,)).copy()
                         for d in range(out.info.numberOfDetectors)])
        return out.detector_weights(), out.absorption.copy(), traj

    try:
        a = via_launch()
        api.launch_set_options(api.options(lane_queries=True, grid_cell_tris=32, block_size=256, photons_per_chunk=64))
        b = via_launch()
        api.launch_set_options(api.options(query_batch=16, grid_cell_tris=2))
        c = via_launch()
    finally:
        api.launch_set_options(None)
    for other in (b, c):
        for x, y in zip(a, other):
            assert np.array_equal(x, y)
    _lib.check(_lib.load().xmc_launch_release())
