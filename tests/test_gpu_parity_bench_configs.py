"""Parity at the benchmarked configurations, cell by cell.

The scenes are the ones bench.py times, at their full sizes: the 256 x 256 height-field tissue
(2 x 130,050 triangles, 50 rings x 200 time bins of 5 ps, 100^3 absorption grid), the ellipsoid
target scene (81,920 triangles, 256 x 256 x 128 grid, 100 rings x 200 time bins), the planar
3-layer stack at 1e6 photons and 32 instances of the batched sweep at their own (uneven) budgets,
scaled down by 50 so the FP64 oracle finishes in seconds. Photon counts are reduced where the
oracle would take minutes; the geometry, grids and tallies are not.

Every individual cell is tested, not sums over slabs or shells:
  * absorption-grid voxels, scattering-map cells and every detector's trajectory-map cells: the
    photons are split into B independent batches (photon-id ranges, or LaunchOMP calls with their
    own keys) on both sides, the variance of each cell's total comes from the spread of its batch
    values (batch means), and every cell that all batches of both sides scored must lie within 3
    combined standard errors of the oracle (reference: mcml_kernel.cpp:633-642 absorption += dw,
    :750-810 UpdatePhotonTrajectory / UpdateDetectorTrajectory);
  * every ring and every time bin (mcml_kernel.cpp:744-849), from the per-photon sums of squared
    weights both sides tally (or batch means for the LaunchOMP path, whose OutputInfo carries no
    squares);
  * detected-photon counts per ring (binomial), exact photon accounting and the fixed-point ledger.
The GPU and the oracle draw the same Philox numbers per photon, so most photons take the same path
in FP32 and FP64; the printed max |z| per tally family is therefore far below 3.
"""
import numpy as np
import pytest

from oracle import bind as B
from xmcml_b200 import api, scenes
from xmcml_b200 import batch as XB
from xmcml_b200 import structs as S

from helpers import (WEIGHT_SCALE, BatchStats, cell_zscores, ledger_identity_fx, oracle_opts_for, sum_var,
                     zscores)

pytestmark = pytest.mark.gpu

NB = 8  # independent batches per side for the per-cell variances


def _report(label, family, z, n_cells, n_scored):
    mz = float(np.max(np.abs(z))) if len(z) else 0.0
    print(f"{label}: {family}: {n_cells} cells tested ({n_scored} scored), max|z| {mz:.3f}")
    assert n_cells > 0, f"{label} {family}: no cell scored in every batch"
    assert np.all(np.abs(z) < 3.0), f"{label} {family}: max |z| {mz:.2f}"
    return mz


def _gpu_batches(t, n, seed, maps=False):
    nb = n // NB
    st = {k: BatchStats() for k in ("absorption", "scattering", "trajectory")}
    acc = None
    leds = []
    for b in range(NB):
        led = t.run(nb, seed=seed, first_photon=b * nb)
        assert led["photons_launched"] == nb and led["photons_terminated"] == nb
        assert ledger_identity_fx(led) == nb * 2 ** 31
        tal = t.tallies()
        st["absorption"].add(tal["absorption"].astype(np.float64) / WEIGHT_SCALE)
        if maps:
            mp = t.maps()
            st["scattering"].add(mp["scattering"].astype(np.float64) / WEIGHT_SCALE)
            st["trajectory"].add(mp["trajectory"][:t.n_dets])
        if acc is None:
            acc = {k: v.astype(np.float64) for k, v in tal.items() if k != "absorption"}
        else:
            for k in acc:
                acc[k] += tal[k]
        leds.append(led)
    return st, acc, leds, nb * NB


def _oracle_batches(m, n, seed, opts, maps=False):
    """The oracle over the same NB photon-id ranges, accumulated into one OutputInfo (allocating one
    per batch would zero gigabytes of trajectory maps each time); each batch's values are the
    differences of consecutive snapshots."""
    nb = n // NB
    st = {k: BatchStats() for k in ("absorption", "scattering", "trajectory")}
    dw2_sum = tw2_sum = None
    tgt = 0.0
    D = m.n_detectors
    out = api.Output(m)
    G = out.info.gridSize
    prev = None
    for b in range(NB):
        led, dw2, tw2 = B.oracle_run(m.info, out.info, opts, seed=seed, first=b * nb, n=nb)
        assert led["launched"] == led["terminated"] == nb
        cur = {"absorption": out.absorption.copy()}
        if maps:
            cur["scattering"] = np.ctypeslib.as_array(out.info.scattering, shape=(G,)).copy()
            cur["trajectory"] = np.stack([np.ctypeslib.as_array(out.info.detectorInfo[d].trajectory, shape=(G,))
                                          for d in range(D)])
        for k, v in cur.items():
            st[k].add(v - prev[k] if prev is not None else v)
        prev = cur
        dw2_sum = dw2 if dw2_sum is None else dw2_sum + dw2
        tw2_sum = tw2 if tw2_sum is None else tw2_sum + tw2
        tgt += led["absorbed_target"]
    res = {"det_weight": out.detector_weights(), "det_count": out.detector_counts().astype(np.float64),
           "time_weight": out.time_weights(), "dw2": dw2_sum, "tw2": tw2_sum, "absorbed_target": tgt}
    out.close()
    return st, res


def _rings_and_bins(label, acc, o, n):
    g = acc["det_weight"] / WEIGHT_SCALE
    g2 = acc["det_weight2"] / WEIGHT_SCALE
    z = zscores(g, o["det_weight"], sum_var(g, g2, n), sum_var(o["det_weight"], o["dw2"], n))
    _report(label, "rings", z, len(z), len(z))
    c, oc = acc["det_count"], o["det_count"]
    zc = zscores(c, oc, c * (1 - c / n), oc * (1 - oc / n))
    _report(label, "ring photon counts", zc, len(zc), len(zc))
    gt = acc["time_weight"] / WEIGHT_SCALE
    gt2 = acc["time_weight2"] / WEIGHT_SCALE
    zt = zscores(gt, o["time_weight"], sum_var(gt, gt2, n), sum_var(o["time_weight"], o["tw2"], n))
    scored = (gt > 0) | (o["time_weight"] > 0)
    _report(label, "time bins", zt[scored], int(scored.sum()), int(scored.sum()))


def test_height_field_full_mesh_cells(tmp_path):
    """The benchmarked 256 x 256 height-field scene (2 x 130,050 triangles + 2 planes, 50 rings x 200
    time bins of 5 ps, 100^3 grid) with the benchmark's roulette semantics."""
    n = 240_000
    sc = scenes.height_field_tissue(photons=n)
    assert sc.n_triangles == 2 * 130_050 + 4 and sc.time_bins == 200
    xml, surf = sc.write(str(tmp_path), "hf")
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True)
    g, acc, leds, n = _gpu_batches(t, n, seed=4242)
    t.close()
    o_st, o = _oracle_batches(m, n, 4242, oracle_opts_for(True, True, 0.0))
    assert sum(l["n_invalid"] for l in leds) == 0
    _rings_and_bins("hf", acc, o, n)
    _report("hf", "absorption voxels", *cell_zscores(g["absorption"], o_st["absorption"]))


def test_height_field_launch_omp_maps_cells(tmp_path):
    """The benchmark's end-to-end path: xmc_launch_omp (the LaunchOMP signature, reference semantics:
    weight cut, Area kill, scattering map and 50 trajectory maps) on the full 256 x 256 height field,
    called NB times into one OutputInfo, against the oracle run with the same keys (the MCG59 value
    of each call) and photon ids. Every accumulated tally is checked cell by cell, and the
    accumulated OutputInfo equals the sum of the per-call increments."""
    n = 200_000
    sc = scenes.height_field_tissue(photons=n)
    xml, surf = sc.write(str(tmp_path), "hfomp")
    m = api.Model(xml, surf)
    nb = n // NB
    m.info.numberOfPhotons = nb
    out = api.Output(m)
    G, D = out.info.gridSize, m.n_detectors
    rng = api.mcg59_init(31, 0, 1)
    keys = []
    g = {k: BatchStats() for k in ("absorption", "scattering", "trajectory", "rings", "counts", "time")}
    prev = None

    def snapshot():
        return {"absorption": out.absorption.copy(),
                "scattering": np.ctypeslib.as_array(out.info.scattering, shape=(G,)).copy(),
                "trajectory": np.stack([np.ctypeslib.as_array(out.info.detectorInfo[d].trajectory, shape=(G,)).copy()
                                        for d in range(D)]),
                "rings": out.detector_weights(), "counts": out.detector_counts().astype(np.float64),
                "time": out.time_weights()}

    for b in range(NB):
        keys.append(rng.value)
        api.launch_omp(m, out, rng, 0)
        cur = snapshot()
        for k in g:
            g[k].add(cur[k] - prev[k] if prev is not None else cur[k])
        prev = cur
    # the OutputInfo holds the sum of the calls
    assert np.array_equal(prev["trajectory"].astype(np.float64), g["trajectory"].total)
    assert out.info.specularReflectance == pytest.approx(0.0277777777777, rel=1e-9)

    opts = oracle_opts_for(False, True, 0.0)
    opts.flags |= B.OFLAG_SCATTERING | B.OFLAG_TRAJECTORY
    o = {k: BatchStats() for k in g}
    oo = api.Output(m)
    prev = None
    for key in keys:
        led, _, _ = B.oracle_run(m.info, oo.info, opts, seed=key, first=0, n=nb)
        assert led["launched"] == led["terminated"] == nb
        cur = {"absorption": oo.absorption.copy(),
               "scattering": np.ctypeslib.as_array(oo.info.scattering, shape=(G,)).copy(),
               "trajectory": np.stack([np.ctypeslib.as_array(oo.info.detectorInfo[d].trajectory, shape=(G,))
                                       for d in range(D)]),
               "rings": oo.detector_weights(), "counts": oo.detector_counts().astype(np.float64),
               "time": oo.time_weights()}
        for k in o:
            o[k].add(cur[k] - prev[k] if prev is not None else cur[k])
        prev = cur
    oo.close()
    for fam in ("rings", "counts", "time", "absorption", "scattering", "trajectory"):
        z, nc, ns = cell_zscores(g[fam], o[fam])
        _report("launch_omp hf", fam, z, nc, ns)
    out.close()


def test_ellipsoid_full_scene_cells(tmp_path):
    """The benchmarked target-region scene: 3 planar layers + the 81,920-triangle ellipsoid, 256 x 256 x
    128 grid over 20 x 20 x 10 mm, 100 rings x 200 time bins, target absorbed weight."""
    n = 120_000
    sc = scenes.ellipsoid_target(photons=n)
    assert sc.n_triangles - 8 == 81_920
    xml, surf = sc.write(str(tmp_path), "ell")
    m = api.Model(xml, surf)
    assert m.grid_shape == (256, 256, 128) and m.n_detectors == 100 and m.info.timeScaleSize == 200
    t = api.Transport(m, roulette=True)
    g, acc, leds, n = _gpu_batches(t, n, seed=99)
    t.close()
    o_st, o = _oracle_batches(m, n, 99, oracle_opts_for(True, True, 0.0))
    assert sum(l["n_invalid"] for l in leds) == 0
    _rings_and_bins("ellipsoid", acc, o, n)
    _report("ellipsoid", "absorption voxels", *cell_zscores(g["absorption"], o_st["absorption"]))
    gt = sum(l["absorbed_target_fx"] for l in leds) / WEIGHT_SCALE
    ot = o["absorbed_target"]
    print(f"ellipsoid: absorbed in target gpu {gt / n:.6f} oracle {ot / n:.6f}")
    assert ot > 0 and abs(gt - ot) / np.sqrt(gt + ot) < 3.0


def test_planar_1e6_cells(tmp_path):
    """The planar 3-layer stack at 1e6 photons (100^3 grid over 10 x 10 x 5 mm, 50 rings), roulette
    1e-4 / 0.1."""
    n = 1_000_000
    xml, surf = scenes.planar(photons=n).write(str(tmp_path), "c1")
    m = api.Model(xml, surf)
    t = api.Transport(m, roulette=True)
    g, acc, leds, n = _gpu_batches(t, n, seed=777)
    t.close()
    o_st, o = _oracle_batches(m, n, 777, oracle_opts_for(True, True, 0.0))
    _rings_and_bins("planar", acc, o, n)
    _report("planar", "absorption voxels", *cell_zscores(g["absorption"], o_st["absorption"]))


def test_batched_sweep_32_sampled_instances(tmp_path):
    """32 instances sampled (fixed seed) from the benchmark's 1024-instance sweep, each at its own
    budget from the sweep's log-uniform [1e5, 1e7] scaled by 1/50 (so [2e3, 2e5], still uneven), in
    one batched launch; each instance against its own oracle run: exact ledger, every ring and time
    bin within 3 sigma."""
    full = XB.sample_instances(2024, 1024, budget=(1e5, 1e7))
    pick = np.sort(np.random.default_rng(5).choice(1024, 32, replace=False))
    inst = full.subset(pick)
    inst.photons = np.maximum((inst.photons // 50).astype(np.uint64), 1)
    R, T = 50, 20
    b = XB.Batch(n_rings=R, n_time=T, max_instances=64)
    res = b.run(inst)
    tal = b.tallies()
    b.close()
    worst = {"rings": 0.0, "time": 0.0}
    for k in range(len(inst)):
        n = int(inst.photons[k])
        L = tal["ledger"][k]
        assert int(L[0]) == n and int(L[8] + L[9] + L[10] + L[11]) == n
        sc = XB.to_scene(inst, k, n_rings=R, n_time=T)
        xml, surf = sc.write(str(tmp_path), f"i{k}")
        m = api.Model(xml, surf)
        out = api.Output(m)
        oled, dw2, tw2 = B.oracle_run(m.info, out.info, oracle_opts_for(True, False, float(inst.beam_radius[k])),
                                      seed=int(inst.seed[k]), n=n)
        g = tal["ring"][k, :, 0].astype(float) / WEIGHT_SCALE
        g2 = tal["ring"][k, :, 2].astype(float) / WEIGHT_SCALE
        ow = out.detector_weights()
        z = zscores(g, ow, sum_var(g, g2, n), sum_var(ow, dw2, n))
        gt = tal["ring_time"][k, :, :, 0].astype(float) / WEIGHT_SCALE
        gt2 = tal["ring_time"][k, :, :, 2].astype(float) / WEIGHT_SCALE
        otw = out.time_weights()
        zt = zscores(gt, otw, sum_var(gt, gt2, n), sum_var(otw, tw2, n))
        worst["rings"] = max(worst["rings"], float(np.max(np.abs(z))))
        worst["time"] = max(worst["time"], float(np.max(np.abs(zt))))
        assert np.all(np.abs(z) < 3.0), (k, n, float(np.max(np.abs(z))))
        assert np.all(np.abs(zt) < 3.0), (k, n, float(np.max(np.abs(zt))))
        assert res["steps"][k] == pytest.approx(oled["steps"], rel=0.02)
        out.close()
    print(f"batched sweep, 32 instances ({int(inst.photons.min())}..{int(inst.photons.max())} photons): "
          f"rings max|z| {worst['rings']:.3f}, time bins max|z| {worst['time']:.3f}")
