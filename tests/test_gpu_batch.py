"""Batched planar instances on the GPU (xmc_batch_*), checked against the FP64 oracle per instance.

Instances are drawn from the layered sweep's distributions (per layer mua log-uniform [0.005, 1],
mus [5, 40], g [0.7, 0.95], n [1.33, 1.45]; L1 / L2 thickness [0.05, 0.3] / [0.5, 2] mm; L3 50 mm)
and every sampled instance is run by the oracle as its own planar model (the reference's input
format: planes, layers, 50 rings of 0.1 mm, 20 time bins of 50 ps) with roulette 1e-4 / 0.1 and no
Area kill. The batch and the oracle draw the same random numbers (Philox keyed by the instance
seed, photon ids 0..N-1), so the checks are the single-model ones: exact photon accounting and
energy ledger per instance, rings and time bins within 3 combined standard errors.
"""
import numpy as np
import pytest

from oracle import bind as B
from xmcml_b200 import api
from xmcml_b200 import batch as XB
from xmcml_b200 import structs as S

from helpers import WEIGHT_SCALE, oracle_opts_for, sum_var, zscores

pytestmark = pytest.mark.gpu

R_, T_ = 50, 20


def _ledger_identity(led, w0_fx_times_n, n):
    """specular + top + bottom + absorbed + roulette killed - gained + budget == N * 2^31, exactly."""
    L = {k: int(led[i]) for i, k in enumerate(S.BATCH_LEDGER_SLOTS)}
    spec = n * 2 ** 31 - w0_fx_times_n
    return spec + L["top_fx"] + L["bottom_fx"] + L["absorbed_fx"] + L["rkilled_fx"] - L["rgained_fx"] + L["budget_fx"]


def _w0_fx(inst, k):
    t = (inst.n_above[k] - inst.n[k, 0]) / (inst.n_above[k] + inst.n[k, 0])
    return int(round((1.0 - t * t) * 2 ** 31))


def _oracle(tmp_path, inst, k):
    sc = XB.to_scene(inst, k, n_rings=R_, n_time=T_)
    xml, surf = sc.write(str(tmp_path), f"inst{k}")
    m = api.Model(xml, surf)
    out = api.Output(m)
    n = int(inst.photons[k])
    led, dw2, tw2 = B.oracle_run(m.info, out.info, oracle_opts_for(True, False, float(inst.beam_radius[k])),
                                 seed=int(inst.seed[k]), n=n)
    return out.detector_weights(), dw2, out.time_weights(), tw2, led, out.detector_counts()


def test_batch_matches_oracle_per_instance(tmp_path):
    inst = XB.sample_instances(11, 12, budget=(20000, 40000), beam_radius=(0.0, 0.4))
    inst.beam_radius[:4] = 0.0  # pencil beam on some instances
    b = XB.Batch(n_rings=R_, n_time=T_, max_instances=64)
    res = b.run(inst)
    tal = b.tallies()
    for k in range(len(inst)):
        n = int(inst.photons[k])
        led = tal["ledger"][k]
        assert int(led[0]) == n == int(res["photons"][k])
        assert int(led[8] + led[9] + led[10] + led[11]) == n  # every photon ends in one cause
        assert _ledger_identity(led, _w0_fx(inst, k) * n, n) == n * 2 ** 31
        ow, dw2, otw, tw2, oled, ocnt = _oracle(tmp_path, inst, k)
        g = tal["ring"][k, :, 0].astype(float) / WEIGHT_SCALE
        g2 = tal["ring"][k, :, 2].astype(float) / WEIGHT_SCALE
        z = zscores(g, ow, sum_var(g, g2, n), sum_var(ow, dw2, n))
        zt = zscores(g.sum(), ow.sum(), sum_var(g.sum(), g2.sum(), n), sum_var(ow.sum(), dw2.sum(), n))
        gt = tal["ring_time"][k, :, :, 0].astype(float) / WEIGHT_SCALE
        gt2 = tal["ring_time"][k, :, :, 2].astype(float) / WEIGHT_SCALE
        ztb = zscores(gt, otw, sum_var(gt, gt2, n), sum_var(otw, tw2, n))
        print(f"instance {k}: n {n} R gpu {g.sum() / n:.4f} oracle {ow.sum() / n:.4f} rings max|z| "
              f"{np.max(np.abs(z)):.2f} total z {zt:.3f} time max|z| {np.max(np.abs(ztb)):.2f} "
              f"steps {res['steps'][k] / n:.0f} / {oled['steps'] / n:.0f}")
        assert np.all(np.abs(z) < 3.0)
        assert np.all(np.abs(ztb) < 3.0)
        assert abs(zt) < 1.0
        # FP64 reduction of the batch equals the fixed-point tallies / N
        assert np.allclose(res["ring"][k], g / n, rtol=1e-12, atol=0)
        assert np.allclose(res["ring_time"][k], gt / n, rtol=1e-12, atol=0)
        assert res["steps"][k] == pytest.approx(oled["steps"], rel=0.02)
        assert res["escaped_top"][k] == pytest.approx(oled["escaped_top"] / n, abs=0.01)
    b.close()


def test_instance_independent_of_batch_composition():
    """An instance's integer tallies are the same alone, at another position and beside others."""
    inst = XB.sample_instances(5, 6, budget=(3000, 30000))
    b = XB.Batch(n_rings=R_, n_time=T_, max_instances=16)
    b.run(inst)
    full = b.tallies()
    for k in (0, 3, 5):
        b.run(inst.subset([k]))
        one = b.tallies()
        assert np.array_equal(one["ring"][0], full["ring"][k])
        assert np.array_equal(one["ring_time"][0], full["ring_time"][k])
        assert np.array_equal(one["ledger"][0], full["ledger"][k])
    perm = [5, 2, 0, 4, 1, 3]
    b.run(inst.subset(perm))
    p = b.tallies()
    for i, k in enumerate(perm):
        assert np.array_equal(p["ring_time"][i], full["ring_time"][k])
        assert np.array_equal(p["ledger"][i], full["ledger"][k])
    b.close()


def test_bit_identical_across_launch_shapes_and_graph():
    inst = XB.sample_instances(9, 10, budget=(2000, 20000))
    ref = None
    for use_graph in (True, False):
        b = XB.Batch(n_rings=R_, n_time=T_, max_instances=16, use_graph=use_graph)
        for bs, ch, sch in [(256, 64, 1), (128, 32, 0), (256, 256, 0), (64, 1, 1)]:
            b.set_tuning(block_size=bs, photons_per_chunk=ch, tally_scheme=sch)
            for rep in range(2):  # replays of the same graph
                res = b.run(inst)
                t = b.tallies()
                cur = (t["ring"].copy(), t["ring_time"].copy(), t["ledger"].copy(), res["ring_time"].copy())
                if ref is None:
                    ref = cur
                for a, r in zip(cur, ref):
                    assert np.array_equal(a, r)
        b.close()


def test_uneven_and_zero_budgets():
    inst = XB.sample_instances(21, 7, budget=(1000, 50000))
    inst.photons[[0, 3, 6]] = 0
    inst.photons[1] = 1
    b = XB.Batch(n_rings=R_, n_time=T_, max_instances=8)
    res = b.run(inst)
    t = b.tallies()
    for k in range(len(inst)):
        n = int(inst.photons[k])
        assert int(t["ledger"][k][0]) == n
        assert _ledger_identity(t["ledger"][k], _w0_fx(inst, k) * n, n) == n * 2 ** 31
        if n == 0:
            assert not t["ring"][k].any() and not t["ring_time"][k].any()
            assert not res["ring"][k].any()
    res0 = b.run(inst.subset([]))
    assert res0["ring"].shape == (0, R_)
    b.close()


def test_autotune_picks_a_shape_that_reproduces():
    inst = XB.sample_instances(2, 16, budget=(5000, 20000))
    b = XB.Batch(n_rings=R_, n_time=T_, max_instances=16)
    b.set_tuning(256, 64, 1)
    b.run(inst)
    before = b.tallies()
    best = b.autotune(inst, photons_cap=4000)
    assert best["block_size"] in (64, 128, 256) and best["photons_per_chunk"] in (32, 64, 128, 256)
    assert best["tally_scheme"] in (0, 1) and best["ms"] > 0 and best["blocks_per_sm"] >= 1
    assert b.tuning == best
    b.run(inst)
    after = b.tallies()
    for key in before:
        assert np.array_equal(before[key], after[key])
    b.close()


def test_step_budget_reported():
    inst = XB.sample_instances(4, 3, budget=(500, 500))
    b = XB.Batch(n_rings=R_, n_time=T_, max_instances=4, max_steps_per_photon=20)
    res = b.run(inst, allow_budget=True)
    assert res["status"] == S.XMC_ERR_BUDGET
    t = b.tallies()
    for k in range(3):
        assert int(t["ledger"][k][11]) > 0  # n_budget
        assert _ledger_identity(t["ledger"][k], _w0_fx(inst, k) * 500, 500) == 500 * 2 ** 31
    b.close()
