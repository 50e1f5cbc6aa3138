"""Train the surrogate on batched Monte Carlo tallies and judge it against high-photon Monte Carlo.

    python -m xmcml_b200.surrogate_study --train 20000 --train-photons 1000000 --test 200 \\
        --test-photons 10000000 --steps 30000 --out result.json

1. Samples `train` + `test` instances of the layered sweep (per layer mua log-uniform [0.005, 1],
   mus [5, 40], g [0.7, 0.95], n [1.33, 1.45]; L1 / L2 thickness [0.05, 0.3] / [0.5, 2] mm; beam
   radius uniform [0, 0.5] mm) and runs them through the batched kernel: 50 rings of 0.1 mm x 20
   time bins of 50 ps, roulette 1e-4 / 0.1.
2. Trains an ensemble of MLPs (15 -> 256 x 4 SiLU -> 1000) on log10 reflectance with Adam on the
   tensor-core kernels.
3. Reports, on the held-out instances, the median relative reflectance error over the cells whose
   reference is known to 1 % (relative standard error from the squared-weight tally), the share of
   queries the gate sends to the network, and the network's evals/s next to the Monte Carlo's.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import batch as XB
from . import surrogate as SG


def run_batched(b: XB.Batch, inst: XB.Instances, chunk: int):
    rt, w2, ms = [], [], 0.0
    for i in range(0, len(inst), chunk):
        sub = inst.subset(np.arange(i, min(i + chunk, len(inst))))
        out = b.run(sub)
        tal = b.tallies()
        rt.append(out["ring_time"])
        w2.append(tal["ring_time"][:, :, :, 2].astype(np.float64) / 2 ** 31)
        ms += out["kernel_ms"]
    return np.concatenate(rt), np.concatenate(w2), ms


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--train", type=int, default=20000)
    p.add_argument("--train-photons", type=float, default=1e6)
    p.add_argument("--test", type=int, default=200)
    p.add_argument("--test-photons", type=float, default=1e7)
    p.add_argument("--members", type=int, default=4)
    p.add_argument("--steps", type=int, default=30000)
    p.add_argument("--batch", type=int, default=4096)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--floor", type=float, default=1e-7)
    p.add_argument("--gate", type=float, default=0.05)
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--unweighted", action="store_true", help="plain (unweighted) mean squared error")
    p.add_argument("--out", default="")
    a = p.parse_args(argv)

    chunk = 4096
    b = XB.Batch(n_rings=50, ring_width=0.1, n_time=20, time_finish=1000 * XB.C_MM_PER_PS, max_instances=chunk,
                 device=a.device)
    train = XB.sample_instances(a.seed, a.train, budget=(a.train_photons, a.train_photons), beam_radius=(0.0, 0.5))
    test = XB.sample_instances(a.seed + 1, a.test, budget=(a.test_photons, a.test_photons), beam_radius=(0.0, 0.5))
    tune = b.autotune(train.subset(np.arange(min(256, a.train))), photons_cap=20000)

    t0 = time.perf_counter()
    rt_tr, _, ms_tr = run_batched(b, train, chunk)
    t_gen = time.perf_counter() - t0
    rt_te, w2_te, ms_te = run_batched(b, test, chunk)

    sur = SG.Surrogate(n_in=15, n_out=1000, members=a.members, max_rows=65536, device=a.device, floor=a.floor,
                       gate=a.gate)
    t0 = time.perf_counter()
    curves = sur.fit(train.features(), SG.reflectance_targets(rt_tr, a.floor), steps=a.steps, batch=a.batch, lr=a.lr,
                     seed=a.seed, weighted=not a.unweighted)
    t_fit = time.perf_counter() - t0
    pred = sur.predict(test.features())
    err = SG.relative_error(pred["log10_r"], rt_te, w2_te, test.photons, floor=a.floor, max_ref_rse=0.01)
    per_inst = np.nanmedian(err, axis=1)
    # time-integrated ring reflectance: sum over the time bins
    ring_pred = (10.0 ** pred["log10_r"] - a.floor).reshape(len(test), 50, 20).sum(2)
    ring_ref = rt_te.reshape(len(test), 50, 20).sum(2)
    ring_w2 = w2_te.reshape(len(test), 50, 20).sum(2)
    ring_err = SG.relative_error(np.log10(ring_pred + a.floor), ring_ref, ring_w2, test.photons, floor=a.floor,
                                 max_ref_rse=0.01)

    m0 = sur.members[0]
    m0.forward(np.zeros((65536, 15), np.float32))
    ms_fwd = m0.forward_timed(65536, reps=50)
    evals = 65536 / (ms_fwd / 1e3) / a.members
    mc_rate = float(test.photons.sum()) / (ms_te / 1e3)
    res = {
        "weighted_loss": not a.unweighted, "floor": a.floor, "train_instances": a.train, "train_photons": a.train_photons, "test_instances": a.test,
        "test_photons": a.test_photons, "members": a.members, "steps": a.steps, "batch": a.batch,
        "autotune": tune,
        "mc_train_photons_per_s": float(train.photons.sum()) / (ms_tr / 1e3), "mc_train_wall_s": t_gen,
        "mc_test_photons_per_s": mc_rate,
        "fit_wall_s": t_fit, "fit_device_ms": sur.train_ms,
        "final_loss": [float(c[-100:].mean()) for c in curves],
        "median_rel_err_cells": float(np.nanmedian(err)),
        "p90_rel_err_cells": float(np.nanpercentile(err, 90)),
        "judged_cells_fraction": float(np.isfinite(err).mean()),
        "median_rel_err_rings": float(np.nanmedian(ring_err)),
        "median_of_instance_medians": float(np.nanmedian(per_inst)),
        "gate_pass_fraction": float(pred["use_network"].mean()),
        "median_rel_err_cells_gated": float(np.nanmedian(err[pred["use_network"]])) if pred["use_network"].any() else None,
        "evals_per_s_ensemble": evals, "forward_ms_65536_rows_one_member": ms_fwd,
        "mc_evals_per_s_1e7": mc_rate / 1e7, "speedup_vs_mc_1e7": evals / (mc_rate / 1e7),
    }
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    sur.close()
    b.close()
    return res


if __name__ == "__main__":
    main()
