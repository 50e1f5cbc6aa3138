"""Train the surrogate on batched Monte Carlo tallies and judge it against high-photon Monte Carlo.

    python -m xmcml_b200.surrogate_study --train 20000 --train-photons 1000000 --test 200 \\
        --test-photons 10000000 --steps 30000 --out result.json
    python -m xmcml_b200.surrogate_study --train-sizes 2000,5000,20000,50000 --test 1000 \\
        --save ensemble.npz --save-size 20000 --out curve.json

1. Samples `train` + `test` instances of the layered sweep (per layer mua log-uniform [0.005, 1],
   mus [5, 40], g [0.7, 0.95], n [1.33, 1.45]; L1 / L2 thickness [0.05, 0.3] / [0.5, 2] mm; beam
   radius uniform [0, 0.5] mm) and runs them through the batched kernel: 50 rings of 0.1 mm x 20
   time bins of 50 ps, roulette 1e-4 / 0.1.
2. Trains an ensemble of MLPs (15 -> 256 x 4 SiLU -> 1000) on log10 reflectance with Adam on the
   tensor-core kernels.
3. Reports, on the held-out instances, the median relative reflectance error over the cells whose
   reference is known to 1 % (relative standard error from the squared-weight tally) and its
   distribution, the share of queries the gate sends to the network, and the network's evals/s next
   to the Monte Carlo's; with several training-set sizes (nested subsets of one generated set), the
   error against the size. --save writes one trained ensemble (Surrogate.save).
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


def evaluate(sur: SG.Surrogate, test: XB.Instances, rt_te, w2_te, floor: float) -> dict:
    """Accuracy of the ensemble on held-out instances against their Monte Carlo tallies: per-cell
    relative error on the cells whose reference is known to 1 %, its distribution, the time-integrated
    rings, and the share of queries the gate lets through."""
    pred = sur.predict(test.features())
    err = SG.relative_error(pred["log10_r"], rt_te, w2_te, test.photons, floor=floor, max_ref_rse=0.01)
    per_inst = np.nanmedian(err, axis=1)
    ring_pred = (10.0 ** pred["log10_r"] - floor).reshape(len(test), 50, 20).sum(2)
    ring_ref = rt_te.reshape(len(test), 50, 20).sum(2)
    ring_w2 = w2_te.reshape(len(test), 50, 20).sum(2)
    ring_err = SG.relative_error(np.log10(ring_pred + floor), ring_ref, ring_w2, test.photons, floor=floor,
                                 max_ref_rse=0.01)
    e = err[np.isfinite(err)]
    pct = {f"p{q}": float(np.percentile(e, q)) for q in (10, 25, 50, 75, 90, 95, 99)}
    return {"median_rel_err_cells": float(np.nanmedian(err)), "p90_rel_err_cells": float(np.nanpercentile(err, 90)),
            "error_percentiles_cells": pct, "cells_within_2pct": float(np.mean(e <= 0.02)),
            "cells_within_5pct": float(np.mean(e <= 0.05)), "judged_cells": int(e.size),
            "judged_cells_fraction": float(np.isfinite(err).mean()),
            "median_rel_err_rings": float(np.nanmedian(ring_err)),
            "median_of_instance_medians": float(np.nanmedian(per_inst)),
            "gate_pass_fraction": float(pred["use_network"].mean()),
            "median_rel_err_cells_gated": float(np.nanmedian(err[pred["use_network"]])) if pred["use_network"].any() else None}


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--train", type=int, default=20000)
    p.add_argument("--train-sizes", default="", help="comma list of training-set sizes (nested subsets of the "
                                                     "largest); default: --train alone")
    p.add_argument("--train-photons", type=float, default=1e6)
    p.add_argument("--test", type=int, default=200)
    p.add_argument("--test-photons", type=float, default=1e7)
    p.add_argument("--members", type=int, default=4)
    p.add_argument("--steps", type=int, default=30000, help="Adam steps per member")
    p.add_argument("--batch", type=int, default=4096)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--floor", type=float, default=1e-7)
    p.add_argument("--gate", type=float, default=0.05)
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--unweighted", action="store_true", help="plain (unweighted) mean squared error")
    p.add_argument("--save", default="", help="write the ensemble of --save-size (default the largest) to this .npz "
                                              "(the package ships xmcml_b200/data/surrogate_ensemble.npz)")
    p.add_argument("--save-size", type=int, default=0)
    p.add_argument("--out", default="")
    a = p.parse_args(argv)

    sizes = sorted({int(v) for v in a.train_sizes.split(",") if v}) or [a.train]
    n_train = max(sizes)
    chunk = 4096
    b = XB.Batch(n_rings=50, ring_width=0.1, n_time=20, time_finish=1000 * XB.C_MM_PER_PS, max_instances=chunk,
                 device=a.device)
    train = XB.sample_instances(a.seed, n_train, budget=(a.train_photons, a.train_photons), beam_radius=(0.0, 0.5))
    test = XB.sample_instances(a.seed + 1, a.test, budget=(a.test_photons, a.test_photons), beam_radius=(0.0, 0.5))
    tune = b.autotune(train.subset(np.arange(min(256, n_train))), photons_cap=20000)

    t0 = time.perf_counter()
    rt_tr, _, ms_tr = run_batched(b, train, chunk)
    t_gen = time.perf_counter() - t0
    rt_te, w2_te, ms_te = run_batched(b, test, chunk)
    mc_rate = float(test.photons.sum()) / (ms_te / 1e3)
    feats, targets = train.features(), SG.reflectance_targets(rt_tr, a.floor)

    curve, res = [], None
    save_size = a.save_size or n_train
    for size in sizes:
        steps = a.steps
        sur = SG.Surrogate(n_in=15, n_out=1000, members=a.members, max_rows=65536, device=a.device, floor=a.floor,
                           gate=a.gate)
        t0 = time.perf_counter()
        curves = sur.fit(feats[:size], targets[:size], steps=steps, batch=a.batch, lr=a.lr, seed=a.seed,
                         weighted=not a.unweighted)
        t_fit = time.perf_counter() - t0
        acc = evaluate(sur, test, rt_te, w2_te, a.floor)
        m0 = sur.members[0]
        m0.forward(np.zeros((65536, 15), np.float32))
        ms_fwd = m0.forward_timed(65536, reps=50)
        evals = 65536 / (ms_fwd / 1e3) / a.members
        entry = {"train_instances": size, "steps": steps, "fit_wall_s": t_fit, "fit_device_ms": sur.train_ms,
                 "final_loss": [float(c[-100:].mean()) for c in curves], **acc}
        curve.append(entry)
        print(json.dumps(entry), flush=True)
        if size == save_size and a.save:
            sur.save(a.save)
        if size == n_train:
            res = {
                "weighted_loss": not a.unweighted, "floor": a.floor, "train_instances": size,
                "train_photons": a.train_photons, "test_instances": a.test, "test_photons": a.test_photons,
                "members": a.members, "steps": steps, "batch": a.batch, "autotune": tune,
                "mc_train_photons_per_s": float(train.photons.sum()) / (ms_tr / 1e3), "mc_train_wall_s": t_gen,
                "mc_test_photons_per_s": mc_rate, "fit_wall_s": t_fit, "fit_device_ms": sur.train_ms,
                "final_loss": entry["final_loss"], **acc,
                "evals_per_s_ensemble": evals, "forward_ms_65536_rows_one_member": ms_fwd,
                "mc_evals_per_s_1e7": mc_rate / 1e7, "speedup_vs_mc_1e7": evals / (mc_rate / 1e7)}
        sur.close()
    res["error_vs_training_size"] = [{k: e[k] for k in ("train_instances", "steps", "median_rel_err_cells",
                                                         "p90_rel_err_cells", "median_rel_err_rings",
                                                         "gate_pass_fraction", "median_rel_err_cells_gated")}
                                     for e in curve]
    if a.save:
        res["saved"] = {"path": a.save, "train_instances": save_size}
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    b.close()
    return res


if __name__ == "__main__":
    main()
