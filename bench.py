"""Throughput benchmark of the photon-transport hot path (LaunchOMP -> ComputePhoton) on B200.

Workload (default): the 3-layer tissue with the top two boundaries triangulated height fields
(256 x 256 vertices over 20 x 20 mm each, 2 x 130,050 triangles, A = 0.05 mm, lam = 2 mm), planar
L2/L3 boundary and bottom, 50 rings of 0.1 mm and 200 time bins of 5 ps, 100^3 absorption grid;
one step = one transport call of 1e7 photons with the reference LaunchOMP's semantics and tallies
(weight cut at MinWeight 1e-4, photons killed outside Area, absorption grid, detectors, time bins,
scattering map and one trajectory map per detector), so the GPU arms and the reference arm do the
same work. Synthetic input generated by xmcml_b200.scenes.

  value : photons/s with the device image resident (xmc_run on a persistent context), device time
          of every run from CUDA events on the library's stream (tally and map zeroing, run pass,
          trajectory replay pass, tally read-back); L2 is flushed between steps (256 MB write).
  e2e   : photons/s through the reference-signature C-ABI xmc_launch_omp(InputInfo*, OutputInfo*,
          MCG59*, int) with host buffers (reference-layout BVH prebuilt once, as the reference's
          launcher does). Every step fingerprints the caller's InputInfo, runs, reads every tally
          and map back and adds them into the FP64 OutputInfo; the device image (triangles, tree,
          tables, detectors) is built and uploaded only when the model's contents change, which
          `cold` measures (one call on a model the library has not seen). Host wall clock around
          the call.
  workloads : the same measurements (fewer steps) on the planar 3-layer stack and on the ellipsoid
          target scene, each with its own reference CPU baseline and roofline.
  --impl reference : the reference's own OpenMP LaunchOMP (compiled from its sources into
          oracle/_ref, -O3, all host threads) on a bounded sample of the same workload.
Multi-GPU (torchrun): independent replicas on disjoint photon-id ranges (weak scaling); the only
collectives are the barriers and the max-over-ranks of the timings.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "photons/s (3-layer, BVH mesh)"
UNIT = "photons/s"


SEMANTICS = ("reference LaunchOMP: weight cut at MinWeight 1e-4, photons killed outside Area; absorption grid, "
             "detectors, time bins, scattering map and one trajectory map per detector")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["heightfield", "planar", "ellipsoid", "batch"], default="heightfield")
    p.add_argument("--instances", type=int, default=1024)
    p.add_argument("--budget-scale", type=float, default=1.0)
    p.add_argument("--photons", type=int, default=10_000_000)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-surrogate", action="store_true")
    p.add_argument("--extra-workloads", default="planar,ellipsoid,batch",
                   help="workloads measured beside the headline one (comma list, '' for none)")
    p.add_argument("--extra-steps", type=int, default=3)
    p.add_argument("--no-roulette-variant", action="store_true")
    p.add_argument("--no-autotune", action="store_true",
                   help="fixed launch shape instead of the autotuner's (profiling runs): block 512, 32 photon ids "
                        "per claim, cooperative queries in rounds of 8, 8 triangles per grid cell")
    return p.parse_args()


def make_scene(workload, photons):
    """Scene and config of a workload; the config is the same in every arm (ours and reference)."""
    from xmcml_b200 import scenes
    if workload == "heightfield":
        return scenes.height_field_tissue(photons=photons), {
            "workload": f"heightfield-3layer-256x256-{photons:.0e}", "surfaces": "2 height fields 256x256 (2x130050 tris) + 2 planes",
            "rings": 50, "time_bins": "200 x 5 ps", "grid": "100x100x100 over 10x10x5 mm",
            "photons_per_step": photons, "semantics": SEMANTICS}
    if workload == "ellipsoid":
        sc = scenes.ellipsoid_target(photons=photons)
        return sc, {
            "workload": f"ellipsoid-target-3layer-{photons:.0e}", "surfaces": f"4 planes + icosphere ellipsoid 2x2x1 mm "
            f"({sc.n_triangles - 8} tris) at depth 2.5", "rings": 100, "time_bins": "200 x 5 ps",
            "grid": "256x256x128 over 20x20x10 mm", "photons_per_step": photons, "semantics": SEMANTICS}
    return scenes.planar(photons=photons), {
        "workload": f"planar-3layer-{photons:.0e}", "rings": 50, "grid": "100x100x100 over 10x10x5 mm",
        "photons_per_step": photons, "semantics": SEMANTICS}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(prefix="xmc_clocks_", suffix=".csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _ref_sample_size(info, seconds, threads):
    """Photon count for about `seconds` of the reference's LaunchOMP, from growing probe runs."""
    from oracle import bind as OB
    n = max(threads * 50, 500)
    while True:
        out = OB.ref_new_output(info, fast=True)
        t0 = time.perf_counter()
        OB.ref_launch(info, out, 5, threads, fast=True, n=n)
        dt = time.perf_counter() - t0
        OB.ref(True).ref_free_output(C.byref(out))
        if dt > min(2.0, seconds / 4) or n > 5e7:
            return int(max(threads * 50, min(n / dt * seconds, 5e7)))
        n *= 4


def cpu_reference_rate(xml, surf, seconds, threads, seed=777):
    """The reference's LaunchOMP (oracle/_ref/libxmcml_ref_fast.so, -O3, all threads) on a bounded
    sample of the workload; returns (photons/s, photons, seconds)."""
    from oracle import bind as OB
    info = OB.ref_load_model(xml, surf, fast=True)
    OB.ref(True).ref_generate_bvh(C.byref(info))  # prebuilt tree, outside the timed region
    n2 = _ref_sample_size(info, seconds, threads)
    out2 = OB.ref_new_output(info, fast=True)
    t0 = time.perf_counter()
    OB.ref_launch(info, out2, seed + 1, threads, fast=True, n=n2)
    dt = time.perf_counter() - t0
    OB.ref(True).ref_free_output(C.byref(out2))
    return n2 / dt, n2, dt


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    d = tempfile.mkdtemp(prefix="xmc_bench_ref_")
    inst = None
    if args.workload == "batch":
        # the instances one after the other through the reference's LaunchOMP (the reference has no
        # batched form): a bounded sample of photons from instance k at step k
        from xmcml_b200 import batch as XB
        inst = XB.sample_instances(2024, args.instances, budget=(1e5 * args.budget_scale, 1e7 * args.budget_scale))
        sc = XB.to_scene(inst, 0)
        cfg = batch_config(args, inst)
    else:
        sc, cfg = make_scene(args.workload, args.photons)
    xml, surf = sc.write(d, "bench")
    from oracle import bind as OB
    if not OB.ref_available(fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libxmcml_ref_fast.so missing"}))
        return
    threads = os.cpu_count() or 1
    info = OB.ref_load_model(xml, surf, fast=True)
    OB.ref(True).ref_generate_bvh(C.byref(info))
    # size one step at about 8 s of work from growing probe runs
    n_step = _ref_sample_size(info, 8.0, threads)
    out = OB.ref_new_output(info, fast=True)
    for w in range(args.warmup):
        OB.ref_launch(info, out, 100 + w, threads, fast=True, n=max(n_step // 8, threads * 10))
    OB.ref(True).ref_free_output(C.byref(out))
    times = []
    for k in range(args.steps):
        if inst is not None and k > 0:  # the sweep's next instance, same sample size
            xml, surf = XB.to_scene(inst, k % len(inst)).write(d, f"bench{k}")
            info = OB.ref_load_model(xml, surf, fast=True)
            OB.ref(True).ref_generate_bvh(C.byref(info))
        out = OB.ref_new_output(info, fast=True)
        t0 = time.perf_counter()
        OB.ref_launch(info, out, 777 + k, threads, fast=True, n=n_step)
        times.append(time.perf_counter() - t0)
        OB.ref(True).ref_free_output(C.byref(out))
    tot = sum(times)
    value = n_step * args.steps / tot
    metric = "photons/s (batched 3-layer instances)" if inst is not None else METRIC
    line = {"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "arm": {"parallelism": f"OpenMP x{threads} (host CPU)",
                    "sample": ("instance k of the sweep at step k, " if inst is not None else "") +
                              f"{n_step} photons per step"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{n_step} photons per step of the same workload, LaunchOMP with {threads} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_e2e(m, N, e2e_steps, rank, local, world, barrier, dist, torch, tuned=None):
    """e2e photons/s through xmc_launch_omp with host InputInfo/OutputInfo (see module docstring).

    value: repeated LaunchOMP calls on one model (the library keeps the device image while the
    model's contents are unchanged), each call fingerprinting the host InputInfo, running both
    passes and adding every tally and map into the host OutputInfo. cold: one call on a model the
    library has not seen (device image built and uploaded inside the call)."""
    from xmcml_b200 import api, _lib
    lib = _lib.load()
    tree = lib.xmc_generate_bvh_tree(m.info.surface, m.info.numberOfSurfaces)  # prebuilt once, like the reference launcher
    m.info.bvhTree = tree
    m.info.numberOfPhotons = N
    out = api.Output(m)
    rng = api.mcg59_init(777 + rank, 0, 1)
    lib.xmc_launch_release()
    barrier()
    t0 = time.perf_counter()
    api.launch_omp(m, out, rng, 0)  # cold: image build + upload + run + read-back
    cold_s = time.perf_counter() - t0
    barrier()
    e2e_t = []
    for k in range(e2e_steps):
        t0 = time.perf_counter()
        api.launch_omp(m, out, rng, 0)
        e2e_t.append(time.perf_counter() - t0)
    barrier()
    from xmcml_b200 import replicas
    dev = torch.device(f"cuda:{local}")
    e2e_s = replicas.max_over_ranks(sum(e2e_t), dist, dev)
    cold_s = replicas.max_over_ranks(cold_s, dist, dev)
    e2e_value = world * e2e_steps * N / e2e_s
    lib.xmc_launch_release()
    grid = out.info.gridSize
    D = out.info.numberOfDetectors
    T = m.info.timeScaleSize
    out.close()
    # where a warm call's time goes: the same run through a context with LaunchOMP's options
    t = api.Transport(m, tuned) if tuned is not None else api.Transport(m, roulette=False, scattering=True,
                                                                        trajectories=True, device=local)
    out2 = api.Output(m)
    t.run(N, seed=777 + rank, output=out2)  # first run of a fresh context (staging allocation)
    t0 = time.perf_counter()
    led = t.run(N, seed=777 + rank, output=out2)
    wall_ms = (time.perf_counter() - t0) * 1e3
    image_b = led["h2d_bytes"]
    # read back per call, as the library counts it: absorption and scattering maps (u64), detector and
    # time-bin tallies, the run and replay ledgers, status, and the trajectory maps as their non-zero
    # cells (u32 cell + u64 count each, after the per-block offsets)
    d2h = led["d2h_bytes"]
    dense_d2h = 8 * grid * (2 + D) + 32 * D + 32 * D * T + 2 * 8 * 32 + 16
    t.close()
    out2.close()
    m.info.bvhTree = None
    lib.xmc_free_bvh_tree(tree)
    return {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(d2h),
            "via": "xmc_launch_omp (LaunchOMP signature), host InputInfo/OutputInfo",
            "h2d_note": "the model's device image is uploaded when the model's contents change (cold); "
                        "a warm call copies no input buffer (seed and counts travel as kernel arguments)",
            "cold": {"value": world * N / cold_s, "unit": UNIT, "h2d_bytes": int(image_b), "d2h_bytes": int(d2h),
                     "seconds": cold_s},
            "d2h_dense_bytes": int(dense_d2h),
            "breakdown_ms": {"kernels": led["kernel_ms"], "device_total": led["total_ms"], "host_wall": wall_ms,
                             "trajectory_replayed": led["n_trajectory_replayed"]}}


def atomic_peak(local):
    """Measured throughput of scattered 64-bit atomic adds into an L2-resident 8 MB array (the
    tallies' access pattern) on this GPU, adds/s."""
    from xmcml_b200 import _lib
    rate, ms = C.c_double(0), C.c_double(0)
    _lib.check(_lib.load().xmc_atomic_throughput(local, 20, 256, C.byref(rate), C.byref(ms)))
    return rate.value


def roofline(led, kernel_ms, clocks, n_photons, atomics_per_s=None, traj_adds=0):
    """Roofline of the transport kernel from the per-step cost model, three roofs:
      issue   : 48 FP32 flop + ~45 INT32 ops (Philox) per walk iteration, plus 16 flop per BVH/grid
                node test and 30 per triangle test, against the nominal SIMT peak 148 SMs x 128
                lanes x SM clock;
      mufu    : 6 MUFU ops per iteration against 148 SMs x 16 MUFU lanes x SM clock;
      atomics : one 64-bit absorption add per iteration (an upper bound: boundary iterations drop no
                weight) plus one scattering-map add per z-plane crossing and one trajectory-map add
                per crossing of a detected photon, against the measured L2 atomic throughput.
    The largest fraction names the bound."""
    steps = led["steps"]
    nodes = led["n_node_visits"]
    tris = led["n_triangle_tests"]
    ops = steps * (48 + 45) + nodes * 16 + tris * 30
    t = kernel_ms / 1e3
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    peak_ops = 148 * 128 * sm_mhz * 1e6
    achieved = ops / t
    mufu = steps * 6 / t
    mufu_peak = 148 * 16 * sm_mhz * 1e6
    roofs = {"issue": achieved / peak_ops, "mufu": mufu / mufu_peak}
    adds = steps + led.get("n_plane_crossings", 0) + traj_adds
    if atomics_per_s:
        roofs["atomics"] = adds / t / atomics_per_s
    bound = max(roofs, key=roofs.get)
    if bound == "atomics":
        head = {"achieved": adds / t / 1e9, "peak": atomics_per_s / 1e9, "unit": "G adds/s"}
    elif bound == "mufu":
        head = {"achieved": mufu / 1e12, "peak": mufu_peak / 1e12, "unit": "T MUFU ops/s"}
    else:
        head = {"achieved": achieved / 1e12, "peak": peak_ops / 1e12, "unit": "TOP/s"}
    return {"bound": bound, **head, "frac": roofs[bound], "traffic": None, "roofs": roofs,
            "model": {"ops_per_step": (48 + 45), "node_tests_per_step": nodes / max(steps, 1),
                      "triangle_tests_per_step": tris / max(steps, 1), "steps_per_photon": steps / max(n_photons, 1),
                      "atomic_adds_per_step": adds / max(steps, 1), "atomic_adds_per_s": adds / t,
                      "atomic_peak_adds_per_s": atomics_per_s,
                      "peak_source": "issue: nominal 148 SMs x 128 FP32/INT32 lanes x median sampled SM clock "
                                     "(MEASURED_PEAKS.json has no SIMT figure; the walk is not HBM- or tensor-bound); "
                                     "atomics: measured in this run (xmc_atomic_throughput, 8 MB array)"}}


def surrogate_inference(local):
    """Surrogate evals/s: the 15 -> 256 x 4 (SiLU) -> 1000 network (random He-uniform weights: the
    speed does not depend on their values) on a 65,536-row batch on the tensor cores; device time of
    the resident forward pass (the fused kernel, one launch for all five layers, replayed from a CUDA
    graph) and host-to-host time of one call."""
    import numpy as np
    from xmcml_b200 import surrogate as SG
    rows = 65536
    m = SG.MLP(15, 1000, 256, 4, max_rows=rows, device=local)
    m.set_params(SG.he_uniform(np.random.default_rng(0), 15, 256, 4, 1000))
    x = np.random.default_rng(1).standard_normal((rows, 15)).astype(np.float32)
    m.forward(x)
    t0 = time.perf_counter()
    m.forward(x)
    e2e_s = time.perf_counter() - t0
    ms = m.forward_timed(rows, reps=50)
    m.close()
    algo = 2.0 * rows * (15 * 256 + 3 * 256 * 256 + 256 * 1000)   # multiply-adds of the network x 2
    issued = 2.0 * rows * (64 * 256 + 3 * 256 * 256 + 256 * 1024)  # with the padded input / output tiles
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]
    except Exception:
        pass
    evals = rows / (ms / 1e3)
    # the Monte Carlo the network stands in for: batched planar 3-layer instances on this GPU
    from xmcml_b200 import batch as XB
    b = XB.Batch(device=local, max_instances=64)
    inst = XB.sample_instances(3, 64, budget=(1e6, 1e6))
    b.run(inst.with_photons(20000))
    mc = b.run(inst)
    b.close()
    mc_rate = float(inst.photons.sum()) / (mc["kernel_ms"] / 1e3)
    mc_evals = mc_rate / 1e7
    return {"metric": "surrogate evals/s", "value": evals, "batch": rows, "ms_per_batch": ms,
            "e2e": {"value": rows / e2e_s, "unit": "evals/s", "h2d_bytes_per_step": rows * 15 * 4,
                    "d2h_bytes_per_step": rows * 1000 * 4},
            "roofline": {"bound": "tensor", "achieved": algo / (ms / 1e3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": (algo / (ms / 1e3) / 1e12 / peak) if peak else None,
                         "issued_tflops": issued / (ms / 1e3) / 1e12,
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst, cuBLAS 8192^3)"},
            "vs_mc_1e7_photon_evals": evals / mc_evals, "mc_evals_per_s_at_1e7_photons": mc_evals,
            "mc_batched_photons_per_s": mc_rate, "error": surrogate_accuracy(local)}


def surrogate_accuracy(local, n_test=100, photons=1e7):
    """Accuracy of the committed trained ensemble (xmcml_b200/data/surrogate_ensemble.npz, written by
    xmcml_b200.surrogate_study --save) in this run: fresh held-out instances of the sweep's
    distributions (a seed the training never used), their ring x time reflectance from the batched
    Monte Carlo at `photons` each, and the network's median relative error on the cells the Monte
    Carlo resolves to 1 %."""
    import numpy as np
    from xmcml_b200 import batch as XB
    from xmcml_b200 import surrogate as SG
    from xmcml_b200 import surrogate_study as SS
    if not os.path.exists(SG.DEFAULT_ENSEMBLE):
        return {"value": None, "note": f"{os.path.relpath(SG.DEFAULT_ENSEMBLE, ROOT)} missing"}
    sur = SG.Surrogate.load(SG.DEFAULT_ENSEMBLE, device=local)
    test = XB.sample_instances(90210, n_test, budget=(photons, photons), beam_radius=(0.0, 0.5))
    b = XB.Batch(n_rings=50, ring_width=0.1, n_time=20, time_finish=1000 * XB.C_MM_PER_PS, max_instances=n_test,
                 device=local)
    rt, w2, ms = SS.run_batched(b, test, n_test)
    b.close()
    acc = SS.evaluate(sur, test, rt, w2, sur.floor)
    sur.close()
    return {"value": acc["median_rel_err_cells"], "unit": "median relative error (cells resolved to 1 %)",
            "p90": acc["p90_rel_err_cells"], "rings": acc["median_rel_err_rings"],
            "gate_pass_fraction": acc["gate_pass_fraction"], "gated": acc["median_rel_err_cells_gated"],
            "judged_cells": acc["judged_cells"],
            "reference": f"batched Monte Carlo, {n_test} held-out instances x {photons:.0e} photons ({ms / 1e3:.1f} s)",
            "ensemble": os.path.relpath(SG.DEFAULT_ENSEMBLE, ROOT)}


def batch_config(args, inst):
    """Config of the batched sweep, the same in both arms."""
    return {"workload": f"batched-{len(inst)}-instances-3layer", "photons_per_step": int(inst.photons.sum()),
            "budgets": f"log-uniform [{1e5 * args.budget_scale:.0e}, {1e7 * args.budget_scale:.0e}]",
            "rings": 50, "time_bins": "20 x 50 ps",
            "semantics": "GPU: roulette 1e-4 / 0.1, no Area kill (the sweep's semantics); reference arm: its LaunchOMP "
                         "(weight cut; the reference has no roulette) on instance k at step k"}


def run_batch_workload(args, rank, world, local, dist, torch, barrier):
    """`--workload batch`: the batched sweep's line on its own (measure_batch)."""
    line = measure_batch(args, rank, world, local, dist, torch, barrier, args.steps, args.warmup, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_batch(args, rank, world, local, dist, torch, barrier, n_steps, n_warmup, cpu_seconds):
    """Batched sweep: `instances` 3-layer planar instances (the sweep's distributions, photon budgets
    log-uniform in [1e5, 1e7] x budget_scale) in one persistent launch per step, replayed from a
    CUDA graph, launch shape from the autotuner. value: photons / device time of the transport
    kernel; e2e: photons / host wall time of xmc_batch_run (instance table upload, zeroing, kernel,
    FP64 reduction and read-back of [instances x 50 x 20] reflectance and the ledgers)."""
    import numpy as np
    from xmcml_b200 import batch as XB
    from xmcml_b200 import replicas
    K = args.instances
    inst = XB.sample_instances(2024 + rank, K, budget=(1e5 * args.budget_scale, 1e7 * args.budget_scale))
    total = int(inst.photons.sum())
    b = XB.Batch(max_instances=K, device=local)
    tune = b.autotune(inst.subset(np.arange(min(128, K))), photons_cap=20000)
    for w in range(n_warmup):
        b.run(inst)
    barrier()
    kms, walls, steps = [], [], 0
    with ClockSampler(local) as clk:
        barrier()
        for k in range(n_steps):
            t0 = time.perf_counter()
            out = b.run(inst)
            walls.append(time.perf_counter() - t0)
            kms.append(out["kernel_ms"])
            steps = int(out["steps"].sum())
        barrier()
    clocks = clk.summary()
    dev = torch.device(f"cuda:{local}")
    ker_ms = replicas.max_over_ranks(sum(kms), dist, dev)
    wall_s = replicas.max_over_ranks(sum(walls), dist, dev)
    value = world * n_steps * total / (ker_ms / 1e3)
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    t = ker_ms / n_steps / 1e3
    ops = steps * (48 + 45)
    peak = 148 * 128 * sm_mhz * 1e6
    rl = {"bound": "issue", "achieved": ops / t / 1e12, "peak": peak / 1e12, "unit": "TOP/s", "frac": ops / t / peak,
          "traffic": None, "model": {"ops_per_step": 93, "steps_per_photon": steps / total,
                                     "peak_source": "nominal 148 SMs x 128 lanes x median sampled SM clock"}}
    cpu = None
    if rank == 0 and world == 1 and cpu_seconds > 0 and not args.no_cpu_baseline:
        try:
            from oracle import bind as OB
            if OB.ref_available(fast=True):
                d = tempfile.mkdtemp(prefix="xmc_bench_batch_")
                rates = []
                for k in range(4):
                    xml, surf = XB.to_scene(inst, k).write(d, f"i{k}")
                    r, n_cpu, secs = cpu_reference_rate(xml, surf, cpu_seconds / 4, os.cpu_count() or 1)
                    rates.append(r)
                cpu = {"value": float(np.mean(rates)), "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference",
                       "sample": "the reference's LaunchOMP on the first 4 instances as planar models, "
                                 f"{cpu_seconds / 4:.0f} s each, mean rate (weight cut semantics)"}
        except Exception as e:
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference", "sample": f"failed: {e}"}
    b.close()
    R, T = 50, 20
    line = {"metric": "photons/s (batched 3-layer instances)", "value": value, "unit": UNIT, "n_gpus": world,
            "steps": n_steps, "warmup": n_warmup, "ms_per_step": ker_ms / n_steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": batch_config(args, inst),
            "arm": {"autotune": tune, "parallelism": f"replicas x{world} (disjoint instance sets)",
                    "l2": "instance table re-uploaded and 24.6 MB of tallies zeroed every step"},
            "clocks": clocks,
            "e2e": {"value": world * n_steps * total / wall_s, "unit": UNIT,
                    "h2d_bytes_per_step": K * (32 + 5 * 48), "d2h_bytes_per_step": K * (R * T * 8 + R * 8 + 16 * 8) + 4,
                    "via": "xmc_batch_run with host instance table and host result arrays"},
            "gpu_launches": 2 * n_steps, "roofline": rl, "cpu_baseline": cpu,
            "walk": {"steps_per_photon": steps / total}}
    if cpu and cpu.get("value"):
        cpu["gpu_value_over_cpu"] = value / cpu["value"]
    return line


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    if args.workload == "batch":
        run_batch_workload(args, rank, world, local, dist, torch, barrier)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    atom = None
    try:
        atom = atomic_peak(local)
    except Exception:
        atom = None
    line = measure_transport(args, args.workload, args.photons, args.steps, args.warmup, args.e2e_steps, rank, world,
                             local, dist, torch, barrier, atom, cpu_seconds=args.cpu_seconds)
    if not args.no_roulette_variant:
        # the same scene with roulette 1e-4 / 0.1 and no maps (the sweep's semantics), device time only
        line["roulette_variant"] = measure_transport(args, args.workload, args.photons, args.extra_steps, 3, 0, rank,
                                                     world, local, dist, torch, barrier, atom, roulette=True,
                                                     cpu_seconds=0)
    extra = {}
    for wl in [w for w in args.extra_workloads.split(",") if w and w != args.workload]:
        if wl == "batch":  # the batched sweep at its own config: 3 warm-up and 2 timed steps of ~14 s
            extra[wl] = measure_batch(args, rank, world, local, dist, torch, barrier, 2, 3, args.cpu_seconds)
            continue
        extra[wl] = measure_transport(args, wl, args.photons, args.extra_steps, 3, min(args.e2e_steps, 2), rank, world,
                                      local, dist, torch, barrier, atom, cpu_seconds=args.cpu_seconds * 0.75)
    if extra:
        line["workloads"] = extra
    if not args.no_surrogate:
        try:
            line["surrogate"] = surrogate_inference(local)
        except Exception as e:  # reported, not fatal
            line["surrogate"] = {"metric": "surrogate evals/s", "value": None, "error": str(e)}
    line["gpu_launches"] = line["gpu_launches"] + sum(v["gpu_launches"] for v in extra.values()) + (
        line["roulette_variant"]["gpu_launches"] if "roulette_variant" in line else 0)
    line["gpu_launches_note"] = ("transport kernel launches (run pass + trajectory replay pass per call) of the timed "
                                 "steps of the headline, the roulette variant and the extra workloads, and the batched "
                                 "sweep's kernel and reduction per timed step")
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def measure_transport(args, workload, N, steps, warmup, e2e_steps, rank, world, local, dist, torch, barrier, atom,
                      roulette=False, cpu_seconds=12.0):
    """Device-timed photons/s of `steps` transport calls of N photons on `workload` (L2 flushed
    between steps), its roofline, the e2e rates through xmc_launch_omp and the reference's CPU rate
    on the same scene. roulette=False: the reference LaunchOMP's semantics and tallies (the work the
    reference arm does); True: roulette 1e-4 / 0.1 without maps."""
    from xmcml_b200 import api, replicas
    from xmcml_b200 import structs as S
    d = tempfile.mkdtemp(prefix=f"xmc_bench_{rank}_")
    sc, cfg = make_scene(workload, N)
    xml, surf = sc.write(d, "bench")
    m = api.Model(xml, surf)
    maps = not roulette
    kw = dict(roulette=roulette, scattering=maps, trajectories=maps, device=local)
    if args.no_autotune:
        tuned, tune_ms = api.options(block_size=512, photons_per_chunk=32, query_batch=8, grid_cell_tris=8, **kw), None
    else:  # the project's launch-shape autotuner
        tuned, tune_ms = api.autotune(m, sample_photons=min(N, 2_000_000), **kw)
    t = api.Transport(m, tuned)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    for w in range(warmup):  # disjoint photon ids per rank and step
        t.run(N, seed=777, first_photon=replicas.photon_range(rank, world, N, w)[0])
    barrier()
    leds = []
    with ClockSampler(local) as clk:
        barrier()
        for k in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            leds.append(t.run(N, seed=777, first_photon=replicas.photon_range(rank, world, N, warmup + k)[0]))
        barrier()
    clocks = clk.summary()
    dev = torch.device(f"cuda:{local}")
    dev_ms = replicas.max_over_ranks(sum(l["total_ms"] for l in leds), dist, dev)
    ker_ms = replicas.max_over_ranks(sum(l["kernel_ms"] for l in leds), dist, dev)
    value = world * steps * N / (dev_ms / 1e3)
    last = leds[-1]
    traj_adds = int(t.maps()["trajectory"].sum()) if maps else 0  # one atomic add per counted crossing
    launches = sum(1 + (1 if l["n_trajectory_replayed"] > 0 else 0) for l in leds)
    shape = {"block": tuned.block_size or 256, "photons_per_claim": tuned.photons_per_chunk,
             "queries": "lane by lane" if tuned.flags & S.XMC_LANE_QUERIES else "warp-cooperative",
             "query_batch": max(1, tuned.query_batch), "grid_cell_tris": tuned.grid_cell_tris or 2,
             "autotune_sample_ms": tune_ms}
    t.close()
    del flush

    rl = roofline(last, last["kernel_ms"], clocks, N, atom, traj_adds)
    prof = os.path.join(ROOT, "profiles", f"transport_kernel_{workload}_dram.json")
    if os.path.exists(prof) and not roulette:
        try:
            pj = json.load(open(prof))
            rl["traffic"] = pj.get("dram_bytes_per_launch")
            rl["traffic_note"] = pj.get("note")
        except Exception:
            pass

    e2e = None
    if e2e_steps > 0:
        api.launch_set_options(tuned)  # the LaunchOMP replacement runs with the tuned shape as well
        try:
            e2e = run_e2e(m, N, e2e_steps, rank, local, world, barrier, dist, torch, tuned)
        finally:
            api.launch_set_options(None)

    cpu = None
    if rank == 0 and world == 1 and cpu_seconds > 0 and not args.no_cpu_baseline:
        try:
            from oracle import bind as OB
            if OB.ref_available(fast=True):
                rate, n_cpu, secs = cpu_reference_rate(xml, surf, cpu_seconds, os.cpu_count() or 1)
                cpu = {"value": rate, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference",
                       "sample": f"{n_cpu} photons of the same workload through the reference's LaunchOMP "
                                 f"({secs:.1f} s, -O3, all tallies incl. scattering and trajectory maps)"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference", "sample": f"failed: {e}"}
    if cpu and cpu.get("value"):
        cpu["gpu_value_over_cpu"] = value / cpu["value"]
        if e2e:
            cpu["gpu_e2e_over_cpu"] = e2e["value"] / cpu["value"]
            cpu["gpu_e2e_cold_over_cpu"] = e2e["cold"]["value"] / cpu["value"]
    m.close()
    return {"metric": METRIC if workload == "heightfield" else f"photons/s ({workload})", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": dev_ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": cfg if not roulette else dict(cfg, semantics="roulette 1e-4 / 0.1, photons killed outside Area; "
                                                                   "absorption grid, detectors and time bins (no maps)"),
            "arm": {"parallelism": f"replicas x{world} (disjoint photon ids)", "launch": shape,
                    "l2": "flushed between timed steps (256 MB write)"},
            "clocks": clocks, "e2e": e2e, "gpu_launches": launches, "roofline": rl, "cpu_baseline": cpu,
            "kernel_ms_per_step": ker_ms / steps,
            "walk": {"steps_per_photon": last["steps"] / N, "detected_fraction": last["n_detected"] / N,
                     "fp64_retests_per_step": last["n_fp64_retests"] / max(last["steps"], 1),
                     "plane_crossings_per_step": last["n_plane_crossings"] / max(last["steps"], 1),
                     "trajectory_replayed": last["n_trajectory_replayed"],
                     "escaped_top": last["escaped_top"], "absorbed": last["absorbed"],
                     "absorbed_target": last["absorbed_target"]}}


if __name__ == "__main__":
    main()
