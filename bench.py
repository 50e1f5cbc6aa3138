"""Throughput benchmark of the photon-transport hot path (LaunchOMP -> ComputePhoton) on B200.

Workload (default): the 3-layer tissue with the top two boundaries triangulated height fields
(256 x 256 vertices over 20 x 20 mm each, 2 x 130,050 triangles, A = 0.05 mm, lam = 2 mm), planar
L2/L3 boundary and bottom, 50 rings of 0.1 mm and 200 time bins of 5 ps, roulette 1e-4 / 0.1;
one step = one transport call of 1e7 photons. Synthetic input generated by xmcml_b200.scenes.

  value : photons/s with the device image resident (xmc_run on a persistent context), device time
          of every run from CUDA events on the library's stream (tally zeroing, kernel, read-back);
          L2 is flushed between steps (256 MB write).
  e2e   : photons/s through the reference-signature C-ABI xmc_launch_omp(InputInfo*, OutputInfo*,
          MCG59*, int) with host buffers (reference-layout BVH prebuilt once, as the reference's
          launcher does). Every step fingerprints the caller's InputInfo, runs, reads every tally
          and map back and adds them into the FP64 OutputInfo; the device image (triangles, tree,
          tables, detectors) is built and uploaded only when the model's contents change, which
          `cold` measures (one call on a model the library has not seen). Host wall clock around
          the call.
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
    return p.parse_args()


def make_scene(workload, photons):
    from xmcml_b200 import scenes
    if workload == "heightfield":
        return scenes.height_field_tissue(photons=photons), {
            "workload": f"heightfield-3layer-256x256-{photons:.0e}", "surfaces": "2 height fields 256x256 (2x130050 tris) + 2 planes",
            "rings": 50, "time_bins": "200 x 5 ps", "roulette": "1e-4 / 0.1", "grid": "100x100x100"}
    if workload == "ellipsoid":
        sc = scenes.ellipsoid_target(photons=photons)
        return sc, {
            "workload": f"ellipsoid-target-3layer-{photons:.0e}", "surfaces": f"4 planes + icosphere ellipsoid 2x2x1 mm "
            f"({sc.n_triangles - 8} tris) at depth 2.5", "rings": 100, "time_bins": "200 x 5 ps",
            "grid": "256x256x128 over 20x20x10 mm", "roulette": "1e-4 / 0.1"}
    return scenes.planar(photons=photons), {
        "workload": f"planar-3layer-{photons:.0e}", "rings": 50, "grid": "100x100x100 over 10x10x5 mm",
        "roulette": "1e-4 / 0.1"}


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
        cfg = {"workload": f"batched-{args.instances}-instances-3layer", "rings": 50, "time_bins": "20 x 50 ps",
               "sample": "instance k at step k"}
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
    cfg = dict(cfg)
    cfg["parallelism"] = f"OpenMP x{threads} (host CPU)"
    cfg["semantics"] = "reference: weight cut at MinWeight 1e-4, Area kill (no roulette in the reference)"
    metric = "photons/s (batched 3-layer instances)" if inst is not None else METRIC
    line = {"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{n_step} photons per step of the same workload, LaunchOMP with {threads} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_e2e(args, m, N, rank, local, world, barrier, dist, torch):
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
    for k in range(args.e2e_steps):
        t0 = time.perf_counter()
        api.launch_omp(m, out, rng, 0)
        e2e_t.append(time.perf_counter() - t0)
    barrier()
    from xmcml_b200 import replicas
    dev = torch.device(f"cuda:{local}")
    e2e_s = replicas.max_over_ranks(sum(e2e_t), dist, dev)
    cold_s = replicas.max_over_ranks(cold_s, dist, dev)
    e2e_value = world * args.e2e_steps * N / e2e_s
    # where a warm call's time goes: the same run through a context with LaunchOMP's options
    t = api.Transport(m, roulette=False, scattering=True, trajectories=True, device=local)
    out2 = api.Output(m)
    t.run(N, seed=777 + rank, output=out2)  # first run of a fresh context (staging allocation)
    t0 = time.perf_counter()
    led = t.run(N, seed=777 + rank, output=out2)
    wall_ms = (time.perf_counter() - t0) * 1e3
    image_b = led["h2d_bytes"]
    t.close()
    out2.close()
    grid = out.info.gridSize
    D = out.info.numberOfDetectors
    T = m.info.timeScaleSize
    # read back per call: absorption, scattering and D trajectory maps (u64), detector and time-bin
    # tallies (4 u64 each), two ledgers, status, replay count
    d2h = 8 * grid * (2 + D) + 32 * D + 32 * D * T + 2 * 8 * 32 + 16 + 8
    m.info.bvhTree = None
    lib.xmc_free_bvh_tree(tree)
    return {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(d2h),
            "via": "xmc_launch_omp (LaunchOMP signature), host InputInfo/OutputInfo",
            "h2d_note": "the model's device image is uploaded when the model's contents change (cold); "
                        "a warm call copies no input buffer (seed and counts travel as kernel arguments)",
            "cold": {"value": world * N / cold_s, "unit": UNIT, "h2d_bytes": int(image_b), "d2h_bytes": int(d2h),
                     "seconds": cold_s},
            "breakdown_ms": {"kernels": led["kernel_ms"], "device_total": led["total_ms"], "host_wall": wall_ms,
                             "trajectory_replayed": led["n_trajectory_replayed"]}}

def roofline(led, kernel_ms, clocks, n_photons):
    """Issue-bound roofline of the transport kernel from the per-step cost model (48 FP32 flop,
    6 MUFU and ~45 INT32 ops of Philox per walk iteration, plus 16 flop per BVH node test and
    30 flop per triangle test), against the nominal SIMT peak 148 SMs x 128 lanes x SM clock."""
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
    # the step cost model's two compute roofs; the larger fraction names the bound (the walk's tally
    # atomics have no measured peak here and are not claimed as a roof)
    roofs = {"issue": achieved / peak_ops, "mufu": mufu / mufu_peak}
    bound = max(roofs, key=roofs.get)
    return {"bound": bound, "achieved": achieved / 1e12, "peak": peak_ops / 1e12, "unit": "TOP/s",
            "frac": achieved / peak_ops, "traffic": None, "roofs": roofs,
            "model": {"ops_per_step": (48 + 45), "node_tests_per_step": nodes / max(steps, 1),
                      "triangle_tests_per_step": tris / max(steps, 1), "steps_per_photon": steps / max(n_photons, 1),
                      "mufu_frac": mufu / mufu_peak,
                      "peak_source": "nominal 148 SMs x 128 FP32/INT32 lanes x median sampled SM clock (MEASURED_PEAKS.json "
                                     "has no SIMT figure; the walk is not HBM- or tensor-bound)"}}


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
            "mc_batched_photons_per_s": mc_rate,
            "error_note": "accuracy of the trained ensemble is measured by xmcml_b200.surrogate_study, not here"}


def run_batch_workload(args, rank, world, local, dist, torch, barrier):
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
    for w in range(args.warmup):
        b.run(inst)
    barrier()
    kms, walls, steps = [], [], 0
    with ClockSampler(local) as clk:
        barrier()
        for k in range(args.steps):
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
    value = world * args.steps * total / (ker_ms / 1e3)
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    t = ker_ms / args.steps / 1e3
    ops = steps * (48 + 45)
    peak = 148 * 128 * sm_mhz * 1e6
    rl = {"bound": "issue", "achieved": ops / t / 1e12, "peak": peak / 1e12, "unit": "TOP/s", "frac": ops / t / peak,
          "traffic": None, "model": {"ops_per_step": 93, "steps_per_photon": steps / total,
                                     "peak_source": "nominal 148 SMs x 128 lanes x median sampled SM clock"}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import bind as OB
            if OB.ref_available(fast=True):
                d = tempfile.mkdtemp(prefix="xmc_bench_batch_")
                rates = []
                for k in range(4):
                    xml, surf = XB.to_scene(inst, k).write(d, f"i{k}")
                    r, n_cpu, secs = cpu_reference_rate(xml, surf, args.cpu_seconds / 4, os.cpu_count() or 1)
                    rates.append(r)
                cpu = {"value": float(np.mean(rates)), "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference",
                       "sample": "the reference's LaunchOMP on the first 4 instances as planar models, "
                                 f"{args.cpu_seconds / 4:.0f} s each, mean rate (weight cut semantics)"}
        except Exception as e:
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference", "sample": f"failed: {e}"}
    b.close()
    R, T = 50, 20
    line = {"metric": "photons/s (batched 3-layer instances)", "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ker_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched-{K}-instances-3layer", "photons_per_step": total,
                       "budgets": f"log-uniform [{1e5 * args.budget_scale:.0e}, {1e7 * args.budget_scale:.0e}]",
                       "rings": R, "time_bins": f"{T} x 50 ps", "roulette": "1e-4 / 0.1", "autotune": tune,
                       "parallelism": f"replicas x{world} (disjoint instance sets)",
                       "l2": "instance table re-uploaded and 24.6 MB of tallies zeroed every step"},
            "clocks": clocks,
            "e2e": {"value": world * args.steps * total / wall_s, "unit": UNIT,
                    "h2d_bytes_per_step": K * (32 + 5 * 48), "d2h_bytes_per_step": K * (R * T * 8 + R * 8 + 16 * 8) + 4,
                    "via": "xmc_batch_run with host instance table and host result arrays"},
            "gpu_launches": 2 * args.steps, "roofline": rl, "cpu_baseline": cpu,
            "walk": {"steps_per_photon": steps / total}}
    if rank == 0:
        print(json.dumps(line), flush=True)


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

    from xmcml_b200 import api, _lib
    from xmcml_b200 import structs as S
    d = tempfile.mkdtemp(prefix=f"xmc_bench_{rank}_")
    sc, cfg = make_scene(args.workload, args.photons)
    xml, surf = sc.write(d, "bench")
    m = api.Model(xml, surf)
    N = args.photons
    t = api.Transport(m, roulette=True, device=local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    from xmcml_b200 import replicas
    for w in range(args.warmup):  # disjoint photon ids per rank and step
        t.run(N, seed=777, first_photon=replicas.photon_range(rank, world, N, w)[0])
    barrier()
    leds = []
    with ClockSampler(local) as clk:
        barrier()
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            leds.append(t.run(N, seed=777, first_photon=replicas.photon_range(rank, world, N, args.warmup + k)[0]))
        barrier()
    clocks = clk.summary()
    dev = torch.device(f"cuda:{local}")
    dev_ms = replicas.max_over_ranks(sum(l["total_ms"] for l in leds), dist, dev)
    ker_ms = replicas.max_over_ranks(sum(l["kernel_ms"] for l in leds), dist, dev)
    value = world * args.steps * N / (dev_ms / 1e3)
    tal = t.tallies()
    last = leds[-1]

    # ---- e2e through the reference-signature C-ABI with host buffers ----
    e2e = None
    if args.e2e_steps > 0:
        e2e = run_e2e(args, m, N, rank, local, world, barrier, dist, torch)
    line_e2e = e2e

    sur = None
    if not args.no_surrogate:
        try:
            sur = surrogate_inference(local)
        except Exception as e:  # reported, not fatal
            sur = {"metric": "surrogate evals/s", "value": None, "error": str(e)}

    rl = roofline(last, last["kernel_ms"], clocks, N)
    prof = os.path.join(ROOT, "profiles", f"transport_kernel_{args.workload}_dram.json")
    if os.path.exists(prof):
        try:
            pj = json.load(open(prof))
            rl["traffic"] = pj.get("dram_bytes_per_launch")
            rl["traffic_note"] = pj.get("note")
        except Exception:
            pass

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import bind as OB
            if OB.ref_available(fast=True):
                rate, n_cpu, secs = cpu_reference_rate(xml, surf, args.cpu_seconds, os.cpu_count() or 1)
                cpu = {"value": rate, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference",
                       "sample": f"{n_cpu} photons of the same workload through the reference's LaunchOMP "
                                 f"({secs:.1f} s, -O3, reference semantics: weight cut, no roulette)"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference", "sample": f"failed: {e}"}

    cfg = dict(cfg)
    cfg["photons_per_step"] = N
    cfg["parallelism"] = f"replicas x{world} (disjoint photon ids)"
    cfg["l2"] = "flushed between timed steps (256 MB write)"
    cfg["launch"] = {"block": t.opts.block_size or 256}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": cfg, "clocks": clocks,
            "e2e": line_e2e,
            "gpu_launches": args.steps, "roofline": rl, "cpu_baseline": cpu, "surrogate": sur,
            "kernel_ms_per_step": ker_ms / args.steps,
            "walk": {"steps_per_photon": last["steps"] / N, "detected_fraction": last["n_detected"] / N,
                     "fp64_retests_per_step": last["n_fp64_retests"] / max(last["steps"], 1),
                     "escaped_top": last["escaped_top"], "absorbed": last["absorbed"],
                     "absorbed_target": last["absorbed_target"]}}
    t.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
