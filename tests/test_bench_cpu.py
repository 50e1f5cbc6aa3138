"""bench.py parts that run without a GPU: the reference arm (the reference's own LaunchOMP on the
host cores) keeps the JSON-line contract with the same config as the GPU arm, and the transport
roofline picks its bound from the step cost model's issue, MUFU and L2-atomic roofs."""
import json
import os
import subprocess
import sys

import pytest

from oracle import bind as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.mark.skipif(not B.ref_available(fast=True), reason="reference build oracle/_ref missing")
def test_reference_arm_prints_one_json_line():
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "photons/s" and d["value"] > 0
    assert d["metric"] == "photons/s (3-layer, BVH mesh)" and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("heightfield")
    # the GPU arm's config for the same workload is the same dict (same work in both arms)
    import bench
    _, cfg = bench.make_scene("heightfield", 10_000_000)
    assert d["config"] == json.loads(json.dumps(cfg))


def test_roofline_bound_is_the_larger_roof():
    import bench
    led = {"steps": 5.5e9, "n_node_visits": 1.9e9, "n_triangle_tests": 1.2e9, "n_plane_crossings": 2.0e9}
    r = bench.roofline(led, 465.0, {"sm_mhz": 1965.0}, 10_000_000)
    assert set(r["roofs"]) == {"issue", "mufu"}
    assert r["bound"] == max(r["roofs"], key=r["roofs"].get) == "issue"
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    ops = 5.5e9 * 93 + 1.9e9 * 16 + 1.2e9 * 30
    assert r["achieved"] == pytest.approx(ops / 0.465 / 1e12)
    # with a measured atomic peak the third roof counts one add per step, per crossing and per
    # trajectory-map count
    r = bench.roofline(led, 465.0, {"sm_mhz": 1965.0}, 10_000_000, atomics_per_s=1e11, traj_adds=1.5e9)
    adds = 5.5e9 + 2.0e9 + 1.5e9
    assert r["roofs"]["atomics"] == pytest.approx(adds / 0.465 / 1e11)
    assert r["bound"] == max(r["roofs"], key=r["roofs"].get)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    r = bench.roofline(led, 465.0, {"sm_mhz": 1965.0}, 10_000_000, atomics_per_s=1e10, traj_adds=1.5e9)
    assert r["bound"] == "atomics" and r["unit"] == "G adds/s"
    assert r["achieved"] == pytest.approx(adds / 0.465 / 1e9)
