"""The C-ABI as a C caller sees it: tests/c_abi/launcher_stub.c is compiled with gcc as C11 against
include/xmcml_b200.h, linked with libxmcml_b200.so, and run on a model (parse, InitOutput replacement,
specular reflectance, layout table); the GPU test also runs the LaunchOMP replacement from C."""
import os
import shutil
import subprocess

import pytest

from xmcml_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "xmcml_b200")


def _build(tmp_path):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    exe = str(tmp_path / "stub")
    cmd = ["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "c_abi", "launcher_stub.c"), "-L", LIBDIR, "-lxmcml_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_parses_and_sizes_outputs(tmp_path):
    exe = _build(tmp_path)
    xml, surf = scenes.planar(photons=100).write(str(tmp_path), "c")
    r = subprocess.run([exe, xml, surf], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "layers 4 surfaces 4 detectors 50 grid 1000000" in r.stdout
    assert "rsp 0.027777777778" in r.stdout
    assert "layout fields" in r.stdout


@pytest.mark.gpu
def test_c_caller_runs_launch_omp(tmp_path):
    exe = _build(tmp_path)
    xml, surf = scenes.planar(photons=20000).write(str(tmp_path), "c")
    r = subprocess.run([exe, xml, surf, "--run"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    w = float(r.stdout.split("detected weight")[1])
    assert 20000 * 0.2 < w < 20000 * 0.6
