"""xmc_run_noalloc, the transport run for callers that cannot allocate GPU memory (code inside a host
framework that owns all device memory through its own pool, or a process that must not grow its
device footprint once running). The caller brings its own output buffers; the model image and the
photon-id dispenser live in the library's static device scratch array.

Checked through the C-ABI against the existing entry point (xmc_create / xmc_run /
xmc_read_tallies) with the same seed and photon range, on two calls in a row. The tallies are 64-bit
fixed-point integers and the path of every photon depends only on (seed, photon id), so the
tolerance is the one the determinism tests use: exact equality. The second call also checks that
the dispenser left in the scratch by the first call is cleared. This file is collected last."""
import ctypes as C

import numpy as np
import pytest
import torch

from xmcml_b200 import _lib, api, scenes
from xmcml_b200 import structs as S

pytestmark = pytest.mark.gpu

# raw ledger slots (LedgerSlot in xmc_internal.h)
SLOT = {"photons_launched": 0, "photons_terminated": 1, "steps": 2, "n_detected": 11,
        "absorbed_fx": 15, "escaped_top_fx": 17, "lost_area_fx": 19, "roulette_killed_fx": 24, "roulette_gained_fx": 25}


def _existing_entry_point(m, opts, seed, first, n):
    t = api.Transport(m, opts)
    led = t.run(n, seed=seed, first_photon=first)
    tal = t.tallies()
    t.close()
    return led, tal


def _noalloc(m, opts, seed, first, n):
    lib = _lib.load()
    D = max(1, m.n_detectors)
    T = m.info.timeScaleSize
    G = int(np.prod(m.grid_shape))
    dev = torch.device("cuda", opts.device)
    # the caller's own buffers, deliberately not zero: the call must clear them
    out = {"absorption": torch.full((G,), 7, dtype=torch.int64, device=dev),
           "detectors": torch.full((4 * D,), 7, dtype=torch.int64, device=dev),
           "time_bins": torch.full((4 * D * T,), 7, dtype=torch.int64, device=dev),
           "ledger": torch.full((32,), 7, dtype=torch.int64, device=dev)}
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.xmc_run_noalloc(C.byref(m.info), C.byref(opts), seed, first, n, out["absorption"].data_ptr(),
                             out["detectors"].data_ptr(), out["time_bins"].data_ptr(), out["ledger"].data_ptr(),
                             stream)
    assert st == S.XMC_OK, _lib.last_error()
    return {k: v.cpu().numpy().view(np.uint64) for k, v in out.items()}, D, T


def _compare(na, D, T, led, tal):
    assert np.array_equal(na["absorption"], tal["absorption"])
    det = na["detectors"].reshape(D, 4)
    for k, name in enumerate(["det_weight", "det_count", "det_target", "det_weight2"]):
        assert np.array_equal(det[:, k], tal[name]), name
    tb = na["time_bins"].reshape(D, T, 4)
    for k, name in enumerate(["time_weight", "time_count", "time_target", "time_weight2"]):
        assert np.array_equal(tb[:, :, k], tal[name]), name
    for name, slot in SLOT.items():
        assert int(na["ledger"][slot]) == int(led[name]), name


@pytest.mark.parametrize("which", ["planar", "heightfield"])
def test_noalloc_matches_existing_entry_point_twice(tmp_path, which):
    if which == "planar":
        sc = scenes.planar(photons=1)
    else:
        sc = scenes.height_field_tissue(photons=1, grid=64, time_bins=40)
    xml, surf = sc.write(str(tmp_path), which)
    m = api.Model(xml, surf)
    opts = api.options(roulette=True)
    n = 30_000
    for call, (seed, first) in enumerate([(11, 0), (12, 5_000)]):
        na, D, T = _noalloc(m, opts, seed, first, n)
        led, tal = _existing_entry_point(m, opts, seed, first, n)
        assert int(na["ledger"][SLOT["photons_launched"]]) == n, f"call {call}"
        _compare(na, D, T, led, tal)


def test_noalloc_rejects_a_model_beyond_the_scratch(tmp_path):
    xml, surf = scenes.height_field_tissue(photons=1).write(str(tmp_path), "big")  # 2 x 130,050 triangles
    m = api.Model(xml, surf)
    lib = _lib.load()
    opts = api.options()
    dummy = C.c_void_p(1)
    st = lib.xmc_run_noalloc(C.byref(m.info), C.byref(opts), 1, 0, 10, dummy, dummy, dummy, dummy, None)
    assert st == S.XMC_ERR_RANGE
    msg = _lib.last_error()
    assert "scratch" in msg and str(8 << 20) in msg
