"""Host side of the batched planar path (no GPU): the instance sampler of the layered sweep, the
instance -> reference-model conversion used by the oracle checks, and the library's validation of
batch specs and instance tables (xmc_batch_validate runs on the host only)."""
import numpy as np
import pytest

from xmcml_b200 import batch as XB
from xmcml_b200 import structs as S


def test_sampler_distributions_and_reproducibility():
    a = XB.sample_instances(7, 4096)
    b = XB.sample_instances(7, 4096)
    for k in a.__dataclass_fields__:
        assert np.array_equal(getattr(a, k), getattr(b, k))
    assert a.mua.min() >= 0.005 and a.mua.max() <= 1.0
    # log-uniform: log10 mua roughly uniform over [-2.3, 0]
    assert abs(np.log10(a.mua).mean() - (np.log10(0.005) / 2)) < 0.05
    assert a.mus.min() >= 5 and a.mus.max() <= 40 and a.g.min() >= 0.7 and a.g.max() <= 0.95
    assert a.n.min() >= 1.33 and a.n.max() <= 1.45
    assert a.thickness[:, 0].min() >= 0.05 and a.thickness[:, 0].max() <= 0.3
    assert a.thickness[:, 1].min() >= 0.5 and a.thickness[:, 1].max() <= 2.0
    assert np.all(a.thickness[:, 2] == 50.0)
    assert a.photons.min() >= 1e5 and a.photons.max() <= 1e7
    # expected total of log-uniform [1e5, 1e7] budgets: (1e7 - 1e5) / ln(100) per instance
    assert a.photons.astype(float).mean() == pytest.approx((1e7 - 1e5) / np.log(100), rel=0.05)
    assert len(set(a.seed.tolist())) == len(a)
    assert a.features().shape == (4096, 15)


def test_to_scene_layers_and_detectors():
    inst = XB.sample_instances(3, 2)
    sc = XB.to_scene(inst, 1, n_rings=50, n_time=20)
    assert len(sc.layers) == 4 and sc.layers[0].n == 1.0
    for l in range(3):
        L = sc.layers[l + 1]
        assert (L.mua, L.mus, L.g, L.n) == (inst.mua[1, l], inst.mus[1, l], inst.g[1, l], inst.n[1, l])
    zs = [float(v[0, 2]) for v, _ in sc.surfaces]
    assert np.allclose(zs, np.concatenate([[0.0], np.cumsum(inst.thickness[1])]))
    assert len(sc.rings) == 50 and sc.time_bins == 20
    assert sc.time_finish == pytest.approx(1000 * 0.299792458)
    inst.n_below[1] = 1.33
    with pytest.raises(ValueError):
        XB.to_scene(inst, 1)


def test_validate_accepts_and_rejects():
    inst = XB.sample_instances(1, 8, budget=(10, 100))
    assert XB.validate(inst) == S.XMC_OK
    assert XB.validate(inst.subset([])) == S.XMC_OK
    cases = [("g", (2, 1), 1.0), ("g", (0, 0), -1.0), ("mua", (1, 2), -0.1), ("n", (3, 0), 0.0),
             ("thickness", (4, 1), 0.0), ("mus", (5, 0), float("nan"))]
    for field, ij, v in cases:
        bad = inst.subset(range(8))
        getattr(bad, field)[ij] = v
        assert XB.validate(bad) == S.XMC_ERR_INVALID_INPUT, field
    bad = inst.subset(range(8))
    bad.mua[0, 0] = 0.0
    bad.mus[0, 0] = 0.0
    assert XB.validate(bad) == S.XMC_ERR_INVALID_INPUT
    bad = inst.subset(range(8))
    bad.beam_radius[2] = -1.0
    assert XB.validate(bad) == S.XMC_ERR_INVALID_INPUT
    bad = inst.subset(range(8))
    bad.photons[0] = 2 ** 50
    assert XB.validate(bad) == S.XMC_ERR_RANGE
    assert XB.validate(inst, max_instances=4) == S.XMC_ERR_RANGE
    assert XB.validate(inst, n_rings=0) == S.XMC_ERR_RANGE
    assert XB.validate(inst, n_time=0) == S.XMC_ERR_RANGE
    assert XB.validate(inst, ring_width=0.0) == S.XMC_ERR_INVALID_INPUT
    assert XB.validate(inst, roulette_chance=0.0) == S.XMC_ERR_INVALID_INPUT
    assert XB.validate(inst, min_weight=1.0) == S.XMC_ERR_INVALID_INPUT
    assert XB.validate(inst, time_start=5.0, time_finish=1.0) == S.XMC_ERR_INVALID_INPUT
    assert XB.validate(inst, ring_angle=0.0) == S.XMC_ERR_INVALID_INPUT


def test_struct_sizes_match_the_header():
    import ctypes as C
    assert C.sizeof(S.BatchSpec) == 112
    assert C.sizeof(S.BatchInstance) == 280
    assert C.sizeof(S.BatchTuning) == 24
    assert C.sizeof(S.BatchResult) == 112


def test_features_round_trip():
    a = XB.sample_instances(8, 16, beam_radius=(0.0, 0.5))
    b = XB.from_features(a.features(), photons=7, seed=100)
    for k in ("mua", "mus", "g", "n", "thickness", "beam_radius"):
        assert np.allclose(getattr(a, k), getattr(b, k), rtol=1e-12), k
    assert np.all(b.photons == 7) and list(b.seed[:2]) == [100, 101]
