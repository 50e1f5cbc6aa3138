"""Batched planar instances: many optical-property sets of one planar layer stack in one persistent
GPU launch (xmc_batch_* in libxmcml_b200.so). No counterpart in the reference, whose LaunchOMP
(base/xmcml/xmcmlLauncher/launcher_omp.cpp:123-163) runs one model per call; an instance here is
the planar model a caller would run through it (see `to_scene` for the equivalent input files).

    b = Batch(n_layers=3, n_rings=50, ring_width=0.1, n_time=20, time_finish=299.792458)
    inst = sample_instances(seed=1, count=1024)     # the layered sweep's distributions
    out = b.run(inst)                               # rings / ring x time / per-instance ledger
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import numpy as np

from . import structs as S
from ._lib import XmcError, check, load

C_MM_PER_PS = 0.299792458


@dataclass
class Instances:
    """Instance table as arrays: per-layer properties [K, L]; per-instance scalars [K]."""
    mua: np.ndarray
    mus: np.ndarray
    g: np.ndarray
    n: np.ndarray
    thickness: np.ndarray
    photons: np.ndarray
    seed: np.ndarray
    beam_radius: np.ndarray
    n_above: np.ndarray
    n_below: np.ndarray

    def __len__(self) -> int:
        return int(self.mua.shape[0])

    @property
    def n_layers(self) -> int:
        return int(self.mua.shape[1])

    def subset(self, idx) -> "Instances":
        idx = np.asarray(idx, dtype=np.int64)
        return Instances(**{k: np.asarray(getattr(self, k))[idx].copy() for k in self.__dataclass_fields__})

    def with_photons(self, photons) -> "Instances":
        out = self.subset(np.arange(len(self)))
        out.photons = np.broadcast_to(np.asarray(photons, dtype=np.uint64), (len(self),)).copy()
        return out

    def features(self) -> np.ndarray:
        """Surrogate inputs [K, 4 L + (L - 1) + 1]: per layer (log10 mua, mus, g, n), the finite layer
        thicknesses and the beam radius (float64)."""
        L = self.n_layers
        cols = [np.log10(self.mua), self.mus, self.g, self.n, self.thickness[:, :L - 1], self.beam_radius[:, None]]
        return np.concatenate([np.asarray(c, dtype=np.float64).reshape(len(self), -1) for c in cols], axis=1)

    def to_ctypes(self):
        K, L = len(self), self.n_layers
        if L > S.XMC_BATCH_MAX_LAYERS:
            raise ValueError("too many layers")
        arr = (S.BatchInstance * max(K, 1))()
        for k in range(K):
            I = arr[k]
            for l in range(L):
                I.mua[l] = float(self.mua[k, l]); I.mus[l] = float(self.mus[k, l]); I.g[l] = float(self.g[k, l])
                I.n[l] = float(self.n[k, l]); I.thickness[l] = float(self.thickness[k, l])
            I.n_above = float(self.n_above[k]); I.n_below = float(self.n_below[k])
            I.beam_radius = float(self.beam_radius[k])
            I.photons = int(self.photons[k]); I.seed = int(self.seed[k])
        return arr


def make_instances(mua, mus, g, n, thickness, photons, seed, beam_radius=0.0, n_above=1.0, n_below=1.0) -> Instances:
    mua = np.atleast_2d(np.asarray(mua, dtype=np.float64))
    K = mua.shape[0]
    f = lambda a: np.broadcast_to(np.asarray(a, dtype=np.float64), mua.shape).copy()
    v = lambda a, dt=np.float64: np.broadcast_to(np.asarray(a, dtype=dt), (K,)).copy()
    return Instances(mua.copy(), f(mus), f(g), f(n), f(thickness), v(photons, np.uint64), v(seed, np.uint64),
                     v(beam_radius), v(n_above), v(n_below))


def from_features(features: np.ndarray, photons: int, seed: int = 0, last_thickness: float = 50.0,
                  n_ambient: float = 1.0) -> Instances:
    """Inverse of Instances.features() for 3-layer instances: [log10 mua x3, mus x3, g x3, n x3,
    L1 and L2 thickness, beam radius] -> instance table (L3 `last_thickness`)."""
    f = np.atleast_2d(np.asarray(features, dtype=np.float64))
    K = f.shape[0]
    th = np.concatenate([f[:, 12:14], np.full((K, 1), last_thickness)], axis=1)
    return make_instances(10 ** f[:, 0:3], f[:, 3:6], f[:, 6:9], f[:, 9:12], th, photons,
                          np.uint64(seed) + np.arange(K, dtype=np.uint64), f[:, 14], n_ambient, n_ambient)


def sample_instances(seed: int, count: int = 1024, budget=(1e5, 1e7), beam_radius=(0.0, 0.0),
                     last_thickness: float = 50.0) -> Instances:
    """`count` 3-layer instances drawn with numpy.random.default_rng(seed): per layer mua
    log-uniform [0.005, 1], mus uniform [5, 40], g uniform [0.7, 0.95], n uniform [1.33, 1.45];
    L1 / L2 thickness uniform [0.05, 0.3] / [0.5, 2] mm, L3 `last_thickness` (semi-infinite);
    photon budgets log-uniform in `budget`; beam radius uniform in `beam_radius`; instance seeds
    seed * 2^20 + k."""
    rng = np.random.default_rng(seed)
    L = 3
    mua = 10 ** rng.uniform(np.log10(0.005), 0.0, (count, L))
    mus = rng.uniform(5.0, 40.0, (count, L))
    g = rng.uniform(0.7, 0.95, (count, L))
    n = rng.uniform(1.33, 1.45, (count, L))
    th = np.empty((count, L))
    th[:, 0] = rng.uniform(0.05, 0.3, count)
    th[:, 1] = rng.uniform(0.5, 2.0, count)
    th[:, 2] = last_thickness
    lo, hi = budget
    photons = np.round(10 ** rng.uniform(np.log10(lo), np.log10(hi), count)).astype(np.uint64)
    br = rng.uniform(beam_radius[0], beam_radius[1], count) if beam_radius[1] > 0 else np.zeros(count)
    seeds = (np.uint64(seed) << np.uint64(20)) + np.arange(count, dtype=np.uint64)
    return make_instances(mua, mus, g, n, th, photons, seeds, br)


def to_scene(inst: Instances, k: int, n_rings: int = 50, ring_width: float = 0.1, n_time: int = 20,
             time_finish: float = 1000.0 * C_MM_PER_PS, min_weight: float = 1e-4):
    """The reference-format model (planes + layers + rings + time bins) of instance k, for the oracle
    and for the single-model path; ambient above and below must have the same index (the reference
    models both with one layer)."""
    from . import scenes
    if float(inst.n_above[k]) != float(inst.n_below[k]):
        raise ValueError("to_scene needs n_above == n_below")
    props = [(float(inst.thickness[k, l]), float(inst.mua[k, l]), float(inst.mus[k, l]), float(inst.g[k, l]),
              float(inst.n[k, l])) for l in range(inst.n_layers)]
    return scenes.planar(props=props, photons=int(inst.photons[k]), ambient_n=float(inst.n_above[k]), n_rings=n_rings,
                         ring_width=ring_width, time_bins=n_time, time_finish=time_finish, min_weight=min_weight)


class Batch:
    """Device tables and launch shape for batched runs of up to `max_instances` instances."""

    def __init__(self, n_layers: int = 3, n_rings: int = 50, ring_width: float = 0.1, n_time: int = 20,
                 time_start: float = 0.0, time_finish: float = 1000.0 * C_MM_PER_PS, ring_angle: float = 90.0,
                 min_weight: float = 1e-4, roulette_chance: float = 0.1, max_instances: int = 1024,
                 use_graph: bool = True, device: int = 0, max_steps_per_photon: int = 0):
        self._lib = load()
        s = S.BatchSpec()
        s.struct_size = C.sizeof(S.BatchSpec)
        s.n_layers, s.n_rings, s.n_time = n_layers, n_rings, n_time
        s.ring_width, s.time_start, s.time_finish, s.ring_angle = ring_width, time_start, time_finish, ring_angle
        s.min_weight, s.roulette_chance = min_weight, roulette_chance
        s.max_steps_per_photon = max_steps_per_photon
        s.max_instances, s.use_graph, s.device = max_instances, 1 if use_graph else 0, device
        self.spec = s
        self._b = C.c_void_p()
        check(self._lib.xmc_batch_create(C.byref(s), C.byref(self._b)))
        self.n_layers, self.n_rings, self.n_time = n_layers, n_rings, n_time
        self.last_n = 0

    # ---- runs ----
    def run(self, inst: Instances, allow_budget: bool = False) -> Dict[str, np.ndarray]:
        K, R, T = len(inst), self.n_rings, self.n_time
        if inst.n_layers != self.n_layers:
            raise ValueError("instance layer count differs from the batch's")
        arr = inst.to_ctypes()
        rt = np.zeros((max(K, 1), R, T))
        rg = np.zeros((max(K, 1), R))
        res = (S.BatchResult * max(K, 1))()
        ms = C.c_double(0.0)
        pd = C.POINTER(C.c_double)
        st = self._lib.xmc_batch_run(self._b, arr, K, rt.ctypes.data_as(pd), rg.ctypes.data_as(pd), res, C.byref(ms))
        if st != S.XMC_OK and not (allow_budget and st == S.XMC_ERR_BUDGET):
            check(st)
        self.last_n = K
        out = {"ring_time": rt[:K], "ring": rg[:K], "kernel_ms": ms.value, "status": st}
        for name, _ in S.BatchResult._fields_:
            out[name] = np.array([getattr(res[k], name) for k in range(K)])
        return out

    def tallies(self, n: Optional[int] = None) -> Dict[str, np.ndarray]:
        """Integer tallies of the last run: ring [n, R, 3], ring_time [n, R, T, 3] (weight_fx, count,
        weight^2_fx) and the ledger [n, 16]."""
        n = self.last_n if n is None else n
        R, T = self.n_rings, self.n_time
        ring = np.zeros((max(n, 1), R, 3), dtype=np.uint64)
        rt = np.zeros((max(n, 1), R, T, 3), dtype=np.uint64)
        led = np.zeros((max(n, 1), S.XMC_BATCH_LEDGER), dtype=np.uint64)
        P = C.POINTER(C.c_uint64)
        check(self._lib.xmc_batch_read_tallies(self._b, n, ring.ctypes.data_as(P), rt.ctypes.data_as(P),
                                               led.ctypes.data_as(P)))
        return {"ring": ring[:n], "ring_time": rt[:n], "ledger": led[:n]}

    # ---- launch shape ----
    @property
    def tuning(self) -> dict:
        t = S.BatchTuning()
        check(self._lib.xmc_batch_get_tuning(self._b, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, block_size: int = 256, photons_per_chunk: int = 64, tally_scheme: int = 1,
                   blocks_per_sm: int = 0) -> dict:
        t = S.BatchTuning(block_size, blocks_per_sm, photons_per_chunk, tally_scheme, 0.0)
        check(self._lib.xmc_batch_set_tuning(self._b, C.byref(t)))
        return self.tuning

    def autotune(self, sample: Instances, photons_cap: int = 20000) -> dict:
        t = S.BatchTuning()
        arr = sample.to_ctypes()
        check(self._lib.xmc_batch_autotune(self._b, arr, len(sample), photons_cap, C.byref(t)))
        return t.as_dict()

    def close(self):
        if self._b:
            self._lib.xmc_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def validate(inst: Instances, n_rings: int = 50, n_time: int = 20, ring_width: float = 0.1, max_instances: int = 1024,
             **spec) -> int:
    """Host-only check (no GPU): the status xmc_batch_run would return for this table."""
    s = S.BatchSpec()
    s.struct_size = C.sizeof(S.BatchSpec)
    s.n_layers, s.n_rings, s.n_time, s.ring_width = inst.n_layers, n_rings, n_time, ring_width
    s.time_start = spec.get("time_start", 0.0)
    s.time_finish = spec.get("time_finish", 1000.0 * C_MM_PER_PS)
    s.ring_angle = spec.get("ring_angle", 90.0)
    s.min_weight = spec.get("min_weight", 1e-4)
    s.roulette_chance = spec.get("roulette_chance", 0.1)
    s.max_instances = max_instances
    arr = inst.to_ctypes()
    return load().xmc_batch_validate(C.byref(s), arr, len(inst))
