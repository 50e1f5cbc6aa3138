"""Shared helpers of the test suite: scene files, oracle/GPU runs and Monte Carlo comparisons."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from xmcml_b200 import api, scenes
from xmcml_b200 import structs as S

WEIGHT_SCALE = float(2 ** 31)


def write_scene(sc: scenes.Scene, directory: str, stem: str):
    return sc.write(directory, stem)


def small_planar(photons=20000, **kw) -> scenes.Scene:
    return scenes.planar(photons=photons, **kw)


def rich_planar(photons=3000) -> scenes.Scene:
    """Planar 3-layer stack with a glass cover layer, cube detectors with layer filters and angles,
    ring detectors with mixed filters (exercising the detector re-ordering), target-range layers and
    time bins: every branch of the walk and of the detector code."""
    props = [(0.2, 0.0, 0.0, 0.0, 1.5),  # glass layer
             (0.1, 0.3, 10.0, 0.8, 1.4), (1.0, 0.05, 20.0, 0.9, 1.4), (50.0, 0.02, 15.0, 0.85, 1.37)]
    sc = scenes.planar(props, photons=photons, n_rings=0, name="rich")
    sc.rings = [scenes.Ring(0.0, 0.3, filter=[1, 2, 3, 4]), scenes.Ring(0.3, 0.6, filter=[3]),
                scenes.Ring(0.6, 1.0, angle=60.0), scenes.Ring(1.0, 2.0), scenes.Ring(2.0, 4.0, filter=[4], angle=80.0)]
    sc.cubes = [scenes.Cube((0.5, 0.5, 0.0), (0.4, 0.4, 0.01)), scenes.Cube((-1.0, 0.0, 0.0), (1.0, 1.0, 0.01), filter=[2, 3])]
    sc.time_start, sc.time_finish, sc.time_bins = 1.0, 30.0, 12
    sc.target_layers = [2, 3]
    sc.min_weight = 1e-3
    return sc


def ledger_identity_fx(led: dict) -> int:
    """Sum of all fixed-point ledger terms (roulette gains subtracted)."""
    tot = 0
    for k in S.LEDGER_TERMS:
        v = led[k + "_fx"]
        tot += -v if k == "roulette_gained" else v
    # biasing: weight created (gained) and removed (lost) by the weight-table factor
    return tot - led.get("bias_gained_fx", 0) + led.get("bias_lost_fx", 0)


def zscores(g, o, var_g, var_o):
    g, o = np.asarray(g, float), np.asarray(o, float)
    den = np.sqrt(np.maximum(np.asarray(var_g, float) + np.asarray(var_o, float), 0.0))
    with np.errstate(divide="ignore", invalid="ignore"):
        z = np.where(den > 0, (g - o) / np.where(den > 0, den, 1.0), np.where(g == o, 0.0, np.inf))
    return z


def sum_var(total, total_sq, n):
    """Variance of a sum of n per-photon scores from the sum and the sum of squares."""
    return np.maximum(np.asarray(total_sq, float) - np.asarray(total, float) ** 2 / n, 0.0)


def oracle_opts_for(roulette=False, area_kill=True, beam_radius=0.0, nthreads=None):
    from oracle import bind as B
    flags = (B.OFLAG_ROULETTE if roulette else 0) | (0 if area_kill else B.OFLAG_NO_AREA_KILL)
    return B.default_opts(rng_kind=B.RNG_PHILOX, flags=flags, beam_radius=beam_radius,
                          nthreads=nthreads or os.cpu_count() or 1)


class BatchStats:
    """Running sum and sum of squares of a per-batch tally array over independent batches (photon-id
    ranges or keys). The variance of the total is estimated from the spread of the batch values
    (batch means): var(total) = B / (B - 1) * sum_b (x_b - total / B)^2."""

    def __init__(self):
        self.s1 = None
        self.s2 = None
        self.nz = None
        self.k = 0

    def add(self, x):
        x = np.asarray(x, dtype=np.float64)
        if self.s1 is None:
            self.s1 = np.zeros_like(x)
            self.s2 = np.zeros_like(x)
            self.nz = np.zeros(x.shape, dtype=np.uint8)
        self.s1 += x
        self.s2 += x * x
        self.nz += x != 0
        self.k += 1

    @property
    def total(self):
        return self.s1

    def var_total(self):
        k = self.k
        if k < 2:
            return np.full_like(self.s1, np.inf)
        return np.maximum(self.s2 - self.s1 * self.s1 / k, 0.0) * k / (k - 1)


def cell_zscores(g: BatchStats, o: BatchStats, min_batches=None):
    """Per-cell z-scores of two batch-mean tallies over the cells that every batch of both sides
    scored (so both variance estimates rest on all batches); returns (z of those cells, their count,
    the number of cells either side scored)."""
    kb = g.k if min_batches is None else min_batches
    sel = (g.nz >= kb) & (o.nz >= kb)
    z = zscores(g.total[sel], o.total[sel], g.var_total()[sel], o.var_total()[sel])
    return z, int(sel.sum()), int(((g.nz > 0) | (o.nz > 0)).sum())
