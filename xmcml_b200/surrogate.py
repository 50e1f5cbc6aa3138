"""Learned surrogate of the batched Monte Carlo: a SiLU MLP trained and evaluated on the GPU's tensor
cores (xmc_mlp_* / tcgen05 kernels in libxmcml_b200.so), with an ensemble-variance gate and the
Monte Carlo as fallback. No counterpart in the reference.

    MLP         one network (FP32 master weights on the device, BF16 compute)
    Surrogate   normalisation + an ensemble of MLPs + the training hull; predict() returns the mean,
                the ensemble spread and whether each query may use the network; reflectance()
                answers from the network where allowed and from the batched Monte Carlo otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import structs as S
from ._lib import check, load

FP = C.POINTER(C.c_float)

# The trained ensemble shipped with the package, written by `python -m xmcml_b200.surrogate_study
# --save` (4 members trained on the batched Monte Carlo of the layered sweep, 1e6 photons per training
# instance, 50 rings x 20 time bins of 50 ps).
DEFAULT_ENSEMBLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "surrogate_ensemble.npz")


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def pad_rows(n: int) -> int:
    return (n + 127) // 128 * 128


class MLP:
    """n_in -> hidden x n_hidden (SiLU) -> n_out network on one GPU."""

    def __init__(self, n_in: int, n_out: int, hidden: int = 256, n_hidden: int = 4, max_rows: int = 65536,
                 device: int = 0, fused_forward: bool = True):
        self._lib = load()
        s = S.MlpSpec()
        s.struct_size = C.sizeof(S.MlpSpec)
        s.n_in, s.hidden, s.n_hidden, s.n_out, s.max_rows, s.device = n_in, hidden, n_hidden, n_out, max_rows, device
        s.forward_kernel = 0 if fused_forward else 1
        self._m = C.c_void_p()
        check(self._lib.xmc_mlp_create(C.byref(s), C.byref(self._m)))
        self.n_in, self.n_out, self.hidden, self.n_hidden, self.max_rows = n_in, n_out, hidden, n_hidden, max_rows
        self.n_params = int(self._lib.xmc_mlp_param_count(self._m))

    @property
    def dims(self):
        return self.n_in, self.hidden, self.n_hidden, self.n_out

    def set_params(self, p: np.ndarray) -> None:
        p = _f32(p)
        if p.size != self.n_params:
            raise ValueError("parameter count mismatch")
        check(self._lib.xmc_mlp_set_params(self._m, p.ctypes.data_as(FP)))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        check(self._lib.xmc_mlp_get_params(self._m, p.ctypes.data_as(FP)))
        return p

    def set_output_weights(self, w: Optional[np.ndarray]) -> None:
        """Per-output weights of the squared error (None: all 1)."""
        if w is None:
            check(self._lib.xmc_mlp_set_output_weights(self._m, None))
        else:
            w = _f32(w)
            if w.size != self.n_out:
                raise ValueError("need one weight per output")
            self._w = w
            check(self._lib.xmc_mlp_set_output_weights(self._m, w.ctypes.data_as(FP)))

    def forward(self, x: np.ndarray) -> Tuple[np.ndarray, float]:
        """(outputs [n, n_out] float32, device ms); rows padded to a multiple of 128 internally."""
        x = _f32(x)
        n = x.shape[0]
        outs, ms = [], 0.0
        for i in range(0, n, self.max_rows):
            xb = x[i:i + self.max_rows]
            r = xb.shape[0]
            rp = pad_rows(r)
            if rp != r:
                xb = np.concatenate([xb, np.zeros((rp - r, self.n_in), np.float32)])
            y = np.empty((rp, self.n_out), dtype=np.float32)
            t = C.c_double(0.0)
            check(self._lib.xmc_mlp_forward(self._m, xb.ctypes.data_as(FP), rp, y.ctypes.data_as(FP), C.byref(t)))
            outs.append(y[:r])
            ms += t.value
        if len(outs) == 1:
            return outs[0], ms
        return np.concatenate(outs) if outs else np.zeros((0, self.n_out), np.float32), ms

    def forward_timed(self, rows: int, reps: int = 20) -> float:
        t = C.c_double(0.0)
        check(self._lib.xmc_mlp_forward_timed(self._m, rows, reps, C.byref(t)))
        return t.value

    def gradients(self, x: np.ndarray, t: np.ndarray) -> Tuple[np.ndarray, float]:
        x, t = _f32(x), _f32(t)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_float(0.0)
        check(self._lib.xmc_mlp_gradients(self._m, x.ctypes.data_as(FP), t.ctypes.data_as(FP), x.shape[0],
                                          g.ctypes.data_as(FP), C.byref(loss)))
        return g, loss.value

    def set_dataset(self, x: np.ndarray, t: np.ndarray) -> None:
        x, t = _f32(x), _f32(t)
        self._ds = (x, t)
        check(self._lib.xmc_mlp_set_dataset(self._m, x.ctypes.data_as(FP), t.ctypes.data_as(FP), x.shape[0]))

    def train(self, steps: int, batch: int = 4096, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
              eps: float = 1e-8, seed: int = 1) -> Tuple[np.ndarray, float]:
        losses = np.zeros(max(steps, 1), dtype=np.float32)
        ms = C.c_double(0.0)
        check(self._lib.xmc_mlp_train(self._m, steps, batch, lr, beta1, beta2, eps, seed, losses.ctypes.data_as(FP),
                                      C.byref(ms)))
        return losses[:steps], ms.value

    def close(self):
        if self._m:
            self._lib.xmc_mlp_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gemm_bf16(a_bits: np.ndarray, b_bits: np.ndarray, bn: int = 256, splits: int = 1) -> np.ndarray:
    """D = A . B^T on the tensor cores; a_bits [M, K], b_bits [N, K] uint16 BF16 patterns."""
    a = np.ascontiguousarray(a_bits, dtype=np.uint16)
    b = np.ascontiguousarray(b_bits, dtype=np.uint16)
    M, K = a.shape
    N = b.shape[0]
    d = np.zeros((M, N), dtype=np.float32)
    P16 = C.POINTER(C.c_uint16)
    check(load().xmc_gemm_bf16(a.ctypes.data_as(P16), b.ctypes.data_as(P16), M, N, K, bn, splits, d.ctypes.data_as(FP)))
    return d


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round float32 to BF16 (nearest even) and return the 16-bit patterns."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    return (((a + 0x7FFF + ((a >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32)


# ---------------------------------------------------------------------------------------------
# Surrogate of the batched Monte Carlo

def reflectance_targets(ring_time: np.ndarray, floor: float = 1e-8) -> np.ndarray:
    """Network targets from MC tallies: log10 of the ring x time reflectance (fraction of launched
    weight per cell) with a floor below the MC's resolution; [n, rings * time]."""
    r = np.asarray(ring_time, dtype=np.float64).reshape(len(ring_time), -1)
    return np.log10(np.maximum(r, 0.0) + floor)


def relative_error(pred_log: np.ndarray, ref: np.ndarray, ref_w2: np.ndarray, photons: np.ndarray,
                   floor: float = 1e-8, max_ref_rse: float = 0.01) -> np.ndarray:
    """Per-cell |R_pred / R_ref - 1| on the cells whose reference is known to max_ref_rse (relative
    standard error from the tally of squared weights); other cells are NaN."""
    ref = np.asarray(ref, dtype=np.float64).reshape(len(ref), -1)
    w2 = np.asarray(ref_w2, dtype=np.float64).reshape(len(ref), -1)
    n = np.asarray(photons, dtype=np.float64)[:, None]
    # per-photon variance of the cell's score: E[w^2] - E[w]^2 (fractions of launched weight)
    var = np.maximum(w2 / n - ref * ref, 0.0) / n
    rse = np.sqrt(var) / np.maximum(ref, 1e-300)
    pred = 10.0 ** np.asarray(pred_log, dtype=np.float64) - floor
    err = np.abs(pred / np.maximum(ref, 1e-300) - 1.0)
    err[(ref <= 0) | (rse > max_ref_rse)] = np.nan
    return err


def he_uniform(rng: np.random.Generator, n_in: int, hidden: int, n_hidden: int, n_out: int) -> np.ndarray:
    """Initial parameters in the flat layout: He-uniform weights, zero biases."""
    dims = [n_in] + [hidden] * n_hidden + [n_out]
    parts = []
    for i in range(len(dims) - 1):
        lim = np.sqrt(6.0 / dims[i])
        parts += [rng.uniform(-lim, lim, dims[i + 1] * dims[i]), np.zeros(dims[i + 1])]
    return np.concatenate(parts).astype(np.float32)


class Surrogate:
    """Ensemble of MLPs over standardised features and targets, with the training hull and an
    ensemble-spread gate; `reflectance` falls back to the batched Monte Carlo where either check
    fails."""

    def __init__(self, n_in: int = 15, n_out: int = 1000, members: int = 4, hidden: int = 256, n_hidden: int = 4,
                 max_rows: int = 65536, device: int = 0, floor: float = 1e-8, gate: float = 0.02,
                 hull_margin: float = 0.0, gate_floor: float = 1e-5):
        self.members = [MLP(n_in, n_out, hidden, n_hidden, max_rows, device) for _ in range(members)]
        self.n_in, self.n_out, self.floor, self.gate, self.hull_margin = n_in, n_out, floor, gate, hull_margin
        self.gate_floor = gate_floor
        self.hidden, self.n_hidden = hidden, n_hidden
        self.x_mean = np.zeros(n_in); self.x_std = np.ones(n_in)
        self.y_mean = np.zeros(n_out); self.y_std = np.ones(n_out)
        self.lo = np.full(n_in, -np.inf); self.hi = np.full(n_in, np.inf)
        self.train_ms = 0.0

    # ---- training ----
    def fit(self, features: np.ndarray, targets: np.ndarray, steps: int = 4000, batch: int = 4096, lr: float = 2e-3,
            seed: int = 1, phases: int = 4, weighted: bool = False) -> List[np.ndarray]:
        """Standardise, then train every member from its own initialisation and minibatch stream
        with Adam; the learning rate drops by 3x at each of `phases` equal phases. With `weighted`,
        each output's squared error is weighted by the share of training rows in which it is above
        gate_floor (at least 0.05; mean 1), so that outputs the Monte Carlo rarely resolves do not
        dominate the fit. Returns the loss curves (standardised units)."""
        f = np.asarray(features, dtype=np.float64)
        y = np.asarray(targets, dtype=np.float64)
        self.x_mean, self.x_std = f.mean(0), f.std(0) + 1e-12
        self.y_mean, self.y_std = y.mean(0), y.std(0) + 1e-6
        self.lo, self.hi = f.min(0), f.max(0)
        xs = ((f - self.x_mean) / self.x_std).astype(np.float32)
        ys = ((y - self.y_mean) / self.y_std).astype(np.float32)
        w = None
        if weighted:
            share = np.mean(y > np.log10(max(self.gate_floor, self.floor)), axis=0)
            w = np.maximum(share, 0.05)
            w = w / w.mean()
        curves = []
        self.train_ms = 0.0
        for i, m in enumerate(self.members):
            rng = np.random.default_rng(seed * 1000 + i)
            m.set_params(he_uniform(rng, self.n_in, self.hidden, self.n_hidden, self.n_out))
            m.set_output_weights(w)
            m.set_dataset(xs, ys)
            curve = []
            per = max(1, steps // phases)
            done = 0
            for ph in range(phases):
                n = per if ph < phases - 1 else steps - done
                if n <= 0:
                    break
                losses, ms = m.train(n, batch=batch, lr=lr / 3 ** ph, seed=seed * 7919 + i)
                curve.append(losses)
                self.train_ms += ms
                done += n
            curves.append(np.concatenate(curve) if curve else np.zeros(0))
        return curves

    # ---- inference ----
    def in_hull(self, features: np.ndarray) -> np.ndarray:
        f = np.asarray(features, dtype=np.float64)
        span = self.hi - self.lo
        return np.all((f >= self.lo - self.hull_margin * span) & (f <= self.hi + self.hull_margin * span), axis=1)

    def predict(self, features: np.ndarray) -> Dict[str, np.ndarray]:
        """mean / spread of log10 reflectance over the ensemble, and the gate: in the training hull
        and median ensemble spread (in relative reflectance, ln 10 x std of log10) below `gate`."""
        f = np.asarray(features, dtype=np.float64)
        xs = ((f - self.x_mean) / self.x_std).astype(np.float32)
        outs, ms = [], 0.0
        for m in self.members:
            y, t = m.forward(xs)
            outs.append(y.astype(np.float64) * self.y_std + self.y_mean)
            ms += t
        stack = np.stack(outs)
        mean = stack.mean(0)
        spread = stack.std(0) * np.log(10.0) if len(outs) > 1 else np.zeros_like(mean)
        # the spread that matters is where the reflectance is well above the Monte Carlo's resolution
        sig = mean > np.log10(max(self.gate_floor, self.floor))
        med = np.array([np.median(s[g]) if g.any() else 0.0 for s, g in zip(spread, sig)])
        ok = self.in_hull(f) & (med <= self.gate)
        return {"log10_r": mean, "spread": med, "use_network": ok, "ms": ms}

    def reflectance(self, inst, batch=None, fallback_photons: int = 10 ** 6) -> Dict[str, np.ndarray]:
        """Ring x time reflectance [n, n_out] of the instances: from the network where the gate
        allows it, else from the batched Monte Carlo with `fallback_photons` photons each."""
        p = self.predict(inst.features())
        r = 10.0 ** p["log10_r"] - self.floor
        fb = np.nonzero(~p["use_network"])[0]
        if fb.size:
            from .batch import Batch
            own = batch is None
            b = batch or Batch(n_layers=inst.n_layers, max_instances=max(int(fb.size), 1))
            sub = inst.subset(fb).with_photons(fallback_photons)
            out = b.run(sub)
            r[fb] = out["ring_time"].reshape(len(fb), -1)
            if own:
                b.close()
        return {"reflectance": r, "from_network": p["use_network"], "spread": p["spread"]}

    # ---- inverse fitting ----
    def mean_log10(self, features: np.ndarray) -> np.ndarray:
        """Ensemble mean of log10 reflectance (no gate), for search loops."""
        xs = ((np.asarray(features, dtype=np.float64) - self.x_mean) / self.x_std).astype(np.float32)
        acc = None
        for m in self.members:
            y, _ = m.forward(xs)
            y = y.astype(np.float64) * self.y_std + self.y_mean
            acc = y if acc is None else acc + y
        return acc / len(self.members)

    def inverse_fit(self, target_log10: np.ndarray, start: np.ndarray, free: List[int], pop: int = 8192,
                    iters: int = 15, elite: float = 0.02, seed: int = 0, batch=None, verify_photons: int = 0,
                    refine: int = 16) -> Dict[str, object]:
        """Fit the `free` input features to a measured log10 reflectance with the network standing in for
        the Monte Carlo: a cross-entropy search (`pop` candidates per round, the best `elite` share
        refits a Gaussian), candidates kept inside the training hull, misfit = mean squared log10
        difference over the cells where the target is above gate_floor. With verify_photons > 0 the
        batched Monte Carlo checks the winner; when the winner fails the gate (ensemble spread), the
        Monte Carlo also ranks the `refine` best candidates of the last round and picks the best."""
        rng = np.random.default_rng(seed)
        t = np.asarray(target_log10, dtype=np.float64).ravel()
        mask = t > np.log10(max(self.gate_floor, self.floor))
        free = list(free)
        base = np.asarray(start, dtype=np.float64).copy()
        mu = self.x_mean[free].copy()
        sd = self.x_std[free].copy()
        lo, hi = self.lo[free], self.hi[free]
        best, best_loss, hist, evals = base.copy(), np.inf, [], 0
        cand = None
        for it in range(iters):
            cand = np.repeat(base[None, :], pop, axis=0)
            cand[:, free] = np.clip(rng.normal(mu, sd, (pop, len(free))), lo, hi)
            pred = self.mean_log10(cand)
            evals += pop
            loss = np.mean((pred[:, mask] - t[mask]) ** 2, axis=1)
            order = np.argsort(loss)
            k = max(2, int(elite * pop))
            el = cand[order[:k]][:, free]
            mu, sd = el.mean(0), np.maximum(el.std(0), 1e-4 * self.x_std[free])
            if loss[order[0]] < best_loss:
                best_loss, best = float(loss[order[0]]), cand[order[0]].copy()
            hist.append(best_loss)
        out = {"features": best, "loss_network": best_loss, "history": np.array(hist), "network_evals": evals}
        gate = self.predict(best[None, :])
        out["gated"] = bool(gate["use_network"][0])
        if verify_photons > 0:
            from .batch import from_features
            fb = best[None, :]
            if not out["gated"] and cand is not None:  # fallback: the Monte Carlo ranks the last round's best
                pred = self.mean_log10(cand)
                loss = np.mean((pred[:, mask] - t[mask]) ** 2, axis=1)
                fb = np.concatenate([best[None, :], cand[np.argsort(loss)[:refine]]])
            inst = from_features(fb, photons=verify_photons, seed=seed + 1)
            r = batch.run(inst)["ring_time"].reshape(len(fb), -1)
            mc_loss = np.mean((np.log10(r[:, mask] + self.floor) - t[mask]) ** 2, axis=1)
            j = int(np.argmin(mc_loss))
            out["features"], out["loss_mc"], out["mc_evals"] = fb[j], float(mc_loss[j]), len(fb)
        return out

    # ---- persistence ----
    def save(self, path: str) -> None:
        """Write the ensemble to an .npz file: the standardisation, the training hull, the gate
        settings, and per member the weights as BF16 bit patterns (the precision the tensor-core
        kernels compute in) and the biases in FP32."""
        dims = [self.n_in] + [self.hidden] * self.n_hidden + [self.n_out]
        arrays = {"dims": np.array(dims, dtype=np.int64), "x_mean": self.x_mean, "x_std": self.x_std,
                  "y_mean": self.y_mean, "y_std": self.y_std, "lo": self.lo, "hi": self.hi,
                  "settings": np.array([self.floor, self.gate, self.hull_margin, self.gate_floor])}
        for i, m in enumerate(self.members):
            p = m.get_params()
            w_parts, b_parts, o = [], [], 0
            for l in range(len(dims) - 1):
                nw = dims[l] * dims[l + 1]
                w_parts.append(p[o:o + nw]); o += nw
                b_parts.append(p[o:o + dims[l + 1]]); o += dims[l + 1]
            arrays[f"w{i}"] = to_bf16_bits(np.concatenate(w_parts))
            arrays[f"b{i}"] = np.concatenate(b_parts).astype(np.float32)
        np.savez_compressed(path, **arrays)

    @classmethod
    def load(cls, path: str, max_rows: int = 65536, device: int = 0) -> "Surrogate":
        """An ensemble written by `save`, ready for predict / reflectance / inverse_fit."""
        z = np.load(path)
        dims = [int(v) for v in z["dims"]]
        members = sum(1 for k in z.files if k.startswith("w"))
        floor, gate, hull_margin, gate_floor = (float(v) for v in z["settings"])
        sur = cls(n_in=dims[0], n_out=dims[-1], members=members, hidden=dims[1], n_hidden=len(dims) - 2,
                  max_rows=max_rows, device=device, floor=floor, gate=gate, hull_margin=hull_margin,
                  gate_floor=gate_floor)
        for k in ("x_mean", "x_std", "y_mean", "y_std", "lo", "hi"):
            setattr(sur, k, np.asarray(z[k], dtype=np.float64))
        for i, m in enumerate(sur.members):
            w = from_bf16_bits(z[f"w{i}"])
            b = np.asarray(z[f"b{i}"], dtype=np.float32)
            parts, ow, ob = [], 0, 0
            for l in range(len(dims) - 1):
                nw = dims[l] * dims[l + 1]
                parts += [w[ow:ow + nw], b[ob:ob + dims[l + 1]]]
                ow += nw
                ob += dims[l + 1]
            m.set_params(np.concatenate(parts))
        return sur

    def close(self):
        for m in self.members:
            m.close()
