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
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import structs as S
from ._lib import check, load

FP = C.POINTER(C.c_float)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def pad_rows(n: int) -> int:
    return (n + 127) // 128 * 128


class MLP:
    """n_in -> hidden x n_hidden (SiLU) -> n_out network on one GPU."""

    def __init__(self, n_in: int, n_out: int, hidden: int = 256, n_hidden: int = 4, max_rows: int = 65536,
                 device: int = 0):
        self._lib = load()
        s = S.MlpSpec()
        s.struct_size = C.sizeof(S.MlpSpec)
        s.n_in, s.hidden, s.n_hidden, s.n_out, s.max_rows, s.device = n_in, hidden, n_hidden, n_out, max_rows, device
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
            y = np.zeros((rp, self.n_out), dtype=np.float32)
            t = C.c_double(0.0)
            check(self._lib.xmc_mlp_forward(self._m, xb.ctypes.data_as(FP), rp, y.ctypes.data_as(FP), C.byref(t)))
            outs.append(y[:r])
            ms += t.value
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
