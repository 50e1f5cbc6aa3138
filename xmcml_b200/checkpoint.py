"""Checkpoint / resume of a long transport run.

With a counter-based RNG the state of a run is small and exact: the seed, the next photon id, and
the integer (2^31 fixed point) tallies accumulated so far. A run of N photons is cut into portions
[first, first + portion) on one device context; after each portion the tallies are added (64-bit
integer sums, exact in any order) and the state is written atomically (temporary file + rename).
Resuming from the file continues at the next photon id, so an interrupted and resumed run gives
bit-identical tallies to an uninterrupted one. The reference's backup files
(base/xmcml/xmcmlLauncher/reader.cpp, writer.cpp backups in launcher_mpi.cpp:357-380) store FP64
partial outputs and the MCG59 states instead; its reader is broken in `base` and is not mirrored.
"""
from __future__ import annotations

import os
import tempfile
from typing import Callable, Dict, Optional

import numpy as np

FORMAT = 1
LEDGER_KEYS = ("photons_launched", "photons_terminated", "steps", "n_escaped_top", "n_escaped_bottom", "n_area",
               "n_cut", "n_roulette", "n_glass", "n_budget", "n_invalid", "n_detected", "specular_fx",
               "absorbed_fx", "absorbed_outside_fx", "escaped_top_fx", "escaped_bottom_fx", "lost_area_fx",
               "lost_cut_fx", "lost_glass_fx", "lost_budget_fx", "lost_invalid_fx", "roulette_killed_fx",
               "roulette_gained_fx", "absorbed_target_fx")


class RunState:
    """Seed, progress and accumulated integer tallies of a portioned run."""

    def __init__(self, seed: int, total: int, portion: int):
        if total < 0 or portion <= 0:
            raise ValueError("total must be >= 0 and portion > 0")
        self.seed, self.total, self.portion = int(seed), int(total), int(portion)
        self.next_id = 0
        self.tallies: Dict[str, np.ndarray] = {}
        self.ledger = {k: 0 for k in LEDGER_KEYS}

    @property
    def done(self) -> bool:
        return self.next_id >= self.total

    def add(self, tallies: Dict[str, np.ndarray], ledger: dict, n: int) -> None:
        for k, v in tallies.items():
            v = np.asarray(v, dtype=np.uint64)
            if k in self.tallies:
                self.tallies[k] = self.tallies[k] + v  # uint64 wrap-around never reached: < 2^63 by design
            else:
                self.tallies[k] = v.copy()
        for k in LEDGER_KEYS:
            self.ledger[k] += int(ledger.get(k, 0))
        self.next_id += int(n)

    # ---- file ----
    def save(self, path: str) -> None:
        d = os.path.dirname(os.path.abspath(path))
        fd, tmp = tempfile.mkstemp(prefix=".ckpt_", dir=d)
        os.close(fd)
        arrays = {"t_" + k: v for k, v in self.tallies.items()}
        led = np.array([self.ledger[k] for k in LEDGER_KEYS], dtype=np.uint64)
        meta = np.array([FORMAT, self.seed, self.total, self.portion, self.next_id], dtype=np.uint64)
        with open(tmp, "wb") as f:
            np.savez(f, meta=meta, ledger=led, **arrays)
            f.flush()
            os.fsync(f.fileno())
        os.replace(tmp, path)

    @classmethod
    def load(cls, path: str) -> "RunState":
        with np.load(path) as z:
            meta = z["meta"]
            if int(meta[0]) != FORMAT:
                raise ValueError(f"checkpoint format {int(meta[0])} is not {FORMAT}")
            st = cls(int(meta[1]), int(meta[2]), int(meta[3]))
            st.next_id = int(meta[4])
            led = z["ledger"]
            st.ledger = {k: int(led[i]) for i, k in enumerate(LEDGER_KEYS)}
            st.tallies = {k[2:]: z[k].copy() for k in z.files if k.startswith("t_")}
        if st.next_id > st.total:
            raise ValueError("checkpoint is past its own total")
        return st


def run_portions(transport, state: RunState, path: Optional[str] = None,
                 after_portion: Optional[Callable[[RunState], None]] = None) -> RunState:
    """Run the remaining portions of `state` on `transport` (an api.Transport or anything with
    run(n, seed, first_photon) -> ledger dict and tallies() -> dict of uint64 arrays), saving after
    each portion when `path` is given. `after_portion` is called after each save (tests use it to
    stop a run part-way, as a crash would)."""
    while not state.done:
        n = min(state.portion, state.total - state.next_id)
        led = transport.run(n, seed=state.seed, first_photon=state.next_id)
        state.add(transport.tallies(), led, n)
        if path:
            state.save(path)
        if after_portion:
            after_portion(state)
    return state
