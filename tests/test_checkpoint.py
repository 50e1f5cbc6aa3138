"""Checkpoint / resume of portioned runs (host logic, no GPU): a fake transport whose tallies are
a deterministic function of the photon ids stands in for the device, and a run stopped part-way
by an exception (as a crash would stop it) and resumed from its file gives the same integer tallies
and ledger as an uninterrupted run."""
import numpy as np
import pytest

from xmcml_b200 import checkpoint as CK


class FakeTransport:
    """Tallies of photons [first, first + n): per-id values hashed from (seed, id)."""

    def __init__(self):
        self._t = None
        self.calls = []

    def run(self, n, seed, first_photon):
        self.calls.append((first_photon, n))
        ids = np.arange(first_photon, first_photon + n, dtype=np.uint64)
        h = (ids * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)) >> np.uint64(40)
        self._t = {"absorption": np.bincount((h % np.uint64(97)).astype(np.int64), minlength=97).astype(np.uint64) * 3,
                   "det_weight": np.array([int(h.sum() % (1 << 40))], dtype=np.uint64)}
        return {"photons_launched": n, "photons_terminated": n, "steps": int(h.sum() % 100000), "absorbed_fx": int(n) * 5}

    def tallies(self):
        return self._t


class Crash(RuntimeError):
    pass


def test_resume_equals_uninterrupted(tmp_path):
    full = CK.run_portions(FakeTransport(), CK.RunState(seed=77, total=10_000, portion=1_500))
    path = str(tmp_path / "run.ckpt")

    def crash_after_3(st):
        if st.next_id >= 3 * 1500:
            raise Crash()

    with pytest.raises(Crash):
        CK.run_portions(FakeTransport(), CK.RunState(seed=77, total=10_000, portion=1_500), path, crash_after_3)
    st = CK.RunState.load(path)
    assert st.next_id == 4500 and not st.done
    t2 = FakeTransport()
    res = CK.run_portions(t2, st, path)
    assert t2.calls[0] == (4500, 1500) and t2.calls[-1] == (9000, 1000)
    assert res.done and res.next_id == 10_000
    for k in full.tallies:
        assert np.array_equal(full.tallies[k], res.tallies[k])
    assert full.ledger == res.ledger
    again = CK.RunState.load(path)
    assert again.done and again.ledger == full.ledger


def test_checkpoint_rejects_bad_files(tmp_path):
    st = CK.RunState(1, 100, 10)
    p = str(tmp_path / "a.ckpt")
    st.save(p)
    with np.load(p) as z:
        arrs = dict(z)
    arrs["meta"] = arrs["meta"].copy()
    arrs["meta"][0] = 99
    with open(p, "wb") as f:
        np.savez(f, **arrs)
    with pytest.raises(ValueError):
        CK.RunState.load(p)
    with pytest.raises(ValueError):
        CK.RunState(1, -1, 10)
