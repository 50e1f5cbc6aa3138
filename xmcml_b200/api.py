"""Python host interface over the C-ABI (ctypes), mirroring the reference launcher's calls:

    ParseInputFile / ParseSurfaceFile   -> Model(xml, surface)
    InitOutput / FreeOutput             -> Output(model)
    LaunchOMP(input, output, rng, n)    -> launch_omp(model, output, rng)
    WriteOutputToFile                   -> Output.write(path)

plus Transport, a persistent device context (xmc_create / xmc_run / xmc_destroy) for repeated runs
with the tallies read back as numpy arrays. All compute goes through libxmcml_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import structs as S
from ._lib import XmcError, check, last_error, load

WEIGHT_SCALE = float(2 ** 31)


class Model:
    """A tissue model parsed from the reference's XML + .surface files (InputInfo owned by the library)."""

    def __init__(self, xml_path: str, surface_path: str):
        self._lib = load()
        self.info = S.InputInfo()
        if not self._lib.xmc_parse_input_file(xml_path.encode(), C.byref(self.info)):
            err = last_error()
            self._lib.xmc_free_input(C.byref(self.info))
            raise XmcError(S.XMC_ERR_IO, err)
        if not self._lib.xmc_parse_surface_file(surface_path.encode(), C.byref(self.info)):
            err = last_error()
            self._lib.xmc_free_input(C.byref(self.info))
            raise XmcError(S.XMC_ERR_IO, err)
        self._open = True

    @property
    def n_detectors(self) -> int:
        return self.info.numberOfCubeDetectors + self.info.numberOfRingDetectors

    @property
    def grid_shape(self):
        p = self.info.area.contents.partitionNumber
        return (p.x, p.y, p.z)

    def close(self):
        if getattr(self, "_open", False):
            self._lib.xmc_free_input(C.byref(self.info))
            self._open = False

    def __del__(self):
        self.close()


class Output:
    """OutputInfo allocated like the reference's InitOutput (launcher_omp.cpp:10-58)."""

    def __init__(self, model: Model):
        self._lib = load()
        self.info = S.OutputInfo()
        self._lib.xmc_init_output(C.byref(model.info), C.byref(self.info))
        self._model = model
        self._open = True

    @property
    def absorption(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.info.absorption, shape=(self.info.gridSize,))

    def detector_weights(self) -> np.ndarray:
        return np.array([self.info.detectorInfo[i].weight for i in range(self.info.numberOfDetectors)])

    def detector_counts(self) -> np.ndarray:
        return np.array([self.info.detectorInfo[i].numberOfPhotons for i in range(self.info.numberOfDetectors)],
                        dtype=np.uint64)

    def detector_target_weights(self) -> np.ndarray:
        return np.array([self.info.detectorInfo[i].targetWeight for i in range(self.info.numberOfDetectors)])

    def time_weights(self) -> np.ndarray:
        D = self.info.numberOfDetectors
        if D == 0:
            return np.zeros((0, 0))
        T = self.info.detectorInfo[0].timeScaleSize
        return np.array([[self.info.detectorInfo[d].timeScale[j].weight for j in range(T)] for d in range(D)])

    def write(self, path: str) -> None:
        if not self._lib.xmc_write_output_file(C.byref(self._model.info), C.byref(self.info), path.encode()):
            raise XmcError(S.XMC_ERR_IO, last_error())

    def close(self):
        if getattr(self, "_open", False):
            self._lib.xmc_free_output(C.byref(self.info))
            self._open = False

    def __del__(self):
        self.close()


def options(roulette: bool = False, area_kill: bool = True, beam_radius: float = 0.0, chance: float = 0.1,
            device: int = 0, block_size: int = 0, blocks_per_sm: int = 0, photons_per_chunk: int = 0,
            smem_nodes: int = 0, max_steps: int = 0, large_grid: bool = False, scattering: bool = False,
            trajectories: bool = False, trajectory_log: int = 0, gpu_bvh: bool = False,
            lane_queries: bool = False, query_batch: int = 0, grid_cell_tris: int = 0) -> S.XmcOptions:
    o = S.XmcOptions()
    load().xmc_default_options(C.byref(o))
    o.flags = (S.XMC_ROULETTE if roulette else 0) | (0 if area_kill else S.XMC_NO_AREA_KILL) | \
              (S.XMC_LARGE_GRID if large_grid else 0) | (S.XMC_SCATTERING_MAP if scattering else 0) | \
              (S.XMC_DETECTOR_TRAJ if trajectories else 0) | (S.XMC_GPU_BVH if gpu_bvh else 0) | \
              (S.XMC_LANE_QUERIES if lane_queries else 0)
    o.roulette_chance = chance
    o.beam_radius = beam_radius
    o.device = device
    o.block_size = block_size
    o.blocks_per_sm = blocks_per_sm
    if photons_per_chunk:
        o.photons_per_chunk = photons_per_chunk
    o.smem_nodes = smem_nodes
    o.trajectory_log = trajectory_log
    o.query_batch = query_batch
    o.grid_cell_tris = grid_cell_tris
    if max_steps:
        o.max_steps_per_photon = max_steps
    return o


class Transport:
    """Persistent device context of one model: geometry, BVH and tallies resident on the GPU."""

    def __init__(self, model: Model, opts: Optional[S.XmcOptions] = None, **kw):
        self._lib = load()
        self.model = model
        self.opts = opts if opts is not None else options(**kw)
        self._ctx = C.c_void_p()
        check(self._lib.xmc_create(C.byref(model.info), C.byref(self.opts), C.byref(self._ctx)))
        self.n_dets = model.n_detectors
        self.n_time = model.info.timeScaleSize
        self.grid = int(np.prod(model.grid_shape))

    def run(self, n: int, seed: int = 777, first_photon: int = 0, output: Optional[Output] = None,
            allow_budget: bool = False) -> dict:
        led = S.XmcLedger()
        st = self._lib.xmc_run(self._ctx, seed, first_photon, n, C.byref(output.info) if output else None,
                               C.byref(led))
        if st != S.XMC_OK and not (allow_budget and st == S.XMC_ERR_BUDGET):
            raise XmcError(st, last_error())
        return led.as_dict()

    def tallies(self) -> dict:
        D, T = max(self.n_dets, 1), self.n_time
        arr = {k: np.zeros(s, dtype=np.uint64) for k, s in [
            ("absorption", self.grid), ("det_weight", D), ("det_count", D), ("det_target", D), ("det_weight2", D),
            ("time_weight", D * T), ("time_count", D * T), ("time_target", D * T), ("time_weight2", D * T)]}
        P = C.POINTER(C.c_uint64)
        ptrs = [a.ctypes.data_as(P) for a in arr.values()]
        check(self._lib.xmc_read_tallies(self._ctx, *ptrs))
        for k in ("time_weight", "time_count", "time_target", "time_weight2"):
            arr[k] = arr[k].reshape(D, T)
        return arr

    def maps(self) -> dict:
        """Scattering map [grid] (weight fixed point) and trajectory maps [detectors, grid] (counts)."""
        res = {}
        P = C.POINTER(C.c_uint64)
        if self.opts.flags & S.XMC_SCATTERING_MAP:
            a = np.zeros(self.grid, dtype=np.uint64)
            check(self._lib.xmc_read_maps(self._ctx, a.ctypes.data_as(P), None))
            res["scattering"] = a
        if self.opts.flags & S.XMC_DETECTOR_TRAJ:
            a = np.zeros(max(self.n_dets, 1) * self.grid, dtype=np.uint64)
            check(self._lib.xmc_read_maps(self._ctx, None, a.ctypes.data_as(P)))
            res["trajectory"] = a.reshape(max(self.n_dets, 1), self.grid)
        return res

    def cancel(self):
        self._lib.xmc_cancel(self._ctx)

    def close(self):
        if self._ctx:
            self._lib.xmc_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(model: Model, sample_photons: int = 1_000_000, **kw) -> tuple:
    """The transport kernel's fastest launch shape for `model` (xmc_autotune): options built from
    `kw` (semantics, maps, device) with the tuned block size, photons per warp claim and query
    scheme, and the sample's kernel ms."""
    base = options(**kw)
    best = S.XmcOptions()
    ms = C.c_double(0.0)
    check(load().xmc_autotune(C.byref(model.info), C.byref(base), sample_photons, C.byref(best), C.byref(ms)))
    return best, ms.value


def launch_set_options(opts: Optional[S.XmcOptions]) -> None:
    """Options xmc_launch_omp uses from now on (e.g. autotune's result); None restores the defaults."""
    check(load().xmc_launch_set_options(C.byref(opts) if opts is not None else None))


def launch_omp(model: Model, output: Output, rng: S.MCG59, num_threads: int = 0) -> int:
    """LaunchOMP(InputInfo*, OutputInfo*, MCG59*, int) on the GPU (launcher_omp.cpp:123-163)."""
    st = load().xmc_launch_omp(C.byref(model.info), C.byref(output.info), C.byref(rng), num_threads)
    if st not in (S.XMC_OK, S.XMC_ERR_BUDGET):
        raise XmcError(st, last_error())
    return st


def mcg59_init(seed: int, ident: int = 0, step: int = 1) -> S.MCG59:
    """InitMCG59 (base/xmcml/xmcml/mcml_mcg59.cpp:24-32) in Python integers."""
    C59 = 302875106592253
    M = (1 << 59) - 1
    g = S.MCG59()
    g.value = ((2 * seed + 1) * pow(C59, ident, 1 << 64)) & M
    g.offset = pow(C59, step, 1 << 64)
    return g
