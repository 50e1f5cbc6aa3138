"""ORACLE — TEST INFRASTRUCTURE ONLY: ctypes bindings of the FP64 oracle (liboracle.so) and of the
reference build (_ref/libxmcml_ref.so). Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py; never by the xmcml_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from xmcml_b200 import structs as S

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libxmcml_ref.so")
REF_FAST_LIB = os.path.join(HERE, "_ref", "libxmcml_ref_fast.so")

RNG_MCG59 = 0
RNG_PHILOX = 1
OFLAG_ROULETTE = 1 << 0
OFLAG_NO_AREA_KILL = 1 << 1
OFLAG_SCATTERING = 1 << 2
OFLAG_TRAJECTORY = 1 << 3


class OracleOpts(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("rng_kind", C.c_int32), ("roulette_chance", C.c_double),
                ("beam_radius", C.c_double), ("max_steps", C.c_uint64), ("nthreads", C.c_int32), ("pad", C.c_int32)]


_CNT = ["launched", "terminated", "steps", "n_escaped_top", "n_escaped_bottom", "n_area", "n_cut", "n_roulette",
        "n_glass", "n_budget", "n_invalid", "n_detected"]
_TERMS = ["specular", "absorbed", "absorbed_outside", "escaped_top", "escaped_bottom", "lost_area", "lost_cut",
          "lost_glass", "lost_budget", "lost_invalid", "roulette_killed", "roulette_gained"]


class OracleLedger(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in _CNT] + [(n, C.c_double) for n in _TERMS] + [("absorbed_target", C.c_double), ("bias_gained", C.c_double),
                                                                                   ("bias_lost", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


def build(force: bool = False) -> None:
    """Build liboracle.so, and _ref when the environment variable XMC_REFERENCE_DIR names a reference
    checkout that is present."""
    ref_dir = os.environ.get("XMC_REFERENCE_DIR", "")
    with_ref = bool(ref_dir) and os.path.isdir(ref_dir)
    targets = ["oracle"] + (["ref", f"REF={ref_dir}"] if with_ref else [])
    cmd = ["make", "-C", HERE] + (["-B"] if force else []) + targets
    subprocess.run(cmd, check=True, capture_output=True)


_oracle = None
_ref = {}


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        lib = C.CDLL(ORACLE_LIB)
        P = C.POINTER
        D = C.c_double
        pd = P(C.c_double)
        lib.oracle_run.restype = C.c_int
        lib.oracle_run.argtypes = [P(S.InputInfo), P(S.OutputInfo), P(OracleOpts), C.c_uint64, C.c_uint64, C.c_uint64,
                                   P(S.MCG59), P(OracleLedger), pd, pd]
        lib.oracle_default_opts.argtypes = [P(OracleOpts)]
        lib.oracle_mcg59_init.argtypes = [P(S.MCG59), C.c_uint64, C.c_uint32, C.c_uint32]
        lib.oracle_mcg59_next.restype = D
        lib.oracle_mcg59_next.argtypes = [P(S.MCG59)]
        lib.oracle_philox4x32_10.argtypes = [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
        lib.oracle_specular_reflectance.restype = D
        lib.oracle_specular_reflectance.argtypes = [P(S.LayerInfo)]
        lib.oracle_hg_cos.restype = D
        lib.oracle_hg_cos.argtypes = [D, D]
        lib.oracle_transmit_cos.restype = D
        lib.oracle_transmit_cos.argtypes = [D, D, D]
        lib.oracle_fresnel.restype = D
        lib.oracle_fresnel.argtypes = [D, D, D, D]
        lib.oracle_critical_cos.restype = D
        lib.oracle_critical_cos.argtypes = [P(S.LayerInfo), C.c_int, C.c_int]
        lib.oracle_find_layer.restype = C.c_int
        lib.oracle_find_layer.argtypes = [P(S.InputInfo), C.c_int, C.c_int]
        lib.oracle_area_index.restype = C.c_int
        lib.oracle_kat_cosine_theta.restype = D
        lib.oracle_kat_cosine_theta.argtypes = [D, P(S.MCG59)]
        lib.oracle_kat_new_direction.argtypes = [pd, D, P(S.MCG59), pd]
        lib.oracle_kat_step_size.restype = D
        lib.oracle_kat_step_size.argtypes = [D, D, P(S.MCG59)]
        lib.oracle_kat_drop.restype = D
        lib.oracle_kat_drop.argtypes = [D, D, D, pd]
        lib.oracle_kat_area_index.restype = D
        lib.oracle_kat_area_index.argtypes = [pd, P(S.Area)]
        lib.oracle_kat_triangle.restype = D
        lib.oracle_kat_triangle.argtypes = [pd, pd, pd, pd, pd]
        lib.oracle_kat_reflect.argtypes = [pd, pd, pd]
        lib.oracle_kat_refract.argtypes = [D, D, pd, pd, pd]
        lib.oracle_detector_id.restype = C.c_int
        lib.oracle_detector_id.argtypes = [P(S.InputInfo), S.double3, S.double3, P(C.c_bool)]
        lib.oracle_kat_nearest_batch.restype = C.c_int
        lib.oracle_kat_nearest_batch.argtypes = [P(S.InputInfo), C.c_int, pd, D, C.c_int, pd, P(C.c_int), pd]
        lib.oracle_weight_integral.restype = D
        lib.oracle_weight_integral.argtypes = [D, D, D, C.c_uint]
        lib.oracle_weight_tables.restype = C.c_int
        lib.oracle_weight_tables.argtypes = [P(S.InputInfo)]
        lib.oracle_free_weight_tables.argtypes = [P(S.InputInfo)]
        lib.oracle_kat_nearest.restype = C.c_int
        lib.oracle_kat_nearest.argtypes = [P(S.InputInfo), pd, pd, D, C.c_int, pd, P(C.c_int), pd]
        _oracle = lib
    return _oracle


def ref_available(fast: bool = False) -> bool:
    return os.path.exists(REF_FAST_LIB if fast else REF_LIB)


def ref(fast: bool = False) -> C.CDLL:
    key = "fast" if fast else "pin"
    if key not in _ref:
        path = REF_FAST_LIB if fast else REF_LIB
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing (the reference build needs the reference sources)")
        lib = C.CDLL(path)
        P = C.POINTER
        D = C.c_double
        pd = P(C.c_double)
        lib.ref_parse_input.restype = C.c_int
        lib.ref_parse_input.argtypes = [C.c_char_p, P(S.InputInfo)]
        lib.ref_parse_surface.restype = C.c_int
        lib.ref_parse_surface.argtypes = [C.c_char_p, P(S.InputInfo)]
        lib.ref_dummy_weight_table.argtypes = [P(S.InputInfo)]
        lib.ref_init_output.argtypes = [P(S.InputInfo), P(S.OutputInfo)]
        lib.ref_free_output.argtypes = [P(S.OutputInfo)]
        lib.ref_generate_bvh.argtypes = [P(S.InputInfo)]
        lib.ref_init_mcg59.argtypes = [P(S.MCG59), C.c_uint64, C.c_uint, C.c_uint]
        lib.ref_next_mcg59.restype = D
        lib.ref_next_mcg59.argtypes = [P(S.MCG59)]
        lib.ref_init_threads_mcg59.argtypes = [P(S.MCG59), C.c_uint64, C.c_int]
        lib.ref_launch_omp.argtypes = [P(S.InputInfo), P(S.OutputInfo), P(S.MCG59), C.c_int]
        lib.ref_write_output.restype = C.c_int
        lib.ref_write_output.argtypes = [P(S.InputInfo), P(S.OutputInfo), C.c_char_p]
        lib.ref_specular.restype = D
        lib.ref_specular.argtypes = [P(S.LayerInfo)]
        lib.ref_cosine_theta.restype = D
        lib.ref_cosine_theta.argtypes = [D, P(S.MCG59)]
        lib.ref_new_direction.argtypes = [pd, D, P(S.MCG59), pd]
        lib.ref_transmit_cos.restype = D
        lib.ref_transmit_cos.argtypes = [D, D, D]
        lib.ref_fresnel.restype = D
        lib.ref_fresnel.argtypes = [D, D, D, D]
        lib.ref_critical_cos.restype = D
        lib.ref_critical_cos.argtypes = [P(S.LayerInfo), C.c_int, C.c_int]
        lib.ref_find_layer.restype = C.c_int
        lib.ref_find_layer.argtypes = [P(S.InputInfo), C.c_int, C.c_int]
        lib.ref_step_size.restype = D
        lib.ref_step_size.argtypes = [D, D, P(S.MCG59)]
        lib.ref_drop.restype = D
        lib.ref_drop.argtypes = [D, D, D, pd]
        lib.ref_area_index.restype = D
        lib.ref_area_index.argtypes = [pd, P(S.Area)]
        lib.ref_triangle.restype = D
        lib.ref_triangle.argtypes = [pd, pd, pd, pd, pd]
        lib.ref_reflect.argtypes = [pd, pd, pd]
        lib.ref_refract.argtypes = [D, D, pd, pd, pd]
        lib.ref_detector_id.restype = C.c_int
        lib.ref_detector_id.argtypes = [P(S.InputInfo), pd, pd, P(C.c_ubyte)]
        lib.ref_bvh_intersection.restype = C.c_int
        lib.ref_bvh_intersection.argtypes = [P(S.InputInfo), pd, pd, D, C.c_int, pd, P(C.c_int), pd]
        lib.ref_layout_offsets.restype = C.c_int
        lib.ref_layout_offsets.argtypes = [P(C.c_int64), C.c_int]
        _ref[key] = lib
    return _ref[key]


def default_opts(**kw) -> OracleOpts:
    o = OracleOpts()
    oracle().oracle_default_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def ref_load_model(xml: str, surface: str, fast: bool = False) -> S.InputInfo:
    """ParseInputFile + ParseSurfaceFile + the dummy weight table, as main.cpp:87-153 does."""
    lib = ref(fast)
    info = S.InputInfo()
    if not lib.ref_parse_input(xml.encode(), C.byref(info)):
        raise RuntimeError("reference ParseInputFile failed")
    if not lib.ref_parse_surface(surface.encode(), C.byref(info)):
        raise RuntimeError("reference ParseSurfaceFile failed")
    if info.useBiasing:  # the reference's own weight tables (weight_integral.cpp:34-65), as its launcher makes them
        lib.ref_weight_tables.argtypes = [C.POINTER(S.InputInfo), C.c_int]
        lib.ref_weight_tables(C.byref(info), os.cpu_count() or 1)
    else:
        lib.ref_dummy_weight_table(C.byref(info))
    return info


def ref_new_output(info: S.InputInfo, fast: bool = False) -> S.OutputInfo:
    out = S.OutputInfo()
    ref(fast).ref_init_output(C.byref(info), C.byref(out))
    return out


def ref_launch(info: S.InputInfo, out: S.OutputInfo, seed: int, nthreads: int, fast: bool = False,
               n: Optional[int] = None) -> None:
    """GenerateBVHTree (once) + per-thread MCG59 init (main.cpp:105-112) + LaunchOMP."""
    lib = ref(fast)
    if not info.bvhTree:
        lib.ref_generate_bvh(C.byref(info))
    if n is not None:
        info.numberOfPhotons = n
    gens = (S.MCG59 * max(1, nthreads))()
    lib.ref_init_threads_mcg59(gens, seed, nthreads)
    lib.ref_launch_omp(C.byref(info), C.byref(out), gens, nthreads)


def output_arrays(out: S.OutputInfo, with_traj: bool = False) -> dict:
    """Copy of an OutputInfo's tallies as numpy arrays."""
    G, D = out.gridSize, out.numberOfDetectors
    res = {
        "specular": out.specularReflectance,
        "absorption": np.ctypeslib.as_array(out.absorption, shape=(G,)).copy(),
        "scattering": np.ctypeslib.as_array(out.scattering, shape=(G,)).copy(),
        "det_weight": np.array([out.detectorInfo[i].weight for i in range(D)]),
        "det_count": np.array([out.detectorInfo[i].numberOfPhotons for i in range(D)], dtype=np.uint64),
        "det_target": np.array([out.detectorInfo[i].targetWeight for i in range(D)]),
    }
    T = out.detectorInfo[0].timeScaleSize if D else 0
    res["time_weight"] = np.array([[out.detectorInfo[d].timeScale[j].weight for j in range(T)] for d in range(D)])
    res["time_count"] = np.array([[out.detectorInfo[d].timeScale[j].numberOfPhotons for j in range(T)] for d in range(D)],
                                 dtype=np.uint64)
    res["time_target"] = np.array([[out.detectorInfo[d].timeScale[j].targetWeight for j in range(T)] for d in range(D)])
    if with_traj:
        res["trajectory"] = np.stack([np.ctypeslib.as_array(out.detectorInfo[d].trajectory, shape=(G,)).copy()
                                      for d in range(D)]) if D else np.zeros((0, G), dtype=np.uint64)
    return res


def oracle_run(info: S.InputInfo, out: S.OutputInfo, opts: OracleOpts, seed: int = 777, first: int = 0,
               n: Optional[int] = None, mcg: Optional[S.MCG59] = None):
    """Run the FP64 oracle; returns (ledger dict, det_w2, time_w2)."""
    lib = oracle()
    n = info.numberOfPhotons if n is None else n
    D = out.numberOfDetectors
    T = out.detectorInfo[0].timeScaleSize if D else 1
    dw2 = np.zeros(max(D, 1))
    tw2 = np.zeros(max(D * T, 1))
    led = OracleLedger()
    g = mcg
    if g is None:
        g = S.MCG59()
        lib.oracle_mcg59_init(C.byref(g), seed, 0, 1)
    pd = C.POINTER(C.c_double)
    lib.oracle_run(C.byref(info), C.byref(out), C.byref(opts), seed, first, n, C.byref(g), C.byref(led),
                   dw2.ctypes.data_as(pd), tw2.ctypes.data_as(pd))
    return led.as_dict(), dw2[:D], tw2[:D * T].reshape(D, T) if D else tw2[:0]
