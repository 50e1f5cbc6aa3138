"""xmcml_b200: xMCML's photon-transport hot path (LaunchOMP -> ComputePhoton) on one B200 GPU.

The compute path is libxmcml_b200.so (hand-written sm_100a CUDA behind a C-ABI, include/xmcml_b200.h);
this package is the Python host interface over it (ctypes) and the synthetic-input generators.
"""
from . import structs
from ._lib import XmcError, load
from .api import Model, Output, Transport, launch_omp, mcg59_init, options

__all__ = ["structs", "XmcError", "load", "Model", "Output", "Transport", "launch_omp", "mcg59_init", "options"]
