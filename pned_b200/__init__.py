"""pned_b200 -- B200 (sm_100a) implementation of pNED's matrix-free H.v and the
Krylov loops built on it (Lanczos, mTPQ/TPS, DSF continued fractions, CG).

The compute runs in libpned_gpu.so (hand-written CUDA, C ABI in
include/pned_gpu.h); this package is the Python host side over that ABI.
"""
from . import couplings, lattice  # noqa: F401
from ._capi import PnedError, lib  # noqa: F401
from .api import (Context, Model, ModelInput, ObservableSpec, SlotBatch, bisec, build_xlocal,  # noqa: F401
                  exec_renbun, hv_noalloc, mk_list12, normalize_dsf, tps_transform, vec12)

__all__ = ["Context", "Model", "ModelInput", "ObservableSpec", "SlotBatch", "PnedError", "bisec", "build_xlocal", "couplings", "exec_renbun", "hv_noalloc",
           "lattice", "lib", "mk_list12", "normalize_dsf", "tps_transform", "vec12"]
