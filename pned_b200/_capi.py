"""ctypes bindings of libpned_gpu.so (the C ABI of include/pned_gpu.h).

The library is built in-tree (pned_b200/build.py).  Loading fails loudly when
it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpned_gpu.so")

PNED_OK = 0
ERRORS = {1: "EINVAL", 2: "ENOMEM", 3: "EBUDGET", 4: "EBREAKDOWN", 5: "ECUDA", 6: "ETIMEOUT", 7: "ENOTSUP"}
PTR_HOST = 0
PTR_DEVICE = 1


class c128(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class ModelDesc(C.Structure):
    _fields_ = [
        ("n_sites", C.c_int32), ("q_spin", C.c_int32), ("tree", C.c_int32), ("n_bonds", C.c_int32),
        ("ipair", C.POINTER(C.c_int32)), ("bond_type", C.POINTER(C.c_int32)),
        ("xlocal", C.c_void_p), ("skip", C.POINTER(C.c_uint8)),
        ("parity_type", C.c_int32), ("total_sz", C.c_int32),
    ]


class DumpInfo(C.Structure):
    """pned_dump_info: the .info file of interval_dump."""
    _fields_ = [("dump_name", C.c_char * 128), ("np", C.c_int32), ("position", C.c_int32 * 7),
                ("max_itr", C.c_int32), ("dsf_comp", C.c_char * 2), ("s_maxitr", C.c_int32), ("n", C.c_int32),
                ("ibond", C.c_int32), ("nvec", C.c_int32), ("total_sz", C.c_int32),
                ("itr_counter", C.c_int32 * 12)]


class DumpData(C.Structure):
    """pned_dump_data: the arrays of interval_dump's data file (null pointers: absent)."""
    _fields_ = [("data_size", C.c_int32), ("vec_size", C.c_int32),
                ("sa", C.POINTER(C.c_double)), ("sb", C.POINTER(C.c_double)), ("sc", C.POINTER(C.c_double)),
                ("se", C.POINTER(C.c_double)), ("n_sa", C.c_int64), ("n_sb", C.c_int64), ("n_sc", C.c_int64),
                ("n_se", C.c_int64), ("vec", C.c_void_p * 5)]


class TilePlan(C.Structure):
    _fields_ = [("row_fixed_bits", C.c_int32), ("window_bits", C.c_int32), ("max_passes", C.c_int32),
                ("j_bits", C.c_int32), ("l1_carveout", C.c_int32), ("stage_partner_tiles", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("objective", C.c_int32),
                ("terms_in_flight", C.c_int32)]


class Observable(C.Structure):
    _fields_ = [
        ("n_terms", C.c_int32), ("a", C.POINTER(C.c_int32)), ("b", C.POINTER(C.c_int32)),
        ("c", C.c_void_p), ("T", c128 * 4),
    ]


class PnedError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pned error {ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None

EXPORTS = [
    "pned_abi_version", "pned_last_error", "pned_set_device", "pned_build_xlocal", "pned_tps_transform",
    "pned_mk_list12", "pned_model_create", "pned_model_destroy", "pned_model_info", "pned_model_plan", "pned_model_set_plan", "pned_tile_plan_export", "pned_qtile_plan_export", "pned_model_tile_staging", "pned_model_sector_segments", "pned_ctx_create",
    "pned_ctx_destroy", "pned_ctx_set_stream", "pned_ctx_synchronize", "pned_ctx_buffer", "pned_ctx_bytes",
    "pned_hv", "pned_inprdct", "pned_calc_beta", "pned_fill_gaussian", "pned_lanczos_run", "pned_tps_run",
    "pned_dsf_run", "pned_dsf_xy_run", "pned_session_begin_dsf_xy", "pned_cg_run", "pned_bisec", "pned_vec12", "pned_exec_renbun", "pned_normalize_dsf",
    "pned_session_begin", "pned_session_begin_dsf", "pned_session_step", "pned_session_read", "pned_session_vector",
    "pned_session_end", "pned_session_profile", "pned_hv_noalloc",
    "pned_slots_create", "pned_slots_destroy", "pned_slots_info", "pned_slots_set_stream", "pned_slots_load",
    "pned_slots_load_szq", "pned_slots_load_vector", "pned_slots_release", "pned_slots_step", "pned_slots_query",
    "pned_slots_synchronize", "pned_slots_read", "pned_gaussian_column", "pned_lanczos_vector", "pned_slots_set_plan", "pned_slots_plan",
    "pned_write_salphasbeta", "pned_read_salphasbeta", "pned_tpq_thermo", "pned_session_save",
    "pned_session_load", "pned_session_info", "pned_write_vec_data", "pned_read_vec_data",
    "pned_write_dsf_alpha_beta", "pned_read_dsf_alpha_beta", "pned_append_dsf_res", "pned_append_sq",
    "pned_write_dsf_vectors", "pned_read_dsf_vectors", "pned_set_max_subrecord",
    "pned_session_lanczos_state", "pned_session_begin_lanczos_at", "pned_write_interval_dump",
    "pned_read_interval_dump_info", "pned_interval_dump_records", "pned_read_interval_dump",
    "pned_session_tps_state", "pned_session_begin_tps_at", "pned_session_begin_dsf_at",
]
SESSION_LANCZOS, SESSION_TPS, SESSION_DSF = 1, 2, 3


def lib() -> C.CDLL:
    """The loaded product library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pned_b200.build` "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int, C.c_int64, C.c_double
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.pned_abi_version.restype = i32
    L.pned_last_error.restype = C.c_char_p
    L.pned_set_device.argtypes = [i32]
    L.pned_build_xlocal.argtypes = [i32, i32, dp, i32, dp, dbl, vp, C.POINTER(C.c_uint8), ip]
    L.pned_tps_transform.argtypes = [i32, i32, i32, dbl, i32, vp, dp]
    L.pned_mk_list12.argtypes = [i32, i32, i32, i32, C.POINTER(i64), vp, vp, vp]
    L.pned_model_create.argtypes = [C.POINTER(ModelDesc), C.POINTER(vp)]
    L.pned_model_destroy.argtypes = [vp]
    L.pned_model_info.argtypes = [vp, C.POINTER(i64), ip, ip]
    L.pned_model_plan.argtypes = [vp, i32, ip, ip, ip]
    L.pned_model_tile_staging.argtypes = [vp, ip, ip]
    L.pned_model_sector_segments.argtypes = [vp, i32, ip]
    L.pned_model_set_plan.argtypes = [vp, i32, C.POINTER(TilePlan)]
    L.pned_tile_plan_export.argtypes = [vp, i32, C.POINTER(TilePlan), C.POINTER(i64), i64, C.POINTER(i64)]
    L.pned_qtile_plan_export.argtypes = [vp, i32, i32, C.POINTER(i64), i64, C.POINTER(i64)]
    L.pned_ctx_create.argtypes = [vp, i32, C.c_size_t, C.POINTER(vp)]
    L.pned_ctx_destroy.argtypes = [vp]
    L.pned_ctx_set_stream.argtypes = [vp, vp]
    L.pned_ctx_synchronize.argtypes = [vp]
    L.pned_ctx_buffer.argtypes = [vp, i32, C.POINTER(vp)]
    L.pned_ctx_bytes.argtypes = [vp, C.POINTER(C.c_size_t)]
    L.pned_hv.argtypes = [vp, vp, vp, dbl, vp, i32]
    L.pned_inprdct.argtypes = [vp, vp, vp, vp, i32]
    L.pned_calc_beta.argtypes = [vp, vp, vp, vp, dp, i32]
    L.pned_fill_gaussian.argtypes = [vp, C.c_uint64, i32, vp]
    L.pned_lanczos_run.argtypes = [vp, vp, i32, i32, dp, dp, dp, ip, i32]
    L.pned_tps_run.argtypes = [vp, dbl, vp, i32, i32, C.POINTER(Observable), dp, dp, dp, i32]
    L.pned_dsf_run.argtypes = [vp, vp, dp, i32, dp, dp, dp, i32]
    L.pned_dsf_xy_run.argtypes = [vp, vp, i32, vp, dp, i32, dp, dp, dp, i32]
    L.pned_session_begin_dsf_xy.argtypes = [vp, vp, i32, vp, dp, i32, dp, i32]
    L.pned_cg_run.argtypes = [vp, dbl, vp, i32, i32, vp, ip, ip, i32]
    L.pned_bisec.argtypes = [dp, dp, i32, dp, i32, dbl]
    L.pned_vec12.argtypes = [dp, dp, dp, i32, i32, dp]
    L.pned_exec_renbun.argtypes = [i32, i32, dbl, dbl, dbl, dp, dp, dp, ip, dp]
    L.pned_normalize_dsf.argtypes = [i32, dbl, dbl, dp]
    L.pned_session_begin.argtypes = [vp, i32, vp, i32, dbl, i32, C.POINTER(Observable), i32]
    L.pned_session_begin_dsf.argtypes = [vp, vp, dp, i32, dp, i32]
    L.pned_session_step.argtypes = [vp, i32]
    L.pned_session_read.argtypes = [vp, dp, dp, dp, ip, ip]
    L.pned_session_vector.argtypes = [vp, C.POINTER(vp), dp]
    L.pned_session_end.argtypes = [vp]
    L.pned_session_profile.argtypes = [vp, i32, dp, dp]
    L.pned_hv_noalloc.argtypes = [vp, i32, vp, vp, dbl, vp, vp]
    L.pned_slots_create.argtypes = [C.POINTER(ModelDesc), i32, i32, C.c_size_t, C.POINTER(vp)]
    L.pned_slots_destroy.argtypes = [vp]
    L.pned_slots_info.argtypes = [vp, C.POINTER(i64), ip, ip, C.POINTER(C.c_size_t)]
    L.pned_slots_set_stream.argtypes = [vp, vp]
    L.pned_slots_load.argtypes = [vp, i32, i32, C.POINTER(ModelDesc), vp, i32, dbl, i32]
    L.pned_slots_load_szq.argtypes = [vp, i32, C.POINTER(ModelDesc), vp, dp, i32, i32]
    L.pned_slots_load_vector.argtypes = [vp, i32, C.POINTER(ModelDesc), vp, i32, dp, dp, dp, vp, i32]
    L.pned_slots_release.argtypes = [vp, i32]
    L.pned_slots_step.argtypes = [vp, i32]
    L.pned_slots_query.argtypes = [vp]
    L.pned_slots_synchronize.argtypes = [vp]
    L.pned_slots_read.argtypes = [vp, i32, ip, ip, ip, dp, dp, dp, dp]
    L.pned_gaussian_column.argtypes = [i64, i32, i32, C.c_uint64, vp, vp]
    L.pned_lanczos_vector.argtypes = [vp, vp, i32, dp, dp, dp, vp, i32]
    L.pned_slots_set_plan.argtypes = [vp, C.POINTER(TilePlan)]
    L.pned_slots_plan.argtypes = [vp, ip, ip, ip]
    L.pned_write_salphasbeta.argtypes = [C.c_char_p, i32, i32, dp, dp, dp]
    L.pned_read_salphasbeta.argtypes = [C.c_char_p, ip, ip, dp, dp, dp, i32]
    L.pned_tpq_thermo.argtypes = [i32, i32, dp, dp, dp, dbl, dbl, i32, dp]
    L.pned_session_save.argtypes = [vp, C.c_char_p]
    L.pned_session_load.argtypes = [vp, C.c_char_p, i32]
    L.pned_session_info.argtypes = [vp, ip, ip, ip, ip]
    L.pned_write_vec_data.argtypes = [C.c_char_p, dbl, vp, i64]
    L.pned_read_vec_data.argtypes = [C.c_char_p, dp, vp, i64]
    L.pned_write_dsf_alpha_beta.argtypes = [C.c_char_p, c128, dp, dp, i32]
    L.pned_read_dsf_alpha_beta.argtypes = [C.c_char_p, C.POINTER(c128), dp, dp, i32]
    L.pned_append_dsf_res.argtypes = [C.c_char_p, dbl, dp, dp, dp, ip, i32]
    L.pned_append_sq.argtypes = [C.c_char_p, i32, dbl, dbl, dbl]
    L.pned_write_dsf_vectors.argtypes = [C.c_char_p, i32, vp, vp, i64]
    L.pned_read_dsf_vectors.argtypes = [C.c_char_p, ip, vp, vp, i64]
    L.pned_session_lanczos_state.argtypes = [vp, vp, vp, i32]
    L.pned_session_begin_lanczos_at.argtypes = [vp, vp, vp, dp, dp, i32, i32, i32]
    L.pned_session_tps_state.argtypes = [vp, vp, vp, vp, i32]
    L.pned_session_begin_dsf_at.argtypes = [vp, vp, vp, dp, dp, i32, i32, i32]
    L.pned_session_begin_tps_at.argtypes = [vp, dbl, vp, vp, dp, dp, dp, i32, i32, i32]
    L.pned_write_interval_dump.argtypes = [C.c_char_p, C.POINTER(DumpInfo), C.POINTER(DumpData)]
    L.pned_read_interval_dump_info.argtypes = [C.c_char_p, C.POINTER(DumpInfo)]
    L.pned_interval_dump_records.argtypes = [C.c_char_p, C.POINTER(i64), i32, ip]
    L.pned_read_interval_dump.argtypes = [C.c_char_p, C.POINTER(DumpData)]
    L.pned_set_max_subrecord.argtypes = [i64]
    _lib = L
    return L


def check(rc: int):
    if rc != PNED_OK:
        raise PnedError(rc, lib().pned_last_error().decode(errors="replace"))
