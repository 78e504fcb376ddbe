"""Load libzoomyfv.so and declare the C ABI of include/zoomy_fv.h.

There is no CPU fallback: if the library is missing or cannot be loaded the
import of the solver fails with the reason.
"""
from __future__ import annotations

import ctypes as C
import pathlib

from ._abi import zfv_amr_level, zfv_config, zfv_status

LIB_PATH = pathlib.Path(__file__).resolve().parent / "lib" / "libzoomyfv.so"

_lib = None

SYMBOLS = ("zfv_last_error", "zfv_version", "zfv_sizeof_config", "zfv_sizeof_status", "zfv_model_info", "zfv_create", "zfv_destroy",
           "zfv_scratch_bytes", "zfv_begin", "zfv_update_state", "zfv_compute_dt", "zfv_evolve",
           "zfv_rhs", "zfv_fill_ghosts", "zfv_total_mass", "zfv_get_status", "zfv_log_capacity",
           "zfv_read_log", "zfv_evolve_static", "zfv_state_import", "zfv_state_export",
           "zfv_batch_create", "zfv_batch_destroy", "zfv_batch_scratch_bytes", "zfv_batch_bind",
           "zfv_batch_import", "zfv_batch_export", "zfv_batch_begin", "zfv_batch_evolve",
           "zfv_batch_status", "zfv_batch_units", "zfv_tile_variants", "zfv_batch_set_variant",
           "zfv_run_state_bytes", "zfv_save_run_state", "zfv_load_run_state", "zfv_adj_tape_bytes",
           "zfv_adj_work_bytes", "zfv_adj_record", "zfv_adj_step", "zfv_adj_variants",
           "zfv_adj_set_variant", "zfv_batch_create_grouped", "zfv_batch_set_frames", "zfv_batch_set_dt",
           "zfv_batch_stage", "zfv_batch_descriptors", "zfv_amr_fill", "zfv_amr_average_down", "zfv_amr_tag",
           "zfv_amr_regrid_fill", "zfv_amr_set_dt", "zfv_implicit_global_stats",
           "zfv_batch_compute_dt", "zfv_amr_level_dt",
           "zfv_init_solution", "zfv_set_variant", "zfv_get_variant", "zfv_generic_tile_variants",
           "zfv_adj_steps")


class ZfvError(RuntimeError):
    pass


def lib():
    """The loaded library (built on first use if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ZfvError(f"{LIB_PATH} is not built; run `python -m zoomy_amrex_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.zfv_last_error.restype = C.c_char_p
    L.zfv_version.restype = C.c_char_p
    L.zfv_sizeof_config.restype = C.c_size_t
    L.zfv_sizeof_status.restype = C.c_size_t
    L.zfv_model_info.argtypes = [i, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.zfv_create.argtypes = [C.POINTER(zfv_config), C.POINTER(vp)]
    L.zfv_destroy.argtypes = [vp]
    L.zfv_scratch_bytes.argtypes = [vp]
    L.zfv_scratch_bytes.restype = C.c_size_t
    L.zfv_begin.argtypes = [vp, vp, vp, vp, vp]
    L.zfv_update_state.argtypes = [vp, vp, vp, d, vp]
    L.zfv_init_solution.argtypes = [vp, vp, i, vp]
    L.zfv_set_variant.argtypes = [vp, i, vp]
    L.zfv_get_variant.argtypes = [vp]
    L.zfv_compute_dt.argtypes = [vp, vp, vp, vp, vp]
    L.zfv_evolve.argtypes = [vp, vp, vp, vp, i, vp]
    L.zfv_rhs.argtypes = [vp, vp, vp, vp, d, vp]
    L.zfv_fill_ghosts.argtypes = [vp, vp, vp, vp, vp, d, vp]
    L.zfv_total_mass.argtypes = [vp, vp, vp, vp]
    L.zfv_get_status.argtypes = [vp, vp, C.POINTER(zfv_status), vp]
    L.zfv_log_capacity.argtypes = [vp]
    L.zfv_read_log.argtypes = [vp, vp, C.POINTER(d), i, C.POINTER(C.c_int64), C.POINTER(i), vp]
    L.zfv_state_import.argtypes = [vp, vp, vp, vp, vp]
    L.zfv_state_export.argtypes = [vp, vp, vp, vp, vp]
    pp = C.POINTER(C.c_void_p)
    L.zfv_batch_create.argtypes = [C.POINTER(zfv_config), i, C.POINTER(vp)]
    L.zfv_batch_destroy.argtypes = [vp]
    L.zfv_batch_scratch_bytes.argtypes = [vp]
    L.zfv_batch_scratch_bytes.restype = C.c_size_t
    L.zfv_batch_bind.argtypes = [vp, pp, pp, vp, vp]
    L.zfv_batch_import.argtypes = [vp, pp, vp]
    L.zfv_batch_export.argtypes = [vp, pp, vp]
    L.zfv_batch_begin.argtypes = [vp, vp]
    L.zfv_batch_evolve.argtypes = [vp, i, vp]
    L.zfv_batch_status.argtypes = [vp, C.POINTER(zfv_status), vp]
    L.zfv_batch_units.argtypes = [vp]
    L.zfv_tile_variants.argtypes = [C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i), i]
    L.zfv_generic_tile_variants.argtypes = [C.POINTER(i), C.POINTER(i), C.POINTER(i), i]
    L.zfv_batch_set_variant.argtypes = [vp, i, vp]
    L.zfv_evolve_static.argtypes = [vp, vp, vp, i, i, C.POINTER(zfv_status), vp]
    L.zfv_run_state_bytes.restype = C.c_size_t
    L.zfv_save_run_state.argtypes = [vp, vp, vp, vp]
    L.zfv_load_run_state.argtypes = [vp, vp, vp, vp]
    L.zfv_adj_tape_bytes.argtypes = [vp, i]
    L.zfv_adj_tape_bytes.restype = C.c_size_t
    L.zfv_adj_work_bytes.argtypes = [vp]
    L.zfv_adj_work_bytes.restype = C.c_size_t
    L.zfv_adj_record.argtypes = [vp, vp, vp, vp, vp, i, vp]
    L.zfv_adj_step.argtypes = [vp, vp, i, vp, vp, vp, vp, vp]
    L.zfv_adj_steps.argtypes = [vp, vp, i, vp, vp, vp, vp, vp]
    L.zfv_adj_set_variant.argtypes = [i]
    L.zfv_batch_create_grouped.argtypes = [C.POINTER(zfv_config), i, C.POINTER(i), C.POINTER(vp)]
    L.zfv_batch_set_frames.argtypes = [vp, pp, vp]
    L.zfv_batch_set_dt.argtypes = [vp, vp, vp]
    L.zfv_batch_compute_dt.argtypes = [vp, vp]
    L.zfv_amr_level_dt.argtypes = [vp, d, vp, vp]
    L.zfv_batch_stage.argtypes = [vp, i, vp]
    L.zfv_batch_descriptors.argtypes = [vp]
    L.zfv_batch_descriptors.restype = vp
    lv = C.POINTER(zfv_amr_level)
    L.zfv_amr_fill.argtypes = [lv, lv, vp, vp, i, i, i, vp]
    L.zfv_amr_average_down.argtypes = [lv, lv, vp, i, i, vp]
    L.zfv_amr_tag.argtypes = [lv, vp, i, i, d, d, d, i, d, vp, vp]
    L.zfv_amr_regrid_fill.argtypes = [lv, lv, lv, vp, i, i, vp]
    L.zfv_amr_set_dt.argtypes = [pp, pp, C.POINTER(i), i, d, d, d, d, d, vp, vp]
    L.zfv_implicit_global_stats.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                            C.POINTER(C.c_longlong)]
    _lib = L
    return L


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().zfv_last_error().decode(errors="replace")
        raise ZfvError(f"{what} failed ({rc}): {msg}")
