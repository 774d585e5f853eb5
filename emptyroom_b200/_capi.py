"""ctypes bindings of libemptyroom_b200.so (declarations in include/emptyroom_b200.h)."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libemptyroom_b200.so")

c_int = ctypes.c_int
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
c_int64 = ctypes.c_int64
c_uint64 = ctypes.c_uint64
c_size_t = ctypes.c_size_t
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)

# largest n er_henry_stats_noalloc accepts (ER_HENRY_STATS_NOALLOC_MAX_N)
ER_HENRY_STATS_NOALLOC_MAX_N = 2147483647


class ErParticle(ctypes.Structure):
    _fields_ = [("x_f", c_double), ("y_f", c_double), ("z_f", c_double),
                ("eps_with_adsorbate", c_double), ("sig_with_adsorbate_squared", c_double)]


class ErFrameworkDesc(ctypes.Structure):
    _fields_ = [("n_atoms", c_int), ("atoms", c_void_p), ("t_matrix", c_double * 9),
                ("rep", c_int * 3), ("r_cutoff_squared", c_double)]


class ErGridJob(ctypes.Structure):
    _fields_ = [("fw_id", c_int), ("nx", c_int), ("ny", c_int), ("nz", c_int),
                ("out_device", c_void_p)]


class ErSettings(ctypes.Structure):
    _fields_ = [("forcefield", ctypes.c_char * 256), ("verbose", c_int),
                ("grid_resolution", c_double), ("grid_output_format", ctypes.c_char * 16),
                ("r_cutoff_squared", c_double), ("feynman_hibbs", c_int),
                ("energy_threshold", c_double), ("temperature", c_double),
                ("insertions_per_a3", c_int)]


class ErHenryResult(ctypes.Structure):
    _fields_ = [("sum_w", c_double), ("sum_ew", c_double), ("log_scale", c_double),
                ("sum_w_scaled", c_double), ("sum_ew_scaled", c_double),
                ("n_insertions", c_double), ("n_blocked", c_double),
                ("mean_energy", c_double), ("kh_mol_m3_pa", c_double)]


class ErHenryTiming(ctypes.Structure):
    _fields_ = [("bin_ms", c_double), ("sort_ms", c_double), ("energy_ms", c_double),
                ("reduce_ms", c_double)]


class ErJob(ctypes.Structure):
    _fields_ = [("kind", c_int), ("fw_key", c_uint64), ("desc", c_void_p), ("nx", c_int),
                ("ny", c_int), ("nz", c_int), ("temperature", c_double),
                ("n_insertions", c_int64), ("seed", c_uint64), ("grid_out_host", c_void_p)]


class ErJobStatus(ctypes.Structure):
    _fields_ = [("done", c_int), ("status", c_int), ("grid_cache_hit", c_int),
                ("submit_s", c_double), ("start_s", c_double), ("finish_s", c_double),
                ("henry", ErHenryResult)]


# name -> (restype, argtypes); every entry point declared in include/emptyroom_b200.h
SIGNATURES = {
    "er_status_string": (ctypes.c_char_p, [c_int]),
    "er_ctx_create": (c_int, [c_int, ctypes.POINTER(c_void_p)]),
    "er_ctx_destroy": (None, [c_void_p]),
    "er_ctx_last_error": (ctypes.c_char_p, [c_void_p]),
    "er_ctx_synchronize": (c_int, [c_void_p]),
    "er_ctx_stream": (c_int, [c_void_p, ctypes.POINTER(c_void_p)]),
    "er_framework_upload": (c_int, [c_void_p, ctypes.POINTER(ErFrameworkDesc), _ip]),
    "er_framework_upload_many": (c_int, [c_void_p, ctypes.POINTER(ErFrameworkDesc), c_int, _ip]),
    "er_framework_release": (c_int, [c_void_p, c_int]),
    "er_framework_bytes": (c_int, [c_void_p, c_int, ctypes.POINTER(c_size_t)]),
    "er_grid": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p]),
    "er_grid_sheet": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, _dp]),
    "er_accessibility": (c_int, [c_void_p, c_int, c_int, c_int, c_int, _u8p]),
    "er_grid_batch": (c_int, [c_void_p, ctypes.POINTER(ErGridJob), c_int, c_int]),
    "er_batch_plan_create": (c_int, [c_void_p, ctypes.POINTER(ErGridJob), c_int, c_int,
                                     ctypes.POINTER(c_void_p)]),
    "er_batch_plan_run": (c_int, [c_void_p]),
    "er_batch_plan_launches": (c_int, [c_void_p, _ip]),
    "er_batch_plan_destroy": (None, [c_void_p]),
    "er_batch_plan_tile": (c_int, [c_void_p, c_int, _ip]),
    "er_henry": (c_int, [c_void_p, c_int, c_double, c_int64, c_uint64, _u8p, c_int, c_int,
                         c_int, ctypes.POINTER(ErHenryResult), _fp]),
    "er_henry_batch": (c_int, [c_void_p, _ip, c_int, c_double, c_int64, ctypes.POINTER(c_uint64),
                               c_int, c_int, c_int, ctypes.POINTER(ErHenryResult), _ip]),
    "er_henry_stats_noalloc": (c_int, [c_void_p, c_void_p, c_int64, c_double,
                                       ctypes.POINTER(ErHenryResult)]),
    "er_ctx_set_timing": (c_int, [c_void_p, c_int]),
    "er_henry_last_timing": (c_int, [c_void_p, ctypes.POINTER(ErHenryTiming)]),
    "er_block_pockets": (c_int, [c_void_p, _dp, c_int, c_int, c_int, c_double, _ip, _ip]),
    "er_block_pockets_device": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_double,
                                        c_void_p, _ip]),
    "er_grid_interp": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, _dp, c_int64,
                               _dp]),
    "er_cell_matrices": (c_int, [c_double, c_double, c_double, c_double, c_double, c_double,
                                 _dp, _dp, _dp]),
    "er_replication_factors": (c_int, [_dp, c_double, c_int, _ip]),
    "er_philox4x32_10": (None, [_u32p, _u32p, _u32p]),
    "er_insertion_point": (None, [c_uint64, c_uint64, _dp]),
    "er_synth_positions": (c_int, [c_uint64, _dp, c_int, c_double, _dp]),
    "er_server_create": (c_int, [c_void_p, c_size_t, c_int, ctypes.POINTER(c_void_p)]),
    "er_server_submit": (c_int, [c_void_p, ctypes.POINTER(ErJob), ctypes.POINTER(c_uint64)]),
    "er_server_poll": (c_int, [c_void_p, c_uint64, ctypes.POINTER(ErJobStatus)]),
    "er_server_wait": (c_int, [c_void_p, c_uint64, c_double, ctypes.POINTER(ErJobStatus)]),
    "er_server_grid": (c_int, [c_void_p, c_uint64, ctypes.POINTER(c_void_p)]),
    "er_server_now": (c_double, [c_void_p]),
    "er_server_bytes": (c_int, [c_void_p, ctypes.POINTER(c_size_t)]),
    "er_server_destroy": (None, [c_void_p]),
    "er_structure_load": (c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(c_void_p),
                                  ctypes.c_char_p, c_size_t]),
    "er_structure_free": (None, [c_void_p]),
    "er_structure_info": (c_int, [c_void_p, _ip, _dp, _dp, _dp, _dp, _dp]),
    "er_structure_frac": (c_int, [c_void_p, _dp]),
    "er_structure_label": (c_int, [c_void_p, c_int, ctypes.c_char_p, c_size_t]),
    "er_forcefield_load": (c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(c_void_p),
                                   ctypes.c_char_p, c_size_t]),
    "er_forcefield_free": (None, [c_void_p]),
    "er_forcefield_count": (c_int, [c_void_p]),
    "er_forcefield_entry": (c_int, [c_void_p, c_int, ctypes.c_char_p, c_size_t, _dp, _dp]),
    "er_forcefield_find": (c_int, [c_void_p, ctypes.c_char_p, _dp, _dp]),
    "er_mix_particles": (c_int, [c_void_p, c_void_p, c_double, c_double, c_void_p,
                                 ctypes.c_char_p, c_size_t]),
    "er_adsorbate_mw": (c_int, [ctypes.c_char_p, ctypes.c_char_p, _dp, ctypes.c_char_p,
                                c_size_t]),
    "er_read_uc": (c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _ip,
                           ctypes.c_char_p, c_size_t]),
    "er_write_uc": (c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _ip]),
    "er_read_settings": (c_int, [ctypes.c_char_p, c_int, c_void_p, ctypes.c_char_p, c_size_t]),
    "er_write_grid_txt": (c_int, [ctypes.c_char_p, _fp, c_int, c_int, c_int, c_int]),
    "er_write_grid_cube": (c_int, [ctypes.c_char_p, _fp, c_int, c_int, c_int, _dp, c_int]),
    "er_read_grid_txt": (c_int, [ctypes.c_char_p, _dp, c_size_t, _ip, ctypes.c_char_p,
                                 c_size_t]),
    "er_version": (ctypes.c_char_p, []),
    "er_probe_fp32_rate": (c_int, [c_void_p, c_double, _dp]),
    "er_probe_rcp64_seed": (c_int, [c_void_p, _dp]),
    "er_selftest_wait_timeout": (c_int, [c_void_p, c_int]),
}

_lib = None


def lib():
    """Loads the in-tree library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libemptyroom_b200.so not built at {LIB_PATH}: run "
                "`make -C emptyroom_b200/csrc` (or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
