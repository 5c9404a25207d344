"""ctypes binding of libscmf.so (include/scmf.h).

The library is built in-tree (new_arch_b200/_lib/libscmf.so).  There is no
fallback: if the library is missing or the GPU is absent, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libscmf.so")

SCMF_OK = 0
ERRORS = {-1: "INVALID", -2: "CUDA", -3: "NOMEM", -4: "IO", -5: "PARSE", -6: "STATE", -7: "TIMEOUT", -8: "DEVICE",
          -9: "CANCELLED"}

HAM_SCMF0, HAM_LITERAL = 0, 1
FIELD_REFERENCE, FIELD_EVERY = 0, 1


class ScmfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"scmf error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [("reference_nbeads", C.c_int32), ("harmonic_normb", C.c_double), ("smc_a", C.c_double),
                ("seed", C.c_uint64), ("hamiltonian", C.c_int32), ("field_rule", C.c_int32),
                ("count_bits", C.c_int32), ("reserved", C.c_int32)]


class SpecInfo(C.Structure):
    _fields_ = [("n_beads", C.c_int64), ("n_cells", C.c_int64), ("n_chains", C.c_int32), ("n_types", C.c_int32),
                ("n_arch", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double), ("field_scaling", C.c_double),
                ("harmonic_normb", C.c_double), ("smc_a", C.c_double), ("smc_r", C.c_double),
                ("reference_nbeads", C.c_int32), ("count_bits", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("step", C.c_uint64), ("last_accepts", C.c_uint64), ("total_accepts", C.c_uint64),
                ("total_moves", C.c_uint64), ("e_bond", C.c_double), ("e_field", C.c_double),
                ("error_word", C.c_uint32), ("reserved", C.c_uint32)]


class Tune(C.Structure):
    _fields_ = [("chains_per_tile", C.c_int32), ("threads_move", C.c_int32), ("cells_per_tile", C.c_int32),
                ("threads_field", C.c_int32), ("persistent_ctas", C.c_int32), ("use_graph", C.c_int32),
                ("beads_per_tile", C.c_int32), ("reserved", C.c_int32)]


class TuneTrial(C.Structure):
    _fields_ = [("tune", Tune), ("ms", C.c_float), ("reserved", C.c_int32)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_active", C.c_int32), ("sweeps_per_round", C.c_int32),
                ("use_graph", C.c_int32), ("reserved", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int32), ("n_sweeps", C.c_int32), ("e_bond", C.c_double),
                ("e_field", C.c_double), ("accepts", C.c_uint64), ("n_beads", C.c_int64),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("sweeps_done", C.c_int32), ("reserved", C.c_int32)]


class CheckpointHeader(C.Structure):
    _fields_ = [("version", C.c_uint32), ("n_types", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32),
                ("nz", C.c_int32), ("n_chains", C.c_int32), ("n_arch", C.c_int32), ("avg_every", C.c_uint32),
                ("n_beads", C.c_int64), ("n_cells", C.c_int64), ("seed", C.c_uint64), ("spec_hash", C.c_uint64),
                ("step", C.c_uint64), ("last_accepts", C.c_uint64), ("total_accepts", C.c_uint64),
                ("total_moves", C.c_uint64), ("e_field", C.c_double), ("avg_samples", C.c_uint64),
                ("payload_bytes", C.c_uint64), ("payload_hash", C.c_uint64)]


class Observables(C.Structure):
    _fields_ = [("arch", C.c_int32), ("n_chains", C.c_int32), ("n_beads", C.c_int64), ("n_bonds", C.c_int64),
                ("re2", C.c_double * 4), ("rg2", C.c_double * 4), ("bond2", C.c_double * 4), ("msd", C.c_double * 4),
                ("msd_com", C.c_double * 4), ("acc_ratio", C.c_double), ("reserved", C.c_double * 3)]


class Validation(C.Structure):
    _fields_ = [("nonfinite_positions", C.c_uint64), ("positions_out_of_range", C.c_uint64),
                ("count_mismatch_words", C.c_uint64), ("nonfinite_omega", C.c_uint64),
                ("count_sum_error", C.c_int64), ("error_word", C.c_uint32), ("reserved", C.c_uint32)]


# name -> (restype, argtypes)
_vp, _i32, _i64, _u32, _u64, _sz, _f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_size_t, C.c_double
_pvp = C.POINTER(C.c_void_p)
_pf32 = C.POINTER(C.c_float)
_pu32 = C.POINTER(C.c_uint32)
_pi32 = C.POINTER(C.c_int32)
_pf64 = C.POINTER(C.c_double)

SIGNATURES = {
    "scmf_last_error": (C.c_char_p, []),
    "scmf_version": (C.c_char_p, []),
    "scmf_spec_create": (_i32, [_i32, _i32, _i32, _i32, _f64, _f64, _f64, _pvp]),
    "scmf_spec_set_xn": (_i32, [_vp, _pf64, _i32]),
    "scmf_spec_set_params": (_i32, [_vp, C.POINTER(Params)]),
    "scmf_spec_add_arch": (_i32, [_vp, _i32, _i32, _pi32, _i32, _pi32, _f64]),
    "scmf_spec_load_files": (_i32, [C.c_char_p, C.c_char_p, _u64, _pvp]),
    "scmf_spec_get_info": (_i32, [_vp, C.POINTER(SpecInfo)]),
    "scmf_spec_get_params": (_i32, [_vp, C.POINTER(Params)]),
    "scmf_spec_get_xn": (_i32, [_vp, _pf64, _i32]),
    "scmf_spec_get_arch": (_i32, [_vp, _i32, _pi32, _pi32, _pi32, _i32, _pi32, _i32, _pi32, _pf64]),
    "scmf_spec_copy": (_i32, [_vp, _pvp]),
    "scmf_spec_destroy": (None, [_vp]),
    "scmf_system_create": (_i32, [_vp, _vp, _pvp]),
    "scmf_system_create_shard": (_i32, [_vp, _i32, _i32, _vp, _pvp]),
    "scmf_shard_chains": (_i32, [_vp, _i32, _i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _i32]),
    "scmf_shard_init_coords": (_i32, [_vp, _vp]),
    "scmf_shard_move": (_i32, [_vp, _vp]),
    "scmf_shard_field": (_i32, [_vp, _vp, _i32]),
    "scmf_system_destroy": (None, [_vp]),
    "scmf_system_get_info": (_i32, [_vp, C.POINTER(SpecInfo)]),
    "scmf_system_stream": (_i32, [_vp, _pvp]),
    "scmf_init_coords": (_i32, [_vp]),
    "scmf_set_coords": (_i32, [_vp, _pf32, _sz]),
    "scmf_get_coords": (_i32, [_vp, _pf32, _sz]),
    "scmf_set_step": (_i32, [_vp, _u64]),
    "scmf_step": (_i32, [_vp, _i32]),
    "scmf_step_async": (_i32, [_vp, _i32]),
    "scmf_step_profiled": (_i32, [_vp, _i32, _pf32, _pf32, _pf32]),
    "scmf_smc_move": (_i32, [_vp, _i32]),
    "scmf_reset_density_fields": (_i32, [_vp]),
    "scmf_update_omega_fields_scmf0": (_i32, [_vp]),
    "scmf_synchronize": (_i32, [_vp]),
    "scmf_get_counts": (_i32, [_vp, _pu32, _sz]),
    "scmf_get_omega": (_i32, [_vp, _pf32, _sz]),
    "scmf_set_omega": (_i32, [_vp, _pf32, _sz]),
    "scmf_get_stats": (_i32, [_vp, C.POINTER(Stats)]),
    "scmf_get_sweep_stats": (_i32, [_vp, C.POINTER(Stats)]),
    "scmf_step_stats": (_i32, [_vp, _i32, C.POINTER(Stats)]),
    "scmf_step_stats_async": (_i32, [_vp, _i32, _vp]),
    "scmf_debug_math": (_i32, [_u32, _u32, _i32, _pu32, _pf32, _pf32]),
    "scmf_update_omega_noalloc": (_i32, [_vp, _vp, _i32, _i64, _f64, _pf64, _i32, _i32, _vp, _vp]),
    "scmf_write_density": (_i32, [_vp, C.c_char_p, _i64]),
    "scmf_write_coords": (_i32, [_vp, C.c_char_p]),
    "scmf_read_coords_file": (_i32, [C.c_char_p, _i64, _pf32, _sz]),
    "scmf_vtk_convert": (_i32, [C.c_char_p, C.c_char_p, _i32]),
    "scmf_average_start": (_i32, [_vp, _u32]),
    "scmf_average_sample": (_i32, [_vp]),
    "scmf_average_get": (_i32, [_vp, C.POINTER(C.c_uint64), _sz, C.POINTER(C.c_uint64)]),
    "scmf_write_average_density": (_i32, [_vp, C.c_char_p, _i64]),
    "scmf_checkpoint_write": (_i32, [_vp, C.c_char_p]),
    "scmf_checkpoint_read": (_i32, [_vp, C.c_char_p]),
    "scmf_checkpoint_info": (_i32, [C.c_char_p, C.POINTER(CheckpointHeader)]),
    "scmf_spec_hash": (_i32, [_vp, C.POINTER(C.c_uint64)]),
    "scmf_validate": (_i32, [_vp, C.POINTER(Validation)]),
    "scmf_analysis_reference": (_i32, [_vp]),
    "scmf_analyze": (_i32, [_vp, C.POINTER(Observables), _i32]),
    "scmf_batch_create": (_i32, [_pvp, _i32, C.POINTER(Tune), _vp, _pvp]),
    "scmf_batch_step": (_i32, [_vp, _i32]),
    "scmf_batch_step_async": (_i32, [_vp, _i32]),
    "scmf_batch_step_profiled": (_i32, [_vp, _i32, _pf32, _pf32, _pf32]),
    "scmf_batch_autotune": (_i32, [_vp, _i32, C.POINTER(Tune)]),
    "scmf_batch_get_tune": (_i32, [_vp, C.POINTER(Tune)]),
    "scmf_batch_tune_trials": (_i32, [_vp, C.POINTER(TuneTrial), _i32, C.POINTER(C.c_int32)]),
    "scmf_batch_destroy": (None, [_vp]),
    "scmf_batch_run": (_i32, [_pvp, _i32, _i32, C.POINTER(Tune)]),
    "scmf_server_create": (_i32, [C.POINTER(ServerOpts), _pvp]),
    "scmf_server_submit": (_i32, [_vp, _vp, _i32, _pu32, C.POINTER(C.c_uint64)]),
    "scmf_server_poll": (_i32, [_vp, C.POINTER(Result), _i32, _pi32, _i32]),
    "scmf_server_pending": (_i32, [_vp, _pi32, _pi32, C.POINTER(C.c_uint64)]),
    "scmf_server_now": (_f64, [_vp]),
    "scmf_server_cancel": (_i32, [_vp, _u64]),
    "scmf_server_drain": (_i32, [_vp, _i32]),
    "scmf_server_destroy": (None, [_vp]),
}

_lib = None


def lib():
    """Load libscmf.so (building nothing: run new_arch_b200.build first)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ScmfError(-2, f"{LIB_PATH} is not built; run `python -m new_arch_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != SCMF_OK:
        raise ScmfError(rc, lib().scmf_last_error().decode(errors="replace"))
