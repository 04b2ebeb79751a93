"""ctypes binding of ``libpdlp_b200.so`` (declared in ``include/pdlp_b200.h``).

The library is the product: every solve and every kernel-level call goes
through it.  If it cannot be loaded, or no CUDA device is usable, the calls
raise ``RuntimeError`` -- there is no CPU path behind them.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpdlp_b200.so")

PDLP_OK = 0
PDLP_ERR_ARG = -1
PDLP_ERR_OOM = -2
PDLP_ERR_CUDA = -3
PDLP_ERR_BARRIER_TIMEOUT = -4
PDLP_ERR_NUMERICAL = -5
PDLP_ERR_STATE = -6
PDLP_ERR_BOUNDS = -7

PDLP_MEM_DEVICE = 0
PDLP_MEM_HOST = 1

PDLP_SPMV_AUTO = 0
PDLP_SPMV_STREAMED = 1
PDLP_SPMV_ROW_GROUPS = 2
PDLP_SPMV_BANDED = 3
PDLP_SPMV_PLAN_TILES = 0
PDLP_SPMV_PLAN_STREAMED = 1

PDLP_STATUS_RUNNING = -1
PDLP_SLOT_FREE = -2

SCALING = {"pdlp": 0, "none": 1, "ruiz": 2, "pock_chambolle": 3}
PRECISION = {"fp64": 0, "fp32": 1}

_c_p = ctypes.c_void_p


class ProblemDesc(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int32), ("n", ctypes.c_int32), ("nnz", ctypes.c_int64),
                ("rp", _c_p), ("ri", _c_p), ("rx", _c_p),
                ("cp", _c_p), ("ci", _c_p), ("cx", _c_p),
                ("c", _c_p), ("row_lb", _c_p), ("row_ub", _c_p),
                ("col_lb", _c_p), ("col_ub", _c_p), ("kind", _c_p),
                ("obj_offset", ctypes.c_double), ("sense", ctypes.c_int32),
                ("memory", ctypes.c_int32)]


class Params(ctypes.Structure):
    _fields_ = [("eps_abs", ctypes.c_double), ("eps_rel", ctypes.c_double),
                ("feas_cap", ctypes.c_double), ("max_iter", ctypes.c_int64),
                ("time_limit", ctypes.c_double), ("check_every", ctypes.c_int32),
                ("stepsize_every", ctypes.c_int32), ("beta_sufficient", ctypes.c_double),
                ("beta_necessary", ctypes.c_double), ("beta_artificial", ctypes.c_double),
                ("primal_weight_smoothing", ctypes.c_double), ("scaling", ctypes.c_int32),
                ("power_start", _c_p), ("time_used", ctypes.c_double),
                ("history_capacity", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("detect_infeasibility", ctypes.c_int32), ("eps_infeasible", ctypes.c_double),
                ("expected_iterations", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("iterations", ctypes.c_int64),
                ("restarts", ctypes.c_int64), ("rejected_steps", ctypes.c_int64),
                ("primal_res", ctypes.c_double), ("dual_res", ctypes.c_double),
                ("gap", ctypes.c_double), ("primal_obj", ctypes.c_double),
                ("dual_obj", ctypes.c_double), ("step_size", ctypes.c_double),
                ("primal_weight", ctypes.c_double), ("objective", ctypes.c_double),
                ("scale_obj", ctypes.c_double), ("history_len", ctypes.c_int32),
                ("device_seconds", ctypes.c_double), ("device_start_ns", ctypes.c_int64),
                ("device_end_ns", ctypes.c_int64)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("max_slots", ctypes.c_int32), ("persistent", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("tile_rows", ctypes.c_int32),
                ("tile_nnz", ctypes.c_int32), ("lanes_override", ctypes.c_int32),
                ("memory_budget", ctypes.c_int64), ("barrier_timeout_us", ctypes.c_int64),
                ("autotune", ctypes.c_int32), ("test_withhold_arrival", ctypes.c_int32)]


class TuneKey(ctypes.Structure):
    _fields_ = [("rows_bucket", ctypes.c_int32), ("row_len_bucket", ctypes.c_int32),
                ("col_len_bucket", ctypes.c_int32)]


class Tuning(ctypes.Structure):
    _fields_ = [("lanes_rows", ctypes.c_int32), ("lanes_cols", ctypes.c_int32),
                ("tile_rows", ctypes.c_int32), ("tile_nnz", ctypes.c_int32),
                ("us_per_iteration", ctypes.c_double),
                ("default_us_per_iteration", ctypes.c_double)]


class SpmvPlanInfo(ctypes.Structure):
    _fields_ = [("tiles", ctypes.c_int32), ("banded_tiles", ctypes.c_int32),
                ("huge_rows", ctypes.c_int32), ("ctas", ctypes.c_int32),
                ("kernel", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("entries", ctypes.c_int64), ("entries_in_band", ctypes.c_int64),
                ("seconds", ctypes.c_double)]


class CrossoverInfo(ctypes.Structure):
    _fields_ = [("placed", ctypes.c_int32), ("candidates", ctypes.c_int32),
                ("rejected", ctypes.c_int32), ("factorizations", ctypes.c_int32),
                ("repairs", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("seconds", ctypes.c_double)]


class SimplexParamsC(ctypes.Structure):
    _fields_ = [("feas_tol", ctypes.c_double), ("opt_tol", ctypes.c_double),
                ("pivot_tol", ctypes.c_double), ("max_iter", ctypes.c_int64),
                ("time_limit", ctypes.c_double), ("refactor_freq", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class SimplexInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("phase", ctypes.c_int32),
                ("iterations", ctypes.c_int64), ("phase1_iterations", ctypes.c_int64),
                ("bound_flips", ctypes.c_int64), ("degenerate_pivots", ctypes.c_int64),
                ("dual_iterations", ctypes.c_int64), ("cost_shifts", ctypes.c_int64),
                ("factorizations", ctypes.c_int32), ("repairs", ctypes.c_int32),
                ("objective", ctypes.c_double), ("primal_infeasibility", ctypes.c_double),
                ("dual_infeasibility", ctypes.c_double), ("lu_nnz", ctypes.c_int64),
                ("seconds", ctypes.c_double)]


# basis statuses (include/pdlp_b200.h; sovopt lp/basis.py:75-79)
BASIC, AT_LOWER, AT_UPPER, FREE, FIXED = 0, 1, 2, 3, 4


# Every symbol include/pdlp_b200.h declares, with its argument types.
_i32, _i64, _d = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
SIGNATURES = {
    "pdlp_abi_version": ([], ctypes.c_int),
    "pdlp_last_error": ([], ctypes.c_char_p),
    "pdlp_launch_count": ([], ctypes.c_int64),
    "pdlp_params_default": ([ctypes.POINTER(Params)], None),
    "pdlp_solve": ([ctypes.POINTER(ProblemDesc), ctypes.POINTER(Params), _c_p,
                    ctypes.POINTER(Result), _c_p, _c_p, _c_p, _c_p, _i32], ctypes.c_int),
    "pdlp_batch_config_default": ([ctypes.POINTER(BatchConfig)], None),
    "pdlp_batch_create": ([ctypes.POINTER(BatchConfig), _c_p, ctypes.POINTER(_c_p)], ctypes.c_int),
    "pdlp_batch_destroy": ([_c_p], ctypes.c_int),
    "pdlp_batch_admit": ([_c_p, ctypes.POINTER(ProblemDesc), ctypes.POINTER(Params),
                          ctypes.POINTER(_i32)], ctypes.c_int),
    "pdlp_batch_admit_many": ([_c_p, _i32, ctypes.POINTER(ProblemDesc), ctypes.POINTER(Params),
                               _c_p, _c_p], ctypes.c_int),
    "pdlp_batch_step": ([_c_p, _i64, ctypes.POINTER(_i32)], ctypes.c_int),
    "pdlp_batch_poll": ([_c_p, _i32, ctypes.POINTER(Result)], ctypes.c_int),
    "pdlp_batch_fetch": ([_c_p, _i32, _c_p, _c_p, _c_p, _c_p, _i32], ctypes.c_int),
    "pdlp_batch_retire": ([_c_p, _i32], ctypes.c_int),
    "pdlp_batch_collect_many": ([_c_p, _i32, _c_p, ctypes.POINTER(Result), _c_p, _c_p, _c_p, _c_p,
                                 _i32, _i32], ctypes.c_int),
    "pdlp_batch_statuses": ([_c_p, _c_p, _i32], ctypes.c_int),
    "pdlp_batch_cancel": ([_c_p, _i32], ctypes.c_int),
    "pdlp_batch_scaling": ([_c_p, _i32, _c_p, _c_p, ctypes.POINTER(_d), _i32], ctypes.c_int),
    "pdlp_slot_bytes": ([_i32, _i32, _i64], ctypes.c_int64),
    "pdlp_batch_last_timing": ([_c_p, ctypes.POINTER(_d), ctypes.POINTER(_d),
                                ctypes.POINTER(_i64)], ctypes.c_int),
    "pdlp_spmv_f64": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "pdlp_spmv_f32": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "pdlp_spmv_ex_f64": ([_i32, _i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "pdlp_spmv_ex_f32": ([_i32, _i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "pdlp_spmv_tune_f64": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _i32, ctypes.POINTER(_i32),
                            _c_p], ctypes.c_int),
    "pdlp_spmv_tune_f32": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _i32, ctypes.POINTER(_i32),
                            _c_p], ctypes.c_int),
    "pdlp_spmv_plan_create": ([_i32, _i32, _c_p, _c_p, _c_p, ctypes.POINTER(_c_p)], ctypes.c_int),
    "pdlp_spmv_plan_run_f64": ([_c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "pdlp_spmv_plan_run_f32": ([_c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "pdlp_spmv_plan_get_info": ([_c_p, ctypes.POINTER(SpmvPlanInfo)], ctypes.c_int),
    "pdlp_spmv_plan_status": ([_c_p, _c_p], ctypes.c_int),
    "pdlp_spmv_plan_destroy": ([_c_p], None),
    "pdlp_spmm_f64": ([_i32, _i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "pdlp_primal_step": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _d, _c_p], ctypes.c_int),
    "pdlp_dual_step": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _d, _c_p], ctypes.c_int),
    "pdlp_pdhg_primal": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _d, _c_p], ctypes.c_int),
    "pdlp_pdhg_dual": ([_i32, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _d, _c_p], ctypes.c_int),
    "pdlp_pdhg_accum": ([_i32, _c_p, _c_p, _c_p, _c_p, _d, _c_p], ctypes.c_int),
    "pdlp_dot": ([_i64, _c_p, _c_p, ctypes.POINTER(_d), _c_p], ctypes.c_int),
    "pdlp_nrm2": ([_i64, _c_p, ctypes.POINTER(_d), _c_p], ctypes.c_int),
    "pdlp_nrm_inf": ([_i64, _c_p, ctypes.POINTER(_d), _c_p], ctypes.c_int),
    "pdlp_bnr_create": ([ctypes.POINTER(ProblemDesc), _d, _i32, _c_p, ctypes.POINTER(_c_p)],
                        ctypes.c_int),
    "pdlp_bnr_destroy": ([_c_p], ctypes.c_int),
    "pdlp_bnr_solve_batch": ([_c_p, _i32, _c_p, _c_p, _c_p, _c_p, _i32, _d, _d, _c_p, _c_p,
                              _c_p, _c_p, _i32], ctypes.c_int),
    "pdlp_bnr_step_sizes": ([_c_p, _i32, _c_p, _c_p], ctypes.c_int),
    "pdlp_dot_noalloc": ([_i64, _c_p, _c_p, ctypes.POINTER(_d), _c_p], ctypes.c_int),
    "pdlp_tune_key_of": ([_i32, _i32, _i64, ctypes.POINTER(TuneKey)], None),
    "pdlp_tune_lp": ([ctypes.POINTER(ProblemDesc), ctypes.POINTER(Params), _c_p,
                      ctypes.POINTER(Tuning)], ctypes.c_int),
    "pdlp_tune_cache_size": ([], ctypes.c_int),
    "pdlp_tune_cache_get": ([_i32, ctypes.POINTER(TuneKey), ctypes.POINTER(Tuning)],
                            ctypes.c_int),
    "pdlp_tune_cache_put": ([ctypes.POINTER(TuneKey), ctypes.POINTER(Tuning)], ctypes.c_int),
    "pdlp_tune_cache_clear": ([], None),
    "pdlp_basis_from_point": ([ctypes.POINTER(ProblemDesc), _c_p, _c_p, _d, _d, _c_p,
                               ctypes.POINTER(CrossoverInfo)], ctypes.c_int),
    "pdlp_simplex_default_params": ([ctypes.POINTER(SimplexParamsC)], ctypes.c_int),
    "pdlp_simplex_solve": ([ctypes.POINTER(ProblemDesc), ctypes.POINTER(SimplexParamsC), _c_p,
                            _c_p, _c_p, _c_p, _c_p, ctypes.POINTER(SimplexInfo)], ctypes.c_int),
}

_LIB = None


def load():
    """Load (building first if the sources are newer) and bind the library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        try:
            from .build import build
            build()
        except Exception as exc:          # pragma: no cover - environment dependent
            raise RuntimeError(f"GPU backend unavailable (libpdlp_b200.so missing and "
                               f"could not be built: {exc})") from exc
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as exc:
        raise RuntimeError(f"GPU backend unavailable (cannot load {LIB_PATH}: {exc})") from exc
    for name, (argtypes, restype) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = restype
    _LIB = lib
    return lib


class PDLPError(RuntimeError):
    """A non-zero return code of the C ABI, with the library's message."""

    def __init__(self, code, message):
        super().__init__(f"pdlp error {code}: {message}")
        self.code = code


def check(code):
    if code != PDLP_OK:
        msg = load().pdlp_last_error()
        raise PDLPError(code, msg.decode() if msg else "")
    return code
