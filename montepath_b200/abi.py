"""ctypes mirror of ``include/montepath_cuda.h`` and the loader of the CUDA
library ``libmontepath_cuda.so``.

The struct layouts are checked against ``mpc_struct_size`` when the library
loads, so a header change that is not mirrored here fails loudly.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import (
    POINTER,
    Structure,
    c_char,
    c_char_p,
    c_double,
    c_int,
    c_int32,
    c_int64,
    c_size_t,
    c_uint32,
    c_uint64,
    c_void_p,
)

MAX_ASSETS = 8
MAX_EXERCISE_DATES = 64
MAX_LEVELS = 16

# mpc_status_t
OK = 0
E_INVALID_CONFIG = 1
E_UNSUPPORTED = 2
E_NO_DEVICE = 3
E_OOM_BUDGET = 4
E_TIMEOUT = 5
E_CUDA = 6
E_BUSY = 7
E_NOT_FOUND = 8
E_CANCELLED = 9

STATUS_NAMES = {
    OK: "MPC_OK",
    E_INVALID_CONFIG: "MPC_E_INVALID_CONFIG",
    E_UNSUPPORTED: "MPC_E_UNSUPPORTED",
    E_NO_DEVICE: "MPC_E_NO_DEVICE",
    E_OOM_BUDGET: "MPC_E_OOM_BUDGET",
    E_TIMEOUT: "MPC_E_TIMEOUT",
    E_CUDA: "MPC_E_CUDA",
    E_BUSY: "MPC_E_BUSY",
    E_NOT_FOUND: "MPC_E_NOT_FOUND",
    E_CANCELLED: "MPC_E_CANCELLED",
}

# mpc_workload_t
WORKLOAD_EUROPEAN_CALL = 0
WORKLOAD_ARITHMETIC_ASIAN_CALL = 1
WORKLOAD_DOWN_AND_OUT_CALL = 2
WORKLOAD_UP_AND_OUT_CALL = 3
WORKLOAD_LOOKBACK_CALL = 4
WORKLOAD_BASKET_CALL = 5
WORKLOAD_AMERICAN_PUT = 6
WORKLOAD_BERMUDAN_PUT = 7
WORKLOAD_ASIAN_MLMC = 8

WORKLOADS = {
    "european_call": WORKLOAD_EUROPEAN_CALL,
    "arithmetic_asian_call": WORKLOAD_ARITHMETIC_ASIAN_CALL,
    "down_and_out_call": WORKLOAD_DOWN_AND_OUT_CALL,
    "up_and_out_call": WORKLOAD_UP_AND_OUT_CALL,
    "lookback_call": WORKLOAD_LOOKBACK_CALL,
    "basket_call": WORKLOAD_BASKET_CALL,
    "american_put": WORKLOAD_AMERICAN_PUT,
    "bermudan_put": WORKLOAD_BERMUDAN_PUT,
    "arithmetic_asian_mlmc": WORKLOAD_ASIAN_MLMC,
}

MODEL_GBM = 0
MODEL_HESTON = 1
MODEL_MERTON = 2

METHOD_AUTO = 0
METHOD_TERMINAL = 1
METHOD_STEPWISE = 2
METHODS = {
    "auto": METHOD_AUTO,
    "terminal": METHOD_TERMINAL,
    "terminal_distribution": METHOD_TERMINAL,
    "stepwise": METHOD_STEPWISE,
    "stepwise_paths": METHOD_STEPWISE,
}

TECHNIQUE_STANDARD = 0
TECHNIQUE_ANTITHETIC = 1
TECHNIQUE_CONTROL_VARIATE = 2
TECHNIQUES = {
    "standard": TECHNIQUE_STANDARD,
    "antithetic": TECHNIQUE_ANTITHETIC,
    "control_variate": TECHNIQUE_CONTROL_VARIATE,
}

SAMPLING_PSEUDORANDOM = 0
SAMPLING_RANDOMIZED_HALTON = 1
SAMPLING_LATIN_HYPERCUBE = 2
SAMPLING_SCRAMBLED_SOBOL = 3
SAMPLING_SCRAMBLED_SOBOL_BRIDGE = 4
SAMPLING_COUNTER_HASH = 5
SAMPLINGS = {
    "pseudorandom": SAMPLING_PSEUDORANDOM,
    "randomized_halton": SAMPLING_RANDOMIZED_HALTON,
    "latin_hypercube": SAMPLING_LATIN_HYPERCUBE,
    "scrambled_sobol": SAMPLING_SCRAMBLED_SOBOL,
    "scrambled_sobol_brownian_bridge": SAMPLING_SCRAMBLED_SOBOL_BRIDGE,
    "counter_hash": SAMPLING_COUNTER_HASH,
}

PRECISION_FP64_PLAIN = 0
PRECISION_FP32_PATH = 1
PRECISIONS = {"fp64_plain": PRECISION_FP64_PLAIN, "fp32_path": PRECISION_FP32_PATH}

WARN_BASIS_DEGREE_CLAMPED = 0x1
WARN_THREADS_IGNORED = 0x2
WARN_SCHEDULE_NORMALISED = 0x4
WARN_INTRINSIC_FLOOR = 0x8

# mpc_greek_t / mpc_greek_estimator_t
GREEK_DELTA = 0
GREEK_DELTA2 = 1
GREEK_VEGA = 2
GREEK_VEGA2 = 3
GREEK_RHO = 4
GREEK_THETA = 5
GREEK_NAMES = {GREEK_DELTA: "delta", GREEK_DELTA2: "delta2", GREEK_VEGA: "vega", GREEK_VEGA2: "vega2",
               GREEK_RHO: "rho", GREEK_THETA: "theta"}
GREEKS_BUMP_AND_REVALUE = 0
GREEKS_PATHWISE = 1
GREEKS_LIKELIHOOD_RATIO = 2
GREEK_ESTIMATORS = {"bump_and_revalue": GREEKS_BUMP_AND_REVALUE, "pathwise": GREEKS_PATHWISE,
                    "likelihood_ratio": GREEKS_LIKELIHOOD_RATIO}
MAX_GREEKS = 6
GREEK_WARN_ESTIMATOR_UNSUPPORTED = 0x1
GREEK_WARN_PSEUDORANDOM_SHOCKS = 0x2
GREEK_WARN_TECHNIQUE_IGNORED = 0x4


class Request(Structure):
    _fields_ = [
        ("workload", c_int32),
        ("model", c_int32),
        ("method", c_int32),
        ("technique", c_int32),
        ("sampling", c_int32),
        ("precision", c_int32),
        ("n_paths", c_uint64),
        ("n_steps", c_uint32),
        ("n_threads", c_uint32),
        ("seed", c_uint64),
        ("s0", c_double),
        ("k", c_double),
        ("r", c_double),
        ("sigma", c_double),
        ("t", c_double),
        ("barrier", c_double),
        ("v0", c_double),
        ("kappa", c_double),
        ("theta", c_double),
        ("vol_of_vol", c_double),
        ("rho", c_double),
        ("jump_intensity", c_double),
        ("jump_mean", c_double),
        ("jump_volatility", c_double),
        ("n_assets", c_uint32),
        ("_pad0", c_uint32),
        ("spots", c_double * MAX_ASSETS),
        ("sigmas", c_double * MAX_ASSETS),
        ("weights", c_double * MAX_ASSETS),
        ("corr", c_double * (MAX_ASSETS * MAX_ASSETS)),
        ("basis_degree", c_uint32),
        ("n_exercise", c_uint32),
        ("exercise_steps", c_uint32 * MAX_EXERCISE_DATES),
        ("base_steps", c_uint32),
        ("levels", c_uint32),
        ("refinement_factor", c_uint32),
        ("scramble_replicates", c_uint32),
        ("paths_per_level", c_uint64 * MAX_LEVELS),
        ("target_stderr", c_double),
        ("pilot_paths_per_level", c_uint64),
        ("min_step_updates", c_uint64),
        ("max_step_updates", c_uint64),
        ("block_size", c_uint32),
        ("paths_per_thread", c_uint32),
        ("_reserved", c_uint64 * 4),
    ]


class Result(Structure):
    _fields_ = [
        ("price", c_double),
        ("stderr", c_double),
        ("runtime_ms", c_double),
        ("n_samples", c_uint64),
        ("path_steps", c_uint64),
        ("moments", c_double * 6),
        ("early_exercise_count", c_uint64),
        ("maturity_exercise_count", c_uint64),
        ("regression_steps", c_uint32),
        ("basis_degree", c_uint32),
        ("n_levels", c_uint32),
        ("target_met", c_uint32),
        ("max_step_updates_hit", c_uint32),
        ("_pad0", c_uint32),
        ("estimated_stderr", c_double),
        ("total_paths", c_uint64),
        ("total_step_updates", c_uint64),
        ("level_mean", c_double * MAX_LEVELS),
        ("level_variance", c_double * MAX_LEVELS),
        ("level_paths", c_uint64 * MAX_LEVELS),
        ("level_fine_steps", c_uint64 * MAX_LEVELS),
        ("t_enqueue_ms", c_double),
        ("t_admit_ms", c_double),
        ("t_complete_ms", c_double),
        ("status", c_int32),
        ("warnings", c_uint32),
    ]


class DeviceInfo(Structure):
    _fields_ = [
        ("index", c_int32),
        ("sm_count", c_int32),
        ("cc_major", c_int32),
        ("cc_minor", c_int32),
        ("total_memory_bytes", c_uint64),
        ("free_memory_bytes", c_uint64),
        ("clock_khz", c_int32),
        ("l2_bytes", c_int32),
        ("name", c_char * 96),
    ]


class Options(Structure):
    _fields_ = [
        ("device", c_int32),
        ("deterministic", c_int32),
        ("hbm_budget_bytes", c_uint64),
        ("default_block_size", c_uint32),
        ("_pad0", c_uint32),
    ]


class Support(Structure):
    _fields_ = [
        ("supported", c_int32),
        ("reason", c_int32),
        ("estimated_bytes", c_uint64),
        ("message", c_char * 160),
    ]


class Artifact(Structure):
    _fields_ = [
        ("kernel_family", c_int32),
        ("block_size", c_uint32),
        ("paths_per_thread", c_uint32),
        ("tiles", c_uint32),
        ("bytes", c_uint64),
        ("name", c_char * 96),
    ]


class ServerOptions(Structure):
    _fields_ = [
        ("hbm_budget_bytes", c_uint64),
        ("max_slots", c_uint32),
        ("wave_tiles", c_uint32),
        ("mode", c_uint32),
        ("reserve_sms", c_uint32),
    ]


class ServerStats(Structure):
    _fields_ = [
        ("submitted", c_uint64),
        ("admitted", c_uint64),
        ("completed", c_uint64),
        ("rejected", c_uint64),
        ("cancelled", c_uint64),
        ("waves", c_uint64),
        ("live_bytes", c_uint64),
        ("peak_bytes", c_uint64),
        ("p50_ms", c_double),
        ("p99_ms", c_double),
        ("mean_ms", c_double),
        ("max_ms", c_double),
        ("busy_ms", c_double),
        ("wall_ms", c_double),
        ("path_steps", c_uint64),
    ]


class GreekEstimate(Structure):
    _fields_ = [
        ("greek", c_int32),
        ("estimator", c_int32),
        ("value", c_double),
        ("stderr", c_double),
        ("bump_size", c_double),
        ("base_price", c_double),
        ("bumped_up_price", c_double),
        ("bumped_down_price", c_double),
    ]


class GreekReport(Structure):
    _fields_ = [
        ("workload", c_int32),
        ("estimator", c_int32),
        ("paths", c_uint64),
        ("steps", c_uint32),
        ("n_estimates", c_uint32),
        ("seed", c_uint64),
        ("base_price", c_double),
        ("base_stderr", c_double),
        ("runtime_ms", c_double),
        ("estimates", GreekEstimate * MAX_GREEKS),
        ("warnings", c_uint32),
        ("status", c_int32),
    ]


class Cost(Structure):
    _fields_ = [
        ("estimated_compile_ms", c_double),
        ("estimated_runtime_ms", c_double),
        ("estimated_total_ms", c_double),
        ("estimated_peak_memory_mb", c_double),
        ("path_steps_per_sec", c_double),
        ("path_steps", c_uint64),
        ("confidence", c_char * 16),
    ]


STRUCTS = [Request, Result, DeviceInfo, Options, Support, Artifact, ServerOptions, ServerStats, GreekReport, Cost]

# (name, restype, argtypes) of every exported entry point, in header order.
FUNCTIONS = [
    ("mpc_abi_version", c_int, []),
    ("mpc_struct_size", c_size_t, [c_int]),
    ("mpc_status_string", c_char_p, [c_int]),
    ("mpc_device_count", c_int, [POINTER(c_int)]),
    ("mpc_device_info", c_int, [c_int, POINTER(DeviceInfo)]),
    ("mpc_request_defaults", c_int, [POINTER(Request), c_int]),
    ("mpc_validate", c_int, [POINTER(Request), c_char_p, c_size_t]),
    ("mpc_supports", c_int, [POINTER(Request), POINTER(Support)]),
    ("mpc_estimate_bytes", c_int, [POINTER(Request), POINTER(c_uint64)]),
    ("mpc_estimate_cost", c_int, [POINTER(Request), c_int, POINTER(Cost)]),
    ("mpc_estimate_cost_ctx", c_int, [c_void_p, POINTER(Request), POINTER(Cost)]),
    ("mpc_calibrate_cost", c_int, [c_void_p, POINTER(c_double)]),
    ("mpc_create", c_int, [POINTER(Options), POINTER(c_void_p)]),
    ("mpc_destroy", c_int, [c_void_p]),
    ("mpc_last_error_message", c_char_p, [c_void_p]),
    ("mpc_prepare", c_int, [c_void_p, POINTER(Request), POINTER(Artifact)]),
    ("mpc_price", c_int, [c_void_p, POINTER(Request), POINTER(Result)]),
    ("mpc_price_batch", c_int, [c_void_p, POINTER(Request), c_size_t, POINTER(Result)]),
    ("mpc_greeks", c_int, [c_void_p, POINTER(Request), c_int, POINTER(GreekReport)]),
    ("mpc_price_paths", c_int, [c_void_p, POINTER(Request), POINTER(c_double), c_uint64]),
    ("mpc_generate_normals", c_int, [c_void_p, c_int, c_uint64, c_uint64, c_uint32, c_int, c_void_p]),
    ("mpc_counter_hash_u32", c_int, [c_void_p, c_uint32, c_uint32, c_uint32, POINTER(c_uint32)]),
    ("mpc_xorshift_u64", c_int, [c_void_p, c_uint64, c_uint64, c_uint64, POINTER(c_uint64)]),
    (
        "mpc_european_call_stepwise_v1",
        c_int,
        [c_void_p, c_void_p, c_int32, c_int32, c_double, c_double, c_double, c_double, c_double, c_void_p],
    ),
    ("mpc_flush_l2", c_int, [c_void_p]),
    ("mpc_last_timing", c_int, [c_void_p, POINTER(c_double), POINTER(c_uint64)]),
    ("mpc_last_transfer", c_int, [c_void_p, POINTER(c_uint64), POINTER(c_uint64)]),
    ("mpc_measure_peaks", c_int, [c_void_p, POINTER(c_double), POINTER(c_double)]),
    ("mpc_price_fused_noalloc", c_int, [POINTER(Request), POINTER(Result), c_void_p, c_char_p, c_size_t]),
    ("mpc_server_start", c_int, [c_void_p, POINTER(ServerOptions), POINTER(c_void_p)]),
    ("mpc_submit", c_int, [c_void_p, POINTER(Request), POINTER(c_uint64)]),
    ("mpc_poll", c_int, [c_void_p, c_uint64, POINTER(Result)]),
    ("mpc_wait", c_int, [c_void_p, c_uint64, c_int64, POINTER(Result)]),
    ("mpc_cancel", c_int, [c_void_p, c_uint64]),
    ("mpc_server_stats", c_int, [c_void_p, POINTER(ServerStats)]),
    ("mpc_server_stop", c_int, [c_void_p]),
]

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(PACKAGE_DIR, "lib", "libmontepath_cuda.so")

_LIB = None


class LibraryNotBuiltError(RuntimeError):
    """The CUDA library has not been compiled; there is no CPU fallback."""


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load ``libmontepath_cuda.so`` and bind every entry point.

    Raises LibraryNotBuiltError when the library is missing: the backend has
    no CPU fallback by design.
    """

    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    lib_path = path or LIBRARY_PATH
    if not os.path.exists(lib_path):
        raise LibraryNotBuiltError(
            f"{lib_path} is missing; build it with `python -m montepath_b200.build` "
            "(the CUDA backend has no CPU fallback)"
        )
    lib = ctypes.CDLL(lib_path)
    for name, restype, argtypes in FUNCTIONS:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    for index, struct in enumerate(STRUCTS):
        native = lib.mpc_struct_size(index)
        if native != ctypes.sizeof(struct):
            raise RuntimeError(
                f"ABI mismatch: {struct.__name__} is {ctypes.sizeof(struct)} bytes in Python, "
                f"{native} in the library"
            )
    if path is None:
        _LIB = lib
    return lib


def status_name(status: int) -> str:
    return STATUS_NAMES.get(status, f"MPC_STATUS_{status}")
