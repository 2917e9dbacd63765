"""ctypes wrapper of the FP64 CPU oracle (oracle/mp_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU leg (``cpu_baseline`` / ``cpu_leg``, and the reference
arm), to check results and to time the CPU path.  The product
(``montepath_b200``) never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_uint32, c_uint64

import numpy as np

from montepath_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmp_oracle.so")
_SOURCES = [
    os.path.join(HERE, "mp_oracle.cpp"),
    os.path.join(HERE, "..", "include", "montepath_cuda.h"),
    os.path.join(HERE, "..", "montepath_b200", "csrc", "sobol_directions.h"),
]

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with gcc through oracle/Makefile."""

    stale = not os.path.exists(LIB_PATH) or any(
        os.path.getmtime(src) > os.path.getmtime(LIB_PATH) for src in _SOURCES
    )
    if force or stale:
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "or_splitmix64": (c_uint64, [c_uint64]),
        "or_derive_chunk_seed": (c_uint64, [c_uint64, c_uint64]),
        "or_xorshift_u64": (None, [c_uint64, c_uint64, POINTER(c_uint64)]),
        "or_pseudorandom_normals": (None, [c_uint64, c_uint64, POINTER(c_double)]),
        "or_hash_u32": (c_uint32, [c_uint32]),
        "or_counter_hash": (c_uint32, [c_uint32, c_uint32, c_uint32, c_uint32]),
        "or_counter_uniform_f32": (c_float, [c_uint32, c_uint32, c_uint32, c_uint32]),
        "or_stateless_normals_f32": (None, [c_uint64, c_uint64, c_uint64, POINTER(c_float)]),
        "or_inverse_normal": (c_double, [c_double]),
        "or_sobol_unscrambled": (c_uint32, [c_uint32, c_uint32]),
        "or_sobol_owen": (c_uint32, [c_uint32, c_uint32, c_uint32]),
        "or_sobol_point": (c_uint32, [c_uint64, c_uint64, c_uint32]),
        "or_halton": (c_double, [c_uint64, c_uint32]),
        "or_generate_normals": (None, [c_int, c_uint64, c_uint64, c_uint64, POINTER(c_double)]),
        "or_generate_uniforms": (None, [c_int, c_uint64, c_uint64, c_uint64, POINTER(c_double)]),
        "or_price": (c_int, [POINTER(abi.Request), POINTER(abi.Result)]),
        "or_request_defaults": (c_int, [POINTER(abi.Request), c_int]),
        "or_greeks": (c_int, [POINTER(abi.Request), c_int, POINTER(abi.GreekReport)]),
        "or_price_paths": (c_int, [POINTER(abi.Request), POINTER(abi.Result), POINTER(c_double), c_uint64]),
        "or_price_from_f32_normals": (
            None,
            [POINTER(abi.Request), POINTER(c_float), POINTER(abi.Result), POINTER(c_double)],
        ),
        "or_price_threaded": (c_int, [POINTER(abi.Request), c_int, POINTER(abi.Result)]),
        "or_bs_call": (c_double, [c_double] * 5 + [c_int]),
        "or_bs_put": (c_double, [c_double] * 5 + [c_int]),
        "or_bs_greeks": (None, [c_double] * 5 + [c_int, POINTER(c_double)]),
        "or_merton_series": (c_double, [c_double] * 8 + [c_int, c_double, c_int]),
        "or_crr_put": (c_double, [c_double] * 5 + [c_int, POINTER(c_uint32), c_int]),
        "or_heston_call": (c_double, [c_double] * 9),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(arr, ctype):
    return arr.ctypes.data_as(POINTER(ctype))


def xorshift_u64(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    lib().or_xorshift_u64(seed, count, _ptr(out, c_uint64))
    return out


def pseudorandom_normals(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.float64)
    lib().or_pseudorandom_normals(seed, count, _ptr(out, c_double))
    return out


def stateless_normals_f32(seed: int, n_paths: int, n_steps: int) -> np.ndarray:
    out = np.zeros(n_paths * n_steps, dtype=np.float32)
    lib().or_stateless_normals_f32(seed, n_paths, n_steps, _ptr(out, c_float))
    return out


def generate_normals(sampling: int, seed: int, n_points: int, dims: int) -> np.ndarray:
    out = np.zeros(n_points * dims, dtype=np.float64)
    lib().or_generate_normals(sampling, seed, n_points, dims, _ptr(out, c_double))
    return out.reshape(n_points, dims)


def generate_uniforms(sampling: int, seed: int, n_points: int, dims: int) -> np.ndarray:
    out = np.zeros(n_points * dims, dtype=np.float64)
    lib().or_generate_uniforms(sampling, seed, n_points, dims, _ptr(out, c_double))
    return out.reshape(n_points, dims)


def request_defaults(workload: int) -> abi.Request:
    """The reference configs' Default values, from the oracle's own copy."""

    req = abi.Request()
    if lib().or_request_defaults(ctypes.byref(req), int(workload)) != 0:
        raise ValueError(f"unknown workload {workload}")
    return req


def make_request(workload, config=None, **overrides) -> abi.Request:
    """A request built from a config mapping like montepath_b200.requests.make_request,
    with the oracle's defaults: loads nothing from the CUDA library."""

    from montepath_b200.requests import make_request as _make

    return _make(workload, config, defaults=request_defaults, **overrides)


def price(req: abi.Request) -> abi.Result:
    res = abi.Result()
    lib().or_price(ctypes.byref(req), ctypes.byref(res))
    return res


def greeks(req: abi.Request, estimator: int) -> tuple[int, abi.GreekReport]:
    """Greek report of the CPU restatement (cpu.rs:4036-5010): (status, report)."""
    rep = abi.GreekReport()
    status = lib().or_greeks(ctypes.byref(req), int(estimator), ctypes.byref(rep))
    return status, rep


def price_paths(req: abi.Request, capacity: int | None = None) -> tuple[abi.Result, np.ndarray]:
    units = req.n_paths
    if req.technique == abi.TECHNIQUE_ANTITHETIC:
        units = (req.n_paths + 1) // 2
    capacity = capacity or units
    out = np.full(capacity, np.nan, dtype=np.float64)
    res = abi.Result()
    lib().or_price_paths(ctypes.byref(req), ctypes.byref(res), _ptr(out, c_double), capacity)
    return res, out


def price_from_f32_normals(req: abi.Request, normals: np.ndarray) -> tuple[abi.Result, np.ndarray]:
    normals = np.ascontiguousarray(normals, dtype=np.float32)
    res = abi.Result()
    per_path = np.zeros(req.n_paths, dtype=np.float64)
    lib().or_price_from_f32_normals(ctypes.byref(req), _ptr(normals, c_float), ctypes.byref(res), _ptr(per_path, c_double))
    return res, per_path


def price_threaded(req: abi.Request, threads: int) -> abi.Result:
    res = abi.Result()
    lib().or_price_threaded(ctypes.byref(req), threads, ctypes.byref(res))
    return res


def bs_call(s0, k, r, sigma, t, exact: bool = False) -> float:
    return lib().or_bs_call(s0, k, r, sigma, t, 1 if exact else 0)


def bs_put(s0, k, r, sigma, t, exact: bool = False) -> float:
    return lib().or_bs_put(s0, k, r, sigma, t, 1 if exact else 0)


def bs_greeks(s0, k, r, sigma, t, exact: bool = False) -> dict:
    out = (c_double * 5)()
    lib().or_bs_greeks(s0, k, r, sigma, t, 1 if exact else 0, out)
    return dict(zip(("price", "delta", "vega", "rho", "theta"), list(out)))


def merton_series(s0, k, r, sigma, lam, mj, sj, t, max_terms=96, tail_tol=1e-12, exact: bool = False) -> float:
    return lib().or_merton_series(s0, k, r, sigma, lam, mj, sj, t, max_terms, tail_tol, 1 if exact else 0)


def crr_put(s0, k, r, sigma, t, ref_steps, exercise_steps=None) -> float:
    if exercise_steps is None:
        return lib().or_crr_put(s0, k, r, sigma, t, ref_steps, None, 0)
    arr = (c_uint32 * len(exercise_steps))(*exercise_steps)
    return lib().or_crr_put(s0, k, r, sigma, t, ref_steps, arr, len(exercise_steps))


def heston_call(s0, k, r, v0, kappa, theta, xi, rho, t) -> float:
    return lib().or_heston_call(s0, k, r, v0, kappa, theta, xi, rho, t)
