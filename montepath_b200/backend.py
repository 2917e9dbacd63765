"""Python handle on the CUDA backend: a context owning the device, its
stream and its HBM-budgeted buffers, plus the serving loop.

This is the runtime object behind ``NvidiaCudaBackend::execute``
(crates/mc-core/src/backend/cuda.rs:187-193): every call prices on the GPU or
raises; there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
from ctypes import byref, c_double, c_uint64, c_void_p
from typing import Sequence

import numpy as np

from . import abi


class BackendError(RuntimeError):
    """A non-zero status from the C ABI, with its code and message."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.code = abi.status_name(status)
        super().__init__(f"{self.code}: {message}")


class CudaBackend:
    """One device context (``mpc_create``)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = abi.load_library()
        opts = abi.Options(device=device, deterministic=1, hbm_budget_bytes=hbm_budget_bytes)
        handle = c_void_p()
        status = self.lib.mpc_create(byref(opts), byref(handle))
        if status != abi.OK:
            raise BackendError(status, f"mpc_create failed on device {device}")
        self.handle = handle
        self.device = device

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.mpc_destroy(self.handle)
            self.handle = None

    def __enter__(self) -> "CudaBackend":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int) -> None:
        if status != abi.OK:
            raise BackendError(status, self.lib.mpc_last_error_message(self.handle).decode())

    def price(self, req: abi.Request) -> abi.Result:
        res = abi.Result()
        self._check(self.lib.mpc_price(self.handle, byref(req), byref(res)))
        return res

    def price_batch(self, reqs: Sequence[abi.Request]) -> list[abi.Result]:
        n = len(reqs)
        arr = (abi.Request * n)(*reqs)
        out = (abi.Result * n)()
        self._check(self.lib.mpc_price_batch(self.handle, arr, n, out))
        return list(out)

    def greeks(self, req: abi.Request, estimator: int | str = abi.GREEKS_BUMP_AND_REVALUE) -> abi.GreekReport:
        """GreekReport of one request (the reference's ``*_greeks_cpu``):
        bump-and-revalue for every workload with Greeks, pathwise and
        likelihood ratio for the terminal-GBM European call."""
        if isinstance(estimator, str):
            estimator = abi.GREEK_ESTIMATORS[estimator]
        rep = abi.GreekReport()
        self._check(self.lib.mpc_greeks(self.handle, byref(req), int(estimator), byref(rep)))
        return rep

    def price_paths(self, req: abi.Request) -> np.ndarray:
        units = req.n_paths
        if req.technique == abi.TECHNIQUE_ANTITHETIC:
            units = (req.n_paths + 1) // 2
        out = np.zeros(units, dtype=np.float64)
        self._check(self.lib.mpc_price_paths(self.handle, byref(req), out.ctypes.data_as(ctypes.POINTER(c_double)), units))
        return out

    def prepare(self, req: abi.Request) -> abi.Artifact:
        art = abi.Artifact()
        self._check(self.lib.mpc_prepare(self.handle, byref(req), byref(art)))
        return art

    def generate_normals(self, sampling: int, seed: int, n_points: int, dims: int, fp32: bool = False) -> np.ndarray:
        dtype = np.float32 if fp32 else np.float64
        out = np.zeros((n_points, dims), dtype=dtype)
        precision = abi.PRECISION_FP32_PATH if fp32 else abi.PRECISION_FP64_PLAIN
        self._check(
            self.lib.mpc_generate_normals(self.handle, sampling, seed, n_points, dims, precision, out.ctypes.data_as(c_void_p))
        )
        return out

    def counter_hash(self, seed: int, n_paths: int, n_steps: int) -> np.ndarray:
        out = np.zeros(n_paths * n_steps * 2, dtype=np.uint32)
        self._check(
            self.lib.mpc_counter_hash_u32(self.handle, seed, n_paths, n_steps, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        )
        return out.reshape(n_paths, n_steps, 2)

    def xorshift(self, seed: int, offset: int, count: int) -> np.ndarray:
        out = np.zeros(count, dtype=np.uint64)
        self._check(self.lib.mpc_xorshift_u64(self.handle, seed, offset, count, out.ctypes.data_as(ctypes.POINTER(c_uint64))))
        return out

    def flush_l2(self) -> None:
        self._check(self.lib.mpc_flush_l2(self.handle))

    def last_timing(self) -> tuple[float, int]:
        ms = c_double()
        launches = c_uint64()
        self.lib.mpc_last_timing(self.handle, byref(ms), byref(launches))
        return ms.value, launches.value

    def last_transfer(self) -> tuple[int, int]:
        h2d = c_uint64()
        d2h = c_uint64()
        self.lib.mpc_last_transfer(self.handle, byref(h2d), byref(d2h))
        return h2d.value, d2h.value

    def measure_peaks(self) -> tuple[float, float]:
        fp32 = c_double()
        sfu = c_double()
        self._check(self.lib.mpc_measure_peaks(self.handle, byref(fp32), byref(sfu)))
        return fp32.value, sfu.value

    def calibrate_cost(self) -> float:
        """Measures this device's cost-model rates (mpc_calibrate_cost); returns the seconds it took."""
        seconds = c_double()
        self._check(self.lib.mpc_calibrate_cost(self.handle, byref(seconds)))
        return seconds.value

    def estimate_cost(self, req: abi.Request) -> abi.Cost:
        """Cost estimate from this context's rates (mpc_estimate_cost_ctx)."""
        cost = abi.Cost()
        self._check(self.lib.mpc_estimate_cost_ctx(self.handle, byref(req), byref(cost)))
        return cost

    def server(self, hbm_budget_bytes: int = 0, max_slots: int = 0, wave_tiles: int = 0, plain: bool = False,
               mode: str | None = None) -> "Server":
        """mode: "device_loop" (resident device loop), "waves" (host-scheduled
        waves) or "plain" (FIFO FP64, one request per launch); `plain=True`
        selects "plain"; the default is "device_loop"."""
        return Server(self, hbm_budget_bytes, max_slots, wave_tiles, mode or ("plain" if plain else "device_loop"))


SERVER_MODES = {"waves": 0, "plain": 1, "device_loop": 2}


class Server:
    """Serving loop (``mpc_server_start``): the resident device loop,
    host-scheduled waves, or the plain FIFO baseline."""

    def __init__(self, backend: CudaBackend, hbm_budget_bytes: int, max_slots: int, wave_tiles: int, mode: str):
        self.backend = backend
        self.lib = backend.lib
        self.mode = mode
        opts = abi.ServerOptions(
            hbm_budget_bytes=hbm_budget_bytes, max_slots=max_slots, wave_tiles=wave_tiles, mode=SERVER_MODES[mode]
        )
        handle = c_void_p()
        status = self.lib.mpc_server_start(backend.handle, byref(opts), byref(handle))
        if status != abi.OK:
            raise BackendError(status, backend.lib.mpc_last_error_message(backend.handle).decode())
        self.handle = handle

    def submit(self, req: abi.Request) -> int:
        ticket = c_uint64()
        status = self.lib.mpc_submit(self.handle, byref(req), byref(ticket))
        if status != abi.OK:
            raise BackendError(status, "request rejected at submission")
        return ticket.value

    def poll(self, ticket: int) -> abi.Result | None:
        res = abi.Result()
        status = self.lib.mpc_poll(self.handle, ticket, byref(res))
        if status == abi.E_BUSY:
            return None
        if status != abi.OK:
            raise BackendError(status, f"ticket {ticket}")
        return res

    def wait(self, ticket: int, timeout_ms: int = 60_000) -> abi.Result:
        res = abi.Result()
        status = self.lib.mpc_wait(self.handle, ticket, timeout_ms, byref(res))
        if status != abi.OK:
            raise BackendError(status, f"ticket {ticket}")
        return res

    def cancel(self, ticket: int) -> int:
        return self.lib.mpc_cancel(self.handle, ticket)

    def stats(self) -> abi.ServerStats:
        st = abi.ServerStats()
        self.lib.mpc_server_stats(self.handle, byref(st))
        return st

    def stop(self) -> None:
        if self.handle:
            self.lib.mpc_server_stop(self.handle)
            self.handle = None

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> None:
        self.stop()
