"""Backend-selection overlay: the ``nvidia_cuda`` branch of montepath's
production layer, which the reference hard-codes as deferred
(python/montepath/production.py:240-251 reports status ``"deferred"`` and
:397-404 returns ``MC_BACKEND_CUDA_DEFERRED``).

``select_backend("european_call", backend="cuda")`` here reports the CUDA
backend as available when the sm_100a library loads and a device answers,
and ``execute_workload`` prices through the mapping-ABI functions of
``montepath_b200.native``.  Other backend names are left to montepath.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Any, Mapping

from . import abi

NATIVE_MODULE = "montepath_b200.native"

# production.py:92-103
BACKEND_ALIASES = {"cuda": "nvidia_cuda", "nvidia_cuda": "nvidia_cuda"}

CUDA_FUNCTION_BY_WORKLOAD = {
    "european_call": "price_european_call",
    "arithmetic_asian_call": "price_arithmetic_asian_call",
    "down_and_out_call": "price_down_and_out_call",
    "up_and_out_call": "price_up_and_out_call",
    "lookback_call": "price_lookback_call",
    "basket_call": "price_basket_call",
    "american_put": "price_american_put",
    "bermudan_put": "price_bermudan_put",
    "heston_european_call": "price_heston_european_call",
    "merton_jump_diffusion_call": "price_merton_jump_diffusion_call",
    "european_call_parameter_sweep": "price_european_call_parameter_sweep",
    "arithmetic_asian_mlmc": "arithmetic_asian_mlmc",
}


class ProductionCapabilityError(RuntimeError):
    def __init__(self, selection: "BackendSelection"):
        self.selection = selection
        super().__init__("; ".join(d["message"] for d in selection.diagnostics) or "backend unavailable")


@dataclass(frozen=True)
class BackendSelection:
    ok: bool
    backend_id: str
    execution_mode: str
    workload: str
    agent_tool_ready: bool
    diagnostics: tuple = ()
    warnings: tuple = ()
    native_module: str | None = NATIVE_MODULE
    devices: tuple = field(default_factory=tuple)

    def as_dict(self) -> dict[str, Any]:
        return {
            "ok": self.ok,
            "backend_id": self.backend_id,
            "execution_mode": self.execution_mode,
            "workload": self.workload,
            "agent_tool_ready": self.agent_tool_ready,
            "diagnostics": list(self.diagnostics),
            "warnings": list(self.warnings),
            "native_module": self.native_module,
            "devices": list(self.devices),
        }


def cuda_devices() -> list[dict[str, Any]]:
    """Replaces the nvidia-smi parsing of NvidiaCudaBackend::discover_devices (cuda.rs:205-241)."""

    lib = abi.load_library()
    count = ctypes.c_int()
    if lib.mpc_device_count(ctypes.byref(count)) != abi.OK:
        return []
    out = []
    for index in range(count.value):
        info = abi.DeviceInfo()
        if lib.mpc_device_info(index, ctypes.byref(info)) == abi.OK:
            out.append(
                {
                    "index": info.index,
                    "name": info.name.decode(),
                    "compute_capability": f"{info.cc_major}.{info.cc_minor}",
                    "sm_count": info.sm_count,
                    "total_memory_bytes": info.total_memory_bytes,
                    "free_memory_bytes": info.free_memory_bytes,
                }
            )
    return out


def cuda_capability() -> dict[str, Any]:
    """The BackendCapability record of the nvidia_cuda backend (replaces production.py:240-251)."""

    try:
        devices = cuda_devices()
        reason = None if devices else "no CUDA device visible"
    except abi.LibraryNotBuiltError as exc:
        devices, reason = [], str(exc)
    available = bool(devices) and any(d["compute_capability"] == "10.0" for d in devices)
    if devices and not available:
        reason = "the library is compiled for sm_100a (B200) only"
    return {
        "backend_id": "nvidia_cuda",
        "display_name": "NVIDIA CUDA runtime (B200, sm_100a)",
        "status": "available" if available else "unavailable",
        "execution_mode": "native_cuda_sm100a",
        "workloads": sorted(CUDA_FUNCTION_BY_WORKLOAD),
        "agent_tool_ready": available,
        "deterministic": "deterministic for same config, seed, library version and GPU (fixed-order reductions)",
        "reason": reason,
        "native_module": NATIVE_MODULE,
        "devices": devices,
    }


def select_backend(workload: str, *, backend: str = "cuda", native_module: str = NATIVE_MODULE) -> BackendSelection:
    """select_backend for the CUDA branch (production.py:254-412)."""

    normalized = BACKEND_ALIASES.get(backend)
    if normalized is None:
        return BackendSelection(False, backend, "none", workload, False,
                                ({"code": "MC_BACKEND_UNKNOWN", "message": f"{backend!r} is not a CUDA backend name"},))
    if workload not in CUDA_FUNCTION_BY_WORKLOAD:
        return BackendSelection(False, normalized, "none", workload, False,
                                ({"code": "MC_BACKEND_CUDA_WORKLOAD", "message": f"workload {workload!r} has no CUDA kernel"},))
    cap = cuda_capability()
    if cap["status"] != "available":
        return BackendSelection(False, normalized, "none", workload, False,
                                ({"code": "MC_BACKEND_CUDA_UNAVAILABLE", "message": cap["reason"] or "unavailable"},),
                                native_module=native_module)
    return BackendSelection(True, normalized, "native_cuda_sm100a", workload, True,
                            warnings=("FP32-path results carry their stderr; compare against the FP64 oracle tolerance.",),
                            native_module=native_module, devices=tuple(d["name"] for d in cap["devices"]))


def execute_workload(workload: str, config: Mapping[str, Any] | None = None, *, backend: str = "cuda") -> dict[str, Any]:
    """execute_workload (production.py:440-481) on the CUDA backend."""

    selection = select_backend(workload, backend=backend)
    if not selection.ok:
        raise ProductionCapabilityError(selection)
    from . import native

    function = getattr(native, CUDA_FUNCTION_BY_WORKLOAD[workload])
    result = function(dict(config or {}))
    return {
        "ok": True,
        "schema_version": "montepath-execution.v1",
        "workload": workload,
        "selection": selection.as_dict(),
        "result": result,
        "manifest": result["manifest"],
        "warnings": list(result["warnings"]),
    }


def estimate_cost(workload: str, config: Mapping[str, Any] | None = None, *, sm_count: int = 0) -> dict[str, Any]:
    """NvidiaCudaBackend::estimate_cost (crates/mc-core/src/backend/cuda.rs:121-152)
    from the measured cost model (``mpc_estimate_cost``; host only, no GPU needed)."""

    from .requests import make_request

    params = dict(config or {})
    code = {"heston_european_call": "european_call", "merton_jump_diffusion_call": "european_call"}.get(workload, workload)
    if workload == "heston_european_call":
        params.setdefault("model", "heston")
        params.setdefault("method", "stepwise")
    if workload == "merton_jump_diffusion_call":
        params.setdefault("model", "merton")
        params.setdefault("sampling", "counter_hash")
    req = make_request(code, params)
    cost = abi.Cost()
    status = abi.load_library().mpc_estimate_cost(ctypes.byref(req), int(sm_count), ctypes.byref(cost))
    if status != abi.OK:
        raise ValueError(f"MC_CONFIG_INVALID: {abi.status_name(status)}")
    return {
        "backend_id": "nvidia_cuda",
        "estimated_compile_ms": cost.estimated_compile_ms,
        "estimated_runtime_ms": cost.estimated_runtime_ms,
        "estimated_total_ms": cost.estimated_total_ms,
        "estimated_peak_memory_mb": cost.estimated_peak_memory_mb,
        "confidence": cost.confidence.decode(),
        "path_steps": cost.path_steps,
        "path_steps_per_sec": cost.path_steps_per_sec,
    }


def planner_priority(workload: str, config: Mapping[str, Any] | None = None, *,
                     cuda_available: bool | None = None) -> list[str]:
    """Backend order for one run, by estimated total time: the CUDA estimate
    from the measured cost model against the reference's CPU estimate
    (CpuNativeBackend::estimate_cost, backend/mod.rs:292-305: n_paths x n_steps
    / 5e6 per ms).  Stands in for the fixed thresholds of backend_priority
    (planner/mod.rs:509-549) when the CUDA backend is present; Apple Metal is
    never available on this hardware and goes last."""

    cfg = dict(config or {})
    paths = int(cfg.get("n_paths", 10_000))
    steps = int(cfg.get("n_steps", 1)) if workload not in ("european_call",) or cfg.get("method") == "stepwise" else 1
    cpu_ms = max(paths * max(steps, 1) / 5_000_000.0, 0.01)
    if cuda_available is None:
        cuda_available = cuda_capability()["status"] == "available"
    if not cuda_available:
        return ["cpu_native", "nvidia_cuda", "apple_metal"]
    cuda_ms = estimate_cost(workload, cfg)["estimated_total_ms"]
    return (["nvidia_cuda", "cpu_native"] if cuda_ms < cpu_ms else ["cpu_native", "nvidia_cuda"]) + ["apple_metal"]
