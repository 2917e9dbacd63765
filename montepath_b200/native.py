"""Mapping-ABI module for montepath's Python surface, backed by the CUDA library.

montepath's pricing helpers call a native module by name with a config
mapping and expect a mapping back (python/montepath/pricing.py:711-780):

    price_european_call(native_module="montepath_b200.native", ...)

Every function here has the name and the ``fn(mapping) -> dict`` shape of
the reference's PyO3 bridge (crates/montepath-python/src/lib.rs:24-284,
response shape ``pricing_response`` lib.rs:680-707): ``price``, ``stderr``,
``values``, ``manifest`` (``backend: "nvidia_cuda"``) and ``warnings``.  The
``*_cuda`` aliases mirror the naming of the Metal bridge
(``price_european_call_metal``, production.py:80-90).  Pricing always runs on
the GPU; a request the device path cannot run raises with its status code.
"""

from __future__ import annotations

import math
import threading
from typing import Any, Mapping

from . import abi
from .backend import BackendError, CudaBackend
from .requests import ConfigError, make_request, request_to_dict

__version__ = "0.1.0"

_lock = threading.Lock()
_backend: CudaBackend | None = None


def backend() -> CudaBackend:
    """The process-wide device context (created on first use, device 0)."""

    global _backend
    with _lock:
        if _backend is None:
            _backend = CudaBackend(0)
        return _backend


def _manifest(workload: str, function: str, config: Mapping[str, Any], req: abi.Request) -> dict:
    precision = "fp64_plain" if req.precision == abi.PRECISION_FP64_PLAIN else "fp32_path"
    return {
        "schema_version": "python-native-runtime.v1",
        "workload": workload,
        "backend": "nvidia_cuda",
        "execution_mode": "native_cuda_sm100a",
        "function": function,
        "native_module": __name__,
        "config": dict(config),
        "request": request_to_dict(req),
        "precision": precision,
        "reproducibility": (
            "deterministic for identical config, seed, library version and GPU: fixed tile order reductions; "
            "pseudorandom sampling replays the reference MonteCarloRng stream"
        ),
        "performance_claim": "use bench.py artifacts for timing claims",
    }


def _warnings(req: abi.Request, res: abi.Result, config: Mapping[str, Any]) -> list[str]:
    out = []
    if req.precision == abi.PRECISION_FP32_PATH:
        out.append("path arithmetic in FP32 with FP64 accumulation; compare against the FP64 oracle tolerance")
    if config.get("n_threads", 0) == 0 and req.sampling == abi.SAMPLING_PSEUDORANDOM:
        out.append("n_threads=0 runs one deterministic pseudorandom stream (the reference uses the host core count)")
    if res.warnings & abi.WARN_BASIS_DEGREE_CLAMPED:
        out.append("basis_degree was clamped to the supported range [1, 3].")
    if res.warnings & abi.WARN_SCHEDULE_NORMALISED:
        out.append("exercise_steps were sorted, deduplicated and maturity-appended before LSM execution.")
    if res.warnings & abi.WARN_THREADS_IGNORED:
        out.append("n_threads is accepted for API symmetry; the LSM regression runs as one GPU launch.")
    return out


def _values(res: abi.Result, req: abi.Request) -> dict:
    values = {
        "price": res.price,
        "stderr": res.stderr,
        "runtime_ms": res.runtime_ms,
        "samples": res.n_samples,
        "path_steps": res.path_steps,
    }
    if req.workload in (abi.WORKLOAD_AMERICAN_PUT, abi.WORKLOAD_BERMUDAN_PUT):
        values.update(
            early_exercise_count=res.early_exercise_count,
            maturity_exercise_count=res.maturity_exercise_count,
            regression_steps=res.regression_steps,
            regression_basis=f"laguerre_lsm_degree_{res.basis_degree}",
            paths=req.n_paths,
            steps=req.n_steps,
            seed=req.seed,
        )
    if req.workload == abi.WORKLOAD_ASIAN_MLMC:
        levels = []
        for level in range(res.n_levels):
            fine = res.level_fine_steps[level]
            levels.append(
                {
                    "level": level,
                    "paths": res.level_paths[level],
                    "fine_steps": fine,
                    "coarse_steps": None if level == 0 else fine // max(req.refinement_factor, 1),
                    "mean": res.level_mean[level],
                    "variance": res.level_variance[level],
                }
            )
        values.update(
            total_paths=res.total_paths,
            total_step_updates=res.total_step_updates,
            levels=levels,
            target_met=bool(res.target_met) if req.target_stderr > 0 else None,
            estimated_stderr=res.estimated_stderr if req.target_stderr > 0 else None,
        )
    return values


def _price(workload: str, function: str, config: Mapping[str, Any], extra: Mapping[str, Any] | None = None) -> dict:
    cfg = dict(config or {})
    params = dict(cfg)
    params.update(extra or {})
    try:
        req = make_request(workload, params)
    except ConfigError as exc:
        raise ValueError(f"MC_CONFIG_INVALID: {exc}") from exc
    res = abi.Result()
    be = backend()
    try:
        res = be.price(req)
    except BackendError as exc:
        raise ValueError(f"MC_BACKEND_CUDA_{exc.code.replace('MPC_E_', '')}: {exc}") from exc
    return {
        "price": res.price,
        "stderr": res.stderr,
        "values": _values(res, req),
        "manifest": _manifest(workload, function, cfg, req),
        "warnings": _warnings(req, res, cfg),
    }


def price_european_call(config: Mapping[str, Any]) -> dict:
    """european_call_price_mc_cpu (cpu.rs:3009): terminal unless ``method`` says stepwise."""

    return _price("european_call", "price_european_call", config)


def price_arithmetic_asian_call(config: Mapping[str, Any]) -> dict:
    return _price("arithmetic_asian_call", "price_arithmetic_asian_call", config)


def price_down_and_out_call(config: Mapping[str, Any]) -> dict:
    return _price("down_and_out_call", "price_down_and_out_call", config)


def price_up_and_out_call(config: Mapping[str, Any]) -> dict:
    return _price("up_and_out_call", "price_up_and_out_call", config)


def price_lookback_call(config: Mapping[str, Any]) -> dict:
    return _price("lookback_call", "price_lookback_call", config)


def price_basket_call(config: Mapping[str, Any]) -> dict:
    return _price("basket_call", "price_basket_call", config)


def price_american_put(config: Mapping[str, Any]) -> dict:
    return _price("american_put", "price_american_put", config)


def price_bermudan_put(config: Mapping[str, Any]) -> dict:
    return _price("bermudan_put", "price_bermudan_put", config)


def price_heston_european_call(config: Mapping[str, Any]) -> dict:
    return _price("european_call", "price_heston_european_call", config, {"model": "heston", "method": "stepwise"})


def price_merton_jump_diffusion_call(config: Mapping[str, Any]) -> dict:
    """The reference Merton estimator (cpu.rs:3151-3189): terminal sampling from
    the pseudorandom MonteCarloRng stream of each chunk, which the device
    replays exactly (per-path payoffs equal the reference's)."""

    return _price("european_call", "price_merton_jump_diffusion_call", config, {"model": "merton"})


def arithmetic_asian_mlmc(config: Mapping[str, Any]) -> dict:
    out = _price("arithmetic_asian_mlmc", "arithmetic_asian_mlmc", config)
    # workload_response shape (lib.rs:709-727): values + manifest + stderr
    return out


def _standard_normal_cdf(x: float) -> float:
    """standard_normal_cdf (cpu.rs:898-910): Abramowitz-Stegun 7.1.26 erf."""

    sign = -1.0 if x < 0.0 else 1.0
    z = abs(x) / math.sqrt(2.0)
    t = 1.0 / (1.0 + 0.3275911 * z)
    a1, a2, a3, a4, a5 = 0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429
    poly = (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t
    return 0.5 * (1.0 + sign * (1.0 - poly * math.exp(-z * z)))


def black_scholes_european_call_price(s0: float, k: float, r: float, sigma: float, t: float) -> float:
    """black_scholes_european_call_price (cpu.rs:839-860), the sweep's analytic column."""

    if k == 0.0:
        return s0
    if t == 0.0:
        return max(s0 - k, 0.0)
    if sigma == 0.0:
        return max(s0 - k * math.exp(-r * t), 0.0)
    sqrt_t = math.sqrt(t)
    d1 = (math.log(s0 / k) + (r + 0.5 * sigma * sigma) * t) / (sigma * sqrt_t)
    d2 = d1 - sigma * sqrt_t
    return s0 * _standard_normal_cdf(d1) - k * math.exp(-r * t) * _standard_normal_cdf(d2)


# EuropeanCallSweepScenario fields (cpu.rs:5044-5082) and their mapping-ABI aliases
_SWEEP_FIELDS = {
    "s0": ("s0", "spot"), "k": ("k", "strike"), "r": ("r", "rate"), "sigma": ("sigma", "volatility"),
    "t": ("t", "maturity"), "n_paths": ("n_paths", "paths"), "n_steps": ("n_steps", "steps"),
    "sampling": ("sampling",), "technique": ("technique",),
}


def price_european_call_parameter_sweep(config: Mapping[str, Any]) -> dict:
    """price_european_call_parameter_sweep_cpu (cpu.rs:3028-3096) as one batched
    launch: each scenario overrides the base config, takes seed
    base + seed_stride * index unless it names its own (cpu.rs:5071-5074), and
    its row carries the Black-Scholes price and the error in standard errors;
    scenarios more than 4 standard errors away raise a warning, as the
    reference's do."""

    cfg = dict(config or {})
    base = dict(cfg.get("base_config") or {})
    for key in ("n_paths", "n_steps", "seed"):
        if cfg.get(key) is not None:
            base[key] = cfg[key]
    stride = int(cfg.get("seed_stride", 10_000))
    method = cfg.get("method", "terminal_distribution")
    scenarios = cfg.get("scenarios") or [
        {"scenario_id": "atm_base"}, {"scenario_id": "down_10pct", "s0": 90.0}, {"scenario_id": "high_vol", "sigma": 0.35},
    ]  # EuropeanCallParameterSweepConfig::default (cpu.rs:1378-1402)
    reqs, rows_cfg = [], []
    for index, sc in enumerate(scenarios):
        sc = dict(sc)
        scenario_cfg = dict(base)
        for field, keys in _SWEEP_FIELDS.items():
            for key in keys:
                if sc.get(key) is not None:
                    for alias in keys:
                        scenario_cfg.pop(alias, None)
                    scenario_cfg[field] = sc[key]
                    break
        seed = sc.get("seed")
        scenario_cfg["seed"] = int(seed) if seed is not None else (int(base.get("seed", 42)) + stride * index) % (1 << 64)
        scenario_cfg["method"] = sc.get("method") or method
        reqs.append(make_request("european_call", scenario_cfg))
        rows_cfg.append((sc.get("scenario_id", f"scenario_{index}"), scenario_cfg))
    try:
        results = backend().price_batch(reqs)
    except BackendError as exc:
        raise ValueError(f"MC_BACKEND_CUDA_{exc.code.replace('MPC_E_', '')}: {exc}") from exc
    rows, warnings = [], []
    for index, ((sid, sc), req, res) in enumerate(zip(rows_cfg, reqs, results)):
        analytic = black_scholes_european_call_price(req.s0, req.k, req.r, req.sigma, req.t)
        signed = res.price - analytic
        err = abs(signed)
        units = err / res.stderr if res.stderr > 0.0 else (0.0 if err == 0.0 else math.inf)
        if units > 4.0:
            warnings.append(f"scenario '{sid}' is {units:.3f} standard errors from Black-Scholes reference")
        rows.append({"scenario_index": index, "scenario_id": sid, "method": sc["method"], "config": sc,
                     "price": res.price, "stderr": res.stderr, "analytic_price": analytic,
                     "signed_error_vs_black_scholes": signed, "abs_error_vs_black_scholes": err,
                     "abs_error_stderr_units": units})
    return {
        "values": {"schema_version": "european-call-sweep.v1", "scenario_count": len(rows), "rows": rows,
                   "total_paths": sum(r.n_paths for r in reqs), "base_seed": int(base.get("seed", 42)),
                   "seed_stride": stride},
        "manifest": _manifest("european_call_parameter_sweep", "price_european_call_parameter_sweep", cfg, reqs[0]),
        "warnings": warnings,
    }


# ---------------------------------------------------------------- Greeks --
_GREEK_WARNINGS = {
    abi.GREEK_WARN_ESTIMATOR_UNSUPPORTED: "this estimator is not offered for this workload; use bump_and_revalue",
    abi.GREEK_WARN_PSEUDORANDOM_SHOCKS: "single-pass estimators draw pseudorandom terminal shocks whatever the sampling",
    abi.GREEK_WARN_TECHNIQUE_IGNORED: "single-pass estimators ignore the configured variance-reduction technique",
}
_GREEK_WORKLOADS = {
    "european_call": ("european_call", {}),
    "arithmetic_asian_call": ("arithmetic_asian_call", {}),
    "down_and_out_call": ("down_and_out_call", {}),
    "up_and_out_call": ("up_and_out_call", {}),
    "lookback_call": ("lookback_call", {}),
    "basket_call": ("basket_call", {}),
    "heston_european_call": ("european_call", {"model": "heston", "method": "stepwise"}),
}


def greek_report_to_dict(rep: abi.GreekReport, workload: str) -> dict:
    """GreekReport in the field names of the reference's serde shape (cpu.rs:158-182)."""

    estimator = {v: k for k, v in abi.GREEK_ESTIMATORS.items()}[rep.estimator]
    single = rep.estimator != abi.GREEKS_BUMP_AND_REVALUE
    estimates = []
    for i in range(rep.n_estimates):
        e = rep.estimates[i]
        estimates.append({
            "greek": abi.GREEK_NAMES[e.greek],
            "estimator": estimator,
            "value": e.value,
            "stderr": e.stderr,
            "bump_size": None if single else e.bump_size,
            "base_price": e.base_price,
            "bumped_up_price": None if single else e.bumped_up_price,
            "bumped_down_price": None if single else e.bumped_down_price,
            "stderr_estimate_kind": "sample standard error of the single-pass estimator" if single
            else "independent-leg propagation (common random numbers usually make the true error smaller)",
        })
    return {
        "workload": workload,
        "estimator": estimator,
        "paths": rep.paths,
        "steps": rep.steps,
        "seed": rep.seed,
        "base_price": rep.base_price,
        "base_stderr": rep.base_stderr,
        "estimated_runtime_ms": rep.runtime_ms,
        "estimates": estimates,
        "warnings": [text for flag, text in _GREEK_WARNINGS.items() if rep.warnings & flag],
    }


def greeks(config: Mapping[str, Any]) -> dict:
    """``<workload>_greeks_cpu(cfg, estimator)`` (cpu.rs:4036-4356) on the GPU.

    ``config`` carries ``workload`` (one of european_call, arithmetic_asian_call,
    down_and_out_call, up_and_out_call, lookback_call, basket_call,
    heston_european_call), ``estimator`` (bump_and_revalue | pathwise |
    likelihood_ratio) and the workload's pricing fields.
    """

    cfg = dict(config or {})
    workload = cfg.pop("workload", "european_call")
    estimator = cfg.pop("estimator", "bump_and_revalue")
    if workload not in _GREEK_WORKLOADS:
        raise ValueError(f"MC_CONFIG_INVALID: no Greeks for workload {workload!r}")
    code, extra = _GREEK_WORKLOADS[workload]
    params = dict(cfg)
    params.update(extra)
    try:
        req = make_request(code, params)
        rep = backend().greeks(req, estimator)
    except ConfigError as exc:
        raise ValueError(f"MC_CONFIG_INVALID: {exc}") from exc
    except KeyError as exc:
        raise ValueError(f"MC_CONFIG_INVALID: unknown estimator {estimator!r}") from exc
    except BackendError as exc:
        raise ValueError(f"MC_BACKEND_CUDA_{exc.code.replace('MPC_E_', '')}: {exc}") from exc
    out = greek_report_to_dict(rep, workload)
    out["manifest"] = _manifest(workload, "greeks", dict(config or {}), req)
    return out


def price_all_current_greeks_bump_and_revalue(config: Mapping[str, Any]) -> list[dict]:
    """price_all_current_greeks_bump_and_revalue_cpu (cpu.rs:4358-4407): the
    bump-and-revalue report of every workload with Greeks, at default
    configs, seeds ``seed`` .. ``seed + 5``."""

    cfg = dict(config or {})
    n_paths, n_steps, seed = int(cfg.get("n_paths", 10_000)), int(cfg.get("n_steps", 64)), int(cfg.get("seed", 42))
    order = ["european_call", "arithmetic_asian_call", "down_and_out_call", "lookback_call", "basket_call",
             "heston_european_call"]
    reports = []
    for i, workload in enumerate(order):
        params = {"workload": workload, "n_paths": n_paths, "seed": (seed + i) % (1 << 64),
                  "estimator": "bump_and_revalue"}
        if workload != "basket_call":
            params["n_steps"] = n_steps
        for key in ("precision", "sampling"):
            if key in cfg:
                params[key] = cfg[key]
        reports.append(greeks(params))
    return reports


# Aliases in the naming of the Metal bridge.
price_european_call_cuda = price_european_call
price_arithmetic_asian_call_cuda = price_arithmetic_asian_call
price_down_and_out_call_cuda = price_down_and_out_call
price_up_and_out_call_cuda = price_up_and_out_call
price_lookback_call_cuda = price_lookback_call
price_basket_call_cuda = price_basket_call
price_american_put_cuda = price_american_put
price_bermudan_put_cuda = price_bermudan_put
price_heston_european_call_cuda = price_heston_european_call
price_merton_jump_diffusion_call_cuda = price_merton_jump_diffusion_call
arithmetic_asian_mlmc_cuda = arithmetic_asian_mlmc
greeks_cuda = greeks
