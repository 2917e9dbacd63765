"""``mc_cuda_*`` rows in the format of montepath's benchmark harness.

The reference harness (crates/mc-bench/src/harness.rs) times each CPU
pricer at 100,000 paths x 64 steps over three seeds (seed, seed+1, seed+2)
and writes ``BenchmarkReport {generated_at_unix_ms, results: [BenchmarkResult]}``
(crates/mc-bench/src/result.rs:3-23).  This module runs the GPU counterpart
of each throughput row through the public C ABI and emits rows of the same
shape, named ``mc_cuda_<workload>...`` beside the reference's
``mc_cpu_<workload>_rust...``:

* ``backend`` is ``nvidia_cuda``; ``implementation`` names the ABI call;
* ``total_runtime_ms`` / ``per_iteration_us`` are wall-clock times of the
  public call (host request in, result out), like the harness's
  ``Instant::now()`` around the CPU call;
* ``throughput_per_sec`` is paths per second (requests per second for the
  Greeks row), ``metric_value`` the mean price estimate.

    python -m montepath_b200.mc_bench --out mc_cuda_report.json [--compact] [--precision fp64_plain]
"""

from __future__ import annotations

import argparse
import json
import time
from typing import Any, Callable

from . import abi
from .requests import make_request

MC_PATHS = 100_000  # harness.rs:43-45
MC_STEPS = 64
MC_REPEATS = 3
GREEK_PATHS = 50_000
BENCHMARK_VERSION = "0.1"

# (row name, workload, request overrides, methodology)
_PRICING_ROWS: list[tuple[str, str, dict, str]] = [
    ("mc_cuda_european_call", "european_call", {"method": "stepwise"}, "stepwise_paths"),
    ("mc_cuda_european_call_antithetic", "european_call", {"method": "stepwise", "technique": "antithetic"},
     "stepwise_paths_antithetic"),
    ("mc_cuda_european_call_control_variate", "european_call",
     {"method": "stepwise", "technique": "control_variate"}, "stepwise_paths_control_variate"),
    ("mc_cuda_european_call_terminal", "european_call", {}, "terminal_distribution"),
    ("mc_cuda_european_call_terminal_antithetic", "european_call", {"technique": "antithetic"},
     "terminal_distribution_antithetic"),
    ("mc_cuda_european_call_terminal_control_variate", "european_call", {"technique": "control_variate"},
     "terminal_distribution_control_variate"),
    ("mc_cuda_european_call_randomized_halton", "european_call",
     {"method": "stepwise", "sampling": "randomized_halton"}, "stepwise_paths_randomized_halton"),
    ("mc_cuda_european_call_latin_hypercube", "european_call",
     {"method": "stepwise", "sampling": "latin_hypercube"}, "stepwise_paths_latin_hypercube"),
    ("mc_cuda_european_call_scrambled_sobol", "european_call",
     {"method": "stepwise", "sampling": "scrambled_sobol"}, "stepwise_paths_scrambled_sobol"),
    ("mc_cuda_european_call_scrambled_sobol_brownian_bridge", "european_call",
     {"method": "stepwise", "sampling": "scrambled_sobol_brownian_bridge"},
     "stepwise_paths_scrambled_sobol_brownian_bridge"),
    ("mc_cuda_arithmetic_asian_call", "arithmetic_asian_call", {}, "stepwise_paths"),
    ("mc_cuda_arithmetic_asian_call_control_variate", "arithmetic_asian_call", {"technique": "control_variate"},
     "stepwise_paths_control_variate"),
    ("mc_cuda_down_and_out_call", "down_and_out_call", {}, "stepwise_paths"),
    ("mc_cuda_down_and_out_call_control_variate", "down_and_out_call", {"technique": "control_variate"},
     "stepwise_paths_control_variate"),
    ("mc_cuda_lookback_call", "lookback_call", {}, "stepwise_paths"),
    ("mc_cuda_lookback_call_control_variate", "lookback_call", {"technique": "control_variate"},
     "stepwise_paths_control_variate"),
    ("mc_cuda_basket_call", "basket_call", {"n_steps": 1}, "terminal_two_asset"),
    ("mc_cuda_heston_european_call", "european_call", {"model": "heston", "method": "stepwise"},
     "full_truncation_euler"),
    ("mc_cuda_merton_jump_diffusion_call", "european_call", {"model": "merton", "sampling": "counter_hash"},
     "terminal_jump_diffusion_counter_hash"),
    ("mc_cuda_american_put_lsm", "american_put", {"n_steps": 50}, "longstaff_schwartz_laguerre"),
    ("mc_cuda_bermudan_put_lsm", "bermudan_put", {"n_steps": 64, "exercise_steps": [16, 32, 48, 64]},
     "longstaff_schwartz_laguerre"),
]
_COMPACT = {"mc_cuda_european_call", "mc_cuda_european_call_terminal", "mc_cuda_arithmetic_asian_call",
            "mc_cuda_heston_european_call", "mc_cuda_american_put_lsm"}


def _row(name: str, implementation: str, methodology: str | None, runtimes_ms: list[float], units: float,
         metric_name: str | None, metric_value: float | None) -> dict[str, Any]:
    """One BenchmarkResult (result.rs:3-17), field for field."""

    avg = sum(runtimes_ms) / len(runtimes_ms)
    return {
        "benchmark_name": name,
        "benchmark_version": BENCHMARK_VERSION,
        "implementation": implementation,
        "backend": "nvidia_cuda",
        "methodology": methodology,
        "planner_mode": "n/a",
        "iterations": len(runtimes_ms),
        "total_runtime_ms": avg * len(runtimes_ms),
        "per_iteration_us": avg * 1_000.0,
        "throughput_per_sec": units / (avg / 1_000.0) if avg > 0 else units,
        "metric_name": metric_name,
        "metric_value": metric_value,
    }


def _timed(fn: Callable[[], Any]) -> tuple[Any, float]:
    t0 = time.perf_counter()
    out = fn()
    return out, (time.perf_counter() - t0) * 1e3


def run(backend, compact: bool = False, precision: str = "fp32_path", repeats: int = MC_REPEATS,
        seed: int = 42) -> dict[str, Any]:
    """Runs the rows on ``backend`` (a CudaBackend) and returns the BenchmarkReport."""

    suffix = "" if precision == "fp32_path" else "_" + precision
    results = []
    for name, workload, overrides, methodology in _PRICING_ROWS:
        if compact and name not in _COMPACT:
            continue
        params = dict(n_paths=MC_PATHS, n_steps=MC_STEPS, precision=precision)
        params.update(overrides)
        # warm-up: tables, autotuner and scratch on the first call; the second
        # call of a shape captures its CUDA graph, which later calls replay
        for _ in range(2):
            backend.price(make_request(workload, dict(params, seed=seed)))
        runtimes, prices = [], []
        for i in range(repeats):
            res, ms = _timed(lambda: backend.price(make_request(workload, dict(params, seed=seed + i))))
            runtimes.append(ms)
            prices.append(res.price)
        results.append(_row(name + suffix, "montepath_b200::mpc_price", methodology + "_" + precision, runtimes,
                            float(MC_PATHS), "price_estimate", sum(prices) / len(prices)))
    if not compact:
        # price_european_call_parameter_sweep_cpu as one batch (cpu.rs:3028-3096)
        sweep = [make_request("european_call", dict(n_paths=MC_PATHS, s0=s0, sigma=vol, seed=seed + 10_000 * j,
                                                     precision=precision))
                 for j, (s0, vol) in enumerate((s, v) for s in (90.0, 100.0, 110.0) for v in (0.15, 0.2, 0.3))]
        for _ in range(2):  # the second call captures the batch's graph
            backend.price_batch(sweep)
        runtimes = []
        for _ in range(repeats):
            out, ms = _timed(lambda: backend.price_batch(sweep))
            runtimes.append(ms)
        results.append(_row("mc_cuda_european_call_parameter_sweep" + suffix, "montepath_b200::mpc_price_batch",
                            "terminal_distribution_batch_" + precision, runtimes, float(MC_PATHS * len(sweep)),
                            "scenario_count", float(len(sweep))))
        # every workload's bump-and-revalue Greeks (price_all_current_greeks_bump_and_revalue_cpu)
        greek_reqs = [make_request(w, dict(dict(n_paths=GREEK_PATHS, n_steps=MC_STEPS, seed=seed + k,
                                                precision=precision), **kw))
                      for k, (w, kw) in enumerate([("european_call", {}), ("arithmetic_asian_call", {}),
                                                   ("down_and_out_call", {}), ("lookback_call", {}),
                                                   ("basket_call", {"n_steps": 1}),
                                                   ("european_call", {"model": "heston", "method": "stepwise"})])]
        for _ in range(2):
            for r in greek_reqs:
                backend.greeks(r)
        runtimes = []
        for _ in range(repeats):
            _, ms = _timed(lambda: [backend.greeks(r) for r in greek_reqs])
            runtimes.append(ms)
        results.append(_row("mc_cuda_all_workload_greeks_bump" + suffix, "montepath_b200::mpc_greeks",
                            "bump_and_revalue_common_seeds_" + precision, runtimes, float(len(greek_reqs)),
                            "greek_reports", float(len(greek_reqs))))
    return {"generated_at_unix_ms": int(time.time() * 1000), "results": results}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default="-")
    ap.add_argument("--compact", action="store_true")
    ap.add_argument("--precision", default="fp32_path", choices=sorted(abi.PRECISIONS))
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    from .backend import CudaBackend

    be = CudaBackend(args.device)
    try:
        report = run(be, compact=args.compact, precision=args.precision)
    finally:
        be.close()
    text = json.dumps(report, indent=2)
    if args.out == "-":
        print(text)
    else:
        with open(args.out, "w") as f:
            f.write(text + "\n")


if __name__ == "__main__":
    main()
