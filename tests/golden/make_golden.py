"""Regenerates the golden fixtures under tests/golden/ from a reference checkout.

Run where the montepath reference repository is checked out, naming its root
in ``MONTEPATH_REFERENCE``:

    MONTEPATH_REFERENCE=<path to montepath> python tests/golden/make_golden.py

It writes three files, which the tests read; the reference is not needed at
test time:

* ``reference_fixtures.json``: the analytic known-answer values of the
  reference's fixture registry (benchmarks/reference-fixtures.json).
* ``python_reference_runs.json``: outputs of the reference's own pure-Python
  pricer (python/montepath/pricing.py:828-904, ``random.Random(seed).gauss``
  paths) for the plain small configuration.
* ``reference_release_rows.json``: every ``price_estimate`` row the
  reference's Rust CPU runtime published in benchmarks/release-results.json,
  with the configuration its bench harness ran
  (crates/mc-bench/src/harness.rs): 100,000 paths x 64 steps
  (``MC_PATHS``/``MC_STEPS``, harness.rs:42-43), the price averaged over
  seeds s, s+1, s+2 (``MC_REPEATS``, e.g. harness.rs:1741), the config's
  ``Default`` values otherwise (Merton from seed 9,303, harness.rs:4004-4025),
  and ``n_threads`` = 0, which the reference resolves to the publishing
  machine's ``available_parallelism`` (cpu.rs:8912-8920): 8 on the Apple M2
  the rows were measured on.  The MLMC rows first run the tolerance solver at
  seed 42 (harness.rs:2634-2663) and then price the fixed plan at each seed.
"""

from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))

# Row name -> (workload, overrides of the config defaults) as the harness runs
# it.  "seed" overrides the first of the three seeds (42 by default).
RELEASE_ROWS = {
    # harness.rs:1731-1760, 2387-2430 and the control-variate variant
    "mc_cpu_european_call_rust": ("european_call", {"method": "stepwise"}),
    "mc_cpu_european_call_rust_antithetic": ("european_call", {"method": "stepwise", "technique": "antithetic"}),
    "mc_cpu_european_call_rust_control_variate": (
        "european_call", {"method": "stepwise", "technique": "control_variate"}),
    # harness.rs:2218-2260, 2432-2475
    "mc_cpu_european_call_rust_terminal": ("european_call", {"method": "terminal"}),
    "mc_cpu_european_call_rust_terminal_antithetic": (
        "european_call", {"method": "terminal", "technique": "antithetic"}),
    "mc_cpu_european_call_rust_terminal_control_variate": (
        "european_call", {"method": "terminal", "technique": "control_variate"}),
    # harness.rs:2522-2560
    "mc_cpu_arithmetic_asian_call_rust": ("arithmetic_asian_call", {}),
    "mc_cpu_arithmetic_asian_call_rust_control_variate": ("arithmetic_asian_call", {"technique": "control_variate"}),
    # harness.rs:2613-2663 (tolerance-solved plans)
    "mc_cpu_arithmetic_asian_call_rust_mlmc": ("arithmetic_asian_mlmc", {"mlmc_plan": "pseudorandom"}),
    "mc_cpu_arithmetic_asian_call_rust_mlqmc": ("arithmetic_asian_mlmc", {"mlmc_plan": "scrambled_sobol"}),
    # harness.rs:3356-3400 and the Halton / LHS variants
    "mc_cpu_european_call_rust_randomized_halton": (
        "european_call", {"method": "stepwise", "sampling": "randomized_halton"}),
    "mc_cpu_european_call_rust_latin_hypercube": (
        "european_call", {"method": "stepwise", "sampling": "latin_hypercube"}),
    "mc_cpu_european_call_rust_scrambled_sobol": (
        "european_call", {"method": "stepwise", "sampling": "scrambled_sobol"}),
    "mc_cpu_european_call_rust_scrambled_sobol_brownian_bridge": (
        "european_call", {"method": "stepwise", "sampling": "scrambled_sobol_brownian_bridge"}),
    # harness.rs:3520-3560, 3643-3680
    "mc_cpu_down_and_out_call_rust": ("down_and_out_call", {}),
    "mc_cpu_down_and_out_call_rust_control_variate": ("down_and_out_call", {"technique": "control_variate"}),
    "mc_cpu_lookback_call_rust": ("lookback_call", {}),
    "mc_cpu_lookback_call_rust_control_variate": ("lookback_call", {"technique": "control_variate"}),
    # harness.rs:3730-3800
    "mc_cpu_american_put_lsm_rust": ("american_put", {}),
    "mc_cpu_bermudan_put_lsm_rust": ("bermudan_put", {"exercise_steps": [16, 32, 48, 64]}),
    # harness.rs:3923-3960, 4004-4040
    "mc_cpu_heston_european_call_rust": ("european_call", {"model": "heston"}),
    "mc_cpu_merton_jump_diffusion_call_rust": ("european_call", {"model": "merton", "seed": 9303}),
    # harness.rs:4202-4240, 4329-4370, 4456-4500
    "mc_cpu_arithmetic_asian_call_rust_randomized_halton": ("arithmetic_asian_call", {"sampling": "randomized_halton"}),
    "mc_cpu_arithmetic_asian_call_rust_latin_hypercube": ("arithmetic_asian_call", {"sampling": "latin_hypercube"}),
    "mc_cpu_arithmetic_asian_call_rust_scrambled_sobol_brownian_bridge": (
        "arithmetic_asian_call", {"sampling": "scrambled_sobol_brownian_bridge"}),
    "mc_cpu_down_and_out_call_rust_randomized_halton": ("down_and_out_call", {"sampling": "randomized_halton"}),
    "mc_cpu_down_and_out_call_rust_latin_hypercube": ("down_and_out_call", {"sampling": "latin_hypercube"}),
    "mc_cpu_down_and_out_call_rust_scrambled_sobol_brownian_bridge": (
        "down_and_out_call", {"sampling": "scrambled_sobol_brownian_bridge"}),
    "mc_cpu_basket_call_rust": ("basket_call", {}),
    "mc_cpu_basket_call_rust_randomized_halton": ("basket_call", {"sampling": "randomized_halton"}),
    "mc_cpu_basket_call_rust_latin_hypercube": ("basket_call", {"sampling": "latin_hypercube"}),
    "mc_cpu_basket_call_rust_scrambled_sobol": ("basket_call", {"sampling": "scrambled_sobol"}),
}

# The harness's MLMC tolerance configuration (harness.rs:48-53, 2634-2663).
MLMC_PILOT = {
    "base_steps": 8,
    "levels": 4,
    "refinement_factor": 2,
    "paths_per_level": [2048, 2048, 2048, 2048],
    "target_stderr": 0.05,
    "pilot_paths_per_level": 2048,
    "min_step_updates": 100_000,
    "max_step_updates": 2_000_000,
}
MLQMC_REPLICATES = 4  # ASIAN_MLQMC_REPLICATES, harness.rs:54


def reference_root() -> str:
    root = os.environ.get("MONTEPATH_REFERENCE")
    if not root or not os.path.isdir(root):
        raise SystemExit("set MONTEPATH_REFERENCE to the root of a montepath checkout")
    return root


def fixtures(root: str) -> dict:
    with open(os.path.join(root, "benchmarks", "reference-fixtures.json")) as f:
        registry = json.load(f)
    out = {}
    for fx in registry["fixtures"]:
        out[fx["fixture_id"]] = {"parameters": fx["parameters"], "expected": fx["expected"]}
    return out


def release_rows(root: str) -> list[dict]:
    with open(os.path.join(root, "benchmarks", "release-results.json")) as f:
        published = {
            r["benchmark_name"]: r
            for r in json.load(f)["results"]
            if r.get("metric_name") == "price_estimate" and r.get("backend") == "cpu_native"
        }
    rows = []
    for name, (workload, overrides) in RELEASE_ROWS.items():
        row = published[name]
        config = {"n_paths": 100_000, "n_steps": 64, "n_threads": 8}
        config.update(overrides)
        seed = config.pop("seed", 42)
        plan = config.pop("mlmc_plan", None)
        if plan is not None:
            config = dict(MLMC_PILOT, sampling=plan, n_threads=8,
                          scramble_replicates=MLQMC_REPLICATES if plan == "scrambled_sobol" else 1)
        rows.append(
            {
                "name": name,
                "implementation": row["implementation"],
                "methodology": row.get("methodology"),
                "published_price": row["metric_value"],
                "repeats": row["iterations"],
                "workload": workload,
                "config": config,
                "seeds": [seed + i for i in range(row["iterations"])],
                "solve_plan_at_seed": seed if plan is not None else None,
            }
        )
    missing = sorted(set(published) - set(RELEASE_ROWS))
    if missing:
        raise SystemExit(f"release rows without a mapped configuration: {missing}")
    return rows


def python_reference_runs(root: str) -> list[dict]:
    sys.path.insert(0, os.path.join(root, "python"))
    import montepath  # noqa: E402  (the reference package)

    runs = []
    for name, fn, kwargs in (
        ("european_call", montepath.price_european_call, dict(n_paths=20000, n_steps=64, seed=42)),
        ("arithmetic_asian_call", montepath.price_arithmetic_asian_call, dict(n_paths=4000, n_steps=64, seed=7)),
        ("down_and_out_call", montepath.price_down_and_out_call, dict(n_paths=4000, n_steps=64, seed=11, barrier=80.0)),
    ):
        t0 = time.perf_counter()
        res = fn(**kwargs)
        runs.append(
            {
                "workload": name,
                "config": {"spot": 100.0, "strike": 100.0, "rate": 0.03, "volatility": 0.2, "maturity": 1.0, **kwargs},
                "price": res.price,
                "stderr": res.stderr,
                "seconds_1_core": time.perf_counter() - t0,
                "note": "reference pure-Python pricer; its RNG is Python's random.gauss, so it matches other estimators statistically only",
            }
        )
    return runs


def main() -> None:
    root = reference_root()
    with open(os.path.join(HERE, "reference_fixtures.json"), "w") as f:
        json.dump(fixtures(root), f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "reference_release_rows.json"), "w") as f:
        json.dump(release_rows(root), f, indent=1)
        f.write("\n")
    if "--skip-python-runs" not in sys.argv:
        with open(os.path.join(HERE, "python_reference_runs.json"), "w") as f:
            json.dump(python_reference_runs(root), f, indent=1)


if __name__ == "__main__":
    main()
