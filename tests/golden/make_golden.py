"""Regenerates the golden fixtures under tests/golden/ from the reference checkout.

Run in a container where the reference is mounted at /root/reference:

    python tests/golden/make_golden.py

It copies the analytic known-answer values of the reference's fixture
registry (benchmarks/reference-fixtures.json) and records outputs of the
reference's own pure-Python pricer (python/montepath/pricing.py:828-904,
``random.Random(seed).gauss`` paths) for the plain small configuration.
The tests only read the JSON written here; the reference is not needed at
test time.
"""

from __future__ import annotations

import json
import os
import sys
import time

REFERENCE = "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))


def fixtures() -> dict:
    with open(os.path.join(REFERENCE, "benchmarks", "reference-fixtures.json")) as f:
        registry = json.load(f)
    out = {}
    for fx in registry["fixtures"]:
        out[fx["fixture_id"]] = {"parameters": fx["parameters"], "expected": fx["expected"]}
    return out


def python_reference_runs() -> list[dict]:
    sys.path.insert(0, os.path.join(REFERENCE, "python"))
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
    with open(os.path.join(HERE, "reference_fixtures.json"), "w") as f:
        json.dump(fixtures(), f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "python_reference_runs.json"), "w") as f:
        json.dump(python_reference_runs(), f, indent=1)


if __name__ == "__main__":
    main()
