"""Bump-and-revalue Greeks timing: each case's report (all legs in one
scenario launch that draws every normal once) against the same legs priced
as one ``mpc_price_batch``.  Device times from CUDA events, L2 flushed before
each timed call, best of five.  ``python greeks_bench.py`` prints one JSON
object."""

from __future__ import annotations

import argparse
import json
import math
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from montepath_b200 import abi  # noqa: E402
from montepath_b200.backend import CudaBackend  # noqa: E402
from montepath_b200.requests import make_request  # noqa: E402

BASKET5 = {"spots": [100.0, 95.0, 105.0, 90.0, 110.0], "sigmas": [0.2, 0.25, 0.3, 0.35, 0.4], "corr": 0.3}
CASES = {
    "basket5_64_steps_sobol": ("basket_call", {"method": "stepwise", "n_steps": 64, "sampling": "scrambled_sobol",
                                               **BASKET5}),
    "basket5_64_steps_counter_hash": ("basket_call", {"method": "stepwise", "n_steps": 64,
                                                      "sampling": "counter_hash", **BASKET5}),
    "basket2_terminal_pseudorandom": ("basket_call", {}),
    "asian_64_steps_antithetic_sobol": ("arithmetic_asian_call", {"n_steps": 64, "sampling": "scrambled_sobol",
                                                                  "technique": "antithetic"}),
    "european_64_steps_control_variate_counter_hash": ("european_call", {
        "method": "stepwise", "n_steps": 64, "sampling": "counter_hash", "technique": "control_variate"}),
    "heston_64_steps_antithetic_sobol": ("european_call", {"model": "heston", "n_steps": 64,
                                                           "sampling": "scrambled_sobol", "technique": "antithetic"}),
}
# the request field each Greek bumps (basket: first and second asset)
_BASKET_FIELDS = {abi.GREEK_DELTA: ("spots", 0), abi.GREEK_DELTA2: ("spots", 1), abi.GREEK_VEGA: ("sigmas", 0),
                  abi.GREEK_VEGA2: ("sigmas", 1), abi.GREEK_RHO: ("r", None), abi.GREEK_THETA: ("t", None)}
_SINGLE_FIELDS = {abi.GREEK_DELTA: ("s0", None), abi.GREEK_VEGA: ("sigma", None), abi.GREEK_RHO: ("r", None),
                  abi.GREEK_THETA: ("t", None)}


def legs_of(req: abi.Request, workload: str, rep: abi.GreekReport) -> list[abi.Request]:
    """The base request and its up / down legs, as the report bumped them."""

    fields = _BASKET_FIELDS if workload == "basket_call" else _SINGLE_FIELDS
    heston = req.model == abi.MODEL_HESTON
    legs = [req]
    for i in range(rep.n_estimates):
        e = rep.estimates[i]
        name, idx = fields[e.greek]
        for sign in (1.0, -1.0):
            leg = abi.Request.from_buffer_copy(req)
            if heston and e.greek == abi.GREEK_VEGA:  # the Heston vega bumps sqrt(v0)
                leg.v0 = (math.sqrt(req.v0) + sign * e.bump_size) ** 2
            elif idx is None:
                setattr(leg, name, getattr(req, name) + sign * e.bump_size)
            else:
                getattr(leg, name)[idx] = getattr(req, name)[idx] + sign * e.bump_size
            legs.append(leg)
    return legs


def run(backend: CudaBackend, paths: int = 1 << 20, cases: list[str] | None = None, repeats: int = 5) -> dict:
    out = {}
    for name in cases or list(CASES):
        workload, kw = CASES[name]
        req = make_request(workload, dict(n_paths=paths, seed=7, **kw))
        for _ in range(3):
            rep = backend.greeks(req, "bump_and_revalue")
        scenario = []
        for _ in range(repeats):
            backend.flush_l2()
            rep = backend.greeks(req, "bump_and_revalue")
            scenario.append(rep.runtime_ms)
        legs = legs_of(req, workload, rep)
        for _ in range(3):
            backend.price_batch(legs)
        batch = []
        for _ in range(repeats):
            backend.flush_l2()
            backend.price_batch(legs)
            batch.append(backend.last_timing()[0])
        out[name] = {"paths": paths, "legs": len(legs), "scenario_ms": min(scenario), "leg_batch_ms": min(batch),
                     "speedup": min(batch) / min(scenario), "base_price": rep.base_price}
    return out


def main(argv: list[str] | None = None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--paths", type=int, default=1 << 20)
    ap.add_argument("--cases", default="", help="comma list of " + ", ".join(CASES) + " (default: all)")
    ap.add_argument("--repeats", type=int, default=5)
    args = ap.parse_args(argv)
    cases = [c for c in args.cases.split(",") if c] or None
    with CudaBackend(0) as backend:
        print(json.dumps(run(backend, args.paths, cases, args.repeats), indent=1))


if __name__ == "__main__":
    main()
