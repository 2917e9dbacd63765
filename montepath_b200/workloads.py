"""Seeded synthetic workloads of the benchmark configurations.

* ``book(seed)`` -- the heterogeneous batched book: 4,096 contracts, an even
  mix of European, arithmetic Asian, up-and-out barrier and 5-asset basket
  calls; K ~ U[50, 150], sigma ~ U[0.1, 0.6], T ~ U[0.1, 2]; paths
  log-uniform over [1e3, 1e6]; steps uniform over {16..365}; basket
  correlation 0.3, equal weights.  Unstated parameters are fixed here:
  S0 = 100, r = 0.03, barrier ~ U[1.1, 1.5] * max(S0, K), counter-hash
  sampling, FP32 path.
* ``serving_stream(seed)`` -- Poisson arrivals at 2,000 requests/s; each
  request uniformly one of {GBM European (64 steps), Heston European (256
  steps, kappa 2, theta 0.04, xi 0.5, rho -0.7, v0 0.04), arithmetic Asian
  MLMC (levels 0-6, M = 2, base 16 steps, target stderr 1e-3, capped at the
  tolerance solver's default 1e7 step updates), American put LSM (100k paths x
  50 dates, K = 100, r = 0.06, sigma 0.2)}; non-MLMC path counts log-uniform
  over [1e3, 1e6].
"""

from __future__ import annotations

import math

import numpy as np

from . import abi
from .requests import make_request

BOOK_KINDS = ("european_call", "arithmetic_asian_call", "up_and_out_call", "basket_call")


def book(seed: int = 42, n: int = 4096, precision: str = "fp32_path") -> list[abi.Request]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = BOOK_KINDS[i % 4]
        k = float(rng.uniform(50.0, 150.0))
        sigma = float(rng.uniform(0.1, 0.6))
        t = float(rng.uniform(0.1, 2.0))
        paths = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e6)))))
        steps = int(rng.integers(16, 366))
        cfg = dict(s0=100.0, k=k, r=0.03, sigma=sigma, t=t, n_paths=paths, n_steps=steps, seed=seed * 100_003 + i,
                   sampling="counter_hash", precision=precision, method="stepwise")
        if kind == "up_and_out_call":
            cfg["barrier"] = float(rng.uniform(1.1, 1.5)) * max(100.0, k)
        if kind == "basket_call":
            cfg.update(spots=[100.0] * 5, sigmas=[sigma] * 5, weights=[0.2] * 5, corr=0.3)
        out.append(make_request(kind, cfg))
    return out


def book_path_steps(reqs: list[abi.Request]) -> int:
    return sum(r.n_paths * r.n_steps for r in reqs)


SERVING_KINDS = ("gbm_european", "heston_european", "asian_mlmc", "american_put_lsm")


def serving_request(kind: str, rng: np.random.Generator, index: int, precision: str = "fp32_path") -> abi.Request:
    paths = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e6)))))
    seed = 7_000_000 + index
    if kind == "gbm_european":
        return make_request("european_call", dict(method="stepwise", n_paths=paths, n_steps=64, seed=seed,
                                                  sampling="counter_hash", precision=precision))
    if kind == "heston_european":
        return make_request("european_call", dict(model="heston", n_paths=paths, n_steps=256, seed=seed,
                                                  kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7, v0=0.04,
                                                  sampling="scrambled_sobol", precision=precision))
    if kind == "asian_mlmc":
        return make_request("arithmetic_asian_mlmc", dict(levels=7, refinement_factor=2, base_steps=16,
                                                          target_stderr=1e-3, seed=seed, sampling="counter_hash",
                                                          precision=precision))
    return make_request("american_put", dict(n_paths=100_000, n_steps=50, r=0.06, sigma=0.2, k=100.0, s0=100.0,
                                             basis_degree=3, seed=seed, precision=precision))


def serving_stream(seed: int = 42, rate: float = 2000.0, duration_s: float = 60.0,
                   precision: str = "fp32_path") -> list[tuple[float, str, abi.Request]]:
    """(arrival time in seconds, kind, request) sorted by arrival."""

    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    index = 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration_s:
            break
        kind = SERVING_KINDS[int(rng.integers(0, 4))]
        out.append((t, kind, serving_request(kind, rng, index, precision)))
        index += 1
    return out
