"""GPU parity of reference entry points beyond the headline kernels.

* The reference's own Merton estimator (terminal, pseudorandom MonteCarloRng
  stream per chunk, cpu.rs:3151-3189, 6408-6441): per-path payoffs to 1e-11
  relative against the oracle (FP64 transcendentals differ from glibc by at
  most an ulp or two), identical jump counts (so identical stream positions),
  and the published reference price of its bench row reproduced.
* The terminal GBM method, the ``Auto`` default of ``price_european_call``
  (cpu.rs:3191-3226, 6360-6406): FP64 per path to 1e-11, FP32 prices within
  the FP32-path tolerance of the other tests.
* Fused FP32 pseudorandom units whose stream start comes from the per-tile
  jump between a thread's units (eight units per thread, chunk edges inside
  tiles): per-path payoffs against the oracle's FP64 on the same streams.
* MLQMC scramble replicates (cpu.rs:3663-3751): FP64 against the oracle.
* The parameter sweep (cpu.rs:3028-3096) through the mapping ABI.
* The headline pair at full size against the oracle itself.
"""

import json
import os

import numpy as np
import pytest

from montepath_b200 import abi
from montepath_b200.requests import make_request
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_release_rows.json")


def req(workload, **kw):
    return make_request(workload, kw)


MERTON = dict(model="merton", jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15)


# ---------------------------------------------- fused pseudorandom jumps --
@pytest.mark.parametrize("workload,kw", [
    ("european_call", dict()),                                   # terminal (the Auto default): one normal per path
    ("european_call", dict(method="stepwise", n_steps=37)),      # an odd number of normals per path
    ("european_call", dict(model="heston", n_steps=16, kappa=2.0, vol_of_vol=0.5, rho=-0.7)),
    ("arithmetic_asian_call", dict(n_steps=24, technique="antithetic")),
])
@pytest.mark.parametrize("threads", [1, 8])
def test_fused_pseudorandom_stream_jumps(backend, workload, kw, threads):
    base = dict(kw, n_paths=150_001, seed=11, n_threads=threads, sampling="pseudorandom", paths_per_thread=8)
    _, ref = O.price_paths(req(workload, **base, precision="fp64_plain"))
    got = backend.price_paths(req(workload, **base, precision="fp32_path"))
    assert np.allclose(got, ref, rtol=1e-3, atol=2e-3), np.max(np.abs(got - ref))


# ---------------------------------------------------------------- Merton --
@pytest.mark.parametrize("n_paths,threads,kw", [
    (1, 1, {}),
    (2, 1, {}),
    (7, 1, {}),
    (50_000, 1, {}),
    (64_003, 8, {}),                                              # the reference's 8-chunk split, uneven chunks
    (20_000, 1, dict(jump_intensity=6.0, jump_mean=0.02)),        # several jumps per path, long Poisson loops
    (20_000, 3, dict(jump_intensity=0.0)),                        # no Poisson uniform drawn at all
    (30_000, 1, dict(t=0.25, jump_intensity=2.0, s0=90.0, k=95.0)),
    (200_003, 32, {}),                                            # many chunks, each with its own chain
    (65_536, 1, dict(seed=0)),                                    # seed 0 maps to MonteCarloRng's fixed state
])
@pytest.mark.parametrize("precision", ["fp64_plain", "fp32_path"])
def test_merton_pseudorandom_per_path(backend, n_paths, threads, kw, precision):
    cfg = dict(MERTON, n_paths=n_paths, seed=9303, n_threads=threads, precision=precision)
    cfg.update(kw)  # may override the seed
    r = req("european_call", **cfg)
    _, ref = O.price_paths(r)
    got = backend.price_paths(r)
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-12), np.max(np.abs(got - ref))
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-11 * abs(b.price) + 1e-15
    assert abs(a.stderr - b.stderr) <= 1e-9 * abs(b.stderr) + 1e-15
    assert a.n_samples == n_paths


def test_merton_reproduces_published_reference_row(backend):
    """mc_cpu_merton_jump_diffusion_call_rust of benchmarks/release-results.json:
    100,000 paths from seeds 9,303-9,305, 8 chunks, averaged."""

    rows = {r["name"]: r for r in json.load(open(GOLDEN))}
    row = rows["mc_cpu_merton_jump_diffusion_call_rust"]
    prices = [backend.price(make_request(row["workload"], row["config"], seed=s)).price for s in row["seeds"]]
    total = 0.0
    for p in prices:
        total += p
    got = total / len(prices)
    assert abs(got - row["published_price"]) <= 1e-12 * row["published_price"], (got, row["published_price"])


def test_merton_pseudorandom_in_a_batch(backend):
    rs = [req("european_call", **dict(MERTON, n_paths=10_000 + 7 * i, seed=100 + i, n_threads=1 + i % 3))
          for i in range(4)]
    rs.append(req("european_call", n_paths=5000, n_steps=16, method="stepwise", seed=3))
    batch = backend.price_batch(rs)
    for r, b in zip(rs, batch):
        alone = backend.price(r)
        assert abs(alone.price - b.price) <= 1e-12 * abs(alone.price)


# ---------------------------------------------------------- terminal GBM --
@pytest.mark.parametrize("technique", ["standard", "antithetic", "control_variate"])
@pytest.mark.parametrize("threads", [1, 8])
def test_terminal_gbm_per_path_fp64(backend, technique, threads):
    r = req("european_call", method="terminal", n_paths=40_001, seed=42, n_threads=threads, technique=technique,
            precision="fp64_plain")
    _, ref = O.price_paths(r)
    got = backend.price_paths(r)
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-12)
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-11 * abs(b.price)


@pytest.mark.parametrize("sampling", ["pseudorandom", "scrambled_sobol", "counter_hash"])
def test_terminal_gbm_auto_method_fp32(backend, sampling):
    """``method`` left at Auto prices by terminal sampling, as
    european_call_price_mc_cpu does; the FP32 path is within 0.05 standard
    errors of the FP64 oracle on the same samples."""

    r = req("european_call", n_paths=200_000, seed=5, sampling=sampling)
    assert r.method == abi.METHOD_AUTO
    a, b = backend.price(r), O.price(r)
    assert a.path_steps == 200_000
    assert abs(a.price - b.price) < 0.05 * b.stderr, (a.price, b.price, b.stderr)
    assert abs(a.price - 9.413403383853016) < 4 * b.stderr


# ----------------------------------------------------------------- MLQMC --
@pytest.mark.parametrize("precision", ["fp64_plain", "fp32_path"])
def test_mlqmc_replicates_match_oracle(backend, precision):
    r = req("arithmetic_asian_mlmc", base_steps=8, levels=4, refinement_factor=2,
            paths_per_level=[8192, 2048, 1024, 512], sampling="scrambled_sobol", scramble_replicates=4, seed=42,
            precision=precision)
    a, b = backend.price(r), O.price(r)
    assert a.n_levels == b.n_levels == 4
    if precision == "fp64_plain":
        assert abs(a.price - b.price) <= 1e-10 * abs(b.price)
        for lvl in range(4):
            assert abs(a.level_mean[lvl] - b.level_mean[lvl]) <= 1e-10 * max(1.0, abs(b.level_mean[lvl]))
            assert a.level_paths[lvl] == b.level_paths[lvl]
    else:
        assert abs(a.price - b.price) < 0.25 * b.stderr, (a.price, b.price, b.stderr)


# ------------------------------------------------------- parameter sweep --
def test_parameter_sweep_matches_oracle(backend):
    from montepath_b200 import native

    scenarios = [
        {"scenario_id": "atm_base"},
        {"scenario_id": "down_10pct", "s0": 90.0},
        {"scenario_id": "high_vol", "sigma": 0.35},
        {"scenario_id": "short", "t": 0.25, "n_paths": 30_000, "method": "stepwise", "n_steps": 16},
    ]
    cfg = {"base_config": {"n_paths": 50_000, "seed": 42, "precision": "fp64_plain"}, "scenarios": scenarios}
    out = native.price_european_call_parameter_sweep(cfg)
    rows = out["values"]["rows"]
    assert [r["scenario_id"] for r in rows] == [s["scenario_id"] for s in scenarios]
    for i, row in enumerate(rows):
        want = O.price(make_request("european_call", row["config"]))
        assert row["config"]["seed"] == 42 + 10_000 * i  # apply_european_call_sweep_scenario (cpu.rs:5071-5074)
        assert abs(row["price"] - want.price) <= 1e-11 * want.price
        analytic = O.bs_call(row["config"].get("s0", 100.0), 100.0, 0.03, row["config"].get("sigma", 0.2),
                             row["config"].get("t", 1.0))
        assert abs(row["analytic_price"] - analytic) <= 1e-12 * analytic
        assert abs(row["abs_error_stderr_units"] - abs(row["price"] - analytic) / row["stderr"]) < 1e-9
    assert out["values"]["total_paths"] == 50_000 * 3 + 30_000


# ------------------------------------------------- headline vs the oracle --
def test_headline_full_size_against_oracle(backend):
    """1,048,576 paths x 256 steps, scrambled Sobol: the FP64 plain device
    path equals the oracle to 1e-10 and the fused FP32 path sits within 0.05
    standard errors of it, for Heston (seed 42) and Merton (seed 43)."""

    threads = max(1, min(32, os.cpu_count() or 1))
    heston = dict(model="heston", kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7, v0=0.04, seed=42)
    merton = dict(model="merton", method="stepwise", jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15,
                  seed=43)
    for kw in (heston, merton):
        r32 = req("european_call", n_paths=1 << 20, n_steps=256, sampling="scrambled_sobol", **kw)
        r64 = req("european_call", n_paths=1 << 20, n_steps=256, sampling="scrambled_sobol",
                  precision="fp64_plain", **kw)
        ref = O.price_threaded(r64, threads)
        a, b = backend.price(r32), backend.price(r64)
        assert abs(b.price - ref.price) <= 1e-10 * ref.price, (kw["model"], b.price, ref.price)
        assert abs(a.price - ref.price) < 0.05 * ref.stderr, (kw["model"], a.price, ref.price, ref.stderr)
