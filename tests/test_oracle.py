"""CPU oracle pinned against the reference's fixtures, its own statistical
bands (crates/mc-core/tests/cpu_runtime.rs) and independent restatements."""

import json
import math
import os

import numpy as np
import pytest

from montepath_b200 import abi
from montepath_b200.requests import make_request
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def fixture(name):
    with open(os.path.join(GOLDEN, "reference_fixtures.json")) as f:
        return json.load(f)[name]


# ---------------------------------------------------------------- analytic --
def test_black_scholes_fixture():
    # The registry values use an exact normal CDF; the reference's runtime
    # black_scholes_european_call_price (cpu.rs:839-860) uses the A&S 7.1.26
    # erf, about 1e-5 away.  Both restatements are pinned.
    fx = fixture("black_scholes_european_call_atm_1y")
    assert abs(O.bs_call(100, 100, 0.03, 0.2, 1.0, exact=True) - fx["expected"]["price"]) < 1e-12
    assert abs(O.bs_call(100, 100, 0.03, 0.2, 1.0) - fx["expected"]["price"]) < 2e-5


def test_black_scholes_greeks_fixture():
    exp = fixture("black_scholes_european_call_greeks_atm_1y")["expected"]
    g = O.bs_greeks(100, 100, 0.03, 0.2, 1.0, exact=True)
    assert abs(g["price"] - exp["price"]) < 1e-12
    assert abs(g["delta"] - exp["delta"]) < 1e-12
    assert abs(g["vega"] - exp["vega"]) < 1e-10
    assert abs(g["rho"] - exp["rho"]) < 1e-10
    assert abs(g["theta"] - exp["theta_calendar_convention"]) < 1e-10


def test_put_parity_fixture():
    exp = fixture("black_scholes_european_put_atm_1y_lower_bound")["expected"]
    assert abs(O.bs_put(100, 100, 0.03, 0.2, 1.0, exact=True) - exp["european_put_lower_bound"]) < 1e-12


def test_crr_american_fixture():
    exp = fixture("crr_american_put_atm_1y_reference")["expected"]
    assert abs(O.crr_put(100, 100, 0.03, 0.2, 1.0, 512) - exp["crr_binomial_price"]) < 1e-11


def test_crr_bermudan_fixture():
    fx = fixture("crr_bermudan_put_atm_1y_quarterly_reference")
    steps = fx["parameters"]["mapped_reference_exercise_steps"]
    assert abs(O.crr_put(100, 100, 0.03, 0.2, 1.0, 512, steps) - fx["expected"]["crr_binomial_price"]) < 1e-11


def test_merton_series_fixture():
    fx = fixture("merton_jump_diffusion_call_series_reference")
    p = fx["parameters"]
    args = (p["spot"], p["strike"], p["rate"], p["diffusion_volatility"], p["jump_intensity"], p["jump_mean"],
            p["jump_volatility"], p["maturity_years"], p["max_series_terms"], p["tail_tolerance"])
    expected = list(fx["expected"].values())[0]
    assert abs(O.merton_series(*args, exact=True) - expected) < 1e-10
    assert abs(O.merton_series(*args) - expected) < 2e-5


def test_heston_semi_analytic_black_scholes_limit():
    fx = fixture("heston_black_scholes_limit_atm_1y")
    got = O.heston_call(100, 100, 0.03, 0.04, 1.5, 0.04, 0.0, -0.6, 1.0)
    assert abs(got - O.bs_call(100, 100, 0.03, 0.2, 1.0, exact=True)) < 1e-12
    # the fixture comes from the reference's A&S-erf Black-Scholes (~1e-7 accurate)
    assert abs(got - fx["expected"]["black_scholes_limit_price"]) < 1e-6
    # integral form at tiny vol-of-vol converges to the same limit
    small = O.heston_call(100, 100, 0.03, 0.04, 1.5, 0.04, 1e-4, -0.6, 1.0)
    assert abs(small - got) < 1e-4


# ------------------------------------------------------------- integers ----
M64 = (1 << 64) - 1


def py_xorshift(seed, n):
    x = seed or 0x9E3779B97F4A7C15
    out = []
    for _ in range(n):
        x ^= x >> 12
        x ^= (x << 25) & M64
        x ^= x >> 27
        out.append((x * 0x2545F4914F6CDD1D) & M64)
    return out


def py_splitmix(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def py_hash(x):
    M = 0xFFFFFFFF
    x = (x + 0x9E3779B9) & M
    x ^= x >> 16
    x = (x * 0x85EBCA6B) & M
    x ^= x >> 13
    x = (x * 0xC2B2AE35) & M
    return x ^ (x >> 16)


@pytest.mark.parametrize("seed", [0, 1, 42, 0xDEADBEEFCAFEF00D])
def test_xorshift_matches_independent_restatement(seed):
    assert list(O.xorshift_u64(seed, 257)) == py_xorshift(seed, 257)


def test_splitmix64_known_answer_and_restatement():
    # splitmix64 from state 0 (Steele-Lea-Flood 2014 / Vigna): first output
    assert O.lib().or_splitmix64(0) == 0xE220A8397B1DCDAF
    for x in (1, 42, 2**63 + 5):
        assert O.lib().or_splitmix64(x) == py_splitmix(x)
    assert O.lib().or_derive_chunk_seed(42, 3) == py_splitmix((42 + 3 * 0x9E3779B97F4A7C15) & M64)


def test_counter_hash_matches_independent_restatement():
    L = O.lib()
    for seed, path, step, lane in [(42, 0, 0, 0), (42, 7, 63, 1), (0xFFFFFFFF, 123456, 9, 0), (7, 2**31, 2**20, 1)]:
        mixed = (seed ^ ((path * 747796405) & 0xFFFFFFFF) ^ ((step * 2891336453) & 0xFFFFFFFF) ^ ((lane * 277803737) & 0xFFFFFFFF))
        assert L.or_counter_hash(seed, path, step, lane) == py_hash(mixed)
        h = py_hash(mixed)
        assert L.or_counter_uniform_f32(seed, path, step, lane) == np.float32((h + 1.0) / 4294967297.0)


def test_halton_digits():
    # radical inverse in base 3 of 7 = 21_3 -> 0.12_3 = 1/3 + 2/9
    assert abs(O.lib().or_halton(7, 3) - (1 / 3 + 2 / 9)) < 1e-15
    assert O.lib().or_halton(1, 2) == 0.5


def test_inverse_normal_accuracy():
    from scipy.stats import norm

    for p in (1e-10, 0.001, 0.02, 0.3, 0.5, 0.8, 0.975, 0.9999):
        assert abs(O.lib().or_inverse_normal(p) - norm.ppf(p)) < 2e-8 * max(1.0, abs(norm.ppf(p)))


def test_unscrambled_sobol_matches_scipy():
    from scipy.stats import qmc

    d = 64
    pts = qmc.Sobol(d, scramble=False, bits=32).random_base2(8) * 2.0**32
    L = O.lib()
    for p in range(256):
        g = p ^ (p >> 1)
        for dim in range(d):
            assert L.or_sobol_unscrambled(g, dim) == int(pts[p, dim])


def test_scrambled_sobol_is_a_net_per_block():
    # Owen scrambling keeps the (0, m, 1)-net property of every dimension:
    # the first 2^m points of a block fill each of 2^m strata exactly once.
    L = O.lib()
    for dim in (0, 5, 300):
        strata = sorted((L.or_sobol_point(i, dim, 42) >> 22) for i in range(1024))
        assert strata == list(range(1024))


# ------------------------------------------------------ Monte Carlo bands ---
def price(workload, **kw):
    return O.price(make_request(workload, kw))


def test_european_stepwise_close_to_black_scholes():
    # cpu_runtime.rs:753-780 band: within 5 SE
    res = price("european_call", method="stepwise", n_paths=40000, n_steps=32, seed=11, n_threads=1)
    assert abs(res.price - O.bs_call(100, 100, 0.03, 0.2, 1.0)) < 5 * res.stderr


def test_gbm_european_small_statistically_matches_reference_python_pricer():
    with open(os.path.join(GOLDEN, "python_reference_runs.json")) as f:
        runs = {r["workload"]: r for r in json.load(f)}
    ref = runs["european_call"]
    res = price("european_call", method="stepwise", n_paths=20000, n_steps=64, seed=42, n_threads=1)
    combined = math.hypot(res.stderr, ref["stderr"])
    assert abs(res.price - ref["price"]) < 3 * combined
    assert abs(res.price - 9.413403383853016) < 3 * res.stderr


@pytest.mark.parametrize("workload", ["arithmetic_asian_call", "down_and_out_call"])
def test_path_payoffs_statistically_match_reference_python_pricer(workload):
    with open(os.path.join(GOLDEN, "python_reference_runs.json")) as f:
        ref = {r["workload"]: r for r in json.load(f)}[workload]
    res = price(workload, n_paths=20000, n_steps=64, seed=5, n_threads=1, barrier=80.0)
    assert abs(res.price - ref["price"]) < 3.5 * math.hypot(res.stderr, ref["stderr"])


def test_determinism_and_chunking():
    a = price("european_call", method="stepwise", n_paths=20000, n_steps=16, seed=7, n_threads=4)
    b = price("european_call", method="stepwise", n_paths=20000, n_steps=16, seed=7, n_threads=4)
    assert a.price == b.price and a.stderr == b.stderr
    # four chunks of 5000 paths seeded by derive_chunk_seed, merged in order
    total = np.zeros(3)
    for idx in range(4):
        seed = O.lib().or_derive_chunk_seed(7, idx)
        part = price("european_call", method="stepwise", n_paths=5000, n_steps=16, seed=seed, n_threads=1)
        total += np.array(part.moments[:3])
    assert a.moments[1] == total[1] and a.moments[2] == total[2]


def test_merton_matches_series():
    # cpu_runtime.rs:76-90: within 4 SE + 0.10
    res = price("european_call", model="merton", n_paths=120000, seed=10202, n_threads=1)
    ref = O.merton_series(100, 100, 0.03, 0.2, 0.4, -0.08, 0.25, 1.0)
    assert abs(res.price - ref) <= 4 * res.stderr + 0.10


def test_merton_stepwise_sobol_matches_series():
    res = price("european_call", model="merton", method="stepwise", sampling="scrambled_sobol", n_paths=16384,
                n_steps=64, seed=3, jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15)
    ref = O.merton_series(100, 100, 0.03, 0.2, 0.5, -0.1, 0.15, 1.0)
    assert abs(res.price - ref) <= 4 * res.stderr + 0.05


def test_heston_black_scholes_limit():
    # cpu_runtime.rs:1510-1533: within 4 SE + 0.05
    res = price("european_call", model="heston", n_paths=40000, n_steps=64, seed=9, vol_of_vol=0.0, v0=0.04,
                theta=0.04, n_threads=1)
    assert abs(res.price - 9.413403383853016) <= 4 * res.stderr + 0.05


def test_heston_sobol_against_semi_analytic():
    res = price("european_call", model="heston", sampling="scrambled_sobol", n_paths=32768, n_steps=128, seed=1,
                kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7, v0=0.04)
    ref = O.heston_call(100, 100, 0.03, 0.04, 2.0, 0.04, 0.5, -0.7, 1.0)
    # the floored-Euler scheme carries an O(dt) bias of a few cents here
    assert abs(res.price - ref) <= 4 * res.stderr + 0.08


def test_lsm_matches_crr_and_premium():
    # cpu_runtime.rs:1334-1378
    res = price("american_put", n_paths=20000, n_steps=50, seed=5, basis_degree=3, r=0.06)
    crr = O.crr_put(100, 100, 0.06, 0.2, 1.0, 2048)
    assert abs(res.price - crr) <= 5 * res.stderr + 0.15
    assert res.price > O.bs_put(100, 100, 0.06, 0.2, 1.0, exact=True) - 3 * res.stderr
    assert res.regression_steps > 0 and res.early_exercise_count > 0


def test_antithetic_and_control_variate_reduce_stderr():
    base = price("european_call", method="stepwise", n_paths=20000, n_steps=16, seed=3, n_threads=1)
    anti = price("european_call", method="stepwise", n_paths=20000, n_steps=16, seed=3, technique="antithetic")
    cv = price("european_call", method="stepwise", n_paths=20000, n_steps=16, seed=3, technique="control_variate",
               n_threads=1)
    assert anti.stderr < base.stderr and cv.stderr < base.stderr


@pytest.mark.parametrize("sampling", ["randomized_halton", "latin_hypercube", "scrambled_sobol",
                                      "scrambled_sobol_brownian_bridge"])
def test_structured_samplers_deterministic_and_sane(sampling):
    n = O.generate_normals(abi.SAMPLINGS[sampling if "bridge" not in sampling else "scrambled_sobol"], 99, 512, 8)
    assert np.all(np.isfinite(n)) and abs(n.mean()) < 0.2
    a = price("european_call", method="stepwise", sampling=sampling, n_paths=4096, n_steps=32, seed=4)
    b = price("european_call", method="stepwise", sampling=sampling, n_paths=4096, n_steps=32, seed=4)
    assert a.price == b.price
    assert abs(a.price - 9.413403383853016) < 6 * max(a.stderr, 0.05)


def test_basket_two_asset_reference_semantics():
    res = price("basket_call", n_paths=50000, seed=8)
    cv = price("basket_call", n_paths=50000, seed=8, technique="control_variate")
    assert cv.stderr < res.stderr
    assert abs(res.price - cv.price) < 4 * res.stderr


def test_mlmc_matches_plain_asian():
    mlmc = O.price(make_request("arithmetic_asian_mlmc", {"paths_per_level": [40000, 20000, 10000, 5000], "seed": 3}))
    ref = price("arithmetic_asian_call", n_paths=40000, n_steps=128, seed=4)
    assert abs(mlmc.price - ref.price) < 4 * math.hypot(mlmc.stderr, ref.stderr) + 0.02
    assert mlmc.n_levels == 4 and mlmc.level_fine_steps[3] == 128


def test_mlmc_tolerance_solver_plan():
    req = make_request("arithmetic_asian_mlmc", {"target_stderr": 0.05, "seed": 3})
    res = O.price(req)
    assert res.target_met in (0, 1)
    assert res.total_step_updates <= req.max_step_updates * 1.01 + 64
    assert res.stderr < 0.1


def test_same_normals_fp32_functions():
    req = make_request("european_call", n_paths=512, n_steps=16, seed=42)
    z = O.stateless_normals_f32(42, 512, 16)
    res, per = O.price_from_f32_normals(req, z)
    assert np.all(per >= 0) and res.price > 0


# ----------------------------------------------------------------- Greeks --
# european_call_greeks_cpu and siblings (cpu.rs:4036-5010), pinned against the
# Black-Scholes Greeks fixture (reference-fixtures.json:31-58).
@pytest.mark.parametrize("estimator", [abi.GREEKS_BUMP_AND_REVALUE, abi.GREEKS_PATHWISE, abi.GREEKS_LIKELIHOOD_RATIO])
def test_european_greeks_against_black_scholes_fixture(estimator):
    exp = fixture("black_scholes_european_call_greeks_atm_1y")["expected"]
    bs = dict(exp, theta=exp["theta_calendar_convention"])
    req = make_request("european_call", n_paths=200_000, seed=17, precision="fp64_plain")
    status, rep = O.greeks(req, estimator)
    assert status == 0 and rep.warnings == 0
    names = {rep.estimates[i].greek: rep.estimates[i] for i in range(rep.n_estimates)}
    expect = [abi.GREEK_DELTA, abi.GREEK_VEGA, abi.GREEK_RHO] + ([] if estimator == 2 else [abi.GREEK_THETA])
    assert sorted(names) == sorted(expect)
    for greek, key in ((abi.GREEK_DELTA, "delta"), (abi.GREEK_VEGA, "vega"), (abi.GREEK_RHO, "rho"),
                       (abi.GREEK_THETA, "theta")):
        if greek in names:
            e = names[greek]
            assert abs(e.value - bs[key]) < 4 * e.stderr + 1e-3 * abs(bs[key]), (key, e.value, bs[key], e.stderr)
    assert abs(rep.base_price - 9.413403383853016) < 4 * rep.base_stderr


def test_bump_recipe_matches_repricing():
    """push_bump_estimate (cpu.rs:4938-4983): central difference of two
    common-seed repricings, theta sign reversed, floors applied."""

    req = make_request("arithmetic_asian_call", n_paths=20_000, n_steps=24, seed=9, precision="fp64_plain")
    status, rep = O.greeks(req, abi.GREEKS_BUMP_AND_REVALUE)
    assert status == 0 and rep.n_estimates == 4
    up, down = abi.Request.from_buffer_copy(req), abi.Request.from_buffer_copy(req)
    up.sigma, down.sigma = 0.2 + 0.01, 0.2 - 0.01
    vega = rep.estimates[1]
    assert vega.greek == abi.GREEK_VEGA and abs(vega.bump_size - 0.01) < 1e-15
    assert vega.value == (O.price(up).price - O.price(down).price) / (2 * (((0.2 + 0.01) - (0.2 - 0.01)) * 0.5))
    theta = rep.estimates[3]
    h = 1.0 / 365.0
    tu, td = abi.Request.from_buffer_copy(req), abi.Request.from_buffer_copy(req)
    tu.t, td.t = 1.0 + h, 1.0 - h
    assert theta.value == -(O.price(tu).price - O.price(td).price) / (2 * (((1.0 + h) - (1.0 - h)) * 0.5))


def test_greek_reports_of_other_workloads():
    basket = make_request("basket_call", n_paths=20_000, seed=3, precision="fp64_plain")
    status, rep = O.greeks(basket, abi.GREEKS_BUMP_AND_REVALUE)
    assert status == 0 and rep.steps == 2
    assert [rep.estimates[i].greek for i in range(rep.n_estimates)] == [0, 1, 2, 3, 4, 5]
    heston = make_request("european_call", model="heston", n_paths=5_000, n_steps=16, seed=3, precision="fp64_plain")
    status, rep = O.greeks(heston, abi.GREEKS_PATHWISE)
    assert status == 0 and rep.n_estimates == 0 and rep.warnings & abi.GREEK_WARN_ESTIMATOR_UNSUPPORTED
    merton = make_request("european_call", model="merton", n_paths=1_000, seed=3, precision="fp64_plain")
    assert O.greeks(merton, abi.GREEKS_BUMP_AND_REVALUE)[0] == abi.E_UNSUPPORTED
