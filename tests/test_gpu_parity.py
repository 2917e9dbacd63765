"""GPU parity: the CUDA backend through its C ABI against the CPU oracle.

Tolerances (stated per test):
  * integer streams (xorshift64*, counter hash, Sobol, Halton digits): bit-exact;
  * FP64 samples: 1e-13 relative (CUDA vs glibc transcendentals, <= 1-2 ulp);
  * FP64-plain prices / per-path payoffs: 1e-11 relative;
  * FP32-path per-path payoffs fed the same samples: 2e-4 relative + 1e-4 absolute,
    prices within 3 standard errors of the FP64 oracle (and far closer in practice);
  * the Metal same-normals precedent (backend/metal.rs:1155-1164): price 1e-3, stderr 1e-4.
"""

import math

import numpy as np
import pytest

from montepath_b200 import abi
from montepath_b200.requests import make_request
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def req(workload, **kw):
    return make_request(workload, kw)


# --------------------------------------------------------------- generators --
@pytest.mark.parametrize("seed,offset", [(42, 0), (1, 1), (0, 12345), (0xDEADBEEF, 999_999)])
def test_xorshift_jump_ahead_bit_exact(backend, seed, offset):
    count = 4096
    ref = O.xorshift_u64(seed, offset + count)[offset:]
    got = backend.xorshift(seed, offset, count)
    assert np.array_equal(got, ref)


def test_counter_hash_bit_exact(backend):
    got = backend.counter_hash(42, 64, 33)
    L = O.lib()
    for path in (0, 1, 17, 63):
        for step in (0, 5, 32):
            for lane in (0, 1):
                assert got[path, step, lane] == L.or_counter_hash(42, path, step, lane)


def test_counter_hash_fp32_normals(backend):
    got = backend.generate_normals(abi.SAMPLING_COUNTER_HASH, 42, 256, 32, fp32=True)
    ref = O.stateless_normals_f32(42, 256, 32).reshape(256, 32)
    # same u32 hashes and f32 uniforms; logf/cosf differ by a few ulp
    assert np.max(np.abs(got - ref)) < 4e-6


@pytest.mark.parametrize(
    "sampling",
    [abi.SAMPLING_PSEUDORANDOM, abi.SAMPLING_SCRAMBLED_SOBOL, abi.SAMPLING_RANDOMIZED_HALTON, abi.SAMPLING_LATIN_HYPERCUBE],
)
def test_fp64_samples_match_oracle(backend, sampling):
    n, d = 2048, 37
    got = backend.generate_normals(sampling, 7, n, d)
    ref = O.generate_normals(sampling, 7, n, d)
    err = np.abs(got - ref) / np.maximum(1.0, np.abs(ref))
    worst = np.unravel_index(np.argmax(err), err.shape)
    assert err.max() < 1e-13, (float(err.max()), worst, float(got[worst]), float(ref[worst]))


def test_sobol_fp32_normals_same_uniforms(backend):
    n, d = 70_000, 9  # crosses a 2^16-point block boundary
    got = backend.generate_normals(abi.SAMPLING_SCRAMBLED_SOBOL, 5, n, d, fp32=True)
    ref = O.generate_normals(abi.SAMPLING_SCRAMBLED_SOBOL, 5, n, d)
    # same 23-bit uniforms; FP32 inverse CDF vs the FP64 Acklam rational
    err = np.abs(got - ref) / np.maximum(1.0, np.abs(ref))
    assert err.max() < 2e-6, float(err.max())


# -------------------------------------------------------------- plain FP64 --
def test_gbm_european_small_plain_fp64_replays_reference_stream(backend):
    r = req("european_call", method="stepwise", n_paths=20000, n_steps=64, seed=42, n_threads=1,
            precision="fp64_plain")
    got = backend.price(r)
    ref = O.price(r)
    assert abs(got.price - ref.price) <= 1e-11 * ref.price
    assert abs(got.stderr - ref.stderr) <= 1e-9 * ref.stderr
    assert abs(got.price - 9.413403383853016) < 3 * got.stderr


@pytest.mark.parametrize("threads", [1, 4])
@pytest.mark.parametrize("technique", ["standard", "antithetic", "control_variate"])
def test_gbm_stepwise_paths_fp64(backend, technique, threads):
    r = req("european_call", method="stepwise", n_paths=9001, n_steps=33, seed=9, n_threads=threads,
            technique=technique, precision="fp64_plain")
    if threads > 1:
        r.n_paths = 9001 * 4 // 3
    _, ref = O.price_paths(r)
    got = backend.price_paths(r)
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-11)
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-10 * abs(b.price)


@pytest.mark.parametrize("workload", ["arithmetic_asian_call", "down_and_out_call", "up_and_out_call", "lookback_call"])
def test_path_dependent_fp64(backend, workload):
    r = req(workload, n_paths=5000, n_steps=48, seed=21, n_threads=1, precision="fp64_plain",
            barrier=(85.0 if workload == "down_and_out_call" else 125.0))
    _, ref = O.price_paths(r)
    got = backend.price_paths(r)
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("sampling", ["scrambled_sobol", "randomized_halton", "latin_hypercube", "counter_hash"])
def test_heston_and_merton_fp64_structured(backend, sampling):
    for kw in (
        dict(model="heston", kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7, v0=0.04),
        dict(model="merton", method="stepwise", jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15),
    ):
        r = req("european_call", n_paths=3000, n_steps=24, seed=42, sampling=sampling, precision="fp64_plain", **kw)
        _, ref = O.price_paths(r)
        got = backend.price_paths(r)
        # counter-hash normals are FP32 values computed by two libms (a few ulp apart)
        tol = 2e-5 if sampling == "counter_hash" else 1e-10
        assert np.allclose(got, ref, rtol=tol, atol=tol), (sampling, kw["model"], float(np.max(np.abs(got - ref))))


def test_heston_pseudorandom_chunked_fp64(backend):
    r = req("european_call", model="heston", n_paths=12000, n_steps=16, seed=3, n_threads=3, precision="fp64_plain",
            technique="antithetic")
    _, ref = O.price_paths(r)
    assert np.allclose(backend.price_paths(r), ref, rtol=1e-11, atol=1e-11)


def test_basket_reference_two_asset_fp64(backend):
    r = req("basket_call", n_paths=6000, seed=8, precision="fp64_plain")
    _, ref = O.price_paths(r)
    assert np.allclose(backend.price_paths(r), ref, rtol=1e-11, atol=1e-11)


# ------------------------------------------------------------- fused FP32 ---
def test_metal_same_normals_precedent(backend):
    # backend/metal.rs:1127-1164: 4,096 x 32, price within 1e-3, stderr within 1e-4
    r = req("european_call", method="stepwise", n_paths=4096, n_steps=32, seed=42, sampling="counter_hash")
    z = O.stateless_normals_f32(42, 4096, 32)
    ref, _ = O.price_from_f32_normals(r, z)
    got = backend.price(r)
    assert abs(got.price - ref.price) <= 1e-3
    assert abs(got.stderr - ref.stderr) <= 1e-4


@pytest.mark.parametrize("workload", ["european_call", "arithmetic_asian_call", "down_and_out_call", "lookback_call"])
def test_fused_counter_hash_same_normals(backend, workload):
    r = req(workload, method="stepwise", n_paths=4096, n_steps=64, seed=11, sampling="counter_hash")
    z = O.stateless_normals_f32(11, 4096, 64)
    ref, ref_paths = O.price_from_f32_normals(r, z)
    got_paths = backend.price_paths(r)
    close = np.isclose(got_paths, ref_paths, rtol=2e-4, atol=1e-4)
    # a barrier crossing within FP32 rounding of the level may flip a path
    assert close.mean() > 0.999
    got = backend.price(r)
    assert abs(got.price - ref.price) <= 1e-3


@pytest.mark.parametrize("sampling", ["pseudorandom", "scrambled_sobol", "randomized_halton", "counter_hash"])
def test_fused_gbm_against_fp64_oracle(backend, sampling):
    r = req("european_call", method="stepwise", n_paths=8192, n_steps=64, seed=5, sampling=sampling)
    _, ref_paths = O.price_paths(r)
    got_paths = backend.price_paths(r)
    assert np.allclose(got_paths, ref_paths, rtol=2e-4, atol=1e-3)
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) < 0.05 * b.stderr


def test_heston_euler_bias_shrinks_to_semi_analytic(backend):
    """The headline Heston request (1,048,576 paths, Sobol, FP32 path) against
    the semi-analytic price: full-truncation Euler is biased by its time step
    (the Feller condition fails at these parameters), so the gap falls as the
    steps double, and the step-doubling estimate 2 P(2n) - P(n) lands within 3
    of its standard-error bounds sqrt(5) SE(2n)."""

    semi = O.heston_call(100, 100, 0.03, 0.04, 2.0, 0.04, 0.5, -0.7, 1.0)
    prices = {}
    for n in (256, 1024, 2048):
        r = req("european_call", model="heston", n_paths=1 << 20, n_steps=n, seed=42, sampling="scrambled_sobol",
                kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7, v0=0.04)
        prices[n] = backend.price(r)
    gaps = [prices[n].price - semi for n in (256, 1024, 2048)]
    assert gaps[0] > gaps[1] > gaps[2] > -3 * prices[2048].stderr, gaps
    rich = 2 * prices[2048].price - prices[1024].price
    assert abs(rich - semi) < 3 * math.sqrt(5.0) * prices[2048].stderr, (rich, semi)


def test_merton_fp32_jump_counts_match_oracle(backend):
    """FP32 Sobol Merton steps count jumps with integer thresholds on the
    uniform's 23-bit index.  At lambda dt = 0.625 steps with 1, 2, 3 and 4+
    jumps are common (4+ take the FP64 inversion); a count that differed from
    the oracle's sample_poisson would move a path's log-price by a whole jump
    mean (-0.1), far outside the FP32 tolerance, so every path must match."""

    r = req("european_call", model="merton", method="stepwise", n_paths=4096, n_steps=32, seed=13,
            sampling="scrambled_sobol", jump_intensity=20.0, jump_mean=-0.1, jump_volatility=0.15)
    _, ref_paths = O.price_paths(r)
    got_paths = backend.price_paths(r)
    assert np.allclose(got_paths, ref_paths, rtol=1e-3, atol=2e-3), np.max(np.abs(got_paths - ref_paths))


def test_launch_hint_paths_per_thread(backend):
    """A paths_per_thread hint replaces the autotuner's choice (mpc_prepare
    reports it) and changes only the tile partition, so the price moves at
    rounding level."""

    base = req("european_call", model="heston", n_paths=1 << 18, n_steps=64, seed=8, sampling="scrambled_sobol")
    hinted = req("european_call", model="heston", n_paths=1 << 18, n_steps=64, seed=8, sampling="scrambled_sobol",
                 paths_per_thread=4, block_size=256)
    art = backend.prepare(hinted)
    assert art.paths_per_thread == 4 and art.block_size == 256
    assert art.tiles == (1 << 18) // (256 * 4)
    a, b = backend.price(base), backend.price(hinted)
    assert abs(a.price - b.price) <= 1e-12 * abs(a.price)
    assert abs(a.stderr - b.stderr) <= 1e-9 * a.stderr


EDGE_MODELS = [
    ("european_call", dict(method="stepwise")),
    ("arithmetic_asian_call", {}),
    ("european_call", dict(model="heston", method="stepwise", kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7)),
    ("european_call", dict(model="merton", method="stepwise", jump_intensity=0.5, jump_mean=-0.1,
                           jump_volatility=0.15)),
]


@pytest.mark.parametrize("workload,kw", EDGE_MODELS)
@pytest.mark.parametrize("sampling", ["scrambled_sobol", "counter_hash"])
@pytest.mark.parametrize("n_paths,n_steps", [(1, 1), (3, 3), (257, 5), (300, 7)])
def test_edge_sizes_match_oracle(backend, workload, kw, sampling, n_paths, n_steps):
    """Single paths, tile tails (257, 300 paths) and step counts that end in a
    partial quad or Merton chunk (1, 3, 5, 7 steps): FP64 plain per path to
    1e-10 (2e-5 with counter-hash normals, FP32 values from two libms), fused
    FP32 per path within the FP32 tolerance, against the oracle."""

    base = dict(kw, n_paths=n_paths, n_steps=n_steps, seed=21, sampling=sampling)
    r64 = req(workload, precision="fp64_plain", **base)
    _, ref = O.price_paths(r64)
    got64 = backend.price_paths(r64)
    tol = 2e-5 if sampling == "counter_hash" else 1e-10
    assert np.allclose(got64, ref, rtol=tol, atol=tol)
    r32 = req(workload, **base)
    got32 = backend.price_paths(r32)
    assert np.allclose(got32, ref, rtol=1e-3, atol=2e-3), np.max(np.abs(got32 - ref))
    a = backend.price(r32)
    assert math.isfinite(a.price) and a.n_samples == n_paths


@pytest.mark.parametrize("n_paths,n_steps", [(1, 2), (5, 3), (513, 2), (513, 3), (5000, 7), (70001, 9)])
def test_lsm_edge_sizes_match_oracle(backend, n_paths, n_steps):
    """American put with one path (no regression can run), a handful of
    paths and the fewest dates, FP64 against the oracle; the last two cases
    give threads up to four paths with odd step counts, so the stream jump
    between a thread's paths starts them on odd normal indices too."""

    r = req("american_put", n_paths=n_paths, n_steps=n_steps, seed=17, r=0.06, basis_degree=3,
            precision="fp64_plain")
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-9 * max(abs(b.price), 1e-12)
    assert a.early_exercise_count == b.early_exercise_count
    assert a.regression_steps == b.regression_steps


@pytest.mark.parametrize("n_paths", [1, 5, 257])
def test_antithetic_odd_paths_match_oracle(backend, n_paths):
    """Antithetic pairs with an odd path count (the reference prices
    (n + 1) / 2 pairs), FP64 plain per pair against the oracle."""

    r = req("european_call", method="stepwise", n_paths=n_paths, n_steps=9, seed=4, technique="antithetic",
            precision="fp64_plain")
    _, ref = O.price_paths(r)
    got = backend.price_paths(r)
    assert len(got) == (n_paths + 1) // 2
    assert np.allclose(got, ref, rtol=1e-10, atol=1e-10)
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-10 * max(abs(b.price), 1e-12)


def test_server_cancel_queued_request(backend):
    """mpc_cancel: a request still queued (the only slot is held by a larger
    one) is cancelled and its wait reports MPC_E_CANCELLED; a finished or
    unknown ticket is refused."""

    from montepath_b200.backend import BackendError

    big = req("european_call", model="heston", n_paths=1 << 22, n_steps=256, seed=1, sampling="scrambled_sobol")
    small = req("european_call", method="stepwise", n_paths=10000, n_steps=16, seed=2)
    with backend.server(max_slots=1) as srv:
        t1 = srv.submit(big)
        t2 = srv.submit(small)
        assert srv.poll(t2) is None  # queued: mpc_poll answers MPC_E_BUSY
        assert srv.cancel(t2) == abi.OK
        with pytest.raises(BackendError) as err:
            srv.wait(t2, 10_000)
        assert err.value.status == abi.E_CANCELLED
        done = srv.wait(t1, 60_000)
        assert done.status == abi.OK
        assert srv.poll(t1).price == done.price  # finished: mpc_poll returns the result
        assert srv.cancel(t1) == abi.E_BUSY
        assert srv.cancel(t2 + 1000) == abi.E_NOT_FOUND
        assert srv.stats().cancelled == 1


def test_device_info_and_error_message(backend):
    import ctypes

    lib = abi.load_library()
    info = abi.DeviceInfo()
    assert lib.mpc_device_info(0, ctypes.byref(info)) == abi.OK
    assert info.sm_count > 0 and info.cc_major >= 10 and info.total_memory_bytes > 0 and info.name
    assert lib.mpc_device_info(10_000, ctypes.byref(info)) != abi.OK
    from montepath_b200.backend import BackendError

    with pytest.raises(BackendError) as err:
        backend.price(req("european_call", n_paths=0))
    assert err.value.status == abi.E_INVALID_CONFIG and "n_paths" in str(err.value)


def test_empty_batch(backend):
    assert backend.price_batch([]) == []


def test_fused_heston_merton_sobol_small(backend):
    for kw in (
        dict(model="heston", kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7, v0=0.04),
        dict(model="merton", method="stepwise", jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15),
    ):
        r = req("european_call", n_paths=16384, n_steps=256, seed=42, sampling="scrambled_sobol", **kw)
        _, ref_paths = O.price_paths(r)
        got_paths = backend.price_paths(r)
        assert np.isclose(got_paths, ref_paths, rtol=1e-3, atol=2e-3).mean() > 0.999
        a, b = backend.price(r), O.price(r)
        assert abs(a.price - b.price) < 0.1 * b.stderr, kw["model"]


def test_headline_full_size_fp32_against_fp64_plain(backend):
    """The headline pair at full size (1,048,576 paths x 256 steps, scrambled
    Sobol, seeds 42 / 43): the fused FP32 path reads the same Sobol points as
    the FP64 plain path, so its estimator sits within 0.05 standard errors of
    the FP64 one, with the standard error within 0.5%; the Merton price also
    lies within 3 standard errors of the series price (the stepwise scheme is
    exact in distribution)."""

    heston = dict(model="heston", kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7, v0=0.04, seed=42)
    merton = dict(model="merton", method="stepwise", jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15,
                  seed=43)
    for kw in (heston, merton):
        r32 = req("european_call", n_paths=1 << 20, n_steps=256, sampling="scrambled_sobol", **kw)
        r64 = req("european_call", n_paths=1 << 20, n_steps=256, sampling="scrambled_sobol",
                  precision="fp64_plain", **kw)
        a, b = backend.price(r32), backend.price(r64)
        assert a.path_steps == b.path_steps == (1 << 20) * 256
        assert abs(a.price - b.price) < 0.05 * b.stderr, (kw["model"], a.price, b.price, b.stderr)
        assert abs(a.stderr - b.stderr) < 5e-3 * b.stderr
    series = O.merton_series(100.0, 100.0, 0.03, 0.2, 0.5, -0.1, 0.15, 1.0, exact=True)
    assert abs(a.price - series) < 3 * a.stderr, (a.price, series, a.stderr)


def test_fused_basket_five_assets(backend):
    r = req("basket_call", method="stepwise", n_steps=20, n_paths=8000, seed=4, sampling="counter_hash",
            spots=[100, 95, 105, 98, 102], sigmas=[0.2, 0.25, 0.3, 0.15, 0.22], weights=[0.2] * 5, corr=0.3, k=100)
    _, ref_paths = O.price_paths(r)
    got = backend.price_paths(r)
    assert np.allclose(got, ref_paths, rtol=2e-4, atol=1e-3)


@pytest.mark.parametrize("d", [1, 3, 4, 6, 7, 8])
@pytest.mark.parametrize("sampling", ["scrambled_sobol", "counter_hash"])
def test_basket_every_asset_count(backend, d, sampling):
    """The basket unit is compiled per asset count: every count other than
    the 2 and 5 above, stepwise with a partial last quad of dimensions, FP64
    plain per path and fused FP32 per path against the oracle."""

    spots = [100.0 - 3 * i for i in range(d)]
    sigmas = [0.15 + 0.02 * i for i in range(d)]
    r64 = req("basket_call", method="stepwise", n_steps=7, n_paths=1000, seed=31, sampling=sampling, spots=spots,
              sigmas=sigmas, weights=[1.0 / d] * d, corr=0.3, k=95, precision="fp64_plain")
    _, ref = O.price_paths(r64)
    tol = 2e-5 if sampling == "counter_hash" else 1e-10
    assert np.allclose(backend.price_paths(r64), ref, rtol=tol, atol=tol)
    r32 = req("basket_call", method="stepwise", n_steps=7, n_paths=1000, seed=31, sampling=sampling, spots=spots,
              sigmas=sigmas, weights=[1.0 / d] * d, corr=0.3, k=95)
    assert np.allclose(backend.price_paths(r32), ref, rtol=1e-3, atol=2e-3)


# --------------------------------------------------------------------- LSM --
def test_lsm_fp64_plain_matches_oracle(backend):
    r = req("american_put", n_paths=8192, n_steps=50, seed=5, r=0.06, basis_degree=3, precision="fp64_plain")
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-9 * b.price
    assert a.early_exercise_count == b.early_exercise_count
    assert a.regression_steps == b.regression_steps


@pytest.mark.parametrize("s0", [90.0, 100.0, 110.0])
def test_lsm_fp32_within_se(backend, s0):
    r = req("american_put", n_paths=32768, n_steps=50, seed=5, r=0.06, basis_degree=3, s0=s0)
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) < 0.5 * b.stderr + 1e-3
    crr = O.crr_put(s0, 100, 0.06, 0.2, 1.0, 2048)
    assert abs(a.price - crr) < 5 * a.stderr + 0.15


def test_bermudan_fp64(backend):
    r = req("bermudan_put", n_paths=4096, n_steps=64, seed=3, exercise_steps=[48, 16, 32, 16], precision="fp64_plain")
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-9 * b.price
    assert a.warnings & abi.WARN_SCHEDULE_NORMALISED


@pytest.mark.parametrize("precision", ["fp32_path", "fp64_plain"])
def test_lsm_full_size(backend, precision):
    """524,288 paths x 50 dates (the American-put benchmark size): a job that
    spans every SM; repeatable to the bit and within 5 SE of the binomial price."""
    r = req("american_put", n_paths=524288, n_steps=50, seed=42, r=0.06, basis_degree=3, s0=100.0,
            precision=precision)
    a = backend.price(r)
    b = backend.price(r)
    assert a.price == b.price and a.early_exercise_count == b.early_exercise_count
    crr = O.crr_put(100.0, 100, 0.06, 0.2, 1.0, 2048)
    assert abs(a.price - crr) < 5 * a.stderr + 0.05
    assert a.regression_steps == 49


def test_lsm_batch_equals_individual(backend):
    """Several LSM requests packed into shared cooperative launches give the
    same results as one launch each (each job keeps its block partition)."""
    reqs = [req("american_put", n_paths=20000 + 7000 * i, n_steps=30 + 5 * i, seed=10 + i, r=0.06,
                basis_degree=1 + i % 3, s0=90.0 + 10 * i) for i in range(3)]
    reqs += [req("bermudan_put", n_paths=12000, n_steps=40, seed=4, exercise_steps=[10, 20, 30, 40],
                 precision="fp64_plain"),
             req("american_put", n_paths=9000, n_steps=25, seed=8, precision="fp64_plain", s0=95.0)]
    batch = backend.price_batch(reqs)
    for r, got in zip(reqs, batch):
        one = backend.price(r)
        assert got.status == abi.OK
        assert got.price == one.price, (got.price, one.price)
        assert got.early_exercise_count == one.early_exercise_count
        assert got.regression_steps == one.regression_steps


# --------------------------------------------------------- Brownian bridge --
@pytest.mark.parametrize("workload,steps,technique", [
    ("european_call", 64, "standard"),
    ("european_call", 37, "antithetic"),
    ("arithmetic_asian_call", 50, "control_variate"),
    ("down_and_out_call", 33, "standard"),
    ("lookback_call", 1, "standard"),
    ("arithmetic_asian_call", 365, "standard"),
])
def test_bridge_fp64_per_path_matches_oracle(backend, workload, steps, technique):
    """BrownianBridgePlan (cpu.rs:5886-5981): the device walks the same op
    program depth-first; FP64 per-path payoffs within 1e-10 of the oracle."""

    kw = {"method": "stepwise"} if workload == "european_call" else {}
    r = req(workload, n_paths=3000, n_steps=steps, seed=13, sampling="scrambled_sobol_brownian_bridge",
            technique=technique, precision="fp64_plain", barrier=85.0, **kw)
    _, ref = O.price_paths(r)
    got = backend.price_paths(r)
    assert np.allclose(got, ref, rtol=1e-10, atol=1e-10), float(np.max(np.abs(got - ref)))
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-10 * abs(b.price)


def test_bridge_fp32_fused_matches_oracle(backend):
    r = req("arithmetic_asian_call", n_paths=8192, n_steps=96, seed=7, sampling="scrambled_sobol_brownian_bridge")
    _, ref = O.price_paths(r)
    got = backend.price_paths(r)
    assert np.allclose(got, ref, rtol=2e-4, atol=1e-3)
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) < 0.05 * b.stderr
    # in a mixed batch the bridge request keeps its own launch and its result
    plain_sobol = req("arithmetic_asian_call", n_paths=8192, n_steps=96, seed=7, sampling="scrambled_sobol")
    both = backend.price_batch([r, plain_sobol])
    assert both[0].price == a.price and both[1].price == backend.price(plain_sobol).price


def test_bridge_sampling_reads_as_sobol_outside_gbm_steps(backend):
    """Non-stepwise families take bridge Sobol as plain Sobol, as the reference does."""

    kw = dict(model="heston", n_paths=4096, n_steps=16, seed=3, precision="fp64_plain")
    a = backend.price(req("european_call", sampling="scrambled_sobol_brownian_bridge", **kw))
    b = backend.price(req("european_call", sampling="scrambled_sobol", **kw))
    assert a.price == b.price


# ------------------------------------------------------------------ Greeks --
def _estimates(rep):
    return {rep.estimates[i].greek: rep.estimates[i] for i in range(rep.n_estimates)}


@pytest.mark.parametrize("workload,kw", [
    ("european_call", {}),
    ("european_call", {"method": "stepwise", "n_steps": 32}),
    ("arithmetic_asian_call", {"n_steps": 24}),
    ("down_and_out_call", {"n_steps": 24, "barrier": 85.0}),
    ("lookback_call", {"n_steps": 24}),
    ("basket_call", {}),
    ("european_call", {"model": "heston", "n_steps": 16}),
])
def test_bump_greeks_fp64_match_oracle(backend, workload, kw):
    """Bump-and-revalue (cpu.rs:4938-4983): every leg is an FP64-plain repricing
    (prices 1e-10 relative), so each central difference matches to 1e-7."""

    r = req(workload, n_paths=8000, seed=21, precision="fp64_plain", **kw)
    got = backend.greeks(r, "bump_and_revalue")
    status, ref = O.greeks(r, abi.GREEKS_BUMP_AND_REVALUE)
    assert status == 0 and got.n_estimates == ref.n_estimates > 0
    assert abs(got.base_price - ref.base_price) <= 1e-10 * abs(ref.base_price)
    for greek, e in _estimates(ref).items():
        g = _estimates(got)[greek]
        assert abs(g.bump_size - e.bump_size) <= 1e-15 * abs(e.bump_size)
        assert abs(g.value - e.value) <= 1e-7 * abs(e.value) + 1e-9, (greek, g.value, e.value)
        assert abs(g.stderr - e.stderr) <= 1e-7 * e.stderr + 1e-12


@pytest.mark.parametrize("n_paths", [50_000, 3_000_001])
@pytest.mark.parametrize("estimator", ["pathwise", "likelihood_ratio"])
def test_single_pass_greeks_fp64_replay_reference_stream(backend, estimator, n_paths):
    """european_call_pathwise / likelihood_ratio (cpu.rs:4670-4869): the
    terminal shocks are normal i of MonteCarloRng(seed), replayed on the
    device; at 3,000,001 paths (an odd count) each thread of the grid-stride
    loop takes about ten paths, odd and even stream positions alike."""

    r = req("european_call", n_paths=n_paths, seed=17, precision="fp64_plain")
    got = backend.greeks(r, estimator)
    status, ref = O.greeks(r, abi.GREEK_ESTIMATORS[estimator])
    assert status == 0 and got.n_estimates == ref.n_estimates
    for greek, e in _estimates(ref).items():
        g = _estimates(got)[greek]
        assert abs(g.value - e.value) <= 1e-10 * abs(e.value), (greek, g.value, e.value)
        assert abs(g.stderr - e.stderr) <= 1e-8 * e.stderr


def test_greeks_fp32_within_stderr(backend):
    bs = O.bs_greeks(100.0, 100.0, 0.03, 0.2, 1.0, exact=True)
    r = req("european_call", n_paths=1 << 18, seed=5)  # FP32 path, pseudorandom
    for estimator in ("pathwise", "likelihood_ratio", "bump_and_revalue"):
        rep = backend.greeks(r, estimator)
        for greek, key in ((abi.GREEK_DELTA, "delta"), (abi.GREEK_VEGA, "vega"), (abi.GREEK_RHO, "rho")):
            e = _estimates(rep)[greek]
            assert abs(e.value - bs[key]) < 4 * e.stderr + 2e-3 * abs(bs[key]), (estimator, key, e.value, bs[key])
    h = req("european_call", model="heston", n_paths=1 << 16, n_steps=64, seed=3, sampling="scrambled_sobol")
    got = backend.greeks(h, "bump_and_revalue")
    h64 = req("european_call", model="heston", n_paths=1 << 16, n_steps=64, seed=3, sampling="scrambled_sobol",
              precision="fp64_plain")
    ref = backend.greeks(h64, "bump_and_revalue")
    for greek, e in _estimates(ref).items():
        assert abs(_estimates(got)[greek].value - e.value) < 0.5 * e.stderr, greek


@pytest.mark.parametrize("workload,kw", [
    ("european_call", {"method": "stepwise", "n_steps": 64, "sampling": "scrambled_sobol"}),
    ("european_call", {"sampling": "counter_hash"}),
    ("arithmetic_asian_call", {"n_steps": 32}),
    ("up_and_out_call", {"n_steps": 32, "barrier": 130.0, "sampling": "counter_hash"}),
    ("lookback_call", {"n_steps": 32, "sampling": "scrambled_sobol"}),
    ("european_call", {"model": "heston", "n_steps": 32, "sampling": "scrambled_sobol"}),
])
def test_scenario_bump_legs_equal_separate_pricing(backend, workload, kw):
    """FP32 bump legs that share each normal in one scenario launch price like
    the same legs priced as separate requests: the same FP32 expressions per
    leg, but the two kernels may contract a*b+c into FMAs differently (1 ulp
    on a path) and sum in a different order, so prices agree to 1e-7."""

    r = req(workload, n_paths=20000, seed=31, **kw)
    rep = backend.greeks(r, "bump_and_revalue")
    base = backend.price(r)
    assert abs(rep.base_price - base.price) <= 1e-7 * abs(base.price)
    assert abs(rep.base_stderr - base.stderr) <= 1e-6 * base.stderr
    delta = _estimates(rep)[abi.GREEK_DELTA]
    up, down = abi.Request.from_buffer_copy(r), abi.Request.from_buffer_copy(r)
    up.s0, down.s0 = r.s0 + delta.bump_size, r.s0 - delta.bump_size
    assert abs(delta.bumped_up_price - backend.price(up).price) <= 1e-7 * abs(delta.bumped_up_price)
    assert abs(delta.bumped_down_price - backend.price(down).price) <= 1e-7 * abs(delta.bumped_down_price)


@pytest.mark.parametrize("workload,kw", [
    ("european_call", {"technique": "antithetic"}),
    ("european_call", {"technique": "control_variate", "sampling": "counter_hash"}),
    ("european_call", {"method": "stepwise", "n_steps": 32, "sampling": "scrambled_sobol", "technique": "antithetic"}),
    ("arithmetic_asian_call", {"n_steps": 24, "technique": "control_variate", "sampling": "scrambled_sobol"}),
    ("up_and_out_call", {"n_steps": 24, "barrier": 130.0, "technique": "antithetic", "sampling": "counter_hash"}),
    ("down_and_out_call", {"n_steps": 24, "barrier": 85.0, "technique": "control_variate"}),
    ("lookback_call", {"n_steps": 16, "technique": "antithetic"}),
    ("european_call", {"model": "heston", "n_steps": 16, "technique": "antithetic", "sampling": "scrambled_sobol"}),
    ("european_call", {"model": "heston", "n_steps": 16, "technique": "control_variate", "sampling": "counter_hash"}),
])
def test_scenario_technique_legs_equal_separate_pricing(backend, workload, kw):
    """Antithetic and control-variate bump legs share each normal in one
    scenario launch: each leg's antithetic pair average, or its payoff and
    discounted terminal control, are the single-request unit's FP32
    expressions, summarised by the request's own estimator.  Every leg (base,
    up and down per Greek) prices within 1e-6 of the same leg priced alone
    (FMA contraction and summation order), standard errors within 1e-5."""

    r = req(workload, n_paths=20001, seed=37, **kw)
    rep = backend.greeks(r, "bump_and_revalue")
    base = backend.price(r)
    assert abs(rep.base_price - base.price) <= 1e-6 * abs(base.price)
    assert abs(rep.base_stderr - base.stderr) <= 1e-5 * base.stderr
    est = _estimates(rep)
    for greek, e in est.items():
        for sign, want in ((1.0, e.bumped_up_price), (-1.0, e.bumped_down_price)):
            leg = abi.Request.from_buffer_copy(r)
            if greek == abi.GREEK_DELTA:
                leg.s0 = r.s0 + sign * e.bump_size
            elif greek == abi.GREEK_VEGA and kw.get("model") == "heston":
                leg.v0 = (math.sqrt(r.v0) + sign * e.bump_size) ** 2
            elif greek == abi.GREEK_VEGA:
                leg.sigma = r.sigma + sign * e.bump_size
            elif greek == abi.GREEK_RHO:
                leg.r = r.r + sign * e.bump_size
            else:
                leg.t = r.t + sign * e.bump_size
            got = backend.price(leg).price
            assert abs(want - got) <= 1e-6 * abs(got) + 1e-12, (greek, sign, want, got)


_BASKET5 = {"spots": [100.0, 95.0, 105.0, 90.0, 110.0], "sigmas": [0.2, 0.25, 0.3, 0.35, 0.4], "corr": 0.3}


@pytest.mark.parametrize("kw", [
    {},
    {"method": "stepwise", "n_steps": 16, "sampling": "scrambled_sobol", **_BASKET5},
    {"method": "stepwise", "n_steps": 7, "sampling": "counter_hash", "spots": [100.0, 90.0, 110.0]},
    {"method": "stepwise", "n_steps": 3, "sampling": "pseudorandom", **_BASKET5, "k": 80.0},
])
def test_basket_scenario_legs_equal_separate_pricing(backend, kw):
    """The 13 FP32 basket legs share each path's normal sums in one launch and
    price like the same legs priced one by one.  The scenario kernel regroups
    each asset's log return as T drift + sigma sqrt(dt) (L sum z) instead of
    summing the steps, so FP32 rounding differs per path: leg prices agree to
    2e-5 relative; the Greeks agree with the FP64-plain Greeks of the same
    normals to 0.5 of their standard error."""

    r = req("basket_call", n_paths=30000, seed=23, **kw)
    rep = backend.greeks(r, "bump_and_revalue")
    base = backend.price(r)
    assert abs(rep.base_price - base.price) <= 2e-5 * abs(base.price)
    assert abs(rep.base_stderr - base.stderr) <= 2e-4 * base.stderr
    fields = {abi.GREEK_DELTA: ("spots", 0), abi.GREEK_DELTA2: ("spots", 1), abi.GREEK_VEGA: ("sigmas", 0),
              abi.GREEK_VEGA2: ("sigmas", 1), abi.GREEK_RHO: ("r", None), abi.GREEK_THETA: ("t", None)}
    est = _estimates(rep)
    assert set(est) == set(fields)
    for greek, (name, idx) in fields.items():
        e = est[greek]
        for sign, want in ((1.0, e.bumped_up_price), (-1.0, e.bumped_down_price)):
            leg = abi.Request.from_buffer_copy(r)
            if idx is None:
                setattr(leg, name, getattr(r, name) + sign * e.bump_size)
            else:
                getattr(leg, name)[idx] = getattr(r, name)[idx] + sign * e.bump_size
            got = backend.price(leg).price
            assert abs(want - got) <= 2e-5 * abs(got), (greek, sign, want, got)
    r64 = req("basket_call", n_paths=30000, seed=23, precision="fp64_plain", **kw)
    ref = _estimates(backend.greeks(r64, "bump_and_revalue"))
    for greek, e in ref.items():
        assert abs(est[greek].value - e.value) < 0.5 * e.stderr, (greek, est[greek].value, e.value, e.stderr)


def test_greeks_unsupported_cases(backend):
    from montepath_b200.backend import BackendError

    with pytest.raises(BackendError) as err:
        backend.greeks(req("european_call", model="merton", n_paths=1000, sampling="counter_hash"))
    assert err.value.status == abi.E_UNSUPPORTED
    rep = backend.greeks(req("arithmetic_asian_call", n_paths=2000, n_steps=8), "pathwise")
    assert rep.n_estimates == 0 and rep.warnings & abi.GREEK_WARN_ESTIMATOR_UNSUPPORTED and rep.base_price > 0


# -------------------------------------------------------------------- MLMC --
def test_mlmc_fp64_plain_matches_oracle(backend):
    r = make_request("arithmetic_asian_mlmc", {"paths_per_level": [4000, 2000, 1000, 500], "seed": 3,
                                                "precision": "fp64_plain"})
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) <= 1e-10 * abs(b.price)
    for level in range(4):
        assert abs(a.level_variance[level] - b.level_variance[level]) <= 1e-9 * b.level_variance[level]


def test_mlmc_tolerance_fp32(backend):
    r = make_request("arithmetic_asian_mlmc", {"target_stderr": 0.02, "levels": 5, "seed": 9})
    a, b = backend.price(r), O.price(r)
    assert abs(a.price - b.price) < 3 * math.hypot(a.stderr, b.stderr)
    assert a.total_step_updates <= r.max_step_updates * 1.01 + 64


def test_mlmc_batch_equals_individual(backend):
    """MLMC requests batched (all pilot levels in one launch, all main levels
    in another) give the same results as each request alone."""
    reqs = [make_request("arithmetic_asian_mlmc", {"target_stderr": 0.03, "levels": 4, "seed": 20 + i})
            for i in range(3)]
    reqs.append(make_request("arithmetic_asian_mlmc", {"paths_per_level": [4000, 2000, 1000], "levels": 3,
                                                        "seed": 5, "precision": "fp64_plain"}))
    batch = backend.price_batch(reqs)
    for r, got in zip(reqs, batch):
        one = backend.price(r)
        assert got.status == abi.OK
        assert got.price == one.price and got.stderr == one.stderr
        assert got.total_step_updates == one.total_step_updates


# ------------------------------------------------------ batch and serving ---
def test_batch_equals_individual(backend):
    reqs = [
        req("european_call", method="stepwise", n_paths=3000 + 1000 * i, n_steps=16 + 7 * i, seed=i,
            sampling="counter_hash")
        for i in range(6)
    ] + [req("basket_call", method="stepwise", n_steps=12, n_paths=5000, seed=77, sampling="counter_hash",
             spots=[100] * 5, sigmas=[0.2] * 5, weights=[0.2] * 5, corr=0.3)]
    alone = [backend.price(r) for r in reqs]
    batch = backend.price_batch(reqs)
    for a, b in zip(alone, batch):
        assert a.price == b.price and a.stderr == b.stderr


def test_full_book_batch_equals_individual(backend):
    """The full 4,096-contract heterogeneous book (seed 42; European, Asian,
    up-and-out and 5-asset basket; 1e3-1e6 paths, 16-365 steps) in one batch:
    every result of 32 contracts spread over the book, 8 of each kind, equals
    that contract priced alone bit for bit (tile partials are per request and
    summed in tile order), and every price is finite with a positive count."""

    from montepath_b200 import workloads

    book = workloads.book(42)
    batch = backend.price_batch(book)
    assert len(batch) == 4096
    assert all(math.isfinite(b.price) and b.price >= 0.0 and b.n_samples > 0 for b in batch)
    for i in list(range(0, 4096, 128)):
        alone = backend.price(book[i])
        assert alone.price == batch[i].price and alone.stderr == batch[i].stderr, i


def test_repeated_batches_replay_a_graph(backend):
    """The second identical fused batch is captured as a CUDA graph and later
    ones replay it: same results, same kernel count, new inputs honoured."""

    reqs = [req("european_call", method="stepwise", n_paths=30000, n_steps=32, seed=s, sampling="counter_hash")
            for s in (1, 2)] + [req("european_call", model="heston", n_paths=20000, n_steps=16, seed=3,
                                    sampling="scrambled_sobol")]
    runs = []
    for _ in range(4):  # direct, capture, replay, replay
        runs.append([r.price for r in backend.price_batch(reqs)])
        assert backend.last_timing()[1] == 2
    assert all(run == runs[0] for run in runs)
    changed = [abi.Request.from_buffer_copy(r) for r in reqs]
    changed[0].seed = 99  # same shape, new descriptor contents: the replay reads them
    got = backend.price_batch(changed)
    assert got[0].price == backend.price(changed[0]).price and got[0].price != runs[0][0]
    assert got[2].price == runs[0][2]


def test_serving_alone_equals_mix(backend):
    reqs = [req("european_call", method="stepwise", n_paths=20000 + 5000 * i, n_steps=64, seed=100 + i,
                sampling="counter_hash") for i in range(8)]
    reqs += [req("european_call", model="heston", n_paths=8000, n_steps=32, seed=5, sampling="scrambled_sobol")]
    alone = [backend.price(r) for r in reqs]
    with backend.server(max_slots=4) as srv:
        tickets = [srv.submit(r) for r in reqs]
        mixed = [srv.wait(t) for t in tickets]
        stats = srv.stats()
    for a, b in zip(alone, mixed):
        assert abs(a.price - b.price) <= 1e-12 * abs(a.price)
    assert stats.completed == len(reqs)
    assert stats.p99_ms >= stats.p50_ms > 0


# ------------------------------------------------------ errors and contract --
def test_invalid_config_returns_code(backend):
    from montepath_b200.backend import BackendError

    r = req("european_call", n_paths=0)
    with pytest.raises(BackendError) as err:
        backend.price(r)
    assert err.value.status == abi.E_INVALID_CONFIG
    r = req("european_call", model="merton", method="stepwise", sampling="pseudorandom")
    with pytest.raises(BackendError) as err:
        backend.price(r)
    assert err.value.status == abi.E_UNSUPPORTED


def test_budget_exceeded_returns_code():
    from montepath_b200.backend import BackendError, CudaBackend

    with CudaBackend(0, hbm_budget_bytes=64 << 20) as small:
        r = req("european_call", model="heston", n_paths=1 << 20, n_steps=256, sampling="scrambled_sobol",
                precision="fp64_plain")
        with pytest.raises(BackendError) as err:
            small.price(r)
        assert err.value.status == abi.E_OOM_BUDGET


def test_reference_v1_kernel_contract(backend):
    torch = pytest.importorskip("torch")
    n_paths, n_steps = 5000, 40
    z = O.pseudorandom_normals(42, n_paths * n_steps)
    normals = torch.tensor(z, dtype=torch.float64, device="cuda")
    payoffs = torch.zeros(n_paths, dtype=torch.float64, device="cuda")
    dt = 1.0 / n_steps
    drift, vol, disc = (0.03 - 0.02) * dt, 0.2 * math.sqrt(dt), math.exp(-0.03)
    lib = abi.load_library()
    status = lib.mpc_european_call_stepwise_v1(normals.data_ptr(), payoffs.data_ptr(), n_paths, n_steps,
                                               math.log(100.0), 100.0, drift, vol, disc, None)
    torch.cuda.synchronize()
    assert status == abi.OK
    ref = np.maximum(np.exp(math.log(100.0) + np.cumsum(drift + vol * z.reshape(n_paths, n_steps), axis=1)[:, -1]) - 100.0, 0) * disc
    assert np.allclose(payoffs.cpu().numpy(), ref, rtol=1e-12, atol=1e-12)


# ------------------------------------------------------------ cost model --
@pytest.mark.parametrize("workload,kw", [
    ("european_call", dict(model="heston", method="stepwise", n_steps=128, sampling="scrambled_sobol")),
    ("arithmetic_asian_call", dict(n_steps=96, sampling="counter_hash")),
    ("european_call", dict(method="stepwise", n_steps=64, precision="fp64_plain", sampling="scrambled_sobol")),
    ("american_put", dict(n_steps=50)),
])
def test_cost_model_predicts_device_time(backend, workload, kw):
    """mpc_estimate_cost against the measured device time of the same request (within 2x)."""

    import ctypes

    r = req(workload, n_paths=1 << 19 if workload != "american_put" else 200_000, seed=3, **kw)
    cost = abi.Cost()
    assert abi.load_library().mpc_estimate_cost(ctypes.byref(r), 0, ctypes.byref(cost)) == abi.OK
    times = []
    for _ in range(3):
        backend.price(r)
        times.append(backend.last_timing()[0])
    measured = min(times)
    assert 0.5 < cost.estimated_runtime_ms / measured < 2.0, (cost.estimated_runtime_ms, measured)


def test_cost_model_calibrated_on_this_device(backend):
    """mpc_calibrate_cost measures the rate table on the device in use; the
    calibrated estimates then predict the device time of requests of other
    sizes and shapes within 1.6x (the built-in table: 2x)."""

    seconds = backend.calibrate_cost()
    assert 0.0 < seconds < 60.0
    cases = [
        ("european_call", dict(model="heston", method="stepwise", n_steps=128, sampling="scrambled_sobol")),
        ("european_call", dict(model="merton", method="stepwise", n_steps=96, sampling="scrambled_sobol")),
        ("arithmetic_asian_call", dict(n_steps=96, sampling="counter_hash")),
        ("european_call", dict(method="stepwise", n_steps=64, precision="fp64_plain", sampling="scrambled_sobol")),
        ("down_and_out_call", dict(n_steps=80, barrier=80.0, sampling="pseudorandom")),
        ("european_call", dict(n_paths=1 << 21)),
    ]
    for workload, kw in cases:
        kw = dict(kw)
        r = req(workload, n_paths=kw.pop("n_paths", 1 << 19), seed=3, **kw)
        cost = backend.estimate_cost(r)
        assert cost.confidence.decode() == "calibrated"
        times = []
        for _ in range(3):
            backend.price(r)
            times.append(backend.last_timing()[0])
        measured = min(times)
        assert 1 / 1.6 < cost.estimated_runtime_ms / measured < 1.6, (workload, kw, cost.estimated_runtime_ms, measured)


# ---------------------------------------------------------- harness rows --
def test_mc_bench_compact_rows(backend):
    """mc_cuda_* rows (BenchmarkResult shape) from the real device, compact suite."""

    from montepath_b200 import mc_bench

    report = mc_bench.run(backend, compact=True, repeats=2)
    rows = {r["benchmark_name"]: r for r in report["results"]}
    assert set(rows) == mc_bench._COMPACT
    assert abs(rows["mc_cuda_european_call_terminal"]["metric_value"] - 9.413403383853016) < 0.1
    assert all(r["throughput_per_sec"] > 1e6 for r in rows.values())
