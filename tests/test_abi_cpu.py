"""Host-side checks of the C ABI (no GPU needed): exports, struct layouts,
defaults, validation codes, request mapping and the Python surfaces."""

import ctypes
import os
import re

import pytest

from montepath_b200 import abi
from montepath_b200.requests import ConfigError, make_request

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "montepath_cuda.h")


def lib():
    return abi.load_library()


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(mpc_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 30
    L = lib()
    for name in names:
        assert hasattr(L, name), name
    bound = {name for name, _, _ in abi.FUNCTIONS}
    assert set(names) <= bound, set(names) - bound


def test_struct_layouts_match_header():
    L = lib()
    for index, struct in enumerate(abi.STRUCTS):
        assert L.mpc_struct_size(index) == ctypes.sizeof(struct), struct.__name__


def test_status_strings():
    L = lib()
    assert L.mpc_status_string(abi.E_UNSUPPORTED) == b"MPC_E_UNSUPPORTED"
    assert L.mpc_abi_version() == 1


# Rust `Default` impls (crates/mc-core/src/runtime/cpu.rs:1311-1815)
@pytest.mark.parametrize(
    "workload,expect",
    [
        ("european_call", dict(s0=100.0, k=100.0, r=0.03, sigma=0.2, t=1.0, n_paths=100_000, n_steps=252, seed=42)),
        ("down_and_out_call", dict(barrier=80.0, n_steps=252)),
        ("american_put", dict(n_steps=64, basis_degree=2)),
        ("bermudan_put", dict(n_steps=64, n_exercise=4)),
        ("arithmetic_asian_mlmc", dict(base_steps=16, levels=4, refinement_factor=2, pilot_paths_per_level=2048,
                                       min_step_updates=100_000, max_step_updates=10_000_000)),
    ],
)
def test_defaults_follow_rust_configs(workload, expect):
    r = make_request(workload)
    for key, value in expect.items():
        assert getattr(r, key) == value, key
    assert (r.v0, r.kappa, r.theta, r.vol_of_vol, r.rho) == (0.04, 1.5, 0.04, 0.3, -0.6)
    assert (r.jump_intensity, r.jump_mean, r.jump_volatility) == (0.4, -0.08, 0.25)
    assert list(r.paths_per_level[:4]) == [50000, 25000, 12500, 6250]
    assert list(r.spots[:2]) == [100.0, 95.0] and r.corr[1] == 0.35


def validate(r):
    msg = ctypes.create_string_buffer(256)
    return lib().mpc_validate(ctypes.byref(r), msg, 256), msg.value.decode()


@pytest.mark.parametrize(
    "workload,kw,code",
    [
        ("european_call", dict(n_paths=0), abi.E_INVALID_CONFIG),
        ("european_call", dict(n_steps=0), abi.E_INVALID_CONFIG),
        ("european_call", dict(s0=-1.0), abi.E_INVALID_CONFIG),
        ("european_call", dict(t=0.0), abi.E_INVALID_CONFIG),
        ("european_call", dict(model="heston", rho=1.5), abi.E_INVALID_CONFIG),
        ("european_call", dict(model="heston", vol_of_vol=-0.1), abi.E_INVALID_CONFIG),
        ("european_call", dict(model="merton", method="stepwise", sampling="pseudorandom"), abi.E_UNSUPPORTED),
        ("european_call", dict(model="merton", sampling="pseudorandom", technique="control_variate"),
         abi.E_UNSUPPORTED),
        ("european_call", dict(model="merton", sampling="scrambled_sobol", technique="antithetic"), abi.E_UNSUPPORTED),
        ("european_call", dict(method="stepwise", n_steps=70_000, sampling="scrambled_sobol_brownian_bridge"),
         abi.E_UNSUPPORTED),
        ("arithmetic_asian_mlmc", dict(sampling="scrambled_sobol_brownian_bridge"), abi.E_UNSUPPORTED),
        ("down_and_out_call", dict(barrier=0.0), abi.E_INVALID_CONFIG),
        ("american_put", dict(n_steps=1), abi.E_INVALID_CONFIG),
        ("american_put", dict(sampling="scrambled_sobol"), abi.E_UNSUPPORTED),
        ("bermudan_put", dict(exercise_steps=[0, 16]), abi.E_INVALID_CONFIG),
        ("bermudan_put", dict(exercise_steps=[65]), abi.E_INVALID_CONFIG),
        ("basket_call", dict(spots=[100, 100], corr=[[1, 2], [2, 1]]), abi.E_INVALID_CONFIG),
        ("basket_call", dict(spots=[100, 100, 100], corr=[[1, 0.9, -0.9], [0.9, 1, 0.9], [-0.9, 0.9, 1]]),
         abi.E_INVALID_CONFIG),
        ("arithmetic_asian_mlmc", dict(refinement_factor=1), abi.E_INVALID_CONFIG),
        ("arithmetic_asian_mlmc", dict(levels=0), abi.E_INVALID_CONFIG),
        ("european_call", dict(block_size=192), abi.E_UNSUPPORTED),
        ("european_call", dict(paths_per_thread=65), abi.E_INVALID_CONFIG),
    ],
)
def test_validation_codes(workload, kw, code):
    status, msg = validate(make_request(workload, kw))
    assert status == code, msg
    assert msg


def test_valid_requests_pass():
    for w in ("european_call", "arithmetic_asian_call", "down_and_out_call", "lookback_call", "basket_call",
              "american_put", "bermudan_put", "arithmetic_asian_mlmc"):
        assert validate(make_request(w))[0] == abi.OK, w
    assert validate(make_request("european_call", model="merton", sampling="counter_hash"))[0] == abi.OK
    assert validate(make_request("european_call", model="merton", sampling="pseudorandom"))[0] == abi.OK
    for block in (128, 256, 512):
        assert validate(make_request("european_call", block_size=block, paths_per_thread=4))[0] == abi.OK


def test_unknown_enum_rejected():
    r = make_request("european_call")
    r.sampling = 17
    assert validate(r)[0] == abi.E_INVALID_CONFIG


def test_supports_and_estimate():
    r = make_request("european_call", model="heston", n_paths=1 << 20, n_steps=256, sampling="scrambled_sobol",
                     precision="fp64_plain")
    sup = abi.Support()
    assert lib().mpc_supports(ctypes.byref(r), ctypes.byref(sup)) == abi.OK
    assert sup.supported == 1
    # FP64 plain materialises 2 normals per step in HBM
    assert sup.estimated_bytes >= (1 << 20) * 512 * 8
    r.precision = abi.PRECISION_FP32_PATH
    b = ctypes.c_uint64()
    lib().mpc_estimate_bytes(ctypes.byref(r), ctypes.byref(b))
    assert b.value < 64 << 20


def test_create_without_device_reports_no_device():
    n = ctypes.c_int()
    lib().mpc_device_count(ctypes.byref(n))
    if n.value > 0:
        pytest.skip("a CUDA device is present")
    handle = ctypes.c_void_p()
    assert lib().mpc_create(None, ctypes.byref(handle)) == abi.E_NO_DEVICE


def test_create_rejects_unsupported_block_size():
    # checked before any device call, so it holds with or without a GPU
    handle = ctypes.c_void_p()
    opts = abi.Options(device=0, deterministic=1, hbm_budget_bytes=0, default_block_size=384)
    assert lib().mpc_create(ctypes.byref(opts), ctypes.byref(handle)) == abi.E_UNSUPPORTED
    assert not handle.value


def test_request_aliases():
    r = make_request("european_call", {"spot": 90, "strike": 95, "rate": 0.01, "volatility": 0.3, "maturity": 2,
                                       "paths": 1000, "steps": 12, "technique": "antithetic",
                                       "sampling": "randomized_halton", "method": "stepwise_paths"})
    assert (r.s0, r.k, r.r, r.sigma, r.t, r.n_paths, r.n_steps) == (90, 95, 0.01, 0.3, 2, 1000, 12)
    assert r.technique == abi.TECHNIQUE_ANTITHETIC and r.sampling == abi.SAMPLING_RANDOMIZED_HALTON
    assert r.method == abi.METHOD_STEPWISE
    h = make_request("european_call", {"model": "heston", "initial_variance": 0.05, "mean_reversion": 2.5,
                                       "long_run_variance": 0.03, "vol_of_vol": 0.4, "correlation": -0.5})
    assert (h.v0, h.kappa, h.theta, h.vol_of_vol, h.rho) == (0.05, 2.5, 0.03, 0.4, -0.5)
    b = make_request("basket_call", {"spot_1": 10, "spot_2": 20, "volatility_1": 0.1, "volatility_2": 0.3,
                                     "correlation": -0.2, "weight_1": 0.3, "weight_2": 0.7})
    assert list(b.spots[:2]) == [10, 20] and b.corr[1] == -0.2 and list(b.weights[:2]) == [0.3, 0.7]
    d = make_request("basket_call", {"spots": [1, 2, 3, 4, 5], "corr": 0.3})
    assert d.n_assets == 5 and d.corr[1] == 0.3 and d.corr[6] == 1.0
    with pytest.raises(ConfigError):
        make_request("european_call", {"sampling": "no_such"})


def test_production_overlay_without_device():
    from montepath_b200 import production

    cap = production.cuda_capability()
    assert cap["backend_id"] == "nvidia_cuda"
    if not cap["devices"]:
        assert cap["status"] == "unavailable"
        sel = production.select_backend("european_call", backend="cuda")
        assert not sel.ok and sel.diagnostics[0]["code"] == "MC_BACKEND_CUDA_UNAVAILABLE"
    sel = production.select_backend("inventory_policy", backend="cuda")
    assert not sel.ok


def test_mapping_abi_response_shape(monkeypatch):
    """The native module's fn(mapping) -> dict shape (lib.rs:680-707), with the
    device call replaced by the oracle on the host."""

    from montepath_b200 import native
    from oracle import oracle as O

    class OracleBackend:
        def price(self, req):
            return O.price(req)

    monkeypatch.setattr(native, "backend", lambda: OracleBackend())
    cfg = dict(spot=100.0, strike=100.0, rate=0.03, volatility=0.2, maturity=1.0, n_paths=2000, n_steps=16, seed=42,
               sampling="pseudorandom", technique="standard", n_threads=0)
    out = native.price_european_call(cfg)
    assert set(out) == {"price", "stderr", "values", "manifest", "warnings"}
    assert out["manifest"]["backend"] == "nvidia_cuda"
    assert out["manifest"]["config"] == cfg
    mer = native.price_merton_jump_diffusion_call(dict(cfg, jump_intensity=0.4, jump_mean=-0.08, jump_volatility=0.25))
    ref = O.price(make_request("european_call", dict(model="merton", n_paths=2000, seed=42, jump_intensity=0.4,
                                                     jump_mean=-0.08, jump_volatility=0.25)))
    assert mer["price"] == ref.price  # the reference's own pseudorandom Merton, not a substitute stream
    lsm = native.price_american_put(dict(cfg, basis_degree=5, n_steps=16))
    assert lsm["values"]["regression_basis"] == "laguerre_lsm_degree_3"
    with pytest.raises(ValueError):
        native.price_european_call(dict(cfg, sampling="bogus"))


def test_reference_pricing_surface_accepts_module(monkeypatch):
    """montepath's own price_* helpers (python/montepath/pricing.py:711-780)
    drive this module when a reference checkout is named by MONTEPATH_REFERENCE."""

    root = os.environ.get("MONTEPATH_REFERENCE", "")
    ref_python = os.path.join(root, "python")
    if not root or not os.path.isdir(ref_python):
        pytest.skip("MONTEPATH_REFERENCE does not name a montepath checkout")
    import sys

    monkeypatch.syspath_prepend(ref_python)
    montepath = pytest.importorskip("montepath")
    from montepath_b200 import native
    from oracle import oracle as O

    class OracleBackend:
        def price(self, req):
            return O.price(req)

    monkeypatch.setattr(native, "backend", lambda: OracleBackend())
    res = montepath.price_european_call(native_module="montepath_b200.native", n_paths=4000, n_steps=8, seed=1)
    assert res.manifest["backend"] == "nvidia_cuda" and res.price > 0
    heston = montepath.price_heston_european_call(native_module="montepath_b200.native", n_paths=2000, n_steps=8)
    assert heston.price > 0
    assert "montepath_b200.native" in sys.modules


def test_mc_bench_rows_have_the_harness_shape(monkeypatch):
    """mc_cuda_* rows carry the fields of BenchmarkResult (crates/mc-bench/src/result.rs:3-17);
    the device calls are replaced by the oracle on the host, at a small size."""

    from montepath_b200 import mc_bench
    from oracle import oracle as O

    class OracleBackend:
        def price(self, req):
            return O.price(req)

        def price_batch(self, reqs):
            return [O.price(r) for r in reqs]

        def greeks(self, req):
            return O.greeks(req, abi.GREEKS_BUMP_AND_REVALUE)[1]

    monkeypatch.setattr(mc_bench, "MC_PATHS", 600)
    monkeypatch.setattr(mc_bench, "MC_STEPS", 8)
    monkeypatch.setattr(mc_bench, "GREEK_PATHS", 600)
    report = mc_bench.run(OracleBackend(), compact=False, precision="fp64_plain", repeats=2)
    fields = {"benchmark_name", "benchmark_version", "implementation", "backend", "methodology", "planner_mode",
              "iterations", "total_runtime_ms", "per_iteration_us", "throughput_per_sec", "metric_name",
              "metric_value"}
    assert set(report) == {"generated_at_unix_ms", "results"}
    names = [r["benchmark_name"] for r in report["results"]]
    assert len(names) == len(set(names)) and all(n.startswith("mc_cuda_") and n.endswith("_fp64_plain") for n in names)
    for row in report["results"]:
        assert set(row) == fields and row["backend"] == "nvidia_cuda" and row["iterations"] == 2
        assert row["throughput_per_sec"] > 0 and row["metric_value"] > 0


def test_calibrated_cost_entry_points_reject_null_context():
    import ctypes

    lib = abi.load_library()
    r = make_request("european_call", {"n_paths": 1000})
    cost = abi.Cost()
    assert lib.mpc_estimate_cost_ctx(None, ctypes.byref(r), ctypes.byref(cost)) == abi.E_INVALID_CONFIG
    assert lib.mpc_calibrate_cost(None, None) == abi.E_INVALID_CONFIG


def test_cost_model_and_planner_priority():
    """mpc_estimate_cost (host only) and the planner order it feeds."""

    from montepath_b200 import production

    big = production.estimate_cost("heston_european_call", {"n_paths": 1 << 20, "n_steps": 256,
                                                             "sampling": "scrambled_sobol"})
    # measured headline rate: 268,435,456 path-steps in about 1 ms of device time
    assert 0.6 < big["estimated_runtime_ms"] < 2.0 and big["confidence"] == "measured"
    small = production.estimate_cost("european_call", {"n_paths": 1000})
    assert small["estimated_runtime_ms"] < 0.01 < small["estimated_total_ms"]
    plain = production.estimate_cost("european_call", {"n_paths": 1 << 20, "n_steps": 64, "method": "stepwise",
                                                       "precision": "fp64_plain", "sampling": "scrambled_sobol"})
    fused = production.estimate_cost("european_call", {"n_paths": 1 << 20, "n_steps": 64, "method": "stepwise",
                                                       "sampling": "scrambled_sobol"})
    assert plain["estimated_runtime_ms"] > 5 * fused["estimated_runtime_ms"]
    assert production.planner_priority("heston_european_call", {"n_paths": 1 << 20, "n_steps": 256},
                                       cuda_available=True)[0] == "nvidia_cuda"
    assert production.planner_priority("european_call", {"n_paths": 100}, cuda_available=True)[0] == "cpu_native"
    assert production.planner_priority("european_call", {"n_paths": 10**6}, cuda_available=False)[0] == "cpu_native"


def test_serving_command_line_help():
    """``python -m montepath_b200.serving`` parses its options without a GPU."""

    from montepath_b200 import serving

    with pytest.raises(SystemExit) as done:
        serving.main(["--help"])
    assert done.value.code == 0
