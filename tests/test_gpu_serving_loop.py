"""The resident device-loop server (mpc_server mode 2).

Requests of every kind go through one server: fused FP32 requests under the
three loop samplers (counter hash, scrambled Sobol, the pseudorandom stream),
MLMC with the tolerance solver (pilot levels, then main levels, all through
the loop), and the host-batched kinds (Longstaff-Schwartz, randomized Halton,
the pseudorandom Merton stream replay, FP64 plain).  Each result must equal
the same request priced alone through mpc_price: 1e-12 relative for the
estimators (the tile partition, hence the FP64 summation order, can differ),
identical MLMC allocations.
"""

import time

import pytest

from montepath_b200 import abi
from montepath_b200.requests import make_request

pytestmark = pytest.mark.gpu


def req(workload, **kw):
    return make_request(workload, kw)


def mixed_requests():
    rs = [req("european_call", method="stepwise", n_paths=20_000 + 5_000 * i, n_steps=64, seed=100 + i,
              sampling="counter_hash") for i in range(6)]
    rs += [req("european_call", model="heston", n_paths=30_000 + 1_000 * i, n_steps=64, seed=5 + i,
               sampling="scrambled_sobol", kappa=2.0, vol_of_vol=0.5, rho=-0.7) for i in range(3)]
    rs += [req("arithmetic_asian_call", n_paths=40_000, n_steps=32, seed=9, n_threads=4),
           req("up_and_out_call", n_paths=25_000, n_steps=48, seed=10, sampling="scrambled_sobol", barrier=130.0),
           req("european_call", model="merton", method="stepwise", n_paths=20_000, n_steps=32, seed=11,
               sampling="scrambled_sobol", jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15),
           req("basket_call", method="stepwise", n_steps=16, n_paths=10_000, seed=12, sampling="counter_hash",
               spots=[100, 95, 105], sigmas=[0.2, 0.25, 0.3], weights=[1 / 3] * 3, corr=0.3, k=100)]
    rs += [req("arithmetic_asian_mlmc", levels=5, base_steps=16, refinement_factor=2, target_stderr=0.01,
               seed=200 + i, sampling="counter_hash") for i in range(2)]
    rs += [req("arithmetic_asian_mlmc", levels=4, paths_per_level=[4000, 2000, 1000, 500], seed=210,
               sampling="scrambled_sobol", scramble_replicates=4)]
    rs += [req("american_put", n_paths=50_000, n_steps=50, r=0.06, basis_degree=3, seed=13),
           req("european_call", method="stepwise", n_paths=8_000, n_steps=32, seed=14, sampling="randomized_halton"),
           req("european_call", model="merton", n_paths=30_000, seed=15, jump_intensity=0.5, jump_mean=-0.1,
               jump_volatility=0.15),
           req("european_call", method="stepwise", n_paths=10_000, n_steps=32, seed=16, precision="fp64_plain")]
    return rs


def same(a, b, what):
    assert a.status == 0 and b.status == 0, what
    assert abs(a.price - b.price) <= 1e-12 * max(abs(a.price), 1e-300), (what, a.price, b.price)
    assert abs(a.stderr - b.stderr) <= 1e-10 * max(abs(a.stderr), 1e-300), (what, a.stderr, b.stderr)


def test_device_loop_alone_equals_mix(backend):
    reqs = mixed_requests()
    alone = [backend.price(r) for r in reqs]
    with backend.server(max_slots=8, mode="device_loop") as srv:
        tickets = [srv.submit(r) for r in reqs]
        mixed = [srv.wait(t, 120_000) for t in tickets]
        stats = srv.stats()
    for i, (a, b) in enumerate(zip(alone, mixed)):
        same(a, b, i)
        if reqs[i].workload == abi.WORKLOAD_ASIAN_MLMC:  # MLMC: the same allocation and levels
            assert [a.level_paths[l] for l in range(a.n_levels)] == [b.level_paths[l] for l in range(b.n_levels)]
            assert a.target_met == b.target_met
    assert stats.completed == len(reqs)
    assert stats.p99_ms >= stats.p50_ms > 0


def test_device_loop_reuses_slots_and_relaunches(backend):
    """Two slots and 40 requests: every slot and ring entry is reused many
    times; a pause longer than the loop's idle exit (20 ms) makes the loop
    leave, and the next request relaunches it."""

    reqs = [req("european_call", method="stepwise", n_paths=3_000 + 37 * i, n_steps=16 + (i % 5), seed=300 + i,
                sampling="counter_hash" if i % 3 else "scrambled_sobol") for i in range(40)]
    alone = [backend.price(r) for r in reqs]
    with backend.server(max_slots=2, mode="device_loop") as srv:
        first = [srv.submit(r) for r in reqs[:30]]
        got = [srv.wait(t, 60_000) for t in first]
        time.sleep(0.1)
        rest = [srv.submit(r) for r in reqs[30:]]
        got += [srv.wait(t, 60_000) for t in rest]
        stats = srv.stats()
    for i, (a, b) in enumerate(zip(alone, got)):
        same(a, b, i)
    assert stats.waves >= 2  # loop launches: the idle exit was followed by a relaunch


def test_device_loop_mlmc_meets_rmse_target(backend):
    """An arithmetic Asian MLMC request at levels 0-6, refinement 2, base 16
    steps and target standard error 1e-3 meets its target when the step-update
    cap is lifted, and agrees with the FP64 oracle's estimate at a looser
    target within 3 combined standard errors."""

    from oracle import oracle as O

    cfg = dict(levels=7, base_steps=16, refinement_factor=2, seed=42, sampling="counter_hash")
    r = req("arithmetic_asian_mlmc", target_stderr=1e-3, max_step_updates=20_000_000_000, **cfg)
    with backend.server(mode="device_loop") as srv:
        res = srv.wait(srv.submit(r), 300_000)
    assert res.target_met == 1 and res.max_step_updates_hit == 0
    assert res.estimated_stderr <= 1e-3
    ref = O.price(req("arithmetic_asian_mlmc", target_stderr=2e-2, precision="fp64_plain", **cfg))
    assert abs(res.price - ref.price) < 3 * (res.stderr ** 2 + ref.stderr ** 2) ** 0.5, (res.price, ref.price)


def test_device_loop_budget_cancel_and_stop(backend):
    """Admission under the HBM budget, cancellation of a queued request, a
    request too large for the budget refused with MPC_E_OOM_BUDGET, and a
    stop while work is still running: the loop leaves, the server returns
    promptly and the context prices on afterwards."""

    from montepath_b200.backend import BackendError

    big = req("european_call", model="heston", n_paths=1 << 22, n_steps=256, seed=1, sampling="scrambled_sobol")
    small = req("european_call", method="stepwise", n_paths=10_000, n_steps=16, seed=2, sampling="counter_hash")
    huge = req("european_call", model="heston", n_paths=1 << 30, n_steps=256, seed=3, sampling="scrambled_sobol",
               precision="fp64_plain")
    with backend.server(max_slots=1, mode="device_loop", hbm_budget_bytes=1 << 30) as srv:
        t_big = srv.submit(big)
        t_small = srv.submit(small)
        assert srv.poll(t_small) is None
        assert srv.cancel(t_small) == abi.OK
        with pytest.raises(BackendError) as err:
            srv.wait(t_small, 10_000)
        assert err.value.status == abi.E_CANCELLED
        t_huge = srv.submit(huge)
        done = srv.wait(t_big, 60_000)
        assert done.status == abi.OK
        with pytest.raises(BackendError) as err:
            srv.wait(t_huge, 60_000)
        assert err.value.status == abi.E_OOM_BUDGET
    with backend.server(max_slots=4, mode="device_loop") as srv:
        for i in range(4):
            srv.submit(req("european_call", model="heston", n_paths=1 << 21, n_steps=256, seed=10 + i,
                           sampling="scrambled_sobol"))
        t0 = time.perf_counter()
    assert time.perf_counter() - t0 < 5.0  # stop with work in flight: the loop leaves at its next claim
    after = backend.price(small)
    assert after.status == abi.OK and after.price > 0
