"""The no-allocation entry point, for callers that cannot let a library
allocate device memory (a service whose allocator owns the GPU's memory, or a
latency-critical path where cudaMalloc/cudaFree are forbidden).

mpc_price_fused_noalloc is called through the C ABI, twice in a row per
request, and must agree with mpc_price within the 1e-12 relative tolerance
the other batch/serving equivalence tests use (the two entry points run the
same fused kernel; only the tile size, hence the FP64 summation order, may
differ).  It runs alone in a fresh process as well as after the other tests:
the first call on a device performs its set-up.
"""

import ctypes

import pytest

from montepath_b200 import abi
from montepath_b200.requests import make_request

pytestmark = pytest.mark.gpu


def call_noalloc(lib, req):
    out = abi.Result()
    msg = ctypes.create_string_buffer(256)
    status = lib.mpc_price_fused_noalloc(ctypes.byref(req), ctypes.byref(out), None, msg, 256)
    return status, out, msg.value.decode()


def test_no_alloc_matches_price_two_calls_in_a_row():
    from montepath_b200.backend import CudaBackend

    lib = abi.load_library()
    reqs = [
        make_request("european_call", dict(method="stepwise", n_paths=50_000, n_steps=64, seed=7,
                                           sampling="counter_hash")),
        make_request("european_call", dict(model="heston", n_paths=65_536, n_steps=128, seed=42,
                                           sampling="scrambled_sobol", kappa=2.0, vol_of_vol=0.5, rho=-0.7)),
        make_request("arithmetic_asian_call", dict(n_paths=30_000, n_steps=48, seed=3, technique="antithetic")),
    ]
    with CudaBackend(0) as backend:
        for req in reqs:
            ref = backend.price(req)
            for _ in range(2):
                status, out, msg = call_noalloc(lib, req)
                assert status == abi.OK, msg
                assert abs(out.price - ref.price) <= 1e-12 * abs(ref.price)
                assert abs(out.stderr - ref.stderr) <= 1e-12 * abs(ref.stderr)
                assert out.n_samples == ref.n_samples


def test_no_alloc_rejects_oversize_and_unsupported():
    lib = abi.load_library()
    big = make_request("european_call", dict(method="stepwise", n_paths=(1 << 24) + 1, n_steps=4,
                                             sampling="counter_hash"))
    status, _, msg = call_noalloc(lib, big)
    assert status == abi.E_OOM_BUDGET and "16777216" in msg
    lsm = make_request("american_put", dict(n_paths=1000, n_steps=8))
    status, _, msg = call_noalloc(lib, lsm)
    assert status == abi.E_UNSUPPORTED and msg
