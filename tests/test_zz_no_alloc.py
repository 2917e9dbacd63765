"""The no-allocation entry point, for callers that cannot let a library
allocate device memory (a service whose allocator owns the GPU's memory, or a
latency-critical path where cudaMalloc/cudaFree are forbidden).

mpc_price_fused_noalloc is called through the C ABI, twice in a row per
request, and must agree with mpc_price within the 1e-12 relative tolerance
the other batch/serving equivalence tests use (the two entry points run the
same fused kernel; only the tile size, hence the FP64 summation order, may
differ).  The requests cover the one-path-per-thread tiling, the doubled
tilings of large requests (4,194,305 paths) and the scratch's exact limit
(16,777,216 paths).  One test runs in a fresh process whose first CUDA work is
a no-allocation call, so that the call's own set-up is exercised; the file
also passes when it runs after the other tests.
"""

import ctypes
import os
import subprocess
import sys

import pytest

from montepath_b200 import abi
from montepath_b200.requests import make_request

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAX_PATHS = 1 << 24


def call_noalloc(lib, req):
    out = abi.Result()
    msg = ctypes.create_string_buffer(256)
    status = lib.mpc_price_fused_noalloc(ctypes.byref(req), ctypes.byref(out), None, msg, 256)
    return status, out, msg.value.decode()


def assert_same(out, ref):
    assert abs(out.price - ref.price) <= 1e-12 * abs(ref.price), (out.price, ref.price)
    assert abs(out.stderr - ref.stderr) <= 1e-12 * abs(ref.stderr), (out.stderr, ref.stderr)
    assert out.n_samples == ref.n_samples


REQUESTS = [
    ("european_call", dict(method="stepwise", n_paths=50_000, n_steps=64, seed=7, sampling="counter_hash")),
    ("european_call", dict(model="heston", n_paths=65_536, n_steps=128, seed=42, sampling="scrambled_sobol",
                           kappa=2.0, vol_of_vol=0.5, rho=-0.7)),
    ("arithmetic_asian_call", dict(n_paths=30_000, n_steps=48, seed=3, technique="antithetic")),
    # 4,194,305 paths: 4,097 tiles of 1,024 would overflow the 4,096-tile list, so tiles of 2,048 (ppt 8)
    ("european_call", dict(method="stepwise", n_paths=4_194_305, n_steps=4, seed=11, sampling="counter_hash")),
    # exactly the scratch's limit: 4,096 tiles of 4,096 paths (ppt 16)
    ("european_call", dict(method="stepwise", n_paths=MAX_PATHS, n_steps=2, seed=12, sampling="counter_hash")),
    # a paths_per_thread hint is honoured, as mpc_price honours it
    ("european_call", dict(model="merton", n_paths=300_000, n_steps=16, seed=5, sampling="scrambled_sobol",
                           jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15, paths_per_thread=4)),
]


def test_no_alloc_matches_price_two_calls_in_a_row():
    import torch

    from montepath_b200.backend import CudaBackend

    lib = abi.load_library()
    with CudaBackend(0) as backend:
        refs = [backend.price(make_request(wl, cfg)) for wl, cfg in REQUESTS]
    for (wl, cfg), ref in zip(REQUESTS, refs):
        req = make_request(wl, cfg)
        status, out, msg = call_noalloc(lib, req)  # may perform the device set-up
        assert status == abi.OK, msg
        assert_same(out, ref)
        free_before = torch.cuda.mem_get_info(0)[0]
        status, out, msg = call_noalloc(lib, req)
        assert status == abi.OK, msg
        assert_same(out, ref)
        assert torch.cuda.mem_get_info(0)[0] == free_before, "the no-allocation call changed free device memory"


def test_no_alloc_first_call_in_a_fresh_process():
    """The first CUDA work of the process is a no-allocation call; its result
    then equals mpc_price's in the same process."""

    script = (
        "import sys; sys.path.insert(0, %r)\n"
        "import ctypes\n"
        "from montepath_b200 import abi\n"
        "from montepath_b200.requests import make_request\n"
        "from montepath_b200.backend import CudaBackend\n"
        "lib = abi.load_library()\n"
        "req = make_request('european_call', dict(model='heston', n_paths=200_000, n_steps=64, seed=9,\n"
        "                   sampling='scrambled_sobol', kappa=2.0, vol_of_vol=0.5, rho=-0.7))\n"
        "outs = []\n"
        "for _ in range(2):\n"
        "    out = abi.Result(); msg = ctypes.create_string_buffer(256)\n"
        "    st = lib.mpc_price_fused_noalloc(ctypes.byref(req), ctypes.byref(out), None, msg, 256)\n"
        "    assert st == 0, msg.value\n"
        "    outs.append(out)\n"
        "with CudaBackend(0) as be:\n"
        "    ref = be.price(req)\n"
        "for out in outs:\n"
        "    assert abs(out.price - ref.price) <= 1e-12 * abs(ref.price), (out.price, ref.price)\n"
        "    assert abs(out.stderr - ref.stderr) <= 1e-12 * abs(ref.stderr)\n"
        "print('fresh ok')\n"
    ) % ROOT
    proc = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "fresh ok" in proc.stdout


def test_no_alloc_rejects_oversize_and_unsupported():
    lib = abi.load_library()
    big = make_request("european_call", dict(method="stepwise", n_paths=MAX_PATHS + 1, n_steps=4,
                                             sampling="counter_hash"))
    status, _, msg = call_noalloc(lib, big)
    assert status == abi.E_OOM_BUDGET and "16777216" in msg
    lsm = make_request("american_put", dict(n_paths=1000, n_steps=8))
    status, _, msg = call_noalloc(lib, lsm)
    assert status == abi.E_UNSUPPORTED and msg
    for hint in (3, 32):
        bad = make_request("european_call", dict(method="stepwise", n_paths=10_000, n_steps=4,
                                                 sampling="counter_hash", paths_per_thread=hint))
        status, _, msg = call_noalloc(lib, bad)
        assert status == abi.E_UNSUPPORTED and "paths_per_thread" in msg
    # a valid power of two whose work list would not fit 4,096 tiles
    tight = make_request("european_call", dict(method="stepwise", n_paths=MAX_PATHS, n_steps=2,
                                               sampling="counter_hash", paths_per_thread=8))
    status, _, msg = call_noalloc(lib, tight)
    assert status == abi.E_UNSUPPORTED and "paths_per_thread" in msg
