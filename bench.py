"""Benchmark of the B200 Monte Carlo pricing backend.

Workload (the configuration the headline metric is quoted on): Heston and
Merton European calls, 1,048,576 paths x 256 steps each, scrambled Sobol
samples (2 and 3 dimensions per step), FP32 path arithmetic with FP64
accumulation -- one step prices both requests through ``mpc_price_batch``.
Synthetic inputs: every sample is generated on the device from the seed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  ``value`` is path-steps/s over all ranks with the
requests already resident (device time of each step from CUDA events on the
library stream, summed over K steps, max over ranks); ``e2e`` is the same
metric through the public C ABI with host request structs, wall-clock per
call including the descriptor upload and the result read-back.  The plain
FP64 one-request-per-launch path is timed beside it for the speed-up ratio.
N > 1 runs independent replicas (one per GPU): Monte Carlo paths need no
exchange, so there is no data-path collective.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PATHS = 1_048_576
N_STEPS = 256
SEED = 42
WORKLOAD = "heston_merton_european_sobol_1048576x256"

HESTON = dict(model="heston", s0=100.0, k=100.0, r=0.03, t=1.0, kappa=2.0, theta=0.04, vol_of_vol=0.5, rho=-0.7,
              v0=0.04, n_paths=N_PATHS, n_steps=N_STEPS, seed=SEED, sampling="scrambled_sobol")
MERTON = dict(model="merton", method="stepwise", s0=100.0, k=100.0, r=0.03, sigma=0.2, t=1.0, jump_intensity=0.5,
              jump_mean=-0.1, jump_volatility=0.15, n_paths=N_PATHS, n_steps=N_STEPS, seed=SEED + 1,
              sampling="scrambled_sobol")

# Algorithmic work per path-step (fixed by convention; FMA = 2 flops, one MUFU op = 1 SFU op):
# Sobol + Acklam normal 24 flops + 1 SFU; Heston step 16 flops + 1 SFU (sqrt v+);
# Merton step 4 flops (+ the Sobol uniform of the Poisson dimension, no inverse CDF).
FLOPS_PER_STEP = {"heston": 2 * 24 + 16, "merton": 24 + 4}
SFU_PER_STEP = {"heston": 2 * 1 + 1, "merton": 1}
# Warp instructions the two fused kernels issue per 32 path-steps
# (smsp__inst_executed.sum of the quarter-size ncu capture in profiles/): the
# kernels are issue-bound, so this gives the fraction of the SMs' issue slots
# (4 warp instructions per cycle per SM) the measured rate uses.
WARP_INSTR_PER_32_STEPS = {"heston": 84.7, "merton": 69.8}
# Lane instructions per path-step of the same capture (smsp__thread_inst_executed.sum / path-steps).
LANE_INSTR_PER_STEP = {"heston": 84.6, "merton": 66.4}


def requests(precision: str):
    from montepath_b200.requests import make_request

    h = make_request("european_call", dict(HESTON, precision=precision))
    m = make_request("european_call", dict(MERTON, precision=precision))
    return [h, m]


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu), "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                        rows.append(parts)
        finally:
            try:
                os.remove(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = sorted(float(r[1]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


def reduce_max(pg, value: float, device: str) -> float:
    """Max over ranks (device time of the slowest replica)."""
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate(world: int, path_steps_per_rank: int, steps: int, max_ms: float) -> float:
    """Whole-job path-steps/s: every replica prices the same work (weak scaling)."""
    return world * path_steps_per_rank * steps / (max_ms * 1e-3)


def barrier(pg):
    if pg is not None:
        pg.barrier()


def load_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


def load_traffic() -> dict:
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _cpu_pair(paths: int, threads: int) -> float:
    """Prices the Heston and Merton requests at `paths` paths with the oracle on
    `threads` host threads; returns the wall seconds."""

    from oracle import oracle as O

    t0 = time.perf_counter()
    for cfg in (HESTON, MERTON):
        O.price_threaded(O.make_request("european_call", dict(cfg, n_paths=paths, precision="fp64_plain")), threads)
    return time.perf_counter() - t0


def cpu_baseline(seconds_target: float = 12.0) -> dict:
    """The oracle (FP64 C++ restatement of the reference CPU path) on a
    bounded sample of the same workload, all host threads."""

    from oracle import oracle as O

    O.lib()  # compile/load the oracle before timing
    threads = os.cpu_count() or 1
    paths = 2048
    while True:
        dt = _cpu_pair(paths, threads)
        total_steps = 2 * paths * N_STEPS
        if dt * threads >= seconds_target or paths >= N_PATHS:
            break
        paths = min(N_PATHS, int(paths * max(2.0, seconds_target / max(dt * threads, 1e-3))))
    return {
        "value": total_steps / dt,
        "unit": "path-steps/s",
        "cores": threads,
        "kind": "port",
        "sample": f"Heston + Merton Sobol {paths} paths x {N_STEPS} steps each (of {N_PATHS}), FP64, {dt:.2f} s wall",
    }


# what the GPU legs hand to the CPU leg (requests and GPU prices to check)
_CPU_LEG_INPUTS: dict = {}


def cpu_leg(line: dict) -> None:
    """The CPU leg (rank 0, N = 1; skipped by --no-cpu): the oracle -- the FP64
    C++ restatement of the reference's CPU path -- timed on a bounded sample
    of the workload (`cpu_baseline`), and its reference values for the prices
    this line reports, with the GPU prices' errors against them: the closed
    forms (Heston semi-analytic, Merton series, Black-Scholes), CRR for the
    American put, and FP64 prices on the same samples.  All of the bench's
    use of the oracle happens here, as the checker and as the timed CPU path."""

    from oracle import oracle as O

    line["cpu_baseline"] = cpu_baseline()
    semi = O.heston_call(100, 100, 0.03, 0.04, 2.0, 0.04, 0.5, -0.7, 1.0)
    series = O.merton_series(100, 100, 0.03, 0.2, 0.5, -0.1, 0.15, 1.0, exact=True)
    h, m = line["prices"]["heston"], line["prices"]["merton"]
    # the closed forms are continuous-time; the gap to them includes the
    # 256-step scheme's discretisation bias (see the Heston/Merton leg)
    h["semi_analytic"], h["minus_semi_in_se"] = semi, (h["price"] - semi) / h["stderr"]
    m["series"], m["minus_series_in_se"] = series, (m["price"] - series) / m["stderr"]
    leg_out = line.get("legs", {})
    if "gbm_european_20000x64" in leg_out and "gbm_european_20000x64" in _CPU_LEG_INPUTS:
        c1, r64 = leg_out["gbm_european_20000x64"], _CPU_LEG_INPUTS["gbm_european_20000x64"]
        t0 = time.perf_counter()
        ref = O.price(r64)
        t_cpu = time.perf_counter() - t0
        bs = 9.413403383853016
        c1["fp64_plain"]["err_vs_black_scholes_se"] = (c1["fp64_plain"]["price"] - bs) / c1["fp64_plain"]["stderr"]
        c1["fp64_plain"]["abs_diff_vs_oracle"] = abs(c1["fp64_plain"]["price"] - ref.price)
        c1["cpu_oracle_1_thread"] = {"price": ref.price, "seconds": t_cpu, "path_steps_per_sec": 20000 * 64 / t_cpu}
    if "heston_merton_1048576x256" in leg_out:
        c2 = leg_out["heston_merton_1048576x256"]
        c2["semi_analytic"] = semi
        for row in c2["steps"].values():
            row["minus_semi_in_se"] = (row["price"] - semi) / row["stderr"]
        rich = c2["richardson_1024_2048"]
        rich["minus_semi_in_se"] = (rich["price"] - semi) / rich["stderr_bound"]
    if "american_put_lsm_524288x50" in leg_out:
        for key, row in leg_out["american_put_lsm_524288x50"].items():
            row["crr_2048"] = O.crr_put(float(key.split("_")[1]), 100.0, 0.06, 0.2, 1.0, 2048)
    if "book_4096" in leg_out and "book_4096" in _CPU_LEG_INPUTS:
        diffs_se, worst_abs = [], 0.0
        for req, gpu_price in _CPU_LEG_INPUTS["book_4096"]:
            ref = O.price(req)
            d = abs(gpu_price - ref.price)
            worst_abs = max(worst_abs, d)
            if ref.stderr > 0:
                diffs_se.append(d / ref.stderr)
        leg_out["book_4096"]["vs_fp64_oracle"] = {
            "contracts": len(_CPU_LEG_INPUTS["book_4096"]), "max_abs_diff": worst_abs,
            "max_diff_in_se": max(diffs_se) if diffs_se else None,
            "within_3se": sum(1 for x in diffs_se if x <= 3.0), "with_nonzero_stderr": len(diffs_se)}


def run_reference(args) -> None:
    """The reference arm: the reference's CPU path for this workload -- its C++
    restatement (the oracle; the Rust crate does not build here) -- pricing
    the full Heston + Merton pair, 1,048,576 paths x 256 steps each, in FP64 on
    all host threads (the reference's chunk-per-thread scheme).  Warm-up steps
    price 16,384-path samples; every timed step is the full workload.  Loads
    nothing from the CUDA library."""

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    O.lib()
    threads = os.cpu_count() or 1
    paths = args.paths or N_PATHS
    for _ in range(args.warmup):
        _cpu_pair(min(16_384, paths), threads)
    wall = 0.0
    for _ in range(args.steps):
        wall += _cpu_pair(paths, threads)
    path_steps = 2 * paths * N_STEPS
    value = path_steps * args.steps / wall
    line = {
        "impl": "reference",
        "metric": "path-steps/s",
        "value": value,
        "unit": "path-steps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * wall / max(args.steps, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded scrambled Sobol samples)",
        "config": {"workload": WORKLOAD, "paths": paths, "steps_per_path": N_STEPS, "requests": 2,
                   "host_cores": threads,
                   "note": "the reference CPU path (its C++ restatement) on the full workload every timed step"},
        "cpu_baseline": {"value": value, "unit": "path-steps/s", "cores": threads, "kind": "port",
                         "sample": f"Heston + Merton Sobol {paths} paths x {N_STEPS} steps each (workload: {N_PATHS}), "
                                   f"FP64, {args.steps} steps of {wall / max(args.steps, 1):.2f} s"},
        "e2e": {"value": value, "unit": "path-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    rank, world, local, pg = dist_setup(args.gpus)
    from montepath_b200 import abi
    from montepath_b200.backend import CudaBackend

    backend = CudaBackend(local)
    fused = requests("fp32_path")
    plain = requests("fp64_plain")
    if args.paths:
        for r in fused + plain:
            r.n_paths = args.paths
    path_steps = sum(r.n_paths * r.n_steps for r in fused)
    # compile step (mpc_prepare): the autotuner measures each request kind's block size
    shapes = {}
    for name, r in zip(("heston", "merton"), fused):
        art = backend.prepare(r)
        shapes[name] = {"block": art.block_size, "paths_per_thread": art.paths_per_thread, "tiles": art.tiles}

    for _ in range(max(args.warmup, 3)):
        backend.price_batch(fused)
    # timed region: device time of each step (CUDA events on the library stream)
    barrier(pg)
    device_ms = 0.0
    launches = 0
    results = None
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            backend.flush_l2()  # between steps, outside the events
            results = backend.price_batch(fused)
            ms, n = backend.last_timing()
            device_ms += ms
            launches += n
    barrier(pg)
    clock_info = clocks.summary()
    dev = f"cuda:{local}"
    device_ms = reduce_max(pg, device_ms, dev)
    value = aggregate(world, path_steps, args.steps, device_ms)

    # end to end through the public ABI: host request structs in, results out
    e2e_s = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        backend.price_batch(fused)
        e2e_s += time.perf_counter() - t0
    h2d, d2h = backend.last_transfer()
    e2e_s = reduce_max(pg, e2e_s, dev)
    e2e_value = aggregate(world, path_steps, args.steps, e2e_s * 1e3)

    # plain FP64 one-request-per-launch baseline (same requests, same seeds)
    plain_value = plain_ms = plain_results = None
    if not args.no_plain:
        plain_ms = 0.0
        plain_steps = max(1, min(2, args.steps))
        backend.price_batch(plain)
        for _ in range(plain_steps):
            plain_results = backend.price_batch(plain)
            plain_ms += backend.last_timing()[0]
        plain_ms = reduce_max(pg, plain_ms, dev) / plain_steps
        plain_value = aggregate(world, path_steps, 1, plain_ms)

    # roofline of the fused kernels (compute-bound: FP32 pipe and MUFU)
    fp32_peak, sfu_peak = backend.measure_peaks()
    per_rank_rate = path_steps / (device_ms / args.steps * 1e-3)
    flops = sum(FLOPS_PER_STEP[k] for k in ("heston", "merton")) * (per_rank_rate / 2)
    sfu = sum(SFU_PER_STEP[k] for k in ("heston", "merton")) * (per_rank_rate / 2)
    fr_fp32 = flops / 1e12 / fp32_peak if fp32_peak else None
    fr_sfu = sfu / 1e12 / sfu_peak if sfu_peak else None
    traffic = load_traffic().get("fused_heston_merton_sobol", {}).get("bytes_per_step")
    fr_issue = None
    info = abi.DeviceInfo()
    sm_mhz = clock_info.get("sm_mhz") or clock_info.get("sm_max_mhz")
    if backend.lib.mpc_device_info(local, ctypes.byref(info)) == abi.OK and sm_mhz:
        warp_instr = sum(WARP_INSTR_PER_32_STEPS.values()) / 32.0 * (per_rank_rate / 2)
        fr_issue = warp_instr / (info.sm_count * 4 * sm_mhz * 1e6)
    bound, achieved, peak, unit, frac = "fp32", flops / 1e12, fp32_peak, "TFLOP/s", fr_fp32
    if fr_sfu is not None and fr_fp32 is not None and fr_sfu > fr_fp32:
        bound, achieved, peak, unit, frac = "sfu", sfu / 1e12, sfu_peak, "Tops/s", fr_sfu

    if rank == 0:
        line = {
            "metric": "path-steps/s",
            "value": value,
            "unit": "path-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": device_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 path / f64 accumulation",
            "data": "synthetic (seeded scrambled Sobol samples generated on the device)",
            "config": {
                "workload": WORKLOAD,
                "paths": fused[0].n_paths,
                "steps_per_path": N_STEPS,
                "requests_per_step": 2,
                "precision": "fp32_path",
                "parallelism": f"replicas x{world}",
                "l2": "flushed between steps (256 MiB write); samples never touch HBM",
                "launch_shapes": shapes,
            },
            "e2e": {"value": e2e_value, "unit": "path-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clock_info,
            "roofline": {
                "bound": bound,
                "achieved": achieved,
                "peak": peak,
                "unit": unit,
                "frac": frac,
                "traffic": traffic,
                "fractions": {"fp32": fr_fp32, "sfu": fr_sfu, "issue": fr_issue},
                "lane_instructions_per_path_step": LANE_INSTR_PER_STEP,
                "peak_source": "measured by mpc_measure_peaks on this GPU (FP32 FMA chains / MUFU ex2 chains)",
                "hbm_peak_gbs": load_peaks().get("hbm_gbs"),
            },
            "prices": {
                "heston": {"price": results[0].price, "stderr": results[0].stderr},
                "merton": {"price": results[1].price, "stderr": results[1].stderr},
            },
        }
        if plain_value is not None:
            line["plain_fp64"] = {"value": plain_value, "unit": "path-steps/s", "ms_per_step": plain_ms,
                                  "speedup_fused_vs_plain": value / plain_value}
            for key, i in (("heston", 0), ("merton", 1)):
                line["prices"][key]["fp64_plain"] = plain_results[i].price
                line["prices"][key]["minus_fp64_plain_in_se"] = (results[i].price - plain_results[i].price) / results[i].stderr
        # the configuration legs and the CPU baseline are single-GPU
        # measurements: taken at N = 1 only
        legs = [x for x in args.legs.split(",") if x and x != "none"] if world == 1 else []
        if "all" in legs:
            legs = list(LEGS)
        if legs:
            line["legs"] = {}
            for leg in legs:
                if leg == "book_4096":
                    line["legs"][leg] = leg_book(backend, args.book_contracts)
                else:
                    line["legs"][leg] = LEGS[leg](backend)
        if not args.no_cpu and world == 1:
            cpu_leg(line)
        print(json.dumps(line), flush=True)
    backend.close()
    if pg is not None:
        pg.destroy_process_group()


def _timed(backend, fn):
    res = fn()
    return res, backend.last_timing()[0]


def leg_gbm_european_small(backend) -> dict:
    """Plain method, small: GBM European 20,000 x 64, seed 42, pseudorandom (the
    reference's MonteCarloRng stream replayed), FP64 one request per launch."""

    from montepath_b200.requests import make_request

    cfg = dict(method="stepwise", n_paths=20000, n_steps=64, seed=42, n_threads=1)
    r64 = make_request("european_call", dict(cfg, precision="fp64_plain"))
    r32 = make_request("european_call", dict(cfg, precision="fp32_path"))
    for _ in range(3):
        backend.price(r64)
        backend.price(r32)
    a, t64 = _timed(backend, lambda: backend.price(r64))
    b, t32 = _timed(backend, lambda: backend.price(r32))
    ps = 20000 * 64
    _CPU_LEG_INPUTS["gbm_european_20000x64"] = r64
    return {
        "fp64_plain": {"price": a.price, "stderr": a.stderr, "ms": t64, "path_steps_per_sec": ps / (t64 * 1e-3)},
        "fp32_path": {"price": b.price, "stderr": b.stderr, "ms": t32, "path_steps_per_sec": ps / (t32 * 1e-3)},
    }


def leg_heston_merton(backend) -> dict:
    """Accuracy of the headline Heston request against the semi-analytic
    price as the step count grows (1,048,576 paths, scrambled Sobol, FP32
    path): the full-truncation Euler scheme is biased by its time step (the
    Feller condition fails here, 2 kappa theta = 0.16 < xi^2 = 0.25), the
    closed form is not, so the gap in standard errors shrinks with dt; the
    step-doubling (Richardson) estimate 2 P(2n) - P(n) removes the first-order
    bias.  Its standard error is bounded by sqrt(5) SE(2n) from the two
    estimates' variances (they share the Sobol points, so it is smaller)."""

    from montepath_b200.requests import make_request

    rows = {}
    for n in (256, 512, 1024, 2048):
        r = make_request("european_call", dict(HESTON, n_steps=n, precision="fp32_path"))
        rows[n] = backend.price(r)
    out = {"steps": {str(n): {"price": res.price, "stderr": res.stderr} for n, res in rows.items()}}
    out["richardson_1024_2048"] = {"price": 2.0 * rows[2048].price - rows[1024].price,
                                   "stderr_bound": math.sqrt(5.0) * rows[2048].stderr}
    return out


def leg_american_put_lsm(backend) -> dict:
    """American put by Longstaff-Schwartz, 524,288 paths x 50 dates, S0 in {90, 100, 110}."""

    from montepath_b200.requests import make_request

    out = {}
    for s0 in (90.0, 100.0, 110.0):
        row = {}
        for precision in ("fp32_path", "fp64_plain"):
            r = make_request("american_put", dict(s0=s0, k=100.0, r=0.06, sigma=0.2, t=1.0, n_paths=524288,
                                                  n_steps=50, basis_degree=3, seed=42, precision=precision))
            backend.price(r)
            res, ms = _timed(backend, lambda: backend.price(r))
            row[precision] = {"price": res.price, "stderr": res.stderr, "ms": ms,
                              "path_steps_per_sec": 524288 * 50 / (ms * 1e-3),
                              "early_exercise": res.early_exercise_count, "regressions": res.regression_steps}
        out[f"s0_{int(s0)}"] = row
    return out


def leg_book(backend, contracts: int = 4096) -> dict:
    """4,096-contract heterogeneous book in one batched launch vs plain FP64
    per-request launches (timed on every 63rd contract, which cycles through
    the four contract kinds, and extrapolated by path-steps).  `contracts`
    takes the first contracts of the same book (smaller profiling cases)."""

    from montepath_b200 import workloads
    from montepath_b200.requests import copy_request

    book = workloads.book(42)[:contracts]
    total = workloads.book_path_steps(book)
    blocks = {}
    for r in book:  # the autotuner measures each contract kind once (family, sampler, step bucket)
        b = backend.prepare(r).block_size
        blocks[b] = blocks.get(b, 0) + 1
    backend.price_batch(book)
    res, ms = _timed(backend, lambda: backend.price_batch(book))
    _, launches = backend.last_timing()
    # the contracts small enough (<= 2e6 path-steps) for the CPU leg to price
    # with the oracle on the same samples
    small = [i for i, r in enumerate(book) if r.n_paths * r.n_steps <= 2_000_000][:64]
    _CPU_LEG_INPUTS["book_4096"] = [(book[i], res[i].price) for i in small]
    sample = book[::63]
    plain_ms = 0.0
    for r in sample:
        p = copy_request(r)
        p.precision = 0
        backend.price(p)
        plain_ms += backend.last_timing()[0]
    sample_steps = workloads.book_path_steps(sample)
    plain_rate = sample_steps / (plain_ms * 1e-3)
    return {
        "contracts": len(book),
        "path_steps": total,
        "batched_fp32": {"ms": ms, "path_steps_per_sec": total / (ms * 1e-3), "kernel_launches": launches},
        "plain_fp64_sampled": {"contracts_timed": len(sample), "ms_sample": plain_ms, "path_steps_per_sec": plain_rate,
                               "estimated_ms_full_book": total / plain_rate * 1e3},
        "speedup_batched_vs_plain": (total / (ms * 1e-3)) / plain_rate,
        "contracts_by_block_size": {str(k): v for k, v in sorted(blocks.items())},
        "price_checksum": sum(x.price for x in res),
    }


def leg_merton_reference(backend) -> dict:
    """The reference's own Merton estimator (terminal, pseudorandom
    MonteCarloRng stream per chunk, 8 chunks) at 1,048,576 paths: the stream
    replay of mpc_merton.cu, device time with L2 flushed, median of 10."""

    from montepath_b200.requests import make_request

    r = make_request("european_call", dict(model="merton", n_paths=1 << 20, seed=9303, n_threads=8,
                                           jump_intensity=0.5, jump_mean=-0.1, jump_volatility=0.15))
    for _ in range(3):
        backend.price(r)
    ts = []
    res = None
    for _ in range(10):
        backend.flush_l2()
        res = backend.price(r)
        ts.append(backend.last_timing()[0])
    ms = sorted(ts)[len(ts) // 2]
    return {"paths": r.n_paths, "chunks": 8, "ms": ms, "paths_per_sec": r.n_paths / (ms * 1e-3),
            "price": res.price, "stderr": res.stderr}


def leg_serving(backend) -> dict:
    """Poisson serving stream at 2,000 requests/s, seed 42: the full 60 s
    stream (about 120,000 requests) through the resident device loop; the
    host-scheduled waves and the plain FIFO FP64 baseline at the same offered
    load on the first 10 s and 2 s of the same stream (the FIFO baseline
    cannot keep up with this load, so its queue only grows with the window)."""

    from montepath_b200 import serving, workloads

    loop = serving.replay(backend, workloads.serving_stream(42, duration_s=60.0), mode="device_loop")
    waves = serving.replay(backend, workloads.serving_stream(42, duration_s=10.0), mode="waves")
    plain = serving.replay(backend, workloads.serving_stream(42, duration_s=2.0, precision="fp64_plain"),
                           mode="plain")
    return {"device_loop_60s": loop, "waves_10s": waves, "plain_fifo_2s": plain, "rate_per_s": 2000.0}


LEGS = {"gbm_european_20000x64": leg_gbm_european_small, "heston_merton_1048576x256": leg_heston_merton, "american_put_lsm_524288x50": leg_american_put_lsm, "book_4096": leg_book,
        "serving_2000rps": leg_serving, "merton_reference_1048576": leg_merton_reference}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 plain comparison of the headline")
    ap.add_argument("--paths", type=int, default=0, help="override the path count (profiling cases)")
    ap.add_argument("--legs", default="all", help="comma list of gbm_european_20000x64, heston_merton_1048576x256, american_put_lsm_524288x50, book_4096, serving_2000rps, merton_reference_1048576; all or none")
    ap.add_argument("--book-contracts", type=int, default=4096,
                    help="first contracts of the book in the book_4096 leg (profiling cases)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
