"""Open-loop load generator for the serving loop: submits a timed request
stream to an ``mpc_server`` at its arrival times and reports latency
percentiles and throughput from the server's own timestamps."""

from __future__ import annotations

import threading
import time
from typing import Sequence

from . import abi
from .backend import CudaBackend


def replay(backend: CudaBackend, stream: Sequence[tuple[float, str, abi.Request]], plain: bool = False,
           hbm_budget_bytes: int = 64 << 30, max_slots: int = 256, drain_timeout_s: float = 600.0,
           mode: str | None = None) -> dict:
    """Runs the stream (arrival seconds, kind, request) through a fresh server.

    Arrivals are open-loop: submissions follow the schedule whether or not
    earlier requests have finished.  Returns a summary with per-kind latency
    percentiles, throughput in path-steps/s and the server statistics.
    """

    tickets: list[tuple[int, str, abi.Request]] = []
    lock = threading.Lock()
    mode = mode or ("plain" if plain else "device_loop")
    with backend.server(hbm_budget_bytes=hbm_budget_bytes, max_slots=max_slots, mode=mode) as srv:
        t0 = time.perf_counter()
        lag = 0.0
        for arrival, kind, req in stream:
            delay = arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            else:
                lag = max(lag, -delay)
            ticket = srv.submit(req)
            with lock:
                tickets.append((ticket, kind, req))
        submitted_at = time.perf_counter() - t0
        results = []
        for ticket, kind, req in tickets:
            res = srv.wait(ticket, timeout_ms=int(drain_timeout_s * 1000))
            results.append((kind, req, res))
        wall = time.perf_counter() - t0
        stats = srv.stats()
    lat_all = sorted(r.t_complete_ms - r.t_enqueue_ms for _, _, r in results)

    def pct(values, q):
        if not values:
            return None
        pos = q * (len(values) - 1)
        lo = int(pos)
        hi = min(lo + 1, len(values) - 1)
        return values[lo] + (values[hi] - values[lo]) * (pos - lo)

    per_kind = {}
    for kind in sorted({k for k, _, _ in results}):
        lat = sorted(r.t_complete_ms - r.t_enqueue_ms for k, _, r in results if k == kind)
        per_kind[kind] = {"count": len(lat), "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99)}
    path_steps = sum(r.path_steps for _, _, r in results)
    span_s = (max(r.t_complete_ms for _, _, r in results) - min(r.t_enqueue_ms for _, _, r in results)) / 1e3
    return {
        "mode": {"plain": "plain_fifo_fp64", "waves": "continuous_batching_fp32_waves",
                 "device_loop": "continuous_batching_fp32_device_loop"}[mode],
        "requests": len(results),
        "offered_seconds": stream[-1][0] if stream else 0.0,
        "submit_lag_max_ms": lag * 1e3,
        "submitted_s": submitted_at,
        "wall_s": wall,
        "p50_ms": pct(lat_all, 0.5),
        "p99_ms": pct(lat_all, 0.99),
        "max_ms": lat_all[-1] if lat_all else None,
        "per_kind": per_kind,
        "path_steps": path_steps,
        "path_steps_per_sec": path_steps / span_s if span_s > 0 else None,
        "busy_ms": stats.busy_ms,
        "waves": stats.waves,
        "peak_bytes": stats.peak_bytes,
        "mlmc_target_met": sum(1 for k, _, r in results if k == "asian_mlmc" and r.target_met),
        "mlmc_requests": sum(1 for k, _, _ in results if k == "asian_mlmc"),
        # requests whose allocation the step-update cap cut (cpu.rs:3390-3403), and the
        # standard error they reached instead of the target
        "mlmc_step_cap_hit": sum(1 for k, _, r in results if k == "asian_mlmc" and r.max_step_updates_hit),
        "mlmc_stderr_p50": pct(sorted(r.stderr for k, _, r in results if k == "asian_mlmc"), 0.5),
    }


def main(argv: Sequence[str] | None = None) -> None:
    """``python -m montepath_b200.serving``: replays a seeded Poisson stream
    (default: 2,000 requests/s for 60 s, 64 GB budget) through the
    continuous-batching server and prints the summary as one JSON line."""

    import argparse
    import json

    from . import workloads

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--seconds", type=float, default=60.0, help="arrival window of the stream")
    ap.add_argument("--rate", type=float, default=2000.0, help="mean arrivals per second")
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--budget-gb", type=float, default=64.0, help="HBM budget of the server")
    ap.add_argument("--plain", action="store_true", help="plain FIFO FP64 server, one request per launch")
    ap.add_argument("--mode", default="", choices=["", "device_loop", "waves", "plain"],
                    help="server mode (default device_loop; --plain selects plain)")
    ap.add_argument("--out", default="", help="also write the summary to this file")
    args = ap.parse_args(argv)
    stream = workloads.serving_stream(args.seed, rate=args.rate, duration_s=args.seconds,
                                      precision="fp64_plain" if args.plain else "fp32_path")
    with CudaBackend(0) as backend:
        summary = replay(backend, stream, plain=args.plain, hbm_budget_bytes=int(args.budget_gb * (1 << 30)),
                         mode=args.mode or None)
    summary.update({"rate": args.rate, "seed": args.seed, "budget_gb": args.budget_gb})
    line = json.dumps(summary)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
