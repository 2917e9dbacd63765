"""The reference arm of bench.py (`--impl reference`): the CPU restatement of
the reference's path timed on the host, one JSON line on rank 0 with the
bench contract's keys, nothing on the other ranks.  Runs on the CPU."""

from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env: dict | None = None) -> subprocess.CompletedProcess:
    env = dict(os.environ)
    env.update(extra_env or {})
    # --paths keeps the CPU suite short; the driver's runs price the full 1,048,576 paths per step
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "1", "--paths", "8192"], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_line():
    proc = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [x for x in proc.stdout.splitlines() if x.strip().startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    import bench

    assert line["impl"] == "reference"
    assert line["metric"] == "path-steps/s" and line["unit"] == "path-steps/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1 and line["config"]["paths"] == 8192
    assert line["config"]["workload"] == bench.WORKLOAD
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["unit"] == line["unit"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    proc = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert proc.returncode == 0, proc.stderr[-2000:]
    assert not [x for x in proc.stdout.splitlines() if x.strip().startswith("{")]


def test_reference_arm_loads_no_cuda_library():
    """The reference arm runs the CPU path only: the CUDA library is never mapped."""

    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', "
            "'--paths', '2048']; sys.path.insert(0, %r); import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print('CUDA_LIB_MAPPED' if 'libmontepath_cuda' in maps else 'CUDA_LIB_ABSENT'); "
            "print('ORACLE_MAPPED' if 'libmp_oracle' in maps else 'ORACLE_ABSENT')") % ROOT
    proc = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=dict(os.environ, RANK="0", WORLD_SIZE="1"),
                          capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    assert "CUDA_LIB_ABSENT" in proc.stdout and "ORACLE_MAPPED" in proc.stdout
