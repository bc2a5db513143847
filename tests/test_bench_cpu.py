"""bench.py on the CPU: the rank launcher and the CPU-baseline arithmetic.

``bench.py --gpus N`` started without a launcher starts N ranks itself
(torch.distributed.run on 127.0.0.1, one per GPU).  The reference arm runs
on the host only, so it exercises that path here: two ranks start, rank 0
times the CPU implementation and prints the one JSON line with n_gpus 2,
rank 1 exits without work.
"""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_gpus_flag_starts_its_own_ranks():
    cmd = [sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--impl", "reference", "--steps", "1",
           "--warmup", "0", "--config", "acoustic", "--nt", "60"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["cpu_baseline"]["cores"] >= 1


def test_per_shot_seconds_separates_setup_from_steps():
    import bench
    short = [{"secs": 2.0 + 4 * 0.5, "nt_sample": 4, "nt": 1000, "cells": 10, "migrates_per_shot": 2}]
    long = [{"secs": 2.0 + 16 * 0.5, "nt_sample": 16, "nt": 1000, "cells": 10, "migrates_per_shot": 2}]
    est = bench.per_shot_seconds(short, long)
    assert abs(est["per_step_s"] - 0.5) < 1e-12 and abs(est["setup_s"] - 2.0) < 1e-12
    assert abs(est["per_shot_s"] - 2 * (2.0 + 0.5 * 1000)) < 1e-9


def test_step_shots_cycle_through_the_job_and_split_over_ranks():
    import bench
    from types import SimpleNamespace
    args = SimpleNamespace(shots=4, config="visco")
    seen = [bench.step_shots(args, 64, 2, r, k) for k in range(8) for r in range(2)]
    flat = [i for s in seen for i in s]
    assert sorted(flat) == list(range(64))          # 8 steps x 2 ranks x 4 shots cover the job once
    assert bench.step_shots(args, 64, 2, 0, 8) == [0, 1, 2, 3]   # then wrap around
