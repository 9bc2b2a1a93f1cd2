"""Host logic of bench.py: replica aggregation across ranks (gloo, 2 processes
on the CPU) and the JSON contract of the reference arm on a tiny domain."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _worker(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r processed (r+1)*1000 cells in (r+1) seconds
        value, t_max = bench.replica_throughput(dist, 1000.0 * (rank + 1), float(rank + 1), "cpu")
        out.put((rank, value, t_max))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, value, t_max in results:
        assert t_max == 2.0
        assert value == 3000.0 / 2.0


def test_reference_arm_json_contract():
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--nx", "64", "--ny", "64",
                        "--steps", "2", "--warmup", "1", "--ref-seconds", "0.5"], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] == 1


def test_phase_hbm_fracs():
    """Per-phase fractions from the phase clock: the numbers of a measured
    2048x4096 line (100 steps, 114 attempts, 484 CG passes)."""
    sys.path.insert(0, str(ROOT))
    import bench

    ms = {"propose": 35.553, "setup": 17.785, "apply": 47.882, "update": 41.305, "final": 32.653}
    n = {"propose": 114, "setup": 114, "apply": 484, "update": 484, "final": 114}
    f = bench.phase_hbm_fracs(ms, n, 2048 * 4096, 6551.0)
    assert set(f) == set(ms)
    # UPDATE: 64 B x 8.39 M cells x 484 passes in 41.3 ms
    assert f["update"] == pytest.approx(64 * 2048 * 4096 * 484 / 41.305e-3 / 1e9 / 6551.0, rel=1e-3)
    # APPLY: 114 first passes of 48 B, 370 of 56 B
    assert f["apply"] == pytest.approx((114 * 48 + 370 * 56) * 2048 * 4096 / 47.882e-3 / 1e9 / 6551.0, rel=1e-3)
    assert 0.9 < f["update"] < 1.0 and 0.6 < f["apply"] < 0.8
    assert bench.phase_hbm_fracs({}, {}, 1, 1.0) == {}
