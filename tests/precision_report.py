"""Per-field error of the mixed-precision form against the FP64 GPU path and,
optionally, the FP64 CPU oracle, after N steps of the same workload (a test
helper: it runs the oracle, so it lives with the tests, not in the package).

    python tests/precision_report.py --small --steps 20000 --oracle
    python tests/precision_report.py --nx 4096 --ny 8192 --pairs 128 --steps 20000

--small uses the 128x256 fixed-dt workload (10 K, 4 pairs); otherwise the large
adaptive workload (20 K, seeded spacing and front jitter) at the given size.
The FP64 GPU run records its accepted dt sequence; the mixed run and the
oracle replay it, so all fields are compared at the same times.  Prints one
JSON line: max and rms differences of phi, mu and carbon, total carbon, and
whether each replay followed the sequence."""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
for _p in (str(ROOT), str(ROOT / "fe-c_eutectoid_phase-field_simulation_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def _err(a, b):
    d = a - b
    return {"max": float(np.abs(d).max()), "rms": float(np.sqrt(np.mean(d * d)))}


def _gpu(w, precision, steps, replay=None):
    """Runs `steps` steps; records the accepted dt sequence, or replays `replay`."""
    import pearl_gpu

    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.set_precision(precision)
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        ctx.set_history(steps)
        t0 = time.perf_counter()
        if replay is not None:
            ctx.run_replay(replay)
        else:
            done = 0
            while done < steps:
                done += ctx.run(min(1000, steps - done)).steps
        secs = time.perf_counter() - t0
        hist, _ = ctx.history()
        return ctx.download(), secs, np.array([h.accepted_dt for h in hist])


def main(argv=None) -> int:
    from pearl_gpu import workloads

    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--pairs", type=int, default=0)
    ap.add_argument("--small", action="store_true")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--oracle", action="store_true")
    args = ap.parse_args(argv)
    if args.small:
        w = workloads.plain_small()
    else:
        w = workloads.plain_large(nx=args.nx, ny=args.ny, pairs=args.pairs or max(1, args.nx // 32))
    (p64, c64, mu64, s64), t64, dts = _gpu(w, "fp64", args.steps)
    # the mixed run replays the FP64 run's accepted dt sequence, so both end at the same time
    (pmx, cmx, mumx, smx), tmx, dts_mx = _gpu(w, "mixed", args.steps, replay=dts)
    out = {"workload": w.name, "steps": args.steps,
           "fp64_gpu": {"time": s64.time, "rejected": s64.rejected, "seconds": t64},
           "mixed_gpu_replay": {"time": smx.time, "rejected": smx.rejected, "seconds": tmx,
                                "followed_dt_sequence": bool(np.array_equal(dts, dts_mx))},
           "mixed_vs_fp64_gpu": {"phi": _err(pmx, p64), "mu": _err(mumx, mu64), "carbon": _err(cmx, c64),
                                 "total_carbon_rel": abs(cmx.sum() - c64.sum()) / abs(c64.sum())}}
    if args.oracle:
        from oracle import pyoracle

        port = pyoracle.port()
        po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        so = pyoracle.scalars_from(w.scalars)
        t0 = time.perf_counter()
        rc, why, done, _ = port.advance_n(w.params, po, co, muo, so, args.steps, forced_dt=dts)
        out["oracle"] = {"rc": rc, "steps": done, "time": so.time, "rejected": so.rejected,
                         "seconds": time.perf_counter() - t0}
        out["mixed_vs_oracle"] = {"phi": _err(pmx, po), "mu": _err(mumx, muo), "carbon": _err(cmx, co)}
        out["fp64_vs_oracle"] = {"phi": _err(p64, po), "mu": _err(mu64, muo), "carbon": _err(c64, co)}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
