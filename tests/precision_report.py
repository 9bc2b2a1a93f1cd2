"""Per-field error of the mixed-precision form against the FP64 GPU path and,
optionally, the FP64 CPU oracle, after N steps of the same workload (a test
helper: it runs the oracle, so it lives with the tests, not in the package).

    python tests/precision_report.py --small --steps 20000 --oracle
    python tests/precision_report.py --nx 4096 --ny 8192 --pairs 128 --steps 20000

--small uses the 128x256 fixed-dt workload (10 K, 4 pairs); otherwise the large
adaptive workload (20 K, seeded spacing and front jitter) at the given size.
The FP64 GPU run takes N steps and sets the end time; every mixed form (and
the oracle) runs to exactly that time, its last step clipped to it as the
reference clips a step to an output time, so all fields are compared at the
same physical time whatever dt sequence each form chose.  Prints one JSON
line: per form its steps, rejections, CG iterations and seconds, and max and
rms differences of phi, mu and carbon and the total carbon against the FP64
GPU run and the oracle."""
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


def _gpu(w, precision, steps=None, stop_time=None):
    """Runs `steps` steps, or until exactly `stop_time` (the last step is clipped
    to it, as the reference clips a step to the next output time)."""
    import pearl_gpu

    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.set_precision(precision)
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        t0 = time.perf_counter()
        done, cg = 0, 0
        if stop_time is None:
            while done < steps:
                r = ctx.run(min(1000, steps - done))
                done += r.steps
                cg += r.cg_total
        else:
            while ctx.scalars().time < stop_time:
                r = ctx.run(1000, stop_time=stop_time)
                done += r.steps
                cg += r.cg_total
                if r.reached_stop:
                    break
        secs = time.perf_counter() - t0
        phi, c, mu, s = ctx.download()
        return (phi, c, mu, s), {"time": s.time, "steps": done, "rejected": s.rejected, "cg_iterations": cg,
                                 "seconds": secs}


def _fields(a, b):
    (pa, ca, ma, _), (pb, cb, mb, _) = a, b
    return {"phi": _err(pa, pb), "mu": _err(ma, mb), "carbon": _err(ca, cb),
            "total_carbon_rel": float(abs(ca.sum() - cb.sum()) / abs(cb.sum()))}


def main(argv=None) -> int:
    from pearl_gpu import workloads

    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--pairs", type=int, default=0)
    ap.add_argument("--small", action="store_true")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--forms", default="mixed,mixed_propose,mixed_solve")
    ap.add_argument("--reference-golden", action="store_true",
                    help="--small --steps 2000|20000: also compare with the reference's own run at that step "
                         "(tests/golden/horizon_fields.npz), which ends at the FP64 run's time")
    args = ap.parse_args(argv)
    if args.small:
        w = workloads.plain_small()
    else:
        w = workloads.plain_large(nx=args.nx, ny=args.ny, pairs=args.pairs or max(1, args.nx // 32))
    # the FP64 run sets the end time; every other run is clipped to exactly that time,
    # so the fields are compared at the same physical time whatever dt each form took
    ref, info64 = _gpu(w, "fp64", steps=args.steps)
    end = info64["time"]
    out = {"workload": w.name, "steps": args.steps, "end_time": end, "fp64_gpu": info64}
    runs = {}
    for form in [f for f in args.forms.split(",") if f]:
        runs[form], info = _gpu(w, form, stop_time=end)
        out[f"{form}_gpu"] = info
        out[f"{form}_vs_fp64_gpu"] = _fields(runs[form], ref)
    if args.oracle:
        from oracle import pyoracle

        port = pyoracle.port()
        po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        so = pyoracle.scalars_from(w.scalars)
        t0 = time.perf_counter()
        # run to the end time: the step that would pass it is clipped, the one after finds no time left
        rc, why, done, _ = port.advance_n(w.params, po, co, muo, so, 10 * args.steps + 100, stop_time=end)
        out["oracle"] = {"rc": rc, "steps": done, "time": so.time, "rejected": so.rejected,
                         "seconds": time.perf_counter() - t0}
        orc = (po, co, muo, so)
        out["fp64_vs_oracle"] = _fields(ref, orc)
        for form, r in runs.items():
            out[f"{form}_vs_oracle"] = _fields(r, orc)
    if args.reference_golden:
        ref_f = np.load(ROOT / "tests" / "golden" / "horizon_fields.npz")
        k = f"s{args.steps}"
        assert args.small and f"{k}/phi" in ref_f.files, "the golden holds the small workload at 2000 and 20000 steps"
        assert float(ref_f[f"{k}/scalars"][0]) == end, "the reference's run ends at another time"
        golden = (ref_f[f"{k}/phi"], ref_f[f"{k}/carbon"], ref_f[f"{k}/mu"], None)
        out["fp64_vs_reference"] = _fields(ref, golden)
        for form, r in runs.items():
            out[f"{form}_vs_reference"] = _fields(r, golden)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
