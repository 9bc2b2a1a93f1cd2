"""Generate tests/golden/horizon_golden.json (+ horizon_fields.npz): the
reference solver itself (oracle/_ref/libpearl_ref.so, the unmodified
pearl_serial.cpp behind ref_harness.cpp) run over the small FP64 workload
(pearl_gpu.workloads.plain_small: 128x256, 4 pairs, 10 K, fixed dt = dt_max =
4e-12 s) for 20000 accepted steps, ten times its configured 2000.  Records
every step's retries, accepted dt and CG count, and the fields after 2000 and
after 20000 steps (horizon_fields.npz; the json holds the totals).  About four minutes on one core.

    python tests/golden/make_horizon_golden.py
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (str(ROOT), str(ROOT / "fe-c_eutectoid_phase-field_simulation_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import pyoracle  # noqa: E402
from pearl_gpu import workloads  # noqa: E402

STEPS = 20000
CHECKPOINTS = (2000, 20000)


def main() -> None:
    ref = pyoracle.reference()
    if ref is None:
        raise SystemExit("reference source not available")
    w = workloads.plain_small()
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    fields, record, done_total = {}, {"retries": [], "accepted_dt": [], "cg_iterations": []}, 0
    t0 = time.time()
    for stop in CHECKPOINTS:
        rc, err, done, infos = ref.advance_n(w.params, phi, c, mu, s, stop - done_total)
        assert rc == 0 and done == stop - done_total, err
        done_total = stop
        for i in infos:
            record["retries"].append(int(i.retries))
            record["accepted_dt"].append(float(i.accepted_dt))
            record["cg_iterations"].append(int(i.cg_iterations))
        fields[f"s{stop}/phi"] = phi.copy()
        fields[f"s{stop}/carbon"] = c.copy()
        fields[f"s{stop}/mu"] = mu.copy()
        fields[f"s{stop}/scalars"] = np.array([s.time, s.dt, float(s.step), float(s.rejected)])
    golden = {"workload": w.name, "steps": STEPS, "checkpoints": list(CHECKPOINTS),
              "seconds": time.time() - t0, "rejected": int(sum(record["retries"])),
              "cg_iterations": int(sum(record["cg_iterations"]))}
    (HERE / "horizon_golden.json").write_text(json.dumps(golden, indent=1) + "\n")
    fields["steps/retries"] = np.array(record["retries"], dtype=np.int32)
    fields["steps/accepted_dt"] = np.array(record["accepted_dt"], dtype=np.float64)
    fields["steps/cg_iterations"] = np.array(record["cg_iterations"], dtype=np.int32)
    np.savez_compressed(HERE / "horizon_fields.npz", **fields)


if __name__ == "__main__":
    main()
