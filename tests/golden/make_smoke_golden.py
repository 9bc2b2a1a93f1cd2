"""Generate tests/golden/smoke_golden.json (+ smoke_fields.npz): the reference's
own command-line program (oracle/_ref/pearl_serial) run to completion on the
key-values of its start-up check input (tests/cli_inputs.py case_smoke, the
values of examples/fe_c_phase_diagram_10K_smoke.in).  Records the status
files, diagnostics.csv and the final checkpoint fields.  About a minute on one
core.

    python tests/golden/make_smoke_golden.py
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import cli_inputs  # noqa: E402
from make_cli_golden import read_container  # noqa: E402
from oracle.build_oracle import REF_CLI, build_reference  # noqa: E402


def main() -> None:
    if not build_reference():
        raise SystemExit("reference source not available")
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        inp = cli_inputs.write_input(tmp / "smoke.in", cli_inputs.case_smoke())
        out = tmp / "smoke_out"
        p = subprocess.run([str(REF_CLI), str(inp), str(out)], capture_output=True, text=True, timeout=1800)
        assert p.returncode == 0, p.stderr
        golden = {
            "files": sorted(x.name for x in out.iterdir()),
            "completed": (out / "COMPLETED.txt").read_text(),
            "diagnostics": (out / "diagnostics.csv").read_text(),
            "initialization_report": (out / "initialization_report.txt").read_text(),
        }
        fields = read_container(out / "checkpoint.h5")
    (HERE / "smoke_golden.json").write_text(json.dumps(golden, indent=1) + "\n")
    np.savez_compressed(HERE / "smoke_fields.npz", **fields)


if __name__ == "__main__":
    main()
