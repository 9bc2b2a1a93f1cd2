"""Generate tests/golden/cli_golden.json (+ cli_fields.npz) from the reference's
own command-line program (oracle/_ref/pearl_serial, the unmodified
pearl_serial.cpp built against the HDF5 stand-in).

For every input of tests/cli_inputs.py it records the exit code, the stderr
text and thermodynamics.txt of a --thermo-only run; for the valid inputs it
also records a short real run: diagnostics.csv, initialization_report.txt,
the final status file and the checkpoint fields.

    python tests/golden/make_cli_golden.py
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

import cli_inputs  # noqa: E402
from oracle.build_oracle import REF_CLI, build_reference  # noqa: E402

RUN_STEPS = {"sharp_smooth": 40, "lamella_linear_gp": 30, "direct_flat_mean": 30, "microsim": 30,
             "moving_window": 400}


def read_container(path: Path) -> dict:
    """Datasets of a stand-in HDF5 container (the format written by both programs)."""
    out = {}
    with open(path, "rb") as f:
        assert f.readline().startswith(b"PEARL-H5-STUB 1")
        while True:
            line = f.readline()
            if not line or line.startswith(b"END"):
                break
            parts = line.split()
            if parts[0] == b"D":
                ny, nx = int(parts[2]), int(parts[3])
                out[parts[1].decode()] = np.frombuffer(f.read(8 * ny * nx), dtype="<f8").reshape(ny, nx).copy()
                f.read(1)
            elif parts[0] == b"A" and parts[2] == b"s":
                f.read(int(parts[3]) + 1)
    return out


def run(binary: Path, lines, args, workdir: Path, name: str):
    inp = cli_inputs.write_input(workdir / f"{name}.in", lines)
    out = workdir / f"{name}_out"
    p = subprocess.run([str(binary), str(inp), str(out), *args], capture_output=True, text=True, timeout=900)
    return p, out


def main() -> None:
    if not build_reference() or not REF_CLI.exists():
        raise SystemExit("the reference program is not available here")
    golden = {"thermo_only": {}, "runs": {}}
    fields = {}
    with tempfile.TemporaryDirectory() as tmp:
        work = Path(tmp)
        cases = {**{k: f() for k, f in cli_inputs.VALID.items()}, **cli_inputs.invalid_cases()}
        for name, lines in cases.items():
            p, out = run(REF_CLI, lines, ["--thermo-only"], work, "t_" + name)
            rec = {"rc": p.returncode, "stderr": p.stderr, "stdout": p.stdout}
            thermo = out / "thermodynamics.txt"
            rec["thermodynamics"] = thermo.read_text() if thermo.exists() else None
            golden["thermo_only"][name] = rec
        for name, make in cli_inputs.VALID.items():
            p, out = run(REF_CLI, make(), ["--max-steps", str(RUN_STEPS[name])], work, "r_" + name)
            assert p.returncode == 0, p.stderr
            status = "STOPPED.txt" if (out / "STOPPED.txt").exists() else "COMPLETED.txt"
            golden["runs"][name] = {
                "steps": RUN_STEPS[name],
                "diagnostics": (out / "diagnostics.csv").read_text(),
                "initialization_report": (out / "initialization_report.txt").read_text(),
                "status_file": status,
                "status": (out / status).read_text(),
                "files": sorted(x.name for x in out.iterdir()),
            }
            for k, v in read_container(out / "checkpoint.h5").items():
                fields[f"{name}/{k}"] = v
    (HERE / "cli_golden.json").write_text(json.dumps(golden, indent=1) + "\n")
    np.savez_compressed(HERE / "cli_fields.npz", **fields)
    print("ok", len(golden["thermo_only"]), "thermo-only cases,", len(golden["runs"]), "runs")


if __name__ == "__main__":
    main()
