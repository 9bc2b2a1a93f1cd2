"""Generate tests/golden/examples_golden.json (+ examples_fields.npz): every
example input shipped with the reference (examples/*.in, examples/legacy_direct/*.in),
run by the reference's own program (oracle/_ref/pearl_serial) for 300 steps.
Records each input's key-value lines (comments dropped), the status file,
diagnostics.csv and the final checkpoint fields.

    python tests/golden/make_examples_golden.py
    python tests/golden/make_examples_golden.py --write-input NAME PATH   # one stored input back to a file
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
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))

from make_cli_golden import read_container  # noqa: E402
from oracle.build_oracle import REF_CLI, build_reference, reference_dir  # noqa: E402

STEPS = 300


def key_values(text: str) -> list[list[str]]:
    """The input's entries in file order, without comments or blank lines."""
    out = []
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        if "=" in line:
            k, v = line.split("=", 1)
            out.append([k.strip(), v.strip()])
        else:
            out.append([line, None])
    return out


def main() -> None:
    if not build_reference():
        raise SystemExit("reference source not available")
    ex = reference_dir() / "examples"
    files = sorted(ex.glob("*.in")) + sorted((ex / "legacy_direct").glob("*.in"))
    golden, fields = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        for f in files:
            name = f.stem
            kv = key_values(f.read_text())
            inp = tmp / f"{name}.in"
            inp.write_text("\n".join(k if v is None else f"{k} = {v}" for k, v in kv) + "\n")
            out = tmp / f"{name}_out"
            p = subprocess.run([str(REF_CLI), str(inp), str(out), "--max-steps", str(STEPS)], capture_output=True,
                               text=True, timeout=1800)
            entry = {"input": kv, "rc": p.returncode, "stderr": p.stderr}
            if p.returncode == 0:
                status = "COMPLETED.txt" if (out / "COMPLETED.txt").exists() else "STOPPED.txt"
                entry.update(files=sorted(x.name for x in out.iterdir()), status_file=status,
                             status=(out / status).read_text(), diagnostics=(out / "diagnostics.csv").read_text())
                for k, v in read_container(out / "checkpoint.h5").items():
                    fields[f"{name}/{k}"] = v
            golden[name] = entry
            print(name, p.returncode, flush=True)
    (HERE / "examples_golden.json").write_text(json.dumps(golden, indent=1) + "\n")
    np.savez_compressed(HERE / "examples_fields.npz", **fields)


def write_input(name: str, path: str) -> None:
    """Writes the stored key-values of example `name` as an input file."""
    kv = json.loads((HERE / "examples_golden.json").read_text())[name]["input"]
    Path(path).write_text("\n".join(k if v is None else f"{k} = {v}" for k, v in kv) + "\n")


if __name__ == "__main__":
    if len(sys.argv) == 4 and sys.argv[1] == "--write-input":
        write_input(sys.argv[2], sys.argv[3])
    else:
        main()
