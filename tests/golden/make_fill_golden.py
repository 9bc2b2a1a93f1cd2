"""Generate tests/golden/fill_golden.npz: the initial phase labels that the
reference's own program (oracle/_ref/pearl_serial) paints for every case of
tests/cli_inputs.py FILL_CASES (microsim initialization on 137x250), read
from its init_sharp.h5 (the one-hot phase fields before smoothing) as labels
0 alpha, 1 theta, 2 gamma.  A few seconds on one core.

    python tests/golden/make_fill_golden.py
"""
from __future__ import annotations

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


def labels_of(fields: dict) -> np.ndarray:
    """One-hot phase fields -> labels; asserts they are exactly one-hot."""
    stack = np.stack([fields["alpha"], fields["theta"], fields["gamma"]], axis=-1)
    assert np.all((stack == 0.0) | (stack == 1.0)) and np.all(stack.sum(axis=-1) == 1.0)
    return stack.argmax(axis=-1).astype(np.uint8)


def main() -> None:
    if not build_reference():
        raise SystemExit("reference source not available")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        for name in cli_inputs.FILL_CASES:
            inp = cli_inputs.write_input(tmp / f"{name}.in", cli_inputs.case_fill(name))
            o = tmp / f"{name}_out"
            subprocess.run([str(REF_CLI), str(inp), str(o), "--max-steps", "1"], capture_output=True, text=True,
                           timeout=600)
            sharp = o / "init_sharp.h5"
            assert sharp.exists(), f"{name}: the reference wrote no init_sharp.h5"
            out[name] = labels_of(read_container(sharp))
    np.savez_compressed(HERE / "fill_golden.npz", **out)
    for name, lab in out.items():
        print(name, np.bincount(lab.ravel(), minlength=3).tolist())


if __name__ == "__main__":
    main()
