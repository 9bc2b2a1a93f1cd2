"""The pearl_gpu executable against the reference's own command-line program.

Golden outputs (tests/golden/cli_golden.json, cli_fields.npz) were written by
the unmodified reference (make_cli_golden.py).  On the CPU, --thermo-only runs
compare input parsing, temperature laws, error messages and the
thermodynamics report byte for byte.  On the GPU, short real runs compare the
output files, diagnostics.csv and the checkpoint fields within the FP64
tolerances (phi 1e-10, mu 1e-5 J/mol, total carbon 1e-12 relative).
"""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

import cli_inputs

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def golden():
    return json.loads((GOLDEN / "cli_golden.json").read_text())


@pytest.fixture(scope="module")
def cli(gpu_lib):
    from pearl_gpu import build

    return build.CLI


ALL_CASES = {**{k: f() for k, f in cli_inputs.VALID.items()}, **cli_inputs.invalid_cases()}


def _run(cli, lines, args, tmp_path, name):
    inp = cli_inputs.write_input(tmp_path / f"{name}.in", lines)
    out = tmp_path / f"{name}_out"
    p = subprocess.run([str(cli), str(inp), str(out), *args], capture_output=True, text=True, timeout=600)
    return p, out


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_thermo_only_matches_reference(cli, golden, tmp_path, name):
    ref = golden["thermo_only"][name]
    p, out = _run(cli, ALL_CASES[name], ["--thermo-only"], tmp_path, name)
    assert p.returncode == ref["rc"]
    assert p.stderr == ref["stderr"]
    assert p.stdout == ref["stdout"]
    thermo = out / "thermodynamics.txt"
    assert (thermo.read_text() if thermo.exists() else None) == ref["thermodynamics"]


def test_cli_usage_errors(cli, tmp_path):
    p = subprocess.run([str(cli)], capture_output=True, text=True)
    assert p.returncode == 1 and p.stderr.startswith("ERROR: Usage: pearl input.in NEW_OUTPUT_DIR")
    inp = cli_inputs.write_input(tmp_path / "a.in", cli_inputs.case_sharp_smooth())
    p = subprocess.run([str(cli), str(inp), str(tmp_path / "o"), "--px", "2"], capture_output=True, text=True)
    assert p.stderr == "ERROR: serial build requires px=py=1\n"
    p = subprocess.run([str(cli), str(inp), str(tmp_path / "o"), "--max-steps", "0"], capture_output=True, text=True)
    assert p.stderr == "ERROR: max-steps must be positive\n"
    p = subprocess.run([str(cli), str(inp), str(tmp_path / "o"), "--thermo-only", "--restart", "x.h5"],
                       capture_output=True, text=True)
    assert p.stderr == "ERROR: --thermo-only cannot be combined with --restart\n"
    (tmp_path / "exists").mkdir()
    p = subprocess.run([str(cli), str(inp), str(tmp_path / "exists"), "--thermo-only"], capture_output=True, text=True)
    assert p.stderr == "ERROR: cannot create NEW output directory\n"


def _csv(text):
    lines = text.strip().splitlines()
    head = lines[0].split(",")
    rows = [dict(zip(head, map(float, ln.split(",")))) for ln in lines[1:]]
    return head, rows


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(cli_inputs.VALID))
def test_cli_run_matches_reference(cli, golden, tmp_path, name):
    from golden.make_cli_golden import read_container

    ref = golden["runs"][name]
    p, out = _run(cli, cli_inputs.VALID[name](), ["--max-steps", str(ref["steps"])], tmp_path, name)
    assert p.returncode == 0, p.stderr
    assert sorted(x.name for x in out.iterdir()) == ref["files"]
    assert (out / ref["status_file"]).read_text() == ref["status"]
    head, rows = _csv((out / "diagnostics.csv").read_text())
    rhead, rrows = _csv(ref["diagnostics"])
    assert head == rhead and len(rows) == len(rrows)
    kv = dict(cli_inputs.VALID[name]())
    area = int(kv["nx"]) * int(kv["ny"]) * float(kv["dx"]) ** 2
    for r, g in zip(rows, rrows):
        for k in ("time", "step", "dt_next", "cg_last", "cg_peak", "rejected", "shift_distance"):
            assert r[k] == g[k], k
        assert r["mean_carbon"] == pytest.approx(g["mean_carbon"], rel=1e-13)
        # the ledger is rounding noise of the total carbon: compare on that scale
        total = g["mean_carbon"] * area
        assert abs(r["mass_ledger_error"] - g["mass_ledger_error"]) <= 1e-13 * total
        assert r["reduced_energy"] == pytest.approx(g["reduced_energy"], rel=1e-10)
        assert abs(r["phi_sum_error"] - g["phi_sum_error"]) <= 1e-15
        for k in ("c_min", "c_max"):
            assert abs(r[k] - g[k]) <= 1e-12, k
        for k in ("mu_min", "mu_max"):
            assert abs(r[k] - g[k]) <= 1e-5, k
        assert abs(r["closure_last"] - g["closure_last"]) <= 1e-13
    fields = read_container(out / "checkpoint.h5")
    ref_fields = np.load(GOLDEN / "cli_fields.npz")
    for a in ("alpha", "theta", "gamma"):
        assert np.abs(fields[a] - ref_fields[f"{name}/{a}"]).max() <= 1e-10
    assert np.abs(fields["mu"] - ref_fields[f"{name}/mu"]).max() <= 1e-5
    c, c_ref = fields["carbon"], ref_fields[f"{name}/carbon"]
    assert abs(c.sum() - c_ref.sum()) <= 1e-12 * abs(c_ref.sum())
    rep = dict(ln.split("=", 1) for ln in (out / "initialization_report.txt").read_text().splitlines())
    rep_ref = dict(ln.split("=", 1) for ln in ref["initialization_report"].splitlines())
    for k in ("initialization", "smooth_steps_completed", "smooth_energy_converged", "mu_reference", "NOTE"):
        assert rep[k] == rep_ref[k], k
    for k in ("smooth_energy_initial", "smooth_energy_final", "smooth_final_max_phase_change"):
        assert float(rep[k]) == pytest.approx(float(rep_ref[k]), rel=1e-10), k


@pytest.mark.gpu
def test_cli_restart_from_reference_checkpoint(cli, tmp_path):
    """A checkpoint written by the reference program restarts in pearl_gpu and
    continues like the reference (restart equivalence, VALIDATION.md:33-35)."""
    from oracle.build_oracle import REF_CLI

    if not REF_CLI.exists():
        pytest.skip("reference program not built on this host")
    lines = cli_inputs.case_lamella_linear_gp()
    inp = cli_inputs.write_input(tmp_path / "a.in", lines)
    first = tmp_path / "first"
    p = subprocess.run([str(REF_CLI), str(inp), str(first), "--max-steps", "10"], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    outs = {}
    for tag, binary in (("ref", REF_CLI), ("gpu", cli)):
        o = tmp_path / f"cont_{tag}"
        p = subprocess.run([str(binary), str(inp), str(o), "--restart", str(first / "checkpoint.h5"),
                            "--max-steps", "10"], capture_output=True, text=True)
        assert p.returncode == 0, p.stderr
        outs[tag] = o
    from golden.make_cli_golden import read_container

    a, b = read_container(outs["gpu"] / "checkpoint.h5"), read_container(outs["ref"] / "checkpoint.h5")
    assert np.abs(a["alpha"] - b["alpha"]).max() <= 1e-10
    assert np.abs(a["mu"] - b["mu"]).max() <= 1e-5


@pytest.mark.gpu
def test_cli_smoke_run_matches_reference(cli, tmp_path):
    """Known answer: the reference's start-up check (137x250, sharp_smooth, to
    0.015 microseconds, ~5,500 adaptive steps with ~750 rejections), run by the
    reference program here (make_smoke_golden.py), is reproduced step for step:
    same accepted steps, rejections and total CG iterations, final fields within
    the FP64 tolerances."""
    from golden.make_cli_golden import read_container

    ref = json.loads((GOLDEN / "smoke_golden.json").read_text())
    p, out = _run(cli, cli_inputs.case_smoke(), [], tmp_path, "smoke")
    assert p.returncode == 0, p.stderr
    # the frames are not HDF5: the run says so once
    assert p.stdout.count("written in the PEARL-H5-STUB container, not HDF5") == 1
    assert sorted(x.name for x in out.iterdir()) == ref["files"]
    assert (out / "COMPLETED.txt").read_text() == ref["completed"]
    head, rows = _csv((out / "diagnostics.csv").read_text())
    rhead, rrows = _csv(ref["diagnostics"])
    assert head == rhead and len(rows) == len(rrows)
    for r, g in zip(rows, rrows):
        for k in ("time", "step", "dt_next", "cg_last", "cg_peak", "rejected"):
            assert r[k] == g[k], k
        for k in ("mu_min", "mu_max"):
            assert abs(r[k] - g[k]) <= 1e-5, k
    fields = read_container(out / "checkpoint.h5")
    ref_fields = np.load(GOLDEN / "smoke_fields.npz")
    for a in ("alpha", "theta", "gamma"):
        assert np.abs(fields[a] - ref_fields[a]).max() <= 1e-10
    assert np.abs(fields["mu"] - ref_fields["mu"]).max() <= 1e-5
    c, c_ref = fields["carbon"], ref_fields["carbon"]
    assert abs(c.sum() - c_ref.sum()) <= 1e-12 * abs(c_ref.sum())


@pytest.mark.gpu
def test_cli_stop_restart_is_bitwise(cli, tmp_path):
    """Restart equivalence (VALIDATION.md:33-35): 12 steps, then a restart from
    that checkpoint for 12 more, equal an uninterrupted 24-step run bitwise."""
    from golden.make_cli_golden import read_container

    lines = cli_inputs.case_lamella_linear_gp()
    inp = cli_inputs.write_input(tmp_path / "a.in", lines)

    def run(out, *args):
        p = subprocess.run([str(cli), str(inp), str(tmp_path / out), *args], capture_output=True, text=True)
        assert p.returncode == 0, p.stderr
        return tmp_path / out

    whole = run("whole", "--max-steps", "24")
    first = run("first", "--max-steps", "12")
    second = run("second", "--restart", str(first / "checkpoint.h5"), "--max-steps", "12")
    a, b = read_container(whole / "checkpoint.h5"), read_container(second / "checkpoint.h5")
    assert sorted(a) == sorted(b)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    wa, wb = (whole / "STOPPED.txt").read_text().splitlines(), (second / "STOPPED.txt").read_text().splitlines()
    for k in (1, 2, 4):  # time, step, rejected (CG_total counts the run's own iterations)
        assert wa[k] == wb[k]


EXAMPLES = json.loads((GOLDEN / "examples_golden.json").read_text()) if (GOLDEN / "examples_golden.json").exists() else {}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(EXAMPLES))
def test_cli_reference_examples(cli, tmp_path, name):
    """Every example input shipped with the reference, 300 steps, against the
    reference program's own run (make_examples_golden.py): same files, status
    and step decisions; fields within the FP64 tolerances."""
    from golden.make_cli_golden import read_container

    ref = EXAMPLES[name]
    lines = [(k, v) for k, v in ref["input"]]
    p, out = _run(cli, lines, ["--max-steps", "300"], tmp_path, name)
    assert p.returncode == ref["rc"]
    assert p.stderr == ref["stderr"]
    if ref["rc"]:
        return
    assert sorted(x.name for x in out.iterdir()) == ref["files"]
    assert (out / ref["status_file"]).read_text() == ref["status"]
    head, rows = _csv((out / "diagnostics.csv").read_text())
    rhead, rrows = _csv(ref["diagnostics"])
    assert head == rhead and len(rows) == len(rrows)
    for r, g in zip(rows, rrows):
        for k in ("time", "step", "dt_next", "cg_last", "cg_peak", "rejected", "shift_distance"):
            assert r[k] == g[k], k
    fields = read_container(out / "checkpoint.h5")
    ref_fields = np.load(GOLDEN / "examples_fields.npz")
    for a in ("alpha", "theta", "gamma"):
        assert np.abs(fields[a] - ref_fields[f"{name}/{a}"]).max() <= 1e-10
    assert np.abs(fields["mu"] - ref_fields[f"{name}/mu"]).max() <= 1e-5
    c, c_ref = fields["carbon"], ref_fields[f"{name}/carbon"]
    assert abs(c.sum() - c_ref.sum()) <= 1e-12 * abs(c_ref.sum())
