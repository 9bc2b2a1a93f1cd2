"""The host side of the drop-in executable (input parser, temperature laws,
thermodynamics report, error paths) built with AddressSanitizer and
UndefinedBehaviorSanitizer and run on every --thermo-only input of the CLI
tests: same output as the normal build, and no sanitizer report.  Runs on the
CPU (no device call is made on this path)."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

import cli_inputs
from test_cli import ALL_CASES

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "fe-c_eutectoid_phase-field_simulation_b200"


@pytest.fixture(scope="module")
def asan_cli(tmp_path_factory):
    from pearl_gpu import build

    if not build.LIB.exists():
        pytest.skip("libpearl_gpu.so not built")
    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    out = tmp_path_factory.mktemp("asan") / "pearl_gpu"
    host = PKG / "host"
    cmd = ["g++", "-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
           "-fno-sanitize-recover=undefined", "-ffp-contract=off", f"-I{ROOT / 'include'}", f"-I{host}",
           *[str(host / n) for n in build.CLI_SOURCES], f"-L{build.BUILD}", "-lpearl_gpu",
           f"-Wl,-rpath,{build.BUILD}", "-pthread", "-o", str(out)]
    subprocess.run(cmd, check=True, capture_output=True, timeout=600)
    return out


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_thermo_only_under_sanitizers(asan_cli, tmp_path, name):
    from pearl_gpu import build

    inp = cli_inputs.write_input(tmp_path / f"{name}.in", ALL_CASES[name])
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    a = subprocess.run([str(asan_cli), str(inp), str(tmp_path / "a"), "--thermo-only"], capture_output=True, text=True,
                       env=env, timeout=300)
    b = subprocess.run([str(build.CLI), str(inp), str(tmp_path / "b"), "--thermo-only"], capture_output=True,
                       text=True, timeout=300)
    assert "Sanitizer" not in a.stderr and "runtime error" not in a.stderr, a.stderr
    assert (a.returncode, a.stdout, a.stderr) == (b.returncode, b.stdout, b.stderr)
