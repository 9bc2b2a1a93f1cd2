"""The microsim initial phases on the device (pearl_gpu_fill: filling_phase_at,
pearl_serial.cpp:1393-1514, for every cell) against the labels the reference's
own program paints (tests/golden/make_fill_golden.py, from its
init_sharp.h5): every filling method, rotated arms and ellipses, command
sequences, bit for bit, including the reference's G137 sharp label counts
2520/357/31373 (VALIDATION_READABILITY_20260920_HISTORICAL.md:34).  The
pearl_gpu executable paints its microsim inputs this way; its init_sharp.h5
must hold the same labels.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import cli_inputs

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden():
    return np.load(GOLDEN / "fill_golden.npz")


def _labels(phi: np.ndarray) -> np.ndarray:
    assert np.all((phi == 0.0) | (phi == 1.0)) and np.all(phi.sum(axis=-1) == 1.0)
    return phi.argmax(axis=-1).astype(np.uint8)


@pytest.mark.parametrize("name", sorted(cli_inputs.FILL_CASES))
def test_fill_matches_reference_labels(gpu_lib, name):
    import pearl_gpu
    from pearl_gpu import workloads

    nx, ny = 137, 250
    params = workloads.make_params(nx, ny, 2.79e-9, 10.0, 4e-12)
    cmds = [(m, cli_inputs.fill_params(v)) for m, v in cli_inputs.FILL_CASES[name]]
    with pearl_gpu.Context(params, nx, ny) as ctx:
        z = np.zeros((ny, nx))
        ctx.upload(np.zeros((ny, nx, 3)), z, z)
        ctx.fill(cmds)
        phi = ctx.download()[0]
    got = _labels(phi)
    want = _golden()[name]
    assert np.array_equal(got, want), f"{int((got != want).sum())} cells differ"
    if name == "cube_g137":
        assert np.bincount(got.ravel(), minlength=3).tolist() == [2520, 357, 31373]


def test_fill_rejects_unknown_method(gpu_lib):
    import ctypes as C

    import pearl_gpu
    from pearl_gpu import workloads

    params = workloads.make_params(16, 16, 2e-9, 10.0, 4e-12)
    with pearl_gpu.Context(params, 16, 16) as ctx:
        op = pearl_gpu.PearlFillOp.make("FILLCUBE", [1, 0, 0, 0, 3, 3, 0])
        op.method = 99
        assert gpu_lib.pearl_gpu_fill(ctx.h, C.byref(op), 1) == 1  # PEARL_ERR_INVALID_ARGUMENT
        op.method = 1
        op.nparams = 6
        assert gpu_lib.pearl_gpu_fill(ctx.h, C.byref(op), 1) == 1


@pytest.mark.parametrize("name", ["cube_g137", "sequence"])
def test_cli_microsim_init_sharp_matches_reference(gpu_lib, tmp_path, name):
    from golden.make_cli_golden import read_container
    from pearl_gpu import build

    inp = cli_inputs.write_input(tmp_path / f"{name}.in", cli_inputs.case_fill(name))
    out = tmp_path / "out"
    subprocess.run([str(build.CLI), str(inp), str(out), "--max-steps", "1"], capture_output=True, text=True,
                   timeout=600)
    f = read_container(out / "init_sharp.h5")
    phi = np.stack([f["alpha"], f["theta"], f["gamma"]], axis=-1)
    assert np.array_equal(_labels(phi), _golden()[name])
