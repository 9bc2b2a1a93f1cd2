"""Failure detection with faults injected on the host (no fault, trap or hang
on the GPU): non-finite input fields, a CG iteration cap too small to
converge, restarts from a mismatched or damaged checkpoint, and SIGINT in the
middle of a run.  Each must end the way the reference ends it: same status
and message (pearl_serial.cpp messages), state unchanged on error, and a
restartable checkpoint after a signal."""
from __future__ import annotations

import signal
import subprocess
import time

import numpy as np
import pytest

import cli_inputs

pytestmark = pytest.mark.gpu


def _ctx(w, params=None):
    import pearl_gpu

    ctx = pearl_gpu.Context(params or w.params, w.nx, w.ny)
    ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
    return ctx


def _oracle(port, w, n, params=None):
    from oracle import pyoracle

    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc, why, done, infos = port.advance_n(params or w.params, phi, c, mu, s, n)
    return rc, why, done, s


@pytest.mark.parametrize("field", ["phi", "mu", "carbon"])
def test_non_finite_cell_ends_like_the_reference(gpu_lib, port, field):
    """One NaN cell: the reference throws (mixture check of the step-start energy,
    or every proposal rejected down to dt_min); the device reports the same
    status and leaves the state as uploaded."""
    import pearl_gpu
    from pearl_gpu import workloads

    w = workloads.scaled(64, 48, seed=2, front=12.0)
    if field == "phi":
        w.phi[20, 10, 0] = np.nan
    elif field == "mu":
        w.mu[20, 10] = np.nan
    else:
        w.carbon[20, 10] = np.nan
    rc_o, why_o, done_o, _ = _oracle(port, w, 3)
    assert rc_o != 0 and done_o == 0
    with _ctx(w) as ctx:
        with pytest.raises(pearl_gpu.PearlError) as e:
            ctx.advance()
        assert e.value.status == rc_o
        phi, c, mu, s = ctx.download()
    assert np.array_equal(phi, w.phi, equal_nan=True) and np.array_equal(mu, w.mu, equal_nan=True)
    assert np.array_equal(c, w.carbon, equal_nan=True) and s.step == 0


def test_cg_cap_of_one_iteration(gpu_lib, port):
    """cg_max = 1: the solve fails the linear/closure test until dt is small
    enough; the device takes the same rejections and steps as the reference."""
    import pearl_gpu
    from pearl_gpu import workloads

    w = workloads.scaled(48, 48, seed=4, front=12.0)
    params = dict(w.params, cg_max=1)
    n = 4
    rc_o, why_o, done_o, so = _oracle(port, w, n, params)
    with _ctx(w, params) as ctx:
        done, status = 0, 0
        try:
            for _ in range(n):
                ctx.advance()
                done += 1
        except pearl_gpu.PearlError as e:
            status = e.status
        s = ctx.scalars()
    assert status == rc_o and done == done_o
    assert s.step == so.step and s.rejected == so.rejected and s.dt == so.dt


def _write(tmp_path, name, lines):
    return cli_inputs.write_input(tmp_path / f"{name}.in", lines)


def _cli(cli, inp, out, *args, **kw):
    return subprocess.run([str(cli), str(inp), str(out), *args], capture_output=True, text=True, **kw)


@pytest.fixture(scope="module")
def cli(gpu_lib):
    from pearl_gpu import build

    return build.CLI


def test_restart_from_mismatched_or_damaged_checkpoint(cli, tmp_path):
    """pearl_serial.cpp:1978 (signature) and :1861 (unreadable file)."""
    base = cli_inputs.case_lamella_linear_gp()
    p = _cli(cli, _write(tmp_path, "a", base), tmp_path / "A", "--max-steps", "5")
    assert p.returncode == 0, p.stderr
    ck = tmp_path / "A" / "checkpoint.h5"
    other = _write(tmp_path, "b", [(k, "0.6" if k == "sigma" else v) for k, v in base])
    p = _cli(cli, other, tmp_path / "B", "--restart", str(ck), "--max-steps", "5")
    assert p.returncode == 1 and p.stderr == "ERROR: checkpoint physics signature mismatch\n"
    grid = _write(tmp_path, "g", [(k, "40" if k == "nx" else v) for k, v in base])
    p = _cli(cli, grid, tmp_path / "G", "--restart", str(ck), "--max-steps", "5")
    assert p.returncode == 1 and p.stderr == "ERROR: checkpoint physics signature mismatch\n"
    data = ck.read_bytes()
    (tmp_path / "trunc.h5").write_bytes(data[: len(data) // 2])
    a = _write(tmp_path, "a2", base)
    for bad in (tmp_path / "trunc.h5", tmp_path / "missing.h5"):
        p = _cli(cli, a, tmp_path / f"C_{bad.stem}", "--restart", str(bad), "--max-steps", "5")
        assert p.returncode == 1 and p.stderr == "ERROR: HDF5 open/create failure\n"


def test_sigint_mid_run_stops_cleanly_and_restarts(cli, tmp_path):
    """SIGINT/SIGTERM (pearl_serial.cpp:2250-2251, :2318-2321): the run stops
    between launches, writes checkpoint.h5 and STOPPED.txt, exits 0, and the
    checkpoint restarts."""
    # the start-up check run out to 1.5 us (about a minute), so the signal lands mid-run
    long_run = [(k, "1.5e-6" if k == "end_time" else v) for k, v in cli_inputs.case_smoke()]
    inp = _write(tmp_path, "long", long_run)
    proc = subprocess.Popen([str(cli), str(inp), str(tmp_path / "run")], stdout=subprocess.PIPE,
                            stderr=subprocess.PIPE, text=True)
    # wait until the evolution has started (the first frame is written after initialisation)
    t0 = time.time()
    while not (tmp_path / "run" / "frame_000000.h5").exists() and time.time() - t0 < 120:
        time.sleep(0.05)
    time.sleep(0.5)
    proc.send_signal(signal.SIGINT)
    out, err = proc.communicate(timeout=300)
    assert proc.returncode == 0, err
    status = (tmp_path / "run" / "STOPPED.txt").read_text().splitlines()
    assert status[0] == "status=USER_STOPPED"
    step = int(status[2].split("=")[1])
    assert step > 0
    p = _cli(cli, inp, tmp_path / "again", "--restart", str(tmp_path / "run" / "checkpoint.h5"), "--max-steps", "3",
             timeout=300)
    assert p.returncode == 0, p.stderr
    assert (tmp_path / "again" / "STOPPED.txt").read_text().splitlines()[2] == f"step={step + 3}"
