"""Bit-for-bit parity with the oracle in the device's summation order.

The FP64 path evaluates every per-cell formula with the reference's own
operation order and rounding, so the only way its results may differ from the
reference's is the order of its global sums (CG dot products, carbon mass,
energy): the device sums in a fixed tree, the reference sequentially.  The
oracle's device-order mode (pearl_oracle.c, po_set_device_order) sums the
reference's per-cell values in that tree, given the context's geometry
(pearl_gpu_geometry).  Against it the GPU must agree bitwise:

  * the reductions and the implicit solve of one step;
  * whole runs: 30 adaptive steps, both block shapes on a 1024x1024 domain;
  * the small FP64 configuration for 20000 steps (ten times its horizon),
    where the reference's own order (the golden run of the reference itself,
    tests/golden/make_horizon_golden.py) drifts from the device in mu: the
    device-order oracle drifts by exactly the same amount, so the drift is
    the summation order and nothing else.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _ctx(w):
    import pearl_gpu

    ctx = pearl_gpu.Context(w.params, w.nx, w.ny, device=0)
    ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
    return ctx


def _order(port, ctx):
    g = ctx.geometry()
    return port.device_order(g["warps"], g["blocks"], g["warps_x_log2"], threads=os.cpu_count())


def test_energy_and_mass_bitwise(gpu_lib, port):
    from pearl_gpu import workloads

    w = workloads.scaled(137, 250, seed=2, front=40.0, jitter=0.1)
    with _ctx(w) as ctx:
        e, m = ctx.energy_mass()
        with _order(port, ctx):
            rc, e_o, m_o = port.energy_and_mass(w.params, w.phi, w.carbon)
    assert rc == 0
    assert (e, m) == (e_o, m_o)


@pytest.mark.parametrize("nx,ny,front", [(64, 48, 12.0), (137, 250, 40.0), (37, 19, 6.0)])
def test_implicit_diffusion_bitwise(gpu_lib, port, nx, ny, front):
    from pearl_gpu import workloads

    w = workloads.scaled(nx, ny, seed=5, front=front, jitter=0.1)
    dt = 4e-12
    rc, trial_phi, _ = port.propose_phi(w.params, w.phi, w.mu, dt)
    assert rc == 0
    with _ctx(w) as ctx:
        ctx.upload_trial_phi(trial_phi)
        d = ctx.implicit_diffusion(dt)
        _, c_g, mu_g = ctx.download_trial()
        with _order(port, ctx):
            rc, c_o, mu_o, info = port.implicit_diffusion(w.params, w.carbon, w.mu, trial_phi, dt)
    assert rc == 0 and info.ok == 1 and d["ok"] == 1
    assert d["it"] == info.it
    assert d["residual"] == info.residual
    assert np.array_equal(c_g, c_o)
    assert np.array_equal(mu_g, mu_o)


def _run_both(port, w, n, chunk=None):
    """n steps on the GPU (persistent launches of `chunk` steps) and in the
    device-order oracle; returns both states and step records."""
    from oracle import pyoracle

    with _ctx(w) as ctx:
        ctx.set_history(n)
        done = 0
        while done < n:
            done += ctx.run(min(chunk or n, n - done)).steps
        infos, recorded = ctx.history()
        assert recorded == n
        gpu = ctx.download()
        po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        so = pyoracle.scalars_from(w.scalars)
        with _order(port, ctx):
            rc, why, k, oinfos = port.advance_n(w.params, po, co, muo, so, n)
    assert rc == 0 and k == n, why
    return gpu, (po, co, muo, so), infos, oinfos


def _assert_bitwise(gpu, ora, infos, oinfos):
    phi, c, mu, s = gpu
    po, co, muo, so = ora
    for f in ("retries", "accepted_dt", "cg_iterations", "max_phase_change", "linear_residual", "closure",
              "energy_change"):
        assert [getattr(i, f) for i in infos] == [getattr(i, f) for i in oinfos], f
    assert (s.time, s.dt, s.step, s.rejected) == (so.time, so.dt, so.step, so.rejected)
    assert np.array_equal(phi, po)
    assert np.array_equal(c, co)
    assert np.array_equal(mu, muo)


def test_adaptive_run_bitwise(gpu_lib, port):
    from pearl_gpu import workloads

    w = workloads.scaled(96, 128, seed=7, undercooling=20.0, dt=4e-12, dt_max=8e-12, jitter=0.1, front_jitter=1,
                         front=24.0)
    gpu, ora, infos, oinfos = _run_both(port, w, 30, chunk=7)
    assert sum(i.retries for i in infos) >= 1
    _assert_bitwise(gpu, ora, infos, oinfos)


@pytest.mark.parametrize("warps", [8, 16])
def test_block_shapes_bitwise(gpu_lib, port, monkeypatch, warps):
    from pearl_gpu import workloads

    monkeypatch.setenv("PEARL_GPU_TILE_WARPS", str(warps))
    w = workloads.scaled(1024, 1024, seed=21, undercooling=20.0, dt=4e-12, dt_max=8e-12, front=48.0, pairs=32,
                         jitter=0.1)
    gpu, ora, infos, oinfos = _run_both(port, w, 6)
    _assert_bitwise(gpu, ora, infos, oinfos)


def test_small_workload_20000_steps_bitwise_and_drift_is_summation_order(gpu_lib, port):
    """128x256, fixed dt, 20000 steps: the GPU equals the device-order oracle
    bit for bit at every step; against the reference's own run (same
    decisions at every step) the mu difference of the GPU equals that of the
    device-order oracle, i.e. it comes from the order of the sums alone."""
    from pearl_gpu import workloads

    golden = json.loads((GOLDEN / "horizon_golden.json").read_text())
    ref = np.load(GOLDEN / "horizon_fields.npz")
    n = golden["steps"]
    w = workloads.plain_small()
    gpu, ora, infos, oinfos = _run_both(port, w, n, chunk=5000)
    _assert_bitwise(gpu, ora, infos, oinfos)
    phi, c, mu, s = gpu
    # the reference took the same decisions at every one of the 20000 steps
    assert [i.retries for i in infos] == ref["steps/retries"].tolist()
    assert [i.accepted_dt for i in infos] == ref["steps/accepted_dt"].tolist()
    assert [i.cg_iterations for i in infos] == ref["steps/cg_iterations"].tolist()
    rphi, rc_, rmu = ref[f"s{n}/phi"], ref[f"s{n}/carbon"], ref[f"s{n}/mu"]
    assert s.time == ref[f"s{n}/scalars"][0] and s.rejected == ref[f"s{n}/scalars"][3]
    # phi and carbon stay within the FP64 bars after 20000 steps
    assert np.abs(phi - rphi).max() <= 1e-10
    assert abs(c.sum() - rc_.sum()) <= 1e-12 * abs(rc_.sum())
    # mu drifts with the summation order (1/chi of cementite is ~2e8 J/mol per
    # unit carbon, so 1e-12 carbon moves mu by ~1e-4 J/mol); the device-order
    # oracle, the reference's arithmetic in the device's order, drifts by the
    # very same amount at every cell
    drift = np.abs(mu - rmu)
    assert np.array_equal(drift, np.abs(ora[2] - rmu))
    assert drift.max() <= 1e-3
