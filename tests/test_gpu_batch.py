"""Batched instances (pearl_gpu_batch): many independent domains in one
persistent launch, each following the single-domain step path.

  * With at least as many blocks per group as an instance has tiles, every
    tile of the instance belongs to the same block as in a pearl_gpu_ctx of
    its own and the extra blocks add exact zeros to each sum, so the batch
    reproduces the single-domain result bitwise.
  * With fewer blocks per group, the reductions are ordered differently; the
    instances are then held to the FP64 bars against the oracle (max|dphi| <=
    1e-10, max|dmu| <= 1e-5 J/mol, total carbon 1e-12 relative) with the same
    accepted steps, retries and CG iteration counts.
  * Groups sized per instance (PEARL_BATCH_SIZED_GROUPS) follow the same two
    rules: small instances get a group with at least one block per tile when
    the grid allows it, large ones fewer.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PHI_TOL = 1e-10
MU_TOL = 1e-5
MASS_RTOL = 1e-12


def _cases():
    from pearl_gpu import workloads

    return [
        workloads.scaled(64, 64, seed=1, undercooling=12.0, dt=4e-12, dt_max=8e-12, front=16.0),
        workloads.scaled(40, 48, seed=2, undercooling=30.0, dt=4e-12, dt_max=8e-12, front=12.0, pairs=2),
        workloads.scaled(96, 32, seed=3, undercooling=6.0, dt=4e-12, front=10.0, jitter=0.1),
        workloads.scaled(33, 80, seed=4, undercooling=20.0, dt=4e-12, dt_max=8e-12, front=20.0),
    ]


def _batch(ws, group_blocks):
    import pearl_gpu

    b = pearl_gpu.Batch([(w.params, w.nx, w.ny) for w in ws], group_blocks=group_blocks)
    for i, w in enumerate(ws):
        b.upload(i, w.phi, w.carbon, w.mu, w.scalars)
    return b


def test_batch_bitwise_equals_single_domains(gpu_lib):
    import pearl_gpu

    ws = _cases()
    with _batch(ws, 16) as b:
        reps, st = b.run(20)
        assert st == [0] * len(ws)
        got = [b.download(i) for i in range(len(ws))]
    for w, rep, g in zip(ws, reps, got):
        with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
            ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
            r = ctx.run(20)
            want = ctx.download()
        assert rep.steps == r.steps == 20
        assert rep.cg_total == r.cg_total and rep.cg_peak == r.cg_peak
        for x, y in zip(g[:3], want[:3]):
            assert np.array_equal(x, y)
        assert g[3].time == want[3].time and g[3].dt == want[3].dt and g[3].rejected == want[3].rejected


@pytest.mark.parametrize("group_blocks", [1, 3, -1])
def test_batch_matches_oracle(gpu_lib, port, group_blocks):
    from oracle import pyoracle

    ws = _cases()
    n = 15
    with _batch(ws, group_blocks) as b:
        reps, st = b.run(n)
        assert st == [0] * len(ws)
        got = [b.download(i) for i in range(len(ws))]
    for w, rep, (phi, c, mu, s) in zip(ws, reps, got):
        phi_o, c_o, mu_o = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        so = pyoracle.scalars_from(w.scalars)
        rc, why, done, oinfos = port.advance_n(w.params, phi_o, c_o, mu_o, so, n)
        assert rc == 0 and done == n, why
        assert rep.steps == n
        assert rep.cg_total == sum(i.cg_iterations for i in oinfos)
        assert s.rejected == so.rejected and s.step == so.step and s.time == so.time
        assert np.abs(phi - phi_o).max() <= PHI_TOL
        assert np.abs(mu - mu_o).max() <= MU_TOL
        assert abs(c.sum() - c_o.sum()) <= MASS_RTOL * abs(c_o.sum())


def test_batch_repeated_launches_and_output_stop(gpu_lib):
    """Chunks of launches equal one long launch; stop_time ends every instance at the output time."""
    ws = _cases()[:2]
    with _batch(ws, 8) as a:
        a.run(6)
        a.run(6)
        fa = [a.download(i) for i in range(2)]
    with _batch(ws, 8) as b:
        reps, _ = b.run(12)
        fb = [b.download(i) for i in range(2)]
    for x, y in zip(fa, fb):
        for u, v in zip(x[:3], y[:3]):
            assert np.array_equal(u, v)
    t_out = 5e-12
    with _batch(ws, 8) as c:
        reps, st = c.run(100, stop_time=t_out, output_eps=1e-12 * t_out)
        assert st == [0, 0]
        for i, r in enumerate(reps):
            assert r.reached_stop == 1
            assert c.download(i)[3].time == pytest.approx(t_out, rel=1e-12)


def test_batch_instance_error_is_local(gpu_lib):
    """An instance that hits the configured step limit reports it; the others run on."""
    max_steps_status = 8  # PEARL_ERR_MAX_STEPS
    ws = _cases()[:2]
    with _batch(ws, 4) as b:
        s = dict(ws[1].scalars)
        s["step"] = 5
        b.upload(1, ws[1].phi, ws[1].carbon, ws[1].mu, s)
        reps, st = b.run(6, config_max_steps=7)
        assert st == [0, max_steps_status]
        assert reps[0].steps == 6 and reps[1].steps == 2
        assert b.download(1)[3].step == 7


def test_batch_autotune_keeps_state(gpu_lib):
    ws = _cases()
    with _batch(ws, 4) as a:
        gb, tma, wx = a.autotune(steps=1)
        assert gb in (1, 2, 4, 8, 16, -1) and wx in (1, 2, 4)
        assert a.stats()["group_blocks"] == gb
        assert a.run(10)[1] == [0] * len(ws)
        fa = [a.download(i) for i in range(len(ws))]
    with _batch(ws, gb) as b:
        b.configure(gb, not tma, wx)  # TMA staging moves data only: it changes no value
        b.run(10)
        fb = [b.download(i) for i in range(len(ws))]
    for x, y in zip(fa, fb):
        assert x[3].step == y[3].step == 10
        for u, v in zip(x[:3], y[:3]):
            assert np.array_equal(u, v)


@pytest.mark.parametrize("wx", [2, 4])
def test_batch_tile_shapes_match_oracle(gpu_lib, port, wx):
    """Wider tiles change only which block owns which cells (the order of sums)."""
    from oracle import pyoracle

    ws = _cases()
    n = 12
    with _batch(ws, 4) as b:
        b.configure(4, False, wx)
        reps, st = b.run(n)
        assert st == [0] * len(ws)
        got = [b.download(i) for i in range(len(ws))]
    for w, (phi, c, mu, s) in zip(ws, got):
        phi_o, c_o, mu_o = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        so = pyoracle.scalars_from(w.scalars)
        rc, why, done, _ = port.advance_n(w.params, phi_o, c_o, mu_o, so, n)
        assert rc == 0 and done == n, why
        assert s.rejected == so.rejected and s.step == so.step
        assert np.abs(phi - phi_o).max() <= PHI_TOL
        assert np.abs(mu - mu_o).max() <= MU_TOL
        assert abs(c.sum() - c_o.sum()) <= MASS_RTOL * abs(c_o.sum())


def test_batch_sized_groups(gpu_lib, port):
    """Per-instance group sizes.  The small instances alone (6 to 10 tiles each)
    get a group with a block per tile and equal their single-domain runs
    bitwise.  Beside three 384x384 instances (288 tiles each, more than the
    grid holds for them) every instance shares blocks between tiles and all
    meet the FP64 bars against the oracle."""
    import pearl_gpu
    from pearl_gpu import workloads
    from oracle import pyoracle

    small = _cases()
    n = 8
    with _batch(small, pearl_gpu.BATCH_SIZED_GROUPS) as b:
        assert b.stats()["group_blocks"] == pearl_gpu.BATCH_SIZED_GROUPS
        reps, st = b.run(n)
        assert st == [0] * len(small)
        got = [b.download(i) for i in range(len(small))]
    for w, rep, g in zip(small, reps, got):
        with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
            ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
            r = ctx.run(n)
            want = ctx.download()
        assert rep.cg_total == r.cg_total
        for x, y in zip(g[:3], want[:3]):
            assert np.array_equal(x, y)

    large = [workloads.scaled(384, 384, seed=10 + k, undercooling=15.0 + 5 * k, dt=4e-12, dt_max=8e-12,
                              front=40.0, pairs=6) for k in range(3)]
    ws = large + small
    with _batch(ws, pearl_gpu.BATCH_SIZED_GROUPS) as b:
        assert 0 < b.stats()["grid"] <= 2 * 148
        reps, st = b.run(n)
        assert st == [0] * len(ws)
        got = [b.download(i) for i in range(len(ws))]
    for w, rep, (phi, c, mu, s) in zip(ws, reps, got):
        phi_o, c_o, mu_o = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        so = pyoracle.scalars_from(w.scalars)
        rc, why, done, oinfos = port.advance_n(w.params, phi_o, c_o, mu_o, so, n)
        assert rc == 0 and done == n, why
        assert rep.steps == n and rep.cg_total == sum(i.cg_iterations for i in oinfos)
        assert s.rejected == so.rejected and s.time == so.time
        assert np.abs(phi - phi_o).max() <= PHI_TOL
        assert np.abs(mu - mu_o).max() <= MU_TOL
        assert abs(c.sum() - c_o.sum()) <= MASS_RTOL * abs(c_o.sum())
