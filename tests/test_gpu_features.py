"""GPU path against the reference's own stored outputs (tests/golden, written
by the unmodified reference solver) and against the oracle for the moving
window, output reductions, error semantics and main-loop limits."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from test_oracle import params_from, scalars_from

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
PHI_TOL = 1e-10
MU_TOL = 1e-5
MASS_RTOL = 1e-12


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "pearl_ref_golden.npz"), json.loads((GOLDEN / "pearl_ref_golden.json").read_text())


def _ctx(params, phi, c, mu, s):
    import pearl_gpu

    ny, nx = c.shape
    ctx = pearl_gpu.Context(params, nx, ny, device=0)
    ctx.upload(np.ascontiguousarray(phi), np.ascontiguousarray(c), np.ascontiguousarray(mu),
               {k: getattr(s, k) for k, _ in pearl_gpu.PearlScalars._fields_})
    return ctx


def _close(phi, c, mu, phi_r, c_r, mu_r):
    assert np.abs(phi - phi_r).max() <= PHI_TOL
    assert np.abs(mu - mu_r).max() <= MU_TOL
    assert abs(c.sum() - c_r.sum()) <= MASS_RTOL * abs(c_r.sum())


def test_advance_vs_reference_golden(gpu_lib, golden):
    data, meta = golden
    p = params_from(data["adv_params"], meta)
    with _ctx(p, data["adv_phi0"], data["adv_c0"], data["adv_mu0"], scalars_from(data["adv_s0"], meta)) as ctx:
        infos = [ctx.advance() for _ in range(meta["cases"]["adv"]["steps"])]
        phi, c, mu, s = ctx.download()
    _close(phi, c, mu, data["adv_phi"], data["adv_c"], data["adv_mu"])
    ref_info = data["adv_info"]
    keys = meta["info_keys"]
    assert [i.retries for i in infos] == list(ref_info[:, keys.index("retries")])
    assert [i.cg_iterations for i in infos] == list(ref_info[:, keys.index("cg_iterations")])
    assert [i.accepted_dt for i in infos] == list(ref_info[:, keys.index("accepted_dt")])
    s_ref = data["adv_s"]
    assert s.time == s_ref[meta["scalar_keys"].index("time")]
    assert s.rejected == s_ref[meta["scalar_keys"].index("rejected")]


def test_phase_only_vs_reference_golden(gpu_lib, golden):
    data, meta = golden
    p = params_from(data["po_params"], meta)
    with _ctx(p, data["po_phi0"], data["po_c0"], data["po_mu0"], scalars_from(data["po_s0"], meta)) as ctx:
        for _ in range(8):
            ctx.advance()
        phi, c, mu, s = ctx.download()
    # phase-only steps involve no global sum in the fields: bitwise
    assert np.array_equal(phi, data["po_phi"])
    assert np.array_equal(c, data["po_c"])
    assert np.array_equal(mu, data["po_mu"])


def test_moving_window_vs_reference_golden(gpu_lib, golden):
    data, meta = golden
    p = params_from(data["sh_params"], meta)
    trig, targ, cg = data["sh_args"]
    with _ctx(p, data["sh_phi0"], data["sh_c0"], data["sh_mu0"], scalars_from(data["sh_s0"], meta)) as ctx:
        rows = ctx.maybe_shift(trig, targ, cg)
        phi, c, mu, s = ctx.download()
    assert rows > 0
    # the shift and mu closure are per cell: bitwise
    assert np.array_equal(phi, data["sh_phi"])
    assert np.array_equal(c, data["sh_c"])
    assert np.array_equal(mu, data["sh_mu"])
    sk = meta["scalar_keys"]
    s_ref = data["sh_s"]
    assert s.shifts == s_ref[sk.index("shifts")] and s.shift_distance == s_ref[sk.index("shift_distance")]
    assert s.carbon_added == s_ref[sk.index("carbon_added")]
    assert s.carbon_removed == pytest.approx(s_ref[sk.index("carbon_removed")], rel=1e-13)


def test_moving_window_below_trigger(gpu_lib, port):
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.scaled(64, 64, seed=2, front=12.0)
    with _ctx(w.params, w.phi, w.carbon, w.mu, pyoracle.scalars_from(w.scalars)) as ctx:
        assert ctx.maybe_shift(0.65 * 64 * 2e-9, 0.35 * 64 * 2e-9, 0.0345) == 0
        phi, _, _, s = ctx.download()
    assert s.shifts == 0 and np.array_equal(phi, w.phi)


def test_unsafe_shift_error(gpu_lib):
    """A trigger/target pair that would cut through gamma raises the reference's error."""
    import pearl_gpu
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.scaled(64, 64, seed=2, front=40.0)
    with _ctx(w.params, w.phi, w.carbon, w.mu, pyoracle.scalars_from(w.scalars)) as ctx:
        with pytest.raises(pearl_gpu.PearlError, match="unsafe shift: removed strip contains gamma"):
            ctx.maybe_shift(1e-9, 0.5e-9, 0.0345)


def test_snapshot_reductions(gpu_lib, port):
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.scaled(137, 250, seed=6, front=40.0, jitter=0.1)
    s = pyoracle.scalars_from(w.scalars)
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    rc, why, _, _ = port.advance_n(w.params, phi, c, mu, s, 3)
    assert rc == 0
    with _ctx(w.params, phi, c, mu, s) as ctx:
        d = ctx.snapshot()
    rc, o = port.snapshot(w.params, phi, c, mu, s)
    assert rc == 0
    for k in ("c_min", "c_max", "mu_min", "mu_max", "phi_sum_error"):
        assert getattr(d, k) == getattr(o, k)
    assert d.mass == pytest.approx(o.mass, rel=1e-13)
    assert d.energy == pytest.approx(o.energy, rel=1e-12)
    assert d.ledger == pytest.approx(o.ledger, abs=1e-12 * abs(o.mass))


def test_rejected_below_dt_min_message(gpu_lib, golden):
    import pearl_gpu
    from pearl_gpu import workloads

    data, meta = golden
    w = workloads.scaled(48, 40, seed=1, front=10.0, jitter=0.1, front_jitter=1, dt=2e-10, dt_min=2e-10)
    with _ctx(w.params, w.phi, w.carbon, w.mu, scalars_from(np.array([w.scalars[k] for k in meta["scalar_keys"]]),
                                                              meta)) as ctx:
        with pytest.raises(pearl_gpu.PearlError) as e:
            ctx.advance()
        assert str(e.value) == meta["cases"]["err"]["message"]
        assert e.value.status == 4
        phi, c, mu, s = ctx.download()
    assert np.array_equal(phi, w.phi) and s.step == 0  # state unchanged on error


def test_invalid_advance_time(gpu_lib):
    import pearl_gpu
    from pearl_gpu import workloads

    w = workloads.scaled(32, 16, seed=1, front=6.0)
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        with pytest.raises(pearl_gpu.PearlError, match="invalid advance time"):
            ctx.advance(stop_time=0.0)


def test_run_stops_at_output_time(gpu_lib, port):
    """pearl_gpu_run follows main's loop: output-time clipping and stop (pearl_serial.cpp:2296-2316)."""
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.scaled(64, 48, seed=8, front=12.0)
    out_dt = 2.5e-11  # not a multiple of dt: the last step is clipped
    eps = 1e-12 * max(1e-9, out_dt)
    with _ctx(w.params, w.phi, w.carbon, w.mu, pyoracle.scalars_from(w.scalars)) as ctx:
        rep = ctx.run(1000, stop_time=out_dt, end_time=1e-9, output_eps=eps)
        phi, c, mu, s = ctx.download()
    assert rep.reached_stop == 1
    assert abs(s.time - out_dt) <= eps
    # the oracle with the same stop time takes the same steps
    so = pyoracle.scalars_from(w.scalars)
    phi_o, c_o, mu_o = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    rc, why, done, infos = port.advance_n(w.params, phi_o, c_o, mu_o, so, int(rep.steps), stop_time=out_dt)
    assert rc == 0 and so.time == s.time and so.step == s.step
    assert infos[-1].accepted_dt == rep.last.accepted_dt
    np.testing.assert_allclose(phi, phi_o, rtol=0, atol=PHI_TOL)


def test_config_max_steps_error(gpu_lib):
    import pearl_gpu
    from pearl_gpu import workloads

    w = workloads.scaled(32, 16, seed=1, front=6.0)
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        with pytest.raises(pearl_gpu.PearlError, match="configured max_steps reached before end_time"):
            ctx.run(10, config_max_steps=3)
        assert ctx.scalars().step == 3


def test_large_domain_properties(gpu_lib):
    """2048x1024: deterministic, mass-conserving, energy non-increasing, valid."""
    import pearl_gpu
    from pearl_gpu import workloads

    w = workloads.plain_large(nx=2048, ny=1024, pairs=64)
    results = []
    for _ in range(2):
        with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
            ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
            e0, m0 = ctx.energy_mass()
            infos = [ctx.advance() for _ in range(6)]
            e1, m1 = ctx.energy_mass()
            assert ctx.valid_state()
            results.append(ctx.download())
    for a, b in zip(results[0][:3], results[1][:3]):
        assert np.array_equal(a, b)
    assert abs(m1 - m0) <= 1e-11 * abs(m0)
    assert e1 <= e0
    assert all(i.energy_change <= 1e-12 * abs(e0) + 1e-20 for i in infos)


def test_bounded_wait_reports_and_recovers(gpu_lib):
    """A grid barrier that cannot complete gives up after its limit (4 s) with
    PEARL_ERR_DEVICE_WAIT instead of hanging, and the context keeps working:
    the next step equals a fresh context's step bitwise."""
    import pearl_gpu
    from pearl_gpu import workloads

    w = workloads.scaled(64, 48, seed=5, front=12.0)
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        status, ms = ctx.selftest_wait_limit()
        assert status == 9  # PEARL_ERR_DEVICE_WAIT
        assert 3900.0 <= ms <= 30000.0
        ctx.advance()
        got = ctx.download()
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ref:
        ref.upload(w.phi, w.carbon, w.mu, w.scalars)
        ref.advance()
        want = ref.download()
    for a, b in zip(got[:3], want[:3]):
        assert np.array_equal(a, b)


def test_step_history_ring_and_replay(gpu_lib, port):
    """The device history of a multi-step launch equals the per-step infos of
    single advances, keeps the last `capacity` steps in order, and its accepted
    dt sequence lets the oracle replay the run."""
    import pearl_gpu
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.scaled(96, 128, seed=7, undercooling=20.0, dt=4e-12, dt_max=8e-12, jitter=0.1, front_jitter=1,
                         front=24.0)
    n = 20
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ref:
        ref.upload(w.phi, w.carbon, w.mu, w.scalars)
        infos = [ref.advance() for _ in range(n)]
    fields = [f for f, _ in pearl_gpu.PearlStepInfo._fields_]
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        ctx.set_history(8)
        ctx.run(7)
        ctx.run(n - 7)
        last8, recorded = ctx.history()
        assert recorded == n and len(last8) == 8
        for h, i in zip(last8, infos[-8:]):
            assert all(getattr(h, f) == getattr(i, f) for f in fields)
        ctx.set_history(64)
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        ctx.run(n)
        hist, recorded = ctx.history()
        phi, c, mu, _ = ctx.download()
    assert recorded == n and len(hist) == n
    assert sum(h.retries for h in hist) >= 1
    po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    so = pyoracle.scalars_from(w.scalars)
    rc, why, done, _ = port.advance_n(w.params, po, co, muo, so, n, forced_dt=[h.accepted_dt for h in hist])
    assert rc == 0 and done == n, why
    assert np.abs(phi - po).max() <= 1e-10 and np.abs(mu - muo).max() <= 1e-5


def test_run_replay_reproduces_a_run(gpu_lib):
    """Replaying a run's recorded accepted-dt sequence (rejections included in the
    original) reproduces its fields bitwise with no rejected attempt."""
    import pearl_gpu
    from pearl_gpu import workloads

    w = workloads.scaled(96, 128, seed=7, undercooling=20.0, dt=4e-12, dt_max=8e-12, jitter=0.1, front_jitter=1,
                         front=24.0)
    with pearl_gpu.Context(w.params, w.nx, w.ny) as a:
        a.upload(w.phi, w.carbon, w.mu, w.scalars)
        a.set_history(64)
        a.run(25)
        hist, _ = a.history()
        want = a.download()
    assert sum(h.retries for h in hist) >= 1
    with pearl_gpu.Context(w.params, w.nx, w.ny) as b:
        b.upload(w.phi, w.carbon, w.mu, w.scalars)
        rep = b.run_replay([h.accepted_dt for h in hist])
        got = b.download()
    assert rep.steps == 25 and got[3].rejected == 0
    assert got[3].time == want[3].time
    for x, y in zip(got[:3], want[:3]):
        assert np.array_equal(x, y)
