"""GPU parity of the FP64 hot path against the CPU oracle (pearl_oracle.c,
itself bit-identical to the reference serial solver).

Tolerances (from the reference's own serial-vs-MPI limits and the FP64 bar):
  * per-cell functions that involve no global sum (propose_phi, valid_state)
    must match bitwise;
  * after N accepted steps: max|dphi| <= 1e-10, max|dmu| <= 1e-5 J/mol,
    total carbon within 1e-12 relative;
  * reductions (energy, carbon mass, CG dots) within 1e-12 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PHI_TOL = 1e-10
MU_TOL = 1e-5
MASS_RTOL = 1e-12


def _ctx(w):
    import pearl_gpu

    ctx = pearl_gpu.Context(w.params, w.nx, w.ny, device=0)
    ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
    return ctx


SIZES = [(64, 48, 12.0), (37, 19, 6.0), (137, 250, 40.0), (128, 256, 32.0)]


# Contexts stage tiles through TMA only when every block has several tiles a
# pass (the small domains here run on plain loads by default); PEARL_GPU_TMA=1
# forces the staged path, so both paths meet the same bars.
STAGING = ["default", "1"]


@pytest.mark.parametrize("staging", STAGING)
@pytest.mark.parametrize("nx,ny,front", SIZES)
def test_propose_phi_bitwise(gpu_lib, port, monkeypatch, staging, nx, ny, front):
    from pearl_gpu import workloads

    if staging != "default":
        monkeypatch.setenv("PEARL_GPU_TMA", staging)

    w = workloads.scaled(nx, ny, seed=3, front=front, jitter=0.1, front_jitter=1)
    with _ctx(w) as ctx:
        for dt in (4e-12, 3e-11):
            change = ctx.propose_phi(dt)
            trial, _, _ = ctx.download_trial()
            rc, trial_o, change_o = port.propose_phi(w.params, w.phi, w.mu, dt)
            assert rc == 0
            assert change == change_o
            assert np.array_equal(trial, trial_o)


@pytest.mark.parametrize("nx,ny,front", SIZES[:3])
def test_implicit_diffusion(gpu_lib, port, nx, ny, front):
    from pearl_gpu import workloads

    w = workloads.scaled(nx, ny, seed=5, front=front, jitter=0.1)
    dt = 4e-12
    rc, trial_phi, _ = port.propose_phi(w.params, w.phi, w.mu, dt)
    with _ctx(w) as ctx:
        ctx.upload_trial_phi(trial_phi)
        d = ctx.implicit_diffusion(dt)
        _, c_g, mu_g = ctx.download_trial()
    rc, c_o, mu_o, info = port.implicit_diffusion(w.params, w.carbon, w.mu, trial_phi, dt)
    assert rc == 0 and info.ok == 1 and d["ok"] == 1
    assert d["it"] == info.it
    # the converged true residual is a norm of rounding-level values (~1e-16):
    # different dot-product orders move it in the 5th digit
    assert abs(d["residual"] - info.residual) <= 1e-3 * info.residual + 1e-30
    assert np.abs(mu_g - mu_o).max() <= MU_TOL
    assert np.abs(c_g - c_o).max() <= 1e-14
    assert abs(c_g.sum() - c_o.sum()) <= MASS_RTOL * abs(c_o.sum())


def test_energy_mass_valid(gpu_lib, port):
    from pearl_gpu import workloads

    w = workloads.scaled(137, 250, seed=2, front=40.0, jitter=0.1)
    with _ctx(w) as ctx:
        e, m = ctx.energy_mass()
        v = ctx.valid_state()
    rc, e_o, m_o = port.energy_and_mass(w.params, w.phi, w.carbon)
    assert rc == 0
    assert abs(e - e_o) <= 1e-12 * abs(e_o)
    assert abs(m - m_o) <= 1e-12 * abs(m_o)
    assert v == bool(port.valid_state(w.params, w.phi, w.carbon, w.mu))


def _compare_run(ctx, w, port, nsteps, forced=None):
    infos = [ctx.advance() for _ in range(nsteps)]
    phi, c, mu, s = ctx.download()
    phi_o, c_o, mu_o = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    from oracle import pyoracle

    so = pyoracle.scalars_from(w.scalars)
    dts = [i.accepted_dt for i in infos] if forced else None
    rc, why, done, oinfos = port.advance_n(w.params, phi_o, c_o, mu_o, so, nsteps, forced_dt=dts)
    assert rc == 0 and done == nsteps, why
    if not forced:
        # a replay hands the oracle the accepted dt directly, so it takes no retries
        assert [i.retries for i in infos] == [i.retries for i in oinfos]
    assert [i.accepted_dt for i in infos] == [i.accepted_dt for i in oinfos]
    assert [i.cg_iterations for i in infos] == [i.cg_iterations for i in oinfos]
    assert np.abs(phi - phi_o).max() <= PHI_TOL
    assert np.abs(mu - mu_o).max() <= MU_TOL
    assert abs(c.sum() - c_o.sum()) <= MASS_RTOL * abs(c_o.sum())
    assert s.step == so.step
    if not forced:
        assert s.rejected == so.rejected
        assert s.time == so.time
    return infos, oinfos


@pytest.mark.parametrize("staging", STAGING)
def test_advance_small_fixed_dt(gpu_lib, port, monkeypatch, staging):
    """128x256, 4 pairs, fixed dt 4e-12 s: 25 accepted steps (includes a rejected attempt)."""
    from pearl_gpu import workloads

    if staging != "default":
        monkeypatch.setenv("PEARL_GPU_TMA", staging)

    w = workloads.plain_small()
    with _ctx(w) as ctx:
        infos, _ = _compare_run(ctx, w, port, 25)
    assert sum(i.retries for i in infos) >= 1


def test_small_workload_full_horizon(gpu_lib, port):
    """The small FP64 configuration at its own horizon: 128x256, 4 pairs, 10 K,
    fixed dt = dt_max = 4e-12 s, 2000 accepted steps in persistent launches of
    500 steps, against the oracle's 2000 steps (about 20 s of CPU): every step's
    retries, dt and CG count agree, and the fields meet the FP64 bars."""
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.plain_small()
    n = w.meta["steps"]
    assert n == 2000
    with _ctx(w) as ctx:
        ctx.set_history(n)
        done = 0
        while done < n:
            done += ctx.run(min(500, n - done)).steps
        infos, recorded = ctx.history()
        phi, c, mu, s = ctx.download()
    assert recorded == n
    po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    so = pyoracle.scalars_from(w.scalars)
    rc, why, done, oinfos = port.advance_n(w.params, po, co, muo, so, n)
    assert rc == 0 and done == n, why
    assert [i.retries for i in infos] == [i.retries for i in oinfos]
    assert [i.accepted_dt for i in infos] == [i.accepted_dt for i in oinfos]
    assert [i.cg_iterations for i in infos] == [i.cg_iterations for i in oinfos]
    assert s.step == so.step and s.rejected == so.rejected and s.time == so.time
    assert np.abs(phi - po).max() <= PHI_TOL
    assert np.abs(mu - muo).max() <= MU_TOL
    assert abs(c.sum() - co.sum()) <= MASS_RTOL * abs(co.sum())


def _adaptive():
    from pearl_gpu import workloads

    return workloads.scaled(96, 128, seed=7, undercooling=20.0, dt=4e-12, dt_max=8e-12, jitter=0.1, front_jitter=1,
                            front=24.0)


def test_advance_adaptive_natural(gpu_lib, port):
    """Adaptive dt (dt_max = 2 dt), both sides choosing dt themselves: same decisions."""
    w = _adaptive()
    with _ctx(w) as ctx:
        infos, _ = _compare_run(ctx, w, port, 30)
    assert sum(i.retries for i in infos) >= 1


def test_advance_adaptive_replay(gpu_lib, port):
    """Adaptive dt: the oracle replays the GPU's accepted dt sequence."""
    w = _adaptive()
    with _ctx(w) as ctx:
        _compare_run(ctx, w, port, 30, forced=True)


def test_run_matches_advance(gpu_lib):
    """pearl_gpu_run (many steps per launch) equals repeated pearl_gpu_advance bitwise."""
    from pearl_gpu import workloads

    w = workloads.scaled(64, 80, seed=9, front=20.0)
    with _ctx(w) as a:
        for _ in range(12):
            a.advance()
        fa = a.download()
    with _ctx(w) as b:
        rep = b.run(12)
        fb = b.download()
    assert rep.steps == 12
    for x, y in zip(fa[:3], fb[:3]):
        assert np.array_equal(x, y)


EDGE_SIZES = [(3, 2, 1.0), (3, 5, 2.0), (4, 3, 1.5), (31, 17, 6.0), (33, 16, 8.0), (65, 33, 10.0)]


@pytest.mark.parametrize("staging", STAGING)
@pytest.mark.parametrize("nx,ny,front", EDGE_SIZES)
def test_smallest_and_ragged_domains(gpu_lib, port, monkeypatch, staging, nx, ny, front):
    """The smallest domains the reference accepts (nx >= 3, ny >= 2) and widths
    and heights just off the 32x16 tile: propose_phi bitwise, then 8 coupled
    steps against the oracle with the same decisions; on plain loads (the
    default at these sizes) and staged through TMA."""
    from pearl_gpu import workloads

    if staging != "default":
        monkeypatch.setenv("PEARL_GPU_TMA", staging)

    w = workloads.scaled(nx, ny, seed=3, front=front)
    with _ctx(w) as ctx:
        change = ctx.propose_phi(4e-12)
        trial, _, _ = ctx.download_trial()
    rc, trial_o, change_o = port.propose_phi(w.params, w.phi, w.mu, 4e-12)
    assert rc == 0 and change == change_o
    assert np.array_equal(trial, trial_o)
    with _ctx(w) as ctx:
        _compare_run(ctx, w, port, 8)


def test_full_size_large_workload_replay(gpu_lib, port):
    """The large FP64 configuration at its full size (2048x4096, 64 pairs,
    20 K, adaptive dt): 30 accepted steps on the GPU in one persistent launch,
    then the oracle replays the GPU's accepted dt sequence on the host (about
    90 s of CPU) with the same CG counts, and the fields are held to the FP64
    bars."""
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.plain_large()
    n = 30
    with _ctx(w) as ctx:
        ctx.set_history(n)
        assert ctx.run(n).steps == n
        infos, recorded = ctx.history()
        assert recorded == n
        phi, c, mu, s = ctx.download()
    po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    so = pyoracle.scalars_from(w.scalars)
    rc, why, done, oinfos = port.advance_n(w.params, po, co, muo, so, n, forced_dt=[i.accepted_dt for i in infos])
    assert rc == 0 and done == n, why
    assert [i.cg_iterations for i in infos] == [i.cg_iterations for i in oinfos]
    assert np.abs(phi - po).max() <= PHI_TOL
    assert np.abs(mu - muo).max() <= MU_TOL
    assert abs(c.sum() - co.sum()) <= MASS_RTOL * abs(co.sum())


@pytest.mark.parametrize("warps", [8, 16])
def test_block_shapes_match_oracle(gpu_lib, port, monkeypatch, warps):
    """Both block shapes (256-thread blocks with 32x16 tiles, 512-thread blocks
    with 32x32 tiles; a 1024x1024 domain takes the latter by default) against
    the oracle on the same domain: the shape changes only which block owns
    which cells, so the steps, rejections and CG counts agree and the fields
    meet the FP64 bars."""
    from oracle import pyoracle
    from pearl_gpu import workloads

    monkeypatch.setenv("PEARL_GPU_TILE_WARPS", str(warps))
    w = workloads.scaled(1024, 1024, seed=21, undercooling=20.0, dt=4e-12, dt_max=8e-12, front=48.0, pairs=32,
                         jitter=0.1)
    n = 6
    with _ctx(w) as ctx:
        infos = [ctx.advance() for _ in range(n)]
        phi, c, mu, s = ctx.download()
    po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    so = pyoracle.scalars_from(w.scalars)
    rc, why, done, oinfos = port.advance_n(w.params, po, co, muo, so, n)
    assert rc == 0 and done == n, why
    assert [i.cg_iterations for i in infos] == [i.cg_iterations for i in oinfos]
    assert [i.retries for i in infos] == [i.retries for i in oinfos]
    assert s.time == so.time and s.rejected == so.rejected
    assert np.abs(phi - po).max() <= PHI_TOL
    assert np.abs(mu - muo).max() <= MU_TOL
    assert abs(c.sum() - co.sum()) <= MASS_RTOL * abs(co.sum())
