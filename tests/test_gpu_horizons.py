"""The batched sweep and the adjoint at their configured horizons.

  * Sweep (5000 adaptive steps per instance): three instances of the seeded
    256-instance sweep (the smallest, a high-undercooling one and a mid-sized
    one) run 5000 steps in one batched launch, with groups of 8 blocks.  Each
    equals, bit for bit, the oracle in the device's summation order for a
    group of 8 blocks (pearl_oracle.c, po_set_device_order); the
    high-undercooling instance is also run by the oracle in the reference's
    own order, which takes the same decisions at every step and conserves the
    same carbon; its phase fields drift from the device's by the order of the
    sums alone (measured 5.4e-8 after 5000 steps at 39.5 K: a fast-moving
    front amplifies the last-bit differences of the CG sums; the device-order
    oracle, the same arithmetic in the device's order, equals the device bit
    for bit), held to 1e-6.
  * Adjoint (256x512, 4 pairs, 15 K, 1000 fixed-dt steps, checkpoint every
    50): the device gradient against the CPU reference gradient
    (oracle/pearl_adjoint.c, about two minutes of CPU) and against central
    differences of the device forward (h = 1e-6 relative), both within 1e-4
    relative.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SWEEP_STEPS = 5000
SWEEP_PICK = (176, 149, 72)  # 38x71 at 15.6 K, 42x114 at 39.5 K, 104x239 at 26.7 K
GROUP_BLOCKS = 8


def test_sweep_instances_full_horizon_bitwise(gpu_lib, port):
    import pearl_gpu
    from oracle import pyoracle
    from pearl_gpu import workloads as W

    ws = [W.sweep_one(i, 0) for i in SWEEP_PICK]
    with pearl_gpu.Batch([(w.params, w.nx, w.ny) for w in ws]) as b:
        b.configure(GROUP_BLOCKS, use_tma=True, tile_warps_x=1)
        for i, w in enumerate(ws):
            b.upload(i, w.phi, w.carbon, w.mu, w.scalars)
        reps, st = b.run(SWEEP_STEPS)
        assert st == [0] * len(ws)
        got = [b.download(i) for i in range(len(ws))]
    for w, rep, (phi, c, mu, s) in zip(ws, reps, got):
        assert rep.steps == SWEEP_STEPS
        po, co, muo = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        so = pyoracle.scalars_from(w.scalars)
        with port.device_order(8, GROUP_BLOCKS, 0, threads=os.cpu_count()):
            rc, why, done, oinfos = port.advance_n(w.params, po, co, muo, so, SWEEP_STEPS)
        assert rc == 0 and done == SWEEP_STEPS, why
        assert rep.cg_total == sum(i.cg_iterations for i in oinfos)
        assert (s.time, s.dt, s.step, s.rejected) == (so.time, so.dt, so.step, so.rejected)
        assert np.array_equal(phi, po) and np.array_equal(c, co) and np.array_equal(mu, muo)
        if w is ws[1]:
            # the reference's own summation order: same decisions, FP64 phase and carbon bars
            pr, cr, mr = w.phi.copy(), w.carbon.copy(), w.mu.copy()
            sr = pyoracle.scalars_from(w.scalars)
            rc, why, done, rinfos = port.advance_n(w.params, pr, cr, mr, sr, SWEEP_STEPS)
            assert rc == 0 and done == SWEEP_STEPS, why
            assert [i.retries for i in rinfos] == [i.retries for i in oinfos]
            assert [i.cg_iterations for i in rinfos] == [i.cg_iterations for i in oinfos]
            assert sr.time == s.time and sr.rejected == s.rejected
            assert np.abs(phi - pr).max() <= 1e-6
            assert abs(c.sum() - cr.sum()) <= 1e-12 * abs(cr.sum())


def test_adjoint_full_horizon(gpu_lib, port):
    import pearl_gpu
    from oracle import pyoracle
    from pearl_gpu import workloads as W

    w = W.adjoint_case()
    steps, every = w.meta["steps"], 50
    assert (w.nx, w.ny, steps) == (256, 512, 1000)

    def ctx_for(params):
        ctx = pearl_gpu.Context(params, w.nx, w.ny)
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        return ctx

    with ctx_for(W.perturb(w.params, w.meta["target_rel"])) as ctx:
        assert ctx.run(steps).steps == steps
        target = np.ascontiguousarray(ctx.download()[0][..., 0])
    with ctx_for(w.params) as ctx:
        rep = ctx.adjoint_gradient(steps, every, target)
    assert rep.steps == steps and rep.checkpoints == -(-steps // every)

    # the CPU reference gradient of the same run
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc, orep = port.adjoint_gradient(w.params, phi, c, mu, s, steps, every, target)
    assert rc == 0
    assert rep.objective == pytest.approx(orep.objective, rel=1e-8)
    for k in range(3):
        assert rep.grad[k] == pytest.approx(orep.grad[k], rel=1e-4), W.ADJOINT_PARAMETERS[k]

    # central differences of the device forward
    base = [1.0, w.params["sigma"], w.params["D"][2]]
    h = 1e-6
    for k in range(3):
        J = []
        for sign in (1, -1):
            rel = [0.0, 0.0, 0.0]
            rel[k] = sign * h
            with ctx_for(W.perturb(w.params, rel)) as ctx:
                assert ctx.run(steps).steps == steps
                J.append(float(((ctx.download()[0][..., 0] - target) ** 2).sum()))
        fd = (J[0] - J[1]) / (2 * h * base[k])
        assert rep.grad[k] == pytest.approx(fd, rel=1e-4), W.ADJOINT_PARAMETERS[k]
