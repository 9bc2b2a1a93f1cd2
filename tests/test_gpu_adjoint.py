"""Device adjoint (pearl_gpu_adjoint_gradient) against the CPU reference
gradient (oracle/pearl_adjoint.c) and against central finite differences of
the device forward (h = 1e-6 relative; agreement 1e-4 relative)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = 1e-6
RTOL = 1e-4


def _case(nx=64, ny=96, steps=60, pairs=1):
    from pearl_gpu import workloads as W

    return W.adjoint_case(nx, ny, pairs=pairs, steps=steps, front=24.0)


def _ctx(w, params=None):
    import pearl_gpu

    ctx = pearl_gpu.Context(params or w.params, w.nx, w.ny)
    ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
    return ctx


def _target(w, steps):
    from pearl_gpu import workloads as W

    with _ctx(w, W.perturb(w.params, w.meta["target_rel"])) as ctx:
        ctx.run(steps)
        return np.ascontiguousarray(ctx.download()[0][..., 0])


def _objective(w, params, steps, target):
    with _ctx(w, params) as ctx:
        r = ctx.run(steps)
        assert r.steps == steps
        phi = ctx.download()[0]
    return float(((phi[..., 0] - target) ** 2).sum())


def test_adjoint_matches_cpu_reference_gradient(gpu_lib, port):
    from oracle import pyoracle

    steps = 60
    w = _case(steps=steps)
    target = _target(w, steps)
    with _ctx(w) as ctx:
        rep = ctx.adjoint_gradient(steps, 25, target)
        phi_g = ctx.download()[0]
    with _ctx(w) as ctx:
        ctx.run(steps)
        phi_f = ctx.download()[0]
    # the context is left in the forward's final state
    assert np.array_equal(phi_g, phi_f)
    assert rep.steps == steps and rep.checkpoints == 3
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc, orep = port.adjoint_gradient(w.params, phi, c, mu, s, steps, 25, target)
    assert rc == 0
    assert rep.objective == pytest.approx(orep.objective, rel=1e-8)
    for k in range(3):
        assert rep.grad[k] == pytest.approx(orep.grad[k], rel=RTOL)


def test_adjoint_matches_central_differences(gpu_lib):
    from pearl_gpu import workloads as W

    steps = 60
    w = _case(steps=steps)
    target = _target(w, steps)
    with _ctx(w) as ctx:
        rep = ctx.adjoint_gradient(steps, 20, target)
    base = [1.0, w.params["sigma"], w.params["D"][2]]
    for k in range(3):
        J = []
        for sign in (1, -1):
            rel = [0.0, 0.0, 0.0]
            rel[k] = sign * H
            J.append(_objective(w, W.perturb(w.params, rel), steps, target))
        fd = (J[0] - J[1]) / (2 * H * base[k])
        assert rep.grad[k] == pytest.approx(fd, rel=RTOL), W.ADJOINT_PARAMETERS[k]


def test_adjoint_checkpoint_interval_and_repeat(gpu_lib):
    """The gradient does not depend on the checkpoint interval, and a second call
    from the restored initial state reproduces the first bitwise."""
    steps = 40
    w = _case(nx=96, ny=64, steps=steps, pairs=2)
    target = np.ascontiguousarray(w.phi[..., 0] * 0.9)
    reps = []
    for every in (7, 40):
        with _ctx(w) as ctx:
            reps.append(ctx.adjoint_gradient(steps, every, target))
    with _ctx(w) as ctx:
        again = ctx.adjoint_gradient(steps, 7, target)
    assert reps[0].objective == reps[1].objective
    for k in range(3):
        assert reps[1].grad[k] == pytest.approx(reps[0].grad[k], rel=1e-12)
        assert again.grad[k] == reps[0].grad[k]


def test_autograd_function_wrapper(gpu_lib):
    """The C-ABI gradient as a torch.autograd.Function (test harness only): theta are
    multipliers of (mobility, sigma, D_gamma); backward returns dJ/dtheta."""
    import torch

    from pearl_gpu import workloads as W

    steps = 40
    w = _case(nx=64, ny=64, steps=steps)
    target = _target(w, steps)
    base = [1.0, w.params["sigma"], w.params["D"][2]]

    class Misfit(torch.autograd.Function):
        @staticmethod
        def forward(fctx, theta):
            rel = [float(t) - 1.0 for t in theta.detach().cpu()]
            params = W.perturb(w.params, rel)
            with _ctx(w, params) as ctx:
                rep = ctx.adjoint_gradient(steps, 10, target)
            th = [float(t) for t in theta.detach().cpu()]
            # the context's own mobility scale M multiplies theta_0; sigma and D_gamma scale linearly
            g = [rep.grad[0] / th[0], rep.grad[1] * base[1], rep.grad[2] * base[2]]
            fctx.save_for_backward(torch.tensor(g, dtype=torch.float64))
            return torch.tensor(rep.objective, dtype=torch.float64)

        @staticmethod
        def backward(fctx, gout):
            (g,) = fctx.saved_tensors
            return gout * g

    theta = torch.tensor([1.02, 0.97, 1.01], dtype=torch.float64, requires_grad=True)
    J = Misfit.apply(theta)
    J.backward()
    h = 1e-6
    for k in range(3):
        Js = []
        for sign in (1, -1):
            t = theta.detach().clone()
            t[k] += sign * h
            rel = [float(x) - 1.0 for x in t]
            Js.append(_objective(w, W.perturb(w.params, rel), steps, target))
        fd = (Js[0] - Js[1]) / (2 * h)
        assert float(theta.grad[k]) == pytest.approx(fd, rel=RTOL)


def test_adjoint_refuses_mixed_precision(gpu_lib):
    import pearl_gpu

    w = _case(nx=32, ny=32, steps=4)
    with _ctx(w) as ctx:
        ctx.set_precision("mixed")
        with pytest.raises(pearl_gpu.PearlError, match="FP64"):
            ctx.adjoint_gradient(4, 2, np.zeros((w.ny, w.nx)))
