"""The CPU reference gradient (oracle/pearl_adjoint.c) against central finite
differences of the oracle's own forward (h = 1e-6 relative, agreement 1e-4
relative), and independence of the checkpoint interval."""
from __future__ import annotations

import numpy as np
import pytest

from pearl_gpu import workloads as W

H = 1e-6
RTOL = 1e-4


def _case(nx=48, ny=64, steps=30):
    w = W.adjoint_case(nx, ny, pairs=1, steps=steps, front=16.0)
    return w, steps


def _forward(port, w, params, steps):
    from oracle import pyoracle

    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc, why, done, _ = port.advance_n(params, phi, c, mu, s, steps)
    assert rc == 0, why
    return phi


def _target(port, w, steps):
    return np.ascontiguousarray(_forward(port, w, W.perturb(w.params, w.meta["target_rel"]), steps)[..., 0])


def _gradient(port, w, steps, every, target):
    from oracle import pyoracle

    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc, rep = port.adjoint_gradient(w.params, phi, c, mu, s, steps, every, target)
    assert rc == 0
    return rep, phi


def _objective(port, w, params, steps, target):
    from oracle import pyoracle

    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc, J = port.adjoint_objective(params, phi, c, mu, s, steps, target)
    assert rc == 0
    return J


def test_oracle_gradient_matches_central_differences(port):
    w, steps = _case()
    target = _target(port, w, steps)
    rep, _ = _gradient(port, w, steps, 10, target)
    assert rep.objective > 0
    base = [1.0, w.params["sigma"], w.params["D"][2]]
    for k in range(3):
        J = []
        for sign in (1, -1):
            rel = [0.0, 0.0, 0.0]
            rel[k] = sign * H
            J.append(_objective(port, w, W.perturb(w.params, rel), steps, target))
        fd = (J[0] - J[1]) / (2 * H * base[k])
        assert rep.grad[k] == pytest.approx(fd, rel=RTOL), W.ADJOINT_PARAMETERS[k]


def test_oracle_gradient_checkpoint_independent(port):
    """Segments of 7, 30 and 100 steps give the same gradient and the same final state."""
    w, steps = _case(steps=30)
    target = _target(port, w, steps)
    reps = [_gradient(port, w, steps, every, target) for every in (7, 30, 100)]
    for rep, phi in reps[1:]:
        assert rep.objective == reps[0][0].objective
        assert np.array_equal(phi, reps[0][1])
        for k in range(3):
            assert rep.grad[k] == pytest.approx(reps[0][0].grad[k], rel=1e-12)


def test_oracle_gradient_final_state_is_forward(port):
    w, steps = _case(steps=12)
    target = np.zeros((w.ny, w.nx))
    _, phi = _gradient(port, w, steps, 5, target)
    assert np.array_equal(phi, _forward(port, w, w.params, steps))
