"""The device divides by the reference's constant divisors (Vm, dx, dy, dx*dx,
dy*dy, 3, 2A) with a precomputed reciprocal and two FMA residual corrections.
These tests show that this equals IEEE division bitwise: on the CPU for the
algorithm itself (exact rational FMA), and on the GPU for the device code."""
from __future__ import annotations

from fractions import Fraction

import numpy as np
import pytest


def _fma(a: float, b: float, c: float) -> float:
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _div_by(a: float, b: float, rb: float) -> float:
    q0 = a * rb
    if a == 0.0 or not np.isfinite(q0):
        return q0
    r = _fma(-q0, b, a)
    q = _fma(r, rb, q0)
    r = _fma(-q, b, a)
    return _fma(r, rb, q)


def _divisors():
    from pearl_gpu import workloads

    p = workloads.make_params(128, 256, 2e-9, 10.0, 4e-12)
    out = [p["Vm"], 2e-9, 2.79e-9, 2e-9 * 2e-9, 2.79e-9 * 2.79e-9, 3.0]
    out += [2.0 * A for A in p["A"]]
    for u in (15.0, 20.0, 37.5):
        out += [2.0 * A for A in workloads.make_params(64, 64, 2e-9, u, 4e-12)["A"]]
    return out


def _numerators(rng, n, b):
    mags = 10.0 ** rng.uniform(-150, 150, n)
    a = mags * rng.choice([-1.0, 1.0], n)
    k = rng.integers(-10**6, 10**6, n // 8).astype(np.float64)
    a[: n // 8] = k * b  # exact quotients
    a[n // 8: n // 4] = np.nextafter(b * rng.uniform(0.5, 2.0, n // 8), np.inf)
    a[n // 4: n // 4 + 16] = [0.0, -0.0, 1.0, -1.0, 3.0, 1.5, 0.1, 1e-300, 1e300, 2.0 ** -1000,
                              2.0 ** 1000, 5e-324 * 2**60, 7.0, 1 / 3, 2 / 3, 123456789.0]
    return a


def test_division_algorithm_exact_on_cpu():
    rng = np.random.default_rng(11)
    for b in _divisors():
        rb = 1.0 / b
        for a in _numerators(rng, 400, b):
            q = _div_by(float(a), b, rb)
            ref = float(a) / b
            assert q == ref and np.signbit(q) == np.signbit(ref), (a, b)


def _div_force(a: float, b: float, rb: float) -> float:
    """The proposal's variant: the corrections applied to every numerator, the
    numerator's sign bit OR-ed into the result (no tests on the operands)."""
    q0 = a * rb
    r = _fma(-q0, b, a)
    q = _fma(r, rb, q0)
    r = _fma(-q, b, a)
    q = _fma(r, rb, q)
    return -abs(q) if np.signbit(a) else q


def test_force_division_exact_for_finite_quotients_on_cpu():
    """div_force equals IEEE division, sign of zero included, for the positive
    constant divisors and every finite numerator whose quotient is a normal
    number (the proposal's forces are far inside that range; a non-finite force
    takes the reference's non-finite branch whatever its value)."""
    rng = np.random.default_rng(12)
    for b in _divisors():
        if b <= 0:
            continue
        rb = 1.0 / b
        for a in _numerators(rng, 400, b):
            a = float(a)
            ref = a / b
            if not np.isfinite(ref) or (ref != 0.0 and abs(ref) < np.finfo(float).tiny):
                continue
            q = _div_force(a, b, rb)
            assert q == ref and np.signbit(q) == np.signbit(ref), (a, b)


@pytest.mark.gpu
def test_division_device_exact(gpu_lib):
    import pearl_gpu

    rng = np.random.default_rng(5)
    n = 1 << 21
    total = 0
    for b in _divisors():
        a = _numerators(rng, n, b)
        total += pearl_gpu.selftest_division(a, np.full(n, b))
    # random normal divisors too
    bs = 10.0 ** rng.uniform(-100, 100, n) * rng.choice([-1.0, 1.0], n)
    a = 10.0 ** rng.uniform(-100, 100, n) * rng.choice([-1.0, 1.0], n)
    total += pearl_gpu.selftest_division(a, bs)
    assert total == 0
