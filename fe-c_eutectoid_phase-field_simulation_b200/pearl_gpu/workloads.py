"""Seeded synthetic lamellar pearlite inputs.

The reference publishes no benchmark fields, so every workload here is
generated from a seed with numpy's PCG64 generator, in the reference's axes:
x (``nx``, the lamellar direction) is periodic, y (``ny``, the growth
direction) has zero-flux walls and the transformation front moves towards +y
(pearl_serial.cpp:581-583, :692-693).

Geometry of every workload: lamellar pairs of ferrite (alpha) and cementite
(theta) columns fill the rows below a front; austenite (gamma) fills the rest.
Interfaces are tanh profiles ``0.5*(1 - tanh(d/delta))`` with ``delta`` = 2
cells: 4 cells wide between 12% and 88% (the tanh width 2*delta).  A 1-cell
delta with the +-1-row front jitter is sharper than the model can relax: the
reference itself then shrinks dt below dt_min within ~35 steps.  Phase fractions are built like the
reference's ``lamella`` initialisation (pearl_serial.cpp:1768-1770):
``phi = ((1-Theta)*P, Theta*P, 1-P)``.  The chemical potential starts uniform
at the eutectoid austenite composition and carbon is ``c = chi*mu + c0`` per
cell, so the initial state is closed (pearl_serial.cpp:1823-1826).

Thermodynamics come from the reference's example input
``examples/fe_c_phase_diagram_10K.in`` (supplied eutectoid ABC plus
phase-diagram slopes) evaluated at the requested undercooling with the
``phase_diagram_fixed_curvature`` law (pearl_serial.cpp:236-276), computed in
80-bit extended precision exactly as the reference does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np

# examples/fe_c_phase_diagram_10K.in (values at T_eutectoid = 999.68459774 K)
FE_C_REFERENCE = dict(
    T_eutectoid=999.68459774,
    Aeq=(4724862.6373624019, 100000000.0, 172591.65731409981),
    Beq=(22964.296428571855, -49968654.66102279, 19450.725112218221),
    Ceq=(-42255.03701292308, 6207741.2462954065, -42053.816371518253),
    D=(2e-9, 2e-9, 1e-9),
    ceq=(0.00088690859310575857, 0.25, 0.034458832049305582),
    # alpha on a/g, gamma on a/g, theta on t/g, gamma on t/g  [dc/dT]
    slopes=(-4.6282639461434345e-06, -0.00031198492411304955, 0.0, 0.00010753713136114516),
    Vm=1e-6,
    epsilon=14e-9,
    sigma=0.5,
    triple=10.0,
    tau=(1.72402799784e8, 1.72402799784e8, 7.11828875478e9),
    gamma_carbon=0.034458832049305582,
)


def fma(a: float, b: float, c: float) -> float:
    """Correctly rounded a*b+c (Python 3.12 has no math.fma)."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def phase_diagram_thermo(undercooling: float, ref: dict = FE_C_REFERENCE):
    """A, B, C per phase at T_E - undercooling (pearl_serial.cpp:236-276).

    Uses numpy's 80-bit long double, the same format as the reference's
    ``long double`` on x86-64, in the reference's operation order.
    """
    L = np.longdouble
    A = list(ref["Aeq"])
    B = list(ref["Beq"])
    Cc = list(ref["Ceq"])
    if not math.isfinite(undercooling) or undercooling < 0:
        raise ValueError("undercooling must be finite and nonnegative")
    dT = -L(undercooling)
    gA = L(ref["Aeq"][2])
    gcE = L(ref["ceq"][2])
    for product in (0, 1):
        pA = L(ref["Aeq"][product])
        pcE = L(ref["ceq"][product])
        pcc = dT * L(ref["slopes"][2 * product])
        gcc = dT * L(ref["slopes"][2 * product + 1])
        pc, gc = pcE + pcc, gcE + gcc
        if not (0 <= pc <= 1 and 0 <= gc <= 1):
            raise ValueError("phase-diagram extrapolated carbon outside [0,1]")
        if undercooling == 0:
            continue
        B[product] = float(L(ref["Beq"][product]) + 2 * (gA * gcc - pA * pcc))
        Cc[product] = float(L(ref["Ceq"][product]) + pA * pcc * (2 * pcE + pcc) - gA * gcc * (2 * gcE + gcc))
    return A, B, Cc


@dataclass
class Workload:
    """Initial fields plus the parameters of one synthetic instance."""

    name: str
    nx: int
    ny: int
    params: dict
    phi: np.ndarray  # [ny, nx, 3]
    carbon: np.ndarray  # [ny, nx]
    mu: np.ndarray  # [ny, nx]
    scalars: dict
    meta: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nx * self.ny


def make_params(nx: int, ny: int, dx: float, undercooling: float, dt: float, dt_max: float | None = None,
                dt_min: float | None = None, ref: dict = FE_C_REFERENCE, **controls) -> dict:
    """Solver parameters with the reference's defaults (pearl_serial.cpp:767-773, :1721-1740)."""
    A, B, Cc = phase_diagram_thermo(undercooling, ref)
    dy = controls.pop("dy", dx)
    p = dict(
        A=A, B=B, C=Cc, D=list(ref["D"]),
        Vm=ref["Vm"], epsilon=ref["epsilon"], sigma=ref["sigma"], triple=ref["triple"],
        tau=list(ref["tau"]), dx=dx, dy=dy,
        dt_max=dt if dt_max is None else dt_max,
        dt_min=dt / 1048576.0 if dt_min is None else dt_min,
        max_phase_change=0.04, cg_rtol=1e-11, cg_atol=1e-14, closure_tol=1e-10,
        energy_rtol=1e-11, energy_atol=1e-13 * ref["sigma"] * max(nx * dx, ny * dy),
        cg_max=2000, max_retries=24, check_energy=1, phase_only=0,
    )
    # gamma_carbon -> mu = 2*A_gamma*c + B_gamma (Parabola::mu, pearl_serial.cpp:84; :1734)
    p["mu_reference"] = fma(2.0 * A[2], ref["gamma_carbon"], B[2])
    p.update(controls)
    return p


def _mixture(phi: np.ndarray, params: dict):
    p0, p1, p2 = phi[..., 0], phi[..., 1], phi[..., 2]
    triple = 2.0 * p0 * p1 * p2
    chi = np.zeros(phi.shape[:-1])
    c0 = np.zeros(phi.shape[:-1])
    for q, pq in enumerate((p0, p1, p2)):
        h = pq * pq * (3.0 - 2.0 * pq) + triple
        cq = 1.0 / (2.0 * params["A"][q])
        chi += h * cq
        c0 -= h * cq * params["B"][q]
    return chi, c0


def lamellar_phi(nx: int, ny: int, widths, theta_widths, front_rows, delta: float = 2.0) -> np.ndarray:
    """phi[ny, nx, 3] for lamellar pairs (theta first in each pair) below per-column fronts."""
    widths = np.asarray(widths, dtype=np.int64)
    assert int(widths.sum()) == nx
    xc = np.arange(nx, dtype=np.float64) + 0.5
    theta = np.zeros(nx)
    start = 0
    for w, t in zip(widths, theta_widths):
        a, b = float(start), float(start + t)
        for img in (-nx, 0, nx):
            theta += 0.5 * (np.tanh((xc - (a + img)) / delta) - np.tanh((xc - (b + img)) / delta))
        start += int(w)
    theta = np.clip(theta, 0.0, 1.0)
    yc = np.arange(ny, dtype=np.float64)[:, None] + 0.5
    front = np.asarray(front_rows, dtype=np.float64)[None, :]
    P = 0.5 * (1.0 - np.tanh((yc - front) / delta))
    phi = np.empty((ny, nx, 3))
    phi[..., 0] = (1.0 - theta)[None, :] * P
    phi[..., 1] = theta[None, :] * P
    phi[..., 2] = 1.0 - P
    return np.ascontiguousarray(phi)


def _finish(name, nx, ny, params, phi, meta) -> Workload:
    mu0 = params["mu_reference"]
    chi, c0 = _mixture(phi, params)
    carbon = np.ascontiguousarray(chi * mu0 + c0)
    mu = np.full((ny, nx), mu0)
    dx, dy = params["dx"], params["dy"]
    scalars = dict(time=0.0, dt=meta["dt"], shift_distance=0.0,
                   initial_carbon=float(carbon.sum()) * dx * dy,
                   carbon_added=0.0, carbon_removed=0.0, step=0, shifts=0, rejected=0)
    return Workload(name, nx, ny, params, phi, carbon, mu, scalars, meta)


def jittered_pairs(nx: int, pairs: int, rng: np.random.Generator, jitter: float, ferrite_fraction: float):
    """Integer pair widths with spacing nx/pairs*(1+U(-jitter,jitter)), renormalised to sum nx."""
    raw = (nx / pairs) * (1.0 + rng.uniform(-jitter, jitter, size=pairs))
    raw *= nx / raw.sum()
    widths = np.floor(raw).astype(np.int64)
    rem = nx - int(widths.sum())
    order = np.argsort(-(raw - widths))
    widths[order[:rem]] += 1
    thetas = np.maximum(1, np.rint(widths * (1.0 - ferrite_fraction)).astype(np.int64))
    return widths, thetas


def plain_small(seed: int = 0) -> Workload:
    """FP64 small: nx=128 (4 pairs of 28 alpha + 4 theta), ny=256, front at row 32,
    dx=2 nm, 10 K undercooling, fixed dt = dt_max = 4e-12 s."""
    nx, ny, dx, dt = 128, 256, 2e-9, 4e-12
    params = make_params(nx, ny, dx, undercooling=10.0, dt=dt)
    phi = lamellar_phi(nx, ny, [32] * 4, [4] * 4, np.full(nx, 32.0))
    return _finish("plain_small_128x256", nx, ny, params, phi, dict(dt=dt, seed=seed, pairs=4, steps=2000))


def plain_large(seed: int = 0, nx: int = 2048, ny: int = 4096, pairs: int = 64) -> Workload:
    """FP64 large: nx=2048 (64 pairs, spacing 32 +-10% jitter, ferrite fraction 0.875),
    ny=4096, fronts at row 32 + U{-1,0,1}, 20 K undercooling, adaptive dt, moving window."""
    rng = np.random.default_rng(seed)
    dx, dt = 2e-9, 4e-12
    params = make_params(nx, ny, dx, undercooling=20.0, dt=dt, dt_max=8e-12)
    widths, thetas = jittered_pairs(nx, pairs, rng, 0.10, 0.875)
    fronts = 32.0 + rng.integers(-1, 2, size=nx)
    phi = lamellar_phi(nx, ny, widths, thetas, fronts)
    meta = dict(dt=dt, seed=seed, pairs=pairs, steps=20000, moving_window=True,
                shift_trigger=0.65 * ny * dx, shift_target=0.35 * ny * dx,
                shift_gamma_carbon=FE_C_REFERENCE["gamma_carbon"])
    return _finish(f"plain_large_{nx}x{ny}", nx, ny, params, phi, meta)


def scaled(nx: int, ny: int, seed: int = 0, undercooling: float = 10.0, dt: float = 4e-12,
           dt_max: float | None = None, pairs: int | None = None, jitter: float = 0.0,
           front_jitter: int = 0, front: float = 32.0, **controls) -> Workload:
    """Generic lamellar instance for parity tests at arbitrary sizes."""
    rng = np.random.default_rng(seed)
    dx = controls.pop("dx", 2e-9)
    params = make_params(nx, ny, dx, undercooling=undercooling, dt=dt, dt_max=dt_max, **controls)
    pairs = pairs or max(1, nx // 32)
    widths, thetas = jittered_pairs(nx, pairs, rng, jitter, 0.875)
    fronts = front + (rng.integers(-front_jitter, front_jitter + 1, size=nx) if front_jitter else 0.0)
    phi = lamellar_phi(nx, ny, widths, thetas, np.broadcast_to(fronts, (nx,)))
    return _finish(f"scaled_{nx}x{ny}", nx, ny, params, phi, dict(dt=dt, seed=seed, pairs=pairs))


def sweep_instance(i: int, rng: np.random.Generator, dt: float = 4e-12) -> Workload:
    """One instance of the parameter sweep: 2 lamellar pairs of spacing U{16..96}
    cells across x (nx = 2 spacings), growth length ny = U{64..1024} cells,
    ferrite fraction U(0.85, 0.90), undercooling U(5, 40) K, adaptive dt."""
    spacing = int(rng.integers(16, 97))
    ny = int(rng.integers(64, 1025))
    ferrite = float(rng.uniform(0.85, 0.90))
    undercooling = float(rng.uniform(5.0, 40.0))
    nx = 2 * spacing
    dx = 2e-9
    params = make_params(nx, ny, dx, undercooling=undercooling, dt=dt, dt_max=2 * dt)
    widths, thetas = jittered_pairs(nx, 2, rng, 0.0, ferrite)
    phi = lamellar_phi(nx, ny, widths, thetas, np.full(nx, 32.0))
    meta = dict(dt=dt, index=i, spacing=spacing, ferrite_fraction=ferrite, undercooling=undercooling)
    return _finish(f"sweep_{i}_{nx}x{ny}", nx, ny, params, phi, meta)


def sweep_one(i: int, seed: int = 0) -> Workload:
    """Instance i of the sweep drawn from `seed` (its own stream, so any instance
    can be built alone)."""
    return sweep_instance(i, np.random.default_rng([seed, i]))


def sweep(n: int = 256, seed: int = 0) -> list[Workload]:
    """n sweep instances drawn from one seed (the batched-sweep workload)."""
    return [sweep_one(i, seed) for i in range(n)]


ADJOINT_PARAMETERS = ("mobility", "sigma", "D_gamma")


def perturb(params: dict, rel) -> dict:
    """Parameters with the mobility scale (every 1/tau), sigma and D_gamma scaled by
    (1 + rel[0]), (1 + rel[1]), (1 + rel[2])."""
    p = dict(params)
    p["tau"] = [t / (1.0 + rel[0]) for t in params["tau"]]
    p["sigma"] = params["sigma"] * (1.0 + rel[1])
    D = list(params["D"])
    D[2] = D[2] * (1.0 + rel[2])
    p["D"] = D
    return p


def adjoint_case(nx: int = 256, ny: int = 512, pairs: int = 4, steps: int = 1000, seed: int = 0,
                 undercooling: float = 15.0, dt: float = 2e-12, front: float = 32.0) -> Workload:
    """Adjoint workload: lamellar pairs (spacing nx/pairs, ferrite fraction 0.875), fixed dt
    (dt_max = dt = 2e-12 s, small enough that no step is rejected at 15 K), `steps` steps.
    meta['target_rel'] holds the seeded U(-5%, 5%) perturbation of (mobility, sigma,
    D_gamma) whose forward run defines the target."""
    rng = np.random.default_rng(seed)
    dx = 2e-9
    params = make_params(nx, ny, dx, undercooling=undercooling, dt=dt)
    widths, thetas = jittered_pairs(nx, pairs, rng, 0.0, 0.875)
    phi = lamellar_phi(nx, ny, widths, thetas, np.full(nx, front))
    rel = [float(v) for v in rng.uniform(-0.05, 0.05, size=3)]
    meta = dict(dt=dt, seed=seed, pairs=pairs, steps=steps, target_rel=rel)
    return _finish(f"adjoint_{nx}x{ny}", nx, ny, params, phi, meta)
