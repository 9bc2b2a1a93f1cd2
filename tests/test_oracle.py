"""CPU checks of the test oracle (pearl_oracle.c) against the reference.

1. Golden fixtures written by tests/golden/make_golden.py from the unmodified
   reference solver: the C restatement must reproduce them bitwise (this runs
   everywhere, including hosts where the reference source is absent).
2. Known answers published in the reference's documentation
   (NEW_FREE_ENERGY.md:42-43, :116-133).
3. Where the reference is built here: live bitwise comparison on longer runs.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def golden():
    data = np.load(GOLDEN / "pearl_ref_golden.npz")
    meta = json.loads((GOLDEN / "pearl_ref_golden.json").read_text())
    return data, meta


def params_from(vec, meta) -> dict:
    out, k = {}, 0
    for name in meta["param_keys"]:
        if name in ("A", "B", "C", "D", "tau"):
            out[name] = [float(v) for v in vec[k:k + 3]]
            k += 3
        else:
            v = float(vec[k])
            out[name] = int(v) if name in ("cg_max", "max_retries", "check_energy", "phase_only") else v
            k += 1
    return out


def scalars_from(vec, meta):
    from oracle import pyoracle

    s = pyoracle.PoScalars()
    for name, v in zip(meta["scalar_keys"], vec):
        setattr(s, name, int(v) if name in ("step", "shifts", "rejected") else float(v))
    return s


def _svec(s, meta):
    return np.array([getattr(s, k) for k in meta["scalar_keys"]], dtype=np.float64)


def test_golden_advance(port, golden):
    data, meta = golden
    p = params_from(data["adv_params"], meta)
    phi, c, mu = data["adv_phi0"].copy(), data["adv_c0"].copy(), data["adv_mu0"].copy()
    s = scalars_from(data["adv_s0"], meta)
    rc, why, done, infos = port.advance_n(p, phi, c, mu, s, meta["cases"]["adv"]["steps"])
    assert rc == 0, why
    assert np.array_equal(phi, data["adv_phi"])
    assert np.array_equal(c, data["adv_c"])
    assert np.array_equal(mu, data["adv_mu"])
    assert np.array_equal(_svec(s, meta), data["adv_s"])
    got = np.array([[getattr(i, k) for k in meta["info_keys"]] for i in infos])
    assert np.array_equal(got, data["adv_info"])
    assert s.rejected == meta["cases"]["adv"]["rejected"] > 0


def test_golden_propose_diffusion_energy(port, golden):
    data, meta = golden
    p = params_from(data["adv_params"], meta)
    phi, c, mu = data["adv_phi0"], data["adv_c0"], data["adv_mu0"]
    for tag in ("prop_a", "prop_b"):
        change_ref, dt = data[f"{tag}_change"]
        rc, trial, change = port.propose_phi(p, phi, mu, dt)
        assert rc == 0
        assert change == change_ref
        assert np.array_equal(trial, data[f"{tag}_trial"])
    rc, trial, _ = port.propose_phi(p, phi, mu, 4e-12)
    rc, tc, tmu, info = port.implicit_diffusion(p, c, mu, trial, 4e-12)
    assert rc == 0
    assert np.array_equal(tc, data["diff_c"]) and np.array_equal(tmu, data["diff_mu"])
    assert [info.ok, info.it, info.residual, info.closure] == list(data["diff_info"])
    rc, e, m = port.energy_and_mass(p, phi, c)
    assert [e, m, port.valid_state(p, phi, c, mu)] == list(data["energy_mass"])


def test_golden_phase_only(port, golden):
    data, meta = golden
    p = params_from(data["po_params"], meta)
    assert p["phase_only"] == 1
    phi, c, mu = data["po_phi0"].copy(), data["po_c0"].copy(), data["po_mu0"].copy()
    s = scalars_from(data["po_s0"], meta)
    rc, why, done, infos = port.advance_n(p, phi, c, mu, s, 8)
    assert rc == 0, why
    for got, key in ((phi, "po_phi"), (c, "po_c"), (mu, "po_mu")):
        assert np.array_equal(got, data[key])
    assert np.array_equal(_svec(s, meta), data["po_s"])


def test_golden_moving_window(port, golden):
    data, meta = golden
    p = params_from(data["sh_params"], meta)
    phi, c, mu = data["sh_phi0"].copy(), data["sh_c0"].copy(), data["sh_mu0"].copy()
    s = scalars_from(data["sh_s0"], meta)
    trig, targ, cg = data["sh_args"]
    rc, rows = port.maybe_shift(p, phi, c, mu, s, trig, targ, cg)
    assert rc == 0 and rows > 0
    for got, key in ((phi, "sh_phi"), (c, "sh_c"), (mu, "sh_mu")):
        assert np.array_equal(got, data[key])
    assert np.array_equal(_svec(s, meta), data["sh_s"])


def test_golden_smoothing(port, golden):
    data, meta = golden
    p = params_from(data["adv_params"], meta)
    phi = data["sm_phi0"].copy()
    rc, rep = port.smooth(p, phi, 20, 20, 1e-10, 0.02)
    assert rc == 0
    assert np.array_equal(phi, data["sm_phi"])
    got = [rep.steps, rep.converged, rep.energy_initial, rep.energy_final, rep.final_relative_energy_change,
           rep.final_max_phase_change]
    assert got == list(data["sm_rep"])


def test_golden_error_message(port, golden):
    data, meta = golden
    p = params_from(data["err_params"], meta)
    from pearl_gpu import workloads

    w = workloads.scaled(48, 40, seed=1, front=10.0, jitter=0.1, front_jitter=1, dt=2e-10, dt_min=2e-10)
    from oracle import pyoracle

    s = pyoracle.scalars_from(w.scalars)
    rc, why, done, _ = port.advance_n(p, w.phi.copy(), w.carbon.copy(), w.mu.copy(), s, 1)
    assert rc == 4  # rejected below dt_min
    assert meta["cases"]["err"]["message"] == "step rejected below dt_min: " + why


def test_golden_temperature_law(golden):
    from pearl_gpu import workloads

    data, _ = golden
    for row in data["thermo"]:
        u = row[0]
        A, B, C = workloads.phase_diagram_thermo(u)
        for i in range(3):
            assert (A[i], B[i], C[i]) == tuple(row[1 + 4 * i: 4 + 4 * i])


def test_known_answers_new_free_energy():
    """Known answers of NEW_FREE_ENERGY.md (10 K phase-diagram law)."""
    from oracle import pyoracle
    from pearl_gpu import workloads

    A, B, C = workloads.phase_diagram_thermo(10.0)
    # effective ABC at 10 K (NEW_FREE_ENERGY.md:116-120)
    assert B[0] == pytest.approx(23603.858102865859, rel=1e-15)
    assert C[0] == pytest.approx(-42293.428311015959, rel=1e-15)
    assert B[1] == pytest.approx(-49969025.861257277, rel=1e-15)
    assert C[1] == pytest.approx(6207753.8378329016, rel=1e-15)
    assert (A[2], B[2], C[2]) == (172591.65731409981, 19450.725112218221, -42053.816371518253)
    p = workloads.make_params(64, 64, 2e-9, 10.0, 4e-12)
    # initial chemical potential near 31345.33897721396 J/mol (NEW_FREE_ENERGY.md:42-43)
    assert p["mu_reference"] == pytest.approx(31345.33897721396, abs=1e-9)
    port = pyoracle.port()
    mu = p["mu_reference"]
    # product-minus-gamma grand potential differences (NEW_FREE_ENERGY.md:122-126)
    psi = [port.psi(p, a, mu) for a in range(3)]
    assert psi[0] - psi[2] == pytest.approx(-37.8457083, abs=5e-8)
    assert psi[1] - psi[2] == pytest.approx(-80.2089479, abs=5e-8)
    # shifted pair contacts (NEW_FREE_ENERGY.md:128-133)
    r = workloads.FE_C_REFERENCE
    assert r["ceq"][0] + (-10.0) * r["slopes"][0] == pytest.approx(0.00093319123256719, rel=1e-12)
    assert r["ceq"][2] + (-10.0) * r["slopes"][1] == pytest.approx(0.037578681290436, rel=1e-12)
    assert r["ceq"][2] + (-10.0) * r["slopes"][3] == pytest.approx(0.033383460735694, rel=1e-12)


def test_port_matches_reference_live(port, reference):
    """128x256 lamellar input, 60 coupled steps with rejections: bitwise."""
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.plain_small()
    out = []
    for lib in (port, reference):
        phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        s = pyoracle.scalars_from(w.scalars)
        rc = lib.advance_n(w.params, phi, c, mu, s, 60)
        assert rc[0] == 0
        out.append((phi, c, mu, s.time, s.rejected, [(i.cg_iterations, i.retries) for i in rc[3]]))
    for a, b in zip(out[0], out[1]):
        if isinstance(a, np.ndarray):
            assert np.array_equal(a, b)
        else:
            assert a == b


def test_port_matches_reference_golden_at_config_horizon(port):
    """The small FP64 configuration at its own horizon: 2000 accepted steps of
    the C restatement equal the reference's own run (tests/golden/
    make_horizon_golden.py) bitwise, every step's decisions included (about
    20 s of CPU)."""
    from oracle import pyoracle
    from pearl_gpu import workloads

    ref = np.load(GOLDEN / "horizon_fields.npz")
    w = workloads.plain_small()
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc, why, done, infos = port.advance_n(w.params, phi, c, mu, s, 2000)
    assert rc == 0 and done == 2000, why
    assert [i.retries for i in infos] == ref["steps/retries"][:2000].tolist()
    assert [i.cg_iterations for i in infos] == ref["steps/cg_iterations"][:2000].tolist()
    assert [i.accepted_dt for i in infos] == ref["steps/accepted_dt"][:2000].tolist()
    assert np.array_equal(phi, ref["s2000/phi"])
    assert np.array_equal(c, ref["s2000/carbon"])
    assert np.array_equal(mu, ref["s2000/mu"])
    assert (s.time, s.dt, float(s.step), float(s.rejected)) == tuple(ref["s2000/scalars"])
