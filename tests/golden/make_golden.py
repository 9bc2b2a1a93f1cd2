"""Generate tests/golden/pearl_ref_golden.npz from the reference solver itself.

Runs the UNMODIFIED reference (pearl_serial.cpp, compiled by
oracle/build_oracle.py into oracle/_ref/libpearl_ref.so) on small seeded
inputs and stores inputs and outputs.  Needs the reference source, so it runs
only where that exists; the fixture it writes is committed and pins the C
restatement (and through it the GPU path) everywhere else.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (str(ROOT), str(ROOT / "fe-c_eutectoid_phase-field_simulation_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import pyoracle  # noqa: E402
from pearl_gpu import workloads  # noqa: E402

OUT = HERE / "pearl_ref_golden.npz"
META = HERE / "pearl_ref_golden.json"

PARAM_KEYS = [n for n, _ in pyoracle.PoParams._fields_]
SCALAR_KEYS = [n for n, _ in pyoracle.PoScalars._fields_]
INFO_KEYS = [n for n, _ in pyoracle.PoStepInfo._fields_]


def pvec(params: dict) -> np.ndarray:
    out = []
    for k in PARAM_KEYS:
        v = params[k]
        out.extend(v if isinstance(v, (list, tuple)) else [v])
    return np.array(out, dtype=np.float64)


def svec(s) -> np.ndarray:
    return np.array([getattr(s, k) for k in SCALAR_KEYS], dtype=np.float64)


def ivec(infos) -> np.ndarray:
    return np.array([[getattr(i, k) for k in INFO_KEYS] for i in infos], dtype=np.float64).reshape(-1, len(INFO_KEYS))


def main() -> None:
    ref = pyoracle.reference()
    if ref is None:
        raise SystemExit("the reference solver is not available here")
    data: dict[str, np.ndarray] = {}
    meta: dict = {"param_keys": PARAM_KEYS, "scalar_keys": SCALAR_KEYS, "info_keys": INFO_KEYS, "cases": {}}

    # 1. coupled advance, natural dt (rejections included), 48x40
    w = workloads.scaled(48, 40, seed=1, front=10.0, jitter=0.1, front_jitter=1, dt=8e-12, dt_max=8e-12)
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    data.update(adv_params=pvec(w.params), adv_phi0=w.phi, adv_c0=w.carbon, adv_mu0=w.mu,
                adv_s0=svec(pyoracle.scalars_from(w.scalars)))
    rc, err, done, infos = ref.advance_n(w.params, phi, c, mu, s, 15)
    assert rc == 0, err
    data.update(adv_phi=phi, adv_c=c, adv_mu=mu, adv_s=svec(s), adv_info=ivec(infos))
    meta["cases"]["adv"] = {"nx": 48, "ny": 40, "steps": 15, "rejected": int(s.rejected)}

    # 2. propose_phi and implicit_diffusion on the same input
    for tag, dt in (("prop_a", 4e-12), ("prop_b", 3e-11)):
        rc, trial, change = ref.propose_phi(w.params, w.phi, w.mu, dt)
        assert rc == 0
        data[f"{tag}_trial"] = trial
        data[f"{tag}_change"] = np.array([change, dt])
    rc, trial, _ = ref.propose_phi(w.params, w.phi, w.mu, 4e-12)
    rc, tc, tmu, info = ref.implicit_diffusion(w.params, w.carbon, w.mu, trial, 4e-12)
    assert rc == 0 and info.ok
    data.update(diff_c=tc, diff_mu=tmu, diff_info=np.array([info.ok, info.it, info.residual, info.closure]))

    # 3. energy / mass / valid
    rc, e, m = ref.energy_and_mass(w.params, w.phi, w.carbon)
    data["energy_mass"] = np.array([e, m, ref.valid_state(w.params, w.phi, w.carbon, w.mu)])

    # 4. phase_only advance
    wp = workloads.scaled(40, 32, seed=2, front=8.0, jitter=0.1, dt=4e-12)
    wp.params["phase_only"] = 1
    phi, c, mu = wp.phi.copy(), wp.carbon.copy(), wp.mu.copy()
    s = pyoracle.scalars_from(wp.scalars)
    rc, err, done, infos = ref.advance_n(wp.params, phi, c, mu, s, 8)
    assert rc == 0, err
    data.update(po_params=pvec(wp.params), po_phi0=wp.phi, po_c0=wp.carbon, po_mu0=wp.mu,
                po_s0=svec(pyoracle.scalars_from(wp.scalars)), po_phi=phi, po_c=c, po_mu=mu, po_s=svec(s),
                po_info=ivec(infos))

    # 5. moving window: front high in a 40x48 domain
    ws = workloads.scaled(40, 48, seed=3, front=36.0, jitter=0.1)
    phi, c, mu = ws.phi.copy(), ws.carbon.copy(), ws.mu.copy()
    s = pyoracle.scalars_from(ws.scalars)
    trig, targ = 0.65 * 48 * ws.params["dy"], 0.35 * 48 * ws.params["dy"]
    cg = workloads.FE_C_REFERENCE["gamma_carbon"]
    rc, shifted, err = ref.maybe_shift(ws.params, phi, c, mu, s, trig, targ, cg)
    assert rc == 0 and shifted, err
    data.update(sh_params=pvec(ws.params), sh_phi0=ws.phi, sh_c0=ws.carbon, sh_mu0=ws.mu,
                sh_s0=svec(pyoracle.scalars_from(ws.scalars)), sh_phi=phi, sh_c=c, sh_mu=mu, sh_s=svec(s),
                sh_args=np.array([trig, targ, cg]))

    # 6. capillarity-only smoothing of sharp labels
    sharp = workloads.lamellar_phi(32, 24, [16, 16], [3, 3], np.full(32, 8.0), delta=1e-3)
    sharp = np.round(sharp)
    phi = sharp.copy()
    rc, rep = ref.smooth(w.params, phi, 20, 20, 1e-10, 0.02)
    assert rc == 0
    data.update(sm_phi0=sharp, sm_phi=phi, sm_rep=np.array([rep.steps, rep.converged, rep.energy_initial,
                                                            rep.energy_final, rep.final_relative_energy_change,
                                                            rep.final_max_phase_change]))

    # 7. error text: a rejection with dt_min == dt
    we = workloads.scaled(48, 40, seed=1, front=10.0, jitter=0.1, front_jitter=1, dt=2e-10, dt_min=2e-10)
    phi, c, mu = we.phi.copy(), we.carbon.copy(), we.mu.copy()
    s = pyoracle.scalars_from(we.scalars)
    rc, err, done, infos = ref.advance_n(we.params, phi, c, mu, s, 1)
    assert rc == 1
    data.update(err_params=pvec(we.params))
    meta["cases"]["err"] = {"message": err}

    # 8. phase-diagram law at several undercoolings
    r = workloads.FE_C_REFERENCE
    abcd = []
    for i in range(3):
        abcd += [r["Aeq"][i], r["Beq"][i], r["Ceq"][i], r["D"][i]]
    thermo = []
    for u in (0.0, 10.0, 15.0, 20.0, 37.5):
        rc, out, err = ref.thermo_at_undercooling(1, abcd, list(r["ceq"]) + list(r["slopes"]), u)
        assert rc == 0, err
        thermo.append(np.concatenate([[u], out]))
    data["thermo"] = np.array(thermo)

    np.savez_compressed(OUT, **data)
    META.write_text(json.dumps(meta, indent=1) + "\n")
    print(OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
