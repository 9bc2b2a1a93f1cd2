"""ctypes view of the CPU oracle (TEST INFRASTRUCTURE).

Loads ``oracle/libpearl_oracle.so`` (the C restatement, ``pearl_oracle.c``)
and, when it was built, ``oracle/_ref/libpearl_ref.so`` (the unmodified
reference solver behind ``ref_harness.cpp``).  Both expose the same
operations on the same host layout:

  phi[ny, nx, 3] (alpha, theta, gamma), carbon[ny, nx], mu[ny, nx]

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

D = C.c_double
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


class PoParams(C.Structure):
    _fields_ = [
        ("A", D * 3), ("B", D * 3), ("C", D * 3), ("D", D * 3),
        ("Vm", D), ("epsilon", D), ("sigma", D), ("triple", D),
        ("tau", D * 3),
        ("dx", D), ("dy", D),
        ("dt_max", D), ("dt_min", D), ("max_phase_change", D),
        ("cg_rtol", D), ("cg_atol", D), ("closure_tol", D),
        ("energy_rtol", D), ("energy_atol", D),
        ("cg_max", C.c_int), ("max_retries", C.c_int), ("check_energy", C.c_int), ("phase_only", C.c_int),
        ("mu_reference", D),
    ]


class PoScalars(C.Structure):
    _fields_ = [
        ("time", D), ("dt", D), ("shift_distance", D), ("initial_carbon", D),
        ("carbon_added", D), ("carbon_removed", D),
        ("step", C.c_longlong), ("shifts", C.c_longlong), ("rejected", C.c_longlong),
    ]


class PoStepInfo(C.Structure):
    _fields_ = [
        ("accepted_dt", D), ("max_phase_change", D), ("linear_residual", D), ("closure", D),
        ("energy_change", D), ("cg_iterations", C.c_int), ("retries", C.c_int),
    ]


class PoDiffusionInfo(C.Structure):
    _fields_ = [("ok", C.c_int), ("it", C.c_int), ("residual", D), ("closure", D)]


class PoAdjointReport(C.Structure):
    _fields_ = [("objective", D), ("grad", D * 3), ("steps", C.c_longlong), ("cg_forward", C.c_longlong),
                ("cg_adjoint", C.c_longlong), ("checkpoints", C.c_int)]


class PoDiag(C.Structure):
    _fields_ = [(n, D) for n in ("c_min", "c_max", "mu_min", "mu_max", "phi_sum_error", "mass", "ledger", "energy")]


class PoDeviceOrder(C.Structure):
    _fields_ = [("warps", C.c_int), ("warps_x_log2", C.c_int), ("blocks", C.c_int), ("threads", C.c_int)]


class PoSmoothReport(C.Structure):
    _fields_ = [
        ("steps", C.c_int), ("converged", C.c_int),
        ("energy_initial", D), ("energy_final", D), ("final_relative_energy_change", D),
        ("final_max_phase_change", D), ("phase_fraction_before", D * 3), ("phase_fraction_after", D * 3),
    ]


WHY = {0: "", 1: "phase increment", 2: "linear/closure", 3: "composition/phase bounds",
       4: "mass conservation", 5: "free-energy increase"}


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(DP)


def _params(params) -> PoParams:
    """Accept a PoParams, or any ctypes struct / dict with the same fields."""
    if isinstance(params, PoParams):
        return params
    out = PoParams()
    src = params if isinstance(params, dict) else {n: getattr(params, n) for n, _ in PoParams._fields_}
    for name, typ in PoParams._fields_:
        v = src[name]
        if isinstance(getattr(out, name), C.Array):
            arr = getattr(out, name)
            for i in range(3):
                arr[i] = float(v[i])
        else:
            setattr(out, name, v)
    return out


def scalars_from(obj) -> PoScalars:
    s = PoScalars()
    src = obj if isinstance(obj, dict) else {n: getattr(obj, n) for n, _ in PoScalars._fields_}
    for name, _ in PoScalars._fields_:
        setattr(s, name, src[name])
    return s


class _Lib:
    def __init__(self, path: Path):
        self.path = path
        self.lib = C.CDLL(str(path))


class Port(_Lib):
    """The C restatement (pearl_oracle.c)."""

    def __init__(self):
        from .build_oracle import build_port  # noqa: WPS433 (local import keeps module import cheap)

        super().__init__(build_port())
        L = self.lib
        L.po_propose_phi.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, D, DP]
        L.po_implicit_diffusion.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, DP, DP, D,
                                            C.POINTER(PoDiffusionInfo)]
        L.po_reduced_energy.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP]
        L.po_total_carbon.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP]
        L.po_total_carbon.restype = D
        L.po_valid_state.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP]
        L.po_advance_n.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, C.POINTER(PoScalars),
                                   C.c_int, DP, D, C.POINTER(PoStepInfo), IP, IP]
        L.po_maybe_shift.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, C.POINTER(PoScalars),
                                     D, D, D, IP]
        L.po_front_position.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP]
        L.po_front_position.restype = D
        L.po_snapshot.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, C.POINTER(PoScalars),
                                  C.POINTER(PoDiag)]
        L.po_smooth_interface_only.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, C.c_int, C.c_int, D, D,
                                               C.POINTER(PoSmoothReport)]
        L.po_interface_energy_only.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP]
        L.po_interface_energy_only.restype = D
        L.po_close_mu.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP]
        L.po_set_device_order.argtypes = [C.POINTER(PoDeviceOrder)]
        L.po_set_device_order.restype = None
        L.po_device_sum.argtypes = [C.c_int, C.c_int, DP, C.c_int]
        L.po_device_sum.restype = D
        L.po_psi.argtypes = [C.POINTER(PoParams), C.c_int, D]
        L.po_psi.restype = D
        L.po_adjoint_gradient.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, C.POINTER(PoScalars),
                                          C.c_int, C.c_int, DP, C.POINTER(PoAdjointReport)]
        L.po_adjoint_objective.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP,
                                           C.POINTER(PoScalars), C.c_int, DP, DP]

    def set_device_order(self, warps: int | None, blocks: int = 1, warps_x_log2: int = 0,
                         threads: int | None = None) -> None:
        """Sum in libpearl_gpu's tree order for a grid of `blocks` blocks of
        `warps` warps (see pearl_oracle.h); warps=None restores the reference's
        sequential order."""
        if warps is None:
            self.lib.po_set_device_order(None)
            return
        import os

        o = PoDeviceOrder(warps, warps_x_log2, blocks, threads if threads else (os.cpu_count() or 1))
        self.lib.po_set_device_order(C.byref(o))

    def device_order(self, warps: int, blocks: int, warps_x_log2: int = 0, threads: int | None = None):
        """Context manager: the device's summation order inside, the reference's after."""
        import contextlib

        @contextlib.contextmanager
        def _cm():
            self.set_device_order(warps, blocks, warps_x_log2, threads)
            try:
                yield self
            finally:
                self.set_device_order(None)

        return _cm()

    def device_sum(self, v, reverse: bool = False) -> float:
        """The device's tree sum of v[ny, nx] under the current device order."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        ny, nx = v.shape
        return self.lib.po_device_sum(nx, ny, _p(v), int(reverse))

    def psi(self, params, phase: int, mu: float) -> float:
        return self.lib.po_psi(C.byref(_params(params)), phase, mu)

    def propose_phi(self, params, phi, mu, dt):
        ny, nx = mu.shape
        trial = np.empty_like(phi)
        ch = D()
        rc = self.lib.po_propose_phi(C.byref(_params(params)), nx, ny, _p(phi), _p(mu), _p(trial), dt, C.byref(ch))
        return rc, trial, ch.value

    def implicit_diffusion(self, params, carbon, mu, trial_phi, dt):
        ny, nx = mu.shape
        tc, tmu = carbon.copy(), mu.copy()
        info = PoDiffusionInfo()
        rc = self.lib.po_implicit_diffusion(C.byref(_params(params)), nx, ny, _p(carbon), _p(mu), _p(trial_phi),
                                            _p(tc), _p(tmu), dt, C.byref(info))
        return rc, tc, tmu, info

    def energy_and_mass(self, params, phi, carbon):
        ny, nx = carbon.shape
        e = D()
        pp = _params(params)
        rc = self.lib.po_reduced_energy(C.byref(pp), nx, ny, _p(phi), _p(carbon), C.byref(e))
        m = self.lib.po_total_carbon(C.byref(pp), nx, ny, _p(carbon))
        return rc, e.value, m

    def valid_state(self, params, phi, carbon, mu):
        ny, nx = mu.shape
        return self.lib.po_valid_state(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu))

    def advance_n(self, params, phi, carbon, mu, scalars, nsteps, forced_dt=None, stop_time=1e300):
        """Advance in place.  Returns (rc, why, steps_done, infos)."""
        ny, nx = mu.shape
        infos = (PoStepInfo * max(nsteps, 1))()
        why, done = C.c_int(0), C.c_int(0)
        fd = None
        if forced_dt is not None:
            fd = np.ascontiguousarray(forced_dt, dtype=np.float64)
        rc = self.lib.po_advance_n(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu),
                                   C.byref(scalars), nsteps, _p(fd) if fd is not None else None, stop_time,
                                   infos, C.byref(why), C.byref(done))
        return rc, WHY.get(why.value, "?"), done.value, list(infos)[: done.value]

    def maybe_shift(self, params, phi, carbon, mu, scalars, trigger, target, c_gamma):
        ny, nx = mu.shape
        shifted = C.c_int(0)
        rc = self.lib.po_maybe_shift(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu),
                                     C.byref(scalars), trigger, target, c_gamma, C.byref(shifted))
        return rc, shifted.value

    def front_position(self, params, phi):
        ny, nx = phi.shape[:2]
        return self.lib.po_front_position(C.byref(_params(params)), nx, ny, _p(phi))

    def snapshot(self, params, phi, carbon, mu, scalars):
        ny, nx = mu.shape
        d = PoDiag()
        rc = self.lib.po_snapshot(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu),
                                  C.byref(scalars), C.byref(d))
        return rc, d

    def smooth(self, params, phi, max_steps, min_steps, energy_rtol, max_phase_change):
        ny, nx = phi.shape[:2]
        rep = PoSmoothReport()
        rc = self.lib.po_smooth_interface_only(C.byref(_params(params)), nx, ny, _p(phi), max_steps, min_steps,
                                               energy_rtol, max_phase_change, C.byref(rep))
        return rc, rep

    def close_mu(self, params, phi, carbon):
        ny, nx = carbon.shape
        mu = np.empty_like(carbon)
        rc = self.lib.po_close_mu(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu))
        return rc, mu


    def adjoint_gradient(self, params, phi, carbon, mu, scalars, nsteps, checkpoint_every, target_alpha):
        """Reverse-mode gradient of sum((phi_alpha - target)^2) after nsteps, w.r.t.
        (mobility scale, sigma, D_gamma).  Fields advance in place.  Returns (rc, report)."""
        ny, nx = mu.shape
        rep = PoAdjointReport()
        t = np.ascontiguousarray(target_alpha, dtype=np.float64)
        rc = self.lib.po_adjoint_gradient(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu),
                                          C.byref(scalars), nsteps, checkpoint_every, _p(t), C.byref(rep))
        return rc, rep

    def adjoint_objective(self, params, phi, carbon, mu, scalars, nsteps, target_alpha):
        ny, nx = mu.shape
        J = D()
        t = np.ascontiguousarray(target_alpha, dtype=np.float64)
        rc = self.lib.po_adjoint_objective(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu),
                                           C.byref(scalars), nsteps, _p(t), C.byref(J))
        return rc, J.value


class Reference(_Lib):
    """The unmodified reference solver through ref_harness.cpp (None when not built)."""

    ERRLEN = 512

    def __init__(self, path: Path):
        super().__init__(path)
        L = self.lib
        CP = C.c_char_p
        L.ref_advance_n.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, C.POINTER(PoScalars),
                                    C.c_int, DP, D, C.POINTER(PoStepInfo), IP, CP, C.c_int]
        L.ref_propose_phi.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, D, DP, CP, C.c_int]
        L.ref_implicit_diffusion.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, DP, DP, D,
                                             C.POINTER(PoDiffusionInfo), CP, C.c_int]
        L.ref_energy_and_mass.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, DP, CP, C.c_int]
        L.ref_valid_state.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP]
        L.ref_maybe_shift.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, DP, DP, C.POINTER(PoScalars),
                                      D, D, D, IP, CP, C.c_int]
        L.ref_smooth.argtypes = [C.POINTER(PoParams), C.c_int, C.c_int, DP, C.c_int, C.c_int, D, D,
                                 C.POINTER(PoSmoothReport), CP, C.c_int]
        L.ref_thermo_at_undercooling.argtypes = [C.c_int, DP, DP, D, DP, CP, C.c_int]

    def _err(self):
        return C.create_string_buffer(self.ERRLEN)

    def advance_n(self, params, phi, carbon, mu, scalars, nsteps, forced_dt=None, stop_time=1e300):
        ny, nx = mu.shape
        infos = (PoStepInfo * max(nsteps, 1))()
        done = C.c_int(0)
        err = self._err()
        fd = None
        if forced_dt is not None:
            fd = np.ascontiguousarray(forced_dt, dtype=np.float64)
        rc = self.lib.ref_advance_n(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu),
                                    C.byref(scalars), nsteps, _p(fd) if fd is not None else None, stop_time,
                                    infos, C.byref(done), err, self.ERRLEN)
        return rc, err.value.decode(), done.value, list(infos)[: done.value]

    def propose_phi(self, params, phi, mu, dt):
        ny, nx = mu.shape
        trial = np.empty_like(phi)
        ch = D()
        err = self._err()
        rc = self.lib.ref_propose_phi(C.byref(_params(params)), nx, ny, _p(phi), _p(mu), _p(trial), dt,
                                      C.byref(ch), err, self.ERRLEN)
        return rc, trial, ch.value

    def implicit_diffusion(self, params, carbon, mu, trial_phi, dt):
        ny, nx = mu.shape
        tc, tmu = carbon.copy(), mu.copy()
        info = PoDiffusionInfo()
        err = self._err()
        rc = self.lib.ref_implicit_diffusion(C.byref(_params(params)), nx, ny, _p(carbon), _p(mu), _p(trial_phi),
                                             _p(tc), _p(tmu), dt, C.byref(info), err, self.ERRLEN)
        return rc, tc, tmu, info

    def energy_and_mass(self, params, phi, carbon):
        ny, nx = carbon.shape
        e, m = D(), D()
        err = self._err()
        rc = self.lib.ref_energy_and_mass(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), C.byref(e),
                                          C.byref(m), err, self.ERRLEN)
        return rc, e.value, m.value

    def valid_state(self, params, phi, carbon, mu):
        ny, nx = mu.shape
        return self.lib.ref_valid_state(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu))

    def maybe_shift(self, params, phi, carbon, mu, scalars, trigger, target, c_gamma):
        ny, nx = mu.shape
        shifted = C.c_int(0)
        err = self._err()
        rc = self.lib.ref_maybe_shift(C.byref(_params(params)), nx, ny, _p(phi), _p(carbon), _p(mu),
                                      C.byref(scalars), trigger, target, c_gamma, C.byref(shifted), err,
                                      self.ERRLEN)
        return rc, shifted.value, err.value.decode()

    def smooth(self, params, phi, max_steps, min_steps, energy_rtol, max_phase_change):
        ny, nx = phi.shape[:2]
        rep = PoSmoothReport()
        err = self._err()
        rc = self.lib.ref_smooth(C.byref(_params(params)), nx, ny, _p(phi), max_steps, min_steps, energy_rtol,
                                 max_phase_change, C.byref(rep), err, self.ERRLEN)
        return rc, rep

    def thermo_at_undercooling(self, law: int, ref_abcd, slopes, undercooling):
        a = np.ascontiguousarray(ref_abcd, dtype=np.float64)
        s = np.ascontiguousarray(slopes, dtype=np.float64)
        out = np.zeros(12)
        err = self._err()
        rc = self.lib.ref_thermo_at_undercooling(law, _p(a), _p(s), undercooling, _p(out), err, self.ERRLEN)
        return rc, out, err.value.decode()


_port = None


def port() -> Port:
    global _port
    if _port is None:
        _port = Port()
    return _port


def reference() -> Reference | None:
    from .build_oracle import REF_SO, build_reference

    try:
        build_reference()
    except Exception:  # noqa: BLE001 — a failed compile leaves the reference unavailable
        pass
    return Reference(REF_SO) if REF_SO.exists() else None
