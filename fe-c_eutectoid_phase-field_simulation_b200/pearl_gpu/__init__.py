"""Python view of libpearl_gpu.so, the B200 hot path of the Pearl pearlite solver.

This module only binds the C ABI declared in ``include/pearl_gpu.h`` with
ctypes; all arithmetic runs in the CUDA library.  There is no CPU fallback:
importing the binding fails loudly when the library has not been built, and
creating a context fails when no CUDA device is present.

Host arrays use the reference's gathered layout: ``phi[ny, nx, 3]`` (alpha,
theta, gamma), ``carbon[ny, nx]``, ``mu[ny, nx]``, float64, C-contiguous.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .build import LIB

D = C.c_double
DP = C.POINTER(C.c_double)

STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "invalid advance time",
    4: "step rejected below dt_min", 5: "step retry limit", 6: "Invalid mixture coefficients",
    7: "Simplex projection failed", 8: "configured max_steps reached before end_time",
    9: "device wait limit exceeded", 10: "unsafe shift: removed strip contains gamma",
    11: "Nonfinite total carbon", 12: "no CUDA device",
    13: "domain exceeds the no-allocation scratch limit of 262144 cells", 14: "sharp smoothing failed",
}


class PearlParams(C.Structure):
    """pearl_params (include/pearl_gpu.h)."""

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

    @classmethod
    def from_dict(cls, d: dict) -> "PearlParams":
        p = cls()
        for name, _ in cls._fields_:
            v = d[name]
            if isinstance(getattr(p, name), C.Array):
                arr = getattr(p, name)
                for i in range(3):
                    arr[i] = float(v[i])
            else:
                setattr(p, name, v)
        return p


class PearlScalars(C.Structure):
    """pearl_scalars: the scalar members of pearl::State."""

    _fields_ = [
        ("time", D), ("dt", D), ("shift_distance", D), ("initial_carbon", D),
        ("carbon_added", D), ("carbon_removed", D),
        ("step", C.c_longlong), ("shifts", C.c_longlong), ("rejected", C.c_longlong),
    ]

    @classmethod
    def from_dict(cls, d: dict) -> "PearlScalars":
        s = cls()
        for name, _ in cls._fields_:
            setattr(s, name, d[name])
        return s

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class PearlStepInfo(C.Structure):
    """pearl_step_info: pearl::StepInfo."""

    _fields_ = [
        ("accepted_dt", D), ("max_phase_change", D), ("linear_residual", D), ("closure", D),
        ("energy_change", D), ("cg_iterations", C.c_int), ("retries", C.c_int),
    ]


class PearlSmoothReport(C.Structure):
    _fields_ = [("steps", C.c_int), ("converged", C.c_int), ("energy_initial", D), ("energy_final", D),
                ("final_relative_energy_change", D), ("final_max_phase_change", D),
                ("phase_fraction_before", D * 3), ("phase_fraction_after", D * 3)]


class PearlRunLimits(C.Structure):
    _fields_ = [("max_steps", C.c_longlong), ("config_max_steps", C.c_longlong), ("stop_time", D),
                ("end_time", D), ("output_eps", D)]


class PearlRunReport(C.Structure):
    _fields_ = [("steps", C.c_longlong), ("cg_total", C.c_longlong), ("cg_peak", C.c_int),
                ("reached_stop", C.c_int), ("last", PearlStepInfo)]


class PearlDiag(C.Structure):
    _fields_ = [(n, D) for n in ("c_min", "c_max", "mu_min", "mu_max", "phi_sum_error", "mass", "ledger", "energy")]


EXPORTS = [
    "pearl_gpu_create", "pearl_gpu_destroy", "pearl_gpu_set_stream", "pearl_gpu_set_params", "pearl_gpu_upload",
    "pearl_gpu_download", "pearl_gpu_get_scalars", "pearl_gpu_set_scalars", "pearl_gpu_advance", "pearl_gpu_run",
    "pearl_gpu_maybe_shift", "pearl_gpu_snapshot", "pearl_gpu_propose_phi", "pearl_gpu_upload_trial_phi",
    "pearl_gpu_implicit_diffusion", "pearl_gpu_download_trial", "pearl_gpu_energy_mass", "pearl_gpu_valid_state",
    "pearl_gpu_status_string", "pearl_gpu_last_error", "pearl_gpu_stats", "pearl_gpu_phase_times",
    "pearl_gpu_selftest_division", "pearl_gpu_advance_noalloc", "pearl_gpu_smooth_interface",
    "pearl_gpu_mixture_sums", "pearl_gpu_init_composition", "pearl_gpu_batch_create", "pearl_gpu_batch_destroy",
    "pearl_gpu_batch_upload", "pearl_gpu_batch_download", "pearl_gpu_batch_run", "pearl_gpu_batch_autotune",
    "pearl_gpu_batch_stats", "pearl_gpu_batch_last_error", "pearl_gpu_adjoint_gradient", "pearl_gpu_set_precision",
    "pearl_gpu_batch_set_precision", "pearl_gpu_selftest_wait_limit", "pearl_gpu_batch_configure",
    "pearl_gpu_set_history", "pearl_gpu_get_history", "pearl_gpu_run_replay", "pearl_gpu_batch_plan",
    "pearl_gpu_selftest_fp64_peak", "pearl_gpu_geometry", "pearl_gpu_fill",
]

# Filling commands (PEARL_FILL_*): method name -> code
FILL_METHODS = {"FILLCUBE": 1, "FILLCYLINDER": 2, "FILLCENTERBOX2D": 3, "FILLYJUNCTION2D": 4,
                "FILLYJUNCTIONLAMELLAE2D": 5, "FILLADHEREDPEARLITEARM2D": 6, "FILLPEARLITEELLIPSE2D": 7}


class PearlFillOp(C.Structure):
    _fields_ = [("method", C.c_int), ("nparams", C.c_int), ("p", D * 16)]

    @classmethod
    def make(cls, method: str, params) -> "PearlFillOp":
        o = cls()
        o.method = FILL_METHODS[method]
        o.nparams = len(params)
        for j, v in enumerate(params):
            o.p[j] = float(v)
        return o

# fp64: the reference's arithmetic; mixed: FP32 proposal + FP32 inner solve;
# mixed_propose / mixed_solve: one of the two
PRECISION = {"fp64": 0, "mixed": 1, "mixed_propose": 2, "mixed_solve": 3}
# Batch group_blocks value for groups sized per instance (PEARL_BATCH_SIZED_GROUPS)
BATCH_SIZED_GROUPS = -1

PHASES = ["propose", "setup", "apply", "update", "true_residual", "reset", "final", "energy", "final_phase_only",
          "mixture", "shift", "snapshot", "smooth", "init", "adjoint", "apply32"]

_lib = None


def library(path: Path | None = None) -> C.CDLL:
    """Load libpearl_gpu.so; raises if it is missing (build with __graft_entry__.build())."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB
    if not p.exists():
        raise ImportError(f"{p} is missing: the CUDA library must be built (python -m pearl_gpu.build)")
    L = C.CDLL(str(p))
    V = C.c_void_p
    L.pearl_gpu_create.argtypes = [C.POINTER(PearlParams), C.c_int, C.c_int, C.c_int, C.POINTER(V)]
    L.pearl_gpu_destroy.argtypes = [V]
    L.pearl_gpu_destroy.restype = None
    L.pearl_gpu_set_stream.argtypes = [V, V]
    L.pearl_gpu_set_params.argtypes = [V, C.POINTER(PearlParams)]
    L.pearl_gpu_upload.argtypes = [V, DP, DP, DP, C.POINTER(PearlScalars)]
    L.pearl_gpu_download.argtypes = [V, DP, DP, DP, C.POINTER(PearlScalars)]
    L.pearl_gpu_get_scalars.argtypes = [V, C.POINTER(PearlScalars)]
    L.pearl_gpu_set_scalars.argtypes = [V, C.POINTER(PearlScalars)]
    L.pearl_gpu_advance.argtypes = [V, D, C.POINTER(PearlStepInfo)]
    L.pearl_gpu_run.argtypes = [V, C.POINTER(PearlRunLimits), C.POINTER(PearlRunReport)]
    L.pearl_gpu_maybe_shift.argtypes = [V, D, D, D, C.POINTER(C.c_int)]
    L.pearl_gpu_snapshot.argtypes = [V, C.POINTER(PearlDiag)]
    L.pearl_gpu_propose_phi.argtypes = [V, D, DP]
    L.pearl_gpu_upload_trial_phi.argtypes = [V, DP]
    L.pearl_gpu_implicit_diffusion.argtypes = [V, D, C.POINTER(C.c_int), C.POINTER(C.c_int), DP, DP]
    L.pearl_gpu_download_trial.argtypes = [V, DP, DP, DP]
    L.pearl_gpu_energy_mass.argtypes = [V, DP, DP]
    L.pearl_gpu_valid_state.argtypes = [V, C.POINTER(C.c_int)]
    L.pearl_gpu_status_string.argtypes = [C.c_int]
    L.pearl_gpu_status_string.restype = C.c_char_p
    L.pearl_gpu_last_error.argtypes = [V]
    L.pearl_gpu_last_error.restype = C.c_char_p
    L.pearl_gpu_stats.argtypes = [V, C.POINTER(C.c_longlong), C.POINTER(C.c_int), DP]
    L.pearl_gpu_geometry.argtypes = [V, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pearl_gpu_fill.argtypes = [V, C.POINTER(PearlFillOp), C.c_int]
    L.pearl_gpu_phase_times.argtypes = [V, DP, C.POINTER(C.c_longlong)]
    L.pearl_gpu_selftest_division.argtypes = [C.c_int, DP, DP, C.c_longlong, C.POINTER(C.c_ulonglong)]
    L.pearl_gpu_selftest_fp64_peak.argtypes = [C.c_int, DP]
    L.pearl_gpu_smooth_interface.argtypes = [V, C.c_int, C.c_int, D, D, C.POINTER(PearlSmoothReport)]
    L.pearl_gpu_mixture_sums.argtypes = [V, DP, DP]
    L.pearl_gpu_init_composition.argtypes = [V, D, DP]
    L.pearl_gpu_advance_noalloc.argtypes = [C.POINTER(PearlParams), C.c_int, C.c_int, V, V, V,
                                            C.POINTER(PearlScalars), D, C.POINTER(PearlStepInfo), V]
    IP = C.POINTER(C.c_int)
    L.pearl_gpu_adjoint_gradient.argtypes = [V, C.c_longlong, C.c_int, DP, C.POINTER(PearlAdjointReport)]
    L.pearl_gpu_set_precision.argtypes = [V, C.c_int]
    L.pearl_gpu_set_history.argtypes = [V, C.c_longlong]
    L.pearl_gpu_run_replay.argtypes = [V, DP, C.c_longlong, C.POINTER(PearlRunReport)]
    LLP = C.POINTER(C.c_longlong)
    L.pearl_gpu_get_history.argtypes = [V, C.POINTER(PearlStepInfo), C.c_longlong, LLP, LLP]
    L.pearl_gpu_selftest_wait_limit.argtypes = [V, C.POINTER(C.c_int), DP]
    L.pearl_gpu_batch_set_precision.argtypes = [V, C.c_int]
    L.pearl_gpu_batch_create.argtypes = [C.c_int, C.POINTER(PearlParams), IP, IP, C.c_int, C.c_int, C.POINTER(V)]
    L.pearl_gpu_batch_destroy.argtypes = [V]
    L.pearl_gpu_batch_destroy.restype = None
    L.pearl_gpu_batch_upload.argtypes = [V, C.c_int, DP, DP, DP, C.POINTER(PearlScalars)]
    L.pearl_gpu_batch_download.argtypes = [V, C.c_int, DP, DP, DP, C.POINTER(PearlScalars)]
    L.pearl_gpu_batch_run.argtypes = [V, C.POINTER(PearlRunLimits), C.POINTER(PearlRunReport), IP]
    L.pearl_gpu_batch_autotune.argtypes = [V, C.c_int, IP, IP, IP]
    L.pearl_gpu_batch_configure.argtypes = [V, C.c_int, C.c_int, C.c_int]
    L.pearl_gpu_batch_plan.argtypes = [C.c_int, LLP, C.c_int, C.c_int, C.c_double, IP, IP, IP, DP]
    L.pearl_gpu_batch_stats.argtypes = [V, C.POINTER(C.c_longlong), IP, IP, DP]
    L.pearl_gpu_batch_last_error.argtypes = [V]
    L.pearl_gpu_batch_last_error.restype = C.c_char_p
    if path is None:
        _lib = L
    return L


def batch_plan(tiles, grid_blocks: int, group_blocks: int = BATCH_SIZED_GROUPS, pass_overhead_tiles: float = 4.0):
    """The groups a batch launch would use (pearl_gpu_batch_plan; host only):
    (group of each instance, size of each group, modelled longest group time)."""
    L = library()
    t = np.ascontiguousarray(tiles, dtype=np.int64)
    goi = np.zeros(len(t), dtype=np.int32)
    gsz = np.zeros(max(grid_blocks, 1), dtype=np.int32)
    ng, longest = C.c_int(), C.c_double()
    rc = L.pearl_gpu_batch_plan(len(t), t.ctypes.data_as(C.POINTER(C.c_longlong)), grid_blocks, group_blocks,
                                pass_overhead_tiles, goi.ctypes.data_as(C.POINTER(C.c_int)),
                                gsz.ctypes.data_as(C.POINTER(C.c_int)), C.byref(ng), C.byref(longest))
    if rc:
        raise PearlError(rc, f"pearl_gpu_batch_plan failed: {STATUS.get(rc, rc)}")
    return goi, gsz[: ng.value].copy(), longest.value


def selftest_division(a: np.ndarray, b: np.ndarray, device: int = 0) -> int:
    """Number of elements where the device's exact constant-divisor division differs from a/b."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = C.c_ulonglong(0)
    rc = library().pearl_gpu_selftest_division(device, _p(a), _p(b), a.size, C.byref(n))
    if rc:
        raise PearlError(rc, STATUS.get(rc, str(rc)))
    return int(n.value)


def fp64_peak_tflops(device: int = 0) -> float:
    """Measured FP64 throughput of the device (independent FMA chains, full grid)."""
    t = C.c_double(0)
    rc = library().pearl_gpu_selftest_fp64_peak(device, C.byref(t))
    if rc:
        raise PearlError(rc, STATUS.get(rc, str(rc)))
    return t.value


class PearlAdjointReport(C.Structure):
    """pearl_adjoint_report: objective, gradient (mobility scale, sigma, D_gamma), counters, timings."""

    _fields_ = [("objective", D), ("grad", D * 3), ("steps", C.c_longlong), ("cg_forward", C.c_longlong),
                ("cg_adjoint", C.c_longlong), ("checkpoints", C.c_int), ("forward_ms", D), ("recompute_ms", D),
                ("adjoint_ms", D)]


class PearlError(RuntimeError):
    """A non-zero pearl_status; ``str()`` is the reference-style message."""

    def __init__(self, status: int, message: str):
        super().__init__(message or STATUS.get(status, f"status {status}"))
        self.status = status


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(DP)


class Context:
    """One device-resident domain (pearl_gpu_ctx)."""

    def __init__(self, params: dict | PearlParams, nx: int, ny: int, device: int = 0, stream: int | None = None):
        self.lib = library()
        self.nx, self.ny = nx, ny
        self.params = params if isinstance(params, PearlParams) else PearlParams.from_dict(params)
        h = C.c_void_p()
        rc = self.lib.pearl_gpu_create(C.byref(self.params), nx, ny, device, C.byref(h))
        if rc:
            raise PearlError(rc, f"pearl_gpu_create failed: {STATUS.get(rc, rc)}")
        self.h = h
        if stream is not None:
            self._check(self.lib.pearl_gpu_set_stream(self.h, C.c_void_p(stream)))

    def _check(self, rc: int) -> None:
        if rc:
            raise PearlError(rc, self.lib.pearl_gpu_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.pearl_gpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    # ---- state transfer (Domain::load_global / gather)
    def upload(self, phi, carbon, mu, scalars: dict | PearlScalars | None = None) -> None:
        s = None
        if scalars is not None:
            s = scalars if isinstance(scalars, PearlScalars) else PearlScalars.from_dict(scalars)
        self._check(self.lib.pearl_gpu_upload(self.h, _p(phi), _p(carbon), _p(mu), C.byref(s) if s else None))

    def download(self, out=None):
        """(phi, carbon, mu, scalars); `out` = (phi, carbon, mu) arrays to write into
        (e.g. pinned host buffers), else new arrays."""
        if out is None:
            phi = np.empty((self.ny, self.nx, 3))
            carbon = np.empty((self.ny, self.nx))
            mu = np.empty((self.ny, self.nx))
        else:
            phi, carbon, mu = out
        s = PearlScalars()
        self._check(self.lib.pearl_gpu_download(self.h, _p(phi), _p(carbon), _p(mu), C.byref(s)))
        return phi, carbon, mu, s

    def scalars(self) -> PearlScalars:
        s = PearlScalars()
        self._check(self.lib.pearl_gpu_get_scalars(self.h, C.byref(s)))
        return s

    def set_scalars(self, s: dict | PearlScalars) -> None:
        s = s if isinstance(s, PearlScalars) else PearlScalars.from_dict(s)
        self._check(self.lib.pearl_gpu_set_scalars(self.h, C.byref(s)))

    # ---- hot path
    def advance(self, stop_time: float = 1e300) -> PearlStepInfo:
        info = PearlStepInfo()
        self._check(self.lib.pearl_gpu_advance(self.h, stop_time, C.byref(info)))
        return info

    def run(self, max_steps: int, stop_time: float = 1e300, end_time: float = 1e300, output_eps: float = 0.0,
            config_max_steps: int = 2**62) -> PearlRunReport:
        lim = PearlRunLimits(max_steps, config_max_steps, stop_time, end_time, output_eps)
        rep = PearlRunReport()
        self._check(self.lib.pearl_gpu_run(self.h, C.byref(lim), C.byref(rep)))
        return rep

    def maybe_shift(self, trigger: float, target: float, c_gamma: float) -> int:
        rows = C.c_int(0)
        self._check(self.lib.pearl_gpu_maybe_shift(self.h, trigger, target, c_gamma, C.byref(rows)))
        return rows.value

    def snapshot(self) -> PearlDiag:
        d = PearlDiag()
        self._check(self.lib.pearl_gpu_snapshot(self.h, C.byref(d)))
        return d

    # ---- initialisation (pearl::initialize)
    def smooth_interface(self, max_steps: int = 100, min_steps: int = 100, energy_rtol: float = 1e-10,
                         max_phase_change: float = 0.02) -> PearlSmoothReport:
        rep = PearlSmoothReport()
        self._check(self.lib.pearl_gpu_smooth_interface(self.h, max_steps, min_steps, energy_rtol, max_phase_change,
                                                        C.byref(rep)))
        return rep

    def fill(self, commands) -> None:
        """Paint the current phase fields with filling commands [(method, params), ...]
        (pearl_gpu_fill: filling_phase_at of every cell, on the device)."""
        ops = (PearlFillOp * max(len(commands), 1))(*[PearlFillOp.make(m, p) for m, p in commands])
        self._check(self.lib.pearl_gpu_fill(self.h, ops, len(commands)))

    def mixture_sums(self):
        a, b = D(), D()
        self._check(self.lib.pearl_gpu_mixture_sums(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def init_composition(self, mu: float) -> float:
        m = D()
        self._check(self.lib.pearl_gpu_init_composition(self.h, mu, C.byref(m)))
        return m.value

    # ---- single functions of the hot path
    def propose_phi(self, dt: float) -> float:
        ch = D()
        self._check(self.lib.pearl_gpu_propose_phi(self.h, dt, C.byref(ch)))
        return ch.value

    def upload_trial_phi(self, phi) -> None:
        self._check(self.lib.pearl_gpu_upload_trial_phi(self.h, _p(phi)))

    def implicit_diffusion(self, dt: float):
        ok, it = C.c_int(), C.c_int()
        res, clo = D(), D()
        self._check(self.lib.pearl_gpu_implicit_diffusion(self.h, dt, C.byref(ok), C.byref(it), C.byref(res),
                                                          C.byref(clo)))
        return dict(ok=ok.value, it=it.value, residual=res.value, closure=clo.value)

    def download_trial(self):
        phi = np.empty((self.ny, self.nx, 3))
        carbon = np.empty((self.ny, self.nx))
        mu = np.empty((self.ny, self.nx))
        self._check(self.lib.pearl_gpu_download_trial(self.h, _p(phi), _p(carbon), _p(mu)))
        return phi, carbon, mu

    def energy_mass(self):
        e, m = D(), D()
        self._check(self.lib.pearl_gpu_energy_mass(self.h, C.byref(e), C.byref(m)))
        return e.value, m.value

    def valid_state(self) -> bool:
        v = C.c_int()
        self._check(self.lib.pearl_gpu_valid_state(self.h, C.byref(v)))
        return bool(v.value)

    def run_replay(self, accepted_dt) -> PearlRunReport:
        """Steps whose first attempt uses accepted_dt[k] (an oracle-style replay)."""
        dts = np.ascontiguousarray(accepted_dt, dtype=np.float64)
        rep = PearlRunReport()
        self._check(self.lib.pearl_gpu_run_replay(self.h, _p(dts), dts.size, C.byref(rep)))
        return rep

    def set_history(self, capacity: int) -> None:
        """Record every accepted step's PearlStepInfo in a device ring of `capacity` entries."""
        self._check(self.lib.pearl_gpu_set_history(self.h, capacity))

    def history(self, max_entries: int | None = None):
        """(entries oldest first, steps recorded since set_history)."""
        n = max_entries if max_entries is not None else 1 << 20
        buf = (PearlStepInfo * max(n, 1))()
        got, rec = C.c_longlong(), C.c_longlong()
        self._check(self.lib.pearl_gpu_get_history(self.h, buf, n, C.byref(got), C.byref(rec)))
        return list(buf)[: got.value], rec.value

    def selftest_wait_limit(self):
        """(status, device ms) of a grid barrier that cannot complete (see pearl_gpu.h)."""
        st, ms = C.c_int(), D()
        self._check(self.lib.pearl_gpu_selftest_wait_limit(self.h, C.byref(st), C.byref(ms)))
        return st.value, ms.value

    def set_precision(self, precision: str) -> None:
        """'fp64' (default, the reference's arithmetic), 'mixed' (FP32 proposal forces and FP32
        inner solve rounds), 'mixed_propose' or 'mixed_solve' (one of the two)."""
        self._check(self.lib.pearl_gpu_set_precision(self.h, PRECISION[precision]))

    def adjoint_gradient(self, nsteps: int, checkpoint_every: int, target_alpha) -> PearlAdjointReport:
        """Gradient of sum((phi_alpha - target)^2) after nsteps w.r.t. (mobility scale, sigma,
        D_gamma); the context ends in the forward's final state."""
        t = np.ascontiguousarray(target_alpha, dtype=np.float64)
        assert t.shape == (self.ny, self.nx)
        rep = PearlAdjointReport()
        self._check(self.lib.pearl_gpu_adjoint_gradient(self.h, nsteps, checkpoint_every, _p(t), C.byref(rep)))
        return rep

    def phase_times(self) -> dict:
        """{phase: (ms, count)} of the last launch."""
        ms = (D * 16)()
        cnt = (C.c_longlong * 16)()
        self._check(self.lib.pearl_gpu_phase_times(self.h, ms, cnt))
        return {name: (ms[k], cnt[k]) for k, name in enumerate(PHASES) if cnt[k]}

    def geometry(self) -> dict:
        """warps per block, warps side by side in x (log2) and grid blocks: the
        tree every global sum follows (oracle: set_device_order)."""
        w, wx, g = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.pearl_gpu_geometry(self.h, C.byref(w), C.byref(wx), C.byref(g)))
        return dict(warps=w.value, warps_x_log2=wx.value, blocks=g.value)

    def stats(self):
        n, g, ms = C.c_longlong(), C.c_int(), D()
        self._check(self.lib.pearl_gpu_stats(self.h, C.byref(n), C.byref(g), C.byref(ms)))
        return dict(launches=n.value, grid=g.value, last_ms=ms.value)


class Batch:
    """Many independent domains advanced in one persistent launch (pearl_gpu_batch).

    ``cases`` is a sequence of (params, nx, ny).  Each instance follows the
    same step path as a :class:`Context` of its own.
    """

    def __init__(self, cases, device: int = 0, group_blocks: int = 0):
        self.lib = library()
        self.n = len(cases)
        self.shapes = [(int(nx), int(ny)) for _, nx, ny in cases]
        prm = (PearlParams * self.n)()
        for i, (p, _, _) in enumerate(cases):
            prm[i] = p if isinstance(p, PearlParams) else PearlParams.from_dict(p)
        nx = (C.c_int * self.n)(*[s[0] for s in self.shapes])
        ny = (C.c_int * self.n)(*[s[1] for s in self.shapes])
        h = C.c_void_p()
        rc = self.lib.pearl_gpu_batch_create(self.n, prm, nx, ny, device, group_blocks, C.byref(h))
        if rc:
            raise PearlError(rc, f"pearl_gpu_batch_create failed: {STATUS.get(rc, rc)}")
        self.h = h

    def _check(self, rc: int) -> None:
        if rc:
            raise PearlError(rc, self.lib.pearl_gpu_batch_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.pearl_gpu_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def upload(self, i: int, phi, carbon, mu, scalars: dict | PearlScalars | None = None) -> None:
        s = None
        if scalars is not None:
            s = scalars if isinstance(scalars, PearlScalars) else PearlScalars.from_dict(scalars)
        self._check(self.lib.pearl_gpu_batch_upload(self.h, i, _p(phi), _p(carbon), _p(mu),
                                                    C.byref(s) if s else None))

    def download(self, i: int, out=None):
        nx, ny = self.shapes[i]
        if out is None:
            phi = np.empty((ny, nx, 3))
            carbon = np.empty((ny, nx))
            mu = np.empty((ny, nx))
        else:
            phi, carbon, mu = out
        s = PearlScalars()
        self._check(self.lib.pearl_gpu_batch_download(self.h, i, _p(phi), _p(carbon), _p(mu), C.byref(s)))
        return phi, carbon, mu, s

    def run(self, max_steps: int, stop_time: float = 1e300, end_time: float = 1e300, output_eps: float = 0.0,
            config_max_steps: int = 2**62):
        """Returns (reports, statuses), one entry per instance."""
        lim = PearlRunLimits(max_steps, config_max_steps, stop_time, end_time, output_eps)
        reps = (PearlRunReport * self.n)()
        st = (C.c_int * self.n)()
        self._check(self.lib.pearl_gpu_batch_run(self.h, C.byref(lim), reps, st))
        return list(reps), list(st)

    def set_precision(self, precision: str) -> None:
        self._check(self.lib.pearl_gpu_batch_set_precision(self.h, PRECISION[precision]))

    def configure(self, group_blocks: int, use_tma: bool = True, tile_warps_x: int = 1) -> None:
        self._check(self.lib.pearl_gpu_batch_configure(self.h, group_blocks, int(use_tma), tile_warps_x))

    def autotune(self, steps: int = 2):
        """Chooses (group blocks, TMA staging, warps side by side in x of the tile)."""
        g, t, w = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.pearl_gpu_batch_autotune(self.h, steps, C.byref(g), C.byref(t), C.byref(w)))
        return g.value, bool(t.value), w.value

    def stats(self):
        n, grid, gb, ms = C.c_longlong(), C.c_int(), C.c_int(), D()
        self._check(self.lib.pearl_gpu_batch_stats(self.h, C.byref(n), C.byref(grid), C.byref(gb), C.byref(ms)))
        return dict(launches=n.value, grid=grid.value, group_blocks=gb.value, last_ms=ms.value)
