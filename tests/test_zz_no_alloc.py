"""pearl_gpu_advance_noalloc: one accepted step for callers that cannot allocate
device memory (their GPU memory belongs to another allocator, or they run
loops that must not pay for cudaMalloc/cudaFree).  The caller hands in device
planes; the library's scratch is a fixed array compiled into it.

Checked here through the C ABI against the context-based entry point
(pearl_gpu_advance) on the same input, for two calls in a row, with the
tolerances of the other parity tests.  The context pads every row to a
multiple of 32 doubles; this entry point runs on the caller's dense rows
(pitch = nx), so widths that are not multiples of 32 (37, 100, 513) exercise
its own row layout and periodic x wrap.  A phase-only case covers the trial
carbon and mu that the proposal itself writes into the scratch.  After the
first call, a second call must leave the device's free memory unchanged.
This file is collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PHI_TOL = 1e-10
MU_TOL = 1e-5
MASS_RTOL = 1e-12


def _planes(w):
    import torch

    phi = torch.from_numpy(np.ascontiguousarray(np.moveaxis(w.phi, -1, 0))).cuda()  # [3, ny, nx]
    c = torch.from_numpy(w.carbon.copy()).cuda()
    mu = torch.from_numpy(w.mu.copy()).cuda()
    return phi, c, mu


def _noalloc_step(lib, params, w, phi, c, mu, scalars):
    import torch

    import pearl_gpu

    info = pearl_gpu.PearlStepInfo()
    stream = torch.cuda.current_stream()
    rc = lib.pearl_gpu_advance_noalloc(C.byref(params), w.nx, w.ny, C.c_void_p(phi.data_ptr()),
                                       C.c_void_p(c.data_ptr()), C.c_void_p(mu.data_ptr()), C.byref(scalars),
                                       1e300, C.byref(info), C.c_void_p(stream.cuda_stream))
    return rc, info


CASES = [
    # (nx, ny, front, extra controls)
    (96, 72, 20.0, {}),
    (100, 72, 20.0, {}),         # row length not a multiple of 32
    (37, 19, 6.0, {}),           # ragged in both directions, smaller than one tile
    (513, 511, 40.0, {}),        # 262143 cells: just under the scratch limit
    (100, 72, 20.0, {"phase_only": 1}),
]


@pytest.mark.parametrize("nx,ny,front,controls", CASES,
                         ids=["96x72", "100x72", "37x19", "513x511", "100x72-phase-only"])
def test_noalloc_matches_context_entry_point(gpu_lib, nx, ny, front, controls):
    import torch

    import pearl_gpu
    from pearl_gpu import workloads

    torch.cuda.set_device(0)
    w = workloads.scaled(nx, ny, seed=4, front=front, jitter=0.1, front_jitter=1, **controls)
    params = pearl_gpu.PearlParams.from_dict(w.params)
    phi, c, mu = _planes(w)
    scalars = pearl_gpu.PearlScalars.from_dict(w.scalars)
    with pearl_gpu.Context(w.params, w.nx, w.ny, device=0) as ctx:
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        for call in range(2):
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            rc, info = _noalloc_step(gpu_lib, params, w, phi, c, mu, scalars)
            assert rc == 0, pearl_gpu.STATUS.get(rc, rc)
            free_after = torch.cuda.mem_get_info()[0]
            if call == 1:
                # the first call may load the library's module (and its static
                # scratch) onto the device; later calls allocate nothing
                assert free_after == free_before
            ref = ctx.advance()
            assert info.retries == ref.retries
            assert info.cg_iterations == ref.cg_iterations
            assert info.accepted_dt == ref.accepted_dt
            phi_r, c_r, mu_r, s_r = ctx.download()
            torch.cuda.synchronize()
            phi_n = np.moveaxis(phi.cpu().numpy(), 0, -1)
            assert np.abs(phi_n - phi_r).max() <= PHI_TOL
            assert np.abs(mu.cpu().numpy() - mu_r).max() <= MU_TOL
            c_n = c.cpu().numpy()
            assert abs(c_n.sum() - c_r.sum()) <= MASS_RTOL * abs(c_r.sum())
            assert scalars.step == s_r.step and scalars.time == s_r.time and scalars.dt == s_r.dt


def test_noalloc_rejects_oversized_domain(gpu_lib):
    import torch

    import pearl_gpu
    from pearl_gpu import workloads

    torch.cuda.set_device(0)
    params = pearl_gpu.PearlParams.from_dict(workloads.make_params(1024, 512, 2e-9, 10.0, 4e-12))
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    scalars = pearl_gpu.PearlScalars()
    ptr = C.c_void_p(dummy.data_ptr())
    rc = gpu_lib.pearl_gpu_advance_noalloc(C.byref(params), 1024, 512, ptr, ptr, ptr, C.byref(scalars), 1e300,
                                           None, None)
    assert rc == 13  # PEARL_ERR_TOO_LARGE, before any device work
