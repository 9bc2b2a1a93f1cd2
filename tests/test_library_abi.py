"""The C ABI library loads without a GPU and exports every entry point that
include/pearl_gpu.h declares (no compute calls here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "pearl_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pearl_gpu_\w+)\s*\(", text)))


def test_header_declares_the_hot_path():
    names = declared_functions()
    for must in ("pearl_gpu_create", "pearl_gpu_upload", "pearl_gpu_advance", "pearl_gpu_run",
                 "pearl_gpu_download", "pearl_gpu_maybe_shift", "pearl_gpu_snapshot", "pearl_gpu_destroy",
                 "pearl_gpu_propose_phi", "pearl_gpu_implicit_diffusion", "pearl_gpu_valid_state",
                 "pearl_gpu_energy_mass"):
        assert must in names


def test_library_exports_every_declared_symbol(gpu_lib):
    import pearl_gpu

    lib = ctypes.CDLL(str(pearl_gpu.build.LIB))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing
    assert set(pearl_gpu.EXPORTS) == set(declared_functions())


def test_status_strings_without_device(gpu_lib):
    gpu_lib.pearl_gpu_status_string.restype = ctypes.c_char_p
    assert gpu_lib.pearl_gpu_status_string(5) == b"step retry limit"
    assert gpu_lib.pearl_gpu_status_string(4) == b"step rejected below dt_min"


def test_create_without_device_fails_cleanly(gpu_lib):
    """With no GPU the library reports PEARL_ERR_NO_DEVICE instead of falling back."""
    import torch

    import pearl_gpu
    from pearl_gpu import workloads

    if torch.cuda.is_available():
        return
    p = pearl_gpu.PearlParams.from_dict(workloads.make_params(16, 16, 2e-9, 10.0, 4e-12))
    h = ctypes.c_void_p()
    assert gpu_lib.pearl_gpu_create(ctypes.byref(p), 16, 16, 0, ctypes.byref(h)) == 12
