"""In-tree build of libpearl_gpu.so (sm_100a) and the pearl_gpu host executable.

nvcc cross-compiles for sm_100a without a GPU, so this runs on any host with
the CUDA 12.9 toolchain.  Outputs go to ``<package>/build/`` (git-ignored, but
shipped with the repository snapshot to GPU hosts).
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent.parent  # fe-c_eutectoid_phase-field_simulation_b200/
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
INCLUDE = ROOT / "include"
BUILD = PKG / "build"
LIB = BUILD / "libpearl_gpu.so"
CLI = BUILD / "pearl_gpu"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# FP64 path: -fmad=false keeps every multiply and add separately rounded, as in
# the reference built for plain x86-64, so per-cell results match bitwise.
# (object, source, flags); the phases and kernels are compiled once per block
# shape: 8 warps (namespace g8) and 16 warps (namespace g16).
CU_SOURCES = [
    ("pearl_fp64_g8", "pearl_fp64.cu", ["-fmad=false", "-DPEARL_TILE_WARPS=8"]),    # phases and kernels
    ("pearl_fp64_g16", "pearl_fp64.cu", ["-fmad=false", "-DPEARL_TILE_WARPS=16"]),
    ("pearl_ctx", "pearl_ctx.cu", ["-fmad=false"]),            # context, transfers, single-domain C ABI
    ("pearl_batch", "pearl_batch.cu", ["-fmad=false"]),        # batched instances
    ("pearl_adjoint_host", "pearl_adjoint_host.cu", ["-fmad=false"]),  # adjoint gradient driver
    ("pearl_noalloc", "pearl_noalloc.cu", ["-fmad=false"]),    # step without device allocation
]
# host driver (the pearl_gpu executable): C++17, linked against libpearl_gpu.so
CLI_SOURCES = ["config.cpp", "io.cpp", "main.cpp"]


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _newer(out: Path, inputs: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in inputs if p.exists())


def sources() -> list[Path]:
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp"))
    deps += list(HOST.glob("*.cpp")) + list(HOST.glob("*.hpp")) + list(INCLUDE.glob("*.h"))
    return deps


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    deps = sources() + [Path(__file__)]
    if force or _newer(LIB, deps):
        objs, cmds = [], []
        for stem, name, extra in CU_SOURCES:
            obj = BUILD / (stem + ".o")
            cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", *extra, "-Xcompiler", "-fPIC",
                   f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(CSRC / name), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            cmds.append(cmd)
            objs.append(obj)
        # the translation units are independent: compile them side by side
        with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
            for f in [pool.submit(_run, c) for c in cmds]:
                f.result()
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(LIB)])
    if force or _newer(CLI, deps + [LIB]):
        # -ffp-contract=off: host arithmetic that mirrors the reference (temperature
        # laws, initial geometry) is rounded operation by operation like it
        _run(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-ffp-contract=off", f"-I{INCLUDE}", f"-I{HOST}",
              *[str(HOST / n) for n in CLI_SOURCES], f"-L{BUILD}", "-lpearl_gpu", "-Wl,-rpath,$ORIGIN",
              "-pthread", "-o", str(CLI)])
    return LIB


if __name__ == "__main__":
    import sys

    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
