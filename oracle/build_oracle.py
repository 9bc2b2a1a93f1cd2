"""Build recipe for the test oracle (test infrastructure, not the product).

* ``oracle/libpearl_oracle.so`` — the C restatement ``pearl_oracle.c``.
* ``oracle/_ref/libpearl_ref.so`` and ``oracle/_ref/pearl_serial`` — the
  UNMODIFIED reference solver compiled from its own single source file where
  it lies (``PEARL_REFERENCE_DIR``, default ``/root/reference``), against the
  stand-in ``oracle/hdf5_stub/hdf5.h`` because libhdf5 is not installed.
  The harness #includes the reference file; nothing is copied.

Outputs go to ``oracle/`` (ignored ``*.so``) and ``oracle/_ref/`` (ignored).
Both travel with the repository snapshot to a GPU host, where the reference
source itself is absent; ``build()`` therefore skips the reference part when
the source directory is missing and keeps an existing prebuilt copy.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
ORACLE_SO = HERE / "libpearl_oracle.so"
REF_SO = REF_OUT / "libpearl_ref.so"
REF_CLI = REF_OUT / "pearl_serial"

# The reference's own CMake adds -Wall -Wextra -Wpedantic; -O3 -DNDEBUG is the
# optimised serial build used for every CPU timing.  No -march: the reference
# build targets plain x86-64, so no multiply-add is contracted.
REF_FLAGS = ["-std=c++17", "-O3", "-DNDEBUG", "-Wall", "-Wextra", "-Wpedantic"]


def reference_dir() -> Path:
    return Path(os.environ.get("PEARL_REFERENCE_DIR", "/root/reference"))


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(out: Path, *inputs: Path) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.exists() and p.stat().st_mtime > t for p in inputs)


def build_port(force: bool = False) -> Path:
    src = HERE / "pearl_oracle.c"
    adj = HERE / "pearl_adjoint.c"
    hdr = HERE / "pearl_oracle.h"
    if force or _stale(ORACLE_SO, src, adj, hdr):
        # -fopenmp: the device-order mode runs its per-cell loops on host threads
        # (off by default; results do not depend on the thread count)
        _run(["gcc", "-std=c99", "-O3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-Wall", "-Wextra",
              "-Wno-maybe-uninitialized", str(src), str(adj), "-o", str(ORACLE_SO), "-lm"])
    return ORACLE_SO


def build_reference(force: bool = False) -> bool:
    """Compile the reference harness and CLI.  Returns False when the source is absent."""
    ref = reference_dir()
    src = ref / "pearl_serial.cpp"
    if not src.exists():
        return REF_SO.exists()
    REF_OUT.mkdir(exist_ok=True)
    stub = HERE / "hdf5_stub"
    deps = (src, stub / "hdf5.h", HERE / "ref_harness.cpp", HERE / "pearl_oracle.h")
    if force or _stale(REF_SO, *deps):
        _run(["g++", *REF_FLAGS, "-fPIC", "-shared", f"-I{stub}", f"-I{HERE}", f"-I{ref}",
              str(HERE / "ref_harness.cpp"), "-o", str(REF_SO)])
    if force or _stale(REF_CLI, src, stub / "hdf5.h"):
        _run(["g++", *REF_FLAGS, f"-I{stub}", str(src), "-o", str(REF_CLI)])
    return True


def build(force: bool = False) -> None:
    build_port(force)
    build_reference(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(ORACLE_SO, REF_SO if REF_SO.exists() else "(reference not built)")
