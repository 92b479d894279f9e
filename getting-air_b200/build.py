"""Builds the sm_100a shared library `liblbm.so` in this package directory.

Every CUDA source under csrc/ is compiled by nvcc for sm_100a only
(`-gencode arch=compute_100a,code=sm_100a`), linked against the CUDA
runtime, and written in-tree so that the library travels with the source
tree. Run as a script or call `build()`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "liblbm.so"
NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-ffp-contract=off",
    "-Xcompiler", "-fvisibility=hidden",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles csrc/*.cu into liblbm.so (skips the work when up to date)."""
    srcs = sources()
    deps = srcs + sorted(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "lbm.h"]
    if LIB.exists() and not extra:
        t = LIB.stat().st_mtime
        if all(p.stat().st_mtime <= t for p in deps):
            return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    procs = []
    for src in srcs:
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc, *NVCC_FLAGS, *(extra or []), "-I", str(HERE.parent / "include"),
               "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0 or verbose:
            sys.stdout.write(out.decode(errors="replace"))
        if pr.returncode != 0:
            failed.append(src.name)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *map(str, objs),
           "-o", str(tmp), "-cudart", "static"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, extra=[a for a in sys.argv[1:] if a != "-v"])
    print(LIB)
