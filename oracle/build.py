"""Builds the oracle (test infrastructure) into oracle/_build/liboracle.so.

The oracle is a CPU restatement of the reference's shader arithmetic and is
only ever loaded by the tests, by the smoke check and by the benchmark's
CPU-baseline leg.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "liboracle.so"
SOURCES = ["dense_oracle.cpp", "amr2d_oracle.cpp", "amr3d_oracle.cpp", "sample_oracle.cpp"]
FLAGS = ["-std=c++17", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared"]


def _cxx() -> str:
    # The system g++ carries libgomp; a wrapper named by $CXX may not.
    for cand in ("/usr/bin/g++", os.environ.get("CXX"), "g++"):
        if cand and (os.path.sep not in cand or Path(cand).exists()):
            return cand
    return "g++"


def build() -> Path:
    srcs = [HERE / s for s in SOURCES]
    deps = srcs + [HERE / "common.h", HERE / "body.h", HERE / "dense3.h", HERE.parent / "include" / "lbm.h"]
    if OUT.exists() and all(p.stat().st_mtime <= OUT.stat().st_mtime for p in deps):
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    subprocess.run([_cxx(), *FLAGS, *map(str, srcs), "-o", str(tmp)], check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build())
