"""Build the in-tree CUDA library ``ertm_b200/libertm_b200.so`` for sm_100a.

    python challenge-cup_b200/build.py [--verbose-ptxas]

nvcc cross-compiles without a GPU.  The shared library is written next to
the Python package so it travels with the repository snapshot.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "ertm_b200" / "libertm_b200.so"
SOURCES = [CSRC / "ertm_b200.cu"]
DEPS = sorted(CSRC.glob("*.cu*")) + [HERE.parent / "include" / "ertm_b200.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else "nvcc"


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    built = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= built for p in DEPS + [Path(__file__)])


def build(force: bool = False, ptxas_verbose: bool = False) -> Path:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC,-O3", "-shared", "-o", str(OUT), *map(str, SOURCES), "-lcufft"]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    tmp = OUT.with_suffix(".so.tmp")
    cmd[cmd.index(str(OUT))] = str(tmp)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc failed with exit code {res.returncode}")
    if ptxas_verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    p = build(force=True, ptxas_verbose="--verbose-ptxas" in sys.argv)
    print(p)
