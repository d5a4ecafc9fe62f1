"""Build libirs_b200.so in this folder (nvcc, sm_100a only).

    python irsounderlbl.jl_b200/build.py [--force] [-v]

The library is built in-tree so that it travels with the repository to the GPU
host; there is no JIT cache and no other architecture.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SO = HERE / "libirs_b200.so"
SOURCES = [HERE / "csrc" / "irs_b200.cu", HERE / "csrc" / "noalloc.cu", HERE / "csrc" / "surrogate.cu",
           HERE / "csrc" / "irs_host.cpp", HERE / "csrc" / "relmat.cpp", HERE / "csrc" / "shard.cpp"]
DEPS = SOURCES + sorted((HERE / "csrc").glob("*.cuh")) + sorted((HERE / "csrc").glob("*.h")) + \
    [HERE.parent / "include" / "irs_b200.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# -fcx-limited-range: host complex products and quotients by the textbook formulas (the
# eigensolver of relmat.cpp; its values are finite and moderate) instead of libgcc calls.
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fcx-limited-range", "-shared"]


def up_to_date() -> bool:
    return SO.exists() and all(SO.stat().st_mtime >= d.stat().st_mtime for d in DEPS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return SO
    cmd = [NVCC, *FLAGS, *(["-Xptxas", "-v"] if verbose else []), *map(str, SOURCES), "-o", str(SO)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stderr)
    return SO


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
