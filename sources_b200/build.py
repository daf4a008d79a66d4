"""Builds libsphg.so in-tree with nvcc for sm_100a.

    python -m sources_b200.build        (or __graft_entry__.build())

The library is a plain shared object with a C ABI (include/sphg.h); it links
only the CUDA runtime.  -Xptxas -v output goes to _build/ptxas.log.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = [os.path.join(HERE, "csrc", "sphg_api.cu"), os.path.join(HERE, "csrc", "sphg_noalloc.cu"),
       os.path.join(HERE, "csrc", "sphg_io.cpp"), os.path.join(HERE, "csrc", "sphg_scenes.cpp"),
       os.path.join(HERE, "csrc", "sphg_umma.cu"),
       os.path.join(HERE, "csrc", "sphg_gnn.cu")]
OUT = os.path.join(HERE, "libsphg.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    d = os.path.join(HERE, "csrc")
    inc = os.path.join(ROOT, "include")
    return [os.path.join(d, f) for f in sorted(os.listdir(d))] + [os.path.join(inc, f) for f in sorted(os.listdir(inc))]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force: bool = False, verbose: bool = False, defines=(), out: str = OUT) -> str:
    if not force and out == OUT and up_to_date():
        return OUT
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    tmp = out + ".tmp"
    # -prec-div/-prec-sqrt=false only affect float arithmetic (the FP32 pair
    # mode); double division and sqrt stay IEEE.
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-prec-div=false", "-prec-sqrt=false",
           "-shared", "-Xcompiler", "-fPIC",
           "-Xptxas", "-v", *["-D" + d for d in defines], "-o", tmp, *SRC, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(HERE, "_build", "ptxas.log") if out == OUT else out + ".ptxas.log"
    with open(log, "w") as f:
        f.write(r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-8000:])
        raise RuntimeError("nvcc failed building libsphg.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
