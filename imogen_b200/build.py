"""Build the in-tree CUDA library libimogen_b200.so for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "imogen_b200.cu")
OUT = os.path.join(HERE, "libimogen_b200.so")
DEPS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
DEPS.append(os.path.join(ROOT, "include", "imogen_b200.h"))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date(out=OUT, deps=DEPS):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    """Compile csrc/imogen_b200.cu into libimogen_b200.so (static cudart, -fPIC).

    IMOGEN_CHECKED=1 in the environment adds -DIMG_CHECKED (access checks that record instead of
    faulting), for diagnosing a kernel on a small case."""
    if os.environ.get("IMOGEN_CHECKED") == "1":
        extra = tuple(extra) + ("-DIMG_CHECKED",)
        force = True
    if not force and up_to_date():
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-cudart", "static", "-I", os.path.join(ROOT, "include"), SRC, "-o", OUT + ".tmp", *extra]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed for libimogen_b200.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
