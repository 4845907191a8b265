"""Build the in-tree CUDA library libimogen_b200.so for sm_100a (nvcc, no JIT cache).

The kernels are split over several translation units (host code; fluid and magnet sweeps per
precision; the MAT-file slice reader/writer, host C++ linked with zlib) that compile in parallel and
link into one shared library with the CUDA runtime linked statically."""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
UNITS = ["imogen_b200.cu", "fluid_f32.cu", "fluid_f64.cu", "magnet_f32.cu", "magnet_f64.cu", "fluid_cluster.cu",
         "matfile.cpp", "server.cpp"]
# per-unit ptxas options: the batched cluster fluid kernels are compiled at -O1 (fluid_cluster.cu says why)
UNIT_FLAGS = {"fluid_cluster.cu": ["-Xptxas", "-O1"]}
OUT = os.path.join(HERE, "libimogen_b200.so")
HEADER = os.path.join(ROOT, "include", "imogen_b200.h")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [HEADER]


def up_to_date(out=OUT):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in sources() if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    """Compile csrc/*.cu (one process per translation unit) and link libimogen_b200.so."""
    if not force and up_to_date():
        return OUT
    cc = nvcc()
    tmp = tempfile.mkdtemp(prefix="imogen_b200_build_")
    try:
        def compile_unit(unit):
            obj = os.path.join(tmp, os.path.splitext(unit)[0] + ".o")
            cmd = [cc, *ARCH, *FLAGS, *UNIT_FLAGS.get(unit, []), "-I", os.path.join(ROOT, "include"), "-c",
                   os.path.join(CSRC, unit), "-o", obj, *extra]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            return unit, obj, r

        with concurrent.futures.ThreadPoolExecutor(len(UNITS)) as ex:
            results = list(ex.map(compile_unit, UNITS))
        for unit, _, r in results:
            if verbose or r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {unit}")
        link = [cc, *ARCH, "-shared", "-cudart", "static", *[o for _, o, _ in results], "-lz", "-o", OUT + ".tmp"]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libimogen_b200.so failed")
        os.replace(OUT + ".tmp", OUT)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
