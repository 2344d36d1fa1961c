"""Build libmag_b200.so in-tree with nvcc for sm_100a (no JIT cache, no torch).

    python -m mag_b200.build            # incremental
    python -m mag_b200.build --force    # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmag_b200.so")
SOURCES = ["kernels_force.cu", "kernels_update.cu", "kernels_wloop.cu", "kernels_nersc.cu", "kernels_demon.cu", "kernels_matrix.cu", "kernels_multi.cu", "mag_api.cu",
           "mag_nersc_api.cu", "mag_dd.cu", "mag_multi_api.cu",
           "noalloc.cu",
           "nersc_host.cpp"]
HEADERS = ["su3.cuh", "lattice.cuh", "gauge_ops.cuh", "rng.cuh", "kernels.h", "nersc_host.h", "ctx.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "mag_c.h"), os.path.join(ROOT, "include", "mag_diag.h")]
    if _newer(obj, deps):
        cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        with open(obj.replace(".o", ".log"), "w") as f:
            f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-4000:]}")
    return obj


def build(force: bool = False, verbose_ptxas: bool = True) -> str:
    """Compile every CUDA source for sm_100a and link libmag_b200.so."""
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for f in os.listdir(OBJ):
            if f.endswith(".o"):
                os.remove(os.path.join(OBJ, f))
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    if _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
