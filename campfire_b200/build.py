"""Build libcampfire_gas.so in-tree with nvcc for sm_100a.

    python -m campfire_b200.build            # incremental
    python -m campfire_b200.build --force    # rebuild everything
    python -m campfire_b200.build --ptxas-v  # print registers / spills / smem per kernel

Device code is compiled with -fmad=false: every f32 operation of the WGSL
expressions is rounded separately, as in the CPU restatement of the reference.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcampfire_gas.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]
SOURCES = ["k_advect.cu", "k_diffsrc.cu", "k_forces.cu", "k_mg.cu", "k_mgf.cu", "k_mgc.cu", "k_misc.cu", "k_render.cu", "noalloc.cu", "engine.cu",
           "capi.cpp", "scene.cpp", "serve.cpp", "wood.cpp", "rigid.cpp"]
HEADERS = ["gas_dev.cuh", "kernels.h", "reduce.cuh", "engine.h", "tma.cuh", "wood.h", "rigid.h", "mg_common.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_header() -> float:
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "campfire_gas.h")]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _compile(src: str, force: bool, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), _newest_header()):
        return obj
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc()] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                                 "-I" + os.path.join(HERE, "..", "include"), "-x", "c++", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    if r.stderr.strip() and ("-Xptxas" in extra):
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_v else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force or ptxas_v, extra), SOURCES))
    if force or ptxas_v or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_v=a.ptxas_v))
