"""Build libdaw_b200.so (and the main_redatum_daw driver) in-tree for sm_100a.

    python build.py [--force] [-j N]

Objects go to _build/ beside this file; the shared library and the driver
executable are written next to this file so they travel with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libdaw_b200.so")
EXE = os.path.join(HERE, "main_redatum_daw")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          f"-I{INCLUDE}", f"-I{CSRC}"]
LIB_SOURCES = ["hicks.cpp", "engine.cu", "stencil_plain.cu", "stencil_fused.cu", "stencil_tma.cu", "stencil_step.cu",
               "minres.cu",
               "filter.cu", "filter_noalloc.cu", "driver.cpp"]


def _needs(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "daw_b200.h"))
    return hs


def _compile(src: str, verbose: bool) -> str:
    out = os.path.join(OBJ, os.path.basename(src) + ".o")
    cmd = [NVCC, *ARCH, *COMMON, "-c", src, "-o", out]
    if src.endswith(".cu"):
        cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    return out


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    todo = [s for s in srcs
            if force or _needs(os.path.join(OBJ, os.path.basename(s) + ".o"), [s, *hdrs])]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            list(ex.map(lambda s: _compile(s, verbose), todo))
    objs = [os.path.join(OBJ, os.path.basename(s) + ".o") for s in srcs]
    if force or _needs(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        subprocess.run(cmd, check=True)
    main_src = os.path.join(CSRC, "main.cpp")
    if force or _needs(EXE, [main_src, LIB, *hdrs]):
        cmd = [NVCC, *ARCH, *COMMON, main_src, "-o", EXE, f"-L{HERE}", "-ldaw_b200",
               f"-Xlinker=-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
