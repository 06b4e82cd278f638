"""Build libglc.so (the CUDA product) in-tree for sm_100a.

    python g-leco_b200/build.py [--verbose-ptxas]

Compiles every csrc/*.cu with nvcc (-gencode arch=compute_100a,code=sm_100a -lineinfo -O3) and
links g-leco_b200/glc/libglc.so.  Objects go to g-leco_b200/_build/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "glc", "libglc.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "glc.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps) and not verbose_ptxas:
        return obj
    cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        # export only the C ABI (glc_*): the exports of the shared object are include/glc.h
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-Xcompiler", "-fvisibility=hidden"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_dropin()
    build_percall()
    return OUT


def build_percall() -> str:
    """Compile the per-call request loop the serving benchmark compares against
    (g-leco_b200/percall/percall.cpp -> _build/libglc_percall.so, linked to libglc)."""
    src = os.path.join(HERE, "percall", "percall.cpp")
    so = os.path.join(BUILD, "libglc_percall.so")
    hdr = os.path.join(ROOT, "include", "glc.h")
    if os.path.exists(so) and all(os.path.getmtime(so) >= os.path.getmtime(d) for d in (src, OUT, hdr)):
        return so
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I" + os.path.join(ROOT, "include"), src, "-L" + os.path.dirname(OUT), "-lglc",
           "-Wl,-rpath,$ORIGIN/../glc", "-o", so]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"per-call loop failed to compile:\n{r.stderr}")
    return so


def build_dropin() -> str:
    """Compile the C++ caller of the drop-in LeCoGPU<T> header (tests/cpp/leco_dropin.cpp)."""
    src = os.path.join(ROOT, "tests", "cpp", "leco_dropin.cpp")
    exe = os.path.join(BUILD, "leco_dropin")
    hdrs = [os.path.join(ROOT, "include", h) for h in ("glc.h", "glc_leco.hpp", "glc_io.hpp")]
    if os.path.exists(exe) and all(os.path.getmtime(exe) >= os.path.getmtime(d) for d in [src, OUT] + hdrs):
        return exe
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(
        subprocess.run(["which", NVCC], capture_output=True, text=True).stdout.strip() or "/usr/local/cuda/bin/nvcc"))),
        "include")
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-I" + cuda_inc,
           src, "-L" + os.path.dirname(OUT), "-lglc", "-Wl,-rpath,$ORIGIN/../glc", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"drop-in caller failed to compile:\n{r.stderr}")
    return exe


if __name__ == "__main__":
    print(build("--verbose-ptxas" in sys.argv))
