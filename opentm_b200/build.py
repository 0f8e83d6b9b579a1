"""Build the sm_100a CUDA library ``libopentm_b200.so`` in-tree with nvcc.

Usage: ``python -m opentm_b200.build`` (or ``opentm_b200.build.build()``). The library is
written next to this file so that it travels with the source tree; nothing is installed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD_DIR = os.path.join(HERE, "_build")
LIB_NAME = "libopentm_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = [
    "otm_template.cpp",
    "otm_homo.cu",
    "otm_filter.cu",
    "otm_oc.cu",
    "otm_mma.cu",
    "otm_server.cu",
    "otm_noalloc.cu",
    "otm_pool.cu",
    "otm_init.cu",
    "otm_driver.cu",
]


def nvcc_path() -> str:
    cand = [os.environ.get("CUDACXX"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build opentm_b200")


def host_compiler() -> list[str]:
    # The image's $CXX may be a compiler without its runtime pieces; use the system g++.
    gxx = shutil.which("g++")
    return ["-ccbin", gxx] if gxx else []


def _compile(src: str, verbose: bool) -> str:
    nvcc = nvcc_path()
    obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc, *host_compiler(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd.insert(-4, "-x")
        cmd.insert(-4, "cu")
    if verbose:
        cmd.insert(-4, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False, jobs: int = 6) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(o) for o in objs):
        return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc_path(), *host_compiler(), *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static",
           "-Xlinker", "--exclude-libs,ALL"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
