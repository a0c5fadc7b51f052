"""Build recipe: libdmm.so (sm_100a kernels + C ABI) and the `dynex` CLI.

    python dynex-neuromorphic-chip_b200/build.py [--force] [--debug]

Outputs (in-tree, git-ignored): ``lib/libdmm.so`` and ``bin/dynex`` next to this file.
Every translation unit is compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``
with the system g++ as host compiler (libstdc++ linked dynamically, so the library can be
loaded into processes that already hold one).
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
LIB_DIR = os.path.join(HERE, "lib")
BIN_DIR = os.path.join(HERE, "bin")
OBJ_DIR = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(LIB_DIR, "libdmm.so")
CLI = os.path.join(BIN_DIR, "dynex")

SOURCES = ["pack.cu", "cnf.cpp", "capi.cpp", "server.cpp", "noalloc.cu", "devmem.cpp"]
HEADERS = ["dmm_device.cuh", "dmm_kernels.cuh", "dmm_step.cuh", "dmm_inst.cuh", "dmm_xpose.cuh", "dmm_xprep.cuh",
           "dmm_pack.h", "devmem.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if p and os.path.exists(p):
            return p
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _flags(debug: bool) -> list[str]:
    f = ARCH + ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", _host_cxx(),
                "-I", os.path.join(ROOT, "include"), "-Xptxas", "-warn-spills"]
    f += ["-O0", "-G"] if debug else ["-O3"]
    return f


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    warn = (r.stdout + r.stderr).strip()
    if warn and "spill" in warn:
        print(warn, file=sys.stderr)


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    """Compiles the library and the CLI if any source is newer than the outputs."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "dmm.h")]
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ_DIR, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            jobs.append([nvcc, "-x", "cu", "-c", src, "-o", obj] + _flags(debug))
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for fut in [ex.submit(_run, j) for j in jobs]:
            fut.result()
    if force or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-ccbin", _host_cxx()])
    cli_src = os.path.join(HERE, "cli", "dynex.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB, hdrs[-1]])):
        _run([_host_cxx(), "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), cli_src,
              "-o", CLI, "-L", LIB_DIR, "-ldmm", "-Wl,-rpath,$ORIGIN/../lib"])
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    a = ap.parse_args()
    build(force=a.force, debug=a.debug, verbose=True)
