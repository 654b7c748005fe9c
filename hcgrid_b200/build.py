"""Compile the gridder's shared library in-tree for sm_100a.

    python -m hcgrid_b200.build

Produces hcgrid_b200/lib/libhcgrid_b200.so (CUDA runtime linked
statically) from hcgrid_b200/csrc/. Host code is compiled with
-ffp-contract=off so the host-side HEALPix setup rounds like the reference.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libhcgrid_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["hcg_field.cu", "hcg_grid.cu", "hcg_batch.cu", "hcg_noalloc.cu", "hcg_tc.cu", "hcg_capi.cu",
              "hcg_shard.cu"]
CXX_SOURCES = ["hcg_wcs.cpp", "hcg_fits.cpp", "hcg_compat.cpp", "hcg_server.cpp"]
CLI = os.path.join(PKG, "bin", "HCGrid")


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: %s" % os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    objs = []
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "hcgrid_c.h")]
    newest_dep = max(os.path.getmtime(d) for d in deps)
    log = ""
    for src in CU_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep and not ptxas_info:
            continue
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
               "-Xcompiler", "-fPIC,-ffp-contract=off", *inc, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        log += _run(cmd)
    for src in CXX_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
            continue
        cmd = ["g++", "-O2", "-fPIC", "-ffp-contract=off", "-std=c++17", "-pthread", *inc,
               "-I", "/usr/local/cuda/include", "-c", os.path.join(CSRC, src), "-o", obj]
        log += _run(cmd)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        log += _run([nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-Xlinker", "-lpthread"])
    # flag-compatible command line (HCGrid/HCGrid.cpp) linked against the library
    cli_src = os.path.join(CSRC, "hcg_cli.cpp")
    if not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(LIB), os.path.getmtime(cli_src)):
        os.makedirs(os.path.dirname(CLI), exist_ok=True)
        log += _run(["g++", "-O2", "-std=c++17", *inc, cli_src, "-o", CLI, "-L", LIBDIR, "-lhcgrid_b200",
                     "-Wl,-rpath,$ORIGIN/../lib"])
    if verbose and log:
        print(log)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
