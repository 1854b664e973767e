"""Build libparalanczos_b200.so (sm_100a) in-tree with nvcc.

    python -m paralanczos_b200.build [--verbose-ptxas] [--jobs N]

Each translation unit under csrc/ is compiled separately (in parallel) and
linked into paralanczos_b200/libparalanczos_b200.so with the CUDA runtime
linked statically, so the library loads in any process (with or without
PyTorch) and does not depend on a JIT cache.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libparalanczos_b200.so")
# PTX of the reference-named kernels, for MATLAB's parallel.gpu.CUDAKernel
PTX = os.path.join(PKG, "ParaLanczos.ptx")
UNITS = ["pl_api.cu", "pl_dropin.cu", "pl_compat.cu", "pl_gram.cu", "pl_serve.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    "-diag-suppress", "177,550",
]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _sources():
    return [u for u in UNITS if os.path.exists(os.path.join(CSRC, u))]


def _deps_mtime() -> float:
    m = 0.0
    for f in os.listdir(CSRC):
        m = max(m, os.path.getmtime(os.path.join(CSRC, f)))
    m = max(m, os.path.getmtime(os.path.join(PKG, "..", "include", "paralanczos.h")))
    return m


def up_to_date() -> bool:
    return os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime()


def build(verbose_ptxas: bool = False, jobs: int = 0, force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    host = shutil.which("g++") or "/usr/bin/g++"
    objs = []
    cmds = []
    for u in _sources():
        obj = os.path.join(BUILD, u.replace(".cu", ".o"))
        cmd = [cc, *NVCC_FLAGS, "-ccbin", host, "-c", os.path.join(CSRC, u), "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        cmds.append(cmd)
        objs.append(obj)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(cmds))) as ex:
        for cmd, r in ex.map(run, cmds):
            if r.returncode != 0 or verbose_ptxas:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
    link = [cc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-ccbin", host, *objs,
            "-o", LIB + ".tmp", "-cudart", "static"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(LIB + ".tmp", LIB)
    compat = os.path.join(CSRC, "pl_compat.cu")
    if os.path.exists(compat):
        r = subprocess.run([cc, "-arch=compute_100a", "-std=c++17", "--expt-relaxed-constexpr",
                            "-diag-suppress", "177,550", "-ptx", compat, "-o", PTX],
                           capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("ptx failed")
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose_ptxas, a.jobs, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
