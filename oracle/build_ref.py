"""Compile the reference's own host-compilable routines into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  The product never loads what this script builds.

The reference (ParaLanczos v0.21) keeps its tridiagonal eigensolver in plain C
marked ``__device__``: ``TQLRAT`` (ParaLanczos.cu:32-189) and ``DET_TRIDIAG``
(ParaLanczos.cu:243-269), with the macros they use in ParaLanczos0.h:13-32.
This recipe cuts those two functions and the macro block out of the read-only
reference tree *at build time*, drops the ``__device__``/``__inline__``
qualifiers, and compiles them with gcc into ``oracle/_ref/libplref.so``.  The
extracted source is written under ``oracle/_ref/`` only, which is git-ignored:
no reference source enters the repository.  Tests use the library to pin the
oracle's own restatement (oracle/pl_oracle.c) bit-for-bit.

It also compiles the reference's first example program (example1.cu, its
caller of calculate_subeigs) against the reference's own ParaLanczos.h into
``oracle/_ref/example1.o`` (object only), so a test can link that unchanged
caller to libparalanczos_b200.so and run it.

The reference tree is found at $PL_REFERENCE_DIR, else at the default below.

Usage: python oracle/build_ref.py [--ref DIR]
Exit status 0 also when the reference tree is absent (nothing to build).
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
DEFAULT_REF = "/root/reference"


def reference_dir() -> str | None:
    """The reference tree ($PL_REFERENCE_DIR or the default), if present."""
    d = os.environ.get("PL_REFERENCE_DIR") or DEFAULT_REF
    return d if os.path.isfile(os.path.join(d, "ParaLanczos.cu")) else None


def _cut_function(src: str, name: str) -> str:
    """Return the full definition of function `name` (signature to closing brace)."""
    m = re.search(r"^[^\n;{}]*\b" + re.escape(name) + r"\s*\([^)]*\)\s*\{", src, re.M)
    if not m:
        raise RuntimeError(f"function {name} not found in reference source")
    start = m.start()
    depth = 0
    i = src.index("{", m.start())
    while i < len(src):
        if src[i] == "{":
            depth += 1
        elif src[i] == "}":
            depth -= 1
            if depth == 0:
                return src[start:i + 1]
        i += 1
    raise RuntimeError(f"unbalanced braces in {name}")


def _macro_block(hdr: str) -> str:
    keep = ("DBL_EPSILON", "_POW2", "_ABS", "_PYTHAG", "_SIGN", "_EPSILON")
    lines = []
    for line in hdr.splitlines():
        s = line.strip()
        if s.startswith("#define"):
            parts = s.split()
            macro = parts[1].split("(")[0] if len(parts) > 1 else ""
            if macro in keep:
                lines.append(f"#undef {macro}")
                lines.append(s)
    return "\n".join(lines)


def build(ref_dir: str) -> str | None:
    cu = os.path.join(ref_dir, "ParaLanczos.cu")
    h0 = os.path.join(ref_dir, "ParaLanczos0.h")
    if not (os.path.isfile(cu) and os.path.isfile(h0)):
        return None
    with open(cu, encoding="utf-8", errors="replace") as f:
        src = f.read()
    with open(h0, encoding="utf-8", errors="replace") as f:
        hdr = f.read()
    parts = [
        "/* Extracted at build time from the reference tree; not part of the repository. */",
        "#include <math.h>",
        _macro_block(hdr),
    ]
    for name in ("TQLRAT", "DET_TRIDIAG"):
        body = _cut_function(src, name)
        body = re.sub(r"\b__device__\b|\b__inline__\b|\b__host__\b", "", body)
        parts.append(body)
    parts.append("int plref_tqlrat(int n, double *d, double *e2) { return TQLRAT(n, d, e2); }")
    parts.append("double plref_det_tridiag(int n, double *a, double *b) { return DET_TRIDIAG(n, a, b); }")
    os.makedirs(OUT_DIR, exist_ok=True)
    c_path = os.path.join(OUT_DIR, "ref_tqlrat.c")
    with open(c_path, "w") as f:
        f.write("\n\n".join(parts) + "\n")
    so_path = os.path.join(OUT_DIR, "libplref.so")
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-w", c_path, "-o", so_path, "-lm"]
    subprocess.run(cmd, check=True)
    return so_path


def build_example(ref_dir: str) -> str | None:
    """example1.cu compiled, unchanged, against the reference's ParaLanczos.h."""
    src = os.path.join(ref_dir, "example1.cu")
    if not (os.path.isfile(src) and os.path.isfile(os.path.join(ref_dir, "ParaLanczos.h"))):
        return None
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    obj = os.path.join(OUT_DIR, "example1.o")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-I", ref_dir, "-w", "-c", src,
                    "-o", obj], check=True)
    return obj


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference tree (default: $PL_REFERENCE_DIR or the default)")
    a = ap.parse_args()
    ref = a.ref or reference_dir()
    out = build(ref) if ref else None
    print(out if out else "reference tree absent; nothing built")
    if ref:
        ex = build_example(ref)
        if ex:
            print(ex)
    return 0


if __name__ == "__main__":
    sys.exit(main())
