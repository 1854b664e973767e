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

Usage: python oracle/build_ref.py [--ref DIR]   (default DIR: /root/reference)
Exit status 0 also when the reference tree is absent (nothing to build).
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")


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


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    out = build(a.ref)
    print(out if out else "reference tree absent; nothing built")
    return 0


if __name__ == "__main__":
    sys.exit(main())
