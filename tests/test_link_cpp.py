"""Link compatibility with the reference's C++ callers.

The reference's examples include ParaLanczos.h and call calculate_subeigs3 /
calculate_eigs with C++ linkage (their objects reference
_Z18calculate_subeigs3PdiiS_S_Pii).  These tests link such callers to
libparalanczos_b200.so with no other change, run them on the GPU and check
the eigenvalues and determinants against LAPACK dsyev: a small C++ program of
this project compiled against include/ParaLanczos.h, and the reference's own
example1.cu compiled unchanged against the reference's header.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include "ParaLanczos.h"

// A = B^T B for a fixed 24 x 16 B (so A is symmetric positive definite).
int main() {
  const int n = 16, m = 24, k = 8, nsets = 4;
  double B[m * n], A[n * n];
  unsigned s = 12345u;
  for (int i = 0; i < m * n; ++i) {
    s = s * 1103515245u + 12345u;
    B[i] = ((double)((s >> 8) & 0xffff) / 65536.0 - 0.5) / 3.0;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double a = 0.0;
      for (int r = 0; r < m; ++r) a += B[r * n + i] * B[r * n + j];
      A[i * n + j] = a;
    }
  int S[nsets * k];
  for (int t = 0; t < nsets; ++t)
    for (int c = 0; c < k; ++c) S[t * k + c] = (3 * t + 5 * c) % n;
  double eig[nsets * k], det[nsets], all[n], detall;
  calculate_subeigs3(A, nsets * k, n, eig, det, S, k);
  calculate_eigs(A, n, all, &detall);
  for (int i = 0; i < n * n; ++i) printf("A %.17g\n", A[i]);
  for (int i = 0; i < nsets * k; ++i) printf("S %d\n", S[i]);
  for (int i = 0; i < nsets * k; ++i) printf("E %.17g\n", eig[i]);
  for (int i = 0; i < nsets; ++i) printf("D %.17g\n", det[i]);
  for (int i = 0; i < n; ++i) printf("F %.17g\n", all[i]);
  printf("G %.17g\n", detall);
  return 0;
}
"""


def test_cpp_program_links_and_runs(tmp_path):
    from oracle import oracle as O
    from paralanczos_b200 import _lib
    _lib.lib()  # built
    cxx = shutil.which("g++")
    assert cxx, "g++ not found"
    src = tmp_path / "caller.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "paralanczos_b200")
    cmd = [cxx, "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L", libdir,
           "-lparalanczos_b200", f"-Wl,-rpath,{libdir}"]
    # the library file is libparalanczos_b200.so: -l finds it by that name
    subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=120)
    r = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120)
    vals = {}
    for line in r.stdout.splitlines():
        tag, v = line.split()
        vals.setdefault(tag, []).append(float(v))
    n, k = 16, 8
    A = np.array(vals["A"]).reshape(n, n)
    S = np.array(vals["S"], dtype=int).reshape(-1, k)
    E = np.array(vals["E"]).reshape(-1, k)
    for t in range(S.shape[0]):
        w = O.dsyev_eigs(A[np.ix_(S[t], S[t])])
        assert np.max(np.abs(E[t] - w)) <= 1e-5 * np.max(np.abs(w))
        assert abs(vals["D"][t] - np.prod(w)) <= 1e-4 * abs(np.prod(w))
    w = O.dsyev_eigs(A)
    assert np.max(np.abs(np.array(vals["F"]) - w)) <= 1e-5 * np.max(np.abs(w))
    assert abs(vals["G"][0] - np.prod(w)) <= 1e-4 * abs(np.prod(w))


EXAMPLE1_OBJ = os.path.join(ROOT, "oracle", "_ref", "example1.o")


def _link_example1(tmp_path):
    """The reference's own example1.cu, compiled unchanged against the
    reference's ParaLanczos.h at build time (oracle/build_ref.py writes
    oracle/_ref/example1.o), linked to libparalanczos_b200.so."""
    from paralanczos_b200 import _lib
    _lib.lib()
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    libdir = os.path.join(ROOT, "paralanczos_b200")
    exe = tmp_path / "example1"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", EXAMPLE1_OBJ, "-o", str(exe), "-L", libdir,
                    "-lparalanczos_b200", "-Xlinker", f"-rpath={libdir}"], check=True, capture_output=True,
                   text=True, timeout=300)
    return exe


@pytest.mark.skipif(not os.path.exists(EXAMPLE1_OBJ), reason="reference example1 object not built")
def test_reference_example1_runs_against_the_library(tmp_path):
    """example1.cu (ParaLanczos example1.cu:14-54): calculate_subeigs on its 8 x 8
    matrix (example1.cu:19-26) with the subset {1, 3, 5, 7} (example1.cu:39-42).
    It allocates Eigenvalues[8] and one Det, enough for the 4 eigenvalues and the
    determinant the call writes.  With PL_VERBOSE=1 the library prints the
    reference's "%d eigenvalue: %g" lines, checked against dsyev."""
    import json

    from oracle import oracle as O
    exe = _link_example1(tmp_path)
    env = dict(os.environ, PL_VERBOSE="1")
    r = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120, env=env)
    got = [float(line.split(":")[1]) for line in r.stdout.splitlines() if "eigenvalue:" in line]
    fx = json.load(open(os.path.join(ROOT, "tests", "golden", "fixture8.json")))
    g = np.array(fx["matrix"]).reshape(8, 8)
    w = O.dsyev_eigs(g[np.ix_([1, 3, 5, 7], [1, 3, 5, 7])])
    assert len(got) == 4, r.stdout
    # %g prints six significant digits
    np.testing.assert_allclose(got, w, rtol=1e-5)
