"""The C-ABI library loads and exports every symbol the public headers declare;
host-only entry points and argument validation work without a GPU."""
import os
import re
import subprocess

import numpy as np

from paralanczos_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_c_symbols():
    src = open(os.path.join(ROOT, "include", "paralanczos.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pl_[a-z0-9_]+)\s*\(", src)))


def _exported():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_library_exports_every_declared_c_symbol():
    decl = _declared_c_symbols()
    assert len(decl) >= 15
    exp = _exported()
    missing = [s for s in decl if s not in exp]
    assert not missing, missing
    # the ctypes binding covers exactly the declared surface
    assert sorted(_lib.SIGNATURES) == decl


def test_library_exports_reference_cxx_symbols():
    # mangled names the reference's objects link against (ParaLanczos.h:39-47;
    # `nm example3.o` references _Z18calculate_subeigs3PdiiS_S_Pii)
    exp = _exported()
    for sym in ["_Z18calculate_subeigs3PdiiS_S_Pii", "_Z17calculate_subeigsPdiS_S_Pii",
                "_Z18calculate_subeigs2PdiiS_S_Pii", "_Z14calculate_eigsPdiS_S_",
                "_Z17print_tridiagonalPdS_i"]:
        assert sym in exp, sym


def test_cxx_header_declares_reference_signatures():
    src = open(os.path.join(ROOT, "include", "ParaLanczos.h")).read()
    for sig in ["void calculate_subeigs3(double *mat, int subIndexLen, int matsize, double *Eigenvalues, "
                "double *Det, int *subIndex, int subn)",
                "void calculate_subeigs(double *mat, int n, double *Eigenvalues, double *Det, int *subIndex, "
                "int subn)"]:
        assert " ".join(sig.split()) in " ".join(src.split())


def test_host_entry_points_without_gpu():
    L = _lib.lib()
    assert L.pl_version() == 100
    assert L.pl_status_string(0) == b"ok"
    assert L.pl_num_bins() >= 6
    assert [L.pl_bin_kmax(b) for b in range(L.pl_num_bins())][-1] == _lib.PL_KMAX
    # argument validation happens before any device work
    A = np.zeros((4, 4), np.float32)
    idx = np.zeros(4, np.int32)
    assert L.pl_solve(A.ctypes.data, 4, 3, idx.ctypes.data, None, 1, 4, 0, None, None, None, None,
                      None, None, None) == _lib.PL_EINVAL          # lda < n
    assert L.pl_solve(A.ctypes.data, 4, 4, idx.ctypes.data, None, 1, 600, 0, None, None, None, None,
                      None, None, None) == _lib.PL_ENOTSUP         # k > PL_KMAX
    assert L.pl_solve(A.ctypes.data, 4, 4, idx.ctypes.data, None, 1, 0, 0, None, None, None, None,
                      None, None, None) == _lib.PL_EINVAL          # k < 1
    assert L.pl_solve(A.ctypes.data, 4, 4, idx.ctypes.data, None, 1, 4, 7, None, None, None, None,
                      None, None, None) == _lib.PL_EINVAL          # unknown form
    assert L.pl_solve(A.ctypes.data, 4, 4, idx.ctypes.data, None, 0, 4, 0, None, None, None, None,
                      None, None, None) == _lib.PL_OK              # empty batch
    assert L.pl_gen_sets(1, 0, 10, 4, 8, None, None) == _lib.PL_EINVAL


def test_dropin_reference_validation_messages(capfd):
    # calculate_subeigs3 keeps the reference's checks and messages
    # (ParaLanczos.cu:1814-1824) and returns before touching the GPU
    from paralanczos_b200 import api
    mat = np.eye(8)
    eig = np.zeros(128)
    det = np.zeros(32)
    sub = np.zeros(128, np.int32)
    assert api.calculate_subeigs3(mat, 128, 8, eig, det, sub, 6) == _lib.PL_EINVAL
    assert "'int subn' must be divisible by 4" in capfd.readouterr().err
    assert api.calculate_subeigs3(mat, 120, 8, eig, det, sub, 4) == _lib.PL_EINVAL
    assert "'subIndexLen' must be divisible by 32" in capfd.readouterr().err


def test_reference_example1_object_links(tmp_path):
    """The reference's example1.cu, compiled against the reference's own
    ParaLanczos.h (oracle/_ref/example1.o, built when the reference tree is
    present), resolves every symbol it needs from libparalanczos_b200.so."""
    import shutil

    import pytest
    obj = os.path.join(ROOT, "oracle", "_ref", "example1.o")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(obj) or not os.path.exists(nvcc):
        pytest.skip("reference example1 object or nvcc absent")
    _lib.lib()
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", obj, "-o", str(tmp_path / "example1"),
                    "-L", libdir, "-lparalanczos_b200", "-Xlinker", f"-rpath={libdir}"], check=True,
                   capture_output=True, text=True, timeout=300)
    undef = subprocess.run(["nm", "-u", obj], capture_output=True, text=True, check=True).stdout
    assert "_Z17calculate_subeigsPdiS_S_Pii" in undef
