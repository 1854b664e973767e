"""On-the-fly Gram form: A[S,S] = Phi_S^T Phi_S formed on the tensor cores.

Spec: the reference's subset Gram kernel DSG_B (ParaLanczos.cu:364-382),
restated in the oracle as ``dsg_b`` (FP64).  The GPU forms the block from a
bf16 split of the FP32 frame (x = hi + lo, lo2 = 2 lo rounded to bf16) as
F = hi hi^T + hi lo2^T + lo2 lo2^T / 4 with FP32 accumulation and returns
d_i d_j (F + F^T)_ij / 2, where d_c = ||Phi_c|| / ||hi_c + lo_c|| compensates
the split's residual per column.  Checked three ways: against that arithmetic
evaluated in FP64 (only the FP32 accumulation differs), against the oracle's
FP64 DSG_B (the split's truncation, below 2^-16 relative per entry), and the eigenvalues
of the solve against LAPACK dsyev on the FP64 Gram of the FP32 frame
(<= 1e-5 relative).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _frame(m, n, kind, seed):
    rng = np.random.default_rng(seed)
    if kind == "gauss":
        return (rng.standard_normal((m, n)) / np.sqrt(m)).astype(np.float32)
    return (rng.choice([-1.0, 1.0], size=(m, n)) / np.sqrt(m)).astype(np.float32)


def _sets(nsets, n, k, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.choice(n, size=k, replace=False) for _ in range(nsets)]).astype(np.int32)


def _split_model(Phi, S):
    """The kernel's arithmetic in FP64: bf16 pieces, exact products, and the
    per-column compensation d (rounded to FP32, as the kernel stores it)."""
    import torch
    X = torch.from_numpy(np.ascontiguousarray(Phi[:, S].T))          # k x m FP32
    hi = X.to(torch.bfloat16).float()
    lo2 = (2.0 * (X - hi)).to(torch.bfloat16).float()
    H, L = hi.double().numpy(), lo2.double().numpy()
    F = H @ H.T + H @ L.T + (L @ L.T) / 4.0
    Xr = H + L / 2.0
    ex = np.sum(X.double().numpy() ** 2, axis=1)
    rp = np.sum(Xr ** 2, axis=1)
    d = np.where((rp > 0) & (ex > 0), np.sqrt(ex / np.where(rp > 0, rp, 1.0)), 1.0).astype(np.float32)
    d = d.astype(np.float64)
    return (F + F.T) / 2.0 * np.outer(d, d)


def _gpu_frame(Phi):
    import torch

    from paralanczos_b200.api import GramFrame
    return GramFrame(torch.from_numpy(Phi).cuda())


@pytest.mark.parametrize("m,n,k", [(300, 1000, 128), (2048, 4096, 128), (130, 700, 37), (64, 500, 1),
                                   (77, 300, 64)])
def test_gram_blocks_match_split_model_and_dsg_b(m, n, k):
    import torch

    from oracle import oracle as O
    Phi = _frame(m, n, "gauss", 11)
    nsets = 40
    S = _sets(nsets, n, k, 12)
    gf = _gpu_frame(Phi)
    blocks, err = gf.blocks(torch.from_numpy(S.reshape(-1)).cuda(), k)
    blocks = blocks.cpu().numpy().astype(np.float64)
    assert (err.cpu().numpy() == 0).all()
    # exactly symmetric by construction
    assert np.array_equal(blocks, np.transpose(blocks, (0, 2, 1)))
    Phi64 = Phi.astype(np.float64)
    for s in range(nsets):
        model = _split_model(Phi, S[s])
        # FP32 accumulation over m products: a few ulps of the row scale
        scale = np.sqrt(np.outer(np.diag(model), np.diag(model))) + 1e-30
        assert np.max(np.abs(blocks[s] - model) / scale) < 2e-6, s
        ref = O.dsg_b(Phi64, S[s])
        assert np.max(np.abs(blocks[s] - ref) / scale) < 1e-5, s


def test_gram_rademacher_frame_compensated_to_fp32_accumulation():
    """A frame whose entries share one magnitude (+-1/sqrt(m)) is represented
    by the split as the same multiple of itself everywhere; the per-column
    compensation removes that factor, so the blocks agree with the FP64 DSG_B
    to the FP32 accumulation (without it they are off by ~4e-6 relative)."""
    import torch

    from oracle import oracle as O
    m, n, k = 2048, 4096, 128
    Phi = _frame(m, n, "rademacher", 13)
    S = _sets(24, n, k, 14)
    blocks, err = _gpu_frame(Phi).blocks(torch.from_numpy(S.reshape(-1)).cuda(), k)
    blocks = blocks.cpu().numpy().astype(np.float64)
    assert (err.cpu().numpy() == 0).all()
    Phi64 = Phi.astype(np.float64)
    for s in range(len(S)):
        ref = O.dsg_b(Phi64, S[s])
        scale = np.sqrt(np.outer(np.diag(ref), np.diag(ref)))
        assert np.max(np.abs(blocks[s] - ref) / scale) < 1e-6, s


def test_gram_many_sets_every_cta_wraps_the_ring():
    """More sets than 2 x SMs: every CTA reuses both accumulator buffers and
    wraps the stage ring many times; spot-check sets across the range."""
    import torch
    m, n, k, nsets = 256, 2000, 128, 1000
    Phi = _frame(m, n, "rad", 3)
    S = _sets(nsets, n, k, 4)
    gf = _gpu_frame(Phi)
    blocks, err = gf.blocks(torch.from_numpy(S.reshape(-1)).cuda(), k)
    blocks = blocks.cpu().numpy().astype(np.float64)
    assert (err.cpu().numpy() == 0).all()
    for s in list(range(0, nsets, 97)) + [nsets - 1]:
        model = _split_model(Phi, S[s])
        assert np.max(np.abs(blocks[s] - model)) < 2e-6 * np.max(np.abs(model)), s


def test_gram_bad_index_flagged_others_intact():
    import torch
    m, n, k = 128, 400, 16
    Phi = _frame(m, n, "gauss", 5)
    S = _sets(6, n, k, 6)
    S[2, 5] = n        # out of range
    S[4, 0] = -1
    gf = _gpu_frame(Phi)
    idx = torch.from_numpy(S.reshape(-1)).cuda()
    _, err = gf.blocks(idx, k)
    err = err.cpu().numpy()
    assert err[2] == 4 and err[4] == 4
    assert (err[[0, 1, 3, 5]] == 0).all()
    out = gf.solve(idx, k)
    e = out["err"].cpu().numpy()
    lmin = out["lmin"].cpu().numpy()
    assert e[2] == 4 and e[4] == 4 and np.isnan(lmin[2]) and np.isnan(lmin[4])
    assert ((e[[0, 1, 3, 5]] & ~1) == 0).all() and np.isfinite(lmin[[0, 1, 3, 5]]).all()


def test_gram_rejects_unsupported_k():
    import torch

    from paralanczos_b200._lib import PLError
    Phi = _frame(64, 300, "gauss", 1)
    gf = _gpu_frame(Phi)
    idx = torch.zeros(129 * 2, dtype=torch.int32, device="cuda")
    with pytest.raises(PLError):
        gf.solve(idx, 129)


@pytest.mark.parametrize("kind", ["gauss", "rad"])
@pytest.mark.parametrize("form", ["batched", "plain"])
def test_gram_solve_eigenvalues_vs_dsyev(kind, form):
    """C4 shape at reduced n: Phi 2048 x 4096, k = 128; lambda_min and
    lambda_max within 1e-5 relative of dsyev on the FP64 Gram of the FP32 frame."""
    import torch

    from oracle import oracle as O
    m, n, k, nsets = 2048, 4096, 128, 200
    Phi = _frame(m, n, kind, 21)
    S = _sets(nsets, n, k, 22)
    gf = _gpu_frame(Phi)
    out = gf.solve(torch.from_numpy(S.reshape(-1)).cuda(), k, form=form)
    err = out["err"].cpu().numpy()
    assert ((err & ~1) == 0).all()
    lmin, lmax = out["lmin"].cpu().numpy(), out["lmax"].cpu().numpy()
    delta = out["delta"].cpu().numpy()
    Phi64 = Phi.astype(np.float64)
    worst = 0.0
    for s in range(nsets):
        X = Phi64[:, S[s]]
        w = O.dsyev_eigs(X.T @ X)
        worst = max(worst, abs(lmin[s] - w[0]) / abs(w[0]), abs(lmax[s] - w[-1]) / abs(w[-1]))
        assert delta[s] == max(1 - lmin[s], lmax[s] - 1)
    assert worst <= 1e-5, worst


def test_gram_all_eigenvalues_and_det():
    import torch

    from oracle import oracle as O
    m, n, k, nsets = 512, 1024, 32, 50
    Phi = _frame(m, n, "gauss", 8)
    S = _sets(nsets, n, k, 9)
    gf = _gpu_frame(Phi)
    out = gf.solve(torch.from_numpy(S.reshape(-1)).cuda(), k, want_all=True)
    eig = out["eig"].cpu().numpy().reshape(nsets, k)
    det = out["det"].cpu().numpy()
    Phi64 = Phi.astype(np.float64)
    for s in range(nsets):
        X = Phi64[:, S[s]]
        w = O.dsyev_eigs(X.T @ X)
        assert np.max(np.abs(eig[s] - w) / np.abs(w).max()) < 1e-5
        assert abs(det[s] - np.prod(w)) <= 1e-4 * abs(np.prod(w))


_CHUNK_SCRIPT = r"""
import numpy as np, torch, sys
sys.path.insert(0, {root!r})
from paralanczos_b200.api import GramFrame
rng = np.random.default_rng(1)
Phi = (rng.standard_normal((256, 3000)) / 16.0).astype(np.float32)
S = np.stack([rng.choice(3000, 128, replace=False) for _ in range(700)]).astype(np.int32)
gf = GramFrame(torch.from_numpy(Phi).cuda())
o = gf.solve(torch.from_numpy(S.reshape(-1)).cuda(), 128)
np.save({path!r}, np.stack([o["lmin"].cpu().numpy(), o["lmax"].cpu().numpy()]))
"""


def test_gram_chunking_is_invisible(tmp_path):
    """700 sets through 16 MiB chunks (256 sets each) equal one chunk, bit for bit."""
    res = []
    for mb in ("16", "4096"):
        path = str(tmp_path / f"r{mb}.npy")
        env = dict(os.environ, PL_GRAM_CHUNK_MB=mb)
        subprocess.run([sys.executable, "-c", _CHUNK_SCRIPT.format(root=ROOT, path=path)],
                       check=True, env=env, timeout=300)
        res.append(np.load(path))
    assert np.array_equal(res[0], res[1])


_HOLD_SCRIPT = r"""
import numpy as np, torch, sys
sys.path.insert(0, {root!r})
from paralanczos_b200._lib import PLError, PL_ETIMEDOUT
from paralanczos_b200.api import GramFrame
import os
rng = np.random.default_rng(2)
Phi = (rng.standard_normal((256, 1000)) / 16.0).astype(np.float32)
S = np.stack([rng.choice(1000, 64, replace=False) for _ in range(300)]).astype(np.int32)
gf = GramFrame(torch.from_numpy(Phi).cuda())
idx = torch.from_numpy(S.reshape(-1)).cuda()
os.environ["PL_GRAM_TEST_HOLD"] = "1"
try:
    gf.blocks(idx, 64)
    print("no timeout")
    sys.exit(1)
except PLError as e:
    assert e.status == PL_ETIMEDOUT, e.status
os.environ["PL_GRAM_TEST_HOLD"] = "0"
b, err = gf.blocks(idx, 64)            # the context is still usable
X = torch.from_numpy(Phi[:, S[0]]).double()
ref = (X.T @ X).numpy()
assert np.max(np.abs(b[0].cpu().numpy() - ref)) < 1e-5
print("ok")
"""


def test_gram_bounded_waits_time_out_cleanly():
    """With the MMA thread held back (a test switch), every bounded wait of the
    Gram kernel gives up after 2 s: the call returns PL_ETIMEDOUT, TMEM is
    freed, and the next call in the same process succeeds."""
    r = subprocess.run([sys.executable, "-c", _HOLD_SCRIPT.format(root=ROOT)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
