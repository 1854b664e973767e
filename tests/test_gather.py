"""The gather alone (pl_gather_blocks): A[S,S] blocks bit for bit.

Spec: the reference's gather LOAD_SMS4H / LOAD_SMS4HF (ParaLanczos.cu:455-490),
A_S[r][c] = mat[S[r] * n + S[c]].  For a symmetric FP32 matrix the blocks must
equal plain indexing exactly (no arithmetic is involved), bad indices are
flagged per set, and uneven leading dimensions are honoured.  The kernel reads
only A[S_i, S_j] with i <= j (A is symmetric), so for a matrix that is not
symmetric block s is the upper triangle of A[S, S] mirrored: that is checked
too, as the documented behaviour.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 5, 16, 64, 128, 300, 512])
def test_gather_blocks_exact(k):
    import torch

    from paralanczos_b200 import api
    rng = np.random.default_rng(k)
    n, lda, nsets = 700, 720, 97
    full = rng.standard_normal((n, lda)).astype(np.float32)
    full[:, :n] = np.triu(full[:, :n]) + np.triu(full[:, :n], 1).T   # symmetric n x n part
    A = torch.from_numpy(full).cuda()[:, :n]          # row stride lda > n
    assert A.stride(0) == lda
    S = np.stack([rng.choice(n, size=k, replace=False) for _ in range(nsets)]).astype(np.int32)
    blocks, err = api.gather_blocks(A, torch.from_numpy(S.reshape(-1)).cuda(), k)
    blocks = blocks.cpu().numpy()
    assert (err.cpu().numpy() == 0).all()
    for s in range(nsets):
        assert np.array_equal(blocks[s], full[np.ix_(S[s], S[s])])


@pytest.mark.parametrize("k", [3, 64, 130])
def test_gather_reads_one_triangle(k):
    import torch

    from paralanczos_b200 import api
    rng = np.random.default_rng(100 + k)
    n, nsets = 400, 9
    full = rng.standard_normal((n, n)).astype(np.float32)       # not symmetric
    S = np.stack([rng.choice(n, size=k, replace=False) for _ in range(nsets)]).astype(np.int32)
    blocks, _ = api.gather_blocks(torch.from_numpy(full).cuda(), torch.from_numpy(S.reshape(-1)).cuda(), k)
    blocks = blocks.cpu().numpy()
    for s in range(nsets):
        G = full[np.ix_(S[s], S[s])]
        assert np.array_equal(blocks[s], np.triu(G) + np.triu(G, 1).T)


def test_gather_bad_index_flagged():
    import torch

    from paralanczos_b200 import api
    rng = np.random.default_rng(1)
    n, k, nsets = 300, 24, 6
    A = torch.from_numpy(rng.standard_normal((n, n)).astype(np.float32)).cuda()
    S = np.stack([rng.choice(n, size=k, replace=False) for _ in range(nsets)]).astype(np.int32)
    S[2, 3] = -1
    S[5, 0] = n
    blocks, err = api.gather_blocks(A, torch.from_numpy(S.reshape(-1)).cuda(), k)
    e = err.cpu().numpy()
    assert e[2] == 4 and e[5] == 4 and (e[[0, 1, 3, 4]] == 0).all()
    assert (blocks[2].cpu().numpy() == 0).all()
