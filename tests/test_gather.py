"""The gather alone (pl_gather_blocks): A[S,S] blocks bit for bit.

Spec: the reference's gather LOAD_SMS4H / LOAD_SMS4HF (ParaLanczos.cu:455-490),
A_S[r][c] = mat[S[r] * n + S[c]].  The blocks must equal plain indexing of the
same FP32 matrix exactly (no arithmetic is involved), bad indices are flagged
per set, and uneven leading dimensions are honoured.
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
    A = torch.from_numpy(full).cuda()[:, :n]          # row stride lda > n
    assert A.stride(0) == lda
    S = np.stack([rng.choice(n, size=k, replace=False) for _ in range(nsets)]).astype(np.int32)
    blocks, err = api.gather_blocks(A, torch.from_numpy(S.reshape(-1)).cuda(), k)
    blocks = blocks.cpu().numpy()
    assert (err.cpu().numpy() == 0).all()
    for s in range(nsets):
        assert np.array_equal(blocks[s], full[np.ix_(S[s], S[s])])


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
