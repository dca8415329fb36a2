"""Leading eigenvectors by subspace iteration (cud_syev_top), the partial
eigensolver behind the Tucker factors (the reference asks cuSOLVER's
syevdx for the leading eigenpairs, src/tucker_hosvd.cu:43-61), against
numpy.linalg.eigh on matrices with a planted spectrum.

Shapes cover the cluster fast path (r <= 32, n <= 2048) at its edges --
n below the cluster's eight row blocks, an odd r (one unpaired index per
Jacobi round), n = 2048 (the largest shared-memory layout) -- and the
generic path (r > 32, n > 2048).  Eigenvectors are compared through
residuals and subspaces (signs are arbitrary).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def planted(n, r, seed, tail=0.3):
    """G = Q diag(lam) Q^T: the r leading eigenvalues spread over [1, 2],
    the rest in [0, tail] (lam_{r+1} / lam_r <= tail)."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.concatenate([np.linspace(1.0, 2.0, r), tail * rng.random(n - r)])
    return (Q * lam) @ Q.T


def run(cd, G, n, r, U0=None, max_iters=300):
    dG = torch.from_numpy(np.asfortranarray(G).reshape(-1, order="F").copy()).cuda()
    U = torch.full((n * r,), 7.0, dtype=torch.float32, device="cuda")
    u0 = None if U0 is None else torch.from_numpy(U0.reshape(-1, order="F").astype(np.float32)).cuda()
    st = cd.syev_top(dG, n, r, U, u0, max_iters=max_iters)
    torch.cuda.synchronize()
    return st, U.cpu().numpy().reshape(n, r, order="F").astype(np.float64)


def check(G, U, r):
    w, V = np.linalg.eigh(G)
    W = V[:, -r:]
    lam = w[-r:]
    assert np.linalg.norm(U @ U.T - W @ W.T) <= 2e-5 * np.sqrt(r)
    assert np.linalg.norm(U.T @ U - np.eye(r)) <= 2e-5 * np.sqrt(r)
    ritz = np.einsum("ij,ik,kj->j", U, G, U)
    assert np.all(np.diff(ritz) >= -1e-6)                      # ascending, the largest last
    np.testing.assert_allclose(ritz, lam, rtol=1e-6)
    res = np.linalg.norm(G @ U - U * ritz, axis=0)
    assert res.max() <= 2e-5 * np.abs(lam).max()


@pytest.mark.parametrize("n,r", [(20, 3), (64, 1), (100, 17), (512, 32), (2048, 32), (300, 40), (2049, 8)])
def test_leading_eigenvectors(cd, n, r):
    G = planted(n, r, seed=n + r)
    st, U = run(cd, G, n, r)
    assert st == cd.OK
    check(G, U, r)


def test_deterministic(cd):
    G = planted(512, 16, seed=5)
    _, U1 = run(cd, G, 512, 16)
    _, U2 = run(cd, G, 512, 16)
    assert np.array_equal(U1, U2)


def test_warm_start_and_rank_deficient_start(cd):
    n, r = 384, 24
    G = planted(n, r, seed=9)
    W = np.linalg.eigh(G)[1][:, -r:]
    rng = np.random.default_rng(10)
    st, U = run(cd, G, n, r, U0=W + 1e-3 * rng.standard_normal(W.shape))
    assert st == cd.OK
    check(G, U, r)
    # a zero start block fails CholQR; the solver restarts from a random block
    st, U = run(cd, G, n, r, U0=np.zeros((n, r)))
    assert st == cd.OK
    check(G, U, r)


def test_not_converged_leaves_output(cd):
    n, r = 256, 8
    G = planted(n, r, seed=11, tail=0.95)
    st, U = run(cd, G, n, r, max_iters=1)
    assert st == cd.ERR_NOT_CONVERGED
    assert np.all(U == 7.0)


def test_invalid_arguments(cd):
    G = torch.zeros(16, dtype=torch.float64, device="cuda")
    U = torch.zeros(16 * 5, dtype=torch.float32, device="cuda")
    with pytest.raises(cd.CudError):
        cd.syev_top(G, 4, 5, U)          # r > n
    with pytest.raises(cd.CudError):
        cd.syev_top(G, 4, 0, U)
