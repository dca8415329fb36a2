"""Tucker path on the GPU: generators, mode products (TTM), unfolding Grams,
the FP64 Jacobi eigensolver, HOSVD and HOOI against the oracle.

Eigenvector signs and the order within degenerate eigenspaces are arbitrary
(src/tucker_hosvd.cu:68-70 takes whatever cuSOLVER returns), so factors are
compared as subspaces: ||U U^T - W W^T||_F <= 1e-4, and cores through their
norm and the reconstruction error.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def dev_t(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_golden_generators(cd, golden):
    A, B, C, core = (dev_t(golden[k]) for k in ("gen_A", "gen_B", "gen_C", "gen_core"))
    rec = torch.empty(8, device="cuda")
    cd.gencp(rec, [A, B, C], (2, 2, 2), 2)
    np.testing.assert_array_equal(host(rec), golden["gen_cp"])
    cd.gentucker(rec, core, [A, B, C], (2, 2, 2), (2, 2, 2))
    np.testing.assert_array_equal(host(rec), golden["gen_tucker"])
    hA, hB, hC, hG = (dev_t(golden[k]) for k in ("ht_A", "ht_B", "ht_C", "ht_G"))
    rec = torch.empty(24, device="cuda")
    cd.gentucker(rec, hG, [hA, hB, hC], (3, 4, 2), (2, 2, 2))
    np.testing.assert_array_equal(host(rec), golden["ht_rec"])


@pytest.mark.parametrize("dims,R", [((30, 20, 10), 5), ((9, 8, 7, 6), 4), ((200, 3, 5), 2)])
def test_gencp_random(cd, dims, R):
    rng = np.random.default_rng(R)
    facs = [rng.random(d * R).astype(np.float32) for d in dims]
    rec = torch.empty(int(np.prod(dims)), device="cuda")
    cd.gencp(rec, [dev_t(f) for f in facs], dims, R)
    assert rel(host(rec).astype(np.float64), oracle.gencp(dims, facs, R)) <= 1e-6


@pytest.mark.parametrize("flag", [1, 2, 3])
def test_golden_ttm(cd, golden, flag):
    X = dev_t(golden["ttm_X"])
    U = dev_t(golden[f"ttm_U{flag}"])
    n = {1: 2 * 9, 2: 3 * 2 * 3, 3: 9 * 2}[flag]
    out = torch.empty(n, device="cuda")
    cd.ttm(X, U, out, flag, 3, 3, 3, 2, precision=cd.PREC_FP32)
    assert rel(host(out).astype(np.float64), golden[f"ttm_out{flag}"]) <= 1e-6
    cd.ttm(X, U, out, flag, 3, 3, 3, 2, precision=cd.PREC_FP16)
    want = oracle.ttm(golden["ttm_X"], golden[f"ttm_U{flag}"], flag, 3, 3, 3, 2, round_fp16=True)
    assert rel(host(out).astype(np.float64), want) <= 1e-6


@pytest.mark.parametrize("dims", [(40, 30, 20), (7, 9, 11, 5), (100, 1, 3)])
def test_mode_product_and_gram(cd, dims):
    rng = np.random.default_rng(sum(dims))
    X = rng.standard_normal(int(np.prod(dims))).astype(np.float32)
    dX = dev_t(X)
    for mode in range(len(dims)):
        J = 3 + mode
        W = rng.standard_normal(J * dims[mode]).astype(np.float32)
        out_dims = list(dims)
        out_dims[mode] = J
        Y = torch.empty(int(np.prod(out_dims)), device="cuda")
        cd.mode_product(dX, dims, mode, dev_t(W), J, Y)
        want, _ = oracle.mode_product(X, dims, mode, W, J)
        assert rel(host(Y).astype(np.float64), want) <= 1e-5
        G = torch.empty(dims[mode] ** 2, dtype=torch.float64, device="cuda")
        cd.unfold_gram(dX, dims, mode, G)
        assert rel(host(G).reshape(dims[mode], dims[mode]), oracle.unfold_gram(X, dims, mode)) <= 1e-6


@pytest.mark.parametrize("n", [2, 16, 33, 100, 257])
def test_jacobi_eigensolver(cd, n):
    rng = np.random.default_rng(n)
    Z = rng.standard_normal((n, n))
    A = Z @ Z.T + np.diag(np.linspace(0, 1, n))
    dA = dev_t(A.reshape(-1, order="F"), np.float64)
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    V = torch.empty(n * n, dtype=torch.float64, device="cuda")
    st = cd.syev_jacobi(dA, n, W, V)
    assert st == cd.OK
    w = host(W)
    v = host(V).reshape(n, n, order="F")
    we = np.linalg.eigvalsh(A)
    assert np.all(np.diff(w) >= -1e-12 * abs(we).max())
    np.testing.assert_allclose(w, we, atol=1e-11 * abs(we).max())
    assert np.linalg.norm(A @ v - v * w) <= 1e-10 * np.linalg.norm(A)
    assert np.linalg.norm(v.T @ v - np.eye(n)) <= 1e-10 * n


def tucker_data(dims, ranks, seed, noise=1e-3):
    rng = np.random.default_rng(seed)
    core = rng.standard_normal(int(np.prod(ranks)))
    facs = [np.linalg.qr(rng.standard_normal((d, r)))[0].reshape(-1, order="F") for d, r in zip(dims, ranks)]
    X = oracle.gentucker(core, ranks, facs, dims)
    X = X + noise * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)
    return X.astype(np.float32)


def subspace_gap(u, w, d, r):
    U = u.reshape(d, r, order="F").astype(np.float64)
    W = w.reshape(d, r, order="F")
    return np.linalg.norm(U @ U.T - W @ W.T)


@pytest.mark.parametrize("dims,ranks", [((40, 36, 32), (4, 5, 6)), ((16, 14, 12, 10), (3, 3, 2, 2)),
                                        ((130, 20, 18), (8, 4, 4))])
@pytest.mark.parametrize("method", ["hosvd", "hooi"])
def test_tucker_vs_oracle(cd, dims, ranks, method):
    X = tucker_data(dims, ranks, seed=sum(dims))
    dX = dev_t(X)
    U = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
    core = torch.empty(int(np.prod(ranks)), device="cuda")
    if method == "hosvd":
        cd.tucker_hosvd(dX, dims, ranks, core, U)
        core_or, facs_or = oracle.tucker_hosvd(X, dims, ranks)
    else:
        cd.tucker_hooi(dX, dims, ranks, core, U, sweeps=3)
        core_or, facs_or = oracle.tucker_hooi(X, dims, ranks, sweeps=3)
    for u, w, d, r in zip(U, facs_or, dims, ranks):
        assert subspace_gap(host(u), w, d, r) <= 1e-4
        uu = host(u).reshape(d, r, order="F").astype(np.float64)
        assert np.linalg.norm(uu.T @ uu - np.eye(r)) <= 1e-5
    g = host(core).astype(np.float64)
    assert abs(np.linalg.norm(g) - np.linalg.norm(core_or)) <= 1e-5 * np.linalg.norm(core_or)
    # reconstruction error equals the oracle's
    rec = torch.empty(X.size, device="cuda")
    cd.gentucker(rec, core, U, dims, ranks)
    err = rel(host(rec).astype(np.float64), X.astype(np.float64))
    err_or = rel(oracle.gentucker(core_or, ranks, facs_or, dims), X.astype(np.float64))
    assert abs(err - err_or) <= 1e-5


@pytest.mark.parametrize("dims,ranks", [((64, 48, 40), (8, 6, 5)), ((32, 24, 16, 40), (4, 3, 2, 5))])
@pytest.mark.parametrize("precision", ["bf16x3", "bf16"])
@pytest.mark.parametrize("method", ["hosvd", "hooi"])
def test_tucker_tensor_cores_vs_oracle(cd, dims, ranks, precision, method):
    """Tensor-core Grams (BF16 / three-term split) and BF16 TTM chains against
    the FP64 oracle: the factor subspaces, and the core through the
    reconstruction error."""
    X = tucker_data(dims, ranks, seed=sum(dims) + len(precision))
    dX = dev_t(X)
    U = [torch.zeros(d * r, device="cuda") for d, r in zip(dims, ranks)]
    core = torch.zeros(int(np.prod(ranks)), device="cuda")
    prec = cd.PRECISIONS[precision]
    if method == "hosvd":
        cd.tucker_hosvd(dX, dims, ranks, core, U, precision=prec)
        core_or, facs_or = oracle.tucker_hosvd(X, dims, ranks)
    else:
        cd.tucker_hooi(dX, dims, ranks, core, U, sweeps=3, precision=prec)
        core_or, facs_or = oracle.tucker_hooi(X, dims, ranks, sweeps=3)
    # three-term Grams are FP32-accurate; a BF16 operand (the one-term Gram,
    # and HOOI's projections of the BF16 copy of X) perturbs X by about
    # 2^-9 relative -- as much again as the data's own 1e-3 noise
    gap_tol = 2e-4 if (precision == "bf16x3" and method == "hosvd") else 2e-2
    for u, w, d, r in zip(U, facs_or, dims, ranks):
        assert subspace_gap(host(u), w, d, r) <= gap_tol
    rec = torch.empty(int(np.prod(dims)), device="cuda")
    cd.gentucker(rec, core, U, dims, ranks)
    err = float(torch.linalg.norm((dX - rec).double()) / torch.linalg.norm(dX.double()))
    rec_or = oracle.gentucker(core_or, ranks, facs_or, dims)
    err_or = float(np.linalg.norm(X.astype(np.float64) - rec_or) / np.linalg.norm(X.astype(np.float64)))
    # BF16 TTM inputs: the core carries relative errors of about 2^-9
    assert err <= err_or + 5e-3
