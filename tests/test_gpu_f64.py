"""FP64 CP-ALS and MTTKRP (the reference's decomposition/GPU/normal/dprice/
cp_als.cu and 4_cp_als.cu) against the FP64 oracle.  The tensor holds
float32 values so the oracle (which reads float X) sees the same numbers;
everything else is FP64 on both sides, so the results agree to rounding."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def dev64(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


@pytest.mark.parametrize("dims,R", [((20, 17, 13), 5), ((9, 8, 7, 6), 3), ((64, 33, 40), 12)])
def test_mttkrp_f64_matches_oracle(cd, dims, R):
    rng = np.random.default_rng(sum(dims) + R)
    X = rng.standard_normal(int(np.prod(dims))).astype(np.float32)
    facs = [rng.standard_normal(d * R) for d in dims]
    dX = dev64(X)
    dF = [dev64(f) for f in facs]
    for mode in range(len(dims)):
        out = torch.empty(dims[mode] * R, dtype=torch.float64, device="cuda")
        cd.mttkrp_f64(dX, dims, dF, mode, R, out)
        torch.cuda.synchronize()
        want = oracle.mttkrp(X, dims, facs, mode, R)
        got = out.cpu().numpy()
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want), mode


@pytest.mark.parametrize("dims,R,sweeps", [((20, 17, 13), 4, 8), ((9, 8, 7, 6), 3, 6)])
def test_cp_als_f64_matches_oracle(cd, dims, R, sweeps):
    rng = np.random.default_rng(7 + R)
    true = [rng.random(d * R) for d in dims]
    X = oracle.gencp(dims, true, R)
    X = (X + 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)).astype(np.float32)
    init = [rng.random(d * R) for d in dims]
    want, fits, n = oracle.cp_als(X, dims, R, init, sweeps)
    U = [dev64(f) for f in init]
    res = cd.cp_als_f64(dev64(X), dims, R, U, max_sweeps=sweeps)
    torch.cuda.synchronize()
    assert res.sweeps == sweeps == n
    for m in range(len(dims)):
        got = U[m].cpu().numpy()
        assert np.linalg.norm(got - want[m]) <= 1e-9 * np.linalg.norm(want[m]), m
    assert abs(res.fit - fits[-1]) <= 1e-10
    assert abs(res.fit - oracle.cp_fit(X, dims, [u.cpu().numpy() for u in U], R)) <= 1e-10


def test_cp_als_f64_stops(cd):
    dims, R = (24, 20, 16), 3
    rng = np.random.default_rng(3)
    X = oracle.gencp(dims, [rng.random(d * R) for d in dims], R).astype(np.float32)
    init = [rng.random(d * R) for d in dims]
    res = cd.cp_als_f64(dev64(X), dims, R, [dev64(f) for f in init], max_sweeps=500, tol=1e-9)
    assert 1 < res.sweeps < 500 and res.fit > 0.99
    res2 = cd.cp_als_f64(dev64(X), dims, R, [dev64(f) for f in init], max_sweeps=500, target_fit=0.9)
    assert res2.fit >= 0.9 and res2.sweeps <= res.sweeps


def test_cp_als_f64_rejects_bad_arguments(cd):
    X = torch.zeros(8, dtype=torch.float64, device="cuda")
    U = [torch.zeros(2 * 2, dtype=torch.float64, device="cuda") for _ in range(3)]
    with pytest.raises(cd.CudError):
        cd.cp_als_f64(X, (2, 2, 2), 0, U)
    with pytest.raises(cd.CudError):
        cd.cp_als_f64(X, (2, 2, 0), 2, U)


def subspace_gap(u, w, d, r):
    U = u.reshape(d, r, order="F")
    W = w.reshape(d, r, order="F")
    return np.linalg.norm(U @ U.T - W @ W.T)


@pytest.mark.parametrize("dims,ranks,method", [((30, 26, 22), (4, 5, 3), "hosvd"), ((12, 11, 10, 9), (3, 3, 2, 2), "hosvd"),
                                               ((30, 26, 22), (4, 5, 3), "hooi"), ((12, 11, 10, 9), (3, 3, 2, 2), "hooi")])
def test_tucker_f64_matches_oracle(cd, dims, ranks, method):
    rng = np.random.default_rng(sum(dims))
    core0 = rng.standard_normal(int(np.prod(ranks)))
    facs0 = [np.linalg.qr(rng.standard_normal((d, r)))[0].reshape(-1, order="F") for d, r in zip(dims, ranks)]
    X = oracle.gentucker(core0, ranks, facs0, dims)
    X = (X + 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)).astype(np.float32)
    core = torch.empty(int(np.prod(ranks)), dtype=torch.float64, device="cuda")
    U = [torch.empty(d * r, dtype=torch.float64, device="cuda") for d, r in zip(dims, ranks)]
    if method == "hosvd":
        st = cd.tucker_hosvd_f64(dev64(X), dims, ranks, core, U)
        core_or, facs_or = oracle.tucker_hosvd(X, dims, ranks)
    else:
        st = cd.tucker_hooi_f64(dev64(X), dims, ranks, core, U, sweeps=3)
        core_or, facs_or = oracle.tucker_hooi(X, dims, ranks, sweeps=3)
    torch.cuda.synchronize()
    assert st == cd.OK
    for u, w, d, r in zip(U, facs_or, dims, ranks):
        assert subspace_gap(u.cpu().numpy(), w, d, r) <= 1e-9
    g = core.cpu().numpy()
    assert abs(np.linalg.norm(g) - np.linalg.norm(core_or)) <= 1e-10 * np.linalg.norm(core_or)
    rec = oracle.gentucker(g, ranks, [u.cpu().numpy() for u in U], dims)
    rec_or = oracle.gentucker(core_or, ranks, facs_or, dims)
    assert np.linalg.norm(rec - rec_or) <= 1e-9 * np.linalg.norm(rec_or)
