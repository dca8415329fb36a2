"""CP-ALS on the GPU against the oracle's restatement of src/cp_als.cu and
src/cp4_als.cu (same initial factors).

Tolerances: the fit after a fixed number of sweeps within 1e-4 of the FP64
oracle (the final-fit bar), factors within 1e-3 relative Frobenius norm.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def dev_t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def low_rank(dims, R, seed, noise=1e-3):
    rng = np.random.default_rng(seed)
    true = [rng.random(d * R) for d in dims]
    X = oracle.gencp(dims, true, R)
    X = X + noise * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)
    init = [rng.random(d * R).astype(np.float32) for d in dims]
    return X.astype(np.float32), init


@pytest.mark.parametrize("layout", [1, 2])
@pytest.mark.parametrize("prec", ["fp32", "bf16x3", "default"])
@pytest.mark.parametrize("dims,R", [((30, 25, 20), 4), ((16, 12, 10, 8), 3), ((64, 64, 64), 16)])
def test_fixed_sweeps_match_oracle(cd, prec, dims, R, layout):
    """Both sweep layouts: 1 (split reduce, update with Gram, V^-1 beside the
    MTTKRP) and 2 (partials summed in the update, Gram and next V^-1 beside
    the next MTTKRP, four sweeps a graph: 15 = 3 x 4 + 3 singles)."""
    X, init = low_rank(dims, R, seed=len(dims) * 100 + R)
    sweeps = 15
    facs_or, fits_or, n_or = oracle.cp_als(X, dims, R, init, sweeps)
    U = [dev_t(f) for f in init]
    res = cd.cp_als(dev_t(X), dims, R, U, max_sweeps=sweeps, tol=0.0,
                    precision=cd.PRECISIONS[prec], layout=layout)
    assert res.sweeps == sweeps
    assert abs(res.fit - fits_or[-1]) <= 1e-4, (res.fit, fits_or[-1])
    for u, f in zip(U, facs_or):
        g = u.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(g - f) / np.linalg.norm(f) <= 1e-3


def test_stopping_rule_matches_oracle(cd):
    dims, R = (40, 36, 32), 5
    X, init = low_rank(dims, R, seed=7)
    facs_or, fits_or, n_or = oracle.cp_als(X, dims, R, init, 50, tol=1e-6)
    U = [dev_t(f) for f in init]
    res = cd.cp_als(dev_t(X), dims, R, U, max_sweeps=50, tol=1e-6)
    assert abs(res.sweeps - n_or) <= 2, (res.sweeps, n_or)
    assert abs(res.fit - fits_or[-1]) <= 1e-4


@pytest.mark.parametrize("layout", [1, 2])
def test_graph_and_eager_agree(cd, layout):
    dims, R = (24, 20, 18), 4
    X, init = low_rank(dims, R, seed=9)
    Ua = [dev_t(f) for f in init]
    Ub = [dev_t(f) for f in init]
    ra = cd.cp_als(dev_t(X), dims, R, Ua, max_sweeps=12, use_graph=True, layout=layout)
    rb = cd.cp_als(dev_t(X), dims, R, Ub, max_sweeps=12, use_graph=False, layout=layout)
    assert ra.fit == rb.fit
    for a, b in zip(Ua, Ub):
        assert torch.equal(a, b)


@pytest.mark.parametrize("check_every,layout", [(1, 1), (3, 1), (2, 2)])
def test_device_loop_stops_like_host_loop(cd, check_every, layout):
    """With a Delta-fit tolerance the sweeps run in a graph whose WHILE node
    judges the tolerance on the device; the eager path (no graph) keeps the
    host loop.  Same sweep count, same fit, same factors."""
    dims, R = (40, 36, 32), 5
    X, init = low_rank(dims, R, seed=17, noise=1e-2)
    Ua = [dev_t(f) for f in init]
    Ub = [dev_t(f) for f in init]
    ra = cd.cp_als(dev_t(X), dims, R, Ua, max_sweeps=200, tol=1e-5, check_every=check_every, layout=layout)
    rb = cd.cp_als(dev_t(X), dims, R, Ub, max_sweeps=200, tol=1e-5, check_every=check_every, layout=layout,
                   use_graph=False)
    assert 2 <= ra.sweeps < 200 and ra.sweeps % check_every == 0
    assert ra.sweeps == rb.sweeps and ra.fit == rb.fit
    for a, b in zip(Ua, Ub):
        assert torch.equal(a, b)


def test_four_sweep_graph_equals_single_sweeps(cd):
    """Layout 2 replays four sweeps as one graph (each sweep's last Gram and
    fit beside the next sweep's first MTTKRP); the factors and fits must be
    the ones four single-sweep replays give, bit for bit."""
    dims, R = (96, 80, 72), 16
    X, init = low_rank(dims, R, seed=13)
    dX = dev_t(X)
    Ua = [dev_t(f) for f in init]
    Ub = [dev_t(f) for f in init]
    pa = cd.CpPlan(dX, dims, R, Ua, precision=cd.PREC_BF16X3, layout=2)
    pb = cd.CpPlan(dX, dims, R, Ub, precision=cd.PREC_BF16X3, layout=2)
    pa.run(8)
    for _ in range(8):
        pb.run(1)
    torch.cuda.synchronize()
    assert pa.fit() == pb.fit()
    for a, b in zip(Ua, Ub):
        assert torch.equal(a, b)
    pa.close(); pb.close()


def test_layouts_agree_at_benchmark_size(cd):
    """512 x 512 x 512 rank 64, BF16x3: 8 sweeps in each layout from the same
    start reach the same fit to 1e-6 and factors to 1e-3, the oracle bar (they
    differ only in the order of the split sums, which ALS amplifies in the
    factors, not in the fit)."""
    dims, R = (512, 512, 512), 64
    X, _ = cd.make_cp_tensor(dims, R, seed=5)
    init = cd.make_init(dims, R, seed=6)
    res = {}
    for layout in (1, 2):
        U = [u.clone() for u in init]
        r = cd.cp_als(X, dims, R, U, max_sweeps=8, precision=cd.PREC_BF16X3, layout=layout)
        res[layout] = (r.fit, [u.double() for u in U])
    assert abs(res[1][0] - res[2][0]) <= 1e-6, (res[1][0], res[2][0])
    for a, b in zip(res[1][1], res[2][1]):
        assert float(torch.linalg.norm(a - b) / torch.linalg.norm(a)) <= 1e-3


def test_curand_init_and_500_sweeps_like_reference(cd):
    """cp_als() of src/cp_als.cu:20-24,42: cuRAND seed 1234 init of B then C,
    500 sweeps; checked against the oracle from the same initial factors."""
    dims, R = (12, 10, 8), 3
    X, _ = low_rank(dims, R, seed=21)
    U = [torch.zeros(d * R, device="cuda") for d in dims]
    cd.cp_init_curand(dims, R, U, 1234)
    init = [u.cpu().numpy() for u in U]
    assert init[1].min() >= 0 and init[1].max() <= 1 and init[2].std() > 0.1
    facs_or, fits_or, _ = oracle.cp_als(X, dims, R, init, 500)
    res = cd.cp_als(dev_t(X), dims, R, U, max_sweeps=500)
    assert abs(res.fit - fits_or[-1]) <= 1e-4


def test_singular_normal_equations_fall_back(cd):
    """Two identical factor columns make the Hadamard of Grams singular: the
    Cholesky fails and the pseudo-inverse path must keep the update finite."""
    dims, R = (10, 9, 8), 2
    rng = np.random.default_rng(4)
    X = rng.random(int(np.prod(dims))).astype(np.float32)
    init = []
    for d in dims:
        col = rng.random(d)
        init.append(np.concatenate([col, col]).astype(np.float32))
    U = [dev_t(f) for f in init]
    res = cd.cp_als(dev_t(X), dims, R, U, max_sweeps=3)
    assert res.fallbacks >= 1
    for u in U:
        assert torch.isfinite(u).all()


def test_fit_matches_reconstruction(cd):
    dims, R = (20, 16, 12), 3
    X, init = low_rank(dims, R, seed=31, noise=1e-2)
    U = [dev_t(f) for f in init]
    res = cd.cp_als(dev_t(X), dims, R, U, max_sweeps=20)
    rec = torch.empty(int(np.prod(dims)), device="cuda")
    cd.gencp(rec, U, dims, R)
    Xd = dev_t(X)
    direct = 1.0 - torch.linalg.norm((Xd - rec).double()) / torch.linalg.norm(Xd.double())
    assert abs(res.fit - float(direct)) <= 1e-5


@pytest.mark.parametrize("dims,R", [((20, 16, 12), 3), ((37, 23, 11), 70), ((6, 5, 4, 7), 3),
                                    ((130, 9, 5), 129)])
def test_cp_residual_matches_reconstruction(cd, dims, R):
    """src/rse.cu:4 (norm of X - gencp(U)) against an FP64 reconstruction;
    ranks above 64 take the multi-pass branch, mode 0 above 64 several
    row tiles."""
    rng = np.random.default_rng(len(dims) * 100 + R)
    X = rng.random(int(np.prod(dims))).astype(np.float32)
    facs = [rng.random(d * R).astype(np.float32) for d in dims]
    rec = oracle.gencp(dims, [f.astype(np.float64) for f in facs], R)
    want_r2 = float(np.sum((X.astype(np.float64) - rec) ** 2))
    want_x2 = float(np.sum(X.astype(np.float64) ** 2))
    r2, x2 = cd.cp_residual(dev_t(X), dims, [dev_t(f) for f in facs], R)
    assert abs(x2 - want_x2) <= 1e-12 * want_x2
    assert abs(r2 - want_r2) <= 1e-5 * want_r2


@pytest.mark.parametrize("dims,R", [((256, 200, 64), 16), ((96, 96, 40, 12), 32), ((512, 512, 32), 64),
                                    ((132, 260, 9), 40)])
def test_cp_residual_tensor_core_near_its_data(cd, dims, R):
    """The tensor-core residual (order >= 3, R <= 64: BF16x3 reconstruction
    in TMEM) on a model at fit ~0.999 of its tensor, where the residual is a
    small difference: the residual within 1e-3 (relative) and the fit within
    1e-6 of FP64 (ragged row tiles and U_1 chunks included)."""
    rng = np.random.default_rng(sum(dims) + R)
    facs = [rng.standard_normal(d * R).astype(np.float32) for d in dims]
    rec = oracle.gencp(dims, [f.astype(np.float64) for f in facs], R)
    X = (rec + 1e-3 * np.linalg.norm(rec) / np.sqrt(rec.size) * rng.standard_normal(rec.size)).astype(np.float32)
    Xd = X.astype(np.float64)
    want_r2 = float(np.sum((Xd - rec) ** 2))
    want_x2 = float(np.sum(Xd ** 2))
    r2, x2 = cd.cp_residual(dev_t(X), dims, [dev_t(f) for f in facs], R)
    assert abs(x2 - want_x2) <= 1e-12 * want_x2
    assert abs(r2 - want_r2) <= 1e-3 * want_r2, (r2, want_r2)
    fit, want_fit = 1 - np.sqrt(r2 / x2), 1 - np.sqrt(want_r2 / want_x2)
    assert abs(fit - want_fit) <= 1e-6, (fit, want_fit)


def test_plan_true_fit_matches_direct(cd):
    dims, R = (40, 32, 24), 5
    X, init = low_rank(dims, R, seed=41, noise=1e-2)
    U = [dev_t(f) for f in init]
    Xd = dev_t(X)
    plan = cd.CpPlan(Xd, dims, R, U, precision=cd.PREC_FP32)
    plan.run(15)
    tf = plan.true_fit()
    rec = torch.empty(int(np.prod(dims)), device="cuda")
    cd.gencp(rec, U, dims, R)
    direct = 1.0 - torch.linalg.norm((Xd - rec).double()) / torch.linalg.norm(Xd.double())
    assert abs(tf - float(direct)) <= 1e-6
    plan.close()


def test_repeated_call_reuses_plan_and_matches_a_fresh_one(cd):
    """cud_cp_als keeps its plan for a call with the same buffers: after the
    tensor's and the factors' contents change, the cached plan must give
    exactly what a freshly built plan gives (||X||^2 and the Grams come from
    the data on every call)."""
    rng = np.random.default_rng(21)
    dims, R = (64, 48, 40), 8
    n = int(np.prod(dims))
    X = torch.from_numpy(rng.random(n).astype(np.float32)).cuda()
    U = [torch.from_numpy(rng.random(d * R).astype(np.float32)).cuda() for d in dims]
    cd.cp_als(X, dims, R, U, max_sweeps=6)          # builds and keeps the plan
    X2 = rng.random(n).astype(np.float32)
    init2 = [rng.random(d * R).astype(np.float32) for d in dims]
    X.copy_(torch.from_numpy(X2))
    for u, i in zip(U, init2):
        u.copy_(torch.from_numpy(i))
    a = cd.cp_als(X, dims, R, U, max_sweeps=6)      # the kept plan
    got = [u.cpu().numpy().copy() for u in U]
    cd.cp_als_release()
    for u, i in zip(U, init2):
        u.copy_(torch.from_numpy(i))
    b = cd.cp_als(X, dims, R, U, max_sweeps=6)      # a fresh plan
    for g, u in zip(got, U):
        np.testing.assert_array_equal(g, u.cpu().numpy())
    assert a.fit == b.fit and a.sweeps == b.sweeps


def test_cp_tensorcore_drop_in_fp16(cd, capfd):
    """cp_tensorcore (src/tensorcore_cp.cu:3-150): cuRAND's default generator
    seeded 1234 for B then C, 500 ALS sweeps with FP16 MTTKRP operands, the
    relative error printed.  Our drop-in (C++ symbol, through the library)
    against the FP64 oracle's ALS from the same start: the FP16 operand
    rounding (11-bit mantissas) moves the fit by at most 2e-3."""
    import ctypes
    rng = np.random.default_rng(22)
    dims, R = (40, 32, 24), 4
    true = [rng.random(d * R) for d in dims]
    X = oracle.gencp(dims, true, R)
    X = (X + 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)).astype(np.float32)
    dX = torch.from_numpy(X).cuda()
    U = [torch.zeros(d * R, device="cuda") for d in dims]
    # the start the drop-in draws (A is not drawn: the first update overwrites it)
    ref_init = [torch.zeros(d * R, device="cuda") for d in dims]
    cd.cp_init_curand(dims, R, ref_init, seed=1234)
    init = [u.cpu().numpy() for u in ref_init]
    lib = cd.library()
    f = getattr(lib, "_Z13cp_tensorcorePfS_S_S_llll")
    f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_long] * 4
    f.restype = None
    capfd.readouterr()
    f(dX.data_ptr(), *[u.data_ptr() for u in U], *dims, R)
    torch.cuda.synchronize()
    printed = float(capfd.readouterr().out.strip().splitlines()[-1])
    got = [u.cpu().numpy() for u in U]
    fit_ours = oracle.cp_fit(X, dims, got, R)
    _, fits, _ = oracle.cp_als(X, dims, R, init, 500)
    assert abs(fit_ours - fits[-1]) <= 2e-3, (fit_ours, fits[-1])
    assert abs((1.0 - printed) - fit_ours) <= 1e-5, (printed, fit_ours)
