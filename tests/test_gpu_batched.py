"""Batched CP-ALS (one persistent kernel per sweep over many small tensors of
uneven shape and rank): every tensor's fit must match running it through the
plain single-tensor path from the same start within 1e-4, and the oracle's
restatement of src/cp_als.cu on a few of them."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def make_batch(cd, n, seed, dlo=16, dhi=40, rlo=2, rhi=8):
    rng = np.random.default_rng(seed)
    dims = [tuple(int(x) for x in rng.integers(dlo, dhi + 1, 3)) for _ in range(n)]
    ranks = [int(x) for x in rng.integers(rlo, rhi + 1, n)]
    b = cd.Batch(dims, ranks)
    inits = []
    for t, (d, r) in enumerate(zip(dims, ranks)):
        true = [rng.random(x * r) for x in d]
        X = oracle.gencp(d, true, r)
        X = X + 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)
        b.x_view(t).copy_(torch.from_numpy(X.astype(np.float32)))
        init = [rng.random(x * r).astype(np.float32) for x in d]
        for m in range(3):
            b.u_view(t, m).copy_(torch.from_numpy(init[m]))
        inits.append(init)
    return b, inits


def test_batched_matches_plain_path(cd):
    b, inits = make_batch(cd, 40, seed=1)
    fits, sweeps, launches = cd.cp_als_batched(b, max_sweeps=25, tol=0.0)
    assert all(s == 25 for s in sweeps)
    assert launches >= 25
    for t in range(b.n):
        d, r = b.dims[t], b.ranks[t]
        U = [torch.from_numpy(f).cuda() for f in inits[t]]
        res = cd.cp_als(b.x_view(t).clone(), d, r, U, max_sweeps=25, precision=cd.PREC_FP32)
        assert abs(fits[t] - res.fit) <= 1e-4, (t, fits[t], res.fit)


def test_batched_matches_oracle(cd):
    b, inits = make_batch(cd, 6, seed=2)
    fits, _, _ = cd.cp_als_batched(b, max_sweeps=20, tol=0.0)
    for t in range(b.n):
        X = b.x_view(t).cpu().numpy()
        facs, fo, _ = oracle.cp_als(X, b.dims[t], b.ranks[t], inits[t], 20)
        assert abs(fits[t] - fo[-1]) <= 1e-4
        for m in range(3):
            got = b.u_view(t, m).cpu().numpy().astype(np.float64)
            assert np.linalg.norm(got - facs[m]) <= 1e-3 * np.linalg.norm(facs[m])


def test_batched_per_tensor_convergence_and_ragged_shapes(cd):
    dims = [(16, 16, 16), (96, 17, 31), (1, 40, 23), (33, 1, 9), (96, 96, 96), (20, 30, 1)]
    ranks = [4, 16, 3, 2, 8, 5]
    b = cd.Batch(dims, ranks)
    rng = np.random.default_rng(3)
    for t, (d, r) in enumerate(zip(dims, ranks)):
        b.x_view(t).copy_(torch.from_numpy(rng.random(int(np.prod(d))).astype(np.float32)))
        for m in range(3):
            b.u_view(t, m).copy_(torch.from_numpy(rng.random(d[m] * r).astype(np.float32)))
    Ucopy = b.U.clone()
    fits, sweeps, _ = cd.cp_als_batched(b, max_sweeps=60, tol=1e-5)
    assert all(1 <= s <= 60 for s in sweeps)
    assert all(np.isfinite(f) for f in fits)
    assert torch.isfinite(b.U).all()
    # deterministic: the same start gives bit-identical factors
    U1 = b.U.clone()
    b.U.copy_(Ucopy)
    fits2, sweeps2, _ = cd.cp_als_batched(b, max_sweeps=60, tol=1e-5)
    assert fits2 == fits and sweeps2 == sweeps
    assert torch.equal(U1, b.U)


def test_autotuner_picks_a_candidate(cd):
    b, _ = make_batch(cd, 64, seed=4)
    th, cps = cd.cp_batched_tune(b)
    assert th in (128, 192, 256, 384) and 1 <= cps <= 4
    fits, sweeps, _ = cd.cp_als_batched(b, max_sweeps=5, tol=0.0)
    assert all(np.isfinite(f) for f in fits)
