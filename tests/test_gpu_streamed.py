"""Out-of-core CP-ALS (streamed.py, after decomposition/GPU/large/
slice_cp_als.cu): the tensor stays in pinned host memory and every mode's
MTTKRP streams it slab by slab.  The result must match the same sweep run
on the device-resident tensor (one slab holding everything), up to the
order in which the slab partials are summed."""
import numpy as np
import pytest
import torch

import distributed
import streamed

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("precision,slab,nbuf", [("fp32", 7, 2), ("fp32", 4, 3), ("bf16x3", 9, 2)])
def test_streamed_matches_in_core(cd, precision, slab, nbuf):
    dims, R, sweeps = (40, 36, 30), 6, 3
    prec = cd.PRECISIONS[precision]
    X, _ = cd.make_cp_tensor(dims, R, seed=3)
    init = cd.make_init(dims, R, seed=4)
    ref = distributed.ShardedCP(distributed.CudaOps(cd, prec), streamed.LocalComm(), X, list(dims), R,
                                [u.clone() for u in init])
    for _ in range(sweeps):
        ref.sweep()
    fit_ref = ref.fit()
    Xh = X.cpu().pin_memory()
    sc = streamed.StreamedCP(cd, Xh, dims, R, [u.clone() for u in init], slab=slab, precision=prec, nbuf=nbuf)
    for _ in range(sweeps):
        sc.sweep()
    fit = sc.fit()
    torch.cuda.synchronize()
    for m in range(3):
        assert rel(sc.U[m], ref.U[m]) <= 1e-4, m
    assert abs(fit - fit_ref) <= 1e-6
    assert fit > 0.9
    # the whole tensor crossed the host link once for the norm and once per mode per sweep
    assert sc.h2d_bytes == 4 * int(np.prod(dims)) * (1 + 3 * sweeps)


def test_streamed_order4_last_mode_rows(cd):
    dims, R = (12, 10, 8, 11), 4
    X, _ = cd.make_cp_tensor(dims, R, seed=5)
    init = cd.make_init(dims, R, seed=6)
    ref = distributed.ShardedCP(distributed.CudaOps(cd, cd.PREC_FP32), streamed.LocalComm(), X, list(dims), R,
                                [u.clone() for u in init])
    sc = streamed.StreamedCP(cd, X.cpu().pin_memory(), dims, R, [u.clone() for u in init], slab=3,
                             precision=cd.PREC_FP32)
    for _ in range(2):
        ref.sweep()
        sc.sweep()
    torch.cuda.synchronize()
    for m in range(4):
        assert rel(sc.U[m], ref.U[m]) <= 1e-4, m


def _gap(u, w, d, r):
    U = u.cpu().numpy().reshape(d, r, order="F").astype(np.float64)
    W = w.cpu().numpy().reshape(d, r, order="F").astype(np.float64)
    return np.linalg.norm(U @ U.T - W @ W.T)


@pytest.mark.parametrize("dims,ranks,slab", [((24, 20, 30), (4, 3, 5), 7), ((10, 9, 8, 11), (3, 2, 2, 3), 4)])
def test_streamed_hosvd_matches_in_core(cd, dims, ranks, slab):
    """Out-of-core HOSVD (decomposition/GPU/large/slice_tucker_hosvd.cu)
    against the device-resident FP32 HOSVD: same factor subspaces and core."""
    X, _, _ = cd.make_tucker_tensor(dims, ranks, seed=9)
    n = int(np.prod(ranks))
    core = torch.empty(n, device="cuda")
    U = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
    cd.tucker_hosvd(X, dims, ranks, core, U, precision=cd.PREC_FP32)
    st = streamed.StreamedTucker(cd, X.cpu().pin_memory(), dims, slab)
    core2 = torch.empty(n, device="cuda")
    U2 = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
    assert st.hosvd(ranks, core2, U2) == cd.OK
    torch.cuda.synchronize()
    for u, w, d, r in zip(U2, U, dims, ranks):
        assert _gap(u, w, d, r) <= 1e-5
    rec = torch.empty(X.numel(), device="cuda")
    rec2 = torch.empty(X.numel(), device="cuda")
    cd.gentucker(rec, core, U, dims, ranks)
    cd.gentucker(rec2, core2, U2, dims, ranks)
    torch.cuda.synchronize()
    assert rel(rec2, rec) <= 1e-5
    # host traffic: the tensor for the leading Grams and for the core, and
    # each slab s held once plus the later slabs streamed past it
    P = int(np.prod(dims[:-1]))
    r = streamed.slab_ranges(dims[-1], slab)
    pairs = sum((k1 - k0) + sum(t1 - t0 for t0, t1 in r[s + 1:]) for s, (k0, k1) in enumerate(r[:-1]))
    assert st.h2d_bytes == 4 * P * (2 * dims[-1] + pairs)
