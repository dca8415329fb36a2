"""Parity at the benchmark configurations' own sizes, against FP64 on the host.

* MTTKRP at 512x512x512 rank 64 and 96x96x96x96 rank 32 (FP32 CUDA cores
  and the BF16x3 tensor cores): sampled output rows of every mode against
  an FP64 contraction of the same rows, relative Frobenius <= 1e-5.
* CP-ALS at 128x128x128 rank 16 (seeded rank-16 tensor + 1e-3 noise, seeded
  uniform start, 50 sweeps or delta-fit < 1e-6): final fit within 1e-4 of
  the FP64 oracle's CP-ALS of src/cp_als.cu:44-119 from the same start.
* Tucker at 512x512x512 multilinear rank (32,32,32) and 128^4 rank 16^4, in
  FP32, BF16x3 and BF16:
  HOSVD factors against the leading eigenvectors (numpy eigh) of the FP64
  unfolding Grams, as the largest principal angle; the reconstruction error
  against that of the FP64 HOSVD; 10 HOOI sweeps checked as a fixed point
  (each factor spans the leading eigenvectors of the FP64 Gram of X
  projected by the other returned factors) and never worse than HOSVD.

The inputs are generated on the device by the library's seeded generators
(make_cp_tensor, make_tucker_tensor); every checker value is FP64 on the
host.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def logical(Xflat, dims):
    """View of a flat column-major tensor with index order reversed:
    T[i_{N-1}, ..., i_0] = X(i_0, ..., i_{N-1})."""
    return Xflat.view(*reversed(dims))


def fp64_rows(T, facs, dims, mode, rows, R):
    """FP64 MTTKRP rows: M[q, r] = sum over the other indices of
    X(.., q, ..) * prod_{m != mode} U_m(i_m, r), for q in rows."""
    N = len(dims)
    axis = N - 1 - mode                      # position of `mode` in T
    letters = "abcdefgh"[:N]
    others = [m for m in range(N) if m != mode]
    # T's axes are modes N-1 .. 0; drop the `mode` axis for a row slice
    sl_axes = [letters[N - 1 - m] for m in range(N - 1, -1, -1) if m != mode]
    spec = "".join(sl_axes) + "," + ",".join(letters[N - 1 - m] + "z" for m in others) + "->z"
    mats = [facs[m].reshape(dims[m], R, order="F") for m in others]
    out = np.zeros((len(rows), R))
    for i, q in enumerate(rows):
        S = T.select(axis, int(q)).double().cpu().numpy()
        out[i] = np.einsum(spec, S, *mats, optimize="greedy")
    return out


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
@pytest.mark.parametrize("dims,R", [((512, 512, 512), 64), ((96, 96, 96, 96), 32)])
def test_mttkrp_full_size_sampled_rows(cd, prec, dims, R):
    X, _ = cd.make_cp_tensor(dims, R, seed=3)
    U = cd.make_init(dims, R, seed=4)
    facs = [u.double().cpu().numpy() for u in U]
    T = logical(X, dims)
    rng = np.random.default_rng(7)
    for mode in range(len(dims)):
        out = torch.empty(dims[mode] * R, device="cuda")
        cd.mttkrp(X, dims, U, mode, R, out, cd.PRECISIONS[prec])
        torch.cuda.synchronize()
        got = out.double().cpu().numpy().reshape(dims[mode], R, order="F")
        rows = np.unique(np.concatenate([[0, dims[mode] - 1], rng.integers(0, dims[mode], 14)]))
        want = fp64_rows(T, facs, dims, mode, rows, R)
        err = rel(got[rows], want)
        assert err <= 1e-5, (mode, err)
        assert np.isfinite(got).all()


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
def test_cp_als_128_r16_fit_vs_fp64_oracle(cd, prec):
    dims, R = (128, 128, 128), 16
    X, _ = cd.make_cp_tensor(dims, R, seed=0)
    U = cd.make_init(dims, R, seed=1)
    init = [u.cpu().numpy() for u in U]
    Xh = X.cpu().numpy()
    _, fits, sweeps = oracle.cp_als(Xh, dims, R, init, 50, tol=1e-6)
    res = cd.cp_als(X, dims, R, U, max_sweeps=50, tol=1e-6, precision=cd.PRECISIONS[prec])
    assert abs(res.fit - fits[-1]) <= 1e-4, (res.fit, fits[-1], res.sweeps, sweeps)
    # the returned factors' own fit, in FP64 on the host, is the reported one
    got = [u.cpu().numpy() for u in U]
    assert abs(oracle.cp_fit(Xh, dims, got, R) - res.fit) <= 1e-5


def _host_tensor(X, dims):
    return X.double().cpu().numpy()


def _unfold(Xd, dims, n):
    """Mode-n unfolding (dims[n] x rest) of the flat column-major FP64 X."""
    T = Xd.reshape(tuple(reversed(dims)))
    return np.moveaxis(T, len(dims) - 1 - n, 0).reshape(dims[n], -1)


def _max_angle(U, W):
    """Largest principal angle between span(U) and span(W) (W orthonormal)."""
    Q, _ = np.linalg.qr(U)
    s = np.linalg.norm(Q - W @ (W.T @ Q), 2)
    return float(np.arcsin(min(1.0, s)))


def _project_all_but(Xd, dims, facs, skip):
    """X x_m U_m^T for every m != skip (FP64, BLAS), returns tensor with
    axis order reversed (T[i_{N-1}, ..., i_0])."""
    T = Xd.reshape(tuple(reversed(dims)))
    N = len(dims)
    for m in range(N):
        if m == skip:
            continue
        ax = N - 1 - m
        T = np.moveaxis(np.tensordot(T, facs[m], axes=([ax], [0])), -1, ax)
    return T


def _recon_error(Xd, dims, facs):
    """||X - X x_m U_m U_m^T (all m)|| / ||X|| for orthonormal U_m."""
    C = _project_all_but(Xd, dims, facs, skip=-1)
    N = len(dims)
    for m in range(N):
        ax = N - 1 - m
        C = np.moveaxis(np.tensordot(C, facs[m].T, axes=([ax], [0])), -1, ax)
    return float(np.linalg.norm(Xd - C.reshape(-1)) / np.linalg.norm(Xd))


# FP32 and BF16x3 (three-term Grams and TTM steps) at FP32-level bars; BF16
# (single-term Grams and TTM chains, 8-bit mantissas) at the BF16 bars.
@pytest.mark.parametrize("prec,angle_bar,err_tol", [("fp32", 1e-4, 1e-6), ("bf16x3", 1e-4, 1e-6),
                                                    ("bf16", 2e-2, 2e-4)])
@pytest.mark.parametrize("dims,ranks", [((512, 512, 512), (32, 32, 32)), ((128, 128, 128, 128), (16, 16, 16, 16))])
def test_tucker_full_size_vs_fp64(cd, prec, angle_bar, err_tol, dims, ranks):
    X, _, _ = cd.make_tucker_tensor(dims, ranks, seed=20)
    Xd = _host_tensor(X, dims)
    N = len(dims)
    W = []
    for n in range(N):
        A = _unfold(Xd, dims, n)
        G = A @ A.T
        W.append(np.linalg.eigh(G)[1][:, dims[n] - ranks[n]:])
    e64 = _recon_error(Xd, dims, W)

    core = torch.empty(int(np.prod(ranks)), device="cuda")
    U = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
    cd.tucker_hosvd(X, dims, ranks, core, U, precision=cd.PRECISIONS[prec])
    torch.cuda.synchronize()
    Uh = [u.double().cpu().numpy().reshape(d, r, order="F") for u, d, r in zip(U, dims, ranks)]
    angles = [_max_angle(Uh[n], W[n]) for n in range(N)]
    assert max(angles) <= angle_bar, angles
    e_hosvd = _recon_error(Xd, dims, Uh)
    assert abs(e_hosvd - e64) <= err_tol, (e_hosvd, e64)

    cd.tucker_hooi(X, dims, ranks, core, U, sweeps=10, precision=cd.PRECISIONS[prec])
    torch.cuda.synchronize()
    Uh = [u.double().cpu().numpy().reshape(d, r, order="F") for u, d, r in zip(U, dims, ranks)]
    for n in range(N):
        Y = _project_all_but(Xd, dims, Uh, skip=n)
        A = np.moveaxis(Y, N - 1 - n, 0).reshape(dims[n], -1)
        Wn = np.linalg.eigh(A @ A.T)[1][:, dims[n] - ranks[n]:]
        a = _max_angle(Uh[n], Wn)
        assert a <= angle_bar, (n, a)
    e_hooi = _recon_error(Xd, dims, Uh)
    assert e_hooi <= e_hosvd + err_tol, (e_hooi, e_hosvd)
