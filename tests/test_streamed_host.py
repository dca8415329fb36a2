"""Host logic of the out-of-core CP-ALS: the slab partition of the last mode."""
import pytest

import streamed


def test_slab_ranges_cover_the_mode_once():
    for extent in (1, 7, 30, 64, 513):
        for slab in (1, 3, 7, 64, 1000):
            r = streamed.slab_ranges(extent, slab)
            assert r[0][0] == 0 and r[-1][1] == extent
            assert all(b0 == a1 for (_, a1), (b0, _) in zip(r, r[1:]))
            assert all(0 < k1 - k0 <= slab for k0, k1 in r)


def test_slab_ranges_rejects_empty_slab():
    with pytest.raises(ValueError):
        streamed.slab_ranges(10, 0)


def test_slab_decomposition_of_hosvd_pieces():
    """The identities the out-of-core HOSVD rests on, in FP64 on the host:
    slab Grams sum to the leading modes' Grams, slab-pair blocks assemble the
    last mode's Gram, and the slab projections sum to the core."""
    import numpy as np

    import oracle

    rng = np.random.default_rng(4)
    dims, ranks, slab = (7, 6, 11), (3, 2, 4), 4
    X = rng.standard_normal(int(np.prod(dims))).astype(np.float32)
    P = dims[0] * dims[1]
    r = streamed.slab_ranges(dims[-1], slab)
    slabs = [X[k0 * P:k1 * P] for k0, k1 in r]
    for n in range(2):
        G = sum(oracle.unfold_gram(Xs, (dims[0], dims[1], k1 - k0), n) for Xs, (k0, k1) in zip(slabs, r))
        np.testing.assert_allclose(G, oracle.unfold_gram(X, dims, n), rtol=1e-12, atol=1e-12)
    Glast = np.zeros((dims[-1], dims[-1]))
    for (k0, k1), A in zip(r, slabs):
        for (t0, t1), B in zip(r, slabs):
            Am = A.astype(np.float64).reshape(k1 - k0, P).T
            Bm = B.astype(np.float64).reshape(t1 - t0, P).T
            Glast[k0:k1, t0:t1] = Am.T @ Bm
    np.testing.assert_allclose(Glast, oracle.unfold_gram(X, dims, 2), rtol=1e-12, atol=1e-12)
    facs = [np.linalg.qr(rng.standard_normal((d, q)))[0] for d, q in zip(dims, ranks)]
    W = [np.asfortranarray(f.T).reshape(-1, order="F") for f in facs]
    full, _ = oracle.mode_product(X, dims, 0, W[0], ranks[0])
    full, cur = oracle.mode_product(full, [ranks[0], dims[1], dims[2]], 1, W[1], ranks[1])
    full, _ = oracle.mode_product(full, cur, 2, W[2], ranks[2])
    core = np.zeros(int(np.prod(ranks)))
    for (k0, k1), Xs in zip(r, slabs):
        Y, c = oracle.mode_product(Xs, (dims[0], dims[1], k1 - k0), 0, W[0], ranks[0])
        Y, c = oracle.mode_product(Y, c, 1, W[1], ranks[1])
        Wl = np.asfortranarray(facs[2][k0:k1].T).reshape(-1, order="F")
        Y, _ = oracle.mode_product(Y, c, 2, Wl, ranks[2])
        core += Y
    np.testing.assert_allclose(core, full, rtol=1e-10, atol=1e-12)
