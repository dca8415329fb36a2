"""Pins the CPU oracle against the golden vectors (no GPU).

The golden vectors come from the reference's own driver fixtures
(test/test_mttkrp.cpp, test/test_gen.cpp, test/test_t2m.cpp, test/test_kr.cpp,
test/test_hadmard.cpp, test/test_tensor_product.cpp, test/test_ttm.cpp and the
hand tensors of decomposition/GPU/normal/{cp,tucker}/de_*.cpp) with answers
computed exactly by tests/golden/make_golden.py.
"""
import numpy as np
import pytest

import oracle


def test_fixture_generators_restate_the_drivers(golden):
    X, A, B, C = oracle.rand_int_fixture(2, [27, 6, 6, 6])
    for got, key in ((X, "mt_X"), (A, "mt_A"), (B, "mt_B"), (C, "mt_C")):
        np.testing.assert_array_equal(got, golden[key])
    (T,) = oracle.rand_frac_fixture(2, [24])
    np.testing.assert_array_equal(T, golden["t2m_T"])
    tX, U1 = oracle.rand_frac_fixture(2, [27, 6], shift=-0.5)
    np.testing.assert_array_equal(tX, golden["ttm_X"])
    np.testing.assert_array_equal(U1, golden["ttm_U1"])
    kA, kB = oracle.rand_frac_fixture(None, [6, 6])
    np.testing.assert_array_equal(kA, golden["kr_A"])
    np.testing.assert_array_equal(kB, golden["kr_B"])


def test_elementwise_bit_exact(golden):
    np.testing.assert_array_equal(oracle.hadmard(golden["hd_A"], golden["hd_B"]), golden["hd_C"])
    np.testing.assert_array_equal(oracle.kr(golden["kr_A"], golden["kr_B"], 3, 3, 2), golden["kr_out"])
    np.testing.assert_array_equal(oracle.tensor_product(golden["tp_A"], golden["tp_B"], 2, 2, 3, 3),
                                  golden["tp_C"])


@pytest.mark.parametrize("flag", [1, 2, 3])
def test_t2m_bit_exact(golden, flag):
    np.testing.assert_array_equal(oracle.t2m(golden["t2m_T"], flag, 4, 3, 2), golden[f"t2m_{flag}"])


def test_t2m_bad_flag_is_rejected(golden):
    assert oracle.t2m(golden["t2m_T"], 4, 4, 3, 2) is None


def test_mttkrp_reference_fixture_exact(golden):
    X, A, B, C = (golden[k] for k in ("mt_X", "mt_A", "mt_B", "mt_C"))
    # the three calls of test/test_mttkrp.cpp:60-62, public FP16 semantics
    np.testing.assert_array_equal(oracle.mttkrp_legacy(X, C, B, 1, 3, 3, 3, 2), golden["mt_out1"])
    np.testing.assert_array_equal(oracle.mttkrp_legacy(X, C, A, 2, 3, 3, 3, 2), golden["mt_out2"])
    np.testing.assert_array_equal(oracle.mttkrp_legacy(X, B, A, 3, 3, 3, 3, 2), golden["mt_out3"])
    # general FP64 MTTKRP
    for mode, key in ((0, "mt_out1"), (1, "mt_out2"), (2, "mt_out3")):
        facs = [A, B, C]
        np.testing.assert_array_equal(oracle.mttkrp(X, (3, 3, 3), facs, mode, 2), golden[key])


@pytest.mark.parametrize("prefix,order", [("mt2", 3), ("mt4", 4)])
def test_mttkrp_integer_fixtures_exact(golden, prefix, order):
    X = golden[f"{prefix}_X"]
    dims = tuple(int(d) for d in golden[f"{prefix}_dims"])
    R = int(golden[f"{prefix}_R"])
    facs = [golden[f"{prefix}_U{i}"] for i in range(order)]
    for mode in range(order):
        np.testing.assert_array_equal(oracle.mttkrp(X, dims, facs, mode, R), golden[f"{prefix}_out{mode}"])


def test_gencp_gentucker_exact(golden):
    A, B, C, core = (golden[k] for k in ("gen_A", "gen_B", "gen_C", "gen_core"))
    np.testing.assert_array_equal(oracle.gencp((2, 2, 2), [A, B, C], 2), golden["gen_cp"])
    np.testing.assert_array_equal(oracle.gentucker(core, (2, 2, 2), [A, B, C], (2, 2, 2)),
                                  golden["gen_tucker"])
    np.testing.assert_array_equal(
        oracle.gentucker(golden["ht_G"], (2, 2, 2), [golden["ht_A"], golden["ht_B"], golden["ht_C"]],
                         (3, 4, 2)), golden["ht_rec"])


def test_rse(golden):
    X = golden["gen_X"]
    rec = golden["gen_tucker"].astype(np.float32)
    diff, err = oracle.rse(X, rec)
    np.testing.assert_array_equal(diff, (X - rec).astype(np.float32))
    want = np.linalg.norm((X - rec).astype(np.float64)) / np.linalg.norm(X.astype(np.float64))
    assert abs(err - want) <= 1e-6 * want


@pytest.mark.parametrize("flag", [1, 2, 3])
def test_ttm(golden, flag):
    U = golden[f"ttm_U{flag}"]
    got = oracle.ttm(golden["ttm_X"], U, flag, 3, 3, 3, 2)
    np.testing.assert_allclose(got, golden[f"ttm_out{flag}"], rtol=1e-12, atol=1e-12)


def test_cp_first_update_exact(golden):
    """First A update of src/cp_als.cu:46-63 on the hand tensor of
    decomposition/GPU/normal/cp/de_cp.cpp:11-19."""
    X, B, C = golden["hc_X"], golden["hc_B"], golden["hc_C"]
    for use_lu in (True, False):
        facs, fits, sweeps = oracle.cp_als(X, (3, 2, 2), 2, [np.zeros(6), B, C], 1, use_lu=use_lu)
        np.testing.assert_allclose(facs[0], golden["hc_A1"], rtol=1e-12, atol=1e-12)
        assert sweeps == 1


def test_cp_als_converges_on_exact_low_rank():
    rng = np.random.default_rng(0)
    dims, R = (9, 8, 7), 3
    true = [rng.random(d * R) for d in dims]
    X = oracle.gencp(dims, true, R).astype(np.float32)
    init = [rng.random(d * R) for d in dims]
    facs, fits, sweeps = oracle.cp_als(X, dims, R, init, 200, tol=1e-10)
    assert fits[-1] > 0.999
    assert abs(oracle.cp_fit(X, dims, facs, R) - fits[-1]) < 1e-6


def test_hosvd_hooi_recover_exact_tucker(golden):
    rec = golden["ht_rec"].astype(np.float32)
    dims, ranks = (3, 4, 2), (2, 2, 2)
    core, facs = oracle.tucker_hosvd(rec, dims, ranks)
    back = oracle.gentucker(core, ranks, facs, dims)
    np.testing.assert_allclose(back, rec, atol=1e-9 * np.abs(rec).max())
    core2, facs2 = oracle.tucker_hooi(rec, dims, ranks, sweeps=2)
    back2 = oracle.gentucker(core2, ranks, facs2, dims)
    np.testing.assert_allclose(back2, rec, atol=1e-9 * np.abs(rec).max())


def test_numpy_baseline_matches_oracle_sweep():
    rng = np.random.default_rng(1)
    dims, R = (6, 5, 4), 3
    X = rng.random(int(np.prod(dims))).astype(np.float32)
    init = [rng.random(d * R) for d in dims]
    facs, _, _ = oracle.cp_als(X, dims, R, init, 1)
    X3 = X.reshape(dims, order="F").astype(np.float64)
    F = [f.reshape(d, R, order="F").copy() for f, d in zip(init, dims)]
    oracle.numpy_cp_als_sweep(X3, F)
    for f, g, d in zip(F, facs, dims):
        np.testing.assert_allclose(f.reshape(-1, order="F"), g, rtol=1e-9, atol=1e-12)


def test_cpu_baseline_als_matches_oracle():
    """The C++/OpenMP CPU baseline (oracle/cpu_als.cpp) computes the same ALS
    as the FP64 oracle: in FP64 the factors and fits agree to rounding, and
    its MTTKRP matches at orders 3 and 4."""
    rng = np.random.default_rng(12)
    for dims, R in (((20, 16, 12), 4), ((9, 8, 7, 6), 3)):
        X = oracle.gencp(dims, [rng.random(d * R) for d in dims], R) + 1e-3 * rng.standard_normal(int(np.prod(dims)))
        X = X.astype(np.float32).astype(np.float64)
        init = [rng.random(d * R).astype(np.float32).astype(np.float64) for d in dims]
        for mode in range(len(dims)):
            got = oracle.cpu_mttkrp(X, dims, init, mode, R, threads=3)
            want = oracle.mttkrp(X, dims, init, mode, R)
            assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
        facs, fits, sweeps, _ = oracle.cpu_cp_als(X, dims, R, init, 8, threads=3)
        wfacs, wfits, wsweeps = oracle.cp_als(X, dims, R, init, 8)
        assert sweeps == wsweeps == 8
        assert np.abs(fits - wfits).max() <= 1e-9
        for f, w in zip(facs, wfacs):
            assert np.abs(f - w).max() <= 1e-7 * np.abs(w).max()
        # FP32 arithmetic stays close to FP64
        f32, fits32, _, _ = oracle.cpu_cp_als(X.astype(np.float32), dims, R, [i.astype(np.float32) for i in init], 8,
                                              threads=3)
        assert abs(fits32[-1] - wfits[-1]) <= 1e-4
