"""Index arithmetic of the sm_100a kernels, restated on the CPU: every access
stays inside its buffer and every output element has exactly one writer.
The restatements follow the kernels line by line (the constants are the
kernels' own); a change there that breaks a property shows up here before
the code reaches a GPU."""
import numpy as np
import pytest


# ---- tucker_tc.cu k_unfold_t64: 64 x 64 tiles, float4 reads, 8-wide BF16 writes
def unfold_t64_accesses(Q, S):
    writes = np.zeros(Q * S, np.int32)
    tq, ts = -(-Q // 64), -(-S // 64)
    t = np.arange(256)
    reads_max, smem_max = -1, -1
    for tt in range(tq * ts):
        q0, s0 = (tt % tq) * 64, (tt // tq) * 64
        q4 = (t & 15) * 4
        for i in range(4):
            sl = (t >> 4) + 16 * i
            ok = (q0 + q4 < Q) & (s0 + sl < S)
            if ok.any():
                reads_max = max(reads_max, int((q0 + q4 + 3 + Q * (s0 + sl))[ok].max()))
            smem_max = max(smem_max, int((sl * 68 + q4 + 3).max()))
        for i in range(2):
            u = t + 256 * i
            p = u >> 1
            ql, c = p & 63, 2 * (p >> 6) + (u & 1)
            q, sb = q0 + ql, s0 + 8 * c
            ok = (q < Q) & (sb < S)
            for j in range(8):
                smem_max = max(smem_max, int(((8 * c + j) * 68 + ql).max()))
                np.add.at(writes, (q * S + sb + j)[ok], 1)
    return writes, reads_max, smem_max


@pytest.mark.parametrize("Q,S", [(4, 8), (64, 64), (68, 72), (132, 520), (512, 136), (4, 4096)])
def test_unfold_t64_covers_each_output_once_in_bounds(Q, S):
    writes, rmax, smax = unfold_t64_accesses(Q, S)
    assert np.all(writes == 1)
    assert rmax < Q * S          # float4 reads: Q % 4 == 0 keeps a vector inside
    assert smax < 64 * 68        # tile[64][68]


# ---- subspace.cu cluster layout: 8 CTAs own row blocks of the iterate
CL_N, CL_T, CL_RS = 8, 256, 33


def cl_layout_total(n):
    nl = -(-n // CL_N)
    blk = nl * CL_RS
    return nl, 2 * blk + 2 * 32 * 32 + CL_T * 16 + 2 * 32 * CL_RS


@pytest.mark.parametrize("n", [1, 7, 8, 20, 100, 512, 1000, 2047, 2048])
def test_cluster_rows_partition_and_fit(n):
    nl, total = cl_layout_total(n)
    owned = np.zeros(n, np.int32)
    for rank in range(CL_N):
        i0 = rank * nl
        cnt = max(0, min(nl, n - i0))
        owned[i0:i0 + cnt] += 1
    assert np.all(owned == 1)
    assert 8 * total <= 200 * 1024            # the dynamic shared-memory opt-in
    # the 4 x 4 tile partials: ntiles * groups <= CL_T slots of 16 doubles
    for r in range(1, 33):
        nt = -(-r // 4)
        for sym in (True, False):
            ntiles = nt * (nt + 1) // 2 if sym else nt * nt
            ng = min(8, CL_T // ntiles)
            assert ntiles * ng <= CL_T and 4 * nt <= 32


# ---- batched.cu mttkrp_lanes: lanes along i, warps split the outer index,
# recursive-halving lane sums, partials combined in a fixed order
BMAXD, BMAXR, RS = 96, 16, 16


def lane_sum_restated(v):
    """lane_sum<RP>: v is 32 lanes x RP values; returns the per-lane result
    and checks lane l holds the total of rank l >> (5 - L)."""
    RP = v.shape[1]
    L = {16: 4, 8: 3, 4: 2}[RP]
    v = v.copy()
    lanes = np.arange(32)
    for l in range(L):
        off, n = 16 >> l, RP >> (l + 1)
        up = (lanes & off) != 0
        send = np.where(up[:, None], v[:, :n], v[:, n:2 * n])
        keep = np.where(up[:, None], v[:, n:2 * n], v[:, :n])
        v = keep + send[lanes ^ off]
    s = v[:, 0].copy()
    off = 16 >> L
    while off >= 1:
        s = s + s[lanes ^ off]
        off >>= 1
    return s, lanes >> (5 - L)


@pytest.mark.parametrize("RP", [4, 8, 16])
def test_lane_sum_totals_each_rank(RP):
    rng = np.random.default_rng(RP)
    v = rng.integers(-50, 50, (32, RP)).astype(np.float64)
    s, rank = lane_sum_restated(v)
    np.testing.assert_array_equal(s, v.sum(0)[rank])


def batched_mttkrp_restated(X, dims, F, mode, R, NW):
    """mttkrp_lanes<NW, RP> on the CPU: returns M (Q x R) and checks every
    load in bounds, every output row written by one warp group."""
    I, J, K = dims
    RP = 4 if R <= 4 else 8 if R <= 8 else 16
    Fp = [np.zeros((BMAXD, RS)) for _ in range(3)]
    for m in range(3):
        Fp[m][:dims[m], :R] = F[m]
    LI = -(-I // 32)
    NG = NW // LI
    O = J if mode == 1 else K
    Nn = K if mode == 1 else J
    so, sn = (I, I * J) if mode == 1 else (I * J, I)
    Vf = Fp[2] if mode == 1 else Fp[1]
    Q = dims[mode]
    Mp = np.full((NW, BMAXD * RS), np.nan)
    lanes = np.arange(32)
    written = np.zeros(O, int)
    for warp in range(NW):
        ic, g = warp % LI, warp // LI
        i = ic * 32 + lanes
        valid = i < I
        o0 = O * g // NG if g < NG else O
        o1 = O * (g + 1) // NG if g < NG else O
        acc = np.zeros((32, RP))
        for o in range(o0, o1, 2):
            two = o + 1 < o1
            t = [np.zeros((32, RP)), np.zeros((32, RP))]
            for k, oo in enumerate((o, o + 1 if two else o)):
                ok = valid & (two or k == 0)
                for n in range(Nn):
                    addr = np.where(valid, i, 0) + so * oo + sn * n
                    assert (addr[ok] < X.size).all()
                    x = np.where(ok, X[np.where(ok, addr, 0)], 0.0)
                    assert n < BMAXD
                    t[k] += x[:, None] * Vf[n, :RP][None, :]
            if mode == 0:
                acc += t[0] * Fp[2][o, :RP] + t[1] * Fp[2][o + 1 if two else o, :RP]
            else:
                a = Fp[0][np.where(valid, i, 0), :RP]
                for k, oo in enumerate((o, o + 1)):
                    if k == 1 and not two:
                        break
                    s, rank = lane_sum_restated(t[k] * a)
                    SH = {16: 1, 8: 2, 4: 3}[RP]
                    w = (lanes & ((1 << SH) - 1)) == 0
                    Mp[ic, oo * RS + rank[w]] = s[w]
                    if ic == 0:
                        written[oo] += 1
        if mode == 0 and g < NG:
            for l in np.nonzero(valid)[0]:
                Mp[g, i[l] * RS:i[l] * RS + RP] = acc[l]
    nparts = NG if mode == 0 else LI
    M = np.zeros((Q, R))
    for q in range(Q):
        for r in range(R):
            M[q, r] = sum(Mp[p, q * RS + r] for p in range(nparts))
    assert not np.isnan(M).any()
    if mode != 0:
        assert (written == 1).all()
    return M


@pytest.mark.parametrize("dims,R,NW", [((16, 20, 17), 4, 6), ((37, 16, 24), 7, 4), ((64, 19, 33), 12, 6),
                                       ((96, 50, 18), 16, 12), ((70, 33, 41), 5, 8), ((33, 96, 16), 9, 6)])
def test_batched_mttkrp_lanes_restated_matches_oracle(dims, R, NW):
    import oracle
    rng = np.random.default_rng(sum(dims) + R + NW)
    X = rng.random(int(np.prod(dims))).astype(np.float32).astype(np.float64)
    F = [rng.random((d, R)).astype(np.float32).astype(np.float64) for d in dims]
    for mode in range(3):
        M = batched_mttkrp_restated(X, dims, F, mode, R, NW)
        want = oracle.mttkrp(X, dims, [f.reshape(-1, order="F") for f in F], mode, R).reshape(dims[mode], R, order="F")
        assert np.abs(M - want).max() <= 1e-12 * np.abs(want).max()


def test_batched_shared_memory_fits():
    # BatchSmem: F[3], M, Mp[3] (floats, BMAXD x RS each; Mp holds the row
    # chunks' partials of modes 2 and 3, mode 1 adds its groups into M in
    # turn), V and the pivot rows (doubles); the CTAs per SM of every tuning
    # candidate fit in 228 KB (1 KB reserved per CTA), and their warps
    # within the launch bounds' budgets
    min_ctas = {4: 5, 6: 3, 8: 2, 12: 2}
    for threads, ctas in ((128, 4), (128, 5), (192, 3), (256, 2), (384, 2)):
        NW = threads // 32
        smem = 4 * BMAXD * RS * (4 + 3) + 8 * (BMAXR * BMAXR + 2 * BMAXR + 32) + 16
        assert ctas * (smem + 1024) <= 228 * 1024, (NW, ctas, smem)
        assert ctas <= min_ctas[NW] or NW * ctas <= 24
        # partial buffers: at most ceil(96 / 32) = 3 row chunks
        assert -(-BMAXD // 32) == 3


# ---- gemm_tc.cu skinny GEMM: B resident for K <= 1024 plus an 8-deep A ring
def test_skinny_gemm_shared_memory_fits():
    GBM, GBK, SK_BN, SK_ST = 128, 64, 32, 8
    kblocks = 1024 // GBK
    smem = 1024 + 1024 + kblocks * SK_BN * GBK * 2 + SK_ST * GBM * GBK * 2
    assert smem <= 232448


# ---- mttkrp_tc.cu pre-packed-B path: launch plan, stage split, segments, B pack
BQ, BKS, SEG, PB_RING, NSM = 128, 32, 16, 6, 148
X_STAGE, PB_CTRL = BQ * BKS * 4, 2048


def b_tile_bytes(rpad):
    return rpad * BKS * 2


def pb_plan(dims, mode, R):
    P = int(np.prod(dims[:mode])) if mode else 1
    Q = dims[mode]
    S = int(np.prod(dims[mode + 1:]))
    kind0 = mode == 0
    rpad = max(16, -(-R // 16) * 16)
    psteps = 1 if kind0 else -(-P // BKS)
    stages = -(-S // BKS) if kind0 else S * psteps
    qtiles = -(-Q // BQ)
    rows0 = dims[1] if kind0 else dims[0]
    # factors folded into the packed B (gen, then outer) while a block is
    # shorter than a segment and the packed tiles stay within 8 MiB
    fl = [d for m, d in enumerate(dims) if m != mode and (kind0 or m < mode)]
    fl += [] if kind0 else list(dims[mode + 1:])
    fold, frows = 1, rows0
    while frows // BKS < SEG and fold < len(fl) and frows * fl[fold] * rpad * 4 <= 8 << 20:
        frows *= fl[fold]
        fold += 1
    if rows0 % BKS or frows // BKS < 2:
        return None                                    # not the pre-packed path
    blk = frows // BKS
    smem = lambda n: 1024 + PB_CTRL + n * (X_STAGE + 2 * b_tile_bytes(rpad))
    cps = nring = 0
    for n in range(PB_RING, 2, -1):
        if smem(n) <= 115712 and 2 * rpad + 32 * n <= 256:
            cps, nring = 2, n
            break
    if not cps:
        for n in range(PB_RING, 2, -1):
            if smem(n) <= 232448 and 2 * rpad + 32 * n <= 512:
                cps, nring = 1, n
                break
    want = max(1, (cps * NSM - 2) // qtiles)
    splits = min(want, stages)
    chunk = -(-stages // splits)
    splits = -(-stages // chunk)
    return dict(stages=stages, qtiles=qtiles, blk=blk, rpad=rpad, rows0=rows0, cps=cps, nring=nring,
                splits=splits, chunk=chunk, smem=smem(nring), fold=fold, frows=frows, fl=fl, P=P, psteps=psteps)


def segments(beg, end, blk):
    pos, out, cur = beg % blk, [], 0
    for i in range(end - beg):
        cur += 1
        stop = pos == blk - 1 or (pos & (SEG - 1)) == SEG - 1 or i == end - beg - 1
        pos = 0 if pos + 1 == blk else pos + 1
        if stop:
            out.append((beg + i - cur + 1, cur))
            cur = 0
    return out


@pytest.mark.parametrize("dims,R", [((512, 512, 512), 64), ((384, 384, 384), 64), ((96, 96, 96, 96), 32),
                                    ((512, 512, 512), 16), ((256, 160, 96), 128)])
def test_mttkrp_pb_plan_partitions_stages(dims, R):
    for mode in range(len(dims)):
        p = pb_plan(dims, mode, R)
        assert p is not None
        assert p["cps"] in (1, 2) and p["nring"] >= 3
        assert p["smem"] <= (115712 if p["cps"] == 2 else 232448)
        assert p["qtiles"] * p["splits"] <= p["cps"] * NSM          # one wave
        assert (p["splits"] - 1) * p["chunk"] < p["stages"] <= p["splits"] * p["chunk"]
        blk = p["blk"]
        covered = 0
        for z in range(p["splits"]):
            beg, end = z * p["chunk"], min(p["stages"], (z + 1) * p["chunk"])
            for s0, n in segments(beg, end, blk):
                assert 1 <= n <= SEG
                assert s0 // blk == (s0 + n - 1) // blk           # never across a constant-row block
            covered += end - beg
        assert covered == p["stages"]


@pytest.mark.parametrize("dims,R", [((96, 96, 96, 96), 32), ((128, 64, 32), 8), ((64, 40, 36), 4),
                                    ((32, 96, 6, 5), 3), ((512, 512, 512), 64)])
def test_mttkrp_pb_fold_reproduces_khatri_rao(dims, R):
    """Stage g's B rows (packed row 32 (g mod blk) + i, the product of the
    folded factors) times its constant row (the other factors at the digits
    of 32 g / frows) equal the Khatri-Rao row of contraction position
    l = 32 g + i, digits over gen then outer."""
    rng = np.random.default_rng(sum(dims) + R)
    for mode in range(len(dims)):
        p = pb_plan(dims, mode, R)
        if p is None:
            continue
        kind0 = mode == 0
        facs = [m for m in range(len(dims)) if m != mode and (kind0 or m < mode)]
        facs += [] if kind0 else list(range(mode + 1, len(dims)))
        U = {m: rng.integers(1, 7, (dims[m], R)).astype(np.float64) for m in facs}
        fold, frows, blk = p["fold"], p["frows"], p["blk"]
        assert np.prod([dims[m] for m in facs[:fold]]) == frows
        packed = np.ones((frows, R))
        for rho in range(frows):
            lin = rho
            for m in facs[:fold]:
                packed[rho] *= U[m][lin % dims[m]]
                lin //= dims[m]
        total = int(np.prod([dims[m] for m in facs]))
        for g in rng.choice(p["stages"], min(40, p["stages"]), replace=False):
            lin = (32 * int(g)) // frows
            c = np.ones(R)
            for m in facs[fold:]:
                c *= U[m][lin % dims[m]]
                lin //= dims[m]
            pos = int(g) % blk
            for i in range(32):
                l = 32 * int(g) + i
                if l >= total:
                    continue
                want = np.ones(R)
                ll = l
                for m in facs:
                    want *= U[m][ll % dims[m]]
                    ll //= dims[m]
                np.testing.assert_array_equal(packed[32 * pos + i] * c, want)


@pytest.mark.parametrize("rows0,R", [(512, 64), (96, 32), (64, 128), (512, 5)])
def test_mttkrp_pack_b_in_bounds(rows0, R):
    rpad = max(16, -(-R // 16) * 16)
    blk = rows0 // BKS
    bbytes = b_tile_bytes(rpad)
    n = blk * 4 * rpad
    ids = np.arange(n)
    t = ids // (4 * rpad)
    rem = ids - t * 4 * rpad
    kc, r = rem // rpad, rem % rpad
    row_max = (32 * t + 8 * kc + 7)[r < R].max()
    assert row_max < rows0                                       # U0 rows read
    off = r * 16 + kc * rpad * 16
    assert (off + 16).max() <= bbytes                            # inside each hi / lo half
    assert ((t * 2 + 1) * bbytes + off + 16).max() <= blk * 2 * bbytes   # inside the packed buffer
    # each 16-byte chunk of every tile half written exactly once
    assert len(np.unique(t * bbytes * 2 + off)) == n


# ---- mttkrp_simt.cu k_mttkrp_ffma: the plain FP32 FFMA MTTKRP, restated on
# the CPU with the kernel's own tile arithmetic (float4 A loads, transposing
# swizzled stores, B = pre-packed U0 rows x the constant row, split partials)
FQ, FK, FT = 128, 32, 128


def _swz(q, k):
    return q ^ (k & 28)


def ffma_plan(dims, mode, R, sms=148):
    order = len(dims)
    P = int(np.prod(dims[:mode])) if mode else 1
    Q = dims[mode]
    S = int(np.prod(dims[mode + 1:])) if mode + 1 < order else 1
    kind = 0 if mode == 0 else 1
    rows0 = dims[1] if mode == 0 else dims[0]
    if rows0 % FK or (kind == 0 and Q % 4):
        return None
    BR = 32 if R <= 32 else 64
    rtiles = -(-R // BR)
    Rp = rtiles * BR
    qtiles = -(-Q // FQ)
    psteps = P // FK if kind else 0
    steps = S * psteps if kind else S // FK
    want = -(-(2 * sms) // (qtiles * rtiles))
    splits = max(1, min(want, steps))
    chunk = -(-steps // splits)
    splits = -(-steps // chunk)
    return dict(P=P, Q=Q, S=S, kind=kind, rows0=rows0, BR=BR, rtiles=rtiles, Rp=Rp, qtiles=qtiles,
                psteps=psteps, steps=steps, chunk=chunk, splits=splits)


def ffma_restated(X, dims, facs, mode, R, sms=148):
    """FP64 evaluation of the kernel's data movement; asserts every global
    and shared access in bounds and returns the summed result (Q x R)."""
    p = ffma_plan(dims, mode, R, sms)
    P, Q, kind, rows0, BR, Rp = p["P"], p["Q"], p["kind"], p["rows0"], p["BR"], p["Rp"]
    order = len(dims)
    gen = [m for m in range(order) if m != mode and (kind == 0 or m < mode)]
    outer = [m for m in range(order) if m != mode and kind == 1 and m > mode]
    U = [f.reshape(dims[m], R, order="F") for m, f in enumerate(facs)]
    U0p = np.zeros((rows0, Rp))
    U0p[:, :R] = U[gen[0]]
    part = np.zeros((p["splits"], R, Q))
    t = np.arange(FT)
    rv, kb, kstep = t % (BR // 4), t // (BR // 4), FT // (BR // 4)
    NB = BR * FK // 4 // FT
    blk_stages = rows0 // FK
    nX = X.size
    for bx in range(p["qtiles"] * p["splits"]):
        q0, z = (bx % p["qtiles"]) * FQ, bx // p["qtiles"]
        for by in range(p["rtiles"]):
            r0 = by * BR
            acc = np.zeros((FQ, BR))
            sbeg, send = z * p["chunk"], min(p["steps"], z * p["chunk"] + p["chunk"])
            for st in range(sbeg, send):
                As = np.full((FK, FQ), np.nan)
                Bs = np.full((FK, BR), np.nan)
                if kind == 0:
                    k0 = st * FK
                    i0 = k0 % rows0
                    blk, s = k0 // rows0, 0
                    for i in range(8):
                        e = t + FT * i
                        k, qv = e >> 5, e & 31
                        q = q0 + 4 * qv
                        ok = q < Q
                        addr = q + Q * (k0 + k)
                        assert (addr[ok] + 3 < nX).all() and (addr[ok] % 4 == 0).all()
                        for j in range(4):
                            col = _swz(4 * qv, k) + j
                            assert (col < FQ).all()
                            As[k, col] = np.where(ok, X[np.where(ok, addr + j, 0)], 0.0)
                else:
                    s = st // p["psteps"]
                    p0 = (st - s * p["psteps"]) * FK
                    i0 = p0 % rows0
                    blk = p0 // rows0
                    for i in range(8):
                        e = t + FT * i
                        pv, q = e & 7, e >> 3
                        ok = q0 + q < Q
                        addr = p0 + 4 * pv + P * (q0 + q + Q * s)
                        assert (addr[ok] + 3 < nX).all() and (addr[ok] % 4 == 0).all()
                        for j in range(4):
                            k = 4 * pv + j
                            As[k, _swz(q, k)] = np.where(ok, X[np.where(ok, addr + j, 0)], 0.0)
                # constant row: other generating factors (digits of blk), outer (digits of s)
                c = np.ones(Rp)
                b = blk
                for m in gen[1:]:
                    c[:R] *= U[m][b % dims[m]]
                    b //= dims[m]
                ss = s
                for m in outer:
                    c[:R] *= U[m][ss % dims[m]]
                    ss //= dims[m]
                for i in range(NB):
                    row = i0 + kb + kstep * i
                    assert (row < rows0).all() and (r0 + 4 * rv + 3 < Rp).all()
                    for j in range(4):
                        Bs[kb + kstep * i, 4 * rv + j] = U0p[row, r0 + 4 * rv + j] * c[r0 + 4 * rv + j]
                assert not np.isnan(As).any() and not np.isnan(Bs).any()
                # compute: thread (tq, tr) reads logical q = 8 tq + i at swz
                A = np.empty((FK, FQ))
                for k in range(FK):
                    for g in range(FQ // 4):
                        A[k, 4 * g:4 * g + 4] = As[k, _swz(4 * g, k):_swz(4 * g, k) + 4]
                acc += A.T @ Bs
            for r in range(BR):
                if r0 + r < R:
                    n = min(FQ, Q - q0)
                    part[z, r0 + r, q0:q0 + n] = acc[:n, r]
    return part.sum(0).T


@pytest.mark.parametrize("dims,R,mode", [((128, 64, 32), 16, 0), ((128, 64, 32), 16, 1), ((128, 64, 32), 16, 2),
                                         ((36, 96, 40), 40, 0), ((64, 20, 12), 70, 1), ((32, 9, 7), 5, 2),
                                         ((32, 64, 3, 5), 12, 3), ((260, 32, 6), 8, 0)])
def test_ffma_mttkrp_restated_matches_oracle(dims, R, mode):
    import oracle
    rng = np.random.default_rng(sum(dims) + R + mode)
    X = rng.random(int(np.prod(dims))).astype(np.float32).astype(np.float64)
    facs = [rng.random(d * R).astype(np.float32).astype(np.float64) for d in dims]
    got = ffma_restated(X, dims, facs, mode, R, sms=3)
    want = oracle.mttkrp(X, dims, facs, mode, R)
    assert np.abs(got.reshape(-1, order="F") - want).max() <= 1e-12 * np.abs(want).max()


def test_ffma_plan_limits():
    # eligible shapes and the ones that fall back to the general kernel
    assert ffma_plan((512, 512, 512), 0, 64)["splits"] * 4 <= 2 * 148 + 4
    assert ffma_plan((96, 96, 96, 96), 2, 32)["BR"] == 32
    assert ffma_plan((37, 8, 8), 1, 8) is None       # rows0 not a multiple of 32
    assert ffma_plan((38, 64, 8), 0, 8) is None       # mode 0 rows not a multiple of 4


# ---- residual.cu k_residual_ffma: 128 rows x 32-column stages, B = U_1 rows
# x the constant row, 8 x 4 patches per thread, X float4 loads
def residual_ffma_restated(X, dims, facs, R, sms=148):
    I0, rows1 = dims[0], dims[1]
    assert I0 % 4 == 0 and rows1 % 32 == 0 and R <= 64
    rest = int(np.prod(dims[1:]))
    qtiles = -(-I0 // 128)
    stages = rest // 32
    want = -(-(3 * sms) // qtiles)
    splits = max(1, min(want, stages))
    chunk = -(-stages // splits)
    splits = -(-stages // chunk)
    U = [f.reshape(d, R, order="F") for f, d in zip(facs, dims)]
    As = np.zeros((64, 128))
    t = np.arange(128)
    tq, tk = t >> 3, t & 7
    res = xx = 0.0
    parts = 0
    for bx in range(qtiles * splits):
        q0, z = (bx % qtiles) * 128, bx // qtiles
        As[:] = 0
        n = min(128, I0 - q0)
        As[:R, :n] = U[0][q0:q0 + n].T
        for st in range(z * chunk, min(stages, z * chunk + chunk)):
            k0 = st * 32
            i1 = k0 % rows1
            lin = k0 // rows1
            c = np.ones(R)
            for m in range(2, len(dims)):
                c *= U[m][lin % dims[m]]
                lin //= dims[m]
            Bs = np.zeros((64, 32))
            for i in range(4):
                r = tq + 16 * i
                ok = r < R
                addr = i1 + 4 * tk + rows1 * r
                assert (addr[ok] + 3 < rows1 * R).all()
                for j in range(4):
                    Bs[r[ok], 4 * tk[ok] + j] = facs[1][addr[ok] + j] * c[r[ok]]
            H = As.T @ Bs                                 # 128 x 32
            for c4 in range(4):
                col = k0 + 4 * tk + c4
                qa = q0 + 8 * tq
                for half in range(2):
                    ok = qa + 4 * half < I0
                    addr = qa + 4 * half + I0 * col
                    assert (addr[ok] + 3 < X.size).all() and (addr[ok] % 4 == 0).all()
                    for j in range(4):
                        x = np.where(ok, X[np.where(ok, addr + j, 0)], 0.0)
                        h = H[8 * tq + 4 * half + j, 4 * tk + c4]
                        res += float(np.sum(np.where(ok, (x - h) ** 2, 0.0)))
                        xx += float(np.sum(x ** 2))
        parts += 1
    return res, xx, parts


@pytest.mark.parametrize("dims,R", [((128, 64, 32), 16), ((260, 32, 6, 5), 7), ((36, 96, 40), 64), ((4, 32, 3), 3)])
def test_residual_ffma_restated_matches_fp64(dims, R):
    import oracle
    rng = np.random.default_rng(sum(dims) + R)
    facs = [rng.random(d * R) for d in dims]
    X = oracle.gencp(dims, facs, R) + 0.01 * rng.standard_normal(int(np.prod(dims)))
    res, xx, parts = residual_ffma_restated(X, dims, facs, R, sms=2)
    want = float(np.sum((X - oracle.gencp(dims, facs, R)) ** 2))
    assert abs(res - want) <= 1e-9 * want
    assert abs(xx - float(np.sum(X ** 2))) <= 1e-12 * xx


# ---- solve.cu k_normal_inverse_small: 16 x 16 threads own (ty + 16a, tx + 16b)
def normal_inverse_small_restated(V):
    """Gauss-Jordan as k_normal_inverse_small runs it: the owners of row k
    and column k publish them (buffer k & 1), then every thread updates its
    16 entries from the published copies only.  Returns (Vinv, failed)."""
    R = V.shape[0]
    v = np.zeros((64, 64))
    v[:R, :R] = V
    owner_rows = np.arange(64)          # i = ty + 16 a  <->  (ty, a) = (i % 16, i // 16)
    maxdiag = np.max(np.abs(np.diag(V)))
    rowb = np.zeros((2, 64)); colb = np.zeros((2, 64))
    written = np.zeros((2, 64), bool)
    for k in range(R):
        kb, kk, buf = k >> 4, k & 15, k & 1
        # row k: threads ty == kk with a == kb write columns tx + 16 b
        ty, a = owner_rows % 16, owner_rows // 16
        assert ((ty == kk) & (a == kb)).sum() == 1
        rowb[buf] = v[k]; colb[buf] = v[:, k]
        written[buf] = True
        piv = rowb[buf][k]
        if not (piv > 1e-13 * maxdiag) or not np.isfinite(piv):
            return None, True
        inv = 1.0 / piv
        j = np.arange(64)
        rj = np.where(j == k, 1.0, rowb[buf]) * inv
        old = np.where(j[None, :] == k, 0.0, v)
        v = np.where(np.arange(64)[:, None] == k, rj[None, :], old - colb[buf][:, None] * rj[None, :])
    out = 0.5 * (v[:R, :R] + v[:R, :R].T)
    # the padding stays zero
    assert np.all(v[R:, :] == 0) and np.all(v[:, R:] == 0)
    return out, False


@pytest.mark.parametrize("R", [1, 5, 16, 33, 64])
def test_normal_inverse_small_restated_inverts(R):
    rng = np.random.default_rng(R)
    A = rng.standard_normal((3 * R + 2, R))
    B = rng.standard_normal((2 * R + 3, R))
    V = (A.T @ A) * (B.T @ B)          # Hadamard of two Grams: SPD
    Vi, failed = normal_inverse_small_restated(V)
    assert not failed
    assert np.linalg.norm(Vi @ V - np.eye(R)) <= 1e-8 * np.linalg.cond(V)


def test_normal_inverse_small_restated_flags_singular():
    A = np.random.default_rng(0).standard_normal((3, 8))
    V = A.T @ A                          # rank 3 of 8
    _, failed = normal_inverse_small_restated(V)
    assert failed


# ---- solve.cu k_update_fused: rb rows per CTA, split z of an entry by thread z mod T
def update_fused_restated(parts, splits, I, R, zs, qs, rs, NT=256, RBMAX=8):
    rb = min(RBMAX, max(1, -(-I // 256)))
    grid = -(-I // rb)
    vec = rs == 1 and qs % 4 == 0 and zs % 4 == 0 and qs >= -(-R // 4) * 4
    M = np.full(I * R, np.nan)
    count = np.zeros(parts.size, np.int64)
    W = 4 if vec else 1                      # entries per load
    RW = -(-R // W)                          # loads per row
    for b in range(grid):
        q0 = b * rb
        nr = min(rb, I - q0)
        items = nr * RW
        T = 1 if items >= NT else NT // items
        sums = {}
        for t in range(NT):
            if T == 1:
                its, z0 = range(t, items, NT), 0
            else:
                it, z0 = t % items, t // items
                if z0 >= T:
                    continue
                its = [it]
            for it in its:
                row, cw = divmod(it, RW)
                base = (q0 + row) * qs + cw * W * rs
                for z in range(z0, splits, T):
                    for k in range(W):
                        idx = base + k * rs + z * zs
                        assert 0 <= idx < parts.size
                        count[idx] += 1
                        c = cw * W + k
                        if c < R:
                            sums[(row, c)] = sums.get((row, c), 0.0) + parts[idx]
        for (row, c), v in sums.items():
            q = q0 + row
            assert np.isnan(M[q + I * c])
            M[q + I * c] = v
    return M, count


@pytest.mark.parametrize("I,R,splits", [(512, 64, 73), (96, 32, 37), (128, 16, 36), (5, 3, 1), (700, 64, 3),
                                        (4100, 8, 2), (300, 7, 5)])
def test_update_fused_sums_every_split_once(I, R, splits):
    Rp = -(-R // 4) * 4
    rng = np.random.default_rng(I + R)
    parts = rng.standard_normal(splits * I * Rp)
    M, count = update_fused_restated(parts, splits, I, R, I * Rp, Rp, 1)
    want = parts.reshape(splits, I, Rp).sum(0)[:, :R]
    assert np.allclose(M.reshape(R, I).T, want)
    used = count.reshape(splits, I, Rp)
    # every entry of every split once; the float4 loads also touch the padding
    assert np.all(used[:, :, :R] == 1) and np.all(used[:, :, R:] <= 1)
    # the column-major single-split form (an MTTKRP that wrote M itself)
    Mc = rng.standard_normal(I * R)
    M2, count2 = update_fused_restated(Mc, 1, I, R, 0, 1, I)
    assert np.array_equal(M2, Mc) and np.all(count2 == 1)


def test_update_fused_shared_memory_fits():
    # V^-1 (R^2) + M rows (FU_RB R) + 4 NT split sums, FP64, at R = 64
    assert 8 * (64 * 64 + 8 * 64 + 4 * 256) <= 48 * 1024


# ---- solve.cu k_gram_rows: thread t owns the 4 x 4 block tri(t) of the upper triangle
def tri_pq(e):
    q = int((np.sqrt(8.0 * e + 1.0) - 1.0) * 0.5)
    while (q + 1) * (q + 2) // 2 <= e:
        q += 1
    while q * (q + 1) // 2 > e:
        q -= 1
    return e - q * (q + 1) // 2, q


@pytest.mark.parametrize("R", [1, 3, 4, 16, 31, 32, 63, 64])
def test_gram_rows_blocks_cover_triangle_once(R):
    R4 = -(-R // 4)
    nblk = R4 * (R4 + 1) // 2
    assert nblk <= 256
    T = R * (R + 1) // 2
    hits = np.zeros(T, np.int32)
    for t in range(nblk):
        bp, bq = tri_pq(t)
        assert bp <= bq < R4
        for u in range(4):
            for v in range(4):
                p, q = 4 * bp + u, 4 * bq + v
                if p <= q < R:
                    hits[q * (q + 1) // 2 + p] += 1
    assert np.all(hits == 1)
    # the staged rows: 128 x (4 R4 + 4) floats
    assert 4 * 128 * (4 * R4 + 4) <= 48 * 1024


# ---- residual_tc.cu k_residual_tc: tiles, k split, B layout, TMEM and smem budget
def residual_tc_plan(dims, R, sms=148):
    if len(dims) < 3 or R > 64 or dims[0] % 4:
        return None
    Rpad = -(-R // 16) * 16
    nq = -(-dims[1] // 128)
    if 2 * nq * 128 * Rpad * 2 > 128 * 1024:
        return None
    K = int(np.prod(dims[2:]))
    tiles = -(-dims[0] // 128)
    cpt = max(1, min(K, sms // tiles))
    return Rpad, nq, K, tiles, cpt


@pytest.mark.parametrize("dims,R", [((512, 512, 512), 64), ((96, 96, 96, 96), 32), ((20, 16, 12), 3),
                                    ((128, 128, 128), 16), ((4, 1000, 3), 9), ((1000, 200, 7, 3), 64)])
def test_residual_tc_index_math(dims, R):
    p = residual_tc_plan(dims, R)
    assert p is not None
    Rpad, nq, K, tiles, cpt = p
    ctrl, xbytes = 2048, 128 * 32 * 4
    bbytes = nq * 128 * Rpad * 2
    assert bbytes % 4096 == 0                                   # the X ring stays 1024-aligned
    xs = 12                                                     # rt_ring: the deepest ring that fits
    while xs > 2 and 1024 + ctrl + 2 * bbytes + xs * xbytes > 232448:
        xs -= 1
    assert 1024 + ctrl + 2 * bbytes + xs * xbytes <= 232448     # shared memory
    # ring slots and parities: stage x in slot x % xs, phase x // xs
    for x in range(3 * xs + 1):
        assert 0 <= x % xs < 12
    assert 2 * 128 + 2 * 64 <= 512                              # TMEM: accumulators + A' buffers
    # B words: every (chunk, row, k-chunk) once, inside one operand
    kcs = Rpad // 8
    offs = set()
    for q in range(nq):
        for jr in range(0, 128, 37):
            for kc in range(kcs):
                off = q * 128 * Rpad * 2 + jr * 16 + kc * 128 * 16
                assert 0 <= off and off + 16 <= bbytes
                offs.add(off)
    # MMA descriptors: K step kk reads two 2048-byte K chunks of its chunk
    for kk in range(Rpad // 16):
        assert (2 * kk + 2) * 2048 <= 128 * Rpad * 2
    # k ranges of a tile's CTAs partition [0, K)
    covered = []
    for zc in range(cpt):
        kb, ke = K * zc // cpt, K * (zc + 1) // cpt
        assert ke > kb
        covered.extend(range(kb, ke))
    assert covered == list(range(K))
    # TMA coordinates: x (rows) 128-aligned inside the tensor, y and z in int32
    assert (tiles - 1) * 128 < dims[0] and (tiles - 1) * 128 * 4 % 16 == 0
    assert nq * 128 < 2 ** 31 and K < 2 ** 31
    assert tiles * cpt <= 148


def test_residual_tc_slices_reconstruct():
    """The slice identity the kernel uses: Xh[:, :, k] = (U_0 diag(c_k)) U_1^T
    with c_k the product of the slower factors' rows of k's digits."""
    rng = np.random.default_rng(2)
    dims, R = (6, 5, 4, 3), 3
    U = [rng.standard_normal((d, R)) for d in dims]
    full = np.einsum("ir,jr,kr,lr->ijkl", *U)
    K = dims[2] * dims[3]
    for k in range(K):
        d2, d3 = k % dims[2], k // dims[2]
        c = U[2][d2] * U[3][d3]
        sl = (U[0] * c) @ U[1].T
        assert np.allclose(sl, full[:, :, d2, d3])
