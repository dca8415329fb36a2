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


# ---- batched.cu mttkrp_small: RT x 4 register tiles with unguarded loads
BMAXD, BMAXR = 96, 16
SLICE = BMAXD * (BMAXD + 1) + 4
RED3 = 2 * BMAXR * BMAXD


@pytest.mark.parametrize("RT", [2, 4])
def test_batched_tile_reads_stay_in_buffers(RT):
    NGM = BMAXD // RT
    worst_slice = worst_fac = worst_red = -1
    for I in (16, 37, 94, 95, 96):
        for J in (16, 53, 95, 96):
            ld = I + 1
            for mode in (0, 1):
                rows = I if mode == 0 else J
                ngrp = -(-rows // RT)
                rp_max = (ngrp - 1) * RT
                L = J if mode == 0 else I
                if mode == 0:   # sl[rp + v + ld j], F[1][j + J (r0 + c)]
                    worst_slice = max(worst_slice, rp_max + RT - 1 + ld * (L - 1))
                    worst_fac = max(worst_fac, (L - 1) + J * (BMAXR - 1))
                else:           # sl[i + ld (rp + v)], F[0][i + I (r0 + c)]
                    worst_slice = max(worst_slice, (L - 1) + ld * (rp_max + RT - 1))
                    worst_fac = max(worst_fac, (L - 1) + I * (BMAXR - 1))
            ngrp = -(-J // RT)
            worst_red = max(worst_red, (2 * RT * BMAXR - 1) * NGM + ngrp - 1)
    assert worst_slice < SLICE
    assert worst_fac < BMAXD * BMAXR
    assert worst_red < RED3


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
    assert rows0 % BKS == 0 and rows0 // BKS >= 2     # the pre-packed path
    blk = rows0 // BKS
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
                splits=splits, chunk=chunk, smem=smem(nring))


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
