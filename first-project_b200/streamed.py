"""Out-of-core CP-ALS: the tensor stays in (pinned) host memory and every
mode's MTTKRP streams it through the GPU in slabs along the last mode, the
way decomposition/GPU/large/slice_cp_als.cu does (one host-to-device copy
per frontal slice, :77-79 for A, :116-118 for B, :151-155 for C, each
followed by a GEMM that accumulates into the mode's right-hand side).

Here a slab is `slab` consecutive frontal slices (one contiguous host range
in column-major order).  Copies run on their own stream into `nbuf` device
buffers, so slab s+1 (and later ones) crosses the host link while slab s is
contracted; a buffer is refilled only after the MTTKRP that read it has
finished.  Slab partial MTTKRPs of the modes n < N-1 are summed on the
device in slab order (deterministic); the last mode's rows are slab-local.
The sweep itself -- solve, Grams, fit -- is the sharded sweep of
distributed.py with the slabs in place of ranks and an identity all-reduce,
over the same library calls (cud_mttkrp, cud_cp_solve, cud_factor_gram,
cud_cp_fit_terms).
"""
from __future__ import annotations

import numpy as np

from distributed import CudaOps, ShardedCP


def slab_ranges(last_extent: int, slab: int):
    """[(k0, k1), ...] covering 0 .. last_extent in steps of `slab`."""
    if slab <= 0:
        raise ValueError("slab must be positive")
    return [(k0, min(last_extent, k0 + slab)) for k0 in range(0, last_extent, slab)]


class LocalComm:
    """One process holds every slab: the all-reduce is the identity."""

    def all_reduce(self, t):
        return t

    def all_reduce_scalar(self, x):
        return float(x)


class StreamedOps(CudaOps):
    """CudaOps whose MTTKRP and norm read a host-resident tensor slab by slab.

    X passed to mttkrp/norm2 is the host tensor (flat, column-major, FP32,
    pinned for the copies to overlap); `dims` are the full extents."""

    def __init__(self, cd, precision, slab, nbuf=2, stream=None):
        import torch
        super().__init__(cd, precision, stream=None)
        self.slab, self.nbuf = int(slab), max(2, int(nbuf))
        self.compute = stream if stream is not None else torch.cuda.Stream()
        self.copy = torch.cuda.Stream()
        self.stream = self.compute.cuda_stream
        self.bufs = None
        self.h2d_bytes = 0

    def _buffers(self, n):
        torch = self.torch
        if self.bufs is None or self.bufs[0].numel() < n:
            self.bufs = [torch.empty(n, device="cuda") for _ in range(self.nbuf)]
            self.copied = [torch.cuda.Event() for _ in range(self.nbuf)]
            self.used = [None] * self.nbuf

    def _stream_slabs(self, Xh, dims, body, first=0):
        """Calls body(s, k0, k1, slab_tensor) on the compute stream for every
        slab from `first` on, with the copies overlapped."""
        torch = self.torch
        P = 1
        for d in dims[:-1]:
            P *= int(d)
        ranges = slab_ranges(int(dims[-1]), self.slab)[first:]
        self._buffers(P * min(self.slab, int(dims[-1])))

        def issue(s):
            b = s % self.nbuf
            k0, k1 = ranges[s]
            with torch.cuda.stream(self.copy):
                if self.used[b] is not None:
                    self.copy.wait_event(self.used[b])  # the MTTKRP that read this buffer is done
                self.bufs[b][: (k1 - k0) * P].copy_(Xh[k0 * P: k1 * P], non_blocking=True)
                self.copied[b].record(self.copy)
            self.h2d_bytes += 4 * (k1 - k0) * P

        for s in range(min(self.nbuf - 1, len(ranges))):
            issue(s)
        for s, (k0, k1) in enumerate(ranges):
            if s + self.nbuf - 1 < len(ranges):
                issue(s + self.nbuf - 1)
            b = s % self.nbuf
            with torch.cuda.stream(self.compute):
                self.compute.wait_event(self.copied[b])
                body(first + s, k0, k1, self.bufs[b][: (k1 - k0) * P])
                ev = torch.cuda.Event()
                ev.record(self.compute)
                self.used[b] = ev

    def mttkrp(self, Xh, dims, U, mode, R, out=None):
        torch = self.torch
        N = len(dims)
        I = int(dims[mode])
        M = out.zero_() if out is not None else torch.zeros(I * R, device="cuda")
        part = torch.empty(I * R, device="cuda") if mode < N - 1 else None

        def body(s, k0, k1, Xs):
            sd = list(dims[:-1]) + [k1 - k0]
            Us = list(U)
            if mode < N - 1:  # the last factor's rows of this slab
                Us[-1] = U[-1].view(R, int(dims[-1]))[:, k0:k1].contiguous().view(-1)
                self.cd.mttkrp(Xs, sd, Us, mode, R, part, self.precision, stream=self.stream)
                M.add_(part)
            else:
                out = torch.empty((k1 - k0) * R, device="cuda")
                self.cd.mttkrp(Xs, sd, Us, mode, R, out, self.precision, stream=self.stream)
                M.view(R, I)[:, k0:k1].copy_(out.view(R, k1 - k0))

        self._stream_slabs(Xh, dims, body)
        return M

    def norm2(self, Xh):
        """||X||^2 in FP64, summed over the slabs in order."""
        parts = []

        def body(s, k0, k1, Xs):
            parts.append(self.cd.norm2(Xs, stream=self.stream))

        self._stream_slabs(Xh, self.dims, body)
        return float(sum(parts))


class StreamedCP(ShardedCP):
    """CP-ALS of a host-resident tensor, streamed slab by slab.

    X_host: flat FP32 CPU tensor in column-major order (pin it for copy
    overlap); factors: full I_n x R device factors (updated each sweep)."""

    def __init__(self, cd, X_host, dims, R, factors, slab, precision, nbuf=2, stream=None):
        import torch
        ops = StreamedOps(cd, precision, slab, nbuf=nbuf, stream=stream)
        ops.dims = list(dims)
        # every allocation and launch on the compute stream (the caching
        # allocator ties a block to the stream it was allocated on)
        with torch.cuda.stream(ops.compute):
            super().__init__(ops, LocalComm(), X_host, list(dims), R, factors)

    def sweep(self):
        import torch
        with torch.cuda.stream(self.ops.compute):
            super().sweep()

    def fit(self):
        import torch
        with torch.cuda.stream(self.ops.compute):
            return super().fit()

    @property
    def h2d_bytes(self):
        return self.ops.h2d_bytes


class StreamedTucker:
    """Tucker HOSVD of a host-resident tensor, streamed slab by slab along
    the last mode (decomposition/GPU/large/slice_tucker_hosvd.cu:3-160):

    * the Grams of the modes n < N-1 are sums of the slabs' unfolding Grams
      (:36-37), accumulated in FP64 in slab order;
    * the last mode's Gram pairs every slab with every other (:38-40 pairs
      every frontal slice): one pass gives the diagonal blocks, then for
      each slab s a copy is held on the device while the slabs t > s
      stream past, giving the blocks (s, t) and (t, s) (cud_cross_gram);
    * the factors are the leading eigenvectors of each FP64 Gram (full
      Jacobi, ascending order, as syevdx returns them);
    * the core is the sum over slabs of the slab projected on every factor,
      the last one restricted to the slab's rows (:98-104).

    FP32 data and CUDA-core contractions, like the reference's slice path.
    Host traffic: the tensor once for the leading Grams, about p^2 / 2 slabs
    for the last mode's Gram (p slabs), once for the core."""

    def __init__(self, cd, X_host, dims, slab, nbuf=2, stream=None):
        self.cd, self.Xh, self.dims = cd, X_host, [int(d) for d in dims]
        self.ops = StreamedOps(cd, cd.PREC_FP32, slab, nbuf=nbuf, stream=stream)
        self.ops.dims = self.dims

    @property
    def h2d_bytes(self):
        return self.ops.h2d_bytes

    def hosvd(self, ranks, core, factors):
        """core (prod ranks, FP32) and factors[m] (dims[m] x ranks[m], FP32,
        column-major) are device tensors, written in place.  Returns the
        worst eigensolver status."""
        import torch
        cd, ops, dims = self.cd, self.ops, self.dims
        N = len(dims)
        last = dims[-1]
        P = 1
        for d in dims[:-1]:
            P *= d
        ranges = slab_ranges(last, ops.slab)
        worst = cd.OK
        with torch.cuda.stream(ops.compute):
            G = [torch.zeros(d * d, dtype=torch.float64, device="cuda") for d in dims]
            tmp = torch.empty(max([d * d for d in dims[:-1]] + [1]), dtype=torch.float64, device="cuda")
            held = torch.empty(P * min(ops.slab, last), device="cuda")

            def leading(s, k0, k1, Xs):
                sd = dims[:-1] + [k1 - k0]
                for n in range(N - 1):
                    cd.unfold_gram(Xs, sd, n, tmp[: dims[n] * dims[n]], stream=ops.stream)
                    G[n].add_(tmp[: dims[n] * dims[n]])
                cd.cross_gram(Xs, Xs, P, k1 - k0, k1 - k0, G[-1][k0 + last * k0:], last, stream=ops.stream)

            ops._stream_slabs(self.Xh, dims, leading)
            for s, (k0, k1) in enumerate(ranges[:-1]):
                ks = k1 - k0
                hs = held[: ks * P]
                hs.copy_(self.Xh[k0 * P: k1 * P], non_blocking=True)  # on the compute stream
                ops.h2d_bytes += 4 * ks * P

                def cross(t, t0, t1, Xt, k0=k0, ks=ks, hs=hs):
                    kt = t1 - t0
                    cd.cross_gram(hs, Xt, P, ks, kt, G[-1][k0 + last * t0:], last, stream=ops.stream)
                    cd.cross_gram(Xt, hs, P, kt, ks, G[-1][t0 + last * k0:], last, stream=ops.stream)

                ops._stream_slabs(self.Xh, dims, cross, first=s + 1)
            for n in range(N):
                W = torch.empty(dims[n], dtype=torch.float64, device="cuda")
                V = torch.empty(dims[n] * dims[n], dtype=torch.float64, device="cuda")
                st = cd.syev_jacobi(G[n], dims[n], W, V, stream=ops.stream)
                if st != cd.OK:
                    worst = st
                r = int(ranks[n])
                # column-major V: its last r columns are rows n - r .. n - 1 of V.view(n, n)
                factors[n].copy_(V.view(dims[n], dims[n])[dims[n] - r:, :].reshape(-1).float())
            core.zero_()
            # W_m = U_m^T (r_m x d_m, column-major) for the projections
            Wt = [factors[m].view(int(ranks[m]), dims[m]).t().contiguous().view(-1) for m in range(N - 1)]

            def project(s, k0, k1, Xs):
                cur = dims[:-1] + [k1 - k0]
                Y = Xs
                for m in range(N - 1):
                    out = list(cur)
                    out[m] = int(ranks[m])
                    Z = torch.empty(int(np.prod(out)), device="cuda")
                    cd.mode_product(Y, cur, m, Wt[m], int(ranks[m]), Z, stream=ops.stream)
                    Y, cur = Z, out
                rl = int(ranks[-1])
                Wl = factors[-1].view(rl, last)[:, k0:k1].t().contiguous().view(-1)
                Z = torch.empty(core.numel(), device="cuda")
                cd.mode_product(Y, cur, N - 1, Wl, rl, Z, stream=ops.stream)
                core.add_(Z)

            ops._stream_slabs(self.Xh, dims, project)
        ops.compute.synchronize()
        return worst
