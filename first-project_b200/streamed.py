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

    def _stream_slabs(self, Xh, dims, body):
        """Calls body(s, k0, k1, slab_tensor) on the compute stream for every
        slab, with the copies overlapped."""
        torch = self.torch
        P = 1
        for d in dims[:-1]:
            P *= int(d)
        ranges = slab_ranges(int(dims[-1]), self.slab)
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
                body(s, k0, k1, self.bufs[b][: (k1 - k0) * P])
                ev = torch.cuda.Event()
                ev.record(self.compute)
                self.used[b] = ev

    def mttkrp(self, Xh, dims, U, mode, R):
        torch = self.torch
        N = len(dims)
        I = int(dims[mode])
        M = torch.zeros(I * R, device="cuda")
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
