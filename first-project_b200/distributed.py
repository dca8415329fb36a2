"""CP-ALS across ranks (one process per GPU) with the tensor sharded along
its last mode.

Each rank holds a slab X_r = X[..., k0_r:k1_r] and the full factor matrices
of the other modes; the last factor is sharded like X.  Per sweep, for every
mode n:
  * n < N-1: the local MTTKRP over the slab is a partial sum of the global
    one; an all-reduce (sum) makes it global, then every rank computes the
    same solve, so the replicated factors stay identical;
  * n = N-1: the MTTKRP rows are local; each rank solves its own rows and
    the Gram of the last factor is all-reduced.
The fit needs <M_{N-1}, U_{N-1}> (all-reduced) and the Grams.  The collective
is a real exchange of I_n x R partial sums; nothing else moves.

The sweep logic is backend-neutral: `ops` supplies the per-rank compute
(the CUDA library for GPUs, see CudaOps) and `comm` the all-reduce
(torch.distributed over NCCL on GPUs, gloo on CPU in the tests).
"""
from __future__ import annotations

import math


class ShardedCP:
    def __init__(self, ops, comm, X, local_dims, R, factors):
        """factors[m] for m < N-1 are the full I_m x R factors (identical on
        every rank); factors[N-1] holds this rank's rows of the last factor.
        The factors are updated in place; every buffer a sweep touches is
        allocated here, so a sweep can be captured (see capture)."""
        self.ops, self.comm = ops, comm
        self.X, self.dims, self.R = X, list(local_dims), R
        self.U = list(factors)
        self.N = len(local_dims)
        self.M = [ops.alloc(d * R) for d in self.dims]
        self.G = [ops.gram(u, d) for u, d in zip(self.U, self.dims)]
        self.G[-1] = comm.all_reduce(self.G[-1])
        self.normx2 = comm.all_reduce_scalar(ops.norm2(X))
        self.M_last = None
        self.graph = None

    def sweep(self):
        if self.graph is not None:
            self.graph.replay()
            return
        if hasattr(self.ops, "inverse_begin"):
            self._sweep_overlapped()
            return
        N = self.N
        for n in range(N):
            M = self.ops.mttkrp(self.X, self.dims, self.U, n, self.R, out=self.M[n])
            if n < N - 1:
                M = self.comm.all_reduce(M)
            self.U[n] = self.ops.solve(M, self.dims[n], self.R, self.G, n, out=self.U[n])
            G = self.ops.gram(self.U[n], self.dims[n], out=self.G[n])
            self.G[n] = self.comm.all_reduce(G) if n == N - 1 else G
            if n == N - 1:
                self.M_last = M

    def _sweep_overlapped(self):
        """The same sweep with a second stream (ops providing inverse_begin /
        apply / side_gram): V_n^-1 needs only the other modes' Grams, so it
        runs beside MTTKRP_n and its all-reduce; the Gram of U_n (n < N-1)
        and V_{n+1}^-1 follow on the side stream while MTTKRP_{n+1} runs.
        The last mode's Gram is all-reduced on the main stream, and every
        side-stream step is waited for within the sweep (apply)."""
        N, ops = self.N, self.ops
        tok = ops.inverse_begin(self.G, self.R, 0)
        for n in range(N):
            M = ops.mttkrp(self.X, self.dims, self.U, n, self.R, out=self.M[n])
            if n < N - 1:
                M = self.comm.all_reduce(M)
            self.U[n] = ops.apply(M, self.dims[n], self.R, tok, out=self.U[n])
            if n < N - 1:
                self.G[n] = ops.side_gram(self.U[n], self.dims[n], out=self.G[n])
                tok = ops.inverse_begin(self.G, self.R, n + 1)
            else:
                G = ops.gram(self.U[n], self.dims[n], out=self.G[n])
                self.G[n] = self.comm.all_reduce(G)
                self.M_last = M

    def capture(self, torch, stream):
        """Captures one sweep (the per-rank kernels and the NCCL all-reduces)
        in a CUDA graph that sweep() replays; returns False, leaving eager
        sweeps, when the capture is refused.  Call after a warm-up sweep (the
        library's workspaces and the communicator exist) and release() before
        the process group is destroyed."""
        g = torch.cuda.CUDAGraph()
        try:
            # thread-local capture: the communicator's own threads keep
            # making CUDA calls while this thread captures
            with torch.cuda.graph(g, stream=stream, capture_error_mode="thread_local"):
                self.sweep()
        except Exception:
            self.graph = None
            return False
        self.graph = g
        return True

    def release(self):
        self.graph = None

    def fit(self):
        inner, nh = self.ops.fit_terms(self.M_last, self.U[-1], self.G, self.R)
        inner = self.comm.all_reduce_scalar(inner)
        res2 = self.normx2 - 2.0 * inner + nh
        return 1.0 - math.sqrt(max(res2, 0.0)) / math.sqrt(self.normx2)


class TorchComm:
    """all-reduce (sum) through torch.distributed (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, dist):
        self.dist = dist

    def all_reduce(self, t):
        self.dist.all_reduce(t)
        return t

    def all_reduce_scalar(self, x):
        import torch
        dev = "cuda" if self.dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t)
        return float(t.item())


class CudaOps:
    """Per-rank compute on the GPU through the library's C ABI; with `out`
    the result goes into the given buffer (no allocation)."""

    def __init__(self, cd, precision, stream=None):
        import torch
        self.cd, self.precision, self.stream = cd, precision, stream
        self.torch = torch
        self._work = None

    def alloc(self, n):
        return self.torch.empty(n, device="cuda")

    def mttkrp(self, X, dims, U, mode, R, out=None):
        if out is None:
            out = self.torch.empty(dims[mode] * R, device="cuda")
        self.cd.mttkrp(X, dims, U, mode, R, out, self.precision, stream=self.stream)
        return out

    def solve(self, M, I, R, G, mode, out=None):
        if self._work is None or self._work.numel() < 3 * R * R + 2:
            self._work = self.torch.zeros(3 * R * R + 2, dtype=self.torch.float64, device="cuda")
        if out is None:
            out = self.torch.empty(I * R, device="cuda")
        self.cd.cp_solve(M, I, R, G, mode, out, self._work, stream=self.stream)
        return out

    # The side stream: work enqueued there waits for everything queued so far
    # on the current (main) stream; the main stream waits for it through the
    # token apply() takes.  (self.stream must be the current torch stream.)
    def _fork(self):
        torch = self.torch
        if getattr(self, "_side", None) is None:
            self._side = torch.cuda.Stream()
        ev = torch.cuda.Event()
        ev.record()
        self._side.wait_event(ev)
        return self._side

    def inverse_begin(self, G, R, mode):
        if self._work is None or self._work.numel() < 3 * R * R + 2:
            self._work = self.torch.zeros(3 * R * R + 2, dtype=self.torch.float64, device="cuda")
        side = self._fork()
        self.cd.cp_normal_inverse(R, G, mode, self._work, stream=side.cuda_stream)
        done = self.torch.cuda.Event()
        done.record(side)
        return done

    def apply(self, M, I, R, token, out):
        self.torch.cuda.current_stream().wait_event(token)
        self.cd.cp_apply_inverse(M, I, R, self._work, out, stream=self.stream)
        return out

    def side_gram(self, U, I, out):
        side = self._fork()
        self.cd.factor_gram(U, I, U.numel() // I, out, stream=side.cuda_stream)
        return out

    def gram(self, U, I, out=None):
        R = U.numel() // I
        if out is None:
            out = self.torch.empty(R * R, dtype=self.torch.float64, device="cuda")
        self.cd.factor_gram(U, I, R, out, stream=self.stream)
        return out

    def fit_terms(self, M, U, G, R):
        return self.cd.cp_fit_terms(M, U, G, R, stream=self.stream)

    def norm2(self, X):
        return self.cd.norm2(X, stream=self.stream)


# ---------------------------------------------------------------- batched CP-ALS by tensor

def shard_batch(dims, ranks, rank, world):
    """The tensors of a batch that rank `rank` of `world` runs: a
    longest-processing-time assignment by work (elements x rank, the cost of
    an ALS sweep), largest first, ties to the lower rank; every tensor goes
    to exactly one rank and the assignment is the same on every rank.  The
    batch shards with no collective on the data path: the tensors are
    independent."""
    work = sorted(((-int(d[0]) * int(d[1]) * int(d[2]) * int(r), t) for t, (d, r) in enumerate(zip(dims, ranks))))
    load = [0] * world
    mine = []
    for w, t in work:
        k = min(range(world), key=lambda j: (load[j], j))
        load[k] -= w
        if k == rank:
            mine.append(t)
    return sorted(mine)


class ShardedBatch:
    """Batched CP-ALS over ranks: each rank packs its share of the tensors
    (shard_batch) into its own cd.Batch and runs the persistent batched
    kernel on its GPU; fits and sweeps are gathered once at the end (a
    result collective, not a data-path one)."""

    def __init__(self, cd, dims, ranks, rank, world):
        self.cd, self.rank, self.world = cd, rank, world
        self.all_dims, self.all_ranks = [tuple(d) for d in dims], list(ranks)
        self.mine = shard_batch(dims, ranks, rank, world)
        self.batch = cd.Batch([self.all_dims[t] for t in self.mine], [self.all_ranks[t] for t in self.mine])

    def run(self, max_sweeps=50, tol=1e-6, stream=None):
        fits, sweeps, launches = self.cd.cp_als_batched(self.batch, max_sweeps=max_sweeps, tol=tol, stream=stream)
        return dict(zip(self.mine, zip(fits, sweeps))), launches

    @staticmethod
    def gather(dist, local, n):
        """Per-tensor (fit, sweeps) of every rank's share, in tensor order."""
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local)
        out = [None] * n
        for p in parts:
            for t, v in p.items():
                out[t] = v
        return out
