"""Host logic of the sharded (multi-GPU) CP-ALS, run as two gloo ranks on the
CPU: the tensor is split along its last mode, the partial MTTKRPs of the
other modes are all-reduced, the last factor stays sharded.  Per-rank
compute comes from the oracle here (on GPUs it is the CUDA library, see
distributed.CudaOps); the result must equal the single-process oracle ALS
from the same start."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle

DIMS = (9, 8, 12)
R = 3
SWEEPS = 6


def _into(out, t):
    """The ops' `out` convention: write into the given buffer and return it."""
    if out is None:
        return t
    out.copy_(t)
    return out


class OracleOps:
    def alloc(self, n):
        return torch.empty(n, dtype=torch.float64)

    def mttkrp(self, X, dims, U, mode, R, out=None):
        return _into(out, torch.from_numpy(oracle.mttkrp(X, dims, [u.numpy() for u in U], mode, R)))

    def solve(self, M, I, R, G, mode, out=None):
        V = np.ones((R, R))
        for m, g in enumerate(G):
            if m != mode:
                V = V * g.numpy().reshape(R, R, order="F")
        Mm = M.numpy().reshape(I, R, order="F")
        return _into(out, torch.from_numpy(np.linalg.solve(V.T, Mm.T).T.reshape(-1, order="F").copy()))

    def gram(self, U, I, out=None):
        Um = U.numpy().reshape(I, -1, order="F")
        return _into(out, torch.from_numpy((Um.T @ Um).reshape(-1, order="F").copy()))

    def fit_terms(self, M, U, G, R):
        nh = np.ones((R, R))
        for g in G:
            nh = nh * g.numpy().reshape(R, R, order="F")
        return float(np.dot(M.numpy(), U.numpy())), float(nh.sum())

    def norm2(self, X):
        return float(np.dot(X.astype(np.float64), X))


def problem():
    rng = np.random.default_rng(0)
    true = [rng.random(d * R) for d in DIMS]
    X = oracle.gencp(DIMS, true, R).astype(np.float32)
    init = [rng.random(d * R) for d in DIMS]
    return X, init


def worker(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "first-project_b200"))
    from distributed import ShardedCP, TorchComm
    X, init = problem()
    K = DIMS[-1]
    k0, k1 = rank * K // world, (rank + 1) * K // world
    Xg = X.reshape(DIMS, order="F")
    Xl = np.asfortranarray(Xg[:, :, k0:k1]).reshape(-1, order="F")
    ldims = (DIMS[0], DIMS[1], k1 - k0)
    U = [torch.from_numpy(f.copy()) for f in init[:-1]]
    Cl = init[-1].reshape(K, R, order="F")[k0:k1].reshape(-1, order="F").copy()
    U.append(torch.from_numpy(Cl))
    cp = ShardedCP(OracleOps(), TorchComm(dist), Xl, ldims, R, U)
    fits = []
    for _ in range(SWEEPS):
        cp.sweep()
        fits.append(cp.fit())
    np.savez(os.path.join(outdir, f"rank{rank}.npz"), fits=np.array(fits),
             *[u.numpy() for u in cp.U])
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_cp_matches_single_process(tmp_path, world):
    mp.start_processes(worker, args=(world, free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    X, init = problem()
    facs, fits, _ = oracle.cp_als(X, DIMS, R, init, SWEEPS, use_lu=True)
    K = DIMS[-1]
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    for r, p in enumerate(parts):
        np.testing.assert_allclose(p["fits"], fits, rtol=0, atol=1e-9)
        for m in range(len(DIMS) - 1):
            np.testing.assert_allclose(p[f"arr_{m}"], facs[m], rtol=1e-8, atol=1e-10)
    # the sharded last factor, reassembled
    C = np.concatenate([p[f"arr_{len(DIMS) - 1}"].reshape(-1, R, order="F") for p in parts])
    np.testing.assert_allclose(C.reshape(-1, order="F"), facs[-1], rtol=1e-8, atol=1e-10)


def _shard_worker(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import json
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "first-project_b200"))
    from distributed import shard_batch
    rng = np.random.default_rng(30)
    n = 300
    dims = [tuple(int(x) for x in rng.integers(16, 97, 3)) for _ in range(n)]
    ranks = [int(x) for x in rng.integers(4, 17, n)]
    mine = shard_batch(dims, ranks, rank, world)
    parts = [None] * world
    dist.all_gather_object(parts, mine)
    if rank == 0:
        with open(os.path.join(outdir, "shards.json"), "w") as f:
            json.dump({"parts": parts, "work": [int(np.prod(d)) * r for d, r in zip(dims, ranks)]}, f)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_batched_shards_by_tensor(tmp_path, world):
    """Batched CP-ALS shards by tensor: every tensor on exactly one rank, the
    ranks' work within one tensor's work of each other (greedy largest
    first), each rank computing its share on its own (no data-path
    collective)."""
    import json
    mp.start_processes(_shard_worker, args=(world, free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    d = json.loads((tmp_path / "shards.json").read_text())
    parts, work = d["parts"], d["work"]
    allt = sorted(t for p in parts for t in p)
    assert allt == list(range(len(work)))
    loads = [sum(work[t] for t in p) for p in parts]
    assert max(loads) - min(loads) <= max(work)
