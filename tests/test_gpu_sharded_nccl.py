"""The sharded CP-ALS (distributed.ShardedCP with the CUDA ops) over a real
NCCL process group of one rank: its sweeps against the single-GPU plan from
the same start, and one sweep captured in a CUDA graph (kernels and NCCL
all-reduces) against eager sweeps, bit for bit.  (More ranks need more GPUs;
the exchange logic for 2 and 3 ranks is covered on the CPU over gloo.)"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.fixture(scope="module")
def nccl_group():
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    yield dist
    dist.destroy_process_group()


def test_sharded_sweeps_match_plan_and_graph_replay(cd, nccl_group):
    sys.path.insert(0, os.path.join(ROOT, "first-project_b200"))
    from distributed import CudaOps, ShardedCP, TorchComm
    dims, R = (96, 80, 64), 8
    X, _ = cd.make_cp_tensor(dims, R, seed=12)
    init = cd.make_init(dims, R, seed=13)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    comm = TorchComm(nccl_group)
    with torch.cuda.stream(stream):
        Ua = [u.clone() for u in init]
        eager = ShardedCP(CudaOps(cd, cd.PREC_BF16X3, stream=sptr), comm, X, dims, R, Ua)
        for _ in range(6):
            eager.sweep()
        fit_eager = eager.fit()
        Ub = [u.clone() for u in init]
        graphed = ShardedCP(CudaOps(cd, cd.PREC_BF16X3, stream=sptr), comm, X, dims, R, Ub)
        graphed.sweep()                       # warm-up: workspaces sized before capture
        assert graphed.capture(torch, stream)
        for _ in range(5):
            graphed.sweep()                   # replays
        fit_graph = graphed.fit()
    torch.cuda.synchronize()
    graphed.release()
    assert fit_eager == fit_graph
    for a, b in zip(Ua, Ub):
        assert torch.equal(a, b)
    # the single-GPU plan from the same start (its update sums in another
    # order); both fits here are the sweep estimate ||X||^2 - 2<M, U> + ||Xhat||^2
    Uc = [u.clone() for u in init]
    res = cd.cp_als(X, dims, R, Uc, max_sweeps=6, precision=cd.PREC_BF16X3)
    assert abs(res.fit_estimate - fit_eager) <= 2e-5, (res.fit_estimate, fit_eager)
    for a, c in zip(Ua, Uc):
        assert float(torch.linalg.norm(a - c) / torch.linalg.norm(c)) <= 1e-3
