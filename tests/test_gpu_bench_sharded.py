"""The multi-GPU benchmark path (bench.py run under torchrun, sweeps sharded
along the last mode, NCCL all-reduces, one sweep captured in a CUDA graph)
run end to end on one rank: it must exit cleanly and print one JSON line
whose numbers are sane.  (More ranks need more GPUs than a test run here
has; the exchange itself is covered over gloo on the CPU.)"""
import json
import os
import socket
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_sharded_bench_path_one_rank():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "1",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--sharded", "--dims", "128,128,128", "--rank", "16", "--steps", "3", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [x for x in r.stdout.strip().splitlines() if x.startswith("{")][-1]
    d = json.loads(line)
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["value"] > 0
    assert d["sweep_graph"] is True
    assert 0.9 < d["fit_after_timed_sweeps"] < 1.0
    assert d["e2e"]["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0
