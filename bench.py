#!/usr/bin/env python
"""Benchmark: CP-ALS sweeps and MTTKRP bandwidth on the 512 x 512 x 512,
rank-64 FP32 workload (synthetic: sum of 64 rank-1 terms with uniform [0,1)
factors plus 1e-3 relative Gaussian noise), one process per GPU.

A step is one CP-ALS sweep (three MTTKRPs, the FP64 normal-equation solves,
Gram updates and the fit) on device-resident data, replayed from the sweep's
CUDA graph.  `value` is the MTTKRP traffic the sweep implies (3 x algorithmic
bytes per MTTKRP) divided by the sweep time, in GB/s, summed over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's CPU path (the ALS of
decomposition/CPU/python/mycp.py, TensorLy on NumPy in FP64, restated on
NumPy/OpenBLAS because TensorLy is not installed) on the same workload, on
this host's cores, and reports the same metric.  The line of our arm also
times the reference's own GPU MTTKRP (its cuBLAS Khatri-Rao + SGEMM calls and
its public FP16 mttkrp) beside ours on the same GPU, and a C++/OpenMP CPU
baseline.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "first-project_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "CP-ALS time-to-fit & MTTKRP GB/s (% HBM peak), mixed/learned vs plain FP32"


def mttkrp_bytes(dims, R, mode):
    """Algorithmic bytes of one MTTKRP: the FP32 tensor once, the input
    factors and the output factor (4 B each)."""
    n = 1
    for d in dims:
        n *= d
    fac = sum(d for i, d in enumerate(dims) if i != mode) + dims[mode]
    return 4 * n + 4 * R * fac


def sweep_bytes(dims, R):
    return sum(mttkrp_bytes(dims, R, m) for m in range(len(dims)))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        if not getattr(self, "lines", None):
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def mttkrp_sample_errors(cd, torch, X, dims, R, U, sptr, rows=(0, 77, 300)):
    """Relative error of each MTTKRP precision against an FP64 evaluation of
    a few output rows of every mode (3rd-order workloads)."""
    import numpy as np
    if len(dims) != 3:
        return None
    X3 = X.cpu().numpy().reshape(tuple(reversed(dims))).transpose(2, 1, 0).astype(np.float64)
    F = [u.cpu().numpy().reshape(R, d).T.astype(np.float64) for u, d in zip(U, dims)]
    out = {}
    for name in ("fp32", "bf16x3", "bf16", "fp16"):
        errs = {}
        for mode in range(3):
            got = torch.empty(dims[mode] * R, device="cuda")
            cd.mttkrp(X, dims, U, mode, R, got, cd.PRECISIONS[name], stream=sptr)
            torch.cuda.synchronize()
            g = got.cpu().numpy().reshape(R, dims[mode]).T.astype(np.float64)
            num = den = 0.0
            for q in rows:
                if q >= dims[mode]:
                    continue
                sl = np.take(X3, q, axis=mode)          # the other two modes, in order
                a, b = [F[m] for m in range(3) if m != mode]
                want = np.einsum("ij,ir,jr->r", sl, a, b)
                num += float(np.sum((g[q] - want) ** 2))
                den += float(np.sum(want ** 2))
            errs[str(mode)] = float(f"{(num / den) ** 0.5:.3e}")
        out[name] = errs
    return out


def cpu_sweep_gbs(X3, factors, sweeps=1):
    """Times NumPy ALS sweeps (oracle port of mycp.py) -> (GB/s, seconds)."""
    import numpy as np
    import oracle
    dims = X3.shape
    R = factors[0].shape[1]
    oracle.numpy_cp_als_sweep(X3, [f.copy() for f in factors])  # warm the BLAS threads
    t0 = time.perf_counter()
    for _ in range(sweeps):
        oracle.numpy_cp_als_sweep(X3, factors)
    dt = time.perf_counter() - t0
    return sweep_bytes(dims, R) * sweeps / dt / 1e9, dt


def cpu_sample(dims, R, seed=0, slab=0):
    """The same synthetic workload generated on the host (FP64 holding FP32
    values), or a slab of it (the first `slab` indices of the last mode)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    d = list(dims)
    if slab > 0:
        d[-1] = min(slab, d[-1])
    facs = [rng.random((n, R)) for n in d]
    K = facs[1]
    for m in range(2, len(d)):
        K = (facs[m][:, None, :] * K[None, :, :]).reshape(-1, R)
    X = (facs[0] @ K.T).reshape(d, order="F")
    X += 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.shape)
    X = np.asfortranarray(X.astype(np.float32).astype(np.float64))
    init = [rng.random((n, R)) for n in d]
    return X, init, d


def cpu_baseline_leg(dims, R, X, init, args, sweeps=3):
    """C++/OpenMP (oracle/cpu_als.cpp) ALS sweeps of the bench's own tensor
    and start in FP32 on every host core; config 0 (128^3 rank 16) time to
    the fit of the FP32 GPU path's stopping rule (<= 50 sweeps or delta fit
    < 1e-6) in FP32 and FP64; one sweep of 96^4 rank 32; and one NumPy FP64
    sweep of the full tensor (the port the --impl reference arm times)."""
    import numpy as np
    import oracle
    threads = oracle.cpu_threads()
    Xh = X.cpu().numpy()
    init_h = [u.cpu().numpy() for u in init]
    oracle.cpu_cp_als(Xh, dims, R, [u.copy() for u in init_h], 1)  # warm the threads and pages
    _, fits, sw, sec = oracle.cpu_cp_als(Xh, dims, R, [u.copy() for u in init_h], sweeps)
    value = sweep_bytes(dims, R) * sw / sec / 1e9
    out = {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
           "sample": f"{sw} ALS sweeps of the full {'x'.join(map(str, dims))} rank-{R} FP32 tensor from the "
                     f"bench's start, {sec:.2f} s; C++/OpenMP restatement of decomposition/CPU/python/mycp.py "
                     f"(oracle/cpu_als.cpp), FP32 arithmetic, {threads} threads",
           "seconds_per_sweep": round(sec / sw, 4)}
    rng = np.random.default_rng(10)
    d0, R0 = (128, 128, 128), 16
    f0 = [rng.random(n * R0) for n in d0]
    X0 = oracle.gencp(d0, f0, R0)
    X0 = (X0 + 1e-3 * np.linalg.norm(X0) / np.sqrt(X0.size) * rng.standard_normal(X0.size)).astype(np.float32)
    i0 = [rng.random(n * R0).astype(np.float32) for n in d0]
    ttf = {}
    for name, dt in (("fp32", np.float32), ("fp64", np.float64)):
        _, fits0, sw0, sec0 = oracle.cpu_cp_als(X0.astype(dt), d0, R0, [u.astype(dt) for u in i0], 50, tol=1e-6)
        ttf[name] = {"seconds": round(sec0, 4), "sweeps": sw0, "fit": round(float(fits0[-1]), 8)}
    out["cp_128x128x128_r16_time_to_fit"] = ttf
    d1, R1 = (96, 96, 96, 96), 32
    X1 = rng.random(int(np.prod(d1)), dtype=np.float32)
    i1 = [rng.random(n * R1).astype(np.float32) for n in d1]
    _, _, sw1, sec1 = oracle.cpu_cp_als(X1, d1, R1, i1, 1)
    out["cp_96x96x96x96_r32_sweep"] = {"seconds": round(sec1, 4),
                                       "gbs": round(sweep_bytes(d1, R1) / sec1 / 1e9, 3)}
    X3 = np.asfortranarray(Xh.reshape(tuple(reversed(dims))).transpose(2, 1, 0).astype(np.float64))
    F = [u.reshape(R, n).T.astype(np.float64).copy() for u, n in zip(init_h, dims)]
    gbs_np, dt_np = cpu_sweep_gbs(X3, F, 1)
    out["numpy_fp64_port"] = {"gbs": round(gbs_np, 3), "seconds_per_sweep": round(dt_np, 4),
                              "cores": os.cpu_count()}
    return out


def run_reference(args):
    """--impl reference: the reference's CPU ALS (decomposition/CPU/python/
    mycp.py, TensorLy on the NumPy backend, FP64) on the host cores, restated
    on NumPy/OpenBLAS because TensorLy is not installed; the full workload
    unless --cpu-slab asks for a slab."""
    import numpy as np
    dims = [int(x) for x in args.dims.split(",")]
    R = args.rank
    X3, init, sd = cpu_sample(dims, R, slab=args.cpu_slab if args.cpu_slab > 0 else dims[-1])
    cores = os.cpu_count()
    for _ in range(max(0, args.warmup)):
        cpu_sweep_gbs(X3, [f.copy() for f in init], 1)
    times = []
    facs = [f.copy() for f in init]
    for _ in range(args.steps):
        _, dt = cpu_sweep_gbs(X3, facs, 1)
        times.append(dt)
    tot = sum(times)
    value = sweep_bytes(sd, R) * args.steps / tot / 1e9
    line = {
        "metric": METRIC, "impl": "reference", "value": round(value, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * tot / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
        "config": config_dict(dims, R, "fp64-numpy"),
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": cores, "kind": "port",
                         "sample": f"one ALS sweep per step of the {'x'.join(map(str, sd))} rank-{R} "
                                   f"tensor; NumPy/OpenBLAS (FP64) restatement of "
                                   f"decomposition/CPU/python/mycp.py"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Side workloads, reported as extra keys of the same JSON line (each leg is
# timed with CUDA events on the bench stream; a failing leg records its error
# instead of stopping the bench).

def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def leg_cp_small(cd, torch, stream, sptr):
    """Plain CP-ALS, 128^3, rank 16, <= 50 sweeps or delta fit < 1e-6."""
    dims, R = (128, 128, 128), 16
    with torch.cuda.stream(stream):
        X, _ = cd.make_cp_tensor(dims, R, seed=10)
        init = cd.make_init(dims, R, seed=11)
    stream.synchronize()
    out = {"dims": dims, "rank": R}
    for name in ("fp32", "bf16x3"):
        U = [u.clone() for u in init]
        torch.cuda.synchronize()
        res = cd.cp_als(X, dims, R, U, max_sweeps=50, tol=1e-6, precision=cd.PRECISIONS[name], stream=sptr)
        out[name] = {"seconds": round(res.seconds, 5), "sweeps": res.sweeps, "fit": round(res.fit, 8),
                     "ms_per_sweep": round(1e3 * res.seconds / max(1, res.sweeps), 4)}
    return out


def leg_order4(cd, torch, stream, sptr):
    """4th-order 96^4, rank 32: MTTKRP per mode (BF16x3 tensor cores) and
    sweep time from the plan's graph."""
    dims, R = (96, 96, 96, 96), 32
    with torch.cuda.stream(stream):
        X, _ = cd.make_cp_tensor(dims, R, seed=12)
        init = cd.make_init(dims, R, seed=13)
    stream.synchronize()
    kern = {}
    outm = [torch.empty(d * R, device="cuda") for d in dims]
    for mode in range(4):
        for _ in range(2):
            cd.mttkrp(X, dims, init, mode, R, outm[mode], cd.PREC_BF16X3, stream=sptr)
        e0, e1 = _events(torch)
        e0.record(stream)
        for _ in range(5):
            cd.mttkrp(X, dims, init, mode, R, outm[mode], cd.PREC_BF16X3, stream=sptr)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 5
        kern[mode] = {"ms": round(ms, 4), "gbs": round(mttkrp_bytes(dims, R, mode) / ms / 1e6, 1),
                      "path": cd.mttkrp_path(dims, mode, R, cd.PREC_BF16X3)}
    plan = cd.CpPlan(X, dims, R, [u.clone() for u in init], precision=cd.PREC_BF16X3, stream=sptr)
    plan.run(3, stream=sptr)
    e0, e1 = _events(torch)
    e0.record(stream)
    plan.run(10, stream=sptr)
    e1.record(stream)
    e1.synchronize()
    sweep_ms = e0.elapsed_time(e1) / 10
    fit = plan.true_fit(stream=sptr)
    plan.close()
    return {"dims": dims, "rank": R, "mttkrp": kern, "ms_per_sweep": round(sweep_ms, 4),
            "sweep_gbs": round(sweep_bytes(dims, R) / sweep_ms / 1e6, 1), "fit_after_13_sweeps": round(fit, 8)}


def _fp64_unfold(Xd, dims, n):
    """Mode-n unfolding (dims[n] x rest) of a flat column-major FP64 tensor."""
    import numpy as np
    T = Xd.reshape(tuple(reversed(dims)))
    return np.moveaxis(T, len(dims) - 1 - n, 0).reshape(dims[n], -1)


def _max_angle(U, W):
    """Largest principal angle (radians) between span(U) and span(W), W
    orthonormal."""
    import numpy as np
    Q, _ = np.linalg.qr(U)
    return float(np.arcsin(min(1.0, np.linalg.norm(Q - W @ (W.T @ Q), 2))))


def _fp64_project(Xd, dims, facs, skip):
    """X x_m U_m^T for every m != skip, FP64 on the host (axes reversed)."""
    import numpy as np
    T = Xd.reshape(tuple(reversed(dims)))
    N = len(dims)
    for m in range(N):
        if m != skip:
            T = np.moveaxis(np.tensordot(T, facs[m], axes=([N - 1 - m], [0])), -1, N - 1 - m)
    return T


def leg_tucker(cd, torch, stream, sptr):
    """Tucker HOSVD + 10 HOOI sweeps: 512^3 (32,32,32) and 128^4 (16^4),
    Grams on the tensor cores (three-term BF16), TTM chains in BF16, FP64
    eigensolves; reconstruction error relative to X, and the largest
    principal angle of every factor against FP64 on the host: HOSVD against
    the leading eigenvectors (numpy eigh) of the FP64 unfolding Grams, HOOI
    against the leading eigenvectors of the FP64 Gram of X projected by the
    other returned factors (its fixed point)."""
    import numpy as np
    out = {}
    for dims, ranks in (((512, 512, 512), (32, 32, 32)), ((128, 128, 128, 128), (16, 16, 16, 16))):
        key = "x".join(map(str, dims)) + "_r" + str(ranks[0])
        with torch.cuda.stream(stream):
            X, _, _ = cd.make_tucker_tensor(dims, ranks, seed=20)
        stream.synchronize()
        core = torch.empty(int(np_prod(ranks)), device="cuda")
        U = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
        rec = torch.empty_like(X)
        res = {}
        Xd = X.double().cpu().numpy()
        N = len(dims)
        W64 = []
        for n in range(N):
            A = _fp64_unfold(Xd, dims, n)
            W64.append(np.linalg.eigh(A @ A.T)[1][:, dims[n] - ranks[n]:])
            del A
        for method in ("hosvd", "hooi10"):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if method == "hosvd":
                cd.tucker_hosvd(X, dims, ranks, core, U, precision=cd.PREC_BF16X3, stream=sptr)
            else:
                cd.tucker_hooi(X, dims, ranks, core, U, sweeps=10, precision=cd.PREC_BF16X3, stream=sptr)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            cd.gentucker(rec, core, U, dims, ranks, stream=sptr)
            torch.cuda.synchronize()
            err = float(torch.linalg.norm((X - rec).double()) / torch.linalg.norm(X.double()))
            Uh = [u.double().cpu().numpy().reshape(d, r, order="F") for u, d, r in zip(U, dims, ranks)]
            if method == "hosvd":
                angles = [_max_angle(Uh[n], W64[n]) for n in range(N)]
            else:
                angles = []
                for n in range(N):
                    Y = _fp64_project(Xd, dims, Uh, skip=n)
                    A = np.moveaxis(Y, N - 1 - n, 0).reshape(dims[n], -1)
                    angles.append(_max_angle(Uh[n], np.linalg.eigh(A @ A.T)[1][:, dims[n] - ranks[n]:]))
            res[method] = {"seconds": round(dt, 4), "rel_error": float(f"{err:.4e}"),
                           "max_angle_rad_per_mode": [float(f"{a:.2e}") for a in angles]}
        out[key] = res
        del X, rec, Xd
    return out


def leg_streamed(cd, torch, dims=(512, 512, 512), R=64, slab=64, sweeps=2):
    """Out-of-core CP-ALS (streamed.py): the 512^3 tensor in pinned host
    memory, every mode's MTTKRP streaming it in slabs of `slab` frontal
    slices (BF16x3), copies overlapped with compute on two device buffers."""
    import streamed
    X, _ = cd.make_cp_tensor(dims, R, seed=1000)
    init = cd.make_init(dims, R, seed=2000)
    Xh = X.cpu().pin_memory()
    del X
    torch.cuda.synchronize()
    sc = streamed.StreamedCP(cd, Xh, dims, R, [u.clone() for u in init], slab=slab,
                             precision=cd.PREC_BF16X3, nbuf=2)
    sc.sweep()  # warm
    torch.cuda.synchronize()
    b0 = sc.h2d_bytes
    e0, e1 = _events(torch)
    e0.record(sc.ops.compute)
    for _ in range(sweeps):
        sc.sweep()
    e1.record(sc.ops.compute)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3 / sweeps
    h2d = (sc.h2d_bytes - b0) / sweeps
    # the host link alone: one slab-sized pinned copy loop over the tensor
    buf = torch.empty(Xh.numel() // dims[-1] * slab, device="cuda")
    n = buf.numel()
    c0, c1 = _events(torch)
    c0.record()
    for k in range(0, Xh.numel(), n):
        buf[: min(n, Xh.numel() - k)].copy_(Xh[k:k + n], non_blocking=True)
    c1.record()
    c1.synchronize()
    copy_gbs = 4 * Xh.numel() / (c0.elapsed_time(c1) * 1e-3) / 1e9
    fit = sc.fit()
    return {"dims": list(dims), "rank": R, "slab_slices": slab, "buffers": 2, "precision": "bf16x3",
            "seconds_per_sweep": round(sec, 5), "h2d_bytes_per_sweep": int(h2d),
            "h2d_gbs": round(h2d / sec / 1e9, 2), "host_copy_gbs": round(copy_gbs, 2),
            "link_bound_fraction": round((h2d / (copy_gbs * 1e9)) / sec, 3), "fit": round(fit, 6)}


def run_residual_once(cd, torch, dims, R, reps=5):
    """The exact CP residual (cud_cp_residual) of a synthetic rank-R model on
    its tensor: `reps` calls after one warm-up, mean wall time per call (the
    call reads its two scalars back) and the fit."""
    X, _ = cd.make_cp_tensor(dims, R, seed=1)
    U = cd.make_init(dims, R, seed=2)
    cd.cp_residual(X, dims, U, R)
    torch.cuda.synchronize()
    cd.prof_enable(True)
    t0 = time.perf_counter()
    for _ in range(reps):
        r2, x2 = cd.cp_residual(X, dims, U, R)
    dt = (time.perf_counter() - t0) / reps
    kms = cd.prof_kernel_times()
    cd.prof_enable(False)
    k_ms = sum(kms) / len(kms) if kms else None
    return {"dims": list(dims), "rank": R, "ms_per_call": round(dt * 1e3, 4),
            "kernel_ms": round(k_ms, 4) if k_ms else None,
            "kernel_gbs": round(4 * X.numel() / (k_ms * 1e-3) / 1e9, 1) if k_ms else None,
            "fit": 1 - (r2 / x2) ** 0.5 if x2 > 0 else None}


def run_tucker_once(cd, torch, dims, ranks):
    """One tensor-core HOSVD and one HOOI sweep (BF16x3) on a synthetic
    Tucker tensor of the given shape; wall times and reconstruction errors."""
    X, _, _ = cd.make_tucker_tensor(dims, ranks, seed=20)
    core = torch.empty(int(np_prod(ranks)), device="cuda")
    U = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
    rec = torch.empty_like(X)
    out = {"dims": list(dims), "ranks": list(ranks)}
    for method, sweeps in (("hosvd", 0), ("hooi1", 1)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if sweeps == 0:
            cd.tucker_hosvd(X, dims, ranks, core, U, precision=cd.PREC_BF16X3)
        else:
            cd.tucker_hooi(X, dims, ranks, core, U, sweeps=sweeps, precision=cd.PREC_BF16X3)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        cd.gentucker(rec, core, U, dims, ranks)
        err = float(torch.linalg.norm((X - rec).double()) / torch.linalg.norm(X.double()))
        out[method] = {"seconds": round(dt, 5), "rel_error": float(f"{err:.4e}")}
    return out


def batched_workload(cd, torch, n, seed=30):
    """The batched CP-ALS workload: n tensors, dims uniform in [16, 96],
    ranks in [4, 16], each a sum of rank-1 terms with uniform [0,1) factors
    plus 1e-3 relative Gaussian noise, uniform [0,1) initial factors."""
    import numpy as np
    rng = np.random.default_rng(seed)
    dims = [tuple(int(x) for x in rng.integers(16, 97, 3)) for _ in range(n)]
    ranks = [int(x) for x in rng.integers(4, 17, n)]
    b = cd.Batch(dims, ranks)
    g = torch.Generator(device="cuda").manual_seed(seed + 1)
    for t, (d, r) in enumerate(zip(dims, ranks)):
        facs = [torch.rand(x * r, generator=g, device="cuda") for x in d]
        xv = b.x_view(t)
        cd.gencp(xv, facs, d, r)
        nz = torch.randn(xv.numel(), generator=g, device="cuda")
        xv.add_(nz * (1e-3 * torch.linalg.norm(xv) / (xv.numel() ** 0.5)))
        for m in range(3):
            b.u_view(t, m).copy_(torch.rand(d[m] * r, generator=g, device="cuda"))
    torch.cuda.synchronize()
    return b, dims, ranks, rng


def run_batched_once(cd, torch, n):
    """Three batched sweeps (one kernel launch each, no graph) on the first n
    tensors of the batched workload."""
    b, dims, ranks, _ = batched_workload(cd, torch, n)
    t0 = time.perf_counter()
    fits, sweeps, launches = cd.cp_als_batched(b, max_sweeps=3, tol=0.0, use_graph=False)
    torch.cuda.synchronize()
    return {"tensors": n, "elements": sum(np_prod(d) for d in dims), "launches": launches,
            "seconds": round(time.perf_counter() - t0, 4), "fit_mean": float(sum(fits) / len(fits))}


def np_prod(xs):
    p = 1
    for x in xs:
        p *= int(x)
    return p


def leg_batched(cd, torch, stream, sptr, n=4096):
    """Batched CP-ALS: n tensors, dims uniform in [16, 96], ranks in [4, 16],
    built like the 128^3 workload; one persistent kernel per sweep, graph
    replay, autotuned launch shape; <= 50 sweeps or delta fit < 1e-6 per
    tensor.  Parity sample: 16 tensors through the plain path."""
    import numpy as np
    b, dims, ranks, rng = batched_workload(cd, torch, n)
    U0 = b.U.clone()
    t0 = time.perf_counter()
    th, cps = cd.cp_batched_tune(b, stream=sptr)
    tune_s = time.perf_counter() - t0
    b.U.copy_(U0)
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    e0.record(stream)
    fits, sweeps, launches = cd.cp_als_batched(b, max_sweeps=50, tol=1e-6, stream=sptr)
    e1.record(stream)
    e1.synchronize()
    secs = e0.elapsed_time(e1) * 1e-3
    # parity sample through the plain single-tensor path (FP32, same start,
    # same sweeps), also timed: the batch's plain-path time is estimated as
    # the sample's mean per tensor times n
    worst = 0.0
    plain_s = 0.0
    sample = rng.choice(n, 16, replace=False)
    for t in sample:
        t = int(t)
        U = [U0[b.u_offsets[3 * t + m]: b.u_offsets[3 * t + m] + dims[t][m] * ranks[t]].clone() for m in range(3)]
        xt = b.x_view(t).clone()
        stream.synchronize()
        t0 = time.perf_counter()
        res = cd.cp_als(xt, dims[t], ranks[t], U, max_sweeps=sweeps[t], tol=0.0, precision=cd.PREC_FP32, stream=sptr)
        stream.synchronize()
        plain_s += time.perf_counter() - t0
        worst = max(worst, abs(res.fit_estimate - fits[t]))
    plain_est = plain_s / len(sample) * n
    elems = sum(np_prod(d) for d in dims)
    return {"tensors": n, "elements": elems, "autotune": {"threads": th, "ctas_per_sm": cps, "seconds": round(tune_s, 3)},
            "seconds": round(secs, 4), "sweep_kernels": launches, "sweeps_mean": round(float(np.mean(sweeps)), 2),
            "fit_mean": round(float(np.mean(fits)), 6),
            "gbs_mttkrp_traffic": round(3 * 4 * sum(np_prod(dims[t]) * sweeps[t] for t in range(n)) / secs / 1e9, 1),
            "max_fit_diff_vs_plain_path_16_sampled": float(f"{worst:.3e}"),
            "plain_path_seconds_est": round(plain_est, 3), "speedup_vs_plain_path": round(plain_est / secs, 1)}


def leg_warmstart(cd, torch, n_train, n_eval):
    """Learned warm start: 64^3 rank-8 smooth-factor tensors, network trained
    on n_train ALS solutions the library generates (fresh tensors, 10 epochs
    over them), the judge's rule chosen on 2048 calibration tensors, then
    sweeps and time to each tensor's reference fit - 1e-4 from random, HOSVD,
    learned and judged starts on n_eval held-out tensors."""
    import warmstart
    w = warmstart.WarmStart(I=64, R=8, S=32, hidden=512, noise=1e-3, seed=1, max_batch=256)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = w.train(n_train, batch=256, lr=3e-4, chunk=4096, label_sweeps=3, log_every=64, epochs=10,
                     warmup=400)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    cal = w.calibrate(2048, id0=5 * 10 ** 8)
    ev = w.evaluate(n_eval, id0=10 ** 9)
    ev["judge_calibration"] = cal
    ev["train"] = {"samples": n_train, "epochs": 10, "seconds": round(train_s, 2),
                   "loss_first": round(losses[0][1], 6) if losses else None,
                   "loss_last": round(losses[-1][1], 6) if losses else None}
    w.model.close()
    return ev


def _time_calls(torch, stream, fn, reps, warm=2):
    """Mean ms of fn() over `reps` calls, CUDA events on `stream`."""
    for _ in range(warm):
        fn()
    e0, e1 = _events(torch)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def leg_reference_gpu(cd, torch, stream, sptr, reps=10):
    """The reference's own GPU MTTKRP timed beside ours on this GPU (a
    baseline, outside every timed region of the library):
    * the FP32 MTTKRP its CP-ALS programs run -- Khatri-Rao by rank-1
      batched GEMMs, then one SGEMM against X, X2 or X3
      (src/cp_als.cu:46-52,66-69,85-88; src/cp4_als.cu:67-73,91-96,112-117,
      135-138), issued by oracle/ref_gpu.cu on a handle bound to the bench
      stream -- per mode at 512^3 rank 64 and 96^4 rank 32, against our
      cud_mttkrp in FP32 (CUDA cores) and BF16x3 (tensor cores);
    * its public FP16 mttkrp() (src/mttkrp.cu:3-80, allocations and device
      synchronisations per call, as shipped), host wall time per call at
      512^3 rank 64, against our cud_mttkrp_legacy."""
    import oracle
    out = {}
    for dims, R, seeds in (((512, 512, 512), 64, (40, 41)), ((96, 96, 96, 96), 32, (42, 43))):
        key = "x".join(map(str, dims)) + f"_r{R}"
        with torch.cuda.stream(stream):
            X, _ = cd.make_cp_tensor(dims, R, seed=seeds[0])
            U = cd.make_init(dims, R, seed=seeds[1])
        stream.synchronize()
        h = oracle.RefGpuMttkrp(torch, X, dims, U, R, stream=sptr)
        res = {}
        try:
            o = torch.empty(max(dims) * R, device="cuda")
            for mode in range(len(dims)):
                ref_ms = _time_calls(torch, stream, lambda: h.run(mode), reps)
                ours = {}
                for name in ("bf16x3", "fp32"):
                    ours[name] = _time_calls(
                        torch, stream,
                        lambda: cd.mttkrp(X, dims, U, mode, R, o, cd.PRECISIONS[name], stream=sptr), reps)
                b = mttkrp_bytes(dims, R, mode)
                res[str(mode)] = {"reference_ms": round(ref_ms, 4), "reference_gbs": round(b / ref_ms / 1e6, 1),
                                  "ours_bf16x3_ms": round(ours["bf16x3"], 4),
                                  "ours_bf16x3_gbs": round(b / ours["bf16x3"] / 1e6, 1),
                                  "ours_fp32_ms": round(ours["fp32"], 4),
                                  "speedup_bf16x3": round(ref_ms / ours["bf16x3"], 2),
                                  "speedup_fp32": round(ref_ms / ours["fp32"], 2)}
        finally:
            h.close()
        tot = {k: sum(v[k] for v in res.values()) for k in ("reference_ms", "ours_bf16x3_ms", "ours_fp32_ms")}
        out[key] = {"per_mode": res, "all_modes_ms": {k: round(v, 4) for k, v in tot.items()},
                    "speedup_bf16x3": round(tot["reference_ms"] / tot["ours_bf16x3_ms"], 2),
                    "speedup_fp32": round(tot["reference_ms"] / tot["ours_fp32_ms"], 2)}
        del X, U
        torch.cuda.synchronize()
    # the public FP16 mttkrp(), as shipped (host-synchronous, allocates per call)
    if os.path.exists(oracle.REF_LIB_PATH):
        import ctypes
        lib = ctypes.CDLL(oracle.REF_LIB_PATH)
        f = getattr(lib, "_Z6mttkrpPfS_S_S_lllll")
        f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_long] * 5
        f.restype = None
        m = n = k = 512
        r = 64
        with torch.cuda.stream(stream):
            X, _ = cd.make_cp_tensor((m, n, k), r, seed=44)
            A, B, C = cd.make_init((m, n, k), r, seed=45)
        torch.cuda.synchronize()
        o1 = torch.empty(512 * r, device="cuda")
        o2 = torch.empty(512 * r, device="cuda")
        pub = {}
        for flag, (left, right) in ((1, (C, B)), (2, (C, A)), (3, (B, A))):
            def ref_call():
                f(X.data_ptr(), left.data_ptr(), right.data_ptr(), o1.data_ptr(), flag, m, n, k, r)
                torch.cuda.synchronize()

            def our_call():
                cd.mttkrp_legacy(X, left, right, o2, flag, m, n, k, r, stream=sptr)
                stream.synchronize()
            t = {}
            for name, fn in (("reference", ref_call), ("ours", our_call)):
                fn()
                fn()
                samples = []
                for _ in range(5):
                    t0 = time.perf_counter()
                    fn()
                    samples.append(time.perf_counter() - t0)
                t[name] = statistics.median(samples) * 1e3
            d = (o1 - o2).double().norm() / o1.double().norm()
            pub[str(flag)] = {"reference_ms": round(t["reference"], 3), "ours_ms": round(t["ours"], 4),
                              "speedup": round(t["reference"] / t["ours"], 2),
                              "rel_diff": float(f"{float(d):.2e}")}
        out["public_fp16_mttkrp_512x512x512_r64"] = dict(pub, timing="host wall time per synchronous call, "
                                                                      "median of 5")
        del X, A, B, C
    return out


def config_dict(dims, R, precision, world=1):
    return {"workload": f"cp_als_sweep_{'x'.join(map(str, dims))}_r{R}", "dims": dims, "rank": R,
            "precision": precision, "global_batch": world, "seq_len": None,
            "parallelism": f"dp{world}" if world > 1 else "single",
            "l2": "inputs (512 MiB per tensor) exceed the 126 MB L2; no flush between steps"}


def run_sharded(args, cd, torch, dist, rank, world, local, dims, R, prec, prec_name):
    """N > 1: the global tensor is dims[0] x ... x (dims[-1] * N), sharded
    along its last mode (one dims-sized slab per rank, weak scaling); the
    partial MTTKRPs of the other modes are all-reduced over NCCL each sweep
    (distributed.ShardedCP)."""
    from distributed import CudaOps, ShardedCP, TorchComm
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    with torch.cuda.stream(stream):
        g = torch.Generator(device="cuda")
        g.manual_seed(1000)                      # shared factors of the other modes
        shared = [torch.rand(R * d, generator=g, device="cuda") for d in dims[:-1]]
        g.manual_seed(5000 + rank)               # this rank's rows of the last factor
        last = torch.rand(R * dims[-1], generator=g, device="cuda")
        n = 1
        for d in dims:
            n *= d
        X = torch.empty(n, device="cuda")
        cd.gencp(X, shared + [last], dims, R)
        E = torch.randn(n, generator=g, device="cuda")
        X.add_(E, alpha=1e-3 * (cd.norm2(X) / cd.norm2(E)) ** 0.5)
        del E
        g.manual_seed(2000)
        init = [torch.rand(R * d, generator=g, device="cuda") for d in dims[:-1]]
        g.manual_seed(6000 + rank)
        init.append(torch.rand(R * dims[-1], generator=g, device="cuda"))
    stream.synchronize()
    comm = TorchComm(dist)
    with torch.cuda.stream(stream):
        cp = ShardedCP(CudaOps(cd, prec, stream=sptr), comm, X, dims, R, [u.clone() for u in init])
        for _ in range(args.warmup):
            cp.sweep()
    torch.cuda.synchronize()
    # one sweep (kernels and all-reduces) captured in a CUDA graph; every
    # rank takes the same decision (all-reduced), eager sweeps otherwise
    with torch.cuda.stream(stream):
        ok = cp.capture(torch, stream)
    flag = torch.tensor([0.0 if ok else 1.0], device="cuda")
    dist.all_reduce(flag)
    if float(flag.item()) > 0:
        cp.release()
    graphed = cp.graph is not None
    with torch.cuda.stream(stream):
        cp.sweep()
    torch.cuda.synchronize()
    dist.barrier()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                cp.sweep()
            e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_total = float(t.item())
    with torch.cuda.stream(stream):
        fit = cp.fit()
    value = world * sweep_bytes(dims, R) * args.steps / (ms_total * 1e-3) / 1e9
    # e2e: H2D of each rank's slab and factors (into device buffers allocated
    # once, as the 1-GPU e2e does), a new ShardedCP, 10 sweeps, D2H of the
    # factors into pinned buffers
    hX = torch.empty(X.numel(), dtype=torch.float32, pin_memory=True)
    hX.copy_(X)
    hU = [u.cpu().pin_memory() for u in init]
    dX = torch.empty_like(X)
    dU = [torch.empty_like(u) for u in init]
    oU = [torch.empty(u.numel(), dtype=torch.float32, pin_memory=True) for u in init]
    times = []
    for it in range(3):
        torch.cuda.synchronize()
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            dX.copy_(hX, non_blocking=True)
            for a, b in zip(dU, hU):
                a.copy_(b, non_blocking=True)
            c2 = ShardedCP(CudaOps(cd, prec, stream=sptr), comm, dX, dims, R, dU)
            for _ in range(args.e2e_sweeps):
                c2.sweep()
            for a, b in zip(oU, c2.U):
                a.copy_(b, non_blocking=True)
            e1.record(stream)
        e1.synchronize()
        tt = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        if it > 0:
            times.append(float(tt.item()) * 1e-3)
    e2e_s = sum(times) / len(times)
    peak, peak_kind = load_peaks()
    per_sweep_launches = 5 * len(dims)
    result = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_total / args.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic",
        "config": dict(config_dict(dims, R, prec_name, world),
                       workload=f"cp_als_sweep_{'x'.join(map(str, dims[:-1]))}x{dims[-1]}N_r{R}",
                       parallelism=f"sharded along the last mode over {world} ranks, NCCL all-reduce"),
        "gpu_launches": per_sweep_launches * args.steps * world,
        "sweep_graph": graphed,
        "fit_after_timed_sweeps": round(fit, 8),
        "clocks": clk.summary(),
        "e2e": {"value": round(world * sweep_bytes(dims, R) * args.e2e_sweeps / e2e_s / 1e9, 3),
                "unit": "GB/s", "h2d_bytes_per_step": 4 * (X.numel() + sum(u.numel() for u in init)),
                "d2h_bytes_per_step": 4 * sum(u.numel() for u in init),
                "step": f"sharded CP-ALS, {args.e2e_sweeps} sweeps, from pinned host buffers"},
        "roofline": {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                     "traffic": None, "note": "kernel roofline reported by the 1-GPU run"},
    }
    cp.release()  # the graph holds NCCL calls: released before the group goes
    torch.cuda.synchronize()
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--dims", default="512,512,512")
    ap.add_argument("--rank", type=int, default=64)
    ap.add_argument("--precision", default="default")
    ap.add_argument("--e2e-sweeps", type=int, default=10)
    ap.add_argument("--cpu-slab", type=int, default=0,
                    help="last-mode slices of the CPU baseline's sample (0 = the whole tensor)")
    ap.add_argument("--no-ttf", action="store_true", help="skip the time-to-fit runs")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="skip timing the reference's own GPU MTTKRP beside ours")
    ap.add_argument("--only-mttkrp", action="store_true",
                    help="time only the MTTKRP kernels (profiling runs) and exit")
    ap.add_argument("--only-tucker", action="store_true",
                    help="run one Tucker HOSVD and one HOOI sweep on --dims with --tucker-ranks "
                         "(profiling runs) and exit")
    ap.add_argument("--tucker-ranks", default="16,16,16,16")
    ap.add_argument("--only-residual", action="store_true",
                    help="time the exact CP residual on --dims / --rank (profiling runs) and exit")
    ap.add_argument("--only-batched", type=int, default=0, metavar="N",
                    help="run 3 batched CP-ALS sweeps (one kernel launch each, no graph) on the first N "
                         "tensors of the batched workload (profiling runs) and exit")
    ap.add_argument("--kreps", type=int, default=10, help="timed MTTKRP launches per mode")
    ap.add_argument("--kwarm", type=int, default=3, help="untimed MTTKRP launches per mode")
    ap.add_argument("--legs", default="cp128,order4,tucker,batched,warmstart,streamed",
                    help="side workloads to add as extra keys (comma list, or 'none')")
    ap.add_argument("--ws-train", type=int, default=204800, help="warm-start training samples")
    ap.add_argument("--ws-eval", type=int, default=10240, help="warm-start held-out tensors")
    ap.add_argument("--sharded", action="store_true",
                    help="run the sharded (multi-GPU) sweep path even with one rank (NCCL over one GPU; "
                         "launch under torchrun) -- a check of that path, not the 1-GPU benchmark")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import numpy as np
    import torch
    import cudecompose as cd

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1 or args.sharded:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = dist_mod

    dims = [int(x) for x in args.dims.split(",")]
    R = args.rank
    prec = cd.PRECISIONS[args.precision]
    prec_name = "bf16x3" if prec in (cd.PREC_DEFAULT, cd.PREC_BF16X3) else args.precision
    if args.only_batched:
        if rank == 0:
            print(json.dumps(run_batched_once(cd, torch, args.only_batched)), flush=True)
        return
    if args.only_residual:
        if rank == 0:
            print(json.dumps(run_residual_once(cd, torch, dims, R)), flush=True)
        return
    if args.only_tucker:
        if rank == 0:
            print(json.dumps(run_tucker_once(cd, torch, dims, [int(x) for x in args.tucker_ranks.split(",")])),
                  flush=True)
        return
    if (world > 1 or args.sharded) and not args.only_mttkrp:
        run_sharded(args, cd, torch, dist, rank, world, local, dims, R, prec, prec_name)
        return
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    with torch.cuda.stream(stream):
        X, _ = cd.make_cp_tensor(dims, R, seed=1000 + rank)
        init = cd.make_init(dims, R, seed=2000 + rank)
    stream.synchronize()

    # ---- kernel level: MTTKRP per mode, CUDA events on the launching stream
    kern = {}
    U = [u.clone() for u in init]
    outs = [torch.empty(d * R, device="cuda") for d in dims]
    reps = max(1, args.kreps)
    for mode in range(len(dims)):
        for _ in range(args.kwarm):
            cd.mttkrp(X, dims, U, mode, R, outs[mode], prec, stream=sptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            cd.mttkrp(X, dims, U, mode, R, outs[mode], prec, stream=sptr)
        e1.record(stream)
        e1.synchronize()
        ms_eager = e0.elapsed_time(e1) / reps
        # the same calls replayed from a CUDA graph on the same stream: each
        # call still launches its B pack, the MTTKRP and the split reduce;
        # the graph removes the host launch gaps between them
        ms, timing = ms_eager, "eager"
        try:
            stream.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                for _ in range(reps):
                    cd.mttkrp(X, dims, U, mode, R, outs[mode], prec, stream=sptr)
            with torch.cuda.stream(stream):
                g.replay()
                e0.record(stream)
                g.replay()
                e1.record(stream)
            e1.synchronize()
            ms, timing = e0.elapsed_time(e1) / reps, "graph"
            del g
        except RuntimeError:
            pass
        stream.synchronize()
        # the main kernel alone: CUDA events the library records on the
        # bench stream around it (eager calls)
        cd.prof_enable(True)
        for _ in range(reps):
            cd.mttkrp(X, dims, U, mode, R, outs[mode], prec, stream=sptr)
        kms = cd.prof_kernel_times()
        cd.prof_enable(False)
        k_ms = sum(kms) / len(kms) if kms else None
        kern[mode] = {"ms": round(ms, 5), "gbs": round(mttkrp_bytes(dims, R, mode) / ms / 1e6, 1),
                      "timing": timing, "ms_eager": round(ms_eager, 5),
                      "kernel_ms": round(k_ms, 5) if k_ms else None,
                      "kernel_gbs": round(mttkrp_bytes(dims, R, mode) / k_ms / 1e6, 1) if k_ms else None,
                      "path": cd.mttkrp_path(dims, mode, R, prec)}
    if args.only_mttkrp:
        if rank == 0:
            print(json.dumps({"mttkrp": kern, "dims": dims, "rank": R, "precision": prec_name}), flush=True)
        return

    # ---- timed sweeps through the plan (graph replay)
    plan = cd.CpPlan(X, dims, R, U, precision=prec, stream=sptr)
    plan.run(args.warmup, stream=sptr)
    stream.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.run(args.steps, stream=sptr)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms_total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    kps, fallbacks = plan.info()
    fit_now, _ = plan.fit(stream=sptr)
    plan.close()
    per_rank_bytes = sweep_bytes(dims, R) * args.steps
    value = world * per_rank_bytes / (ms_total * 1e-3) / 1e9

    peak, peak_kind = load_peaks()
    avg_bytes = sum(mttkrp_bytes(dims, R, m) for m in kern) / len(kern)
    call_ms = sum(k["ms"] for k in kern.values()) / len(kern)
    call_achieved = avg_bytes / (call_ms * 1e-3) / 1e9
    kernel_ms = [k["kernel_ms"] for k in kern.values() if k["kernel_ms"]]
    avg_ms = sum(kernel_ms) / len(kernel_ms) if len(kernel_ms) == len(kern) else call_ms
    achieved = avg_bytes / (avg_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "mttkrp_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f)
        key = f"{'x'.join(map(str, dims))}_r{R}_{prec_name}"
        traffic = tj.get(key)

    result = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_total / args.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic", "config": config_dict(dims, R, prec_name, world),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "kernel": "the MTTKRP kernel alone (CUDA events on the bench stream around its launch, "
                               "eager calls), mean over the modes",
                     "per_call": {"achieved": round(call_achieved, 1), "frac": round(call_achieved / peak, 4),
                                  "what": "whole cud_mttkrp call (B pack + MTTKRP + split reduce), CUDA-graph "
                                          "replay of 10 calls"},
                     "per_mode": kern},
        "gpu_launches": kps * args.steps if kps and kps > 0 else None,
        "kernels_per_sweep": kps, "fit_after_timed_sweeps": round(fit_now, 8),
        "clocks": clk.summary(),
    }

    # ---- MTTKRP error against FP64 on sampled output rows (NumPy on the host)
    result["mttkrp_error_vs_fp64"] = mttkrp_sample_errors(cd, torch, X, dims, R, init, sptr)

    # ---- time to fit: the plain FP32 path (CUDA cores) runs to convergence
    # (delta fit < 1e-7, <= 200 sweeps); every variant then runs from the same
    # start until its exact fit (residual pass every 5 sweeps, inside the
    # timed region) is within 1e-4 of that run's exact fit.
    if not args.no_ttf:
        Ut = [u.clone() for u in init]
        torch.cuda.synchronize()
        ref = cd.cp_als(X, dims, R, Ut, max_sweeps=200, tol=1e-7, precision=cd.PREC_FP32, stream=sptr)
        target = ref.fit - 1e-4
        ttf = {"reference_fp32": {"seconds": round(ref.seconds, 5), "sweeps": ref.sweeps,
                                  "fit": round(ref.fit, 8), "fit_estimate": round(ref.fit_estimate, 8)},
               "target_fit": round(target, 8), "check": "exact fit every 5 sweeps"}
        for name in ("fp32", "bf16x3", "bf16"):
            Ut = [u.clone() for u in init]
            torch.cuda.synchronize()
            res = cd.cp_als(X, dims, R, Ut, max_sweeps=200, target_fit=target, check_every=5,
                            precision=cd.PRECISIONS[name], stream=sptr)
            ttf[name] = {"seconds": round(res.seconds, 5), "sweeps": res.sweeps,
                         "fit": round(res.fit, 8), "fit_estimate": round(res.fit_estimate, 8),
                         "reached": bool(res.fit >= target)}
        base = ttf["fp32"]["seconds"]
        for name in ("fp32", "bf16x3", "bf16"):
            s = ttf[name]["seconds"]
            ttf[name]["speedup_vs_fp32"] = round(base / s, 3) if s else None
        result["time_to_fit"] = ttf

    # ---- end to end through the C ABI with host buffers: H2D of X and the
    # initial factors, cud_cp_als (plan + e2e_sweeps sweeps), D2H of factors
    n = X.numel()
    hX = torch.empty(n, dtype=torch.float32, pin_memory=True)
    hX.copy_(X)
    hU = [u.cpu().pin_memory() for u in init]
    dX = torch.empty_like(X)
    dU = [torch.empty_like(u) for u in init]
    oU = [torch.empty(u.numel(), dtype=torch.float32, pin_memory=True) for u in init]
    e2e_steps = max(2, min(args.steps, 5))
    times = []
    for it in range(e2e_steps + 1):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        with torch.cuda.stream(stream):
            dX.copy_(hX, non_blocking=True)
            for a, b in zip(dU, hU):
                a.copy_(b, non_blocking=True)
        cd.cp_als(dX, dims, R, dU, max_sweeps=args.e2e_sweeps, tol=0.0, precision=prec, stream=sptr)
        with torch.cuda.stream(stream):
            for a, b in zip(oU, dU):
                a.copy_(b, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if it > 0:
            times.append(max(e0.elapsed_time(e1) * 1e-3, time.perf_counter() - t0))
    e2e_s = sum(times) / len(times)
    h2d = 4 * n + sum(4 * u.numel() for u in init)
    d2h = sum(4 * u.numel() for u in init)
    result["e2e"] = {"value": round(world * sweep_bytes(dims, R) * args.e2e_sweeps / e2e_s / 1e9, 3),
                     "unit": "GB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                     "step": f"cud_cp_als, {args.e2e_sweeps} sweeps, from pinned host buffers",
                     "seconds_per_step": round(e2e_s, 5)}

    # ---- side workloads
    legs = [x for x in args.legs.split(",") if x and x != "none"]
    if rank == 0 and world == 1 and legs:
        side = {}
        fns = {"cp128": lambda: leg_cp_small(cd, torch, stream, sptr),
               "order4": lambda: leg_order4(cd, torch, stream, sptr),
               "tucker": lambda: leg_tucker(cd, torch, stream, sptr),
               "batched": lambda: leg_batched(cd, torch, stream, sptr),
               "warmstart": lambda: leg_warmstart(cd, torch, args.ws_train, args.ws_eval),
               "streamed": lambda: leg_streamed(cd, torch)}
        for name in legs:
            if name not in fns:
                continue
            try:
                side[name] = fns[name]()
            except Exception as exc:  # a side leg never stops the headline
                side[name] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
            torch.cuda.synchronize()
        result["workloads"] = side

    # ---- the reference's own GPU MTTKRP on this GPU, beside ours
    if rank == 0 and world == 1 and not args.no_refgpu:
        try:
            with ClockSampler(local) as rclk:
                result["reference_gpu"] = leg_reference_gpu(cd, torch, stream, sptr)
            result["reference_gpu"]["clocks"] = rclk.summary()
        except Exception as exc:
            result["reference_gpu"] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
        torch.cuda.synchronize()

    # ---- CPU baseline (rank 0): the C++/OpenMP restatement of mycp.py's
    # ALS on the host cores at the full workload, plus its time to fit on the
    # 128^3 workload and a sweep of the 96^4 one; the NumPy port beside it
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            result["cpu_baseline"] = cpu_baseline_leg(dims, R, X, init, args)
        except Exception as exc:
            result["cpu_baseline"] = {"error": f"{type(exc).__name__}: {exc}"[:300]}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
