"""Python mirror of the cudecompose API over the library's C ABI.

The reference (891922758/first-project) is a cuBLAS-like C++ library
(inc/cudecompose.h): every routine takes device pointers and extents.  This
module exposes the same routines by the same names for PyTorch CUDA tensors
(column-major data is passed as flat or Fortran-ordered tensors), calling the
in-tree shared library `libcudecompose_b200.so` through ctypes.  There is no
fallback: if the library is missing or fails to load, importing this module
raises.

Conventions: tensors are column-major (mode 1 fastest).  A torch tensor that
represents an I x J x K tensor is stored as a flat float32 buffer of I*J*K
elements laid out column-major; `colmajor(t)` / `from_colmajor(buf, shape)`
convert between a logical torch tensor and that buffer.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CUDECOMPOSE_B200_LIB") or os.path.join(_HERE, "libcudecompose_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is not built; run `make -C first-project_b200` "
        "(or __graft_entry__.build()) first")
_lib = ctypes.CDLL(LIB_PATH)

# status codes (include/cudecompose_c.h)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_NO_MEMORY = 3
ERR_NOT_CONVERGED = 4
ERR_UNSUPPORTED = 5
ERR_SINGULAR = 6
ERR_DEVICE_TIMEOUT = 7

# precisions
PREC_FP32 = 0
PREC_BF16 = 1
PREC_FP16 = 2
PREC_BF16X3 = 3
PREC_DEFAULT = 4
PRECISIONS = {"fp32": PREC_FP32, "bf16": PREC_BF16, "fp16": PREC_FP16,
              "bf16x3": PREC_BF16X3, "default": PREC_DEFAULT}

_vp = ctypes.c_void_p
_l = ctypes.c_long
_i = ctypes.c_int
_d = ctypes.c_double


class CpOptions(ctypes.Structure):
    _fields_ = [("max_sweeps", _i), ("tol", _d), ("precision", _i),
                ("use_graph", _i), ("check_every", _i), ("target_fit", _d), ("sweep_layout", _i)]


class GemmEpilogue(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_float), ("bias", _vp), ("relu", _i),
                ("mask", _vp), ("mask_ldm", _l), ("mask_ldn", _l),
                ("out_f32", _vp), ("f32_ldm", _l), ("f32_ldn", _l), ("f32_accumulate", _i),
                ("out_bf16", _vp), ("bf16_ldm", _l), ("bf16_ldn", _l),
                ("out_bf16_2", _vp), ("bf16_2_ldm", _l), ("bf16_2_ldn", _l)]


class CpResult(ctypes.Structure):
    _fields_ = [("sweeps", _i), ("fallbacks", _i), ("fit", _d),
                ("fit_prev", _d), ("seconds", _d), ("kernels_per_sweep", _i),
                ("fit_estimate", _d)]


def _sig(name, argtypes, restype=_i):
    f = getattr(_lib, name)
    f.argtypes = argtypes
    f.restype = restype
    return f


_sig("cud_get_last_error", [])
_sig("cud_status_string", [_i], ctypes.c_char_p)
_sig("cud_last_error_detail", [], ctypes.c_char_p)
_sig("cud_hadmard", [_vp, _vp, _vp, _l, _l, _vp])
_sig("cud_hadmard3", [_vp, _vp, _vp, _vp, _l, _l, _vp])
_sig("cud_elepro3", [_vp, _vp, _vp, _vp, _l, _vp])
_sig("cud_kr", [_vp, _vp, _vp, _l, _l, _l, _vp])
_sig("cud_tensor_product", [_vp, _vp, _vp, _l, _l, _l, _l, _vp])
_sig("cud_f2h", [_vp, _vp, _l, _vp])
_sig("cud_f2bf", [_vp, _vp, _l, _vp])
_sig("cud_t2m", [_vp, _vp, _l, _l, _l, _l, _vp])
_sig("cud_tminust", [_vp, _vp, _l, _vp])
_sig("cud_init_identity", [_vp, _l, _vp])
_sig("cud_rse", [_vp, _vp, _l, ctypes.POINTER(ctypes.c_float), _vp])
_sig("cud_norm2", [_vp, _l, ctypes.POINTER(_d), _vp])
_sig("cud_gencp", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_vp), _l, _vp])
_sig("cud_gentucker", [_vp, _i, ctypes.POINTER(_l), _vp, ctypes.POINTER(_l),
                       ctypes.POINTER(_vp), _vp])
_sig("cud_ttm", [_vp, _vp, _vp, _l, _l, _l, _l, _l, _i, _vp])
_sig("cud_mode_product", [_vp, _i, ctypes.POINTER(_l), _i, _vp, _l, _vp, _i, _vp])
_sig("cud_mttkrp_legacy", [_vp, _vp, _vp, _vp, _l, _l, _l, _l, _l, _i, _vp])
_sig("cud_mttkrp", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_vp), _i, _l, _vp, _i, _vp])
_sig("cud_unfold_gram", [_vp, _i, ctypes.POINTER(_l), _i, _vp, _i, _vp])
_sig("cud_mttkrp_path", [_i, ctypes.POINTER(_l), _i, _l, _i])
_sig("cud_prof_enable", [_i])
_sig("cud_cp_als_release", [])
_sig("cud_prof_kernel_times", [ctypes.POINTER(ctypes.c_float), _i, ctypes.POINTER(_i)])
_sig("cud_syev_jacobi", [_vp, _l, _vp, _vp, _i, _vp])
_sig("cud_cross_gram", [_vp, _vp, _l, _l, _l, _vp, _l, _vp])
_sig("cud_syev_top", [_vp, _l, _l, _vp, _vp, _i, _vp])
_sig("cud_cp_default_options", [ctypes.POINTER(CpOptions)], None)
_sig("cud_cp_als", [_vp, _i, ctypes.POINTER(_l), _l, ctypes.POINTER(_vp),
                    ctypes.POINTER(CpOptions), ctypes.POINTER(CpResult), _vp])
_sig("cud_cp_als_f64", [_vp, _i, ctypes.POINTER(_l), _l, ctypes.POINTER(_vp),
                        ctypes.POINTER(CpOptions), ctypes.POINTER(CpResult), _vp])
_sig("cud_mttkrp_f64", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_vp), _i, _l, _vp, _vp])
_sig("cud_tucker_hosvd_f64", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_l), _vp, ctypes.POINTER(_vp), _vp])
_sig("cud_tucker_hooi_f64", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_l), _vp, ctypes.POINTER(_vp), _i, _vp])
_sig("cud_cp_init_curand", [_i, ctypes.POINTER(_l), _l, ctypes.POINTER(_vp),
                            ctypes.c_ulonglong, _vp])
_sig("cud_cp_plan_create", [_vp, _i, ctypes.POINTER(_l), _l, ctypes.POINTER(_vp),
                            ctypes.POINTER(CpOptions), _vp, ctypes.POINTER(_vp)])
_sig("cud_cp_plan_run", [_vp, _i, _vp])
_sig("cud_cp_plan_fit", [_vp, ctypes.POINTER(_d), ctypes.POINTER(_d), _vp])
_sig("cud_cp_plan_true_fit", [_vp, ctypes.POINTER(_d), _vp])
_sig("cud_cp_plan_info", [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)])
_sig("cud_gemm_bf16", [_vp, _l, _vp, _l, _l, _l, _l, ctypes.POINTER(GemmEpilogue), _vp])
_sig("cud_cp_residual", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_vp), _l, ctypes.POINTER(_d),
                         ctypes.POINTER(_d), _vp])
_sig("cud_cp_plan_destroy", [_vp])
_sig("cud_cp_als_batched", [_i, ctypes.POINTER(_l), ctypes.POINTER(_l), _vp, ctypes.POINTER(_l), _vp,
                            ctypes.POINTER(_l), ctypes.POINTER(CpOptions), ctypes.POINTER(_d),
                            ctypes.POINTER(_i), ctypes.POINTER(_i), _vp])
_sig("cud_cp_als_batched_target", [_i, ctypes.POINTER(_l), ctypes.POINTER(_l), _vp, ctypes.POINTER(_l), _vp,
                                   ctypes.POINTER(_l), ctypes.POINTER(CpOptions), ctypes.POINTER(_d),
                                   ctypes.POINTER(_d), ctypes.POINTER(_i), ctypes.POINTER(_i), _vp])
_sig("cud_ws_model_create", [_i, _i, _i, _i, ctypes.c_ulonglong, ctypes.POINTER(_vp)])
_sig("cud_ws_model_destroy", [_vp])
_sig("cud_ws_model_align", [_vp, _i, _i])
_sig("cud_ws_model_params", [_vp, ctypes.POINTER(_vp), _i])
_sig("cud_ws_model_grads", [_vp, ctypes.POINTER(_vp)])
_sig("cud_ws_backward", [_vp, _vp, _vp, _vp, _i, ctypes.POINTER(_d), _vp])
_sig("cud_ws_train_step", [_vp, _vp, _vp, _vp, _i, ctypes.c_float, ctypes.POINTER(_d), _vp])
_sig("cud_ws_predict", [_vp, _vp, _i, _vp, _vp])
_sig("cud_ws_generate", [_l, _l, ctypes.c_ulonglong, _i, _i, _d, _vp, _vp, _vp, _vp])
_sig("cud_ws_omega", [_i, _i, ctypes.c_ulonglong, _vp, _vp])
_sig("cud_ws_features", [_vp, _l, _i, _vp, _i, _vp, _vp, _vp, _vp])
_sig("cud_ws_canonical", [_vp, _vp, _l, _i, _i, _vp])
_sig("cud_ws_uncanonical", [_vp, _vp, _vp, _l, _i, _i, _vp])
_sig("cud_ws_hosvd_init", [_vp, _l, _i, _i, _vp, _vp])
_sig("cud_cp_batched_tune", [_i, ctypes.POINTER(_l), ctypes.POINTER(_l), _vp, ctypes.POINTER(_l), _vp,
                             ctypes.POINTER(_l), ctypes.POINTER(_i), ctypes.POINTER(_i), _vp])
_sig("cud_factor_gram", [_vp, _l, _l, _vp, _vp])
_sig("cud_cp_solve", [_vp, _l, _l, _i, ctypes.POINTER(_vp), _i, _vp, _vp, _vp])
_sig("cud_cp_normal_inverse", [_l, _i, ctypes.POINTER(_vp), _i, _vp, _vp])
_sig("cud_cp_apply_inverse", [_vp, _l, _l, _vp, _vp, _vp])
_sig("cud_cp_fit_terms", [_vp, _vp, _l, _i, ctypes.POINTER(_vp), _l, ctypes.POINTER(_d),
                          ctypes.POINTER(_d), _vp])
_sig("cud_tucker_hosvd", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_l), _vp,
                          ctypes.POINTER(_vp), _i, _vp])
_sig("cud_tucker_hooi", [_vp, _i, ctypes.POINTER(_l), ctypes.POINTER(_l), _vp,
                         ctypes.POINTER(_vp), _i, _i, _vp])


class CudError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = _lib.cud_status_string(status).decode()
        detail = _lib.cud_last_error_detail().decode()
        super().__init__(f"{where}: status {status} ({msg}) {detail}".strip())
        self.status = status


def library() -> ctypes.CDLL:
    """The loaded shared library (for raw C-ABI calls)."""
    return _lib


def _check(st: int, where: str, allow=(OK,)):
    if st not in allow:
        raise CudError(st, where)
    return st


def _ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("device tensor required")
    if not t.is_contiguous():
        raise ValueError("contiguous tensor required")
    return t.data_ptr()


def _stream(stream=None) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream or None
    return stream


def _longs(xs: Sequence[int]):
    return (_l * len(xs))(*[int(x) for x in xs])


def _ptrs(ts: Sequence[torch.Tensor | None]):
    return (_vp * len(ts))(*[_ptr(t) if t is not None else None for t in ts])


# --------------------------------------------------------------------------
# layout helpers
# --------------------------------------------------------------------------

def colmajor(t: torch.Tensor) -> torch.Tensor:
    """Flat column-major float32 copy of a logical tensor/matrix."""
    return t.float().permute(*reversed(range(t.dim()))).contiguous().reshape(-1)


def from_colmajor(buf: torch.Tensor, shape: Sequence[int]) -> torch.Tensor:
    """Logical tensor view of a flat column-major buffer."""
    return buf.reshape(tuple(reversed(shape))).permute(*reversed(range(len(shape))))


# --------------------------------------------------------------------------
# reference-named routines (device tensors in, device tensors out)
# --------------------------------------------------------------------------

def hadmard(A, B, C, a, b, stream=None):
    _check(_lib.cud_hadmard(_ptr(A), _ptr(B), _ptr(C), a, b, _stream(stream)), "hadmard")


def hadmard3(A, B, C, D, a, b, stream=None):
    _check(_lib.cud_hadmard3(_ptr(A), _ptr(B), _ptr(C), _ptr(D), a, b, _stream(stream)), "hadmard3")


def elepro3(A, B, C, D, n, stream=None):
    _check(_lib.cud_elepro3(_ptr(A), _ptr(B), _ptr(C), _ptr(D), n, _stream(stream)), "elepro3")


def kr(A, B, AkrB, a, b, r, stream=None):
    _check(_lib.cud_kr(_ptr(A), _ptr(B), _ptr(AkrB), a, b, r, _stream(stream)), "kr")


def tensor_product(A, B, C, a, b, c, d, stream=None):
    _check(_lib.cud_tensor_product(_ptr(A), _ptr(B), _ptr(C), a, b, c, d, _stream(stream)),
           "tensor_product")


def f2h(A, B, n, stream=None):
    _check(_lib.cud_f2h(_ptr(A), _ptr(B), n, _stream(stream)), "f2h")


def f2bf(A, B, n, stream=None):
    _check(_lib.cud_f2bf(_ptr(A), _ptr(B), n, _stream(stream)), "f2bf")


def t2m(T1, T2, flag, m, n, k, stream=None):
    _check(_lib.cud_t2m(_ptr(T1), _ptr(T2), flag, m, n, k, _stream(stream)), "t2m")


def tminust(M, N, m, stream=None):
    _check(_lib.cud_tminust(_ptr(M), _ptr(N), m, _stream(stream)), "tminust")


def initMat(A, m, stream=None):
    _check(_lib.cud_init_identity(_ptr(A), m, _stream(stream)), "initMat")


def rse(X, X1, m, stream=None) -> float:
    err = ctypes.c_float(0.0)
    _check(_lib.cud_rse(_ptr(X), _ptr(X1), m, ctypes.byref(err), _stream(stream)), "rse")
    return err.value


def norm2(x, n=None, stream=None) -> float:
    out = _d(0.0)
    n = x.numel() if n is None else n
    _check(_lib.cud_norm2(_ptr(x), n, ctypes.byref(out), _stream(stream)), "norm2")
    return out.value


def gencp(rec, factors, dims, r, stream=None):
    _check(_lib.cud_gencp(_ptr(rec), len(dims), _longs(dims), _ptrs(factors), r,
                          _stream(stream)), "gencp")


def gentucker(rec, core, factors, dims, ranks, stream=None):
    _check(_lib.cud_gentucker(_ptr(rec), len(dims), _longs(dims), _ptr(core), _longs(ranks),
                              _ptrs(factors), _stream(stream)), "gentucker")


def ttm(X, U, XU, flag, a, b, c, d, precision=PREC_FP32, stream=None):
    _check(_lib.cud_ttm(_ptr(X), _ptr(U), _ptr(XU), flag, a, b, c, d, precision,
                        _stream(stream)), "ttm")


def mode_product(X, dims, mode, W, J, Y, precision=PREC_FP32, stream=None):
    _check(_lib.cud_mode_product(_ptr(X), len(dims), _longs(dims), mode, _ptr(W), J, _ptr(Y),
                                 precision, _stream(stream)), "mode_product")


def mttkrp_legacy(X, left, right, XU, flag, m, n, k, r, precision=PREC_FP16, stream=None):
    _check(_lib.cud_mttkrp_legacy(_ptr(X), _ptr(left), _ptr(right), _ptr(XU), flag, m, n, k, r,
                                  precision, _stream(stream)), "mttkrp_legacy")


def mttkrp(X, dims, factors, mode, R, out, precision=PREC_DEFAULT, stream=None):
    """out (dims[mode] x R, column-major) = X_(mode) (KR of the other factors)."""
    _check(_lib.cud_mttkrp(_ptr(X), len(dims), _longs(dims), _ptrs(factors), mode, R,
                           _ptr(out), precision, _stream(stream)), "mttkrp")


def mttkrp_path(dims, mode, R, precision=PREC_DEFAULT) -> str:
    """'tensor-core' or 'cuda-core': the kernel mttkrp() runs for this shape."""
    return "tensor-core" if _lib.cud_mttkrp_path(len(dims), _longs(dims), mode, R, precision) else "cuda-core"


def prof_enable(on=True):
    """Turns the MTTKRP entry points' kernel timing on or off (measurement)."""
    _check(_lib.cud_prof_enable(1 if on else 0), "prof_enable")


def prof_kernel_times(max_n=256):
    """Durations (ms) of the MTTKRP main kernels recorded since the last read."""
    buf = (ctypes.c_float * max_n)()
    n = _i(0)
    _check(_lib.cud_prof_kernel_times(buf, max_n, ctypes.byref(n)), "prof_kernel_times")
    return [buf[i] for i in range(min(n.value, max_n))]


def unfold_gram(X, dims, mode, G, stream=None):
    _check(_lib.cud_unfold_gram(_ptr(X), len(dims), _longs(dims), mode, _ptr(G), 0,
                                _stream(stream)), "unfold_gram")


def cross_gram(A, B, P, ma, mb, G, ldg, stream=None):
    """G[i + ldg j] = sum_p A[p + P i] B[p + P j] (FP32 in, FP64 out); G may be
    a view into a larger float64 matrix."""
    _check(_lib.cud_cross_gram(_ptr(A), _ptr(B), P, ma, mb, _ptr(G), ldg, _stream(stream)), "cross_gram")


def syev_jacobi(A, n, W, V, max_sweeps=60, stream=None):
    return _check(_lib.cud_syev_jacobi(_ptr(A), n, _ptr(W), _ptr(V), max_sweeps,
                                       _stream(stream)), "syev_jacobi",
                  allow=(OK, ERR_NOT_CONVERGED))


def syev_top(G, n, r, U, U0=None, max_iters=300, stream=None):
    """U (n x r, FP32, column-major) = the r leading eigenvectors of the
    symmetric PSD FP64 n x n matrix G, ascending eigenvalue order; U0 seeds
    the iteration.  Returns OK or ERR_NOT_CONVERGED."""
    return _check(_lib.cud_syev_top(_ptr(G), n, r, _ptr(U), _ptr(U0), max_iters, _stream(stream)),
                  "syev_top", allow=(OK, ERR_NOT_CONVERGED))


def cp_default_options() -> CpOptions:
    o = CpOptions()
    _lib.cud_cp_default_options(ctypes.byref(o))
    return o


def cp_als(X, dims, R, factors, max_sweeps=500, tol=0.0, precision=PREC_DEFAULT,
           use_graph=True, check_every=1, target_fit=0.0, stream=None, layout=0) -> CpResult:
    """CP-ALS from the given initial factors (updated in place).  Stops after
    max_sweeps, when |fit - fit_prev| < tol (tol > 0), or when fit >=
    target_fit (target_fit > 0).  layout: the sweep layout (0 by size, 1, 2;
    cud_cp_options.sweep_layout)."""
    opt = CpOptions(max_sweeps, tol, precision, 1 if use_graph else 0, check_every, target_fit, layout)
    res = CpResult()
    _check(_lib.cud_cp_als(_ptr(X), len(dims), _longs(dims), R, _ptrs(factors),
                           ctypes.byref(opt), ctypes.byref(res), _stream(stream)), "cp_als")
    return res


def cp_als_release():
    """Frees the plan cud_cp_als keeps for its next call with the same arguments."""
    _check(_lib.cud_cp_als_release(), "cp_als_release")


def cp_als_f64(X, dims, R, factors, max_sweeps=500, tol=0.0, target_fit=0.0, stream=None) -> CpResult:
    """FP64 CP-ALS (the reference's dprice/cp_als.cu and 4_cp_als.cu) on
    float64 device tensors, factors updated in place.  Stops after
    max_sweeps, when |fit - fit_prev| < tol (tol > 0), or when fit >=
    target_fit (target_fit > 0)."""
    opt = CpOptions(max_sweeps, tol, PREC_FP32, 0, 1, target_fit)
    res = CpResult()
    _check(_lib.cud_cp_als_f64(_ptr(X), len(dims), _longs(dims), R, _ptrs(factors),
                               ctypes.byref(opt), ctypes.byref(res), _stream(stream)), "cp_als_f64")
    return res


def mttkrp_f64(X, dims, factors, mode, R, out, stream=None):
    """out (dims[mode] x R, column-major, float64) = X_(mode) (KR of the other
    factors), all in FP64 on the CUDA cores."""
    _check(_lib.cud_mttkrp_f64(_ptr(X), len(dims), _longs(dims), _ptrs(factors), mode, R,
                               _ptr(out), _stream(stream)), "mttkrp_f64")


class CpPlan:
    """Reusable CP-ALS plan (cud_cp_plan_*): workspace plus the captured
    per-sweep CUDA graph; `run(n)` enqueues n sweeps without synchronising."""

    def __init__(self, X, dims, R, factors, precision=PREC_DEFAULT, use_graph=True, stream=None, layout=0):
        self._keep = (X, list(factors))
        opt = CpOptions(0, 0.0, precision, 1 if use_graph else 0, 1, 0.0, layout)
        h = _vp()
        _check(_lib.cud_cp_plan_create(_ptr(X), len(dims), _longs(dims), R, _ptrs(factors),
                                       ctypes.byref(opt), _stream(stream), ctypes.byref(h)),
               "cp_plan_create")
        self._h = h

    def run(self, sweeps=1, stream=None):
        _check(_lib.cud_cp_plan_run(self._h, sweeps, _stream(stream)), "cp_plan_run")

    def fit(self, stream=None):
        f, fp = _d(0.0), _d(0.0)
        _check(_lib.cud_cp_plan_fit(self._h, ctypes.byref(f), ctypes.byref(fp), _stream(stream)),
               "cp_plan_fit")
        return f.value, fp.value

    def true_fit(self, stream=None):
        """Exact fit of the current factors (cud_cp_plan_true_fit)."""
        f = _d(0.0)
        _check(_lib.cud_cp_plan_true_fit(self._h, ctypes.byref(f), _stream(stream)), "cp_plan_true_fit")
        return f.value

    def info(self):
        k, fb = _i(0), _i(0)
        _check(_lib.cud_cp_plan_info(self._h, ctypes.byref(k), ctypes.byref(fb)), "cp_plan_info")
        return k.value, fb.value

    def close(self):
        if self._h:
            _lib.cud_cp_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _mat_strides(t):
    """(ldm, ldn) of a 2-D tensor seen as out[m, n], or of out.T when
    passed as ('T', tensor)."""
    if isinstance(t, tuple):
        _, t = t
        return t, t.stride(1), t.stride(0)
    return t, t.stride(0), t.stride(1)


def gemm_bf16(A, B, alpha=1.0, bias=None, relu=False, mask=None, out_f32=None, accumulate=False,
              out_bf16=None, out_bf16_2=None, stream=None):
    """C[m, n] = epilogue(alpha * A[m, :] . B[n, :]) on the tensor cores
    (cud_gemm_bf16).  A (M x K) and B (N x K) are contiguous BF16 tensors.
    Each output / the mask is a 2-D tensor indexed [m, n], or ('T', t) for a
    tensor indexed [n, m] (a transposed copy)."""
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16
    M, K = A.shape
    N, K2 = B.shape
    assert K == K2 and A.stride(1) == 1 and B.stride(1) == 1
    e = GemmEpilogue()
    e.alpha = alpha
    e.bias = _ptr(bias) if bias is not None else None
    e.relu = 1 if relu else 0
    if mask is not None:
        t, e.mask_ldm, e.mask_ldn = _mat_strides(mask)
        e.mask = _ptr(t)
    if out_f32 is not None:
        t, e.f32_ldm, e.f32_ldn = _mat_strides(out_f32)
        e.out_f32 = _ptr(t)
        e.f32_accumulate = 1 if accumulate else 0
    if out_bf16 is not None:
        t, e.bf16_ldm, e.bf16_ldn = _mat_strides(out_bf16)
        e.out_bf16 = _ptr(t)
    if out_bf16_2 is not None:
        t, e.bf16_2_ldm, e.bf16_2_ldn = _mat_strides(out_bf16_2)
        e.out_bf16_2 = _ptr(t)
    _check(_lib.cud_gemm_bf16(_ptr(A), A.stride(0), _ptr(B), B.stride(0), M, N, K, ctypes.byref(e),
                              _stream(stream)), "gemm_bf16")


def cp_residual(X, dims, factors, R, stream=None):
    """(||X - [[factors]]||^2, ||X||^2) in FP64 (src/rse.cu:4 + gencp)."""
    r2, x2 = _d(0.0), _d(0.0)
    _check(_lib.cud_cp_residual(_ptr(X), len(dims), _longs(dims), _ptrs(factors), R,
                                ctypes.byref(r2), ctypes.byref(x2), _stream(stream)), "cp_residual")
    return r2.value, x2.value


def cp_true_fit(X, dims, factors, R, stream=None):
    """1 - ||X - [[factors]]|| / ||X||, from cp_residual."""
    r2, x2 = cp_residual(X, dims, factors, R, stream)
    return 1.0 - (r2 ** 0.5) / (x2 ** 0.5 if x2 > 0 else 1.0)


def factor_gram(U, I, R, G, stream=None):
    """G (R x R, float64 device tensor) = U^T U for U (I x R column-major)."""
    _check(_lib.cud_factor_gram(_ptr(U), I, R, _ptr(G), _stream(stream)), "factor_gram")


def cp_solve(M, I, R, grams, mode, U, work, stream=None):
    """U = M * inv(Hadamard of the Grams other than `mode`); work: float64
    device tensor of at least 3 R^2 + 2 elements."""
    _check(_lib.cud_cp_solve(_ptr(M), I, R, len(grams), _ptrs(grams), mode, _ptr(U), _ptr(work),
                             _stream(stream)), "cp_solve")


def cp_normal_inverse(R, grams, mode, work, stream=None):
    """V^-1 (V = Hadamard of the Grams other than `mode`) into the first R^2
    doubles of work (float64 device tensor of at least 3 R^2 + 2)."""
    _check(_lib.cud_cp_normal_inverse(R, len(grams), _ptrs(grams), mode, _ptr(work), _stream(stream)),
           "cp_normal_inverse")


def cp_apply_inverse(M, I, R, work, U, stream=None):
    """U = M * V^-1 with V^-1 from cp_normal_inverse (in work)."""
    _check(_lib.cud_cp_apply_inverse(_ptr(M), I, R, _ptr(work), _ptr(U), _stream(stream)), "cp_apply_inverse")


def cp_fit_terms(M, U, grams, R, stream=None):
    """(<M, U>, sum_{r,s} prod_m G_m[r, s]) computed on the device."""
    inner, nh = _d(0.0), _d(0.0)
    _check(_lib.cud_cp_fit_terms(_ptr(M), _ptr(U), M.numel(), len(grams), _ptrs(grams), R,
                                 ctypes.byref(inner), ctypes.byref(nh), _stream(stream)),
           "cp_fit_terms")
    return inner.value, nh.value


class Batch:
    """A packed batch of small 3rd-order tensors for cp_als_batched: X and
    all factors in two device buffers, with per-tensor offsets (16-byte
    aligned)."""

    def __init__(self, dims, ranks, device="cuda"):
        self.dims = [tuple(int(x) for x in d) for d in dims]
        self.ranks = [int(r) for r in ranks]
        self.n = len(self.dims)
        xo, uo, xs, us = [], [], 0, 0
        for d, r in zip(self.dims, self.ranks):
            xo.append(xs)
            xs += (d[0] * d[1] * d[2] + 3) // 4 * 4
            for m in range(3):
                uo.append(us)
                us += (d[m] * r + 3) // 4 * 4
        self.x_offsets, self.u_offsets = xo, uo
        self.X = torch.zeros(max(xs, 4), device=device)
        self.U = torch.zeros(max(us, 4), device=device)

    def x_view(self, t):
        d = self.dims[t]
        return self.X[self.x_offsets[t]: self.x_offsets[t] + d[0] * d[1] * d[2]]

    def u_view(self, t, m):
        o = self.u_offsets[3 * t + m]
        return self.U[o: o + self.dims[t][m] * self.ranks[t]]

    def _args(self):
        flat = [x for d in self.dims for x in d]
        return (_longs(flat), _longs(self.ranks), _longs(self.x_offsets), _longs(self.u_offsets))


def cp_als_batched(batch, max_sweeps=50, tol=1e-6, use_graph=True, sweeps_per_graph=5, stream=None):
    """Batched CP-ALS (one persistent kernel per sweep).  Returns (fits,
    sweeps, kernel_launches) per tensor; the factors in batch.U are updated."""
    d, r, xo, uo = batch._args()
    opt = CpOptions(max_sweeps, tol, PREC_FP32, 1 if use_graph else 0, sweeps_per_graph, 0.0)
    fits = (_d * batch.n)()
    sw = (_i * batch.n)()
    launches = _i(0)
    _check(_lib.cud_cp_als_batched(batch.n, d, r, _ptr(batch.X), xo, _ptr(batch.U), uo,
                                   ctypes.byref(opt), fits, sw, ctypes.byref(launches),
                                   _stream(stream)), "cp_als_batched")
    return list(fits), list(sw), launches.value


def cp_als_batched_target(batch, targets, max_sweeps=50, use_graph=True, sweeps_per_graph=1, stream=None):
    """Batched CP-ALS where tensor t stops once its fit >= targets[t].
    Returns (fits, sweeps, kernel_launches)."""
    d, r, xo, uo = batch._args()
    opt = CpOptions(max_sweeps, 0.0, PREC_FP32, 1 if use_graph else 0, sweeps_per_graph, 0.0)
    tg = (_d * batch.n)(*[float(x) for x in targets])
    fits = (_d * batch.n)()
    sw = (_i * batch.n)()
    launches = _i(0)
    _check(_lib.cud_cp_als_batched_target(batch.n, d, r, _ptr(batch.X), xo, _ptr(batch.U), uo,
                                          ctypes.byref(opt), tg, fits, sw, ctypes.byref(launches),
                                          _stream(stream)), "cp_als_batched_target")
    return list(fits), list(sw), launches.value


def cp_batched_tune(batch, stream=None):
    """Autotunes the batched sweep's launch shape; returns (threads, ctas_per_sm)."""
    d, r, xo, uo = batch._args()
    Ucopy = batch.U.clone()
    th, cps = _i(0), _i(0)
    _check(_lib.cud_cp_batched_tune(batch.n, d, r, _ptr(batch.X), xo, _ptr(Ucopy), uo,
                                    ctypes.byref(th), ctypes.byref(cps), _stream(stream)),
           "cp_batched_tune")
    return th.value, cps.value


def cp_init_curand(dims, R, factors, seed=1234, stream=None):
    _check(_lib.cud_cp_init_curand(len(dims), _longs(dims), R, _ptrs(factors), seed,
                                   _stream(stream)), "cp_init_curand")


def tucker_hosvd(X, dims, ranks, core, factors, precision=PREC_FP32, stream=None):
    return _check(_lib.cud_tucker_hosvd(_ptr(X), len(dims), _longs(dims), _longs(ranks),
                                        _ptr(core), _ptrs(factors), precision, _stream(stream)),
                  "tucker_hosvd", allow=(OK, ERR_NOT_CONVERGED))


def tucker_hooi(X, dims, ranks, core, factors, sweeps=10, precision=PREC_FP32, stream=None):
    return _check(_lib.cud_tucker_hooi(_ptr(X), len(dims), _longs(dims), _longs(ranks),
                                       _ptr(core), _ptrs(factors), sweeps, precision,
                                       _stream(stream)),
                  "tucker_hooi", allow=(OK, ERR_NOT_CONVERGED))


def tucker_hosvd_f64(X, dims, ranks, core, factors, stream=None):
    """FP64 HOSVD (the reference's dprice/tucker_hosvd.cu, 4_tucker_hosvd.cu)
    on float64 device tensors."""
    return _check(_lib.cud_tucker_hosvd_f64(_ptr(X), len(dims), _longs(dims), _longs(ranks),
                                            _ptr(core), _ptrs(factors), _stream(stream)),
                  "tucker_hosvd_f64", allow=(OK, ERR_NOT_CONVERGED))


def tucker_hooi_f64(X, dims, ranks, core, factors, sweeps=10, stream=None):
    """FP64 HOOI (the reference's dprice/tucker_hooi.cu) on float64 device
    tensors."""
    return _check(_lib.cud_tucker_hooi_f64(_ptr(X), len(dims), _longs(dims), _longs(ranks),
                                           _ptr(core), _ptrs(factors), sweeps, _stream(stream)),
                  "tucker_hooi_f64", allow=(OK, ERR_NOT_CONVERGED))


# --------------------------------------------------------------------------
# seeded synthetic workloads (the shapes and value distributions of the
# reference's benchmark configurations; generated on the device)
# --------------------------------------------------------------------------

def make_cp_tensor(dims, R, seed=0, noise=1e-3, device="cuda"):
    """X = sum_r U1[:,r] o U2[:,r] o ... + noise, factors uniform [0,1), noise
    i.i.d. Gaussian scaled to `noise` * ||X_clean||_F.  Returns the flat
    column-major X and the list of true factors (dims[m] x R column-major)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    facs = [torch.rand(int(R) * int(d), generator=g, device=device, dtype=torch.float32)
            for d in dims]
    n = 1
    for d in dims:
        n *= int(d)
    X = torch.empty(n, device=device, dtype=torch.float32)
    gencp(X, facs, dims, R)
    if noise > 0:
        nrm = norm2(X) ** 0.5
        E = torch.randn(n, generator=g, device=device, dtype=torch.float32)
        enrm = norm2(E) ** 0.5
        X.add_(E, alpha=noise * nrm / enrm)
    return X, facs


def make_init(dims, R, seed=1, device="cuda"):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return [torch.rand(int(R) * int(d), generator=g, device=device, dtype=torch.float32)
            for d in dims]


def make_tucker_tensor(dims, ranks, seed=0, noise=1e-3, device="cuda"):
    """X = G x_1 U1 x_2 U2 ... + noise; G i.i.d. N(0,1), U_n orthonormal
    columns (QR of a seeded Gaussian)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    core = torch.randn(int(torch.tensor(ranks).prod()), generator=g, device=device)
    facs = []
    for d, r in zip(dims, ranks):
        Z = torch.randn(int(d), int(r), generator=g, device=device, dtype=torch.float64)
        Q, _ = torch.linalg.qr(Z)
        facs.append(colmajor(Q.float()))
    n = 1
    for d in dims:
        n *= int(d)
    X = torch.empty(n, device=device, dtype=torch.float32)
    gentucker(X, core, facs, dims, ranks)
    if noise > 0:
        nrm = norm2(X) ** 0.5
        E = torch.randn(n, generator=g, device=device, dtype=torch.float32)
        enrm = norm2(E) ** 0.5
        X.add_(E, alpha=noise * nrm / enrm)
    return X, core, facs
