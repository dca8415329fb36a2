"""The C ABI boundary, checked without a GPU: the library loads, exports every
symbol include/*.h declares, validates arguments on the host, and the
drop-in archive links a program written against the reference's header."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
PKG = os.path.join(ROOT, "first-project_b200")
SO = os.path.join(PKG, "libcudecompose_b200.so")
ARCHIVE = os.path.join(PKG, "libcutensordecomposition.a")


def _c_decls():
    text = open(os.path.join(INC, "cudecompose_c.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cud_\w+)\s*\(", text)))


def _cpp_decls():
    text = open(os.path.join(INC, "cudecompose.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    host = re.findall(r"^\s*(?:void|int)\s+(\w+)\s*\(", text, flags=re.M)
    kernels = re.findall(r"__global__\s+void\s+(\w+)\s*\(", text)
    return sorted(set(host)), sorted(set(kernels))


def test_header_declares_the_reference_api():
    host, kernels = _cpp_decls()
    # inc/cudecompose.h:22-57 of the reference
    for name in ["hadmard", "kr", "tensor_product", "printTensor", "f2h", "ttm", "mttkrp", "t2m",
                 "tminust", "rse", "gencp", "gentucker", "cp_als", "tucker_hosvd", "cp_tensorcore",
                 "tucker_tensorcore", "initMat", "hadmard3", "cp_als4", "tucker_hosvd4", "gencp4",
                 "gentucker4"]:
        assert name in host, name
    for name in ["hardm", "floattohalf", "tensorTomat1", "tensorTomat2", "tensorTomat3", "t_t",
                 "initIdeMat", "hardm3", "elepro3", "elemin"]:
        assert name in kernels, name


def test_library_exports_every_c_symbol():
    lib = ctypes.CDLL(SO)
    missing = [n for n in _c_decls() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(shutil.which("nm") is None, reason="binutils nm missing")
def test_library_exports_every_cpp_symbol():
    out = subprocess.run(["nm", "-DC", "--defined-only", SO], capture_output=True, text=True,
                         check=True).stdout
    host, kernels = _cpp_decls()
    names = set(re.findall(r"\s[TW]\s+(?:cud::)?(\w+)\(", out))
    missing = [n for n in host + kernels if n not in names]
    assert not missing, missing
    # the two initIdeMat overloads of the reference (inc/cudecompose.h:45,56)
    assert "initIdeMat(float*, long)" in out and "initIdeMat(float*, int)" in out


def test_status_side_channel_without_gpu():
    lib = ctypes.CDLL(SO)
    lib.cud_status_string.restype = ctypes.c_char_p
    assert lib.cud_status_string(0) == b"ok"
    assert b"invalid" in lib.cud_status_string(1)
    lib.cud_hadmard.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_long] * 2 + [ctypes.c_void_p]
    assert lib.cud_hadmard(None, None, None, -1, 2, None) == 1
    assert lib.cud_get_last_error() == 1
    lib.cud_t2m.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_long] * 4 + [ctypes.c_void_p]
    assert lib.cud_t2m(None, None, 4, 2, 2, 2, None) == 1  # flag outside 1..3
    lib.cud_mttkrp_legacy.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_long] * 5 + [ctypes.c_int, ctypes.c_void_p]
    assert lib.cud_mttkrp_legacy(None, None, None, None, 0, 2, 2, 2, 2, 0, None) == 1
    lib.cud_cp_als.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_long,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    dims = (ctypes.c_long * 3)(4, 4, 4)
    assert lib.cud_cp_als(None, 3, dims, 0, None, None, None, None) == 1  # R = 0
    # empty extents are a no-op that succeeds without touching the device
    assert lib.cud_hadmard(None, None, None, 0, 5, None) == 0
    assert lib.cud_get_last_error() == 0


def test_extended_entry_points_validate_without_gpu():
    """The FP64 programs, the subspace eigensolver and the cross-Gram block
    reject bad arguments on the host, before any device work."""
    lib = ctypes.CDLL(SO)
    vp, L, I = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
    dims = (ctypes.c_long * 3)(4, 4, 4)
    ranks = (ctypes.c_long * 3)(2, 2, 5)  # rank 5 > extent 4
    lib.cud_syev_top.argtypes = [vp, L, L, vp, vp, I, vp]
    assert lib.cud_syev_top(None, 8, 2, None, None, 10, None) == 1   # null G, U
    lib.cud_cross_gram.argtypes = [vp, vp, L, L, L, vp, L, vp]
    assert lib.cud_cross_gram(None, None, 4, 2, 2, None, 2, None) == 1
    lib.cud_cp_als_f64.argtypes = [vp, I, vp, L, vp, vp, vp, vp]
    assert lib.cud_cp_als_f64(None, 3, dims, 2, None, None, None, None) == 1
    lib.cud_mttkrp_f64.argtypes = [vp, I, vp, vp, I, L, vp, vp]
    assert lib.cud_mttkrp_f64(None, 3, dims, None, 3, 2, None, None) == 1  # mode out of range
    lib.cud_tucker_hosvd_f64.argtypes = [vp, I, vp, vp, vp, vp, vp]
    assert lib.cud_tucker_hosvd_f64(None, 3, dims, ranks, None, None, None) == 1
    lib.cud_tucker_hooi_f64.argtypes = [vp, I, vp, vp, vp, vp, I, vp]
    assert lib.cud_tucker_hooi_f64(None, 3, dims, ranks, None, None, 2, None) == 1
    assert lib.cud_get_last_error() == 1


def test_python_mirror_imports(cd):
    assert os.path.samefile(cd.LIB_PATH, SO)
    opt = cd.cp_default_options()
    assert opt.max_sweeps == 500 and opt.tol == 0.0 and opt.use_graph == 1


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc missing")
def test_drop_in_program_links(tmp_path):
    exe = tmp_path / "drop_in"
    cmd = ["nvcc", "-o", str(exe), os.path.join(ROOT, "tests", "drivers", "drop_in.cpp"),
           "-I", INC, ARCHIVE, "-lcublas", "-lcusolver", "-lcurand"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert exe.exists()
