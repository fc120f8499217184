"""Python binding of libstmg_cuda.so (the C ABI declared in include/stmg.h).

Device memory and streams come from torch; every call goes through the C ABI
by ctypes. There is no CPU fallback: a missing library raises.
"""
import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libstmg_cuda.so")
HEADER = os.path.join(REPO, "include", "stmg.h")

F64, F32, BF16 = 0, 1, 2
DG, CGP = 2, 1
HEAT, WAVE = 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


class StmgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"stmg error {code}: {msg}")
        self.code = code


def header_symbols():
    """Names of the functions include/stmg.h declares."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(stmg_[A-Za-z0-9_]+)\s*\(", text)))


def lib():
    """Loads libstmg_cuda.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: run python dealii-stfem_b200/build.py")
        L = C.CDLL(LIB_PATH)
        L.stmg_last_error.restype = C.c_char_p
        for name in header_symbols():
            fn = getattr(L, name)
            if name not in ("stmg_last_error",):
                fn.restype = C.c_int
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise StmgError(rc, lib().stmg_last_error().decode())


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _dev(t):
    """Raw device pointer of a torch tensor."""
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Mesh:
    """stmg_mesh_t: structured FE_Q(p) mesh level on the device."""

    def __init__(self, dim, n_cells, degree, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), vertices=None, coeff=None,
                 coeff_mode=None):
        n = list(n_cells) + [1] * (3 - len(n_cells))
        self.dim, self.n, self.p = dim, n, degree
        lo_a = np.array(list(lo) + [0.0] * (3 - len(lo)), dtype=np.float64)
        hi_a = np.array(list(hi) + [1.0] * (3 - len(hi)), dtype=np.float64)
        v = None if vertices is None else np.ascontiguousarray(vertices, dtype=np.float64)
        c = None if coeff is None else np.ascontiguousarray(coeff, dtype=np.float64)
        if coeff_mode is None:
            coeff_mode = 0 if c is None else 1
        h = C.c_void_p()
        check(lib().stmg_mesh_create(dim, (C.c_int * 3)(*n), degree, _ptr(lo_a), _ptr(hi_a), _ptr(v), coeff_mode,
                                     _ptr(c), C.byref(h)))
        self.h = h
        nn, nc = C.c_longlong(), C.c_longlong()
        check(lib().stmg_mesh_info(self.h, C.byref(nn), C.byref(nc)))
        self.n_nodes, self.n_cells = nn.value, nc.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.stmg_mesh_destroy(self.h)
            self.h = None


class Operator:
    """stmg_op_t: dst_j = sum_i A(j,i) K src_i + B(j,i) M src_i."""

    def __init__(self, mesh, A, B, dtype=F64):
        A = np.ascontiguousarray(np.atleast_2d(A), dtype=np.float64)
        B = np.ascontiguousarray(np.atleast_2d(B), dtype=np.float64)
        assert A.shape == B.shape
        self.mesh, self.nt_out, self.nt_in, self.dtype = mesh, A.shape[0], A.shape[1], dtype
        h = C.c_void_p()
        check(lib().stmg_op_create(mesh.h, self.nt_out, self.nt_in, _ptr(A), _ptr(B), dtype, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.stmg_op_destroy(self.h)
            self.h = None

    def vmult(self, dst, src, stream=None):
        check(lib().stmg_op_vmult(self.h, _dev(dst), _dev(src), _stream(stream)))

    def Tvmult(self, dst, src, stream=None):
        check(lib().stmg_op_Tvmult(self.h, _dev(dst), _dev(src), _stream(stream)))

    def vmult_add(self, dst, src, stream=None):
        check(lib().stmg_op_vmult_add(self.h, _dev(dst), _dev(src), _stream(stream)))
