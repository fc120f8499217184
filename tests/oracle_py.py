"""ctypes access to the CPU oracle (oracle/build/liboracle.so).

Test infrastructure only: the oracle is what the CUDA path is compared
against; nothing in the product imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "build", "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrcConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("subdiv", C.c_int * 3), ("refine", C.c_int), ("p", C.c_int), ("r", C.c_int),
        ("type", C.c_int), ("problem", C.c_int), ("n_steps", C.c_int), ("n_slabs", C.c_int),
        ("tau", C.c_double), ("lo", C.c_double * 3), ("hi", C.c_double * 3),
        ("smoothing_steps", C.c_int), ("variable", C.c_int), ("estimate_relaxation", C.c_int),
        ("restrict_is_transpose", C.c_int), ("fe_degree_min", C.c_int), ("n_steps_min", C.c_int),
        ("mg_float", C.c_int), ("extrapolate", C.c_int), ("max_iter", C.c_int), ("restart", C.c_int),
        ("rhs_mode", C.c_int), ("compute_errors", C.c_int),
        ("tol", C.c_double), ("abs_tol", C.c_double), ("frequency", C.c_double),
        ("f_nodal", _dp), ("u0_nodal", _dp), ("v0_nodal", _dp), ("fine_vertices", _dp), ("fine_coeff", _dp),
    ]


class OrcResult(C.Structure):
    _fields_ = [("total_iterations", C.c_int), ("n_levels", C.c_int), ("n_blocks", C.c_int),
                ("l8", C.c_double), ("l2", C.c_double), ("h1", C.c_double),
                ("n_dofs", C.c_long), ("n_cells", C.c_long)]


def build():
    """Compile the oracle with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, "-j8"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_last_error.restype = C.c_char_p
        L.orc_mesh_create.restype = C.c_void_p
        L.orc_mesh_create.argtypes = [C.c_int, _ip, C.c_int, _dp, _dp, _dp, C.c_int, _dp]
        L.orc_mesh_destroy.argtypes = [C.c_void_p]
        L.orc_mesh_n_nodes.restype = C.c_long
        L.orc_mesh_n_nodes.argtypes = [C.c_void_p]
        L.orc_node_positions.argtypes = [C.c_void_p, _dp]
        L.orc_st_apply.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, _dp]
        L.orc_st_apply_vec.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, _dp, _dp]
        L.orc_element_matrices.argtypes = [C.c_void_p, C.c_long, _dp, _dp]
        L.orc_vanka_apply.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, _dp, _dp]
        L.orc_patch_matrices.argtypes = [C.c_void_p, C.c_long, _dp, _dp]
        L.orc_h_transfer.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, _dp, _dp]
        L.orc_time_weights.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.orc_time_prolongation.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        L.orc_run.argtypes = [C.POINTER(OrcConfig), C.POINTER(OrcResult), _ip, _dp, _dp]
        L.orc_run_all.argtypes = [C.POINTER(OrcConfig), C.POINTER(OrcResult), _ip, _dp, _dp, _dp]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


DG, CGP = 2, 1
HEAT, WAVE = 1, 2


class Mesh:
    """Structured mesh of FE_Q(p) with optional vertices and coefficient."""

    def __init__(self, dim, n, p, lo=(0, 0, 0), hi=(1, 1, 1), vertices=None, coeff=None, coeff_mode=None):
        n = list(n) + [1] * (3 - len(n))
        self.dim, self.n, self.p = dim, n, p
        self._keep = []
        na = (C.c_int * 3)(*n)
        lo_a = np.array(list(lo) + [0] * (3 - len(lo)), dtype=np.float64)
        hi_a = np.array(list(hi) + [1] * (3 - len(hi)), dtype=np.float64)
        v = None if vertices is None else np.ascontiguousarray(vertices, dtype=np.float64)
        c = None if coeff is None else np.ascontiguousarray(coeff, dtype=np.float64)
        if coeff_mode is None:
            coeff_mode = 0 if c is None else 1
        self._keep += [lo_a, hi_a, v, c]
        self.h = lib().orc_mesh_create(dim, na, p, _ptr(lo_a), _ptr(hi_a), _ptr(v), coeff_mode, _ptr(c))
        self.n_nodes = lib().orc_mesh_n_nodes(self.h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_mesh_destroy(self.h)
            self.h = None

    def node_positions(self):
        x = np.zeros((self.n_nodes, self.dim))
        _check(lib().orc_node_positions(self.h, _ptr(x)))
        return x

    def st_apply(self, Alpha, Beta, src, transpose=False, fp32=False):
        nt = Alpha.shape[0]
        A = np.ascontiguousarray(Alpha, dtype=np.float64)
        B = np.ascontiguousarray(Beta, dtype=np.float64)
        s = np.ascontiguousarray(src, dtype=np.float64)
        d = np.zeros_like(s)
        _check(lib().orc_st_apply(self.h, nt, _ptr(A), _ptr(B), int(transpose), int(fp32), _ptr(d), _ptr(s)))
        return d

    def st_apply_vec(self, a, b, src, dst=None):
        nt = a.shape[0]
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        s = np.ascontiguousarray(src, dtype=np.float64)
        add = dst is not None
        d = np.zeros(nt * self.n_nodes) if dst is None else np.array(dst, dtype=np.float64)
        _check(lib().orc_st_apply_vec(self.h, nt, _ptr(a), _ptr(b), int(add), _ptr(d), _ptr(s)))
        return d

    def element_matrices(self, cell):
        nd = (self.p + 1) ** self.dim
        K = np.zeros((nd, nd))
        M = np.zeros((nd, nd))
        _check(lib().orc_element_matrices(self.h, cell, _ptr(K), _ptr(M)))
        return K, M

    def patch_matrices(self, cell):
        nd = (self.p + 1) ** self.dim
        K = np.zeros((nd, nd))
        M = np.zeros((nd, nd))
        _check(lib().orc_patch_matrices(self.h, cell, _ptr(K), _ptr(M)))
        return K, M

    def vanka_apply(self, Alpha, Beta, src, fp32=False):
        nt = Alpha.shape[0]
        A = np.ascontiguousarray(Alpha, dtype=np.float64)
        B = np.ascontiguousarray(Beta, dtype=np.float64)
        s = np.ascontiguousarray(src, dtype=np.float64)
        d = np.zeros_like(s)
        _check(lib().orc_vanka_apply(self.h, nt, _ptr(A), _ptr(B), int(fp32), _ptr(d), _ptr(s)))
        return d


def h_transfer(fine, coarse, nt, src, restrict=False, dst=None):
    s = np.ascontiguousarray(src, dtype=np.float64)
    n_out = (coarse if restrict else fine).n_nodes * nt
    d = np.zeros(n_out) if dst is None else np.array(dst, dtype=np.float64)
    _check(lib().orc_h_transfer(fine.h, coarse.h, nt, int(restrict), _ptr(d), _ptr(s)))
    return d


def time_weights(ttype, r, tau, n_steps, problem=HEAT):
    nt = (r + 1 if ttype == DG else r) * n_steps
    A = np.zeros((nt, nt))
    B = np.zeros((nt, nt))
    rK = np.zeros(nt)
    rM = np.zeros(nt)
    rV = np.zeros(nt)
    _check(lib().orc_time_weights(ttype, r, tau, n_steps, problem, _ptr(A), _ptr(B), _ptr(rK), _ptr(rM), _ptr(rV)))
    return A, B, rK, rM, rV


def time_prolongation(ttype, kind, r, n_steps):
    """kind 0: k-projection r-1 -> r; kind 1: tau-prolongation."""
    if kind == 0:
        nf = (r + 1 if ttype == DG else r) * n_steps
        nc = (r if ttype == DG else r - 1) * n_steps
    else:
        nf = (r + 1 if ttype == DG else r) * n_steps
        nc = nf // 2
    P = np.zeros((nf, nc))
    _check(lib().orc_time_prolongation(ttype, kind, r, n_steps, _ptr(P)))
    return P


def run(dim=2, subdiv=(1, 1, 1), refine=2, p=2, r=1, ttype=DG, problem=HEAT, n_steps=1, n_slabs=None, tau=None,
        fe_degree_min=-1, n_steps_min=-1, mg_float=True, tol=1e-12, abs_tol=1e-12, frequency=1.0, rhs_mode=0,
        f_nodal=None, u0_nodal=None, v0_nodal=None, fine_vertices=None, fine_coeff=None, compute_errors=True,
        smoothing_steps=1, extrapolate=True, max_iter=200, lo=(0, 0, 0), hi=(1, 1, 1), keep_all=False):
    """The oracle's slab loop; with keep_all the result's "u_all" holds every
    slab's blocks (n_slabs, n_blocks * n_nodes)."""
    if tau is None:
        tau = 2.0 ** -(refine + 1)
    if n_slabs is None:
        n_slabs = int(round(1.0 / (tau * n_steps)))
    c = OrcConfig()
    c.dim, c.refine, c.p, c.r, c.type, c.problem = dim, refine, p, r, ttype, problem
    c.subdiv[:] = list(subdiv) + [1] * (3 - len(subdiv))
    c.n_steps, c.n_slabs, c.tau = n_steps, n_slabs, tau
    c.lo[:] = list(lo) + [0] * (3 - len(lo))
    c.hi[:] = list(hi) + [1] * (3 - len(hi))
    c.smoothing_steps, c.variable, c.estimate_relaxation, c.restrict_is_transpose = smoothing_steps, 1, 1, 1
    c.fe_degree_min, c.n_steps_min, c.mg_float = fe_degree_min, n_steps_min, int(mg_float)
    c.extrapolate, c.max_iter, c.restart, c.rhs_mode = int(extrapolate), max_iter, 30, rhs_mode
    c.compute_errors, c.tol, c.abs_tol, c.frequency = int(compute_errors), tol, abs_tol, frequency
    keep = []

    def arr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return _ptr(a)

    c.f_nodal, c.u0_nodal, c.v0_nodal = arr(f_nodal), arr(u0_nodal), arr(v0_nodal)
    c.fine_vertices, c.fine_coeff = arr(fine_vertices), arr(fine_coeff)
    res = OrcResult()
    its = np.zeros(n_slabs, dtype=np.int32)
    nf = [s << refine for s in c.subdiv[:dim]]
    nn = int(np.prod([n * p + 1 for n in nf]))
    nb = (r + 1 if ttype == DG else r) * n_steps
    u = np.zeros(nb * nn)
    v = np.zeros(nb * nn)
    u_all = np.zeros((n_slabs, nb * nn)) if keep_all else None
    _check(lib().orc_run_all(C.byref(c), C.byref(res), its.ctypes.data_as(_ip), _ptr(u), _ptr(v), _ptr(u_all)))
    return dict(iterations=its, total_iterations=res.total_iterations, n_levels=res.n_levels, linf=res.l8,
                l2=res.l2, h1=res.h1, n_dofs=res.n_dofs, n_cells=res.n_cells, u=u, v=v, u_all=u_all)
