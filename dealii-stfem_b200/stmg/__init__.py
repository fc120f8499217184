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


def kernel_launches():
    n = C.c_longlong()
    check(lib().stmg_kernel_launches(C.byref(n)))
    return n.value


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


def time_weights(time_type, r, tau, n_steps, problem=HEAT):
    """Alpha, Beta, rK, rM, rV of one slab (stmg_time_weights)."""
    nt = (r + 1 if time_type == DG else r) * n_steps
    A, B = np.zeros((nt, nt)), np.zeros((nt, nt))
    rK, rM, rV = np.zeros(nt), np.zeros(nt), np.zeros(nt)
    check(lib().stmg_time_weights(time_type, r, C.c_double(tau), n_steps, problem, _ptr(A), _ptr(B), _ptr(rK),
                                  _ptr(rM), _ptr(rV)))
    return A, B, rK, rM, rV


def time_transfer(time_type, kind, r, n_steps):
    """Time transfer matrix of one slab (stmg_time_transfer): kind 0 the
    k-projection r-1 -> r on n_steps steps, kind 1 the tau-prolongation
    n_steps/2 -> n_steps steps; rows are the fine time dofs."""
    per = r + 1 if time_type == DG else r
    if kind == 0:
        shape = (per * n_steps, (per - 1) * n_steps)
    else:
        shape = (per * n_steps, per * n_steps // 2)
    P = np.zeros(shape)
    check(lib().stmg_time_transfer(time_type, kind, r, n_steps, _ptr(P)))
    return P


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

    def diagonal(self, dst, inverse=False, stream=None):
        """get_matrix_diagonal / get_matrix_diagonal_inverse into dst."""
        check(lib().stmg_op_diagonal(self.h, int(inverse), _dev(dst), _stream(stream)))


class Vanka:
    """stmg_vanka_t: cell-patch space-time Vanka smoother of one level."""

    def __init__(self, mesh, Alpha, Beta, compute=F32, storage=None):
        A = np.ascontiguousarray(Alpha, dtype=np.float64)
        B = np.ascontiguousarray(Beta, dtype=np.float64)
        if storage is None:
            storage = compute
        self.mesh, self.nt = mesh, A.shape[0]
        h = C.c_void_p()
        check(lib().stmg_vanka_create(mesh.h, self.nt, _ptr(A), _ptr(B), compute, storage, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.stmg_vanka_destroy(self.h)
            self.h = None

    def vmult(self, dst, src, stream=None):
        check(lib().stmg_vanka_vmult(self.h, _dev(dst), _dev(src), _stream(stream)))

    def step(self, op, omega, x, b, tmp, stream=None):
        """x += omega P (b - A x) (stmg_relax_step); tmp receives b - A x."""
        check(lib().stmg_relax_step(self.h, op.h, C.c_double(omega), _dev(x), _dev(b), _dev(tmp),
                                    _stream(stream)))


class Transfer:
    """stmg_transfer_t: h-transfer (fine, coarse meshes) or time transfer (P)."""

    def __init__(self, fine=None, coarse=None, nt=1, dtype=F64, mesh=None, P=None, R=None):
        h = C.c_void_p()
        if P is None:
            check(lib().stmg_transfer_h_create(fine.h, coarse.h, nt, dtype, C.byref(h)))
        else:
            P = np.ascontiguousarray(P, dtype=np.float64)
            Rm = None if R is None else np.ascontiguousarray(R, dtype=np.float64)
            self._keep = (P, Rm)
            check(lib().stmg_transfer_t_create(mesh.h, P.shape[0], P.shape[1], _ptr(P), _ptr(Rm), dtype, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.stmg_transfer_destroy(self.h)
            self.h = None

    def prolongate(self, dst, src, stream=None):
        check(lib().stmg_transfer_prolongate(self.h, _dev(dst), _dev(src), _stream(stream)))

    def prolongate_add(self, dst, src, stream=None):
        check(lib().stmg_transfer_prolongate_add(self.h, _dev(dst), _dev(src), _stream(stream)))

    def restrict_add(self, dst, src, stream=None):
        check(lib().stmg_transfer_restrict_add(self.h, _dev(dst), _dev(src), _stream(stream)))


class SolverConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("subdiv", C.c_int * 3), ("refine", C.c_int), ("degree", C.c_int),
        ("time_degree", C.c_int), ("time_type", C.c_int), ("problem", C.c_int), ("n_steps", C.c_int),
        ("tau", C.c_double), ("lo", C.c_double * 3), ("hi", C.c_double * 3),
        ("smoothing_steps", C.c_int), ("fe_degree_min", C.c_int), ("n_steps_min", C.c_int),
        ("mg_dtype", C.c_int), ("vanka_storage", C.c_int),
        ("tol", C.c_double), ("abs_tol", C.c_double),
        ("max_iter", C.c_int), ("restart", C.c_int), ("extrapolate", C.c_int),
        ("rhs_mode", C.c_int), ("frequency", C.c_double),
        ("fine_vertices", _dp), ("fine_coeff", _dp), ("f_nodal", _dp),
    ]


class Solver:
    """stmg_solver_t: FP64 FGMRES + space-time V-cycle slab solver."""

    def __init__(self, dim=2, subdiv=(1, 1, 1), refine=2, degree=2, time_degree=1, time_type=DG, problem=HEAT,
                 n_steps=1, tau=None, lo=(0, 0, 0), hi=(1, 1, 1), smoothing_steps=1, fe_degree_min=-1,
                 n_steps_min=-1, mg_dtype=F32, vanka_storage=None, tol=1e-12, abs_tol=1e-12, max_iter=200,
                 restart=30, extrapolate=True, rhs_mode=0, frequency=1.0, fine_vertices=None, fine_coeff=None,
                 f_nodal=None):
        c = SolverConfig()
        c.dim, c.refine, c.degree, c.time_degree = dim, refine, degree, time_degree
        c.subdiv[:] = list(subdiv) + [1] * (3 - len(subdiv))
        c.time_type, c.problem, c.n_steps = time_type, problem, n_steps
        c.tau = 2.0 ** -(refine + 1) if tau is None else tau
        c.lo[:] = list(lo) + [0] * (3 - len(lo))
        c.hi[:] = list(hi) + [1] * (3 - len(hi))
        c.smoothing_steps, c.fe_degree_min, c.n_steps_min = smoothing_steps, fe_degree_min, n_steps_min
        c.mg_dtype = mg_dtype
        c.vanka_storage = mg_dtype if vanka_storage is None else vanka_storage
        c.tol, c.abs_tol, c.max_iter, c.restart, c.extrapolate = tol, abs_tol, max_iter, restart, int(extrapolate)
        c.rhs_mode, c.frequency = rhs_mode, frequency
        keep = []

        def arr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return _ptr(a)

        c.fine_vertices, c.fine_coeff, c.f_nodal = arr(fine_vertices), arr(fine_coeff), arr(f_nodal)
        h = C.c_void_p()
        check(lib().stmg_solver_create(C.byref(c), C.byref(h)))
        self.h, self.cfg, self.tau = h, c, c.tau
        nn, nb, nl = C.c_longlong(), C.c_int(), C.c_int()
        check(lib().stmg_solver_info(self.h, C.byref(nn), C.byref(nb), C.byref(nl), None))
        self.n_nodes, self.n_blocks, self.n_levels = nn.value, nb.value, nl.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.stmg_solver_destroy(self.h)
            self.h = None

    def omegas(self):
        o = np.zeros(self.n_levels)
        check(lib().stmg_solver_info(self.h, None, None, None, _ptr(o)))
        return o

    def set_initial(self, u0=None, v0=None):
        u = None if u0 is None else np.ascontiguousarray(u0, dtype=np.float64)
        v = None if v0 is None else np.ascontiguousarray(v0, dtype=np.float64)
        check(lib().stmg_solver_set_initial(self.h, _ptr(u), _ptr(v)))

    def set_source(self, f_nodal):
        f = np.ascontiguousarray(f_nodal, dtype=np.float64)
        check(lib().stmg_solver_set_source(self.h, _ptr(f)))

    def point_values(self, points, samples_per_step=0, stream=None):
        """u of the last slab at the points for samples_per_step equidistant
        times per step (stmg_solver_point_values); returns (times, values)
        with values of shape (n_steps * samples, n_points)."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, self.cfg.dim)
        r = self.cfg.time_degree
        samples = samples_per_step if samples_per_step > 0 else (r + 1) ** 2
        rows = self.cfg.n_steps * samples
        times, vals = np.zeros(rows), np.zeros((rows, pts.shape[0]))
        check(lib().stmg_solver_point_values(self.h, pts.shape[0], _ptr(pts), samples, _ptr(times), _ptr(vals),
                                             _stream(stream)))
        return times, vals

    def set_control(self, tol, abs_tol, max_iter):
        """FGMRES ReductionControl of the following slabs (stmg_solver_set_control)."""
        check(lib().stmg_solver_set_control(self.h, C.c_double(tol), C.c_double(abs_tol), int(max_iter)))

    def run(self, n_slabs, stream=None):
        its = np.zeros(n_slabs, dtype=np.int32)
        check(lib().stmg_solver_run(self.h, n_slabs, its.ctypes.data_as(_ip), _stream(stream)))
        return its

    def solution(self, u=None, v=None, want_v=True):
        """Last slab's blocks; u, v may be preallocated (e.g. pinned) arrays."""
        if u is None:
            u = np.zeros(self.n_blocks * self.n_nodes)
        if v is None and want_v:
            v = np.zeros(self.n_blocks * self.n_nodes)
        check(lib().stmg_solver_solution(self.h, _ptr(u), _ptr(v)))
        return u, v

    def solution_async(self, u, v=None, stream=None):
        """Starts copying the last slab's blocks into the host arrays u (and
        v), which should be pinned; the copy overlaps later run() calls and
        is complete after solution_wait(). The arrays must stay alive until
        then."""
        check(lib().stmg_solver_solution_async(self.h, _ptr(u), _ptr(v), _stream(stream)))

    def solution_wait(self):
        check(lib().stmg_solver_solution_wait(self.h))

    def solve(self, x, rhs, stream=None):
        k = C.c_int()
        check(lib().stmg_solver_solve(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(rhs.data_ptr()), C.byref(k),
                                      _stream(stream)))
        return k.value

    def errors(self):
        """(linf, l2, h1) against the manufactured solution since set_initial."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(lib().stmg_solver_errors(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def gradient(self, u_obs, n_slabs=None, checkpoint_every=0, stream=None):
        """Misfit J = 1/2 sum_s |U_s - O_s|^2 of the next n_slabs slabs and
        dJ/dlog(kappa) per fine cell by the adjoint slab sweep
        (stmg_solver_gradient). u_obs: (n_slabs, n_blocks * n_nodes)."""
        obs = np.ascontiguousarray(u_obs, dtype=np.float64).reshape(-1)
        if n_slabs is None:
            n_slabs = obs.size // (self.n_blocks * self.n_nodes)
        assert obs.size == n_slabs * self.n_blocks * self.n_nodes
        ncells = int(np.prod([s << self.cfg.refine for s in list(self.cfg.subdiv)[:self.cfg.dim]]))
        grad = np.zeros(ncells)
        J = C.c_double()
        itf = np.zeros(n_slabs, dtype=np.int32)
        ita = np.zeros(n_slabs, dtype=np.int32)
        check(lib().stmg_solver_gradient(self.h, n_slabs, _ptr(obs), checkpoint_every, C.byref(J), _ptr(grad),
                                         itf.ctypes.data_as(_ip), ita.ctypes.data_as(_ip), _stream(stream)))
        return J.value, grad, itf, ita

    def gmg_vmult(self, dst, src, stream=None):
        check(lib().stmg_gmg_vmult(self.h, _dev(dst), _dev(src), _stream(stream)))

    def system_vmult(self, dst, src, stream=None):
        check(lib().stmg_solver_system_vmult(self.h, _dev(dst), _dev(src), _stream(stream)))
