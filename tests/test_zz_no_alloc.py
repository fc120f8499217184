"""stmg_op_vmult_box_noalloc: the space-time operator on a uniform box for
callers that cannot allocate device memory (a host application whose own
pool or fixed budget owns the GPU's memory, or a solver loop that must not
stall other streams on cudaMalloc's device-wide synchronisation). Its only
scratch, the tiles' face slots, sits in a fixed 16 MiB array inside the
library, so it is checked here against the allocating entry points
(stmg_mesh_create + stmg_op_create + stmg_op_vmult) on two calls in a row,
with the operator tests' tolerances: FP64 1e-12, FP32 2e-5 relative
(max-norm). This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import meshes

torch = pytest.importorskip("torch")

F64, F32 = 0, 1
ERR_ARG, ERR_SHAPE = -1, -3


def _entry():
    import stmg
    fn = stmg.lib().stmg_op_vmult_box_noalloc
    fn.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                   C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _call(dim, n, p, lo, hi, coeff_ptr, A, B, dtype, dst_ptr, src_ptr, stream_ptr):
    nc = (C.c_int * 3)(*(list(n) + [1] * (3 - len(n))))
    lo3 = (C.c_double * 3)(*(list(lo) + [0.0] * (3 - len(lo))))
    hi3 = (C.c_double * 3)(*(list(hi) + [1.0] * (3 - len(hi))))
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    dp = C.POINTER(C.c_double)
    return _entry()(dim, nc, p, lo3, hi3, coeff_ptr, A.shape[0], A.shape[1], A.ctypes.data_as(dp),
                    B.ctypes.data_as(dp), dtype, dst_ptr, src_ptr, stream_ptr)


def test_noalloc_rejects_bad_arguments_without_gpu_work():
    """Argument errors come back as status codes before any device work."""
    A = np.eye(2)
    assert _call(4, (2, 2), 2, (0, 0), (1, 1), None, A, A, F64, C.c_void_p(8), C.c_void_p(8), None) == ERR_ARG
    assert _call(2, (2, 2), 2, (0, 0), (1, 1), None, A, A, F64, None, C.c_void_p(8), None) == ERR_ARG
    assert _call(2, (2, 2), 2, (0, 0), (1, 1), None, A, A, 7, C.c_void_p(8), C.c_void_p(8), None) == ERR_ARG


CASES = [
    # dim, cells, degree, box, coefficient, (nt_out, nt_in)
    (2, (17, 9), 2, ((0.0, 0.0), (1.0, 0.5)), True, (4, 4)),
    (2, (12, 12), 4, ((0.0, 0.0), (1.0, 1.0)), False, (2, 2)),
    (3, (12, 10, 9), 2, ((0.0, 0.0, 0.0), (1.2, 1.0, 0.9)), True, (4, 4)),
    (3, (7, 6, 5), 3, ((-1.0, 0.0, 0.0), (1.0, 1.0, 1.0)), True, (3, 1)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"d{c[0]}-{'x'.join(map(str, c[1]))}-p{c[2]}-nt{c[5][0]}x{c[5][1]}")
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_matches_op_vmult_twice(case, prec):
    import stmg
    dim, n, p, (lo, hi), with_coeff, (nto, nti) = case
    rng = np.random.default_rng(sum(n) + 31 * p)
    coeff = meshes.log_uniform(int(np.prod(n)), 1e-2, 1e2) if with_coeff else None
    A = rng.standard_normal((nto, nti))
    B = rng.standard_normal((nto, nti))
    dtype, tdt, tol = (F64, torch.float64, 1e-12) if prec == "f64" else (F32, torch.float32, 2e-5)
    mesh = stmg.Mesh(dim, n, p, lo=lo, hi=hi, coeff=coeff, coeff_mode=1 if with_coeff else 0)
    op = stmg.Operator(mesh, A, B, dtype=dtype)
    N = mesh.n_nodes
    mask = meshes.boundary_mask(dim, n, p)
    dev_coeff = None if coeff is None else torch.from_numpy(coeff).to("cuda", tdt)
    stream = torch.cuda.current_stream()
    for call in range(2):  # the second call reuses what the first left in the scratch
        src = torch.from_numpy(meshes.random_block_vector(nti, N, mask, seed=call + 1)).to("cuda", tdt)
        ref = torch.empty(nto * N, device="cuda", dtype=tdt)
        out = torch.full((nto * N,), float("nan"), device="cuda", dtype=tdt)
        op.vmult(ref, src)
        rc = _call(dim, n, p, lo, hi, None if dev_coeff is None else C.c_void_p(dev_coeff.data_ptr()), A, B, dtype,
                   C.c_void_p(out.data_ptr()), C.c_void_p(src.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0, stmg.lib().stmg_last_error().decode()
        torch.cuda.synchronize()
        r, o = ref.double().cpu().numpy(), out.double().cpu().numpy()
        assert np.all(np.isfinite(o))
        assert np.abs(o - r).max() <= tol * max(np.abs(r).max(), 1e-300), (call, np.abs(o - r).max())


@pytest.mark.gpu
def test_noalloc_rejects_mesh_beyond_scratch_limit():
    """A mesh whose face slots exceed the fixed scratch is refused with a
    clear message, before any kernel runs."""
    import stmg
    A = np.eye(4)
    x = torch.zeros(4, device="cuda", dtype=torch.float32)
    rc = _call(3, (64, 64, 64), 2, (0, 0, 0), (1, 1, 1), None, A, A, F32, C.c_void_p(x.data_ptr()),
               C.c_void_p(x.data_ptr()), None)
    assert rc == ERR_SHAPE
    assert "scratch" in stmg.lib().stmg_last_error().decode()
