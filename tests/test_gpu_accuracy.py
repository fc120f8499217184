"""Accuracy of the FP32 V-cycle inside the FP64 FGMRES (tests/tp_01.cc:
767,776-777 run the reference as test<double, float>): the slab solutions of
the FP32-multigrid solve, converged to a relative residual of 1e-8, against

* a converged all-FP64 GPU solve (FP64 multigrid, 1e-12) of the large heat
  configuration's shape scaled down to 16^3 Q2 cells, dG(3), dt = 1/8,
  per-cell kappa = 10^U(-1, 1), nodal source f ~ N(0, 1);
* the oracle's all-FP64 solve (1e-13) of the same shape on 8^3 cells;
* the distorted Q3 (dG(2)) and the wave (dG(2), FP32 and BF16 Vanka
  storage) configurations' shapes on 4^3 cells against a converged all-FP64
  GPU solve.

The bar is the 1e-7 relative error (2-norm, per slab) that the FP32
multigrid solve of the large heat configuration is held to.
"""
import numpy as np
import pytest

import meshes
import oracle_py as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

BAR = 1e-7


def _heat_inputs(n, seed=20261203):
    rng = np.random.default_rng(seed)
    kappa = 10.0 ** rng.uniform(-1, 1, n ** 3)
    f = rng.standard_normal((2 * n + 1) ** 3)
    return kappa, f


def _slabs(s, n_slabs, init=None):
    if init is not None:
        s.set_initial(*init)
    out = []
    for _ in range(n_slabs):
        s.run(1)
        out.append(s.solution(want_v=False)[0])
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_fp32_mg_matches_converged_fp64_heat_16cube():
    import stmg
    n, refine = 16, 4
    kappa, f = _heat_inputs(n)
    kw = dict(dim=3, refine=refine, degree=2, time_degree=3, time_type=stmg.DG, problem=stmg.HEAT, n_steps=1,
              tau=1 / 8, rhs_mode=1, f_nodal=f, fine_coeff=kappa, abs_tol=1e-300, max_iter=1000)
    u32 = _slabs(stmg.Solver(mg_dtype=stmg.F32, tol=1e-8, **kw), 3)
    u64 = _slabs(stmg.Solver(mg_dtype=stmg.F64, tol=1e-8, **kw), 3)
    uref = _slabs(stmg.Solver(mg_dtype=stmg.F64, tol=1e-12, **kw), 3)
    for a, b, r in zip(u32, u64, uref):
        assert _rel(a, r) <= BAR, _rel(a, r)
        # and against the all-FP64 solve to the same tolerance
        assert _rel(a, b) <= BAR, _rel(a, b)


def test_fp32_mg_matches_oracle_fp64_heat_8cube():
    import stmg
    n, refine = 8, 3
    kappa, f = _heat_inputs(n, seed=5)
    common = dict(dim=3, refine=refine, n_steps=1, tau=1 / 8, rhs_mode=1, f_nodal=f, fine_coeff=kappa,
                  abs_tol=1e-300)
    ref = orc.run(p=2, r=3, ttype=orc.DG, problem=orc.HEAT, n_slabs=2, mg_float=False, tol=1e-13,
                  compute_errors=False, **common)
    s = stmg.Solver(degree=2, time_degree=3, time_type=stmg.DG, problem=stmg.HEAT, mg_dtype=stmg.F32, tol=1e-8,
                    **common)
    u = _slabs(s, 2)[-1]
    assert _rel(u, ref["u"]) <= BAR, _rel(u, ref["u"])


def test_fp32_mg_matches_converged_fp64_distorted_q3():
    import stmg
    n, refine = 4, 2
    X = meshes.vertices(3, (n, n, n), distort=0.2, seed=41)
    kappa = meshes.log_uniform(n ** 3, 1e-2, 1e2, seed=42)
    kw = dict(dim=3, refine=refine, degree=3, time_degree=2, time_type=stmg.DG, problem=stmg.HEAT, n_steps=1,
              tau=1 / 32, rhs_mode=1, f_nodal=np.ones((3 * n + 1) ** 3), fine_coeff=kappa, fine_vertices=X,
              abs_tol=1e-300, max_iter=1000)
    u32 = _slabs(stmg.Solver(mg_dtype=stmg.F32, tol=1e-8, **kw), 3)
    uref = _slabs(stmg.Solver(mg_dtype=stmg.F64, tol=1e-12, **kw), 3)
    for a, r in zip(u32, uref):
        assert _rel(a, r) <= BAR, _rel(a, r)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_fp32_mg_matches_converged_fp64_wave(storage):
    import stmg
    n, refine = 4, 2
    c2 = np.random.default_rng(43).choice([0.5, 1.0, 4.0], size=n ** 3)
    X = meshes.vertices(3, (2 * n, 2 * n, 2 * n))
    u0 = np.exp(-np.sum((X - 0.5) ** 2, axis=1) / 0.01)
    u0[meshes.boundary_mask(3, (n, n, n), 2)] = 0.0
    init = (u0, np.zeros_like(u0))
    kw = dict(dim=3, refine=refine, degree=2, time_degree=2, time_type=stmg.DG, problem=stmg.WAVE, n_steps=1,
              tau=1 / 128, rhs_mode=2, fine_coeff=c2, abs_tol=1e-300, max_iter=1000)
    st = stmg.F32 if storage == "f32" else stmg.BF16
    u32 = _slabs(stmg.Solver(mg_dtype=stmg.F32, vanka_storage=st, tol=1e-8, **kw), 4, init)
    uref = _slabs(stmg.Solver(mg_dtype=stmg.F64, tol=1e-12, **kw), 4, init)
    for a, r in zip(u32, uref):
        assert _rel(a, r) <= BAR, _rel(a, r)
