"""Failure paths of the slab solve, injected on the host (no GPU fault):
non-convergence (the reference's AssertThrow after SolverFGMRES,
time_integrators.h:172-179) comes back as STMG_ERR_NOCONV, a non-finite
source as STMG_ERR_NONFINITE, and the solver is usable afterwards (the next
run from the same state gives the same iterations and solution as a fresh
solver)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ERR_NONFINITE, ERR_NOCONV = -5, -6


def _solver(**kw):
    import stmg
    base = dict(dim=2, refine=3, degree=2, time_degree=1, time_type=stmg.DG, n_steps=1, fe_degree_min=0,
                n_steps_min=1, rhs_mode=1, f_nodal=np.ones(17 * 17), tol=1e-10, abs_tol=1e-300)
    base.update(kw)
    return stmg.Solver(**base)


def _check_usable(s):
    """After a failure: a fresh start runs as on a fresh solver."""
    ref = _solver()
    ref.set_initial(np.zeros(ref.n_nodes))
    its_ref = ref.run(2)
    u_ref, _ = ref.solution()
    s.set_initial(np.zeros(s.n_nodes))
    s.set_source(np.ones(s.n_nodes))
    its = s.run(2)
    u, _ = s.solution()
    assert np.array_equal(its, its_ref)
    assert np.allclose(u, u_ref, rtol=0, atol=1e-12 * np.abs(u_ref).max())


def test_iteration_limit_gives_noconv_then_solver_recovers():
    import stmg
    s = _solver(max_iter=1)
    with pytest.raises(stmg.StmgError) as e:
        s.run(1)
    assert e.value.code == ERR_NOCONV
    s.set_control(1e-10, 1e-300, 200)
    _check_usable(s)


def test_nonfinite_source_gives_nonfinite_then_solver_recovers():
    import stmg
    s = _solver()
    f = np.ones(s.n_nodes)
    f[s.n_nodes // 2] = np.nan
    s.set_source(f)
    with pytest.raises(stmg.StmgError) as e:
        s.run(1)
    assert e.value.code == ERR_NONFINITE
    _check_usable(s)


def test_nonfinite_initial_state_gives_nonfinite_then_solver_recovers():
    import stmg
    s = _solver()
    u0 = np.zeros(s.n_nodes)
    u0[s.n_nodes // 3] = np.inf
    s.set_initial(u0)
    with pytest.raises(stmg.StmgError) as e:
        s.run(1)
    assert e.value.code == ERR_NONFINITE
    _check_usable(s)
