"""Adjoint gradient of the space-time misfit (stmg_solver_gradient, heat):
dJ/dlog(kappa) per cell against central finite differences of J computed by
forward GPU solves, against finite differences of J from the oracle's FP64
solves, and independent of the checkpoint spacing. Tolerances: 1e-6
relative for the GPU FD check (h = 1e-4, FP64 multigrid, solves to 1e-13),
1e-5 against the oracle."""
import numpy as np
import pytest

import meshes
import oracle_py as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SLABS = 3
BASE = dict(dim=2, refine=3, degree=2, time_degree=1, n_steps=1, tau=1.0 / 8, fe_degree_min=0, n_steps_min=1,
            tol=1e-13, abs_tol=1e-300, rhs_mode=1)


def _problem(seed=3):
    rng = np.random.default_rng(seed)
    ncell = 64
    theta = rng.normal(0.0, 0.5, ncell)
    nn = (8 * 2 + 1) ** 2
    f = rng.standard_normal(nn)
    f[meshes.boundary_mask(2, (8, 8), 2)] = 0.0
    obs = 0.1 * rng.standard_normal((SLABS, 2 * nn))
    obs[:, np.tile(meshes.boundary_mask(2, (8, 8), 2), 2)] = 0.0
    return theta, f, obs


def _solver(theta, f, **kw):
    import stmg
    return stmg.Solver(time_type=stmg.DG, problem=stmg.HEAT, mg_dtype=stmg.F64, f_nodal=f, fine_coeff=np.exp(theta),
                       **BASE, **kw)


def _misfit_gpu(theta, f, obs):
    s = _solver(theta, f)
    J = 0.0
    for k in range(SLABS):
        s.run(1)
        u, _ = s.solution(want_v=False)
        J += 0.5 * float(np.sum((u - obs[k]) ** 2))
    return J


def _misfit_oracle(theta, f, obs):
    J = 0.0
    for k in range(SLABS):
        r = orc.run(dim=2, refine=3, p=2, r=1, ttype=orc.DG, problem=orc.HEAT, n_steps=1, tau=1.0 / 8, n_slabs=k + 1,
                    fe_degree_min=0, n_steps_min=1, mg_float=False, tol=1e-13, abs_tol=1e-300, rhs_mode=1, f_nodal=f,
                    fine_coeff=np.exp(theta), compute_errors=False)
        J += 0.5 * float(np.sum((r["u"] - obs[k]) ** 2))
    return J


def test_gradient_matches_finite_differences():
    theta, f, obs = _problem()
    J, g, itf, ita = _solver(theta, f).gradient(obs)
    assert np.all(itf > 0) and np.all(ita > 0)
    assert abs(J - _misfit_gpu(theta, f, obs)) <= 1e-10 * J
    rng = np.random.default_rng(11)
    h = 1e-4
    for _ in range(3):
        d = rng.standard_normal(theta.size)
        d /= np.linalg.norm(d)
        fd = (_misfit_gpu(theta + h * d, f, obs) - _misfit_gpu(theta - h * d, f, obs)) / (2 * h)
        assert abs(g @ d - fd) <= 1e-6 * max(abs(fd), abs(g @ d)), (g @ d, fd)


def test_gradient_matches_oracle_solves():
    theta, f, obs = _problem(seed=5)
    J, g, _, _ = _solver(theta, f).gradient(obs)
    assert abs(J - _misfit_oracle(theta, f, obs)) <= 1e-8 * J
    d = np.random.default_rng(13).standard_normal(theta.size)
    d /= np.linalg.norm(d)
    h = 1e-4
    fd = (_misfit_oracle(theta + h * d, f, obs) - _misfit_oracle(theta - h * d, f, obs)) / (2 * h)
    assert abs(g @ d - fd) <= 1e-5 * max(abs(fd), abs(g @ d)), (g @ d, fd)


def test_gradient_independent_of_checkpoints():
    theta, f, obs = _problem(seed=7)
    J1, g1, _, _ = _solver(theta, f).gradient(obs, checkpoint_every=1)
    J2, g2, _, _ = _solver(theta, f).gradient(obs, checkpoint_every=SLABS)
    J3, g3, _, _ = _solver(theta, f).gradient(obs)  # ceil(sqrt(n_slabs))
    assert J1 == J2 == J3
    assert np.linalg.norm(g1 - g2) <= 1e-12 * np.linalg.norm(g1)
    assert np.linalg.norm(g1 - g3) <= 1e-12 * np.linalg.norm(g1)


def test_gradient_3d_matches_finite_differences():
    """3-D (4^3 Q2 cells, dG(1), 3 slabs, checkpoints every 2 slabs)."""
    import stmg
    rng = np.random.default_rng(17)
    n = 4
    theta = rng.normal(0.0, 0.5, n ** 3)
    nn = (2 * n + 1) ** 3
    mask = meshes.boundary_mask(3, (n, n, n), 2)
    f = rng.standard_normal(nn)
    f[mask] = 0.0
    obs = 0.1 * rng.standard_normal((SLABS, 2 * nn))
    obs[:, np.tile(mask, 2)] = 0.0
    kw = dict(BASE, dim=3, refine=2)

    def solver(th):
        return stmg.Solver(time_type=stmg.DG, problem=stmg.HEAT, mg_dtype=stmg.F64, f_nodal=f,
                           fine_coeff=np.exp(th), **kw)

    def misfit(th):
        s = solver(th)
        J = 0.0
        for k in range(SLABS):
            s.run(1)
            u, _ = s.solution(want_v=False)
            J += 0.5 * float(np.sum((u - obs[k]) ** 2))
        return J

    J, g, _, _ = solver(theta).gradient(obs, checkpoint_every=2)
    d = rng.standard_normal(theta.size)
    d /= np.linalg.norm(d)
    h = 1e-4
    fd = (misfit(theta + h * d) - misfit(theta - h * d)) / (2 * h)
    assert abs(g @ d - fd) <= 1e-6 * max(abs(fd), abs(g @ d)), (g @ d, fd)


def test_autograd_wrapper_gradcheck_small():
    """The torch.autograd.Function wrapper (stmg.adjoint.misfit) passes
    torch.autograd.gradcheck (central differences in every parameter) on a
    small problem: 2-D 4x4 Q2 cells, dG(1), three slabs."""
    import stmg
    from stmg.adjoint import misfit
    rng = np.random.default_rng(81)
    n = 4
    nn = (2 * n + 1) ** 2
    f = rng.standard_normal(nn)
    f[meshes.boundary_mask(2, (n, n), 2)] = 0.0
    obs = 0.1 * rng.standard_normal((SLABS, 2 * nn))
    obs[:, np.tile(meshes.boundary_mask(2, (n, n), 2), 2)] = 0.0
    kw = dict(BASE, refine=2)

    def make(kappa):
        return stmg.Solver(time_type=stmg.DG, problem=stmg.HEAT, mg_dtype=stmg.F64, f_nodal=f, fine_coeff=kappa, **kw)

    theta = torch.tensor(rng.normal(0.0, 0.5, n * n), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda th: misfit(th, make, obs), (theta,), eps=1e-5, atol=1e-9, rtol=1e-5)


def test_autograd_wrapper_directional_fd_3d():
    """J.backward() through the wrapper against central differences of
    forward solves on random unit directions (3-D 4^3 Q2 cells, dG(1), four
    slabs, checkpoints every two slabs)."""
    import stmg
    from stmg.adjoint import misfit, misfit_value
    rng = np.random.default_rng(82)
    n, S = 4, 4
    nn = (2 * n + 1) ** 3
    f = np.ones(nn)
    obs = 0.05 * rng.standard_normal((S, 2 * nn))
    obs[:, np.tile(meshes.boundary_mask(3, (n, n, n), 2), 2)] = 0.0
    kw = dict(BASE, dim=3, refine=2, tau=1 / 16)

    def make(kappa):
        return stmg.Solver(time_type=stmg.DG, problem=stmg.HEAT, mg_dtype=stmg.F64, f_nodal=f, fine_coeff=kappa, **kw)

    theta = torch.zeros(n ** 3, dtype=torch.float64, requires_grad=True)
    J = misfit(theta, make, obs, 2)
    J.backward()
    g = theta.grad.numpy()
    h = 1e-4
    for _ in range(3):
        d = rng.standard_normal(n ** 3)
        d /= np.linalg.norm(d)
        fd = (misfit_value(h * d, make, obs) - misfit_value(-h * d, make, obs)) / (2 * h)
        assert abs(g @ d - fd) <= 1e-6 * abs(fd), (g @ d, fd)
