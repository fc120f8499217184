"""Point functionals of the slab solution (stmg_solver_point_values,
tests/tp_01.cc:451-619): the GPU values against a numpy evaluation of the
downloaded slab solution (own point location by Newton on the Q1 map, own
Lagrange bases in space (Gauss-Lobatto points) and time (Radau-right for dG,
Lobatto for cGP, time_evaluation matrix of fe_time.h:250-267)), and against
the manufactured solution to the discretisation error."""
import numpy as np
import pytest

import meshes
from test_oracle_operator import gll_points

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def lagrange(pts, i, x):
    v = 1.0
    for j, pj in enumerate(pts):
        if j != i:
            v *= (x - pj) / (pts[i] - pj)
    return v


def time_points(dg, r):
    if dg:  # Radau with the right end point: roots of P_r - P_{r+1}
        P = np.polynomial.legendre.Legendre
        z = (P.basis(r) - P.basis(r + 1)).roots().real
    else:   # Lobatto
        inner = np.polynomial.legendre.Legendre.basis(r).deriv().roots().real if r > 1 else np.array([])
        z = np.concatenate([[-1.0], inner, [1.0]])
    return np.sort(0.5 * (z + 1.0))


def locate(X, n, y):
    """(cell coords, reference coords) of point y in the 2-D Q1 mesh with
    vertices X ((n0+1)(n1+1) x 2)."""
    V = X.reshape(n[1] + 1, n[0] + 1, 2)
    for cy in range(n[1]):
        for cx in range(n[0]):
            c = [V[cy, cx], V[cy, cx + 1], V[cy + 1, cx], V[cy + 1, cx + 1]]
            xi = np.array([0.5, 0.5])
            for _ in range(40):
                s, t = xi
                x = (1 - s) * (1 - t) * c[0] + s * (1 - t) * c[1] + (1 - s) * t * c[2] + s * t * c[3]
                J = np.column_stack([(1 - t) * (c[1] - c[0]) + t * (c[3] - c[2]),
                                     (1 - s) * (c[2] - c[0]) + s * (c[3] - c[1])])
                xi = xi + np.linalg.solve(J, y - x)
            if np.all(xi >= -1e-10) and np.all(xi <= 1 + 1e-10):
                return (cx, cy), np.clip(xi, 0, 1)
    raise AssertionError("point outside the mesh")


@pytest.mark.parametrize("problem,ttype,r,steps", [("heat", "DG", 1, 1), ("heat", "CGP", 2, 2), ("wave", "DG", 2, 1),
                                                   ("heat", "DG", 3, 2)])
def test_point_values_match_numpy_evaluation(problem, ttype, r, steps):
    import stmg
    n, p = (8, 8), r + 1
    X = meshes.vertices(2, n, distort=0.15, seed=71)
    tt = stmg.DG if ttype == "DG" else stmg.CGP
    s = stmg.Solver(dim=2, refine=3, degree=p, time_degree=r, time_type=tt,
                    problem=stmg.HEAT if problem == "heat" else stmg.WAVE, n_steps=steps, tau=1 / 16,
                    fe_degree_min=0 if tt == stmg.DG else 1, n_steps_min=max(1, steps // 2), fine_vertices=X)
    s.run(3)
    pts = np.array([[0.75, 0.1], [0.3, 0.62], [0.5, 0.5]])
    times, vals = s.point_values(pts)
    u, _ = s.solution(want_v=False)
    nt_step = (r + 1) if tt == stmg.DG else r
    N = s.n_nodes
    U = u.reshape(-1, N)
    # the slab's initial value (cGP's first node): the previous slab's last block
    s_prev = stmg.Solver(dim=2, refine=3, degree=p, time_degree=r, time_type=tt,
                         problem=stmg.HEAT if problem == "heat" else stmg.WAVE, n_steps=steps, tau=1 / 16,
                         fe_degree_min=0 if tt == stmg.DG else 1, n_steps_min=max(1, steps // 2), fine_vertices=X)
    s_prev.run(2)
    u_prev = s_prev.solution(want_v=False)[0].reshape(-1, N)[-1]
    xs, nn0 = gll_points(p), n[0] * p + 1
    samples = (r + 1) ** 2
    tq = time_points(tt == stmg.DG, r)
    ref = np.zeros_like(vals)
    for k, y in enumerate(pts):
        (cx, cy), xi = locate(X, n, y)
        wts, idx = [], []
        for ay in range(p + 1):
            for ax in range(p + 1):
                wts.append(lagrange(xs, ax, xi[0]) * lagrange(xs, ay, xi[1]))
                idx.append((cx * p + ax) + nn0 * (cy * p + ay))
        at = lambda vec: float(np.dot(wts, vec[idx]))
        for it in range(steps):
            nodes = [at(U[it * nt_step + q]) for q in range(nt_step)]
            if tt == stmg.CGP:
                nodes = [at(u_prev) if it == 0 else at(U[it * nt_step - 1])] + nodes
            for row in range(samples):
                ts = row / (samples - 1)
                ref[it * samples + row, k] = sum(lagrange(tq, q, ts) * nodes[q] for q in range(len(tq)))
    assert np.abs(vals - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-300)
    tau = 1 / 16
    assert np.allclose(times[:samples], 2 * steps * tau + tau * np.arange(samples) / (samples - 1))
    # against the manufactured solution u = sin(2 pi x) sin(2 pi y) sin(2 pi t)
    # (frequency 1) to the discretisation error
    if problem == "heat":
        ex = np.sin(2 * np.pi * pts[:, 0])[None, :] * np.sin(2 * np.pi * pts[:, 1])[None, :] * \
            np.sin(2 * np.pi * times)[:, None]
        assert np.abs(vals - ex).max() <= 5e-2
