"""Pins the oracle's space-time operator without the reference's help.

The reference has no operator-level golden vector (its tests print solver
iteration counts and error norms only), so the oracle's sum-factorised apply
(oracle/space.cc, st_apply / mf_apply, following tests/include/operators.h:
94-152 and 487-548) is checked here against two independent constructions:

* the global matrices K and M assembled in scipy from the oracle's element
  matrices (a quadrature loop over basis functions, no sum factorisation),
  with the Dirichlet rows and columns removed as the matrix-free operator
  treats them (read as zero, written as zero), and the space-time operator
  (A (x) K + B (x) M) applied as a sparse product;
* on box cells, element matrices built in numpy from the 1-D Lagrange basis
  on Gauss-Lobatto points (FE_Q(p)) and exact 1-D integrals, as tensor
  products.

CPU only.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import meshes
import oracle_py as orc


def cell_dofs(dim, n, p, c):
    """Global lexicographic node numbers of cell c's (p+1)^dim local nodes
    (local index ax + (p+1) ay + (p+1)^2 az, as the oracle numbers them)."""
    p1 = p + 1
    nn = [k * p + 1 for k in n[:dim]] + [1] * (3 - dim)
    ci = [c % n[0], (c // n[0]) % n[1] if dim > 1 else 0, c // (n[0] * n[1]) if dim > 2 else 0]
    loc = np.arange(p1 ** dim)
    a = [loc % p1, (loc // p1) % p1 if dim > 1 else 0 * loc, loc // (p1 * p1) if dim > 2 else 0 * loc]
    return (ci[0] * p + a[0]) + nn[0] * ((ci[1] * p + a[1]) + nn[1] * (ci[2] * p + a[2]))


def assembled(mesh, dim, n, p):
    """Global K, M (scipy CSR) from the oracle's element matrices, Dirichlet
    rows and columns zeroed."""
    ncell = int(np.prod(n[:dim]))
    nd = (p + 1) ** dim
    rows, cols, kv, mv = [], [], [], []
    for c in range(ncell):
        K, M = mesh.element_matrices(c)
        g = cell_dofs(dim, n, p, c)
        rows.append(np.repeat(g, nd))
        cols.append(np.tile(g, nd))
        kv.append(K.reshape(-1))
        mv.append(M.reshape(-1))
    N = mesh.n_nodes
    r, cc = np.concatenate(rows), np.concatenate(cols)
    keep = sp.diags((~meshes.boundary_mask(dim, n, p)).astype(float))
    Kg = keep @ sp.csr_matrix((np.concatenate(kv), (r, cc)), shape=(N, N)) @ keep
    Mg = keep @ sp.csr_matrix((np.concatenate(mv), (r, cc)), shape=(N, N)) @ keep
    return Kg.tocsr(), Mg.tocsr()


def st_apply_assembled(Kg, Mg, A, B, x):
    nt, N = A.shape[1], Kg.shape[0]
    X = x.reshape(nt, N)
    KX = np.stack([Kg @ X[i] for i in range(nt)])
    MX = np.stack([Mg @ X[i] for i in range(nt)])
    return (A @ KX + B @ MX).reshape(-1)


CASES = [
    # dim, cells, p, distortion, coefficient mode (0 none, 1 per cell, 2 per quadrature point)
    (2, (5, 4), 1, 0.0, 0),
    (2, (5, 4), 2, 0.2, 1),
    (2, (4, 3), 3, 0.2, 2),
    (2, (3, 3), 4, 0.15, 1),
    (3, (3, 3, 2), 1, 0.2, 1),
    (3, (3, 2, 2), 2, 0.0, 2),
    (3, (3, 2, 2), 2, 0.2, 1),
    (3, (2, 2, 2), 3, 0.2, 2),
]


@pytest.mark.parametrize("dim,n,p,distort,cmode", CASES, ids=lambda v: str(v))
@pytest.mark.parametrize("transpose", [False, True])
def test_sum_factorised_apply_matches_assembled(dim, n, p, distort, cmode, transpose):
    ncell = int(np.prod(n[:dim]))
    X = meshes.vertices(dim, n, distort=distort, seed=31) if distort else None
    coeff = None
    if cmode == 1:
        coeff = meshes.log_uniform(ncell, 1e-2, 1e2, seed=32)
    elif cmode == 2:
        coeff = meshes.log_uniform(ncell * (p + 1) ** dim, 1e-1, 1e1, seed=33)
    mesh = orc.Mesh(dim, n, p, vertices=X, coeff=coeff, coeff_mode=cmode)
    Kg, Mg = assembled(mesh, dim, list(n) + [1] * (3 - len(n)), p)
    rng = np.random.default_rng(34)
    nt = 3
    A, B = rng.standard_normal((nt, nt)), rng.standard_normal((nt, nt))
    x = meshes.random_block_vector(nt, mesh.n_nodes, meshes.boundary_mask(dim, n, p), seed=35)
    ref = st_apply_assembled(Kg, Mg, A.T if transpose else A, B.T if transpose else B, x)
    got = mesh.st_apply(A, B, x, transpose=transpose)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    # the n_t x 1 form (vmult(BlockVector&, const Vector&), operators.h:182-187)
    a, b = rng.standard_normal((nt, 1)), rng.standard_normal((nt, 1))
    v = x[: mesh.n_nodes]
    ref1 = np.concatenate([a[j, 0] * (Kg @ v) + b[j, 0] * (Mg @ v) for j in range(nt)])
    got1 = mesh.st_apply_vec(a, b, v)
    assert np.abs(got1 - ref1).max() <= 1e-13 * np.abs(ref1).max()


def gll_points(p):
    """Gauss-Lobatto points on [0, 1] (the support points of FE_Q(p))."""
    inner = np.polynomial.legendre.Legendre.basis(p).deriv().roots() if p > 1 else np.array([])
    return np.concatenate([[0.0], 0.5 * (np.sort(inner.real) + 1.0), [1.0]])


def lagrange_1d(p):
    """Mass and stiffness matrices of the 1-D Lagrange basis on the unit
    interval, integrated exactly (Gauss rule of p + 2 points)."""
    x = gll_points(p)
    polys = []
    for i in range(p + 1):
        others = np.delete(x, i)
        polys.append(np.polynomial.Polynomial.fromroots(others) / np.prod(x[i] - others))
    q, w = np.polynomial.legendre.leggauss(p + 2)
    q, w = 0.5 * (q + 1.0), 0.5 * w
    V = np.array([pl(q) for pl in polys])
    D = np.array([pl.deriv()(q) for pl in polys])
    return (V * w) @ V.T, (D * w) @ D.T


@pytest.mark.parametrize("dim,p", [(2, 1), (2, 2), (2, 3), (2, 4), (2, 5), (3, 1), (3, 2), (3, 3), (3, 4)])
def test_box_element_matrices_match_tensor_products(dim, p):
    n = [3, 2, 2][:dim]
    lo, hi = (0.0, -1.0, 0.5), (1.5, 1.0, 1.25)
    h = [(hi[d] - lo[d]) / n[d] for d in range(dim)]
    kappa = 2.5
    mesh = orc.Mesh(dim, n, p, lo=lo, hi=hi, coeff=np.full(int(np.prod(n)), kappa), coeff_mode=1)
    M1, K1 = lagrange_1d(p)
    Ms = [M1 * h[d] for d in range(dim)]
    Ks = [K1 / h[d] for d in range(dim)]

    def kron_all(mats):  # x fastest: kron(z, kron(y, x))
        out = mats[0]
        for m in mats[1:]:
            out = np.kron(m, out)
        return out

    M = kron_all(Ms)
    K = sum(kron_all([Ks[d] if d == j else Ms[d] for d in range(dim)]) for j in range(dim)) * kappa
    Ko, Mo = mesh.element_matrices(int(np.prod(n)) - 1)
    assert np.abs(Mo - M).max() <= 1e-13 * np.abs(M).max()
    assert np.abs(Ko - K).max() <= 1e-13 * np.abs(K).max()
