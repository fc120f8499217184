"""Space-time operator on the GPU against the CPU oracle (SystemMatrix::vmult,
Tvmult, vmult_add of tests/include/operators.h:94-187).
FP64: 1e-12 relative (max-norm); FP32: 2e-5 relative."""
import numpy as np
import pytest

import meshes
import oracle_py as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = [
    # dim, cells, p, distort, coeff_mode, time (type, r, steps)
    (2, (4, 4), 1, 0.0, 0, (orc.DG, 1, 1)),
    (2, (5, 3), 2, 0.0, 1, (orc.DG, 1, 2)),
    (2, (6, 6), 3, 0.2, 1, (orc.CGP, 2, 1)),
    (2, (3, 4), 4, 0.2, 2, (orc.DG, 3, 1)),
    (2, (17, 9), 2, 0.0, 0, (orc.DG, 3, 4)),
    (3, (3, 2, 2), 1, 0.0, 0, (orc.DG, 1, 1)),
    (3, (5, 4, 3), 2, 0.0, 1, (orc.DG, 3, 1)),
    (3, (9, 5, 4), 2, 0.2, 1, (orc.DG, 2, 1)),
    (3, (4, 3, 3), 2, 0.15, 2, (orc.CGP, 2, 2)),
    (3, (3, 3, 2), 3, 0.2, 1, (orc.DG, 2, 1)),
    (3, (2, 2, 2), 4, 0.0, 1, (orc.DG, 1, 1)),
    # several big tiles of degree 3 and 4 (shell faces and the plane fix-up)
    (3, (9, 5, 3), 3, 0.2, 1, (orc.DG, 2, 1)),
    (3, (5, 5, 3), 4, 0.1, 1, (orc.DG, 1, 1)),
    # undistorted boxes with a coefficient per quadrature point
    (2, (6, 5), 2, 0.0, 2, (orc.DG, 1, 2)),
    (3, (5, 4, 3), 2, 0.0, 2, (orc.DG, 3, 1)),
    (3, (3, 3, 2), 3, 0.0, 2, (orc.CGP, 2, 1)),
]


def build(case):
    dim, n, p, distort, cmode, (tt, r, steps) = case
    X = meshes.vertices(dim, n, distort=distort)
    ncell = int(np.prod(n))
    nq = (p + 1) ** dim
    coeff = None
    if cmode == 1:
        coeff = meshes.log_uniform(ncell, 1e-2, 1e2)
    elif cmode == 2:
        coeff = meshes.log_uniform(ncell * nq, 0.1, 10)
    om = orc.Mesh(dim, n, p, vertices=X, coeff=coeff, coeff_mode=cmode)
    import stmg
    gm = stmg.Mesh(dim, n, p, vertices=X, coeff=coeff, coeff_mode=cmode)
    A, B, rK, rM, _ = orc.time_weights(tt, r, 0.25, steps, orc.HEAT)
    return om, gm, A, B, rK, rM


def rel_err(x, y):
    return np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"d{c[0]}-{'x'.join(map(str, c[1]))}-p{c[2]}-dist{c[3]}-c{c[4]}")
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_operator_matches_oracle(case, prec):
    import stmg
    om, gm, A, B, rK, rM = build(case)
    dim, n, p = case[0], case[1], case[2]
    nt = A.shape[0]
    mask = meshes.boundary_mask(dim, n, p)
    src = meshes.random_block_vector(nt, om.n_nodes, mask)
    dt = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-12 if prec == "f64" else 2e-5
    op = stmg.Operator(gm, A, B, dtype=stmg.F64 if prec == "f64" else stmg.F32)
    s = torch.tensor(src, dtype=dt, device="cuda")
    d = torch.full_like(s, 7.0)
    # vmult
    op.vmult(d, s)
    ref = om.st_apply(A, B, src)
    assert rel_err(d.double().cpu().numpy(), ref) < tol
    # Tvmult
    op.Tvmult(d, s)
    refT = om.st_apply(A, B, src, transpose=True)
    assert rel_err(d.double().cpu().numpy(), refT) < tol
    # vmult_add with the n x 1 rhs form (operators.h:155-180)
    if not np.all(rK == 0) or not np.all(rM == 0):
        opv = stmg.Operator(gm, rK.reshape(-1, 1), rM.reshape(-1, 1), dtype=op.dtype)
        v = torch.tensor(src[:om.n_nodes], dtype=dt, device="cuda")
        base = meshes.random_block_vector(nt, om.n_nodes, mask, seed=3)
        dv = torch.tensor(base, dtype=dt, device="cuda")
        opv.vmult_add(dv, v)
        refv = om.st_apply_vec(rK, rM, src[:om.n_nodes], dst=base)
        assert rel_err(dv.double().cpu().numpy(), refv) < tol * 10


def test_operator_deterministic():
    import stmg
    om, gm, A, B, _, _ = build(CASES[7])
    src = meshes.random_block_vector(A.shape[0], om.n_nodes, meshes.boundary_mask(3, CASES[7][1], 2))
    op = stmg.Operator(gm, A, B, dtype=stmg.F32)
    s = torch.tensor(src, dtype=torch.float32, device="cuda")
    d1, d2 = torch.empty_like(s), torch.empty_like(s)
    op.vmult(d1, s)
    op.vmult(d2, s)
    assert torch.equal(d1, d2)


def _assembled_diagonals(om, dim, n, p):
    """Diagonals of K and M summed over the oracle's element matrices
    (interior nodes; Dirichlet rows are left to the caller)."""
    from test_oracle_operator import cell_dofs
    nn = list(n) + [1] * (3 - len(n))
    dK, dM = np.zeros(om.n_nodes), np.zeros(om.n_nodes)
    for c in range(int(np.prod(n))):
        K, M = om.element_matrices(c)
        g = cell_dofs(dim, nn, p, c)
        np.add.at(dK, g, np.diag(K))
        np.add.at(dM, g, np.diag(M))
    return dK, dM


@pytest.mark.parametrize("case", [CASES[i] for i in (1, 2, 3, 7, 8, 9, 14)],
                         ids=lambda c: f"d{c[0]}-{'x'.join(map(str, c[1]))}-p{c[2]}-dist{c[3]}-c{c[4]}")
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_operator_diagonal_matches_assembled(case, prec):
    """stmg_op_diagonal (get_matrix_diagonal[_inverse], operators.h:188-215)
    against the diagonals of the assembled element matrices; Dirichlet rows
    of diag(K) and diag(M) are 1; the inverse follows the reference's
    composition diag(K)^+ / Alpha(i,i) + diag(M)^+ / Beta(i,i)."""
    import stmg
    om, gm, A, B, _, _ = build(case)
    dim, n, p = case[0], case[1], case[2]
    nt = A.shape[0]
    dK, dM = _assembled_diagonals(om, dim, n, p)
    bd = meshes.boundary_mask(dim, n, p)
    dK[bd], dM[bd] = 1.0, 1.0
    ref = np.concatenate([A[j, j] * dK + B[j, j] * dM for j in range(nt)])
    eps = np.finfo(np.float64 if prec == "f64" else np.float32).eps
    inv = lambda d: np.where(np.abs(d) > np.sqrt(eps), 1.0 / d, 1.0)
    ref_inv = np.concatenate([inv(dK) / A[j, j] + inv(dM) / B[j, j] for j in range(nt)])
    op = stmg.Operator(gm, A, B, dtype=stmg.F64 if prec == "f64" else stmg.F32)
    dt = torch.float64 if prec == "f64" else torch.float32
    d = torch.zeros(nt * om.n_nodes, dtype=dt, device="cuda")
    tol = 1e-12 if prec == "f64" else 2e-6
    op.diagonal(d)
    assert rel_err(d.double().cpu().numpy(), ref) < tol
    op.diagonal(d, inverse=True)
    assert rel_err(d.double().cpu().numpy(), ref_inv) < tol


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_relax_step_matches_composition(prec):
    """stmg_relax_step: x + omega P (b - A x), against the operator and the
    smoother applied one after the other."""
    import stmg
    om, gm, A, B, _, _ = build(CASES[7])
    dim, n, p = 3, CASES[7][1], 2
    nt = A.shape[0]
    mask = meshes.boundary_mask(dim, n, p)
    dt = torch.float64 if prec == "f64" else torch.float32
    mode = stmg.F64 if prec == "f64" else stmg.F32
    op = stmg.Operator(gm, A, B, dtype=mode)
    vk = stmg.Vanka(gm, A, B, compute=mode, storage=mode)
    x = torch.tensor(meshes.random_block_vector(nt, om.n_nodes, mask, seed=61), dtype=dt, device="cuda")
    b = torch.tensor(meshes.random_block_vector(nt, om.n_nodes, mask, seed=62), dtype=dt, device="cuda")
    omega = 0.7
    r, pr = torch.empty_like(x), torch.empty_like(x)
    op.vmult(r, x)
    r = b - r
    vk.vmult(pr, r)
    ref = x + omega * pr
    tmp = torch.empty_like(x)
    x1 = x.clone()
    vk.step(op, omega, x1, b, tmp)
    torch.cuda.synchronize()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert torch.linalg.norm(x1 - ref) <= tol * torch.linalg.norm(ref)
    assert torch.linalg.norm(tmp - r) <= tol * torch.linalg.norm(r)


TINY_CASES = [c for c in CASES if c[0] == 3 and c[2] == 2] + [
    (3, (13, 9, 7), 2, 0.1, 1, (orc.DG, 3, 1)),
    (3, (12, 8, 6), 2, 0.0, 2, (orc.DG, 3, 1)),
    (3, (8, 8, 8), 2, 0.0, 1, (orc.DG, 2, 1)),
    (3, (7, 4, 5), 2, 0.0, 0, (orc.CGP, 2, 1)),
]


@pytest.mark.parametrize("case", TINY_CASES, ids=lambda c: f"{'x'.join(map(str, c[1]))}-dist{c[3]}-c{c[4]}-r{c[5][1]}")
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_operator_small_tiles_match_regular_tiles_and_oracle(monkeypatch, case, prec):
    """3-D degree 2 on tiles of 2x2x2 cells with phase B by planes (three
    lanes per (cell, time dof), the z sweeps by shuffles; STMG_OP_TINY=1)
    against the regular tiles with the per-thread phase B (STMG_OP_TINY=0)
    and the oracle, for vmult, Tvmult and the relaxation update: the same
    sums in another order and over other tile faces, so FP64 1e-13 / FP32
    2e-6 between the two."""
    import stmg
    om, gm, A, B, rK, rM = build(case)
    dim, n, p = case[0], case[1], case[2]
    nt = A.shape[0]
    mask = meshes.boundary_mask(dim, n, p)
    src = meshes.random_block_vector(nt, om.n_nodes, mask)
    dt = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-12 if prec == "f64" else 2e-5
    close = 1e-13 if prec == "f64" else 2e-6
    dty = stmg.F64 if prec == "f64" else stmg.F32
    monkeypatch.setenv("STMG_OP_TINY", "1")
    opt = stmg.Operator(gm, A, B, dtype=dty)
    monkeypatch.setenv("STMG_OP_TINY", "0")
    opr = stmg.Operator(gm, A, B, dtype=dty)
    s = torch.tensor(src, dtype=dt, device="cuda")
    for transpose in (False, True):
        dp, dq = torch.full_like(s, 7.0), torch.full_like(s, -7.0)
        (opt.Tvmult if transpose else opt.vmult)(dp, s)
        (opr.Tvmult if transpose else opr.vmult)(dq, s)
        ref = om.st_apply(A, B, src, transpose=transpose)
        got = dp.double().cpu().numpy()
        assert rel_err(got, ref) < tol
        assert rel_err(got, dq.double().cpu().numpy()) < close
    # the residual output mode through a relaxation step (the same FP32 Vanka)
    if prec == "f32":
        vk = stmg.Vanka(gm, A, B, compute=stmg.F32, storage=stmg.F32)
        b = torch.tensor(meshes.random_block_vector(nt, om.n_nodes, mask, seed=5), dtype=dt, device="cuda")
        xt, xr, tmp = s.clone(), s.clone(), torch.empty_like(s)
        vk.step(opt, 0.8, xt, b, tmp)
        vk.step(opr, 0.8, xr, b, tmp)
        torch.cuda.synchronize()
        assert rel_err(xt.double().cpu().numpy(), xr.double().cpu().numpy()) < 1e-5
