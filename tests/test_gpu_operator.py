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
