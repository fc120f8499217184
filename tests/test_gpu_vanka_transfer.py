"""Vanka smoother and multigrid transfers on the GPU against the CPU oracle
(PreconditionVanka::vmult, gmg.h:476-514; MGTwoLevelTransfer via
gmg.h:35-75; MGTwoLevelTransferST, gmg.h:77-136).
Vanka: the oracle inverts each patch matrix with Gauss-Jordan; the GPU applies
the same inverse in factored form. Tolerances (relative, 2-norm): FP64 1e-10,
FP32 2e-4, BF16 storage of the eigenvectors 3e-2. Transfers: FP64 1e-14,
FP32 1e-6."""
import numpy as np
import pytest

import meshes
import oracle_py as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

VANKA_CASES = [
    # dim, cells, p, distort, coeff, (type, r, steps, problem)
    (2, (4, 4), 2, 0.0, False, (orc.DG, 1, 1, orc.HEAT)),
    (2, (5, 3), 3, 0.2, True, (orc.CGP, 2, 2, orc.HEAT)),
    (2, (3, 3), 4, 0.0, False, (orc.DG, 2, 2, orc.WAVE)),
    (2, (4, 4), 1, 0.0, False, (orc.DG, 0, 1, orc.HEAT)),
    (3, (3, 3, 2), 2, 0.0, True, (orc.DG, 3, 1, orc.HEAT)),
    (3, (4, 3, 3), 2, 0.2, True, (orc.DG, 2, 1, orc.HEAT)),
    (3, (2, 2, 2), 3, 0.15, True, (orc.DG, 2, 1, orc.WAVE)),
    # degree 3 over several tiles (chunked apply for every precision)
    (3, (5, 4, 3), 3, 0.2, True, (orc.DG, 2, 1, orc.HEAT)),
]


def rel2(x, y):
    return np.linalg.norm(x - y) / np.linalg.norm(y)


def _setup(case):
    import stmg
    dim, n, p, distort, coeff, (tt, r, steps, prob) = case
    X = meshes.vertices(dim, n, distort=distort)
    c = meshes.log_uniform(int(np.prod(n)), 1e-2, 1e2) if coeff else None
    om = orc.Mesh(dim, n, p, vertices=X, coeff=c)
    gm = stmg.Mesh(dim, n, p, vertices=X, coeff=c)
    A, B, _, _, _ = orc.time_weights(tt, r, 0.125, steps, prob)
    src = meshes.random_block_vector(A.shape[0], om.n_nodes, meshes.boundary_mask(dim, n, p))
    return om, gm, A, B, src


@pytest.mark.parametrize("case", VANKA_CASES, ids=lambda c: f"d{c[0]}-p{c[2]}-nt{c[5][1]}x{c[5][2]}-dist{c[3]}")
@pytest.mark.parametrize("mode", ["f64", "f32", "bf16"])
def test_vanka_matches_oracle(case, mode):
    import stmg
    om, gm, A, B, src = _setup(case)
    ref = om.vanka_apply(A, B, src)
    compute = stmg.F64 if mode == "f64" else stmg.F32
    storage = {"f64": stmg.F64, "f32": stmg.F32, "bf16": stmg.BF16}[mode]
    vk = stmg.Vanka(gm, A, B, compute=compute, storage=storage)
    dt = torch.float64 if mode == "f64" else torch.float32
    s = torch.tensor(src, dtype=dt, device="cuda")
    d = torch.full_like(s, 3.0)
    vk.vmult(d, s)
    got = d.double().cpu().numpy()
    tol = {"f64": 1e-10, "f32": 2e-4, "bf16": 3e-2}[mode]
    assert rel2(got, ref) < tol
    d2 = torch.empty_like(s)
    vk.vmult(d2, s)
    assert torch.equal(d, d2)  # deterministic


H_CASES = [(2, (2, 3), 1), (2, (2, 2), 2), (2, (3, 2), 3), (2, (2, 2), 4), (2, (2, 2), 5), (3, (2, 2, 2), 1), (3, (2, 2, 1), 2),
           (3, (1, 2, 2), 3),
           # several tiles per direction, partial last tiles (FP32 tiles of
           # 16 / 8 / 4 coarse cells for degree 1 in 2-D / 1 in 3-D / 2 in 3-D)
           (2, (20, 9), 1), (3, (10, 3, 9), 1), (3, (9, 5, 6), 2), (3, (3, 4, 5), 4)]


@pytest.mark.parametrize("case", H_CASES, ids=lambda c: f"d{c[0]}-p{c[2]}")
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_h_transfer_matches_oracle(case, prec):
    import stmg
    dim, nc, p = case
    nf = [2 * k for k in nc]
    oc, of = orc.Mesh(dim, nc, p), orc.Mesh(dim, nf, p)
    gc, gf = stmg.Mesh(dim, nc, p), stmg.Mesh(dim, nf, p)
    nt = 2
    dt = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-14 if prec == "f64" else 1e-6
    tr = stmg.Transfer(gf, gc, nt, dtype=stmg.F64 if prec == "f64" else stmg.F32)
    xc = meshes.random_block_vector(nt, oc.n_nodes, meshes.boundary_mask(dim, nc, p), seed=5)
    xf = meshes.random_block_vector(nt, of.n_nodes, meshes.boundary_mask(dim, nf, p), seed=6)
    base_f = meshes.random_block_vector(nt, of.n_nodes, meshes.boundary_mask(dim, nf, p), seed=7)
    base_c = meshes.random_block_vector(nt, oc.n_nodes, meshes.boundary_mask(dim, nc, p), seed=8)
    # prolongate_and_add
    ref = orc.h_transfer(of, oc, nt, xc, restrict=False, dst=base_f)
    d = torch.tensor(base_f, dtype=dt, device="cuda")
    tr.prolongate_add(d, torch.tensor(xc, dtype=dt, device="cuda"))
    assert rel2(d.double().cpu().numpy(), ref) < tol
    # prolongate (zeroes dst)
    ref0 = orc.h_transfer(of, oc, nt, xc, restrict=False)
    tr.prolongate(d, torch.tensor(xc, dtype=dt, device="cuda"))
    assert rel2(d.double().cpu().numpy(), ref0) < tol
    # restrict_and_add
    refr = orc.h_transfer(of, oc, nt, xf, restrict=True, dst=base_c)
    dc = torch.tensor(base_c, dtype=dt, device="cuda")
    tr.restrict_add(dc, torch.tensor(xf, dtype=dt, device="cuda"))
    assert rel2(dc.double().cpu().numpy(), refr) < tol
    # restriction is the transpose of prolongation: <P xc, xf> = <xc, R xf>
    pc = orc.h_transfer(of, oc, nt, xc)
    rf = orc.h_transfer(of, oc, nt, xf, restrict=True)
    assert abs(pc @ xf - xc @ rf) < 1e-12 * np.linalg.norm(pc) * np.linalg.norm(xf)


@pytest.mark.parametrize("kind,ttype,r,steps", [(0, orc.DG, 3, 1), (0, orc.CGP, 2, 2), (1, orc.DG, 1, 2), (1, orc.CGP, 2, 4)])
def test_time_transfer_matches_oracle(kind, ttype, r, steps):
    import stmg
    P = orc.time_prolongation(ttype, kind, r, steps)
    gm = stmg.Mesh(2, (3, 3), 2)
    N = gm.n_nodes
    tr = stmg.Transfer(mesh=gm, P=P, dtype=stmg.F64)
    rng = np.random.default_rng(1)
    xc = rng.standard_normal((P.shape[1], N))
    xf = rng.standard_normal((P.shape[0], N))
    d = torch.zeros(P.shape[0] * N, dtype=torch.float64, device="cuda")
    tr.prolongate_add(d, torch.tensor(xc.reshape(-1), device="cuda"))
    assert np.allclose(d.cpu().numpy().reshape(P.shape[0], N), P @ xc, rtol=1e-14, atol=1e-14)
    dc = torch.zeros(P.shape[1] * N, dtype=torch.float64, device="cuda")
    tr.restrict_add(dc, torch.tensor(xf.reshape(-1), device="cuda"))
    assert np.allclose(dc.cpu().numpy().reshape(P.shape[1], N), P.T @ xf, rtol=1e-14, atol=1e-14)


ROW_CASES = [
    # single-step slabs (time solves in the eigenbasis), cells of up to 32 dofs
    (2, (4, 4), 2, 0.0, False, (orc.DG, 1, 1, orc.HEAT)),
    (2, (6, 5), 3, 0.2, True, (orc.DG, 2, 1, orc.HEAT)),
    (2, (3, 3), 4, 0.0, False, (orc.DG, 3, 1, orc.HEAT)),
    (2, (4, 4), 1, 0.0, False, (orc.DG, 0, 1, orc.HEAT)),
    (3, (3, 3, 2), 1, 0.1, True, (orc.DG, 1, 1, orc.HEAT)),
    (3, (3, 3, 2), 2, 0.0, True, (orc.DG, 3, 1, orc.HEAT)),
    (3, (9, 6, 5), 2, 0.2, True, (orc.DG, 2, 1, orc.WAVE)),
    (3, (12, 8, 8), 2, 0.0, True, (orc.DG, 3, 1, orc.HEAT)),
]


@pytest.mark.parametrize("case", ROW_CASES, ids=lambda c: f"d{c[0]}-p{c[2]}-r{c[5][1]}-n{'x'.join(map(str, c[1]))}")
@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_vanka_row_records_match_streamed_and_oracle(monkeypatch, case, storage):
    """The row-record apply (bulk-copied colour phases, a half-warp per
    cell) against the streamed apply over the same records in the previous
    layout (STMG_VANKA_ROWREC=0) and against the oracle's Gauss-Jordan
    inverses; with alpha/beta output modes through the relaxation update."""
    import stmg
    om, gm, A, B, src = _setup(case)
    ref = om.vanka_apply(A, B, src)
    st = stmg.F32 if storage == "f32" else stmg.BF16
    monkeypatch.setenv("STMG_VANKA_SLOT", "0")  # the colour-phase kernels on these small meshes
    monkeypatch.setenv("STMG_VANKA_ROWREC", "1")
    vr = stmg.Vanka(gm, A, B, compute=stmg.F32, storage=st)
    monkeypatch.setenv("STMG_VANKA_ROWREC", "0")
    vs = stmg.Vanka(gm, A, B, compute=stmg.F32, storage=st)
    s = torch.tensor(src, dtype=torch.float32, device="cuda")
    dr, ds = torch.full_like(s, 3.0), torch.full_like(s, -1.0)
    for _ in range(2):
        vr.vmult(dr, s)
        vs.vmult(ds, s)
    torch.cuda.synchronize()
    got, prev = dr.double().cpu().numpy(), ds.double().cpu().numpy()
    tol = 2e-4 if storage == "f32" else 3e-2
    assert rel2(got, ref) <= tol, rel2(got, ref)
    # same records (up to layout), same maths: agreement to FP32 rounding
    # (BF16 records with 3 or 4 time dofs take the tensor-core apply, whose
    # input keeps ~16 significant bits: 1e-4)
    assert rel2(got, prev) <= (2e-5 if storage == "f32" else 1e-4), rel2(got, prev)


MMA_CASES = [c for c in ROW_CASES if c[5][1] + 1 in (3, 4)] + [
    (3, (16, 8, 8), 2, 0.0, True, (orc.DG, 3, 1, orc.HEAT)),
    (2, (20, 16), 2, 0.1, True, (orc.DG, 2, 1, orc.WAVE)),
]


@pytest.mark.parametrize("case", MMA_CASES, ids=lambda c: f"d{c[0]}-p{c[2]}-r{c[5][1]}-n{'x'.join(map(str, c[1]))}")
def test_vanka_tensor_core_matches_row_kernel(monkeypatch, case):
    """The tensor-core apply (BF16 records, m16n8k16 BF16 MMA with FP32
    accumulation, input split in two BF16 parts) against the FFMA2 row
    kernel on the same BF16 eigenvectors (STMG_VANKA_MMA=0): 1e-4, and the
    oracle's FP64 Gauss-Jordan inverses: 3e-2 (the BF16 storage). The
    relaxation output mode runs in the solver tests with BF16 storage."""
    import stmg
    om, gm, A, B, src = _setup(case)
    ref = om.vanka_apply(A, B, src)
    monkeypatch.setenv("STMG_VANKA_SLOT", "0")
    monkeypatch.setenv("STMG_VANKA_MMA", "1")
    vm = stmg.Vanka(gm, A, B, compute=stmg.F32, storage=stmg.BF16)
    monkeypatch.setenv("STMG_VANKA_MMA", "0")
    vr = stmg.Vanka(gm, A, B, compute=stmg.F32, storage=stmg.BF16)
    s = torch.tensor(src, dtype=torch.float32, device="cuda")
    dm, dr = torch.full_like(s, 5.0), torch.full_like(s, -2.0)
    for _ in range(2):
        vm.vmult(dm, s)
        vr.vmult(dr, s)
    torch.cuda.synchronize()
    got, row = dm.double().cpu().numpy(), dr.double().cpu().numpy()
    assert rel2(got, row) <= 1e-4, rel2(got, row)
    assert rel2(got, ref) <= 3e-2, rel2(got, ref)



SLOT_CASES = ROW_CASES + [
    (3, (16, 16, 16), 2, 0.0, True, (orc.DG, 3, 1, orc.HEAT)),
    (3, (7, 5, 9), 2, 0.15, True, (orc.DG, 2, 1, orc.HEAT)),
    (2, (15, 22), 4, 0.1, True, (orc.CGP, 2, 1, orc.HEAT)),
]


@pytest.mark.parametrize("case", SLOT_CASES, ids=lambda c: f"d{c[0]}-p{c[2]}-r{c[5][1]}-n{'x'.join(map(str, c[1]))}")
@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_vanka_small_tiles_match_row_kernel_and_oracle(monkeypatch, case, storage):
    """The small-tile apply (tiles of 2^dim cells, all cells of a tile at
    once, per-cell output slots summed in colour order; STMG_VANKA_SLOT=1)
    against the colour-phase row kernel over row records of the same
    storage (STMG_VANKA_SLOT=0, tensor-core apply off): the same cell
    arithmetic on other tile boundaries, so agreement to FP32 rounding of
    the node sums (2e-6); and against the oracle's Gauss-Jordan inverses.
    Both the plain apply and the relaxation update x += omega V (b - A x)."""
    import stmg
    om, gm, A, B, src = _setup(case)
    ref = om.vanka_apply(A, B, src)
    st = stmg.F32 if storage == "f32" else stmg.BF16
    monkeypatch.setenv("STMG_VANKA_MMA", "0")
    monkeypatch.setenv("STMG_VANKA_SLOT", "1")
    vt = stmg.Vanka(gm, A, B, compute=stmg.F32, storage=st)
    monkeypatch.setenv("STMG_VANKA_SLOT", "0")
    vr = stmg.Vanka(gm, A, B, compute=stmg.F32, storage=st)
    s = torch.tensor(src, dtype=torch.float32, device="cuda")
    dt, dr = torch.full_like(s, 3.0), torch.full_like(s, -1.0)
    for _ in range(2):
        vt.vmult(dt, s)
        vr.vmult(dr, s)
    torch.cuda.synchronize()
    got, row = dt.double().cpu().numpy(), dr.double().cpu().numpy()
    assert rel2(got, ref) <= (2e-4 if storage == "f32" else 3e-2), rel2(got, ref)
    assert rel2(got, row) <= 2e-6, rel2(got, row)
    # relaxation step through both kernels' output modes
    op = stmg.Operator(gm, A, B, dtype=stmg.F32)
    b = torch.tensor(meshes.random_block_vector(A.shape[0], om.n_nodes, meshes.boundary_mask(case[0], case[1], case[2]),
                                                seed=11), dtype=torch.float32, device="cuda")
    xt, xr = s.clone(), s.clone()
    tmp = torch.empty_like(s)
    vt.step(op, 0.7, xt, b, tmp)
    vr.step(op, 0.7, xr, b, tmp)
    torch.cuda.synchronize()
    assert rel2(xt.double().cpu().numpy(), xr.double().cpu().numpy()) <= 2e-6
