"""The slab solve on the GPU (FP64 FGMRES + FP32 space-time V-cycle) against
the reference's golden 2-D runs (tests/tp_01.output: FGMRES totals per
configuration) and against the CPU oracle (same iteration counts within one
per slab, solution within 1e-7 relative)."""
import json
import os

import numpy as np
import pytest

import meshes
import oracle_py as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tp_01.json")


def _gold():
    with open(GOLDEN) as f:
        return json.load(f)


# directory for the GPU-vs-reference iteration record (unset: no record)
RECORD_DIR = os.environ.get("STMG_TEST_RECORD_DIR")


def _record(g, total):
    """Appends GPU-vs-reference totals for the parity report (best effort)."""
    if not RECORD_DIR:
        return
    try:
        os.makedirs(RECORD_DIR, exist_ok=True)
        with open(os.path.join(RECORD_DIR, "tp01_gpu_iterations.jsonl"), "a") as f:
            f.write(json.dumps(dict(section=g["section"], k=g["k"], refine=g["refine"], slabs=g["slabs"],
                                    reference=g["iterations"], gpu=total)) + "\n")
    except OSError:
        pass


# (section, k, refine) of golden configurations whose totals differ from the
# reference's by rounding of the FP32 V-cycle: none at present
NEAR_TOTALS = set()

GOLD_CASES = [g for g in _gold() if g["refine"] <= 4 and not (g["refine"] == 4 and g["k"] == 3)]


@pytest.mark.parametrize("g", GOLD_CASES, ids=lambda g: f"{g['section']}-k{g['k']}-r{g['refine']}")
def test_gpu_iterations_match_tp01(g):
    import stmg
    ttype = stmg.DG if g["type"] == "DG" else stmg.CGP
    s = stmg.Solver(dim=2, refine=g["refine"], degree=g["k"] + 1, time_degree=g["k"], time_type=ttype,
                    problem=stmg.HEAT if g["problem"] == "heat" else stmg.WAVE, n_steps=g["steps"],
                    fe_degree_min=0 if ttype == stmg.DG else 1, n_steps_min=max(1, g["steps"] // 2))
    assert s.n_nodes == g["s_dofs"]
    its = s.run(g["slabs"])
    total = int(its.sum())
    _record(g, total)
    # the reference's FGMRES total exactly (every one of these configurations
    # reproduced it on the B200); a configuration listed in NEAR_TOTALS would
    # be held to one iteration per slab instead
    if (g["section"], g["k"], g["refine"]) in NEAR_TOTALS:
        assert abs(total - g["iterations"]) <= g["slabs"], (total, g["iterations"])
    else:
        assert total == g["iterations"], (total, g["iterations"])
    # error norms against the manufactured solution, as printed (6 digits)
    linf, l2, h1 = s.errors()
    assert linf == pytest.approx(g["linf"], rel=2e-5)
    assert l2 == pytest.approx(g["l2"], rel=2e-5)
    assert h1 == pytest.approx(g["h1"], rel=2e-5)


@pytest.mark.parametrize("problem,ttype,k,steps", [("heat", "DG", 1, 1), ("heat", "CGP", 2, 1), ("wave", "DG", 1, 1),
                                                   ("heat", "DG", 2, 2)])
def test_gpu_solution_matches_oracle_2d(problem, ttype, k, steps):
    import stmg
    tt = stmg.DG if ttype == "DG" else stmg.CGP
    pb = stmg.HEAT if problem == "heat" else stmg.WAVE
    refine = 3
    ref = orc.run(dim=2, refine=refine, p=k + 1, r=k, ttype=tt, problem=pb, n_steps=steps,
                  fe_degree_min=0 if tt == stmg.DG else 1, n_steps_min=max(1, steps // 2), compute_errors=False)
    s = stmg.Solver(dim=2, refine=refine, degree=k + 1, time_degree=k, time_type=tt, problem=pb, n_steps=steps,
                    fe_degree_min=0 if tt == stmg.DG else 1, n_steps_min=max(1, steps // 2))
    its = s.run(len(ref["iterations"]))
    assert np.all(np.abs(its - ref["iterations"]) <= 1)
    u, _ = s.solution()
    assert np.linalg.norm(u - ref["u"]) <= 1e-7 * np.linalg.norm(ref["u"])


def test_gpu_solution_matches_oracle_3d_coefficient():
    """32^3-style heat slab with a log-uniform per-cell coefficient and a
    nodal random source, scaled down to 4^3 Q2 cells, dG(1)."""
    import stmg
    dim, R = 3, 2
    nf = (4, 4, 4)
    coeff = meshes.log_uniform(64, 1e-1, 1e1, seed=3)
    nn = 9 ** 3
    f = np.random.default_rng(4).standard_normal(nn)
    kw = dict(dim=3, refine=R, r=1, problem=orc.HEAT, n_steps=1, tau=1 / 8, n_slabs=3, rhs_mode=1)
    ref = orc.run(p=2, ttype=orc.DG, f_nodal=f, fine_coeff=coeff, compute_errors=False, tol=1e-10, abs_tol=1e-14, **kw)
    s = stmg.Solver(dim=3, refine=R, degree=2, time_degree=1, time_type=stmg.DG, problem=stmg.HEAT, n_steps=1,
                    tau=1 / 8, rhs_mode=1, f_nodal=f, fine_coeff=coeff, tol=1e-10, abs_tol=1e-14)
    its = s.run(3)
    assert np.all(np.abs(its - ref["iterations"]) <= 1)
    u, _ = s.solution()
    assert np.linalg.norm(u - ref["u"]) <= 1e-7 * np.linalg.norm(ref["u"])


@pytest.mark.parametrize("dim,refine,k,steps", [(2, 3, 1, 1), (2, 3, 2, 2), (3, 2, 1, 2)])
@pytest.mark.parametrize("mg", ["f32", "f64"])
def test_dense_tail_matches_sweeps(monkeypatch, dim, refine, k, steps, mg):
    """The coarsest levels run as one matrix composed in FP64; one V-cycle
    agrees with the sweep-by-sweep V-cycle (STMG_DENSE_TAIL=0) to the
    rounding of the V-cycle's precision."""
    import stmg
    dt, tol = (stmg.F32, 2e-5) if mg == "f32" else (stmg.F64, 1e-10)
    kw = dict(dim=dim, refine=refine, degree=2, time_degree=k, time_type=stmg.DG, n_steps=steps, fe_degree_min=0,
              n_steps_min=max(1, steps // 2), mg_dtype=dt)
    monkeypatch.setenv("STMG_DENSE_TAIL", "1")
    a = stmg.Solver(**kw)
    monkeypatch.setenv("STMG_DENSE_TAIL", "0")
    b = stmg.Solver(**kw)
    n = a.n_nodes * a.n_blocks
    x = torch.from_numpy(np.random.default_rng(5).standard_normal(n)).cuda()
    ya, yb = torch.empty_like(x), torch.empty_like(x)
    for _ in range(2):
        a.gmg_vmult(ya, x)
        b.gmg_vmult(yb, x)
    torch.cuda.synchronize()
    assert torch.linalg.norm(ya - yb) <= tol * torch.linalg.norm(yb)


def test_gpu_distorted_q3_matches_oracle():
    """The 32^3 Q3 distorted-mesh configuration scaled down: 4^3 Q3 cells,
    interior vertices moved by up to 0.2 h per axis, per-cell coefficient
    10^U(-2, 2), f = 1 (nodal), dG(2); GPU and oracle (both FP32 V-cycle)."""
    import stmg
    R, n = 2, 4
    X = meshes.vertices(3, (n, n, n), distort=0.2, seed=21)
    coeff = meshes.log_uniform(n ** 3, 1e-2, 1e2, seed=22)
    f = np.ones((3 * n + 1) ** 3)
    kw = dict(dim=3, refine=R, r=2, problem=orc.HEAT, n_steps=1, tau=1 / 32, n_slabs=2, rhs_mode=1)
    ref = orc.run(p=3, ttype=orc.DG, f_nodal=f, fine_coeff=coeff, fine_vertices=X, compute_errors=False, tol=1e-10,
                  abs_tol=1e-14, **kw)
    s = stmg.Solver(dim=3, refine=R, degree=3, time_degree=2, time_type=stmg.DG, problem=stmg.HEAT, n_steps=1,
                    tau=1 / 32, rhs_mode=1, f_nodal=f, fine_coeff=coeff, fine_vertices=X, tol=1e-10, abs_tol=1e-14)
    its = s.run(2)
    assert np.all(np.abs(its - ref["iterations"]) <= 1), (its, ref["iterations"])
    u, _ = s.solution()
    assert np.linalg.norm(u - ref["u"]) <= 1e-7 * np.linalg.norm(ref["u"])


def test_gpu_wave_bf16_vanka_keeps_iterations():
    """The wave configuration's precision question scaled down (4^3 Q2
    cells, dG(2), c^2 in {0.5, 1, 4} per cell, Gaussian pulse u0, v0 = 0,
    f = 0): BF16-stored Vanka eigenvectors vs FP32-stored, same FP64 FGMRES
    tolerance; iterations within one per slab and solutions within the
    solver tolerance."""
    import stmg
    R, n = 2, 4
    rng = np.random.default_rng(23)
    c2 = rng.choice([0.5, 1.0, 4.0], size=n ** 3)
    kw = dict(dim=3, refine=R, degree=2, time_degree=2, time_type=stmg.DG, problem=stmg.WAVE, n_steps=1,
              tau=1 / 128, rhs_mode=2, fine_coeff=c2, tol=1e-10, abs_tol=1e-14)
    nn1 = 2 * n + 1
    g = np.linspace(0, 1, nn1)
    Z, Y, Xc = np.meshgrid(g, g, g, indexing="ij")
    u0 = np.exp(-((Xc - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2) / 0.01).reshape(-1)
    u0[meshes.boundary_mask(3, (n, n, n), 2)] = 0.0
    out = {}
    for st in (stmg.F32, stmg.BF16):
        s = stmg.Solver(vanka_storage=st, **kw)
        s.set_initial(u0, np.zeros_like(u0))
        its = s.run(4)
        u, _ = s.solution()
        out[st] = (its, u)
    its32, u32 = out[stmg.F32]
    its16, u16 = out[stmg.BF16]
    assert np.all(np.abs(its16 - its32) <= 1), (its16, its32)
    assert np.linalg.norm(u16 - u32) <= 1e-7 * np.linalg.norm(u32)


def test_gpu_c1_plain_fp64_matches_oracle():
    """The plain FP64 configuration: 2-D unit square, 16^2 Q2 cells, dG(1),
    dt = 1/64, 64 slabs, manufactured u = sin(pi x) sin(pi y) sin(pi t)
    (frequency 1/2), 2 pre/post sweeps, all-FP64 multigrid, 1e-10 relative
    residual. GPU and oracle: iterations per slab within one, error norms to
    1e-6."""
    import stmg
    kw = dict(dim=2, refine=4, n_steps=1, tau=1 / 64, fe_degree_min=0, n_steps_min=1, tol=1e-10, abs_tol=1e-14,
              frequency=0.5, smoothing_steps=2)
    ref = orc.run(p=2, r=1, ttype=orc.DG, problem=orc.HEAT, n_slabs=64, mg_float=False, compute_errors=True, **kw)
    s = stmg.Solver(degree=2, time_degree=1, time_type=stmg.DG, problem=stmg.HEAT, mg_dtype=stmg.F64, **kw)
    its = s.run(64)
    assert np.all(np.abs(its - ref["iterations"]) <= 1), (its, ref["iterations"])
    linf, l2, h1 = s.errors()
    assert linf == pytest.approx(ref["linf"], rel=1e-6)
    assert l2 == pytest.approx(ref["l2"], rel=1e-6)
    assert h1 == pytest.approx(ref["h1"], rel=1e-6)


@pytest.mark.parametrize("problem", ["heat", "wave"])
def test_gpu_solution_async_matches_blocking_copy(problem):
    """stmg_solver_solution_async: the host arrays hold the slab the copy was
    started after, although the next slabs run (and overwrite the device
    solution) before the wait; equal to the blocking copy bit for bit."""
    import stmg
    kw = dict(dim=2, refine=3, degree=2, time_degree=1, time_type=stmg.DG, n_steps=1, fe_degree_min=0,
              n_steps_min=1, problem=stmg.HEAT if problem == "heat" else stmg.WAVE)
    ref = stmg.Solver(**kw)
    ref.run(1)
    u1, v1 = ref.solution()
    ref.run(1)
    u2, v2 = ref.solution()
    s = stmg.Solver(**kw)
    n = s.n_blocks * s.n_nodes
    hu = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    hv = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    hu[:] = np.nan
    hv[:] = np.nan
    s.run(1)
    s.solution_async(hu, hv)
    s.run(2)  # moves the device solution on while the copy may still run
    s.solution_wait()
    assert np.array_equal(hu, u1) and np.array_equal(hv, v1)
    s2 = stmg.Solver(**kw)
    s2.run(2)
    s2.solution_async(hu)
    s2.solution_wait()
    assert np.array_equal(hu, u2)


def test_gpu_short_restart_tight_tolerance_fp32_matches_fp64():
    """FGMRES over several restart cycles (restart 8) to a tight tolerance
    (1e-12) on the distorted Q3 shape (4^3 cells, kappa = 10^U(-2, 2),
    dG(2)): each basis vector reaches the FP32 V-cycle scaled by a power of
    two to a norm near one, so the FP32-multigrid solve converges like the
    all-FP64 one and the solutions agree."""
    import stmg
    n = 4
    X = meshes.vertices(3, (n, n, n), distort=0.2, seed=51)
    coeff = meshes.log_uniform(n ** 3, 1e-2, 1e2, seed=52)
    kw = dict(dim=3, refine=2, degree=3, time_degree=2, time_type=stmg.DG, problem=stmg.HEAT, n_steps=1,
              tau=1 / 32, rhs_mode=1, f_nodal=np.ones((3 * n + 1) ** 3), fine_coeff=coeff, fine_vertices=X,
              tol=1e-12, abs_tol=1e-300, restart=8, max_iter=1000)
    s32 = stmg.Solver(mg_dtype=stmg.F32, **kw)
    s64 = stmg.Solver(mg_dtype=stmg.F64, **kw)
    its32, its64 = s32.run(2), s64.run(2)
    assert its32.max() > 8 and np.all(np.abs(its32 - its64) <= 2), (its32, its64)
    u32, _ = s32.solution()
    u64, _ = s64.solution()
    assert np.linalg.norm(u32 - u64) <= 1e-10 * np.linalg.norm(u64)
