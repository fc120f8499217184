#!/usr/bin/env python
"""Benchmark of the space-time multigrid slab solve on B200.

Workload (one GPU): heat equation on the unit cube, 128^3 Q2 cells
(257^3 = 16,974,593 nodes), dG(3) in time (4 time dofs, 67.9M space-time
dofs per slab), 8 slabs of dt = 1/8, per-cell coefficient log-uniform in
[0.1, 10] and a nodal source f_i ~ N(0,1), both seeded; each slab solved by
FP64 FGMRES preconditioned with the FP32 space-time V-cycle (cell-patch
Vanka, h/k transfers) to 1e-8 relative residual. A step is one slab solve.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The JSON line carries the device-timed throughput (`value`), the end-to-end
throughput through the C ABI with host buffers (`e2e`), the all-FP64
V-cycle throughput on the same workload (`fp64_mg`), the roofline of the
finest-level operator and Vanka kernels timed in isolation, the CPU oracle
baseline on a bounded sample, clocks sampled during the timed region, the
number of kernels launched and (`accuracy`) the per-slab relative difference
of the FP32-MG and all-FP64 solutions from a converged all-FP64 solve of the
same 8 slabs.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "dealii-stfem_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))

METRIC = "space-time DoF/s to 1e-8 residual, FP32-MG vs FP64 on one B200; apply GB/s"
SEED = 20261203


def workload(refine=7):
    n = 1 << refine
    return dict(name=f"heat3d-{n}^3-Q2-dG3-8slabs", dim=3, refine=refine, degree=2, time_degree=3, n_steps=1,
                tau=1.0 / 8, n_slabs=8, kappa=(0.1, 10.0), tol=1e-8, cells=n ** 3, nodes=(2 * n + 1) ** 3, nt=4)


def inputs(w, seed=SEED):
    rng = np.random.default_rng(seed)
    kappa = 10.0 ** rng.uniform(np.log10(w["kappa"][0]), np.log10(w["kappa"][1]), size=w["cells"])
    f = rng.standard_normal(w["nodes"])
    return kappa, f


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per cell of one
# finest-level Vanka apply kernel, from ncu captures of the same kernels on
# 64^3 Q2 cells with n_t = 4 (the records exceed L2 there, and the traffic
# grows with the cell count): python bench.py --kernels-only vanka_apply
# --refine 6 [--vanka-storage bf16] under ncu --set full (vanka_row_kernel
# with FP32 records, vanka_mma_kernel with BF16 records).
VANKA_TRAFFIC_PER_CELL = {"f32": 3508.62, "bf16": 2301.93}


def vanka_traffic(refine, storage="f32"):
    """DRAM bytes of one finest-level Vanka apply on (2^refine)^3 cells."""
    return VANKA_TRAFFIC_PER_CELL[storage] * (1 << refine) ** 3


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------- CPU baseline
def cpu_sample(w, seed=SEED, steps=1):
    """The CPU oracle (one thread) on a bounded sample of the workload: the
    same physics on 16^3 Q2 cells, dG(3), one slab per step."""
    import oracle_py as orc
    ws = workload(refine=4)
    kappa, f = inputs(ws, seed)
    t0 = time.perf_counter()
    res = orc.run(dim=3, refine=ws["refine"], p=2, r=3, ttype=orc.DG, problem=orc.HEAT, n_steps=1, tau=ws["tau"],
                  n_slabs=steps, rhs_mode=1, f_nodal=f, fine_coeff=kappa, compute_errors=False, tol=w["tol"],
                  abs_tol=1e-300)
    dt = time.perf_counter() - t0
    dofs = ws["nodes"] * ws["nt"] * steps
    return dict(value=dofs / dt, unit="DoF/s", cores=1, kind="port",
                sample=f"oracle FP64 FGMRES + FP32 V-cycle, 16^3 Q2 cells dG(3), {steps} slab(s) incl. setup "
                       f"({dt:.1f} s, {res['total_iterations']} FGMRES iterations)"), dt


def _reference_sample(n_slabs):
    """One process: the oracle port on the 16^3 sample for n_slabs slabs;
    returns (space-time dofs, seconds, FGMRES iterations)."""
    import oracle_py as orc
    w = workload()
    ws = workload(refine=4)
    kappa, f = inputs(ws)
    t0 = time.perf_counter()
    res = orc.run(dim=3, refine=ws["refine"], p=2, r=3, ttype=orc.DG, problem=orc.HEAT, n_steps=1, tau=ws["tau"],
                  n_slabs=n_slabs, rhs_mode=1, f_nodal=f, fine_coeff=kappa, compute_errors=False, tol=w["tol"],
                  abs_tol=1e-300)
    return ws["nodes"] * ws["nt"] * n_slabs, time.perf_counter() - t0, [int(i) for i in res["iterations"]]


def run_reference(args):
    """--impl reference: the oracle port of the reference's CPU path, timed on
    the host cores (steps = slabs of the bounded 16^3 sample; setup counted
    once). The port is single-threaded, so every host core runs its own copy
    of the sample at the same time (spawned processes) and the throughput is
    the sum over copies / the slowest copy's time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    w = workload()
    n = args.warmup + args.steps
    procs = max(1, min(int(os.environ.get("STMG_REFERENCE_PROCS", os.cpu_count() or 1)), 128))
    if procs == 1:
        results = [_reference_sample(n)]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            results = pool.map(_reference_sample, [n] * procs)
    dofs = sum(r[0] for r in results)
    dt = max(r[1] for r in results)
    value = dofs / dt
    line = dict(metric=METRIC, value=value, unit="DoF/s", impl="reference", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=1e3 * dt / n, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic",
                config=dict(workload=w["name"], sample="16^3 Q2 cells, dG(3), same seeded coefficient and source "
                                                        "distributions", slabs=n, copies=procs),
                cpu_baseline=dict(value=value, unit="DoF/s", cores=procs, kind="port",
                                  sample=f"{procs} concurrent copies x {n} slabs of the 16^3 sample including setup"),
                e2e=dict(value=value, unit="DoF/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                fgmres_iterations=results[0][2])
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------- GPU arm
def max_over_ranks(t, dist=None):
    """The slowest rank's time (replicas run independently; the job takes
    as long as its slowest replica)."""
    if dist is None:
        return t
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    tt = torch.tensor([t], device=dev, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def replica_throughput(world, dofs_per_step, steps, t):
    """Whole-job DoF/s of `world` replicas, each solving `steps` slabs."""
    return world * dofs_per_step * steps / t


# relative residual of the converged FP64 solve the accuracy figures compare
# against (the FP64 FGMRES stagnates near 1e-13 on these systems)
ACC_REF_TOL = 1e-12


def slab_solutions(solver, w, n_slabs):
    """The solver's solution blocks after each of n_slabs slabs run from a
    zero initial state (host FP64 arrays); untimed."""
    out = []
    if n_slabs:
        solver.set_initial(np.zeros(w["nodes"]))
        for _ in range(n_slabs):
            solver.run(1)
            u, _ = solver.solution(want_v=False)
            out.append(u)
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def accuracy_report(u32, u64, uref, tol):
    """Per-slab relative 2-norm differences of the FP32-MG solve (u32) and
    the all-FP64 solve (u64), both to `tol`, against a converged all-FP64
    solve (uref, ACC_REF_TOL), and of u32 against u64."""
    rep = dict(reference=f"all-FP64 multigrid, FGMRES to {ACC_REF_TOL:g} relative residual", slabs=len(uref),
               fp32_mg_vs_reference=[_rel(a, r) for a, r in zip(u32, uref)])
    if u64:
        rep["fp64_mg_vs_reference"] = [_rel(a, r) for a, r in zip(u64, uref)]
        rep["fp32_mg_vs_fp64_mg"] = [_rel(a, b) for a, b in zip(u32, u64)]
    rep["max_fp32_mg_vs_reference"] = max(rep["fp32_mg_vs_reference"])
    rep["target"] = 1e-7
    rep["meets_target"] = rep["max_fp32_mg_vs_reference"] <= 1e-7
    rep["solver_tol"] = tol
    return rep


def vanka_record_bytes(storage_bf16):
    """Bytes of one Q2 cell's Vanka record read per apply: V (27 x 27) in the
    storage type and the 27 FP32 eigenvalues (padding excluded)."""
    return 27 * 27 * (2 if storage_bf16 else 4) + 27 * 4


def kernel_roofline(stmg, torch, w, kappa, hbm, only=None, fp64=False, bf16=False):
    """Finest-level FP32 operator and Vanka apply timed in isolation with CUDA
    events on the launching stream; algorithmic bytes per launch:
      operator: 2 n_t N 4 (read src, write dst) + cells 4 (coefficient)
      Vanka:    cells (nd^2 s + nd 4) (eigenvectors in the storage type s,
                eigenvalues) + 2 n_t N 4
      h-transfer to the next coarser mesh (N_c nodes), FP32:
                prolongate-add n_t (N_c + 2 N) 4, restrict-add n_t (N + 2 N_c) 4."""
    n = 1 << w["refine"]
    mesh = stmg.Mesh(3, (n, n, n), 2, coeff=kappa)
    A, B, _, _, _ = stmg.time_weights(stmg.DG, 3, w["tau"], 1, stmg.HEAT)
    N, nt = w["nodes"], w["nt"]
    x = torch.randn(nt * N, device="cuda", dtype=torch.float64 if fp64 else torch.float32)
    y = torch.empty_like(x)
    s = torch.cuda.current_stream()
    out = {}
    op = stmg.Operator(mesh, A, B, dtype=stmg.F64 if fp64 else stmg.F32) if only in (None, "st_apply") else None
    vk = stmg.Vanka(mesh, A, B, compute=stmg.F32, storage=stmg.BF16 if bf16 else stmg.F32) \
        if only in (None, "vanka_apply") else None
    tr = xc = yc = None
    Nc = (n + 1) ** 3
    if only in (None, "h_transfer"):
        coarse = stmg.Mesh(3, (n // 2,) * 3, 2)
        tr = stmg.Transfer(mesh, coarse, nt, dtype=stmg.F32)
        xc = torch.randn(nt * Nc, device="cuda", dtype=torch.float32)
        yc = torch.zeros_like(xc)
        x32 = x.float()
        y32 = torch.zeros_like(x32)
    sz = 8 if fp64 else 4
    for name, fn, nbytes in (("st_apply", lambda: op.vmult(y, x), 2 * nt * N * sz + w["cells"] * sz),
                             ("vanka_apply", lambda: vk.vmult(y, x), w["cells"] * vanka_record_bytes(bf16) + 2 * nt * N * 4),
                             ("h_prolongate", lambda: tr.prolongate_add(y32, xc), nt * (Nc + 2 * N) * 4),
                             ("h_restrict", lambda: tr.restrict_add(yc, x32), nt * (N + 2 * Nc) * 4)):
        kind = "h_transfer" if name.startswith("h_") else name
        if only is not None and kind != only:
            continue
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        reps = 10
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        gbs = nbytes / t / 1e9
        out[name] = dict(ms=t * 1e3, bytes=nbytes, achieved=gbs, frac=gbs / hbm)
    del op, vk, tr, xc, yc, mesh
    torch.cuda.empty_cache()
    return out


def run_ours(args):
    import torch
    import stmg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    w = workload(args.refine)
    kappa, f = inputs(w, SEED + rank)
    hbm, hbm_kind = peaks()

    bf16 = args.vanka_storage == "bf16"

    def make(mg_dtype, tol=w["tol"], max_iter=200):
        storage = None if mg_dtype == stmg.F64 else (stmg.BF16 if bf16 else stmg.F32)
        return stmg.Solver(dim=3, refine=w["refine"], degree=2, time_degree=3, time_type=stmg.DG,
                           problem=stmg.HEAT, n_steps=1, tau=w["tau"], mg_dtype=mg_dtype, tol=tol,
                           abs_tol=1e-300, rhs_mode=1, f_nodal=f, fine_coeff=kappa, max_iter=max_iter,
                           vanka_storage=storage)

    n_acc = 0 if args.no_accuracy else w["n_slabs"]

    def timed(solver, steps, warmup):
        solver.set_initial(np.zeros(w["nodes"]))
        solver.run(warmup)
        solver.set_initial(np.zeros(w["nodes"]))
        s = torch.cuda.current_stream()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = stmg.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        torch.cuda.nvtx.range_push("timed_slabs")  # lets a profiler restrict itself to the timed slabs
        its = solver.run(steps)
        torch.cuda.nvtx.range_pop()
        e1.record(s)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        launches = stmg.kernel_launches() - l0
        t = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
        return t, its, launches

    t_setup = time.perf_counter()
    solver = make(stmg.F32)
    t_setup = time.perf_counter() - t_setup
    clocks = ClockSampler(local)
    clocks.start()
    t32, its32, launches = timed(solver, args.steps, args.warmup)
    clk = clocks.stop()
    dofs_step = w["nodes"] * w["nt"]
    value = replica_throughput(world, dofs_step, args.steps, t32)

    # end to end through the C ABI with host buffers: per step the slab's
    # source goes host -> device (pinned) and the slab solution comes back
    # (pinned, stmg_solver_solution_async: the download of slab k overlaps
    # the solve of slab k+1; the last one is waited for inside the timing)
    f_host = torch.from_numpy(f).pin_memory()
    u_host = torch.empty(w["nt"] * w["nodes"], dtype=torch.float64).pin_memory()
    solver.set_initial(np.zeros(w["nodes"]))
    torch.cuda.synchronize()
    te = time.perf_counter()
    u_np = u_host.numpy()
    for _ in range(args.steps):
        solver.set_source(f_host.numpy())
        solver.run(1)
        solver.solution_async(u_np)
    solver.solution_wait()
    torch.cuda.synchronize()
    te = time.perf_counter() - te
    e2e = dict(value=world * dofs_step * args.steps / te, unit="DoF/s", h2d_bytes_per_step=w["nodes"] * 8,
               d2h_bytes_per_step=w["nt"] * w["nodes"] * 8)
    u32 = slab_solutions(solver, w, n_acc)
    del solver
    torch.cuda.empty_cache()

    fp64, u64 = None, []
    if not args.no_fp64:
        s64 = make(stmg.F64)
        t64, its64, _ = timed(s64, args.steps, min(args.warmup, 1))
        fp64 = dict(value=world * dofs_step * args.steps / t64, ms_per_step=1e3 * t64 / args.steps,
                    fgmres_iterations=[int(i) for i in its64],
                    speedup_fp32_mg=(world * dofs_step * args.steps / t32) / (world * dofs_step * args.steps / t64))
        u64 = slab_solutions(s64, w, n_acc)
        del s64
        torch.cuda.empty_cache()

    accuracy = None
    if n_acc:
        sref = make(stmg.F64, tol=ACC_REF_TOL, max_iter=1000)
        uref = slab_solutions(sref, w, n_acc)
        del sref
        torch.cuda.empty_cache()
        accuracy = accuracy_report(u32, u64, uref, w["tol"])
    del u32, u64

    kr = kernel_roofline(stmg, torch, w, kappa, hbm, bf16=bf16)
    dom = max(kr, key=lambda k: kr[k]["ms"])
    traffic = vanka_traffic(w["refine"], args.vanka_storage) if dom == "vanka_apply" else None
    roof = dict(kernel=dom, bound="hbm", achieved=kr[dom]["achieved"], peak=hbm, unit="GB/s",
                frac=kr[dom]["frac"], traffic=traffic, peak_kind=hbm_kind,
                kernels={k: dict(ms=v["ms"], algorithmic_bytes=v["bytes"], achieved_gbs=v["achieved"], frac=v["frac"])
                         for k, v in kr.items()})

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, _ = cpu_sample(w)

    if rank == 0:
        line = dict(metric=METRIC, value=value, unit="DoF/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=1e3 * t32 / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f32", data="synthetic",
                    config=dict(workload=w["name"], cells=w["cells"], nodes=w["nodes"], time_dofs=w["nt"],
                                dofs_per_slab=dofs_step, outer="fgmres-fp64", mg="fp32 v-cycle, cell-patch vanka",
                                vanka_storage=args.vanka_storage,
                                tol=w["tol"], l2="inputs larger than L2 (FGMRES basis 30 x 0.54 GB)",
                                parallelism="replicas" if world > 1 else "single-gpu", setup_s=t_setup),
                    fgmres_iterations=[int(i) for i in its32], e2e=e2e, roofline=roof, cpu_baseline=cpu,
                    clocks=clk, gpu_launches=int(launches), fp64_mg=fp64, accuracy=accuracy)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_config(args):
    """--config c1|c2|c3: the other configurations of the slab solve, timed
    the same way as the main line (device events, inputs resident, W warm-up
    slabs then K timed slabs) and compared across multigrid precisions:
      c1  2-D 16^2 Q2, dG(1), dt 1/64, frequency 1/2, 2 sweeps, FP64, tol 1e-10;
      c2  3-D 32^3 Q3, vertices moved +-0.2h, kappa = 10^U(-2,2), dG(2),
          dt 1/32, f = 1: FP32 vs FP64 multigrid;
      c3  3-D wave 64^3 Q2, c^2 in {0.5, 1, 4}, dG(2), dt 1/128, Gaussian
          pulse, v0 = 0, f = 0: Vanka stored in FP32 vs BF16.
    For c2 and c3 a converged all-FP64 solve of the same slabs is run last
    and the line's `accuracy` gives each variant's relative difference from
    it after the last slab."""
    import torch
    import meshes
    import stmg
    rng = np.random.default_rng(SEED)
    init = None
    if args.config == "c1":
        name = "heat2d-16^2-Q2-dG1-c1"
        base = dict(dim=2, refine=4, degree=2, time_degree=1, time_type=stmg.DG, problem=stmg.HEAT, n_steps=1,
                    tau=1 / 64, fe_degree_min=0, n_steps_min=1, tol=1e-10, abs_tol=1e-14, frequency=0.5,
                    smoothing_steps=2)
        variants = {"fp64-mg": dict(mg_dtype=stmg.F64)}
    elif args.config == "c2":
        n = 32
        name = "heat3d-32^3-Q3-dG2-distorted-c2"
        V = meshes.vertices(3, (n, n, n), distort=0.2, seed=SEED)
        kappa = 10.0 ** rng.uniform(-2, 2, n ** 3)
        base = dict(dim=3, refine=5, degree=3, time_degree=2, time_type=stmg.DG, problem=stmg.HEAT, n_steps=1,
                    tau=1 / 32, fe_degree_min=0, n_steps_min=1, tol=1e-8, abs_tol=1e-300, rhs_mode=1,
                    f_nodal=np.ones((3 * n + 1) ** 3), fine_coeff=kappa, fine_vertices=V)
        variants = {"fp32-mg": dict(mg_dtype=stmg.F32), "fp64-mg": dict(mg_dtype=stmg.F64)}
    else:
        n = 64
        name = "wave3d-64^3-Q2-dG2-c3"
        c2 = rng.choice([0.5, 1.0, 4.0], size=n ** 3)
        X = meshes.vertices(3, (2 * n, 2 * n, 2 * n))
        u0 = np.exp(-np.sum((X - 0.5) ** 2, axis=1) / 0.01)
        u0[meshes.boundary_mask(3, (n, n, n), 2)] = 0.0
        init = (u0, np.zeros_like(u0))
        base = dict(dim=3, refine=6, degree=2, time_degree=2, time_type=stmg.DG, problem=stmg.WAVE, n_steps=1,
                    tau=1 / 128, fe_degree_min=0, n_steps_min=1, tol=1e-8, abs_tol=1e-300, rhs_mode=2,
                    fine_coeff=c2)
        variants = {"fp32-vanka": dict(mg_dtype=stmg.F32, vanka_storage=stmg.F32),
                    "bf16-vanka": dict(mg_dtype=stmg.F32, vanka_storage=stmg.BF16)}
    if args.config != "c1":
        # a converged all-FP64 solve of the same slabs, for the accuracy figures
        variants["reference"] = dict(mg_dtype=stmg.F64, tol=ACC_REF_TOL, max_iter=1000)
    out, sols = {}, {}
    for vname, vkw in variants.items():
        s = stmg.Solver(**{**base, **vkw})
        if init is not None:
            s.set_initial(*init)
        s.run(args.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.cuda.nvtx.range_push(f"timed_slabs_{vname}")  # lets a profiler restrict itself to these slabs
        its = s.run(args.steps)
        torch.cuda.nvtx.range_pop()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        dofs = s.n_nodes * s.n_blocks * args.steps
        entry = dict(value=dofs / t, unit="DoF/s", ms_per_step=1e3 * t / args.steps,
                     fgmres_iterations=[int(i) for i in its])
        if args.config == "c1":
            entry["errors"] = dict(zip(("linf", "l2", "h1"), s.errors()))
        else:
            sols[vname] = s.solution(want_v=False)[0]
        out[vname] = entry
        del s
        torch.cuda.empty_cache()
    line = dict(workload=name, steps=args.steps, warmup=args.warmup, slabs=args.warmup + args.steps, variants=out)
    if sols:
        # relative 2-norm difference of each variant's last slab solution
        # (after warmup + steps slabs from the same initial state) from the
        # converged all-FP64 solve
        ref = sols.pop("reference")
        line["accuracy"] = dict(reference=f"all-FP64 multigrid, FGMRES to {ACC_REF_TOL:g} relative residual",
                                target=1e-7, **{f"{k}_vs_reference": _rel(u, ref) for k, u in sols.items()})
        if len(sols) == 2:
            (ka, ua), (kb, ub) = sols.items()
            line["accuracy"][f"{ka}_vs_{kb}"] = _rel(ua, ub)
    print(json.dumps(line), flush=True)
    return 0


def smoothed_field(n, seed, sigma_cells=1.0):
    """White noise N(0, 1) on the n^3 cells, smoothed by a Gaussian of
    sigma_cells cells (scipy.ndimage.gaussian_filter, reflecting edges) and
    scaled back to unit standard deviation."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    w = gaussian_filter(rng.standard_normal((n, n, n)), sigma=sigma_cells, mode="reflect")
    return (w / w.std()).reshape(-1)


def run_adjoint(args):
    """--adjoint: the adjoint-gradient configuration: heat, 32^3 Q2 cells,
    dG(1), 16 slabs of dt = 1/16, f = 1. The true log-coefficient is
    Gaussian-smoothed white noise (sigma = 1 cell, unit standard deviation,
    seeded); the observations are a forward FP64 solve with the true field
    plus 1e-3 relative Gaussian noise; the gradient of the misfit is taken at
    the initial guess theta = 0 with checkpoints every 4 slabs (FP64
    multigrid, 1e-12), through the torch.autograd.Function wrapper, timed,
    and checked against central finite differences of forward solves on
    --fd random unit directions (h = 1e-4). The same construction on 8^3
    cells is checked against central differences of the oracle's FP64 solves
    (--fd-oracle directions)."""
    import torch
    import stmg
    from stmg.adjoint import misfit, misfit_value
    import oracle_py as orc

    def setup(n, S, seed):
        rng = np.random.default_rng(seed)
        truth = smoothed_field(n, seed)
        f = np.ones((2 * n + 1) ** 3)
        kw = dict(dim=3, refine=int(np.log2(n)), degree=2, time_degree=1, time_type=stmg.DG, problem=stmg.HEAT,
                  n_steps=1, tau=1 / 16, fe_degree_min=0, n_steps_min=1, rhs_mode=1, f_nodal=f, tol=1e-12,
                  abs_tol=1e-300, mg_dtype=stmg.F64)

        def make(kappa):
            return stmg.Solver(fine_coeff=kappa, **kw)

        clean = []
        sv = make(np.exp(truth))
        for _ in range(S):
            sv.run(1)
            clean.append(sv.solution(want_v=False)[0])
        clean = np.array(clean)
        obs = clean * (1 + 1e-3 * rng.standard_normal(clean.shape))
        return rng, truth, f, make, obs

    n, S = 32, 16
    rng, truth, f, make, obs = setup(n, S, SEED)
    theta = torch.zeros(n ** 3, dtype=torch.float64, requires_grad=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J = misfit(theta, make, obs, 4)
    J.backward()
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    g = theta.grad.numpy()
    checks = []
    h = 1e-4
    for _ in range(args.fd):
        d = rng.standard_normal(theta.numel())
        d /= np.linalg.norm(d)
        fd = (misfit_value(h * d, make, obs) - misfit_value(-h * d, make, obs)) / (2 * h)
        checks.append(dict(gd=float(g @ d), fd=fd, rel=abs(float(g @ d) - fd) / max(abs(fd), 1e-300)))

    # the same construction on 8^3 cells: GPU gradient against central
    # differences of the oracle's FP64 solves
    n8 = 8
    rng8, truth8, f8, make8, obs8 = setup(n8, S, SEED + 1)
    th8 = torch.zeros(n8 ** 3, dtype=torch.float64, requires_grad=True)
    J8 = misfit(th8, make8, obs8, 4)
    J8.backward()
    g8 = th8.grad.numpy()

    def oracle_misfit(th):
        r = orc.run(dim=3, refine=3, p=2, r=1, ttype=orc.DG, problem=orc.HEAT, n_steps=1, tau=1 / 16, n_slabs=S,
                    fe_degree_min=0, n_steps_min=1, mg_float=False, tol=1e-13, abs_tol=1e-300, rhs_mode=1, f_nodal=f8,
                    fine_coeff=np.exp(th), compute_errors=False, keep_all=True)
        return 0.5 * float(np.sum((r["u_all"] - obs8) ** 2))

    ochecks = []
    for _ in range(args.fd_oracle):
        d = rng8.standard_normal(n8 ** 3)
        d /= np.linalg.norm(d)
        fd = (oracle_misfit(h * d) - oracle_misfit(-h * d)) / (2 * h)
        ochecks.append(dict(gd=float(g8 @ d), fd_oracle=fd, rel=abs(float(g8 @ d) - fd) / max(abs(fd), 1e-300)))
    print(json.dumps(dict(workload="heat3d-32^3-Q2-dG1-16slabs-adjoint", misfit=float(J), gradient_seconds=t,
                          parameters=int(theta.numel()), initial_guess="theta = 0",
                          true_field="Gaussian-smoothed white noise, sigma 1 cell, unit std",
                          checkpoint_every=4, fd_h=h, fd_checks=checks,
                          max_fd_rel=max(c["rel"] for c in checks) if checks else None,
                          oracle_check=dict(workload="heat3d-8^3-Q2-dG1-16slabs", misfit=float(J8),
                                            checks=ochecks))), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--refine", type=int, default=7, help="mesh 2^refine cells per direction (7: 128^3)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the all-FP64 V-cycle comparison")
    ap.add_argument("--vanka-storage", choices=["f32", "bf16"], default="f32",
                    help="storage of the FP32 V-cycle's Vanka eigenvectors")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle sample")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the per-slab comparison of the FP32-MG and FP64-MG solutions with a converged "
                         "FP64 solve")
    ap.add_argument("--kernels-only", choices=["all", "st_apply", "st_apply64", "vanka_apply", "h_transfer"], default=None,
                    help="only time the finest-level operator (FP32 or FP64), Vanka apply and/or h-transfers "
                         "in isolation (profiling)")
    ap.add_argument("--adjoint", action="store_true", help="time the adjoint gradient configuration")
    ap.add_argument("--config", choices=["c1", "c2", "c3"], default=None,
                    help="time one of the other configurations (not the main metric line)")
    ap.add_argument("--fd", type=int, default=8, help="finite-difference directions checked with --adjoint")
    ap.add_argument("--fd-oracle", type=int, default=2,
                    help="directions checked against the oracle's FP64 solves with --adjoint (8^3 cells)")
    args = ap.parse_args()
    if args.adjoint:
        return run_adjoint(args)
    if args.config:
        return run_config(args)
    if args.kernels_only:
        import torch
        import stmg
        w = workload(args.refine)
        kappa, _ = inputs(w)
        hbm, kind = peaks()
        only = None if args.kernels_only == "all" else args.kernels_only.replace("64", "")
        kr = kernel_roofline(stmg, torch, w, kappa, hbm, only, fp64=args.kernels_only == "st_apply64",
                             bf16=args.vanka_storage == "bf16")
        print(json.dumps(dict(workload=w["name"], peak_gbs=hbm, peak_kind=kind, kernels=kr)), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
