// extern "C" entry points of libstmg_cuda.so (declared in include/stmg.h).
#include <atomic>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>

#include "solver.h"
#include "time_fe.h"
#include "st_operator.h"
#include "stmg_internal.h"
#include "transfer.h"
#include "vanka.h"

struct stmg_mesh_s
{
  std::unique_ptr<stmg::Mesh> m;
};
struct stmg_op_s
{
  std::unique_ptr<stmg::StOperator> op;
};
struct stmg_vanka_s
{
  std::unique_ptr<stmg::Vanka> vk;
};
struct stmg_transfer_s
{
  std::unique_ptr<stmg::Transfer> tr;
  long long                       fine_size;
  int                             elem;
};
struct stmg_solver_s
{
  std::unique_ptr<stmg::SlabSolver> s;
};

namespace stmg
{
  namespace
  {
    thread_local std::string last_error;
  }
  void
  set_last_error(const std::string &m)
  {
    last_error = m;
  }

  namespace
  {
    std::atomic<long long> launches{0};
  }
  void
  count_launch()
  {
    launches.fetch_add(1, std::memory_order_relaxed);
  }
  void
  add_launches(long long n)
  {
    launches.fetch_add(n, std::memory_order_relaxed);
  }
  long long
  launch_count()
  {
    return launches.load(std::memory_order_relaxed);
  }

  template <typename F>
  int
  guard(F &&f)
  {
    try
      {
        f();
        return STMG_OK;
      }
    catch (const Error &e)
      {
        last_error = e.what();
        return e.code;
      }
    catch (const std::bad_alloc &)
      {
        last_error = "host allocation failed";
        return STMG_ERR_NOMEM;
      }
    catch (const std::exception &e)
      {
        last_error = e.what();
        return STMG_ERR_ARG;
      }
  }

  const char *
  last_error_cstr()
  {
    return last_error.c_str();
  }
} // namespace stmg

using namespace stmg;

extern "C"
{
  const char *
  stmg_last_error(void)
  {
    return last_error_cstr();
  }

  int
  stmg_version(void)
  {
    return 1;
  }

  int
  stmg_kernel_launches(long long *count)
  {
    return guard([&] {
      STMG_REQUIRE(count, STMG_ERR_ARG, "kernel_launches: null argument");
      *count = launch_count();
    });
  }

  int
  stmg_time_weights(int time_type, int r, double tau, int n_steps, int problem, double *Alpha, double *Beta,
                    double *rK, double *rM, double *rV)
  {
    return guard([&] {
      STMG_REQUIRE(time_type == 1 || time_type == 2, STMG_ERR_ARG, "time_weights: time type 1 (cGP) or 2 (dG)");
      STMG_REQUIRE(problem == 1 || problem == 2, STMG_ERR_ARG, "time_weights: problem 1 (heat) or 2 (wave)");
      STMG_REQUIRE(r >= (time_type == 2 ? 0 : 1) && n_steps >= 1 && tau > 0, STMG_ERR_ARG, "time_weights: bad degree/steps");
      STMG_REQUIRE(Alpha && Beta && rK && rM, STMG_ERR_ARG, "time_weights: null output");
      const auto t  = tfe::Type(time_type);
      auto       wn = tfe::slab_weights(t, r, tau, n_steps);
      const int  nt = wn[0].m;
      if (problem == 1)
        {
          std::copy(wn[0].a.begin(), wn[0].a.end(), Alpha);
          std::copy(wn[1].a.begin(), wn[1].a.end(), Beta);
          for (int i = 0; i < nt; ++i)
            {
              rK[i] = t == tfe::CGP ? wn[2](i, 0) : 0.0;
              rM[i] = t == tfe::CGP ? wn[3](i, 0) : wn[2](i, 0);
              if (rV)
                rV[i] = 0.0;
            }
        }
      else
        {
          auto w1 = tfe::slab_weights(t, r, tau, 1);
          auto ww = tfe::wave_weights(t, w1[0], w1[1], w1[2], w1[3], n_steps);
          std::copy(ww[0].a.begin(), ww[0].a.end(), Alpha);
          std::copy(ww[1].a.begin(), ww[1].a.end(), Beta);
          for (int i = 0; i < nt; ++i)
            {
              rK[i] = ww[2](i, 0);
              rM[i] = ww[3](i, 0);
              if (rV)
                rV[i] = ww[4](i, 0);
            }
        }
    });
  }

  int
  stmg_time_transfer(int time_type, int kind, int r, int n_steps, double *P)
  {
    return guard([&] {
      STMG_REQUIRE(time_type == 1 || time_type == 2, STMG_ERR_ARG, "time_transfer: time type 1 (cGP) or 2 (dG)");
      STMG_REQUIRE(kind == 0 || kind == 1, STMG_ERR_ARG, "time_transfer: kind 0 (k projection) or 1 (tau)");
      STMG_REQUIRE(n_steps >= 1 && P, STMG_ERR_ARG, "time_transfer: bad steps or null output");
      STMG_REQUIRE(kind == 1 || r >= (time_type == 2 ? 1 : 2), STMG_ERR_ARG,
                   "time_transfer: the k projection needs a coarse degree r - 1 of the time type");
      STMG_REQUIRE(kind == 0 || (n_steps % 2 == 0 && r >= (time_type == 2 ? 0 : 1)), STMG_ERR_ARG,
                   "time_transfer: the tau prolongation needs an even step count");
      const auto      t = tfe::Type(time_type);
      const tfe::Mat  M = kind == 0 ? tfe::projection(t, r - 1, r, n_steps) : tfe::prolongation(t, r, n_steps);
      std::copy(M.a.begin(), M.a.end(), P);
    });
  }

  int
  stmg_block_permute(int n_blocks, long long n, const long long *perm, int scatter, const void *src, void *dst,
                     int dtype, void *stream)
  {
    return guard([&] { block_permute(n_blocks, n, perm, scatter, src, dst, dtype, static_cast<cudaStream_t>(stream)); });
  }

  int
  stmg_mesh_create(int dim, const int *n_cells, int degree, const double *lo, const double *hi, const double *vertices,
                   int coeff_mode, const double *coeff, stmg_mesh_t *mesh)
  {
    return guard([&] {
      STMG_REQUIRE(n_cells && lo && hi && mesh, STMG_ERR_ARG, "mesh_create: null argument");
      auto h = new stmg_mesh_s;
      try
        {
          h->m = make_mesh(dim, n_cells, degree, lo, hi, vertices, coeff_mode, coeff);
        }
      catch (...)
        {
          delete h;
          throw;
        }
      *mesh = h;
    });
  }

  int
  stmg_mesh_destroy(stmg_mesh_t mesh)
  {
    return guard([&] {
      STMG_REQUIRE(mesh, STMG_ERR_HANDLE, "mesh_destroy: null handle");
      delete mesh;
    });
  }

  int
  stmg_mesh_info(stmg_mesh_t mesh, long long *n_nodes, long long *n_cells)
  {
    return guard([&] {
      STMG_REQUIRE(mesh && mesh->m, STMG_ERR_HANDLE, "mesh_info: null handle");
      if (n_nodes)
        *n_nodes = mesh->m->v.N;
      if (n_cells)
        *n_cells = mesh->m->v.ncells;
    });
  }

  int
  stmg_op_create(stmg_mesh_t mesh, int nt_out, int nt_in, const double *A, const double *B, int dtype, stmg_op_t *op)
  {
    return guard([&] {
      STMG_REQUIRE(mesh && mesh->m, STMG_ERR_HANDLE, "op_create: null mesh");
      STMG_REQUIRE(A && B && op, STMG_ERR_ARG, "op_create: null argument");
      auto h = new stmg_op_s;
      try
        {
          h->op = std::make_unique<StOperator>(mesh->m.get(), nt_out, nt_in, A, B, dtype);
        }
      catch (...)
        {
          delete h;
          throw;
        }
      *op = h;
    });
  }

  int
  stmg_op_destroy(stmg_op_t op)
  {
    return guard([&] {
      STMG_REQUIRE(op, STMG_ERR_HANDLE, "op_destroy: null handle");
      delete op;
    });
  }

  int
  stmg_op_vmult(stmg_op_t op, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      NvtxScope range("vmult");
      STMG_REQUIRE(op && op->op, STMG_ERR_HANDLE, "op_vmult: null handle");
      op->op->apply(false, src, dst, false, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_op_vmult_box_noalloc(int dim, const int *n_cells, int degree, const double *lo, const double *hi,
                            const void *coeff, int nt_out, int nt_in, const double *A, const double *B, int dtype,
                            void *dst, const void *src, void *stream)
  {
    return guard([&] {
      op_vmult_box_noalloc(dim, n_cells, degree, lo, hi, coeff, nt_out, nt_in, A, B, dtype, src, dst,
                           static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_op_diagonal(stmg_op_t op, int inverse, void *dst, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(op && op->op, STMG_ERR_HANDLE, "op_diagonal: null handle");
      op->op->diagonal(inverse != 0, dst, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_op_Tvmult(stmg_op_t op, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      NvtxScope range("Tvmult");
      STMG_REQUIRE(op && op->op, STMG_ERR_HANDLE, "op_Tvmult: null handle");
      op->op->apply(true, src, dst, false, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_op_vmult_add(stmg_op_t op, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      NvtxScope range("vmult");
      STMG_REQUIRE(op && op->op, STMG_ERR_HANDLE, "op_vmult_add: null handle");
      op->op->apply(false, src, dst, true, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_vanka_create(stmg_mesh_t mesh, int nt, const double *Alpha, const double *Beta, int compute_dtype,
                    int storage_dtype, stmg_vanka_t *vanka)
  {
    return guard([&] {
      STMG_REQUIRE(mesh && mesh->m, STMG_ERR_HANDLE, "vanka_create: null mesh");
      STMG_REQUIRE(Alpha && Beta && vanka, STMG_ERR_ARG, "vanka_create: null argument");
      auto h = std::make_unique<stmg_vanka_s>();
      h->vk  = std::make_unique<Vanka>(mesh->m.get(), nt, Alpha, Beta, compute_dtype, storage_dtype);
      *vanka = h.release();
    });
  }

  int
  stmg_vanka_destroy(stmg_vanka_t vanka)
  {
    return guard([&] {
      STMG_REQUIRE(vanka, STMG_ERR_HANDLE, "vanka_destroy: null handle");
      delete vanka;
    });
  }

  int
  stmg_vanka_vmult(stmg_vanka_t vanka, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      NvtxScope range("vanka");
      STMG_REQUIRE(vanka && vanka->vk, STMG_ERR_HANDLE, "vanka_vmult: null handle");
      vanka->vk->apply(src, dst, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_relax_step(stmg_vanka_t vanka, stmg_op_t op, double omega, void *x, const void *b, void *tmp, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(vanka && vanka->vk && op && op->op, STMG_ERR_HANDLE, "relax_step: null handle");
      STMG_REQUIRE(x && b && tmp, STMG_ERR_ARG, "relax_step: null vector");
      const Vanka      &vk = *vanka->vk;
      const StOperator &A  = *op->op;
      STMG_REQUIRE(A.mesh == vk.mesh && A.nt_in == vk.nt && A.nt_out == vk.nt && A.dtype == vk.compute, STMG_ERR_SHAPE,
                   "relax_step: operator and smoother differ in mesh, time dofs or type");
      const cudaStream_t s = static_cast<cudaStream_t>(stream);
      A.apply_ex(false, x, tmp, -1.0, 0.0, b, s); // tmp = b - A x
      vk.apply_ex(tmp, x, omega, 1.0, s);         // x += omega P tmp
    });
  }

  int
  stmg_transfer_h_create(stmg_mesh_t fine, stmg_mesh_t coarse, int nt, int dtype, stmg_transfer_t *tr)
  {
    return guard([&] {
      STMG_REQUIRE(fine && fine->m && coarse && coarse->m, STMG_ERR_HANDLE, "transfer_h_create: null mesh");
      STMG_REQUIRE(tr && (dtype == STMG_F64 || dtype == STMG_F32), STMG_ERR_ARG, "transfer_h_create: bad argument");
      auto h       = std::make_unique<stmg_transfer_s>();
      h->tr        = std::make_unique<HTransfer>(fine->m.get(), coarse->m.get(), nt, dtype);
      h->fine_size = fine->m->v.N * nt;
      h->elem      = dtype == STMG_F64 ? 8 : 4;
      *tr          = h.release();
    });
  }

  int
  stmg_transfer_t_create(stmg_mesh_t mesh, int nt_fine, int nt_coarse, const double *P, const double *R, int dtype,
                         stmg_transfer_t *tr)
  {
    return guard([&] {
      STMG_REQUIRE(mesh && mesh->m, STMG_ERR_HANDLE, "transfer_t_create: null mesh");
      STMG_REQUIRE(P && tr && (dtype == STMG_F64 || dtype == STMG_F32), STMG_ERR_ARG, "transfer_t_create: bad argument");
      auto h       = std::make_unique<stmg_transfer_s>();
      h->tr        = std::make_unique<TTransfer>(mesh->m.get(), nt_fine, nt_coarse, P, R, dtype);
      h->fine_size = mesh->m->v.N * nt_fine;
      h->elem      = dtype == STMG_F64 ? 8 : 4;
      *tr          = h.release();
    });
  }

  int
  stmg_transfer_destroy(stmg_transfer_t tr)
  {
    return guard([&] {
      STMG_REQUIRE(tr, STMG_ERR_HANDLE, "transfer_destroy: null handle");
      delete tr;
    });
  }

  int
  stmg_transfer_prolongate(stmg_transfer_t tr, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(tr && tr->tr, STMG_ERR_HANDLE, "transfer_prolongate: null handle");
      STMG_REQUIRE(dst && src, STMG_ERR_ARG, "transfer_prolongate: null vector");
      STMG_CUDA(cudaMemsetAsync(dst, 0, tr->fine_size * tr->elem, static_cast<cudaStream_t>(stream)));
      tr->tr->prolongate_add(src, dst, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_transfer_prolongate_add(stmg_transfer_t tr, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(tr && tr->tr, STMG_ERR_HANDLE, "transfer_prolongate_add: null handle");
      STMG_REQUIRE(dst && src, STMG_ERR_ARG, "transfer_prolongate_add: null vector");
      tr->tr->prolongate_add(src, dst, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_transfer_restrict_add(stmg_transfer_t tr, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(tr && tr->tr, STMG_ERR_HANDLE, "transfer_restrict_add: null handle");
      STMG_REQUIRE(dst && src, STMG_ERR_ARG, "transfer_restrict_add: null vector");
      tr->tr->restrict_add(src, dst, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_solver_create(const stmg_solver_config *c, stmg_solver_t *solver)
  {
    return guard([&] {
      STMG_REQUIRE(c && solver, STMG_ERR_ARG, "solver_create: null argument");
      STMG_REQUIRE(c->dim == 2 || c->dim == 3, STMG_ERR_ARG, "solver_create: dim must be 2 or 3");
      STMG_REQUIRE(c->refine >= 0 && c->refine < 16, STMG_ERR_ARG, "solver_create: refine out of range");
      STMG_REQUIRE(c->n_steps >= 1 && c->tau > 0, STMG_ERR_ARG, "solver_create: bad time step");
      SolverConfig s;
      s.dim = c->dim;
      for (int d = 0; d < 3; ++d)
        {
          s.subdiv[d] = d < c->dim ? c->subdiv[d] : 1;
          s.lo[d]     = c->lo[d];
          s.hi[d]     = c->hi[d];
        }
      s.refine          = c->refine;
      s.degree          = c->degree;
      s.time_degree     = c->time_degree;
      s.time_type       = c->time_type;
      s.problem         = c->problem;
      s.n_steps         = c->n_steps;
      s.tau             = c->tau;
      s.smoothing_steps = c->smoothing_steps > 0 ? c->smoothing_steps : 1;
      s.fe_degree_min   = c->fe_degree_min;
      s.n_steps_min     = c->n_steps_min;
      s.mg_dtype        = c->mg_dtype;
      s.vanka_storage   = c->vanka_storage;
      s.tol             = c->tol;
      s.abs_tol         = c->abs_tol;
      s.max_iter        = c->max_iter;
      s.restart         = c->restart > 0 ? c->restart : 30;
      s.extrapolate     = c->extrapolate;
      s.rhs_mode        = c->rhs_mode;
      s.frequency       = c->frequency;
      long long nv = 1, nc = 1, nn = 1;
      for (int d = 0; d < c->dim; ++d)
        {
          const long long n = (long long)s.subdiv[d] << c->refine;
          nv *= n + 1;
          nc *= n;
          nn *= n * c->degree + 1;
        }
      if (c->fine_vertices)
        s.fine_vertices.assign(c->fine_vertices, c->fine_vertices + nv * c->dim);
      if (c->fine_coeff)
        s.fine_coeff.assign(c->fine_coeff, c->fine_coeff + nc);
      if (c->rhs_mode == 1)
        {
          STMG_REQUIRE(c->f_nodal, STMG_ERR_ARG, "solver_create: rhs_mode 1 needs f_nodal");
          s.f_nodal.assign(c->f_nodal, c->f_nodal + nn);
        }
      auto h = std::make_unique<stmg_solver_s>();
      h->s   = std::make_unique<SlabSolver>(s);
      *solver = h.release();
    });
  }

  int
  stmg_solver_destroy(stmg_solver_t solver)
  {
    return guard([&] {
      STMG_REQUIRE(solver, STMG_ERR_HANDLE, "solver_destroy: null handle");
      delete solver;
    });
  }

  int
  stmg_solver_info(stmg_solver_t solver, long long *n_nodes, int *n_blocks, int *n_levels, double *omegas)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_info: null handle");
      if (n_nodes)
        *n_nodes = solver->s->N;
      if (n_blocks)
        *n_blocks = solver->s->nb;
      if (n_levels)
        *n_levels = int(solver->s->gmg->levels.size());
      if (omegas)
        {
          auto o = solver->s->gmg->omegas();
          std::copy(o.begin(), o.end(), omegas);
        }
    });
  }

  int
  stmg_solver_set_initial(stmg_solver_t solver, const double *u0, const double *v0)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_set_initial: null handle");
      solver->s->set_initial(u0, v0);
    });
  }

  int
  stmg_solver_set_source(stmg_solver_t solver, const double *f_nodal)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_set_source: null handle");
      STMG_REQUIRE(f_nodal, STMG_ERR_ARG, "solver_set_source: null source");
      solver->s->set_source(f_nodal);
    });
  }

  int
  stmg_solver_point_values(stmg_solver_t solver, int n_points, const double *points, int samples_per_step,
                           double *times, double *values, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_point_values: null handle");
      const int r       = solver->s->cfg.time_degree;
      const int samples = samples_per_step > 0 ? samples_per_step : (r + 1) * (r + 1);
      solver->s->point_values(n_points, points, samples, times, values, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_solver_set_control(stmg_solver_t solver, double tol, double abs_tol, int max_iter)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_set_control: null handle");
      STMG_REQUIRE(tol >= 0 && abs_tol >= 0 && max_iter >= 1, STMG_ERR_ARG,
                   "solver_set_control: tolerances >= 0 and max_iter >= 1");
      solver->s->cfg.tol      = tol;
      solver->s->cfg.abs_tol  = abs_tol;
      solver->s->cfg.max_iter = max_iter;
    });
  }

  int
  stmg_solver_run(stmg_solver_t solver, int n_slabs, int *iterations, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_run: null handle");
      STMG_REQUIRE(n_slabs >= 0, STMG_ERR_ARG, "solver_run: negative slab count");
      solver->s->run(n_slabs, iterations, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_solver_solution(stmg_solver_t solver, double *u, double *v)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_solution: null handle");
      solver->s->download(u, v);
    });
  }

  int
  stmg_solver_solution_async(stmg_solver_t solver, double *u, double *v, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_solution_async: null handle");
      solver->s->download_async(u, v, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_solver_solution_wait(stmg_solver_t solver)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_solution_wait: null handle");
      solver->s->download_wait();
    });
  }

  int
  stmg_solver_solve(stmg_solver_t solver, double *x, const double *rhs, int *iterations, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_solve: null handle");
      STMG_REQUIRE(x && rhs, STMG_ERR_ARG, "solver_solve: null vector");
      const int k = solver->s->solve(x, rhs, static_cast<cudaStream_t>(stream));
      if (iterations)
        *iterations = k;
    });
  }

  int
  stmg_solver_errors(stmg_solver_t solver, double *linf, double *l2, double *h1)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_errors: null handle");
      STMG_REQUIRE(linf && l2 && h1, STMG_ERR_ARG, "solver_errors: null argument");
      *linf = solver->s->err_l8;
      *l2   = std::sqrt(solver->s->err_l2sq);
      *h1   = std::sqrt(solver->s->err_h1sq);
    });
  }

  int
  stmg_solver_gradient(stmg_solver_t solver, int n_slabs, const double *u_obs, int checkpoint_every, double *misfit,
                       double *grad, int *its_fwd, int *its_adj, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_gradient: null handle");
      STMG_REQUIRE(u_obs && grad && misfit, STMG_ERR_ARG, "solver_gradient: null argument");
      *misfit = solver->s->gradient(n_slabs, u_obs, checkpoint_every, grad, its_fwd, its_adj,
                                    static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_gmg_vmult(stmg_solver_t solver, double *dst, const double *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "gmg_vmult: null handle");
      STMG_REQUIRE(dst && src, STMG_ERR_ARG, "gmg_vmult: null vector");
      solver->s->gmg->vmult(dst, src, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_solver_system_vmult(stmg_solver_t solver, double *dst, const double *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(solver && solver->s, STMG_ERR_HANDLE, "solver_system_vmult: null handle");
      STMG_REQUIRE(dst && src, STMG_ERR_ARG, "solver_system_vmult: null vector");
      solver->s->system_vmult(dst, src, static_cast<cudaStream_t>(stream));
    });
  }
}
