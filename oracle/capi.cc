// Oracle (test infrastructure only): C entry points used by tests/ (through
// ctypes) and by the bench's CPU-baseline leg. Nothing in the product links
// this library.
#include <cstring>
#include <exception>
#include <string>

#include "solver.h"

using namespace oracle;

namespace
{
  thread_local std::string last_error;

  template <typename F>
  int
  guard(F &&f)
  {
    try
      {
        f();
        return 0;
      }
    catch (const std::exception &e)
      {
        last_error = e.what();
        return -1;
      }
  }

  DMat
  to_mat(const double *a, int m, int n)
  {
    DMat M(m, n);
    if (a)
      std::memcpy(M.a.data(), a, sizeof(double) * m * n);
    return M;
  }

  void
  from_mat(const DMat &M, double *out)
  {
    std::memcpy(out, M.a.data(), sizeof(double) * M.a.size());
  }
} // namespace

// Flat configuration record mirrored by tests/oracle_py.py.
struct OrcConfig
{
  int    dim, subdiv[3], refine, p, r, type, problem, n_steps, n_slabs;
  double tau, lo[3], hi[3];
  int    smoothing_steps, variable, estimate_relaxation, restrict_is_transpose;
  int    fe_degree_min, n_steps_min, mg_float, extrapolate, max_iter, restart, rhs_mode,
    compute_errors;
  double tol, abs_tol, frequency;
  const double *f_nodal, *u0_nodal, *v0_nodal, *fine_vertices, *fine_coeff;
};

struct OrcResult
{
  int    total_iterations, n_levels, n_blocks;
  double l8, l2, h1;
  long   n_dofs, n_cells;
};

extern "C"
{
  const char *
  orc_last_error()
  {
    return last_error.c_str();
  }

  void *
  orc_mesh_create(int dim, const int *n, int p, const double *lo, const double *hi, const double *vertices,
                  int coeff_mode, const double *coeff)
  {
    auto *m = new Mesh();
    m->init(dim, n, p, lo, hi);
    if (vertices)
      m->set_vertices(vertices);
    m->coeff_mode = coeff_mode;
    if (coeff_mode == 1)
      m->coeff.assign(coeff, coeff + m->n_cells);
    else if (coeff_mode == 2)
      m->coeff.assign(coeff, coeff + m->n_cells * m->nq);
    return m;
  }

  void
  orc_mesh_destroy(void *m)
  {
    delete static_cast<Mesh *>(m);
  }

  long
  orc_mesh_n_nodes(void *m)
  {
    return long(static_cast<Mesh *>(m)->n_nodes);
  }

  int
  orc_node_positions(void *mp, double *x)
  {
    return guard([&] {
      const Mesh &m = *static_cast<Mesh *>(mp);
      for (std::size_t i = 0; i < m.n_nodes; ++i)
        m.node_position(i, x + i * m.dim);
    });
  }

  int
  orc_st_apply(void *mp, int nt, const double *Alpha, const double *Beta, int transpose, int fp32, double *dst,
               const double *src)
  {
    return guard([&] {
      const Mesh &m = *static_cast<Mesh *>(mp);
      const DMat  A = to_mat(Alpha, nt, nt), B = to_mat(Beta, nt, nt);
      if (fp32)
        {
          const std::size_t  n = m.n_nodes * nt;
          std::vector<float> s(src, src + n), d(n);
          st_apply(m, A, B, transpose != 0, d.data(), s.data());
          std::copy(d.begin(), d.end(), dst);
        }
      else
        st_apply(m, A, B, transpose != 0, dst, src);
    });
  }

  int
  orc_st_apply_vec(void *mp, int nt, const double *a, const double *b, int add, double *dst, const double *src)
  {
    return guard([&] { st_apply_vec(*static_cast<Mesh *>(mp), to_mat(a, nt, 1), to_mat(b, nt, 1), add != 0, dst, src); });
  }

  int
  orc_element_matrices(void *mp, long cell, double *Ke, double *Me)
  {
    return guard([&] {
      const Mesh         &m = *static_cast<Mesh *>(mp);
      std::vector<double> K, M;
      element_matrices(m, std::size_t(cell), K, M);
      std::copy(K.begin(), K.end(), Ke);
      std::copy(M.begin(), M.end(), Me);
    });
  }

  // Cell-patch Vanka apply (setup + one vmult), in FP64 or FP32.
  int
  orc_vanka_apply(void *mp, int nt, const double *Alpha, const double *Beta, int fp32, double *dst, const double *src)
  {
    return guard([&] {
      const Mesh &m = *static_cast<Mesh *>(mp);
      CSR         K, M;
      assemble(m, K, M);
      const DMat        A = to_mat(Alpha, nt, nt), B = to_mat(Beta, nt, nt);
      const std::size_t n = m.n_nodes * nt;
      if (fp32)
        {
          Vanka<float> v;
          v.setup(m, K, M, A, B);
          std::vector<float> s(src, src + n), d(n);
          v.vmult(d.data(), s.data());
          std::copy(d.begin(), d.end(), dst);
        }
      else
        {
          Vanka<double> v;
          v.setup(m, K, M, A, B);
          v.vmult(dst, src);
        }
    });
  }

  // Restriction of the assembled K and M to the dofs of one cell (the
  // reference's Vanka patch matrices), nd x nd each.
  int
  orc_patch_matrices(void *mp, long cell, double *Kp, double *Mp)
  {
    return guard([&] {
      const Mesh &m = *static_cast<Mesh *>(mp);
      CSR         K, M;
      assemble(m, K, M);
      std::vector<std::size_t> idx;
      m.cell_nodes(std::size_t(cell), idx);
      for (int a = 0; a < m.nd; ++a)
        for (int b = 0; b < m.nd; ++b)
          {
            Kp[a * m.nd + b] = K(idx[a], idx[b]);
            Mp[a * m.nd + b] = M(idx[a], idx[b]);
          }
    });
  }

  int
  orc_h_transfer(void *fine, void *coarse, int nt, int restrict_, double *dst, const double *src)
  {
    return guard([&] {
      const Mesh &f = *static_cast<Mesh *>(fine), &c = *static_cast<Mesh *>(coarse);
      if (restrict_)
        h_restrict_add(f, c, nt, dst, src);
      else
        h_prolongate_add(f, c, nt, dst, src);
    });
  }

  // Time weights for one slab: heat (problem 1) fills Alpha, Beta (nt x nt)
  // and the rhs columns rK, rM; wave (problem 2) also rV.
  int
  orc_time_weights(int type, int r, double tau, int n_steps, int problem, double *Alpha, double *Beta, double *rK,
                   double *rM, double *rV)
  {
    return guard([&] {
      const TimeType t  = TimeType(type);
      auto           wn = get_fe_time_weights(t, r, tau, n_steps);
      if (problem == 1)
        {
          from_mat(wn[0], Alpha);
          from_mat(wn[1], Beta);
          const DMat zero(wn[2].m, 1);
          from_mat(t == TimeType::CGP ? wn[2] : zero, rK);
          from_mat(t == TimeType::CGP ? wn[3] : wn[2], rM);
        }
      else
        {
          auto w1 = get_fe_time_weights(t, r, tau, 1);
          auto ww = get_fe_time_weights_wave(t, w1[0], w1[1], w1[2], w1[3], n_steps);
          from_mat(ww[0], Alpha);
          from_mat(ww[1], Beta);
          from_mat(ww[2], rK);
          from_mat(ww[3], rM);
          from_mat(ww[4], rV);
        }
    });
  }

  // Time transfer matrix between levels: kind 0 = k (projection r-1 -> r),
  // kind 1 = tau (prolongation); rows = fine time dofs.
  int
  orc_time_prolongation(int type, int kind, int r, int n_steps, double *P)
  {
    return guard([&] {
      const TimeType t = TimeType(type);
      from_mat(kind == 0 ? get_time_projection_matrix(t, r - 1, r, n_steps) : get_time_prolongation_matrix(t, r, n_steps),
               P);
    });
  }

  int orc_run_all(const OrcConfig *c, OrcResult *res, int *iterations, double *u_last, double *v_last, double *u_all);

  int
  orc_run(const OrcConfig *c, OrcResult *res, int *iterations, double *u_last, double *v_last)
  {
    return orc_run_all(c, res, iterations, u_last, v_last, nullptr);
  }

  // orc_run, and with u_all non-null every slab's blocks (n_slabs x n_blocks x N)
  int
  orc_run_all(const OrcConfig *c, OrcResult *res, int *iterations, double *u_last, double *v_last, double *u_all)
  {
    return guard([&] {
      Config cfg;
      cfg.dim = c->dim;
      for (int d = 0; d < 3; ++d)
        {
          cfg.subdiv[d] = c->subdiv[d];
          cfg.lo[d]     = c->lo[d];
          cfg.hi[d]     = c->hi[d];
        }
      cfg.refine                = c->refine;
      cfg.p                     = c->p;
      cfg.r                     = c->r;
      cfg.type                  = TimeType(c->type);
      cfg.problem               = Problem(c->problem);
      cfg.n_steps               = c->n_steps;
      cfg.n_slabs               = c->n_slabs;
      cfg.tau                   = c->tau;
      cfg.smoothing_steps       = c->smoothing_steps;
      cfg.variable              = c->variable != 0;
      cfg.estimate_relaxation   = c->estimate_relaxation != 0;
      cfg.restrict_is_transpose = c->restrict_is_transpose != 0;
      cfg.fe_degree_min         = c->fe_degree_min;
      cfg.n_steps_min           = c->n_steps_min;
      cfg.mg_float              = c->mg_float != 0;
      cfg.extrapolate           = c->extrapolate != 0;
      cfg.max_iter              = c->max_iter;
      cfg.restart               = c->restart;
      cfg.rhs_mode              = c->rhs_mode;
      cfg.compute_errors        = c->compute_errors != 0;
      cfg.tol                   = c->tol;
      cfg.abs_tol               = c->abs_tol;
      cfg.frequency             = c->frequency;
      cfg.keep_all              = u_all != nullptr;
      const int nf[3]           = {c->subdiv[0] << c->refine, c->subdiv[1] << c->refine, c->subdiv[2] << c->refine};
      std::size_t nn = 1, nc = 1, nv = 1;
      for (int d = 0; d < c->dim; ++d)
        {
          nn *= std::size_t(nf[d]) * c->p + 1;
          nc *= nf[d];
          nv *= nf[d] + 1;
        }
      if (c->f_nodal)
        cfg.f_nodal.assign(c->f_nodal, c->f_nodal + nn);
      if (c->u0_nodal)
        cfg.u0_nodal.assign(c->u0_nodal, c->u0_nodal + nn);
      if (c->v0_nodal)
        cfg.v0_nodal.assign(c->v0_nodal, c->v0_nodal + nn);
      if (c->fine_vertices)
        cfg.fine_vertices.assign(c->fine_vertices, c->fine_vertices + nv * c->dim);
      if (c->fine_coeff)
        cfg.fine_coeff.assign(c->fine_coeff, c->fine_coeff + nc);
      Result r              = run(cfg);
      res->total_iterations = r.total_iterations;
      res->n_levels         = r.n_levels;
      res->n_blocks         = r.n_blocks;
      res->l8               = r.l8;
      res->l2               = r.l2;
      res->h1               = r.h1;
      res->n_dofs           = long(r.n_dofs);
      res->n_cells          = long(r.n_cells);
      if (iterations)
        std::copy(r.iterations.begin(), r.iterations.end(), iterations);
      if (u_last)
        std::copy(r.u_last.begin(), r.u_last.end(), u_last);
      if (v_last)
        std::copy(r.v_last.begin(), r.v_last.end(), v_last);
      if (u_all)
        std::copy(r.u_all.begin(), r.u_all.end(), u_all);
    });
  }
}
