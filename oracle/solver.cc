// Oracle (test infrastructure only): see solver.h for what this restates.
#include "solver.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <sstream>
#include <stdexcept>

namespace oracle
{
  namespace
  {
    const double PI = 3.14159265358979323846;

    template <typename T>
    double
    dot(const std::vector<T> &a, const std::vector<T> &b)
    {
      double s = 0;
      for (std::size_t i = 0; i < a.size(); ++i)
        s += double(a[i]) * double(b[i]);
      return s;
    }
  } // namespace

  // ------------------------------------------------------------- hierarchy
  Hierarchy
  build_hierarchy(const Config &cfg, double tau)
  {
    Hierarchy      h;
    const unsigned n_sp = cfg.refine + 1;
    const int      lowest = cfg.type == TimeType::DG ? 0 : 1;
    int k_min = cfg.fe_degree_min < 0 ? cfg.r - 1 : cfg.fe_degree_min;
    k_min     = std::clamp(k_min, lowest, cfg.r);
    int n_min = cfg.n_steps_min < 0 ? cfg.n_steps / 2 : cfg.n_steps_min;
    n_min     = std::clamp(n_min, 1, cfg.n_steps);
    if (!cfg.space_time_mg)
      k_min = cfg.r, n_min = cfg.n_steps;
    h.seq = get_time_mg_sequence(n_sp, cfg.r, k_min, cfg.n_steps, std::max(n_min, 1), TimeMG::k,
                                 cfg.time_before_space);
    const auto sp = get_space_time_levels(h.seq, n_sp);

    // spatial meshes (coarsening sequence of the finest mesh)
    const int nf[3] = {cfg.subdiv[0] << cfg.refine, cfg.subdiv[1] << cfg.refine,
                       cfg.subdiv[2] << cfg.refine};
    h.meshes.resize(n_sp);
    for (unsigned s = 0; s < n_sp; ++s)
      {
        const int f     = 1 << (cfg.refine - s);
        const int ns[3] = {nf[0] / f, nf[1] / f, nf[2] / f};
        Mesh     &m     = h.meshes[s];
        m.init(cfg.dim, ns, cfg.p, cfg.lo, cfg.hi);
        if (!cfg.fine_vertices.empty())
          {
            const int nvf[3] = {nf[0] + 1, cfg.dim > 1 ? nf[1] + 1 : 1, cfg.dim > 2 ? nf[2] + 1 : 1};
            const int nv[3]  = {ns[0] + 1, cfg.dim > 1 ? ns[1] + 1 : 1, cfg.dim > 2 ? ns[2] + 1 : 1};
            for (int k = 0; k < nv[2]; ++k)
              for (int j = 0; j < nv[1]; ++j)
                for (int i = 0; i < nv[0]; ++i)
                  {
                    const std::size_t v  = i + std::size_t(nv[0]) * (j + std::size_t(nv[1]) * k);
                    const std::size_t vf = std::size_t(i * f) +
                                           std::size_t(nvf[0]) * (std::size_t(j * f) + std::size_t(nvf[1]) * std::size_t(k * f));
                    for (int d = 0; d < cfg.dim; ++d)
                      m.vert[v * cfg.dim + d] = cfg.fine_vertices[vf * cfg.dim + d];
                  }
          }
        if (!cfg.fine_coeff.empty())
          {
            if (f == 1)
              {
                m.coeff_mode = 1;
                m.coeff      = cfg.fine_coeff;
              }
            else
              {
                // coarse level: the fine per-cell field sampled at this level's
                // quadrature points; a point belongs to fine sub-cell
                // min(floor(xi*f), f-1) in each direction.
                m.coeff_mode = 2;
                m.coeff.assign(m.n_cells * m.nq, 0.0);
                const int p1 = cfg.p + 1;
                for (std::size_t c = 0; c < m.n_cells; ++c)
                  {
                    const int ci[3] = {int(c % ns[0]), cfg.dim > 1 ? int((c / ns[0]) % ns[1]) : 0,
                                       cfg.dim > 2 ? int(c / (std::size_t(ns[0]) * ns[1])) : 0};
                    for (int q = 0; q < m.nq; ++q)
                      {
                        const int qi[3] = {q % p1, cfg.dim > 1 ? (q / p1) % p1 : 0, cfg.dim > 2 ? q / (p1 * p1) : 0};
                        int       fi[3] = {0, 0, 0};
                        for (int d = 0; d < cfg.dim; ++d)
                          fi[d] = ci[d] * f + std::min(int(std::floor(m.gx[qi[d]] * f)), f - 1);
                        const std::size_t fc = fi[0] + std::size_t(nf[0]) * (fi[1] + std::size_t(nf[1]) * fi[2]);
                        m.coeff[c * m.nq + q] = cfg.fine_coeff[fc];
                      }
                  }
              }
          }
      }

    // level schedule, coarsest first
    const std::size_t L = h.seq.size() + 1;
    h.levels.resize(L);
    int r = cfg.r, n = cfg.n_steps;
    for (std::size_t l = L; l-- > 0;)
      {
        LevelInfo &li = h.levels[l];
        li.sp         = int(sp[l]);
        li.r          = r;
        li.n_steps    = n;
        li.nt         = cfg.type == TimeType::DG ? (r + 1) * n : r * n;
        li.to_finer   = l + 1 < L ? h.seq[l] : TimeMG::none;
        if (l > 0)
          {
            if (h.seq[l - 1] == TimeMG::k)
              --r;
            else if (h.seq[l - 1] == TimeMG::tau)
              n /= 2;
          }
      }
    if (cfg.problem == Problem::heat)
      {
        auto tw = get_fe_time_weights_levels(cfg.type, cfg.r, tau, cfg.n_steps, h.seq);
        for (std::size_t l = 0; l < L; ++l)
          h.levels[l].Alpha = tw[l][0], h.levels[l].Beta = tw[l][1];
      }
    else
      {
        auto tw = get_fe_time_weights_wave_levels(cfg.type, cfg.r, tau, cfg.n_steps, h.seq);
        for (std::size_t l = 0; l < L; ++l)
          h.levels[l].Alpha = tw[l][0], h.levels[l].Beta = tw[l][1];
      }
    return h;
  }

  // -------------------------------------------------------------------- GMG
  namespace
  {
    // Start vector of the power iteration: deal.II's generic
    // set_initial_guess (all ones, global entry 0 set to zero), which is what
    // PreconditionChebyshev uses for the reference's block vectors.
    template <typename Number>
    void
    initial_guess(std::vector<Number> &v)
    {
      std::fill(v.begin(), v.end(), Number(1));
      v[0] = Number(0);
    }

    template <typename Number>
    class GMG final : public GMGBase
    {
    public:
      GMG(const Config &cfg, const Hierarchy &h)
        : cfg(cfg)
        , h(h)
      {
        const std::size_t L = h.levels.size();
        Ks.resize(h.meshes.size());
        Ms.resize(h.meshes.size());
        for (std::size_t s = 0; s < h.meshes.size(); ++s)
          assemble(h.meshes[s], Ks[s], Ms[s]);
        vanka.resize(L);
        for (std::size_t l = 0; l < L; ++l)
          {
            const auto &li = h.levels[l];
            vanka[l].setup(h.meshes[li.sp], Ks[li.sp], Ms[li.sp], li.Alpha, li.Beta);
          }
        // transfers: P[l] maps level l-1 to level l
        P.resize(L);
        R.resize(L);
        for (std::size_t l = 1; l < L; ++l)
          {
            const TimeMG t  = h.seq[l - 1];
            const auto  &li = h.levels[l];
            if (t == TimeMG::k)
              {
                P[l] = get_time_projection_matrix(cfg.type, li.r - 1, li.r, li.n_steps);
                R[l] = cfg.restrict_is_transpose ? transpose(P[l]) :
                                                   get_time_projection_matrix(cfg.type, li.r, li.r - 1, li.n_steps);
              }
            else if (t == TimeMG::tau)
              {
                P[l] = get_time_prolongation_matrix(cfg.type, li.r, li.n_steps);
                R[l] = cfg.restrict_is_transpose ? transpose(P[l]) :
                                                   get_time_restriction_matrix(cfg.type, li.r, li.n_steps);
              }
          }
        sol.resize(L);
        def.resize(L);
        t.resize(L);
        for (std::size_t l = 0; l < L; ++l)
          {
            const std::size_t n = size(l);
            sol[l].assign(n, 0);
            def[l].assign(n, 0);
            t[l].assign(n, 0);
          }
        omega.assign(L, 1.0);
        if (cfg.estimate_relaxation)
          for (std::size_t l = 1; l < L; ++l)
            omega[l] = estimate_relaxation(l);
      }

      void
      vmult(double *dst, const double *src) override
      {
        const std::size_t L = h.levels.size();
        for (std::size_t l = 0; l < L; ++l)
          std::fill(sol[l].begin(), sol[l].end(), Number(0));
        for (std::size_t i = 0; i < size(L - 1); ++i)
          def[L - 1][i] = Number(src[i]);
        vstep(L - 1);
        for (std::size_t i = 0; i < size(L - 1); ++i)
          dst[i] = double(sol[L - 1][i]);
      }

      std::vector<double>
      omegas() const override
      {
        return omega;
      }

    private:
      std::size_t
      size(std::size_t l) const
      {
        return h.meshes[h.levels[l].sp].n_nodes * h.levels[l].nt;
      }

      void
      A(std::size_t l, Number *dst, const Number *src) const
      {
        const auto &li = h.levels[l];
        st_apply(h.meshes[li.sp], li.Alpha, li.Beta, false, dst, src);
      }

      // PreconditionRelaxation<SystemMatrix, Vanka>::step (deal.II precondition.h)
      void
      relax_step(std::size_t l, std::vector<Number> &x, const std::vector<Number> &b)
      {
        std::vector<Number> r(x.size()), z(x.size());
        A(l, r.data(), x.data());
        for (std::size_t i = 0; i < r.size(); ++i)
          r[i] = b[i] - r[i];
        vanka[l].vmult(z.data(), r.data());
        const Number w = Number(omega[l]);
        for (std::size_t i = 0; i < x.size(); ++i)
          x[i] += w * z[i];
      }

      // MGSmootherPrecondition(steps = 1, variable) (gmg.h:726-730): 2^(L-1-l)
      // smoother steps on level l, each PreconditionRelaxation step running
      // n_iterations = smoothing_steps relaxations (gmg.h:721)
      unsigned
      steps(std::size_t l) const
      {
        unsigned s = 1;
        if (cfg.variable)
          s <<= h.levels.size() - 1 - l;
        return s;
      }

      // MGSmootherPrecondition::apply: first relaxation through vmult
      void
      smooth_apply(std::size_t l, std::vector<Number> &x, const std::vector<Number> &b)
      {
        unsigned s = steps(l);
        // PreconditionRelaxation::vmult: i = 0 -> x = w P b, then further iterations
        vanka[l].vmult(x.data(), b.data());
        const Number w = Number(omega[l]);
        for (auto &v : x)
          v *= w;
        for (int it = 1; it < cfg.smoothing_steps; ++it)
          relax_step(l, x, b);
        for (unsigned i = 1; i < s; ++i)
          for (int it = 0; it < cfg.smoothing_steps; ++it)
            relax_step(l, x, b);
      }

      void
      smooth(std::size_t l, std::vector<Number> &x, const std::vector<Number> &b)
      {
        const unsigned s = steps(l);
        for (unsigned i = 0; i < s; ++i)
          for (int it = 0; it < cfg.smoothing_steps; ++it)
            relax_step(l, x, b);
      }

      void
      restrict_add(std::size_t l, std::vector<Number> &dst, const std::vector<Number> &src) const
      {
        const auto &fi = h.levels[l], &ci = h.levels[l - 1];
        if (h.seq[l - 1] == TimeMG::none)
          h_restrict_add(h.meshes[fi.sp], h.meshes[ci.sp], fi.nt, dst.data(), src.data());
        else
          tensorproduct_add(h.meshes[fi.sp].n_nodes, R[l], dst.data(), src.data());
      }

      void
      prolongate_add(std::size_t l, std::vector<Number> &dst, const std::vector<Number> &src) const
      {
        const auto &fi = h.levels[l], &ci = h.levels[l - 1];
        if (h.seq[l - 1] == TimeMG::none)
          h_prolongate_add(h.meshes[fi.sp], h.meshes[ci.sp], fi.nt, dst.data(), src.data());
        else
          tensorproduct_add(h.meshes[fi.sp].n_nodes, P[l], dst.data(), src.data());
      }

      // Multigrid::level_v_step (deal.II multigrid.templates.h)
      void
      vstep(std::size_t l)
      {
        if (l == 0)
          {
            smooth(0, sol[0], def[0]); // MGCoarseGridApplySmoother
            return;
          }
        smooth_apply(l, sol[l], def[l]);
        A(l, t[l].data(), sol[l].data());
        for (std::size_t i = 0; i < t[l].size(); ++i)
          t[l][i] = def[l][i] - t[l][i];
        std::fill(def[l - 1].begin(), def[l - 1].end(), Number(0));
        restrict_add(l, def[l - 1], t[l]);
        vstep(l - 1);
        prolongate_add(l, sol[l], sol[l - 1]);
        smooth(l, sol[l], def[l]);
      }

      // GMG::estimate_relaxation (gmg.h:792-844) with PreconditionChebyshev's
      // power iteration (20 steps) and its 1.2 safety factor.
      double
      estimate_relaxation(std::size_t l)
      {
        const std::size_t   n = size(l);
        std::vector<Number> x(n), y(n), z(n);
        initial_guess(x);
        double nrm = std::sqrt(dot(x, x));
        for (auto &v : x)
          v = Number(v / nrm);
        double ev = 0;
        for (int it = 0; it < 20; ++it)
          {
            A(l, y.data(), x.data());
            vanka[l].vmult(z.data(), y.data());
            ev  = dot(x, z);
            nrm = std::sqrt(dot(z, z));
            for (std::size_t i = 0; i < n; ++i)
              x[i] = Number(z[i] / nrm);
          }
        ev                  = std::abs(ev);
        const double max_ev = 1.2 * ev, min_ev = ev;
        const double alpha  = std::min(0.9 * max_ev, min_ev);
        return 2.0 / (alpha + max_ev);
      }

      const Config                     cfg;
      const Hierarchy                 &h;
      std::vector<CSR>                 Ks, Ms;
      std::vector<Vanka<Number>>       vanka;
      std::vector<DMat>                P, R;
      std::vector<std::vector<Number>> sol, def, t;
      std::vector<double>              omega;
    };
  } // namespace

  std::unique_ptr<GMGBase>
  make_gmg(const Config &cfg, const Hierarchy &h)
  {
    if (cfg.mg_float)
      return std::make_unique<GMG<float>>(cfg, h);
    return std::make_unique<GMG<double>>(cfg, h);
  }

  // ----------------------------------------------------------------- FGMRES
  int
  fgmres(std::size_t n, const std::function<void(double *, const double *)> &A,
         const std::function<void(double *, const double *)> &P, double *x, const double *b,
         double abs_tol, double reduce, int max_iter, int basis_size)
  {
    // Iteration k checks the residual of the k-dimensional flexible Krylov
    // solution; a restart cycle uses at most basis_size-1 directions (deal.II
    // 9.5 SolverFGMRES). ReductionControl: converged if res <= abs_tol or
    // res <= reduce * initial residual.
    std::vector<double>              aux(n);
    std::vector<std::vector<double>> V(basis_size, std::vector<double>(n)),
      Z(basis_size, std::vector<double>(n));
    int    it = 0;
    double reduced_tol = -1;
    bool   first = true;
    while (true)
      {
        A(aux.data(), x);
        for (std::size_t i = 0; i < n; ++i)
          aux[i] = b[i] - aux[i];
        const double beta = std::sqrt(dot(aux, aux));
        if (first)
          {
            reduced_tol = beta * reduce;
            first       = false;
          }
        if (beta <= reduced_tol || beta <= abs_tol)
          return it;
        if (it >= max_iter || std::isnan(beta))
          throw std::runtime_error("fgmres: no convergence");
        std::vector<std::vector<double>> H(basis_size + 1, std::vector<double>(basis_size, 0.0));
        std::vector<double>              cs(basis_size), sn(basis_size), g(basis_size + 1, 0.0);
        g[0]       = beta;
        for (std::size_t i = 0; i < n; ++i)
          V[0][i] = aux[i] / beta;
        int  used = 0;
        bool done = false;
        for (int j = 0; j + 1 < basis_size; ++j)
          {
            P(Z[j].data(), V[j].data());
            A(aux.data(), Z[j].data());
            for (int i = 0; i <= j; ++i)
              {
                H[i][j] = dot(aux, V[i]);
                for (std::size_t k = 0; k < n; ++k)
                  aux[k] -= H[i][j] * V[i][k];
              }
            H[j + 1][j] = std::sqrt(dot(aux, aux));
            if (H[j + 1][j] != 0)
              for (std::size_t k = 0; k < n; ++k)
                V[j + 1][k] = aux[k] / H[j + 1][j];
            for (int i = 0; i < j; ++i)
              {
                const double t = cs[i] * H[i][j] + sn[i] * H[i + 1][j];
                H[i + 1][j]    = -sn[i] * H[i][j] + cs[i] * H[i + 1][j];
                H[i][j]        = t;
              }
            const double rr = std::hypot(H[j][j], H[j + 1][j]);
            cs[j]           = H[j][j] / rr;
            sn[j]           = H[j + 1][j] / rr;
            H[j][j]         = rr;
            H[j + 1][j]     = 0;
            g[j + 1]        = -sn[j] * g[j];
            g[j]            = cs[j] * g[j];
            used            = j + 1;
            ++it;
            const double res = std::abs(g[j + 1]);
            if (res <= reduced_tol || res <= abs_tol)
              {
                done = true;
                break;
              }
            if (it >= max_iter || std::isnan(res))
              throw std::runtime_error("fgmres: no convergence");
          }
        std::vector<double> y(used);
        for (int i = used - 1; i >= 0; --i)
          {
            double s = g[i];
            for (int k = i + 1; k < used; ++k)
              s -= H[i][k] * y[k];
            y[i] = s / H[i][i];
          }
        for (int j = 0; j < used; ++j)
          for (std::size_t k = 0; k < n; ++k)
            x[k] += y[j] * Z[j][k];
        if (done)
          return it;
      }
  }

  // ------------------------------------------------------------ slab loops
  namespace
  {
    double
    exact_u(const double *x, int dim, double t, double f)
    {
      double v = std::sin(2 * PI * f * t);
      for (int i = 0; i < dim; ++i)
        v *= std::sin(2 * PI * f * x[i]);
      return v;
    }

    void
    exact_grad(const double *x, int dim, double t, double f, double *g)
    {
      const double tv = 2 * PI * f * std::sin(2 * PI * f * t);
      for (int i = 0; i < dim; ++i)
        {
          g[i] = tv;
          for (int j = 0; j < dim; ++j)
            g[i] *= (i == j ? std::cos(2 * PI * f * x[j]) : std::sin(2 * PI * f * x[j]));
        }
    }

    double
    exact_v(const double *x, int dim, double t, double f)
    {
      double v = 2 * PI * f * std::cos(2 * PI * f * t);
      for (int i = 0; i < dim; ++i)
        v *= std::sin(2 * PI * f * x[i]);
      return v;
    }

    double
    rhs_fun(const double *x, int dim, double t, double f, Problem pb)
    {
      double v;
      if (pb == Problem::heat) // exact_solution.h:53-75
        v = dim * 4 * PI * PI * f * f * std::sin(2 * PI * f * t) + 2 * PI * f * std::cos(2 * PI * f * t);
      else // exact_solution.h:164-184
        v = std::pow(2.0, dim) * std::pow(PI * f, 2) * std::sin(2 * PI * f * t);
      for (int i = 0; i < dim; ++i)
        v *= std::sin(2 * PI * f * x[i]);
      return v;
    }

    // VectorTools::create_right_hand_side with QGauss(p+1); constrained rows
    // dropped.
    void
    create_rhs(const Mesh &m, const std::function<double(const double *)> &f, double *rhs)
    {
      std::fill(rhs, rhs + m.n_nodes, 0.0);
      const int                p1 = m.p + 1;
      std::vector<std::size_t> idx;
      for (std::size_t c = 0; c < m.n_cells; ++c)
        {
          m.cell_nodes(c, idx);
          for (int q = 0; q < m.nq; ++q)
            {
              const int qi[3] = {q % p1, m.dim > 1 ? (q / p1) % p1 : 0, m.dim > 2 ? q / (p1 * p1) : 0};
              double    xi[3] = {0, 0, 0}, w = 1;
              for (int d = 0; d < m.dim; ++d)
                xi[d] = m.gx[qi[d]], w *= m.gw[qi[d]];
              double J[3][3], x[3];
              m.jacobian(c, xi, J);
              double det = m.dim == 2 ? J[0][0] * J[1][1] - J[0][1] * J[1][0] :
                                        J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                                          J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                                          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
              m.map_point(c, xi, x);
              const double fv = f(x) * std::abs(det) * w;
              for (int a = 0; a < m.nd; ++a)
                {
                  const int ai[3] = {a % p1, m.dim > 1 ? (a / p1) % p1 : 0, m.dim > 2 ? a / (p1 * p1) : 0};
                  double    phi   = 1;
                  for (int d = 0; d < m.dim; ++d)
                    phi *= lagrange(m.xs, ai[d], xi[d]);
                  if (!m.is_boundary(idx[a]))
                    rhs[idx[a]] += fv * phi;
                }
            }
        }
    }

    // integrate_difference for L2, L-inf and H1-seminorm at QGauss(nq1) per
    // direction; returns the three global values.
    void
    integrate_difference(const Mesh &m, const double *u, int nq1, double t, double f, double &l2,
                         double &l8, double &h1)
    {
      std::vector<double> gx, gw;
      gauss(nq1, gx, gw);
      l2 = 0;
      l8 = 0;
      h1 = 0;
      const int                p1 = m.p + 1;
      std::vector<std::size_t> idx;
      const int                nqt = m.dim == 2 ? nq1 * nq1 : nq1 * nq1 * nq1;
      for (std::size_t c = 0; c < m.n_cells; ++c)
        {
          m.cell_nodes(c, idx);
          double cl2 = 0, cl8 = 0, ch1 = 0;
          for (int q = 0; q < nqt; ++q)
            {
              const int qi[3] = {q % nq1, m.dim > 1 ? (q / nq1) % nq1 : 0, m.dim > 2 ? q / (nq1 * nq1) : 0};
              double    xi[3] = {0, 0, 0}, w = 1;
              for (int d = 0; d < m.dim; ++d)
                xi[d] = gx[qi[d]], w *= gw[qi[d]];
              double J[3][3], x[3];
              m.jacobian(c, xi, J);
              double Ji[3][3];
              double det;
              if (m.dim == 2)
                {
                  det      = J[0][0] * J[1][1] - J[0][1] * J[1][0];
                  Ji[0][0] = J[1][1] / det;
                  Ji[0][1] = -J[0][1] / det;
                  Ji[1][0] = -J[1][0] / det;
                  Ji[1][1] = J[0][0] / det;
                }
              else
                {
                  det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                        J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                        J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
                  Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
                  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
                  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
                  Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
                  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
                  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
                  Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
                  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
                  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
                }
              m.map_point(c, xi, x);
              double uh = 0, gr[3] = {0, 0, 0};
              for (int a = 0; a < m.nd; ++a)
                {
                  const int ai[3] = {a % p1, m.dim > 1 ? (a / p1) % p1 : 0, m.dim > 2 ? a / (p1 * p1) : 0};
                  double    phi   = 1, dphi[3] = {1, 1, 1};
                  for (int d = 0; d < m.dim; ++d)
                    {
                      const double s = lagrange(m.xs, ai[d], xi[d]);
                      phi *= s;
                      for (int j = 0; j < m.dim; ++j)
                        dphi[j] *= (j == d) ? lagrange_d(m.xs, ai[d], xi[d]) : s;
                    }
                  const double ua = u[idx[a]];
                  uh += ua * phi;
                  for (int j = 0; j < m.dim; ++j)
                    gr[j] += ua * dphi[j];
                }
              double gp[3] = {0, 0, 0}, ge[3];
              for (int i = 0; i < m.dim; ++i)
                for (int j = 0; j < m.dim; ++j)
                  gp[i] += Ji[j][i] * gr[j];
              exact_grad(x, m.dim, t, f, ge);
              const double e  = uh - exact_u(x, m.dim, t, f);
              const double JxW = std::abs(det) * w;
              cl2 += JxW * e * e;
              cl8 = std::max(cl8, std::abs(e));
              for (int i = 0; i < m.dim; ++i)
                ch1 += JxW * (gp[i] - ge[i]) * (gp[i] - ge[i]);
            }
          l2 += cl2;
          l8 = std::max(l8, cl8);
          h1 += ch1;
        }
      l2 = std::sqrt(l2);
      h1 = std::sqrt(h1);
    }
  } // namespace

  Result
  run(const Config &cfg)
  {
    const double tau = cfg.tau;
    Hierarchy    h   = build_hierarchy(cfg, tau);
    const Mesh  &m   = h.meshes.back();
    const std::size_t N = m.n_nodes;
    auto gmg = make_gmg(cfg, h);

    auto w1 = get_fe_time_weights(cfg.type, cfg.r, tau, 1);
    auto wn = get_fe_time_weights(cfg.type, cfg.r, tau, cfg.n_steps);
    const int nt_int = cfg.type == TimeType::DG ? cfg.r + 1 : cfg.r;
    const int nb     = nt_int * cfg.n_steps;
    DMat      zero(nb, 1);
    DMat      lhs_K, lhs_M, rhs_K, rhs_M, rhs_vM;
    if (cfg.problem == Problem::wave)
      {
        auto ww = get_fe_time_weights_wave(cfg.type, w1[0], w1[1], w1[2], w1[3], cfg.n_steps);
        lhs_K = ww[0], lhs_M = ww[1], rhs_K = ww[2], rhs_M = ww[3], rhs_vM = ww[4];
      }
    else
      {
        lhs_K = wn[0], lhs_M = wn[1];
        rhs_K = cfg.type == TimeType::CGP ? wn[2] : zero;
        rhs_M = cfg.type == TimeType::CGP ? wn[3] : wn[2];
      }

    Result res;
    res.n_dofs   = N;
    res.n_cells  = m.n_cells;
    res.n_blocks = nb;
    res.n_levels = int(h.levels.size());
    res.omega    = gmg->omegas();

    std::vector<double> x(N * nb, 0.0), v(N * nb, 0.0), prev_x(N), prev_v(N), rhs(N * nb), F(N);
    // initial values (tp_01.cc:528-531), boundary values zero
    for (std::size_t i = 0; i < N; ++i)
      {
        double xp[3];
        m.node_position(i, xp);
        const bool bd = m.is_boundary(i);
        x[(nb - 1) * N + i] = bd ? 0.0 : (cfg.u0_nodal.empty() ? exact_u(xp, cfg.dim, 0.0, cfg.frequency) : cfg.u0_nodal[i]);
        if (cfg.problem == Problem::wave)
          v[(nb - 1) * N + i] = bd ? 0.0 : (cfg.v0_nodal.empty() ? exact_v(xp, cfg.dim, 0.0, cfg.frequency) : cfg.v0_nodal[i]);
      }
    // time-constant nodal source: rhs = M f
    std::vector<double> Mf;
    if (cfg.rhs_mode == 1)
      {
        Mf.resize(N);
        std::vector<double> fz(cfg.f_nodal);
        for (std::size_t i = 0; i < N; ++i)
          if (m.is_boundary(i))
            fz[i] = 0.0; // the FE source is read through the constraints
        mf_apply(m, 0, Mf.data(), fz.data());
      }
    auto force = [&](double t, double *out) {
      if (cfg.rhs_mode == 0)
        create_rhs(m, [&](const double *xp) { return rhs_fun(xp, cfg.dim, t, cfg.frequency, cfg.problem); }, out);
      else if (cfg.rhs_mode == 1)
        std::copy(Mf.begin(), Mf.end(), out);
      else
        std::fill(out, out + N, 0.0);
    };
    std::vector<double> tq_pts = time_basis_points(cfg.type, cfg.r);
    std::vector<double> eq, ew;
    gauss(cfg.r + 1, eq, ew);

    // wave velocity recovery matrices (time_integrators.h:220-234)
    DMat AixB, AixG, AixZ;
    if (cfg.problem == Problem::wave)
      {
        DMat Ai = invert(w1[0]);
        AixB    = mmult(Ai, w1[1]);
        AixG    = mmult(Ai, w1[2]);
        AixZ    = mmult(Ai, w1[3]);
        if (cfg.type == TimeType::DG)
          AixG.scale(-1.0);
        else
          AixZ.scale(-1.0);
      }

    auto Aop = [&](double *dst, const double *src) { st_apply(m, lhs_K, lhs_M, false, dst, src); };
    auto Pop = [&](double *dst, const double *src) { gmg->vmult(dst, src); };

    double time = 0;
    for (int slab = 0; slab < cfg.n_slabs; ++slab)
      {
        std::copy(x.begin() + (nb - 1) * N, x.begin() + nb * N, prev_x.begin());
        if (cfg.problem == Problem::wave)
          std::copy(v.begin() + (nb - 1) * N, v.begin() + nb * N, prev_v.begin());
        // rhs (time_integrators.h:163-170 / 248-252)
        st_apply_vec(m, rhs_K, rhs_M, false, rhs.data(), prev_x.data());
        if (cfg.problem == Problem::wave)
          st_apply_vec(m, zero, rhs_vM, true, rhs.data(), prev_v.data());
        // assemble_force (time_integrators.h:60-87)
        for (int it = 0; it < cfg.n_steps; ++it)
          for (std::size_t j = 0; j < tq_pts.size(); ++j)
            {
              force(time + tau * it + tau * tq_pts[j], F.data());
              if (cfg.type == TimeType::DG)
                {
                  const double a = w1[0](j, j);
                  double      *d = rhs.data() + (j + it * w1[0].m) * N;
                  for (std::size_t k = 0; k < N; ++k)
                    d[k] += a * F[k];
                }
              else if (j == 0)
                {
                  for (std::size_t i = 0; i < w1[2].m; ++i)
                    {
                      double *d = rhs.data() + (i + it * w1[0].m) * N;
                      for (std::size_t k = 0; k < N; ++k)
                        d[k] += -w1[2](i, 0) * F[k];
                    }
                }
              else
                {
                  const double a = w1[0](j - 1, j - 1);
                  double      *d = rhs.data() + (j - 1 + it * w1[0].m) * N;
                  for (std::size_t k = 0; k < N; ++k)
                    d[k] += a * F[k];
                }
            }
        for (int b = 0; b < nb; ++b)
          for (std::size_t k = 0; k < N; ++k)
            x[b * N + k] = cfg.extrapolate ? prev_x[k] : 0.0;
        const int its = fgmres(N * nb, Aop, Pop, x.data(), rhs.data(), cfg.abs_tol, cfg.tol, cfg.max_iter,
                               cfg.restart);
        res.iterations.push_back(its);
        res.total_iterations += its;
        for (std::size_t k = 0; k < N; ++k)
          if (m.is_boundary(k))
            for (int b = 0; b < nb; ++b)
              x[b * N + k] = 0.0;
        if (cfg.problem == Problem::wave)
          {
            // velocity recovery (time_integrators.h:263-279)
            std::fill(v.begin(), v.end(), 0.0);
            const int ntd = int(AixB.m);
            for (int it = 0; it < cfg.n_steps; ++it)
              {
                const double *pu = it == 0 ? prev_x.data() : x.data() + (it * ntd - 1) * N;
                for (int i = 0; i < ntd; ++i)
                  for (int j = 0; j < ntd; ++j)
                    if (AixB(i, j) != 0.0)
                      for (std::size_t k = 0; k < N; ++k)
                        v[(it * ntd + i) * N + k] += AixB(i, j) * x[(it * ntd + j) * N + k];
                if (cfg.type == TimeType::DG)
                  {
                    for (int i = 0; i < ntd; ++i)
                      if (AixG(i, 0) != 0.0)
                        for (std::size_t k = 0; k < N; ++k)
                          v[(it * ntd + i) * N + k] += AixG(i, 0) * pu[k];
                  }
                else
                  {
                    const double *pv = it == 0 ? prev_v.data() : v.data() + (it * ntd - 1) * N;
                    std::vector<double> pvc(pv, pv + N);
                    for (int i = 0; i < ntd; ++i)
                      {
                        if (AixG(i, 0) != 0.0)
                          for (std::size_t k = 0; k < N; ++k)
                            v[(it * ntd + i) * N + k] += AixG(i, 0) * pvc[k];
                        if (AixZ(i, 0) != 0.0)
                          for (std::size_t k = 0; k < N; ++k)
                            v[(it * ntd + i) * N + k] += AixZ(i, 0) * pu[k];
                      }
                  }
              }
          }
        if (cfg.compute_errors && cfg.rhs_mode == 0)
          {
            // ErrorCalculator::evaluate_error (exact_solution.h:217-299)
            std::vector<double> num(N);
            for (int it = 0; it < cfg.n_steps; ++it)
              for (std::size_t q = 0; q < eq.size(); ++q)
                {
                  const double tt = time + tau * it + eq[q] * tau;
                  std::fill(num.begin(), num.end(), 0.0);
                  const double *pu = it == 0 ? prev_x.data() : x.data() + (nt_int * it - 1) * N;
                  for (std::size_t i = 0; i < tq_pts.size(); ++i)
                    {
                      const double b = lagrange(tq_pts, unsigned(i), eq[q]);
                      if (b == 0.0)
                        continue;
                      const double *src = cfg.type == TimeType::DG ? x.data() + (nt_int * it + i) * N :
                                          (i == 0 ? pu : x.data() + (nt_int * it + i - 1) * N);
                      for (std::size_t k = 0; k < N; ++k)
                        num[k] += b * src[k];
                    }
                  for (std::size_t k = 0; k < N; ++k)
                    if (m.is_boundary(k))
                      num[k] = 0.0;
                  double l2, l8, h1;
                  integrate_difference(m, num.data(), cfg.r + 1, tt, cfg.frequency, l2, l8, h1);
                  res.l2 += tau * ew[q] * l2 * l2;
                  res.h1 += tau * ew[q] * h1 * h1;
                  res.l8 = std::max(res.l8, l8);
                }
          }
        if (cfg.keep_all)
          res.u_all.insert(res.u_all.end(), x.begin(), x.end());
        time += cfg.n_steps * tau;
      }
    res.l2     = std::sqrt(res.l2);
    res.h1     = std::sqrt(res.h1);
    res.u_last = x;
    res.v_last = v;
    return res;
  }

  std::string
  convergence_report(const Config &base, int k0, int n_deg, int r0, int n_ref)
  {
    std::ostringstream os;
    for (int k = k0; k < k0 + n_deg; ++k)
      for (int r = r0; r < r0 + n_ref; ++r)
        {
          Config c  = base;
          c.r       = k;
          c.p       = k + 1;
          c.refine  = r;
          c.tau     = std::pow(2.0, -(r + 1));
          c.n_slabs = int(std::lround(1.0 / (c.tau * c.n_steps)));
          Result res = run(c);
          char   buf[256];
          std::snprintf(buf, sizeof(buf), "k=%d r=%d cells=%zu dofs=%zu levels=%d its=%d slabs=%d L8=%.5e L2=%.5e H1=%.5e\n",
                        k, r, res.n_cells, res.n_dofs, res.n_levels, res.total_iterations, c.n_slabs, res.l8,
                        res.l2, res.h1);
          os << buf;
        }
    return os.str();
  }
} // namespace oracle
