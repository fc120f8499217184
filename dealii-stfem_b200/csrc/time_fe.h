// Host-side time finite element algebra of the slab solve: the time weights,
// wave condensation, time-multigrid schedule and time transfer matrices of
// tests/include/fe_time.h. Matrices are dense row-major std::vector<double>.
#pragma once

#include <array>
#include <vector>

namespace stmg
{
  namespace tfe
  {
    enum Type
    {
      CGP = 1,
      DG  = 2
    };
    enum MG
    {
      TAU  = 1,
      K    = 2,
      NONE = 3
    };

    struct Mat
    {
      int                 m = 0, n = 0;
      std::vector<double> a;
      Mat() = default;
      Mat(int m_, int n_)
        : m(m_)
        , n(n_)
        , a(std::size_t(m_) * n_, 0.0)
      {}
      double &operator()(int i, int j) { return a[std::size_t(i) * n + j]; }
      double  operator()(int i, int j) const { return a[std::size_t(i) * n + j]; }
    };

    // time basis support points on [0,1]: Radau-right (dG) or Lobatto (cGP)
    std::vector<double> basis_points(Type t, int r);
    void                gauss(int n, std::vector<double> &x, std::vector<double> &w);
    double              lagrange(const std::vector<double> &pts, int i, double x);

    // one slab of n_steps steps (fe_time.h:292-349): {Alpha, Beta, Gamma, Zeta}
    std::array<Mat, 4> slab_weights(Type t, int r, double tau, int n_steps);
    // wave condensation (fe_time.h:98-246): {lhs_uK, lhs_uM, rhs_uK, rhs_uM, rhs_vM}
    std::array<Mat, 5> wave_weights(Type t, const Mat &A, const Mat &B, const Mat &G, const Mat &Z, int n_steps);

    // level schedule coarsest first (fe_time.h:43-69) and spatial index per level
    std::vector<MG>  mg_sequence(int n_sp, int k_max, int k_min, int n_steps, int n_steps_min);
    std::vector<int> space_levels(const std::vector<MG> &seq, int n_sp);

    // per-level (Alpha, Beta) of the heat or condensed wave system,
    // coarsest first (fe_time.h:351-412)
    std::vector<std::array<Mat, 2>> level_weights(Type t, bool wave, int r, double tau, int n_steps,
                                                  const std::vector<MG> &seq);

    // time transfers, rows = fine dofs (fe_time.h:567-669)
    Mat projection(Type t, int r_src, int r_dst, int n_steps);
    Mat prolongation(Type t, int r, int n_steps);

    Mat inverse(const Mat &A);
    Mat mul(const Mat &A, const Mat &B);
  } // namespace tfe
} // namespace stmg
