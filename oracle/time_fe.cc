// Oracle (test infrastructure only): restatement of the reference's time FE
// algebra (tests/include/fe_time.h). Every function names the lines it follows.
#include "time_fe.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <stdexcept>

namespace oracle
{
  bool
  DMat::all_zero() const
  {
    for (double v : a)
      if (v != 0.0)
        return false;
    return true;
  }

  void
  DMat::scale(double s)
  {
    for (double &v : a)
      v *= s;
  }

  DMat
  mmult(const DMat &A, const DMat &B)
  {
    if (A.n != B.m)
      throw std::runtime_error("mmult: shape mismatch");
    DMat C(A.m, B.n);
    for (std::size_t i = 0; i < A.m; ++i)
      for (std::size_t k = 0; k < A.n; ++k)
        for (std::size_t j = 0; j < B.n; ++j)
          C(i, j) += A(i, k) * B(k, j);
    return C;
  }

  DMat
  transpose(const DMat &A)
  {
    DMat T(A.n, A.m);
    for (std::size_t i = 0; i < A.m; ++i)
      for (std::size_t j = 0; j < A.n; ++j)
        T(j, i) = A(i, j);
    return T;
  }

  DMat
  invert(const DMat &A)
  {
    const std::size_t n = A.m;
    DMat              M = A;
    std::vector<std::size_t> p(n);
    std::iota(p.begin(), p.end(), 0);
    // In-place Gauss-Jordan with row pivoting on the column maximum
    // (the algorithm of dealii::FullMatrix::gauss_jordan).
    for (std::size_t j = 0; j < n; ++j)
      {
        double      max = std::abs(M(j, j));
        std::size_t r   = j;
        for (std::size_t i = j + 1; i < n; ++i)
          if (std::abs(M(i, j)) > max)
            {
              max = std::abs(M(i, j));
              r   = i;
            }
        if (max == 0.0)
          throw std::runtime_error("invert: singular matrix");
        if (r > j)
          {
            for (std::size_t k = 0; k < n; ++k)
              std::swap(M(j, k), M(r, k));
            std::swap(p[j], p[r]);
          }
        const double hr = 1. / M(j, j);
        M(j, j)         = hr;
        for (std::size_t k = 0; k < n; ++k)
          {
            if (k == j)
              continue;
            for (std::size_t i = 0; i < n; ++i)
              {
                if (i == j)
                  continue;
                M(i, k) -= M(i, j) * M(j, k) * hr;
              }
          }
        for (std::size_t i = 0; i < n; ++i)
          {
            M(i, j) *= hr;
            M(j, i) *= -hr;
          }
        M(j, j) = hr;
      }
    std::vector<double> hv(n);
    for (std::size_t i = 0; i < n; ++i)
      {
        for (std::size_t k = 0; k < n; ++k)
          hv[p[k]] = M(i, k);
        for (std::size_t k = 0; k < n; ++k)
          M(i, k) = hv[k];
      }
    return M;
  }

  void
  fill(DMat &dst, const DMat &src, std::size_t di, std::size_t dj, std::size_t si, std::size_t sj)
  {
    const std::size_t rows = std::min(dst.m - di, src.m - si);
    const std::size_t cols = std::min(dst.n - dj, src.n - sj);
    for (std::size_t i = 0; i < rows; ++i)
      for (std::size_t j = 0; j < cols; ++j)
        dst(di + i, dj + j) = src(si + i, sj + j);
  }

  // ---------------------------------------------------------------- quadrature
  namespace
  {
    // Jacobi polynomial P_n^{(al,be)}(x) and its derivative by the three-term
    // recurrence.
    void
    jacobi(unsigned n, double al, double be, double x, double &p, double &dp)
    {
      double p0 = 1.0, p1 = 0.5 * (al - be + (al + be + 2.0) * x);
      if (n == 0)
        {
          p  = 1.0;
          dp = 0.0;
          return;
        }
      double pm = p0, pc = p1;
      for (unsigned k = 2; k <= n; ++k)
        {
          const double a1 = 2.0 * k * (k + al + be) * (2.0 * k + al + be - 2.0);
          const double a2 = (2.0 * k + al + be - 1.0) * (al * al - be * be);
          const double a3 = (2.0 * k + al + be - 2.0) * (2.0 * k + al + be - 1.0) * (2.0 * k + al + be);
          const double a4 = 2.0 * (k + al - 1.0) * (k + be - 1.0) * (2.0 * k + al + be);
          const double pn = ((a2 + a3 * x) * pc - a4 * pm) / a1;
          pm              = pc;
          pc              = pn;
        }
      p = pc;
      // d/dx P_n^{(a,b)} = (n+a+b+1)/2 P_{n-1}^{(a+1,b+1)}
      double q, dq;
      jacobi(n - 1, al + 1.0, be + 1.0, x, q, dq);
      dp = 0.5 * (n + al + be + 1.0) * q;
    }

    // Roots of P_n^{(al,be)} on (-1,1): Chebyshev-like starting guesses,
    // Newton with deflation by the roots already found.
    std::vector<double>
    jacobi_roots(unsigned n, double al, double be)
    {
      std::vector<double> r;
      for (unsigned k = 0; k < n; ++k)
        {
          double x = -std::cos((2.0 * k + 1.0) * M_PI / (2.0 * n));
          if (k > 0)
            x = 0.5 * (x + r.back());
          for (int it = 0; it < 200; ++it)
            {
              double p, dp;
              jacobi(n, al, be, x, p, dp);
              double s = 0.0;
              for (double y : r)
                s += 1.0 / (x - y);
              const double dx = p / (dp - s * p);
              x -= dx;
              if (std::abs(dx) < 1e-17)
                break;
            }
          r.push_back(x);
        }
      std::sort(r.begin(), r.end());
      return r;
    }
  } // namespace

  void
  gauss(unsigned n, std::vector<double> &x, std::vector<double> &w)
  {
    auto r = jacobi_roots(n, 0.0, 0.0);
    x.resize(n);
    w.resize(n);
    for (unsigned i = 0; i < n; ++i)
      {
        double p, dp;
        jacobi(n, 0.0, 0.0, r[i], p, dp);
        x[i] = 0.5 * (r[i] + 1.0);
        w[i] = 1.0 / ((1.0 - r[i] * r[i]) * dp * dp);
      }
  }

  void
  gauss_lobatto(unsigned n, std::vector<double> &x, std::vector<double> &w)
  {
    if (n < 2)
      throw std::runtime_error("gauss_lobatto: n >= 2 required");
    std::vector<double> r{-1.0};
    auto                in = jacobi_roots(n - 2, 1.0, 1.0);
    r.insert(r.end(), in.begin(), in.end());
    r.push_back(1.0);
    x.resize(n);
    w.resize(n);
    for (unsigned i = 0; i < n; ++i)
      {
        double p, dp;
        jacobi(n - 1, 0.0, 0.0, r[i], p, dp);
        x[i] = 0.5 * (r[i] + 1.0);
        w[i] = 1.0 / (n * (n - 1.0) * p * p);
      }
  }

  void
  gauss_radau_right(unsigned n, std::vector<double> &x)
  {
    // Right Radau on [-1,1]: {+1} and the roots of P_{n-1}^{(1,0)}.
    std::vector<double> r = jacobi_roots(n - 1, 1.0, 0.0);
    r.push_back(1.0);
    x.resize(n);
    for (unsigned i = 0; i < n; ++i)
      x[i] = 0.5 * (r[i] + 1.0);
  }

  double
  lagrange(const std::vector<double> &pts, unsigned i, double x)
  {
    double v = 1.0;
    for (unsigned j = 0; j < pts.size(); ++j)
      if (j != i)
        v *= (x - pts[j]) / (pts[i] - pts[j]);
    return v;
  }

  double
  lagrange_d(const std::vector<double> &pts, unsigned i, double x)
  {
    double s = 0.0;
    for (unsigned k = 0; k < pts.size(); ++k)
      {
        if (k == i)
          continue;
        double v = 1.0 / (pts[i] - pts[k]);
        for (unsigned j = 0; j < pts.size(); ++j)
          if (j != i && j != k)
            v *= (x - pts[j]) / (pts[i] - pts[j]);
        s += v;
      }
    return s;
  }

  std::vector<double>
  time_basis_points(TimeType type, unsigned r)
  {
    std::vector<double> x, w;
    if (type == TimeType::CGP)
      gauss_lobatto(r + 1, x, w);
    else
      gauss_radau_right(r + 1, x);
    return x;
  }

  // ------------------------------------------------------------ time weights
  std::array<DMat, 3>
  get_dg_weights(unsigned r)
  {
    const auto          pts = time_basis_points(TimeType::DG, r);
    std::vector<double> qx, qw;
    gauss(r + 2, qx, qw);
    DMat lhs(r + 1, r + 1), jump(r + 1, 1), der(r + 1, r + 1);
    for (unsigned i = 0; i < r + 1; ++i)
      {
        jump(i, 0) = lagrange(pts, i, 0.0);
        for (unsigned j = 0; j < r + 1; ++j)
          for (unsigned q = 0; q < qx.size(); ++q)
            lhs(i, j) += qw[q] * lagrange(pts, i, qx[q]) * lagrange(pts, j, qx[q]);
      }
    for (unsigned i = 0; i < r + 1; ++i)
      for (unsigned j = 0; j < r + 1; ++j)
        {
          der(i, j) += lagrange(pts, i, 0.0) * lagrange(pts, j, 0.0);
          for (unsigned q = 0; q < qx.size(); ++q)
            der(i, j) += qw[q] * lagrange(pts, i, qx[q]) * lagrange_d(pts, j, qx[q]);
        }
    return {{lhs, der, jump}};
  }

  std::array<DMat, 2>
  get_cg_weights(unsigned r)
  {
    const auto                trial = time_basis_points(TimeType::CGP, r);
    const std::vector<double> test(trial.begin() + 1, trial.end());
    std::vector<double>       qx, qw;
    gauss(r + 2, qx, qw);
    DMat mat(r, r + 1), der(r, r + 1);
    for (unsigned i = 0; i < r; ++i)
      for (unsigned j = 0; j < r + 1; ++j)
        for (unsigned q = 0; q < qx.size(); ++q)
          {
            mat(i, j) += qw[q] * lagrange(test, i, qx[q]) * lagrange(trial, j, qx[q]);
            der(i, j) += qw[q] * lagrange(test, i, qx[q]) * lagrange_d(trial, j, qx[q]);
          }
    return {{mat, der}};
  }

  std::array<DMat, 4>
  split_lhs_rhs(const std::array<DMat, 2> &tw)
  {
    const std::size_t m = tw[0].m, n = tw[0].n;
    std::array<DMat, 4> ret{{DMat(m, n - 1), DMat(m, n - 1), DMat(m, 1), DMat(m, 1)}};
    for (std::size_t i = 0; i < m; ++i)
      {
        for (std::size_t j = 1; j < n; ++j)
          {
            ret[0](i, j - 1) = tw[0](i, j);
            ret[1](i, j - 1) = tw[1](i, j);
          }
        ret[2](i, 0) = -tw[0](i, 0);
        ret[3](i, 0) = -tw[1](i, 0);
      }
    return ret;
  }

  std::array<DMat, 4>
  split_lhs_rhs(const std::array<DMat, 3> &tw)
  {
    return {{tw[0], tw[1], tw[2], DMat(tw[2].m, 1)}};
  }

  std::array<DMat, 4>
  get_fe_time_weights(TimeType type, unsigned r, double tau, unsigned n_steps)
  {
    std::array<DMat, 4> tmp;
    if (type == TimeType::CGP)
      {
        tmp = split_lhs_rhs(get_cg_weights(r));
        tmp[2].scale(tau);
      }
    else
      {
        tmp    = split_lhs_rhs(get_dg_weights(r));
        tmp[3] = tmp[2];
        tmp[2] = DMat(tmp[2].m, tmp[2].n);
      }
    tmp[0].scale(tau);
    const std::size_t   ni = tmp[0].m, nt = ni * n_steps;
    std::array<DMat, 4> ret{{DMat(nt, nt), DMat(nt, nt), DMat(nt, 1), DMat(nt, 1)}};
    for (unsigned it = 0; it < n_steps; ++it)
      for (std::size_t i = 0; i < ni; ++i)
        {
          if (it + 1 < n_steps && i == ni - 1)
            for (std::size_t j = 0; j < ni; ++j)
              {
                ret[0](j + (it + 1) * ni, i + it * ni) = -tmp[2](j, 0);
                ret[1](j + (it + 1) * ni, i + it * ni) = -tmp[3](j, 0);
              }
          for (std::size_t j = 0; j < ni; ++j)
            {
              ret[0](i + it * ni, j + it * ni) = tmp[0](i, j);
              ret[1](i + it * ni, j + it * ni) = tmp[1](i, j);
            }
        }
    for (std::size_t i = 0; i < ni; ++i)
      {
        ret[2](i, 0) = tmp[type == TimeType::CGP ? 2 : 3](i, 0);
        ret[3](i, 0) = tmp[type == TimeType::CGP ? 3 : 2](i, 0);
      }
    return ret;
  }

  std::array<DMat, 5>
  get_fe_time_weights_wave(TimeType type, const DMat &Alpha, const DMat &Beta, const DMat &Gamma,
                           const DMat &Zeta, unsigned n_steps)
  {
    const DMat Ai     = invert(Alpha);
    const DMat BxAixB = mmult(mmult(Beta, Ai), Beta);
    const DMat BxAixG = mmult(mmult(Beta, Ai), Gamma);
    const std::size_t last = Gamma.m - 1;
    const double gxai = Gamma(last, 0) / Alpha(last, last);
    DMat         GxAixG = Gamma;
    GxAixG.scale(gxai);
    DMat Beta_row(1, Beta.n);
    for (std::size_t j = 0; j < Beta.n; ++j)
      Beta_row(0, j) = Beta(Beta.m - 1, j);
    DMat GxAixB = mmult(Gamma, Beta_row);
    GxAixB.scale(1.0 / Alpha(last, last));

    const std::size_t   ni = Alpha.m, nt = ni * n_steps;
    std::array<DMat, 5> ret{{DMat(nt, nt), DMat(nt, nt), DMat(nt, 1), DMat(nt, 1), DMat(nt, 1)}};
    if (type == TimeType::CGP)
      {
        const DMat BxAixZ   = mmult(mmult(Beta, Ai), Zeta);
        DMat       ZmBxAixG = Zeta;
        for (std::size_t i = 0; i < ZmBxAixG.a.size(); ++i)
          ZmBxAixG.a[i] -= BxAixG.a[i];
        DMat ZmBxAixB = mmult(ZmBxAixG, Beta_row);
        ZmBxAixB.scale(1.0 / Alpha(last, last));
        const double zxai = Zeta(Zeta.m - 1, 0) / Alpha(Zeta.m - 1, Zeta.m - 1);
        for (unsigned it = 0; it < n_steps; ++it)
          for (unsigned jt = 0; jt <= it; ++jt)
            for (std::size_t i = 0; i < ni; ++i)
              {
                if (it == 0 && jt == 0)
                  {
                    ret[2](i, 0) = Gamma(i, 0);
                    ret[3](i, 0) = BxAixZ(i, 0);
                    ret[4](i, 0) = ZmBxAixG(i, 0);
                  }
                else if (jt == 0)
                  {
                    ret[3](i + it * ni, 0) = -zxai * std::pow(gxai, it - 1.0) * ZmBxAixG(i, 0);
                    ret[4](i + it * ni, 0) = std::pow(gxai, double(it)) * ZmBxAixG(i, 0);
                  }
                if (it == jt + 1)
                  {
                    ret[0](i + it * ni, ni - 1 + jt * ni) = -Gamma(i, 0);
                    ret[1](i + it * ni, ni - 1 + jt * ni) = -BxAixZ(i, 0);
                  }
                if (it == jt)
                  for (std::size_t j = 0; j < ni; ++j)
                    {
                      ret[0](i + it * ni, j + it * ni) = Alpha(i, j);
                      ret[1](i + it * ni, j + it * ni) = BxAixB(i, j);
                    }
                else
                  for (std::size_t j = 0; j < ni; ++j)
                    ret[1](i + it * ni, j + jt * ni) +=
                      -std::pow(gxai, double(it) - jt - 1.0) * ZmBxAixB(i, j) +
                      (it > 1 && it - 1 > jt && j == ni - 1 ?
                         std::pow(gxai, double(it) - jt - 2.0) * zxai * ZmBxAixG(i, 0) :
                         0.0);
              }
      }
    else
      {
        for (unsigned it = 0; it < n_steps; ++it)
          for (std::size_t i = 0; i < ni; ++i)
            {
              if (it == 0)
                {
                  ret[3](i, 0) = BxAixG(i, 0);
                  ret[4](i, 0) = Gamma(i, 0);
                }
              if (it == 1)
                ret[3](ni + i, 0) = -GxAixG(i, 0);
              if (it + 1 < n_steps)
                for (std::size_t j = 0; j < ni; ++j)
                  ret[1](j + (it + 1) * ni, i + it * ni) =
                    -GxAixB(j, i) - (i == ni - 1 ? BxAixG(j, 0) : 0.0);
              if (int(it) < int(n_steps) - 2 && i == ni - 1)
                for (std::size_t j = 0; j < ni; ++j)
                  ret[1](j + (it + 2) * ni, i + it * ni) = GxAixG(j, 0);
              for (std::size_t j = 0; j < ni; ++j)
                {
                  ret[0](i + it * ni, j + it * ni) = Alpha(i, j);
                  ret[1](i + it * ni, j + it * ni) = BxAixB(i, j);
                }
            }
      }
    return ret;
  }

  std::vector<std::array<DMat, 4>>
  get_fe_time_weights_levels(TimeType type, unsigned r, double tau, unsigned n_steps,
                             const std::vector<TimeMG> &seq)
  {
    std::vector<std::array<DMat, 4>> tw(seq.size() + 1);
    auto                             t = tw.rbegin();
    *t                                 = get_fe_time_weights(type, r, tau, n_steps);
    ++t;
    for (auto mgt = seq.rbegin(); mgt != seq.rend(); ++mgt, ++t)
      {
        if (*mgt == TimeMG::k)
          --r;
        else if (*mgt == TimeMG::tau)
          n_steps /= 2, tau *= 2;
        *t = get_fe_time_weights(type, r, tau, n_steps);
      }
    return tw;
  }

  std::vector<std::array<DMat, 5>>
  get_fe_time_weights_wave_levels(TimeType type, unsigned r, double tau, unsigned n_steps,
                                  const std::vector<TimeMG> &seq)
  {
    // Each level condenses that level's (possibly multi-step) heat weights as
    // if they were a single interval, as fe_time.h:394-409 does.
    auto                             tw = get_fe_time_weights_levels(type, r, tau, n_steps, seq);
    std::vector<std::array<DMat, 5>> ww(tw.size());
    for (std::size_t l = 0; l < tw.size(); ++l)
      ww[l] = get_fe_time_weights_wave(type, tw[l][0], tw[l][1], tw[l][2], tw[l][3], 1);
    return ww;
  }

  std::vector<TimeMG>
  get_time_mg_sequence(unsigned n_sp_lvl, unsigned k_max, unsigned k_min, unsigned n_steps,
                       unsigned n_steps_min, TimeMG lower, bool time_before_space)
  {
    const unsigned n_k = k_max - k_min;
    const unsigned n_t = unsigned(std::log2(double(n_steps / n_steps_min)));
    const TimeMG   upper = lower == TimeMG::k ? TimeMG::tau : TimeMG::k;
    const unsigned n_ll  = lower == TimeMG::k ? n_k : n_t;
    const unsigned n_ul  = lower == TimeMG::k ? n_t : n_k;
    std::vector<TimeMG> seq(n_k + n_t + n_sp_lvl - 1, TimeMG::none);
    const unsigned      s_l = time_before_space ? n_sp_lvl - 1 : 0;
    const unsigned      s_u = time_before_space ? n_sp_lvl - 1 + n_ll : n_ll;
    std::fill_n(seq.begin() + s_l, n_ll, lower);
    std::fill_n(seq.begin() + s_u, n_ul, upper);
    return seq;
  }

  std::vector<unsigned>
  get_space_time_levels(const std::vector<TimeMG> &seq, unsigned n_sp_lvl)
  {
    std::vector<unsigned> out(seq.size() + 1);
    unsigned              sp = n_sp_lvl - 1;
    out.back()               = sp;
    for (std::size_t ii = seq.size(); ii-- > 0;)
      {
        if (seq[ii] == TimeMG::none)
          --sp;
        out[ii] = sp;
      }
    return out;
  }

  // --------------------------------------------------------- time transfers
  namespace
  {
    // L2 projection from the Lagrange space on `src` to the one on `dst`
    // over [0,1] (FETools::get_projection_matrix for 1-D elements).
    DMat
    l2_projection(const std::vector<double> &src, const std::vector<double> &dst)
    {
      std::vector<double> qx, qw;
      gauss(unsigned(std::max(src.size(), dst.size())) + 1, qx, qw);
      DMat Mdd(dst.size(), dst.size()), Mds(dst.size(), src.size());
      for (std::size_t q = 0; q < qx.size(); ++q)
        for (std::size_t i = 0; i < dst.size(); ++i)
          {
            const double vi = lagrange(dst, unsigned(i), qx[q]);
            for (std::size_t j = 0; j < dst.size(); ++j)
              Mdd(i, j) += qw[q] * vi * lagrange(dst, unsigned(j), qx[q]);
            for (std::size_t j = 0; j < src.size(); ++j)
              Mds(i, j) += qw[q] * vi * lagrange(src, unsigned(j), qx[q]);
          }
      return mmult(invert(Mdd), Mds);
    }

    // Embedding of the parent basis into child c (interpolation at the
    // child's support points, mapped into the parent interval).
    DMat
    prolongation_child(const std::vector<double> &pts, unsigned c)
    {
      DMat P(pts.size(), pts.size());
      for (std::size_t i = 0; i < pts.size(); ++i)
        for (std::size_t j = 0; j < pts.size(); ++j)
          P(i, j) = lagrange(pts, unsigned(j), 0.5 * (c + pts[i]));
      return P;
    }

    // DG restriction of child c: L2 projection of the child's basis
    // (supported on child c only) onto the parent space.
    DMat
    restriction_child_dg(const std::vector<double> &pts, unsigned c)
    {
      std::vector<double> qx, qw;
      gauss(unsigned(pts.size()) + 1, qx, qw);
      const std::size_t n = pts.size();
      DMat              Mpp(n, n), Mpc(n, n);
      for (std::size_t q = 0; q < qx.size(); ++q)
        for (std::size_t i = 0; i < n; ++i)
          for (std::size_t j = 0; j < n; ++j)
            {
              Mpp(i, j) += qw[q] * lagrange(pts, unsigned(i), qx[q]) * lagrange(pts, unsigned(j), qx[q]);
              const double xp = 0.5 * (c + qx[q]); // parent coordinate of the child point
              Mpc(i, j) += 0.5 * qw[q] * lagrange(pts, unsigned(i), xp) * lagrange(pts, unsigned(j), qx[q]);
            }
      return mmult(invert(Mpp), Mpc);
    }

    // Continuous (FE_Q) restriction of child c: each parent node takes the
    // child's interpolant at that node, from the first child that contains it.
    DMat
    restriction_child_cg(const std::vector<double> &pts, unsigned c)
    {
      const std::size_t n = pts.size();
      DMat              R(n, n);
      for (std::size_t i = 0; i < n; ++i)
        {
          const double x     = pts[i];
          unsigned     first = (x <= 0.5 + 1e-12) ? 0u : 1u;
          if (first != c)
            continue;
          const double xc = 2.0 * x - c;
          for (std::size_t j = 0; j < n; ++j)
            {
              const double v = lagrange(pts, unsigned(j), xc);
              if (std::abs(v) > 1e-10)
                R(i, j) = v;
            }
        }
      return R;
    }
  } // namespace

  DMat
  get_time_projection_matrix(TimeType type, unsigned r_src, unsigned r_dst, unsigned n_steps)
  {
    const bool     dg     = type == TimeType::DG;
    const unsigned ni_dst = dg ? r_dst + 1 : r_dst;
    const unsigned ni_src = dg ? r_src + 1 : r_src;
    const unsigned nd     = dg ? n_steps * (r_dst + 1) : n_steps * r_dst + 1;
    const unsigned ns     = dg ? n_steps * (r_src + 1) : n_steps * r_src + 1;
    const DMat proj = l2_projection(time_basis_points(type, r_src), time_basis_points(type, r_dst));
    DMat       pn(nd, ns);
    for (unsigned it = 0; it < n_steps; ++it)
      fill(pn, proj, it * ni_dst, it * ni_src, 0, 0);
    if (!dg)
      {
        DMat out(nd - 1, ns - 1);
        fill(out, pn, 0, 0, 1, 1);
        return out;
      }
    return pn;
  }

  DMat
  get_time_prolongation_matrix(TimeType type, unsigned r, unsigned n_steps)
  {
    const auto pts = time_basis_points(type, r);
    const DMat L = prolongation_child(pts, 0), R = prolongation_child(pts, 1);
    DMat       P;
    if (type == TimeType::DG)
      {
        P = DMat(2 * (r + 1), r + 1);
        fill(P, L, 0, 0, 0, 0);
        fill(P, R, L.m, 0, 0, 0);
      }
    else
      {
        P = DMat(2 * r, r);
        fill(P, L, 0, 0, 1, 1);
        fill(P, R, r, 0, 1, 1);
      }
    const unsigned ni = type == TimeType::DG ? r + 1 : r;
    DMat           Pn(ni * n_steps, ni * n_steps / 2);
    for (unsigned it = 0; it < n_steps / 2; ++it)
      fill(Pn, P, it * 2 * ni, it * ni, 0, 0);
    return Pn;
  }

  DMat
  get_time_restriction_matrix(TimeType type, unsigned r, unsigned n_steps)
  {
    const auto pts = time_basis_points(type, r);
    DMat       Rm;
    if (type == TimeType::DG)
      {
        const DMat L = restriction_child_dg(pts, 0), R = restriction_child_dg(pts, 1);
        Rm           = DMat(r + 1, 2 * (r + 1));
        fill(Rm, L, 0, 0, 0, 0);
        fill(Rm, R, 0, L.n, 0, 0);
      }
    else
      {
        const DMat L = restriction_child_cg(pts, 0), R = restriction_child_cg(pts, 1);
        Rm           = DMat(r, 2 * r);
        fill(Rm, L, 0, 0, 1, 1);
        fill(Rm, R, 0, r, 1, 1);
      }
    const unsigned ni = type == TimeType::DG ? r + 1 : r;
    DMat           Rn(ni * n_steps / 2, ni * n_steps);
    for (unsigned it = 0; it < n_steps / 2; ++it)
      fill(Rn, Rm, it * ni, it * 2 * ni, 0, 0);
    return Rn;
  }

  DMat
  get_time_evaluation_matrix(const std::vector<double> &pts, unsigned samples)
  {
    const double step = 1.0 / (samples - 1);
    DMat         E(samples, pts.size());
    for (unsigned s = 0; s < samples; ++s)
      for (std::size_t j = 0; j < pts.size(); ++j)
        E(s, j) = lagrange(pts, unsigned(j), s * step);
    return E;
  }

  std::string
  print_formatted(const DMat &M)
  {
    std::string out;
    char        buf[64];
    for (std::size_t i = 0; i < M.m; ++i)
      {
        for (std::size_t j = 0; j < M.n; ++j)
          {
            if (std::abs(M(i, j)) < 0.01)
              out += "       ";
            else
              {
                std::snprintf(buf, sizeof(buf), "%7.2f", M(i, j));
                out += buf;
              }
          }
        out += "\n";
      }
    out += "\n";
    return out;
  }
} // namespace oracle
