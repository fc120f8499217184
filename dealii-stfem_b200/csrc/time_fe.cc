// Time FE algebra of the slab solve (see time_fe.h); each function names
// the reference lines it follows.
#include "time_fe.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace stmg
{
  namespace tfe
  {
    namespace
    {
      double
      leg(int n, double x)
      {
        if (n == 0)
          return 1.0;
        double p0 = 1.0, p1 = x;
        for (int k = 2; k <= n; ++k)
          {
            const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
            p0              = p1;
            p1              = p2;
          }
        return p1;
      }

      // all roots of f in (a, b): bracket on a fine grid, then bisection
      template <typename F>
      std::vector<double>
      roots(F f, double a, double b, int grid = 4000)
      {
        std::vector<double> r;
        double              x0 = a, f0 = f(a);
        for (int i = 1; i <= grid; ++i)
          {
            const double x1 = a + (b - a) * i / grid, f1 = f(x1);
            if (f0 == 0.0)
              r.push_back(x0);
            else if (f0 * f1 < 0)
              {
                double lo = x0, hi = x1, flo = f0;
                for (int it = 0; it < 200 && hi - lo > 1e-17; ++it)
                  {
                    const double mid = 0.5 * (lo + hi), fm = f(mid);
                    if ((fm < 0) == (flo < 0))
                      lo = mid, flo = fm;
                    else
                      hi = mid;
                  }
                r.push_back(0.5 * (lo + hi));
              }
            x0 = x1;
            f0 = f1;
          }
        return r;
      }
    } // namespace

    void
    gauss(int n, std::vector<double> &x, std::vector<double> &w)
    {
      auto z = roots([n](double t) { return leg(n, t); }, -1.0, 1.0);
      x.clear();
      w.clear();
      for (double t : z)
        {
          const double dp = n * (t * leg(n, t) - leg(n - 1, t)) / (t * t - 1.0);
          x.push_back(0.5 * (t + 1.0));
          w.push_back(1.0 / ((1.0 - t * t) * dp * dp));
        }
    }

    std::vector<double>
    basis_points(Type t, int r)
    {
      const int n = r + 1;
      std::vector<double> z;
      if (t == CGP)
        {
          // Gauss-Lobatto: end points and the roots of P'_{n-1}
          z.push_back(-1.0);
          if (n > 2)
            {
              auto in = roots([n](double x) { return n == 1 ? 0.0 : ((n - 1) * (x * leg(n - 1, x) - leg(n - 2, x))); },
                              -1.0 + 1e-12, 1.0 - 1e-12);
              z.insert(z.end(), in.begin(), in.end());
            }
          z.push_back(1.0);
        }
      else
        {
          // Gauss-Radau with the right end point: roots of P_{n-1} - P_n
          if (n > 1)
            z = roots([n](double x) { return leg(n - 1, x) - leg(n, x); }, -1.0, 1.0 - 1e-12);
          z.push_back(1.0);
        }
      std::vector<double> out;
      for (double v : z)
        out.push_back(0.5 * (v + 1.0));
      return out;
    }

    double
    lagrange(const std::vector<double> &pts, int i, double x)
    {
      double v = 1.0;
      for (int j = 0; j < int(pts.size()); ++j)
        if (j != i)
          v *= (x - pts[j]) / (pts[i] - pts[j]);
      return v;
    }

    namespace
    {
      double
      lagrange_d(const std::vector<double> &pts, int i, double x)
      {
        double s = 0.0;
        for (int k = 0; k < int(pts.size()); ++k)
          if (k != i)
            {
              double v = 1.0 / (pts[i] - pts[k]);
              for (int j = 0; j < int(pts.size()); ++j)
                if (j != i && j != k)
                  v *= (x - pts[j]) / (pts[i] - pts[j]);
              s += v;
            }
        return s;
      }
    } // namespace

    Mat
    mul(const Mat &A, const Mat &B)
    {
      Mat C(A.m, B.n);
      for (int i = 0; i < A.m; ++i)
        for (int k = 0; k < A.n; ++k)
          for (int j = 0; j < B.n; ++j)
            C(i, j) += A(i, k) * B(k, j);
      return C;
    }

    Mat
    inverse(const Mat &A)
    {
      const int n = A.m;
      Mat       M(n, 2 * n);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          {
            M(i, j)     = A(i, j);
            M(i, n + j) = i == j;
          }
      for (int c = 0; c < n; ++c)
        {
          int r = c;
          for (int i = c + 1; i < n; ++i)
            if (std::abs(M(i, c)) > std::abs(M(r, c)))
              r = i;
          if (M(r, c) == 0.0)
            throw std::runtime_error("time algebra: singular matrix");
          for (int j = 0; j < 2 * n; ++j)
            std::swap(M(c, j), M(r, j));
          const double d = 1.0 / M(c, c);
          for (int j = 0; j < 2 * n; ++j)
            M(c, j) *= d;
          for (int i = 0; i < n; ++i)
            if (i != c && M(i, c) != 0.0)
              {
                const double f = M(i, c);
                for (int j = 0; j < 2 * n; ++j)
                  M(i, j) -= f * M(c, j);
              }
        }
      Mat I(n, n);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          I(i, j) = M(i, n + j);
      return I;
    }

    std::array<Mat, 4>
    slab_weights(Type t, int r, double tau, int n_steps)
    {
      // single interval: W[0] mass, W[1] derivative (+ jump for dG), and the
      // columns that move to the right-hand side (fe_time.h:292-349,431-555)
      std::vector<double> qx, qw;
      gauss(r + 2, qx, qw);
      const std::vector<double> trial = basis_points(t, r);
      const int                 ni    = t == DG ? r + 1 : r;
      Mat                       a(ni, ni), b(ni, ni), g(ni, 1), z(ni, 1);
      if (t == DG)
        {
          for (int i = 0; i <= r; ++i)
            {
              g(i, 0) = lagrange(trial, i, 0.0); // jump
              for (int j = 0; j <= r; ++j)
                {
                  double m = 0, d = lagrange(trial, i, 0.0) * lagrange(trial, j, 0.0);
                  for (std::size_t q = 0; q < qx.size(); ++q)
                    {
                      m += qw[q] * lagrange(trial, i, qx[q]) * lagrange(trial, j, qx[q]);
                      d += qw[q] * lagrange(trial, i, qx[q]) * lagrange_d(trial, j, qx[q]);
                    }
                  a(i, j) = tau * m;
                  b(i, j) = d;
                }
            }
        }
      else
        {
          const std::vector<double> test(trial.begin() + 1, trial.end());
          for (int i = 0; i < r; ++i)
            for (int j = 0; j <= r; ++j)
              {
                double m = 0, d = 0;
                for (std::size_t q = 0; q < qx.size(); ++q)
                  {
                    m += qw[q] * lagrange(test, i, qx[q]) * lagrange(trial, j, qx[q]);
                    d += qw[q] * lagrange(test, i, qx[q]) * lagrange_d(trial, j, qx[q]);
                  }
                if (j == 0)
                  {
                    g(i, 0) = -tau * m;
                    z(i, 0) = -d;
                  }
                else
                  {
                    a(i, j - 1) = tau * m;
                    b(i, j - 1) = d;
                  }
              }
        }
      // multi-step slab: block bidiagonal coupling through the last dof
      const int          nt = ni * n_steps;
      std::array<Mat, 4> out{{Mat(nt, nt), Mat(nt, nt), Mat(nt, 1), Mat(nt, 1)}};
      const Mat         &low_a = t == DG ? Mat(ni, 1) : g; // dG: no mass term moves to the rhs
      const Mat         &low_b = t == DG ? g : z;
      for (int it = 0; it < n_steps; ++it)
        for (int i = 0; i < ni; ++i)
          {
            for (int j = 0; j < ni; ++j)
              {
                out[0](it * ni + i, it * ni + j) = a(i, j);
                out[1](it * ni + i, it * ni + j) = b(i, j);
              }
            if (it + 1 < n_steps)
              {
                out[0]((it + 1) * ni + i, it * ni + ni - 1) = -low_a(i, 0);
                out[1]((it + 1) * ni + i, it * ni + ni - 1) = -low_b(i, 0);
              }
          }
      for (int i = 0; i < ni; ++i)
        {
          out[2](i, 0) = t == DG ? g(i, 0) : g(i, 0);
          out[3](i, 0) = t == DG ? 0.0 : z(i, 0);
        }
      return out;
    }

    std::array<Mat, 5>
    wave_weights(Type t, const Mat &A, const Mat &B, const Mat &G, const Mat &Z, int n_steps)
    {
      // Beta A^{-1} Beta condensation of the velocity (fe_time.h:98-246)
      const Mat    Ai   = inverse(A);
      const Mat    BAi  = mul(B, Ai);
      const Mat    BAB  = mul(BAi, B);
      const Mat    BAG  = mul(BAi, G);
      const int    ni   = A.m, last = G.m - 1;
      const double gxai = G(last, 0) / A(last, last);
      Mat          GAG  = G;
      for (auto &v : GAG.a)
        v *= gxai;
      Mat brow(1, B.n);
      for (int j = 0; j < B.n; ++j)
        brow(0, j) = B(B.m - 1, j);
      Mat GAB = mul(G, brow);
      for (auto &v : GAB.a)
        v /= A(last, last);
      const int          nt = ni * n_steps;
      std::array<Mat, 5> o{{Mat(nt, nt), Mat(nt, nt), Mat(nt, 1), Mat(nt, 1), Mat(nt, 1)}};
      if (t == CGP)
        {
          const Mat BAZ = mul(BAi, Z);
          Mat       ZmBAG = Z;
          for (std::size_t i = 0; i < ZmBAG.a.size(); ++i)
            ZmBAG.a[i] -= BAG.a[i];
          Mat ZmBAB = mul(ZmBAG, brow);
          for (auto &v : ZmBAB.a)
            v /= A(last, last);
          const double zxai = Z(Z.m - 1, 0) / A(Z.m - 1, Z.m - 1);
          for (int it = 0; it < n_steps; ++it)
            for (int jt = 0; jt <= it; ++jt)
              for (int i = 0; i < ni; ++i)
                {
                  if (it == 0 && jt == 0)
                    {
                      o[2](i, 0) = G(i, 0);
                      o[3](i, 0) = BAZ(i, 0);
                      o[4](i, 0) = ZmBAG(i, 0);
                    }
                  else if (jt == 0)
                    {
                      o[3](i + it * ni, 0) = -zxai * std::pow(gxai, it - 1.0) * ZmBAG(i, 0);
                      o[4](i + it * ni, 0) = std::pow(gxai, double(it)) * ZmBAG(i, 0);
                    }
                  if (it == jt + 1)
                    {
                      o[0](i + it * ni, ni - 1 + jt * ni) = -G(i, 0);
                      o[1](i + it * ni, ni - 1 + jt * ni) = -BAZ(i, 0);
                    }
                  for (int j = 0; j < ni; ++j)
                    {
                      if (it == jt)
                        {
                          o[0](i + it * ni, j + it * ni) = A(i, j);
                          o[1](i + it * ni, j + it * ni) = BAB(i, j);
                        }
                      else
                        o[1](i + it * ni, j + jt * ni) +=
                          -std::pow(gxai, double(it) - jt - 1.0) * ZmBAB(i, j) +
                          ((it > 1 && it - 1 > jt && j == ni - 1) ? std::pow(gxai, double(it) - jt - 2.0) * zxai * ZmBAG(i, 0) : 0.0);
                    }
                }
        }
      else
        {
          for (int it = 0; it < n_steps; ++it)
            for (int i = 0; i < ni; ++i)
              {
                if (it == 0)
                  {
                    o[3](i, 0) = BAG(i, 0);
                    o[4](i, 0) = G(i, 0);
                  }
                if (it == 1)
                  o[3](ni + i, 0) = -GAG(i, 0);
                if (it + 1 < n_steps)
                  for (int j = 0; j < ni; ++j)
                    o[1](j + (it + 1) * ni, i + it * ni) = -GAB(j, i) - (i == ni - 1 ? BAG(j, 0) : 0.0);
                if (it + 2 < n_steps && i == ni - 1)
                  for (int j = 0; j < ni; ++j)
                    o[1](j + (it + 2) * ni, i + it * ni) = GAG(j, 0);
                for (int j = 0; j < ni; ++j)
                  {
                    o[0](i + it * ni, j + it * ni) = A(i, j);
                    o[1](i + it * ni, j + it * ni) = BAB(i, j);
                  }
              }
        }
      return o;
    }

    std::vector<MG>
    mg_sequence(int n_sp, int k_max, int k_min, int n_steps, int n_steps_min)
    {
      // default ordering: all k- then tau-levels at the coarsest space level
      const int       n_k = k_max - k_min;
      const int       n_t = int(std::log2(double(n_steps / n_steps_min)));
      std::vector<MG> seq(n_k + n_t + n_sp - 1, NONE);
      for (int i = 0; i < n_k; ++i)
        seq[i] = K;
      for (int i = 0; i < n_t; ++i)
        seq[n_k + i] = TAU;
      return seq;
    }

    std::vector<int>
    space_levels(const std::vector<MG> &seq, int n_sp)
    {
      std::vector<int> sp(seq.size() + 1);
      int              s = n_sp - 1;
      sp.back()          = s;
      for (int i = int(seq.size()) - 1; i >= 0; --i)
        {
          if (seq[i] == NONE)
            --s;
          sp[i] = s;
        }
      return sp;
    }

    std::vector<std::array<Mat, 2>>
    level_weights(Type t, bool wave, int r, double tau, int n_steps, const std::vector<MG> &seq)
    {
      std::vector<std::array<Mat, 2>> out(seq.size() + 1);
      for (int l = int(seq.size()); l >= 0; --l)
        {
          if (l < int(seq.size()))
            {
              if (seq[l] == K)
                --r;
              else if (seq[l] == TAU)
                n_steps /= 2, tau *= 2;
            }
          auto w = slab_weights(t, r, tau, n_steps);
          if (wave)
            {
              // the levels condense their own (multi-step) heat weights as
              // one interval (fe_time.h:394-409)
              auto ww = wave_weights(t, w[0], w[1], w[2], w[3], 1);
              out[l]  = {ww[0], ww[1]};
            }
          else
            out[l] = {w[0], w[1]};
        }
      return out;
    }

    Mat
    projection(Type t, int r_src, int r_dst, int n_steps)
    {
      // L2 projection between the time bases on one interval, repeated per
      // step; cGP drops the shared first node (fe_time.h:567-623)
      const auto pd = basis_points(t, r_dst), ps = basis_points(t, r_src);
      std::vector<double> qx, qw;
      gauss(int(std::max(pd.size(), ps.size())) + 1, qx, qw);
      Mat Mdd(int(pd.size()), int(pd.size())), Mds(int(pd.size()), int(ps.size()));
      for (std::size_t q = 0; q < qx.size(); ++q)
        for (int i = 0; i < int(pd.size()); ++i)
          {
            const double vi = lagrange(pd, i, qx[q]);
            for (int j = 0; j < int(pd.size()); ++j)
              Mdd(i, j) += qw[q] * vi * lagrange(pd, j, qx[q]);
            for (int j = 0; j < int(ps.size()); ++j)
              Mds(i, j) += qw[q] * vi * lagrange(ps, j, qx[q]);
          }
      const Mat proj = mul(inverse(Mdd), Mds);
      const int di = t == DG ? r_dst + 1 : r_dst, si = t == DG ? r_src + 1 : r_src;
      const int nd = t == DG ? n_steps * (r_dst + 1) : n_steps * r_dst + 1;
      const int ns = t == DG ? n_steps * (r_src + 1) : n_steps * r_src + 1;
      Mat       full(nd, ns);
      for (int it = 0; it < n_steps; ++it)
        for (int i = 0; i < proj.m && it * di + i < nd; ++i)
          for (int j = 0; j < proj.n && it * si + j < ns; ++j)
            full(it * di + i, it * si + j) = proj(i, j);
      if (t == DG)
        return full;
      Mat out(nd - 1, ns - 1);
      for (int i = 0; i < nd - 1; ++i)
        for (int j = 0; j < ns - 1; ++j)
          out(i, j) = full(i + 1, j + 1);
      return out;
    }

    Mat
    prolongation(Type t, int r, int n_steps)
    {
      // interpolation of the coarse interval's basis into its two halves,
      // repeated per pair of steps (fe_time.h:625-669)
      const auto pts = basis_points(t, r);
      const int  n   = int(pts.size());
      const int  ni  = t == DG ? r + 1 : r;
      const int  off = t == DG ? 0 : 1; // cGP drops the first node
      Mat        P(2 * ni, ni);
      for (int c = 0; c < 2; ++c)
        for (int i = off; i < n; ++i)
          for (int j = off; j < n; ++j)
            P(c * ni + i - off, j - off) = lagrange(pts, j, 0.5 * (c + pts[i]));
      Mat Pn(ni * n_steps, ni * n_steps / 2);
      for (int it = 0; it < n_steps / 2; ++it)
        for (int i = 0; i < 2 * ni; ++i)
          for (int j = 0; j < ni; ++j)
            Pn(it * 2 * ni + i, it * ni + j) = P(i, j);
      return Pn;
    }
  } // namespace tfe
} // namespace stmg
