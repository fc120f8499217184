// 1-D tables of FE_Q(p) with Gauss-Lobatto support points and QGauss(p+1)
// quadrature, the element deal.II's FE_Q<dim>(p) and the reference's
// QGauss<dim>(fe.tensor_degree()+1) define (tests/tp_01.cc:76-77).
#include <cmath>
#include <mutex>

#include "stmg_internal.h"

namespace stmg
{
  namespace
  {
    // Legendre P_n and P_n' at x in [-1,1].
    void
    legendre(int n, double x, double &p, double &dp)
    {
      double p0 = 1.0, p1 = x;
      if (n == 0)
        {
          p  = 1.0;
          dp = 0.0;
          return;
        }
      for (int k = 2; k <= n; ++k)
        {
          const double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
          p0              = p1;
          p1              = pk;
        }
      p  = p1;
      dp = n * (x * p1 - p0) / (x * x - 1.0);
    }

    // n-point Gauss-Legendre rule mapped to [0,1].
    void
    gauss_rule(int n, double *x, double *w)
    {
      for (int i = 0; i < n; ++i)
        {
          double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
          for (int it = 0; it < 100; ++it)
            {
              double p, dp;
              legendre(n, z, p, dp);
              const double dz = p / dp;
              z -= dz;
              if (std::abs(dz) < 1e-16)
                break;
            }
          double p, dp;
          legendre(n, z, p, dp);
          // ascending order on [0,1]
          x[n - 1 - i] = 0.5 * (z + 1.0);
          w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
        }
    }

    // n-point Gauss-Lobatto points on [0,1]: the end points and the roots
    // of P'_{n-1}, found by Newton from the Chebyshev-Lobatto points.
    void
    lobatto_points(int n, double *x)
    {
      const int m = n - 1;
      for (int i = 0; i < n; ++i)
        {
          double z = -std::cos(M_PI * i / m);
          if (i > 0 && i < m)
            for (int it = 0; it < 100; ++it)
              {
                double p, dp;
                legendre(m, z, p, dp);
                // (1-z^2) P'' = 2 z P' - m(m+1) P
                const double d2 = (2.0 * z * dp - m * (m + 1.0) * p) / (1.0 - z * z);
                const double dz = dp / d2;
                z -= dz;
                if (std::abs(dz) < 1e-16)
                  break;
              }
          x[i] = 0.5 * (z + 1.0);
        }
    }

    double
    lag(const double *pts, int n, int i, double x)
    {
      double v = 1.0;
      for (int j = 0; j < n; ++j)
        if (j != i)
          v *= (x - pts[j]) / (pts[i] - pts[j]);
      return v;
    }

    double
    lag_d(const double *pts, int n, int i, double x)
    {
      double s = 0.0;
      for (int k = 0; k < n; ++k)
        if (k != i)
          {
            double v = 1.0 / (pts[i] - pts[k]);
            for (int j = 0; j < n; ++j)
              if (j != i && j != k)
                v *= (x - pts[j]) / (pts[i] - pts[j]);
            s += v;
          }
      return s;
    }

    void
    invert_small(int n, double A[MAX_P + 1][MAX_P + 1], double Ai[MAX_P + 1][MAX_P + 1])
    {
      double M[MAX_P + 1][2 * (MAX_P + 1)];
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          {
            M[i][j]     = A[i][j];
            M[i][n + j] = i == j ? 1.0 : 0.0;
          }
      for (int c = 0; c < n; ++c)
        {
          int r = c;
          for (int i = c + 1; i < n; ++i)
            if (std::abs(M[i][c]) > std::abs(M[r][c]))
              r = i;
          for (int j = 0; j < 2 * n; ++j)
            std::swap(M[c][j], M[r][j]);
          const double d = 1.0 / M[c][c];
          for (int j = 0; j < 2 * n; ++j)
            M[c][j] *= d;
          for (int i = 0; i < n; ++i)
            if (i != c)
              {
                const double f = M[i][c];
                for (int j = 0; j < 2 * n; ++j)
                  M[i][j] -= f * M[c][j];
              }
        }
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          Ai[i][j] = M[i][n + j];
    }

    FETables
    compute_tables()
    {
      FETables t{};
      for (int p = 1; p <= MAX_P; ++p)
        {
          const int n = p + 1;
          lobatto_points(n, t.xs[p]);
          gauss_rule(n, t.gx[p], t.gw[p]);
          double S[MAX_P + 1][MAX_P + 1] = {}, Si[MAX_P + 1][MAX_P + 1] = {};
          for (int q = 0; q < n; ++q)
            for (int a = 0; a < n; ++a)
              {
                S[q][a]       = lag(t.xs[p], n, a, t.gx[p][q]);
                t.S[p][q][a]  = S[q][a];
                t.D[p][q][a]  = lag_d(t.xs[p], n, a, t.gx[p][q]);
              }
          invert_small(n, S, Si);
          for (int q = 0; q < n; ++q)
            for (int r = 0; r < n; ++r)
              {
                double s = 0;
                for (int a = 0; a < n; ++a)
                  s += t.D[p][q][a] * Si[a][r];
                t.Dq[p][q][r] = s;
              }
          for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
              {
                double m = 0, k = 0;
                for (int q = 0; q < n; ++q)
                  {
                    m += t.gw[p][q] * t.S[p][q][a] * t.S[p][q][b];
                    k += t.gw[p][q] * t.D[p][q][a] * t.D[p][q][b];
                  }
                t.M1[p][a][b] = m;
                t.K1[p][a][b] = k;
              }
        }
      return t;
    }
  } // namespace

  const FETables &
  host_tables()
  {
    static const FETables t = compute_tables();
    return t;
  }
} // namespace stmg
