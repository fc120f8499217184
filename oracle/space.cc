// Oracle (test infrastructure only): see space.h for what this restates.
#include "space.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <stdexcept>

namespace oracle
{
  // ------------------------------------------------------------------ mesh
  void
  Mesh::init(int dim_, const int *n_, int p_, const double *lo, const double *hi)
  {
    dim = dim_;
    p   = p_;
    n_nodes = 1;
    n_cells = 1;
    for (int d = 0; d < 3; ++d)
      {
        n[d]  = d < dim ? n_[d] : 1;
        nn[d] = d < dim ? n[d] * p + 1 : 1;
        if (d < dim)
          {
            n_nodes *= nn[d];
            n_cells *= n[d];
          }
      }
    nd = nq = 1;
    for (int d = 0; d < dim; ++d)
      nd *= (p + 1), nq *= (p + 1);
    std::vector<double> w;
    gauss_lobatto(p + 1, xs, w);
    gauss(p + 1, gx, gw);
    const int   nv[3] = {n[0] + 1, dim > 1 ? n[1] + 1 : 1, dim > 2 ? n[2] + 1 : 1};
    std::size_t tot   = std::size_t(nv[0]) * nv[1] * nv[2];
    vert.assign(tot * dim, 0.0);
    for (int k = 0; k < nv[2]; ++k)
      for (int j = 0; j < nv[1]; ++j)
        for (int i = 0; i < nv[0]; ++i)
          {
            const std::size_t v   = i + std::size_t(nv[0]) * (j + std::size_t(nv[1]) * k);
            const int         ijk[3] = {i, j, k};
            for (int d = 0; d < dim; ++d)
              vert[v * dim + d] = lo[d] + (hi[d] - lo[d]) * double(ijk[d]) / n[d];
          }
  }

  void
  Mesh::set_vertices(const double *v)
  {
    std::copy(v, v + vert.size(), vert.begin());
  }

  void
  Mesh::cell_nodes(std::size_t c, std::vector<std::size_t> &idx) const
  {
    const int cx = int(c % n[0]);
    const int cy = dim > 1 ? int((c / n[0]) % n[1]) : 0;
    const int cz = dim > 2 ? int(c / (std::size_t(n[0]) * n[1])) : 0;
    idx.resize(nd);
    const int p1 = p + 1;
    for (int a = 0; a < nd; ++a)
      {
        const int a0 = a % p1, a1 = dim > 1 ? (a / p1) % p1 : 0, a2 = dim > 2 ? a / (p1 * p1) : 0;
        idx[a] = std::size_t(cx * p + a0) +
                 std::size_t(nn[0]) * (std::size_t(cy * p + a1) + std::size_t(nn[1]) * std::size_t(cz * p + a2));
      }
  }

  bool
  Mesh::is_boundary(std::size_t node) const
  {
    std::size_t r = node;
    for (int d = 0; d < dim; ++d)
      {
        const std::size_t i = r % nn[d];
        r /= nn[d];
        if (i == 0 || i == std::size_t(nn[d] - 1))
          return true;
      }
    return false;
  }

  namespace
  {
    // vertex index of corner v (bit d = upper side in direction d) of cell c
    std::size_t
    cell_vertex(const Mesh &m, std::size_t c, int v)
    {
      const int cx = int(c % m.n[0]);
      const int cy = m.dim > 1 ? int((c / m.n[0]) % m.n[1]) : 0;
      const int cz = m.dim > 2 ? int(c / (std::size_t(m.n[0]) * m.n[1])) : 0;
      const int nv0 = m.n[0] + 1, nv1 = m.dim > 1 ? m.n[1] + 1 : 1;
      return std::size_t(cx + (v & 1)) +
             std::size_t(nv0) * (std::size_t(cy + ((v >> 1) & 1)) + std::size_t(nv1) * std::size_t(cz + ((v >> 2) & 1)));
    }
  } // namespace

  void
  Mesh::map_point(std::size_t c, const double *xi, double *x) const
  {
    for (int i = 0; i < dim; ++i)
      x[i] = 0;
    for (int v = 0; v < (1 << dim); ++v)
      {
        double w = 1.0;
        for (int d = 0; d < dim; ++d)
          w *= ((v >> d) & 1) ? xi[d] : 1.0 - xi[d];
        const std::size_t vi = cell_vertex(*this, c, v);
        for (int i = 0; i < dim; ++i)
          x[i] += w * vert[vi * dim + i];
      }
  }

  void
  Mesh::jacobian(std::size_t c, const double *xi, double J[3][3]) const
  {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        J[i][j] = 0.0;
    for (int v = 0; v < (1 << dim); ++v)
      {
        const std::size_t vi = cell_vertex(*this, c, v);
        for (int j = 0; j < dim; ++j)
          {
            double w = ((v >> j) & 1) ? 1.0 : -1.0;
            for (int d = 0; d < dim; ++d)
              if (d != j)
                w *= ((v >> d) & 1) ? xi[d] : 1.0 - xi[d];
            for (int i = 0; i < dim; ++i)
              J[i][j] += w * vert[vi * dim + i];
          }
      }
  }

  void
  Mesh::node_position(std::size_t node, double *x) const
  {
    std::size_t r = node;
    int         cell[3] = {0, 0, 0};
    double      xi[3]   = {0, 0, 0};
    for (int d = 0; d < dim; ++d)
      {
        const int i = int(r % nn[d]);
        r /= nn[d];
        cell[d] = std::min(i / p, n[d] - 1);
        xi[d]   = xs[i - cell[d] * p];
      }
    const std::size_t c = cell[0] + std::size_t(n[0]) * (cell[1] + std::size_t(n[1]) * cell[2]);
    map_point(c, xi, x);
  }

  double
  Mesh::coeff_at(std::size_t c, int q) const
  {
    if (coeff_mode == 1)
      return coeff[c];
    if (coeff_mode == 2)
      return coeff[c * nq + q];
    return 1.0;
  }

  namespace
  {
    double
    det_inv(const double J[3][3], int dim, double Ji[3][3])
    {
      if (dim == 2)
        {
          const double d = J[0][0] * J[1][1] - J[0][1] * J[1][0];
          Ji[0][0]       = J[1][1] / d;
          Ji[0][1]       = -J[0][1] / d;
          Ji[1][0]       = -J[1][0] / d;
          Ji[1][1]       = J[0][0] / d;
          return d;
        }
      const double d = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
      Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / d;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / d;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / d;
      Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / d;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / d;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / d;
      Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / d;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / d;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / d;
      return d;
    }

    struct Tables
    {
      int                 p1;
      std::vector<double> S, D; // S[q*p1+a] = phi_a(g_q), D likewise for phi'
    };

    Tables
    tables(const Mesh &m)
    {
      Tables t;
      t.p1 = m.p + 1;
      t.S.resize(t.p1 * t.p1);
      t.D.resize(t.p1 * t.p1);
      for (int q = 0; q < t.p1; ++q)
        for (int a = 0; a < t.p1; ++a)
          {
            t.S[q * t.p1 + a] = lagrange(m.xs, a, m.gx[q]);
            t.D[q * t.p1 + a] = lagrange_d(m.xs, a, m.gx[q]);
          }
      return t;
    }

    // Geometry at quadrature point q of cell c: JxW and the metric
    // G = kappa JxW J^{-1} J^{-T} (dim x dim, row-major 3x3).
    void
    qp_geometry(const Mesh &m, std::size_t c, int q, double &JxW, double G[3][3])
    {
      const int p1 = m.p + 1;
      int       qi[3] = {q % p1, m.dim > 1 ? (q / p1) % p1 : 0, m.dim > 2 ? q / (p1 * p1) : 0};
      double    xi[3] = {0, 0, 0}, w = 1.0;
      for (int d = 0; d < m.dim; ++d)
        {
          xi[d] = m.gx[qi[d]];
          w *= m.gw[qi[d]];
        }
      double J[3][3], Ji[3][3];
      m.jacobian(c, xi, J);
      const double det = det_inv(J, m.dim, Ji);
      JxW              = std::abs(det) * w;
      const double k   = m.coeff_at(c, q) * JxW;
      for (int a = 0; a < m.dim; ++a)
        for (int b = 0; b < m.dim; ++b)
          {
            double s = 0;
            for (int i = 0; i < m.dim; ++i)
              s += Ji[a][i] * Ji[b][i];
            G[a][b] = k * s;
          }
    }

    // Apply the (p+1)x(p+1) matrix A (or A^T) along direction d of a
    // tensor with p+1 entries per direction.
    template <typename T>
    void
    sweep(const std::vector<double> &A, int p1, int dim, int d, bool tr, const T *in, T *out)
    {
      int stride = 1;
      for (int k = 0; k < d; ++k)
        stride *= p1;
      int total = 1;
      for (int k = 0; k < dim; ++k)
        total *= p1;
      const int outer = total / (stride * p1);
      for (int o = 0; o < outer; ++o)
        for (int s = 0; s < stride; ++s)
          {
            const int base = o * stride * p1 + s;
            for (int i = 0; i < p1; ++i)
              {
                T acc = 0;
                for (int k = 0; k < p1; ++k)
                  acc += T(tr ? A[k * p1 + i] : A[i * p1 + k]) * in[base + k * stride];
                out[base + i * stride] = acc;
              }
          }
    }

    // values (comp = -1) or reference derivative in direction comp at the
    // quadrature points, and the transposed integration.
    template <typename T>
    void
    eval_component(const Tables &t, int dim, int comp, bool tr, const T *in, T *out, T *tmp)
    {
      const T *src = in;
      T       *buf[2] = {out, tmp};
      int      which  = (dim % 2 == 1) ? 0 : 1; // so that the last sweep lands in out
      for (int d = 0; d < dim; ++d)
        {
          const std::vector<double> &A = (d == comp) ? t.D : t.S;
          T                         *dst = buf[which];
          sweep(A, t.p1, dim, d, tr, src, dst);
          src   = dst;
          which = 1 - which;
        }
    }
  } // namespace

  void
  element_matrices(const Mesh &m, std::size_t c, std::vector<double> &Ke, std::vector<double> &Me)
  {
    const Tables t  = tables(m);
    const int    p1 = t.p1, nd = m.nd;
    Ke.assign(nd * nd, 0.0);
    Me.assign(nd * nd, 0.0);
    std::vector<double> phi(nd), dphi(nd * 3);
    for (int q = 0; q < m.nq; ++q)
      {
        double JxW, G[3][3];
        qp_geometry(m, c, q, JxW, G);
        const int qi[3] = {q % p1, m.dim > 1 ? (q / p1) % p1 : 0, m.dim > 2 ? q / (p1 * p1) : 0};
        for (int a = 0; a < nd; ++a)
          {
            const int ai[3] = {a % p1, m.dim > 1 ? (a / p1) % p1 : 0, m.dim > 2 ? a / (p1 * p1) : 0};
            double    v     = 1.0;
            for (int d = 0; d < m.dim; ++d)
              v *= t.S[qi[d] * p1 + ai[d]];
            phi[a] = v;
            for (int j = 0; j < m.dim; ++j)
              {
                double g = 1.0;
                for (int d = 0; d < m.dim; ++d)
                  g *= (d == j ? t.D : t.S)[qi[d] * p1 + ai[d]];
                dphi[a * 3 + j] = g;
              }
          }
        for (int a = 0; a < nd; ++a)
          for (int b = 0; b < nd; ++b)
            {
              Me[a * nd + b] += JxW * phi[a] * phi[b];
              double s = 0;
              for (int i = 0; i < m.dim; ++i)
                for (int j = 0; j < m.dim; ++j)
                  s += dphi[a * 3 + i] * G[i][j] * dphi[b * 3 + j];
              Ke[a * nd + b] += s;
            }
      }
  }

  template <typename Number>
  void
  mf_apply(const Mesh &m, int which, Number *dst, const Number *src)
  {
    const Tables t  = tables(m);
    const int    nd = m.nd, dim = m.dim;
    std::fill(dst, dst + m.n_nodes, Number(0));
    // 2^dim colours of cells so that no two cells of one colour share a node
    const int ncol = 1 << dim;
    for (int col = 0; col < ncol; ++col)
      {
#pragma omp parallel
        {
          std::vector<std::size_t> idx;
          std::vector<Number>      u(nd), o(nd), tmp(nd), val(nd), grad(3 * nd), acc(nd);
#pragma omp for schedule(static)
          for (std::size_t c = 0; c < m.n_cells; ++c)
            {
              const int ci[3] = {int(c % m.n[0]), dim > 1 ? int((c / m.n[0]) % m.n[1]) : 0,
                                 dim > 2 ? int(c / (std::size_t(m.n[0]) * m.n[1])) : 0};
              int       cc    = 0;
              for (int d = 0; d < dim; ++d)
                cc |= (ci[d] & 1) << d;
              if (cc != col)
                continue;
              m.cell_nodes(c, idx);
              for (int a = 0; a < nd; ++a)
                u[a] = m.is_boundary(idx[a]) ? Number(0) : src[idx[a]];
              std::fill(o.begin(), o.end(), Number(0));
              if (which == 0)
                {
                  eval_component(t, dim, -1, false, u.data(), val.data(), tmp.data());
                  for (int q = 0; q < m.nq; ++q)
                    {
                      double JxW, G[3][3];
                      qp_geometry(m, c, q, JxW, G);
                      val[q] *= Number(JxW);
                    }
                  eval_component(t, dim, -1, true, val.data(), o.data(), tmp.data());
                }
              else
                {
                  for (int j = 0; j < dim; ++j)
                    eval_component(t, dim, j, false, u.data(), grad.data() + j * nd, tmp.data());
                  for (int q = 0; q < m.nq; ++q)
                    {
                      double JxW, G[3][3];
                      qp_geometry(m, c, q, JxW, G);
                      Number g[3];
                      for (int i = 0; i < dim; ++i)
                        {
                          Number s = 0;
                          for (int j = 0; j < dim; ++j)
                            s += Number(G[i][j]) * grad[j * nd + q];
                          g[i] = s;
                        }
                      for (int i = 0; i < dim; ++i)
                        grad[i * nd + q] = g[i];
                    }
                  for (int j = 0; j < dim; ++j)
                    {
                      eval_component(t, dim, j, true, grad.data() + j * nd, acc.data(), tmp.data());
                      for (int a = 0; a < nd; ++a)
                        o[a] += acc[a];
                    }
                }
              for (int a = 0; a < nd; ++a)
                if (!m.is_boundary(idx[a]))
                  dst[idx[a]] += o[a];
            }
        }
      }
  }

  template <typename Number>
  void
  st_apply(const Mesh &m, const DMat &Alpha, const DMat &Beta, bool transpose, Number *dst,
           const Number *src)
  {
    const std::size_t   N  = m.n_nodes;
    const int           nt = int(Alpha.m);
    std::vector<Number> tmp(N);
    std::fill(dst, dst + N * nt, Number(0));
    for (int pass = 0; pass < 2; ++pass)
      {
        const DMat &T = pass == 0 ? Alpha : Beta;
        for (int i = 0; i < nt; ++i)
          {
            mf_apply(m, pass == 0 ? 1 : 0, tmp.data(), src + i * N);
            for (int j = 0; j < nt; ++j)
              {
                const double c = transpose ? T(i, j) : T(j, i);
                if (c != 0.0)
                  {
                    Number *d = dst + j * N;
                    for (std::size_t k = 0; k < N; ++k)
                      d[k] += Number(c) * tmp[k];
                  }
              }
          }
      }
  }

  template <typename Number>
  void
  st_apply_vec(const Mesh &m, const DMat &a, const DMat &b, bool add, Number *dst, const Number *src)
  {
    const std::size_t   N  = m.n_nodes;
    const int           nt = int(a.m);
    std::vector<Number> tmp(N);
    if (!add)
      std::fill(dst, dst + N * nt, Number(0));
    for (int pass = 0; pass < 2; ++pass)
      {
        const DMat &T = pass == 0 ? a : b;
        if (T.all_zero())
          continue;
        mf_apply(m, pass == 0 ? 1 : 0, tmp.data(), src);
        for (int j = 0; j < nt; ++j)
          if (T(j, 0) != 0.0)
            for (std::size_t k = 0; k < N; ++k)
              dst[j * N + k] += Number(T(j, 0)) * tmp[k];
      }
  }

  // --------------------------------------------------------------- assembly
  double
  CSR::operator()(std::size_t i, std::size_t j) const
  {
    auto b = col.begin() + rowptr[i], e = col.begin() + rowptr[i + 1];
    auto it = std::lower_bound(b, e, j);
    if (it != e && *it == j)
      return val[it - col.begin()];
    return 0.0;
  }

  void
  assemble(const Mesh &m, CSR &K, CSR &M)
  {
    const std::size_t                     N = m.n_nodes;
    std::vector<std::map<std::size_t, std::pair<double, double>>> rows(N);
    std::vector<std::size_t>              idx;
    std::vector<double>                   Ke, Me;
    for (std::size_t c = 0; c < m.n_cells; ++c)
      {
        m.cell_nodes(c, idx);
        element_matrices(m, c, Ke, Me);
        for (int a = 0; a < m.nd; ++a)
          {
            const bool ca = m.is_boundary(idx[a]);
            if (ca)
              {
                auto &e = rows[idx[a]][idx[a]];
                e.first += std::abs(Ke[a * m.nd + a]);
                e.second += std::abs(Me[a * m.nd + a]);
                continue;
              }
            for (int b = 0; b < m.nd; ++b)
              {
                if (m.is_boundary(idx[b]))
                  continue;
                auto &e = rows[idx[a]][idx[b]];
                e.first += Ke[a * m.nd + b];
                e.second += Me[a * m.nd + b];
              }
          }
      }
    for (CSR *A : {&K, &M})
      {
        A->n = N;
        A->rowptr.assign(N + 1, 0);
        A->col.clear();
        A->val.clear();
      }
    for (std::size_t i = 0; i < N; ++i)
      {
        for (auto &kv : rows[i])
          {
            K.col.push_back(kv.first);
            K.val.push_back(kv.second.first);
            M.col.push_back(kv.first);
            M.val.push_back(kv.second.second);
          }
        K.rowptr[i + 1] = K.col.size();
        M.rowptr[i + 1] = M.col.size();
      }
  }

  // ----------------------------------------------------------------- Vanka
  namespace
  {
    // LU with partial pivoting followed by inversion from the factors, in
    // working precision T (the LAPACK getrf/getri path that
    // FullMatrix::gauss_jordan takes for matrices larger than 15x15).
    template <typename T>
    void
    lu_invert(std::vector<T> &A, int n)
    {
      auto             at = [&](int i, int j) -> T & { return A[std::size_t(i) * n + j]; };
      std::vector<int> piv(n);
      for (int k = 0; k < n; ++k)
        {
          int r = k;
          for (int i = k + 1; i < n; ++i)
            if (std::abs(at(i, k)) > std::abs(at(r, k)))
              r = i;
          piv[k] = r;
          if (at(r, k) == T(0))
            throw std::runtime_error("lu_invert: singular");
          if (r != k)
            for (int j = 0; j < n; ++j)
              std::swap(at(k, j), at(r, j));
          const T d = T(1) / at(k, k);
          for (int i = k + 1; i < n; ++i)
            {
              at(i, k) *= d;
              const T l = at(i, k);
              for (int j = k + 1; j < n; ++j)
                at(i, j) -= l * at(k, j);
            }
        }
      // inv(U) in place (upper triangle)
      for (int j = 0; j < n; ++j)
        {
          at(j, j) = T(1) / at(j, j);
          const T ajj = -at(j, j);
          for (int i = 0; i < j; ++i)
            {
              T s = 0;
              for (int k = i; k < j; ++k)
                s += at(i, k) * at(k, j);
              at(i, j) = s * ajj;
            }
        }
      // solve inv(A) L = inv(U) for inv(A), columns right to left
      std::vector<T> work(n);
      for (int j = n - 2; j >= 0; --j)
        {
          for (int i = j + 1; i < n; ++i)
            {
              work[i]  = at(i, j);
              at(i, j) = T(0);
            }
          for (int i = 0; i < n; ++i)
            {
              T s = 0;
              for (int k = j + 1; k < n; ++k)
                s += at(i, k) * work[k];
              at(i, j) -= s;
            }
        }
      // undo the row interchanges as column interchanges
      for (int j = n - 2; j >= 0; --j)
        if (piv[j] != j)
          for (int i = 0; i < n; ++i)
            std::swap(at(i, j), at(i, piv[j]));
    }
  } // namespace

  template <typename T>
  void
  gauss_jordan(std::vector<T> &A, int n)
  {
    if (n > 15)
      {
        lu_invert(A, n);
        return;
      }
    std::vector<int> p(n);
    for (int i = 0; i < n; ++i)
      p[i] = i;
    auto at = [&](int i, int j) -> T & { return A[std::size_t(i) * n + j]; };
    for (int j = 0; j < n; ++j)
      {
        T   max = std::abs(at(j, j));
        int r   = j;
        for (int i = j + 1; i < n; ++i)
          if (std::abs(at(i, j)) > max)
            {
              max = std::abs(at(i, j));
              r   = i;
            }
        if (max == T(0))
          throw std::runtime_error("gauss_jordan: singular");
        if (r > j)
          {
            for (int k = 0; k < n; ++k)
              std::swap(at(j, k), at(r, k));
            std::swap(p[j], p[r]);
          }
        const T hr = T(1) / at(j, j);
        at(j, j)   = hr;
        for (int k = 0; k < n; ++k)
          {
            if (k == j)
              continue;
            for (int i = 0; i < n; ++i)
              {
                if (i == j)
                  continue;
                at(i, k) -= at(i, j) * at(j, k) * hr;
              }
          }
        for (int i = 0; i < n; ++i)
          {
            at(i, j) *= hr;
            at(j, i) *= -hr;
          }
        at(j, j) = hr;
      }
    std::vector<T> hv(n);
    for (int i = 0; i < n; ++i)
      {
        for (int k = 0; k < n; ++k)
          hv[p[k]] = at(i, k);
        for (int k = 0; k < n; ++k)
          at(i, k) = hv[k];
      }
  }

  template <typename Number>
  void
  Vanka<Number>::setup(const Mesh &m, const CSR &K, const CSR &M, const DMat &Alpha, const DMat &Beta)
  {
    mesh = &m;
    nt   = int(Alpha.m);
    idx.resize(m.n_cells);
    valence.assign(m.n_nodes, Number(0));
    for (std::size_t c = 0; c < m.n_cells; ++c)
      {
        m.cell_nodes(c, idx[c]);
        for (auto i : idx[c])
          valence[i] += Number(1);
      }
    const int nd = m.nd, L = nd * nt;
    blocks.resize(m.n_cells);
#pragma omp parallel for schedule(dynamic, 16)
    for (std::size_t c = 0; c < m.n_cells; ++c)
      {
        std::vector<Number> B(std::size_t(L) * L, Number(0));
        std::vector<Number> Kc(nd * nd), Mc(nd * nd);
        for (int k = 0; k < nd; ++k)
          for (int l = 0; l < nd; ++l)
            {
              Kc[k * nd + l] = Number(K(idx[c][k], idx[c][l]));
              Mc[k * nd + l] = Number(M(idx[c][k], idx[c][l]));
            }
        for (int i = 0; i < nt; ++i)
          for (int j = 0; j < nt; ++j)
            if (Beta(i, j) != 0.0 || Alpha(i, j) != 0.0)
              {
                const Number b = Number(Beta(i, j)), a = Number(Alpha(i, j));
                for (int k = 0; k < nd; ++k)
                  for (int l = 0; l < nd; ++l)
                    B[std::size_t(k + i * nd) * L + l + j * nd] = b * Mc[k * nd + l] + a * Kc[k * nd + l];
              }
        gauss_jordan(B, L);
        blocks[c] = std::move(B);
      }
  }

  template <typename Number>
  void
  Vanka<Number>::vmult(Number *dst, const Number *src) const
  {
    const std::size_t N = mesh->n_nodes;
    const int         nd = mesh->nd, L = nd * nt;
    std::fill(dst, dst + N * nt, Number(0));
    std::vector<Number> sl(L), dl(L);
    for (std::size_t c = 0; c < blocks.size(); ++c)
      {
        for (int b = 0, k = 0; b < nt; ++b)
          for (int j = 0; j < nd; ++j, ++k)
            sl[k] = src[b * N + idx[c][j]];
        for (int i = 0; i < L; ++i)
          {
            Number s = 0;
            for (int j = 0; j < L; ++j)
              s += blocks[c][std::size_t(i) * L + j] * sl[j];
            dl[i] = s;
          }
        for (int b = 0, k = 0; b < nt; ++b)
          for (int j = 0; j < nd; ++j, ++k)
            dst[b * N + idx[c][j]] += (damp / valence[idx[c][j]]) * dl[k];
      }
  }

  // ------------------------------------------------------------ h-transfer
  namespace
  {
    // 1-D interpolation stencil of fine node f from the coarse nodes.
    void
    stencil_1d(const Mesh &fine, const Mesh &coarse, int d, int f, std::vector<std::pair<int, double>> &st)
    {
      const int p  = fine.p;
      int       fc = std::min(f / p, fine.n[d] - 1);
      const int a  = f - fc * p;
      const int cc = fc / 2;
      const double xi = 0.5 * ((fc % 2) + fine.xs[a]);
      st.clear();
      for (int b = 0; b <= p; ++b)
        {
          const double v = lagrange(coarse.xs, b, xi);
          if (std::abs(v) > 1e-14)
            st.emplace_back(cc * p + b, v);
        }
    }

    template <typename F>
    void
    for_each_fine(const Mesh &fine, const Mesh &coarse, F &&f)
    {
      std::vector<std::pair<int, double>> s[3];
      const int                           dim = fine.dim;
      for (std::size_t node = 0; node < fine.n_nodes; ++node)
        {
          if (fine.is_boundary(node))
            continue;
          std::size_t r = node;
          for (int d = 0; d < dim; ++d)
            {
              stencil_1d(fine, coarse, d, int(r % fine.nn[d]), s[d]);
              r /= fine.nn[d];
            }
          if (dim == 2)
            s[2] = {{0, 1.0}};
          for (auto &z : s[2])
            for (auto &y : s[1])
              for (auto &x : s[0])
                {
                  const std::size_t cn =
                    x.first + std::size_t(coarse.nn[0]) * (y.first + std::size_t(coarse.nn[1]) * z.first);
                  if (coarse.is_boundary(cn))
                    continue;
                  f(node, cn, x.second * y.second * z.second);
                }
        }
    }
  } // namespace

  template <typename Number>
  void
  h_prolongate_add(const Mesh &fine, const Mesh &coarse, int nt, Number *dst, const Number *src)
  {
    for (int b = 0; b < nt; ++b)
      {
        Number       *d = dst + std::size_t(b) * fine.n_nodes;
        const Number *s = src + std::size_t(b) * coarse.n_nodes;
        std::vector<Number> acc(fine.n_nodes, Number(0));
        for_each_fine(fine, coarse, [&](std::size_t f, std::size_t c, double w) { acc[f] += Number(w) * s[c]; });
        for (std::size_t i = 0; i < fine.n_nodes; ++i)
          d[i] += acc[i];
      }
  }

  template <typename Number>
  void
  h_restrict_add(const Mesh &fine, const Mesh &coarse, int nt, Number *dst, const Number *src)
  {
    for (int b = 0; b < nt; ++b)
      {
        Number       *d = dst + std::size_t(b) * coarse.n_nodes;
        const Number *s = src + std::size_t(b) * fine.n_nodes;
        for_each_fine(fine, coarse, [&](std::size_t f, std::size_t c, double w) { d[c] += Number(w) * s[f]; });
      }
  }

  template <typename Number>
  void
  tensorproduct_add(std::size_t N, const DMat &A, Number *dst, const Number *src)
  {
    for (std::size_t i = 0; i < A.m; ++i)
      for (std::size_t j = 0; j < A.n; ++j)
        if (A(i, j) != 0.0)
          {
            const Number a = Number(A(i, j));
            for (std::size_t k = 0; k < N; ++k)
              dst[i * N + k] += a * src[j * N + k];
          }
  }

#define ORACLE_INST(T)                                                                               \
  template void mf_apply<T>(const Mesh &, int, T *, const T *);                                       \
  template void st_apply<T>(const Mesh &, const DMat &, const DMat &, bool, T *, const T *);          \
  template void st_apply_vec<T>(const Mesh &, const DMat &, const DMat &, bool, T *, const T *);      \
  template struct Vanka<T>;                                                                           \
  template void gauss_jordan<T>(std::vector<T> &, int);                                               \
  template void h_prolongate_add<T>(const Mesh &, const Mesh &, int, T *, const T *);                 \
  template void h_restrict_add<T>(const Mesh &, const Mesh &, int, T *, const T *);                   \
  template void tensorproduct_add<T>(std::size_t, const DMat &, T *, const T *);
  ORACLE_INST(double)
  ORACLE_INST(float)
#undef ORACLE_INST
} // namespace oracle
