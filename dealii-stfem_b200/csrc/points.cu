// Point functionals of the slab solution (tests/tp_01.cc:451-619): the
// solution at given points for every time dof of the last slab
// (RemotePointEvaluation with FEPointEvaluation of FE_Q(p) under MappingQ1),
// mapped to sample times of each step by the time evaluation matrix
// (get_time_evaluation_matrix, tests/include/fe_time.h:250-267).
//
// Points are located on the host: the cell containing the point and its
// reference coordinates by Newton's method on the cell's Q1 map (the mesh's
// vertices), then the (p+1)^dim Lagrange weights at those coordinates. The
// device gathers sum_a w_a u[node_a] per point and time block.
#include <cmath>

#include "solver.h"

namespace stmg
{
  namespace
  {
    // vals[b * n_pts + k] = sum_a w[k * nd + a] u[b * N + node[k * nd + a]]
    __global__ void
    point_gather_kernel(int n_pts, int nd, int n_blocks, long long N, const long long *__restrict__ node,
                        const double *__restrict__ w, const double *__restrict__ u, double *__restrict__ vals)
    {
      const int t = blockIdx.x * blockDim.x + threadIdx.x;
      if (t >= n_pts * n_blocks)
        return;
      const int b = t / n_pts, k = t - b * n_pts;
      double    s = 0.0;
      for (int a = 0; a < nd; ++a)
        s += w[k * nd + a] * u[b * N + node[k * nd + a]];
      vals[t] = s;
    }

    // Q1 map of cell (cx, cy, cz) at reference point xi and its Jacobian
    void
    q1_map(const MeshView &m, const std::vector<double> &vert, const int (&ce)[3], const double (&xi)[3],
           double (&x)[3], double (&J)[3][3])
    {
      for (int d = 0; d < 3; ++d)
        {
          x[d] = 0;
          for (int e = 0; e < 3; ++e)
            J[d][e] = 0;
        }
      for (int vtx = 0; vtx < (1 << m.dim); ++vtx)
        {
          double wv = 1, dw[3] = {1, 1, 1};
          for (int e = 0; e < m.dim; ++e)
            {
              const int    bit = (vtx >> e) & 1;
              const double f   = bit ? xi[e] : 1.0 - xi[e];
              wv *= f;
              for (int k = 0; k < m.dim; ++k)
                dw[k] *= k == e ? (bit ? 1.0 : -1.0) : f;
            }
          const long long vi = (ce[0] + (vtx & 1)) +
                               (long long)(m.n[0] + 1) * ((ce[1] + ((vtx >> 1) & 1)) +
                                                          (m.dim == 3 ? (long long)(m.n[1] + 1) * (ce[2] + ((vtx >> 2) & 1)) : 0));
          for (int d = 0; d < m.dim; ++d)
            {
              const double v = vert[vi * m.dim + d];
              x[d] += wv * v;
              for (int k = 0; k < m.dim; ++k)
                J[d][k] += dw[k] * v;
            }
        }
    }

    // reference coordinates of point y in cell ce (Newton); false if the
    // iteration does not settle or the point lies outside the cell
    bool
    inverse_q1(const MeshView &m, const std::vector<double> &vert, const int (&ce)[3], const double *y, double (&xi)[3])
    {
      xi[0] = xi[1] = xi[2] = 0.5;
      if (m.dim < 3)
        xi[2] = 0;
      for (int it = 0; it < 50; ++it)
        {
          double x[3], J[3][3];
          q1_map(m, vert, ce, xi, x, J);
          double r[3] = {0, 0, 0}, dx[3] = {0, 0, 0};
          for (int d = 0; d < m.dim; ++d)
            r[d] = y[d] - x[d];
          if (m.dim == 2)
            {
              const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
              dx[0]            = (J[1][1] * r[0] - J[0][1] * r[1]) / det;
              dx[1]            = (-J[1][0] * r[0] + J[0][0] * r[1]) / det;
            }
          else
            {
              const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                                 J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                                 J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
              for (int c = 0; c < 3; ++c)
                {
                  double Jc[3][3];
                  for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                      Jc[i][j] = j == c ? r[i] : J[i][j];
                  dx[c] = (Jc[0][0] * (Jc[1][1] * Jc[2][2] - Jc[1][2] * Jc[2][1]) -
                           Jc[0][1] * (Jc[1][0] * Jc[2][2] - Jc[1][2] * Jc[2][0]) +
                           Jc[0][2] * (Jc[1][0] * Jc[2][1] - Jc[1][1] * Jc[2][0])) /
                          det;
                }
            }
          double step = 0;
          for (int d = 0; d < m.dim; ++d)
            {
              xi[d] += dx[d];
              step = std::max(step, std::abs(dx[d]));
            }
          if (!(step < 1e300))
            return false;
          if (step < 1e-14)
            break;
        }
      for (int d = 0; d < m.dim; ++d)
        if (xi[d] < -1e-10 || xi[d] > 1 + 1e-10)
          return false;
      for (int d = 0; d < m.dim; ++d)
        xi[d] = std::min(1.0, std::max(0.0, xi[d]));
      return true;
    }
  } // namespace

  void
  SlabSolver::point_values(int n_pts, const double *pts, int samples, double *times, double *values, cudaStream_t s)
  {
    const Mesh     &fine = *meshes.back();
    const MeshView &m    = fine.v;
    const int       p = m.p, p1 = p + 1;
    const int       nd = m.dim == 2 ? p1 * p1 : p1 * p1 * p1;
    STMG_REQUIRE(n_pts >= 1 && pts && values, STMG_ERR_ARG, "point_values: no points or null output");
    STMG_REQUIRE(samples >= 2, STMG_ERR_ARG, "point_values: at least two samples per step");
    const FETables           &tb = host_tables();
    const std::vector<double> xs(tb.xs[p], tb.xs[p] + p1);
    std::vector<long long>    node(std::size_t(n_pts) * nd);
    std::vector<double>       w(std::size_t(n_pts) * nd);
    for (int k = 0; k < n_pts; ++k)
      {
        const double *y = pts + std::size_t(k) * m.dim;
        // first guess from the bounding box of the vertices, then the
        // neighbouring cells (vertices move by less than a cell)
        double lo[3], hi[3];
        for (int d = 0; d < m.dim; ++d)
          {
            lo[d] = fine.vert_h[d];
            hi[d] = fine.vert_h[(fine.vert_h.size() / m.dim - 1) * m.dim + d];
          }
        int  g[3] = {0, 0, 0}, ce[3] = {0, 0, 0};
        bool found = false;
        double xi[3];
        for (int d = 0; d < m.dim; ++d)
          g[d] = std::min(m.n[d] - 1, std::max(0, int(std::floor((y[d] - lo[d]) / (hi[d] - lo[d]) * m.n[d]))));
        for (int rad = 0; rad <= 2 && !found; ++rad)
          for (int dz = -rad; dz <= rad && !found; ++dz)
            for (int dy = -rad; dy <= rad && !found; ++dy)
              for (int dx = -rad; dx <= rad && !found; ++dx)
                {
                  const int o[3] = {dx, dy, m.dim == 3 ? dz : 0};
                  if (m.dim == 2 && dz != 0)
                    continue;
                  bool ok = true;
                  for (int d = 0; d < m.dim; ++d)
                    {
                      ce[d] = g[d] + o[d];
                      ok    = ok && ce[d] >= 0 && ce[d] < m.n[d];
                    }
                  if (ok && inverse_q1(m, fine.vert_h, ce, y, xi))
                    found = true;
                }
        STMG_REQUIRE(found, STMG_ERR_ARG, "point_values: a point lies outside the mesh");
        for (int a = 0; a < nd; ++a)
          {
            const int ai[3] = {a % p1, (a / p1) % p1, a / (p1 * p1)};
            double    wa    = 1.0;
            long long gi    = 0, stride = 1;
            for (int d = 0; d < m.dim; ++d)
              {
                wa *= tfe::lagrange(xs, ai[d], xi[d]);
                gi += (ce[d] * p + ai[d]) * stride;
                stride *= m.nn[d];
              }
            node[std::size_t(k) * nd + a] = gi;
            w[std::size_t(k) * nd + a]    = wa;
          }
      }
    // point values of the slab's time blocks and of its initial value
    // (prev_x, the previous slab's last block: cGP's first time node)
    DevBuf<long long> dnode(node.size());
    DevBuf<double>    dw(w.size()), dv(std::size_t(n_pts) * (nb + 1));
    STMG_CUDA(cudaMemcpyAsync(dnode.ptr, node.data(), node.size() * sizeof(long long), cudaMemcpyHostToDevice, s));
    STMG_CUDA(cudaMemcpyAsync(dw.ptr, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    point_gather_kernel<<<(n_pts * nb + 127) / 128, 128, 0, s>>>(n_pts, nd, nb, N, dnode.ptr, dw.ptr, x.ptr, dv.ptr);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    point_gather_kernel<<<(n_pts + 127) / 128, 128, 0, s>>>(n_pts, nd, 1, N, dnode.ptr, dw.ptr, prev_x.ptr,
                                                           dv.ptr + std::size_t(n_pts) * nb);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    std::vector<double> pv(std::size_t(n_pts) * (nb + 1));
    STMG_CUDA(cudaMemcpyAsync(pv.data(), dv.ptr, pv.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    STMG_CUDA(cudaStreamSynchronize(s));
    // per step: the time nodes' values (cGP: the step's initial value first),
    // then the Lagrange time basis at the sample times
    const auto                type = tfe::Type(cfg.time_type);
    const std::vector<double> tq   = tfe::basis_points(type, cfg.time_degree);
    const int                 nb1  = int(tq.size());
    const bool                cgp  = type == tfe::CGP;
    const double              t0   = time - cfg.n_steps * cfg.tau; // start of the last slab
    const double              step = 1.0 / (samples - 1);
    for (int it = 0; it < cfg.n_steps; ++it)
      for (int row = 0; row < samples; ++row)
        {
          const double ts = row * step;
          if (times)
            times[it * samples + row] = t0 + cfg.tau * (it + ts);
          for (int k = 0; k < n_pts; ++k)
            {
              double acc = 0.0;
              for (int q = 0; q < nb1; ++q)
                {
                  double u;
                  if (cgp && q == 0)
                    u = it == 0 ? pv[std::size_t(nb) * n_pts + k] : pv[std::size_t(it * ni - 1) * n_pts + k];
                  else
                    u = pv[std::size_t(it * ni + q - (cgp ? 1 : 0)) * n_pts + k];
                  acc += tfe::lagrange(tq, q, ts) * u;
                }
              values[std::size_t(it * samples + row) * n_pts + k] = acc;
            }
        }
  }
} // namespace stmg
