// Slab solve on the GPU (see solver.h).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <utility>

#include "kernels_common.cuh"
#include "op_apply_impl.cuh"
#include "solver.h"

namespace stmg
{
  namespace
  {
    constexpr double PI = 3.14159265358979323846;

    // ------------------------------------------------- error norms
    // ErrorCalculator (exact_solution.h:217-299): at one time point the
    // difference between the FE function and the manufactured solution
    // u = sin(2 pi f t) prod_i sin(2 pi f x_i), integrated per cell with
    // QGauss(nq) per direction on the Q1-mapped cell: L2^2, H1-seminorm^2
    // and the largest |e| at the quadrature points.
    struct ErrTab
    {
      int    nq, p1;
      double gx[MAX_P + 2], gw[MAX_P + 2];
      double phi[MAX_P + 2][MAX_P + 1], dphi[MAX_P + 2][MAX_P + 1];
    };

    template <int DIM>
    __global__ void
    err_cell_kernel(const MeshView m, const __grid_constant__ ErrTab et, const double *__restrict__ u, double t,
                    double f, double *__restrict__ cl2, double *__restrict__ ch1, double *__restrict__ cl8)
    {
      const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (cell >= m.ncells)
        return;
      const int cx = int(cell % m.n[0]), cy = int((cell / m.n[0]) % m.n[1]),
                cz = DIM == 3 ? int(cell / ((long long)m.n[0] * m.n[1])) : 0;
      double X[1 << DIM][DIM];
      load_corners<DIM>(m, cx, cy, cz, X);
      const int p = m.p, p1 = et.p1, nq = et.nq;
      const int nqt = DIM == 3 ? nq * nq * nq : nq * nq, nd = DIM == 3 ? p1 * p1 * p1 : p1 * p1;
      const double tv = sin(2 * 3.14159265358979323846 * f * t), k2 = 2 * 3.14159265358979323846 * f;
      double s2 = 0, sh = 0, s8 = 0;
      for (int q = 0; q < nqt; ++q)
        {
          const int qi[3] = {q % nq, (q / nq) % nq, DIM == 3 ? q / (nq * nq) : 0};
          double    xi[3] = {et.gx[qi[0]], et.gx[qi[1]], DIM == 3 ? et.gx[qi[2]] : 0.0};
          double    w     = et.gw[qi[0]] * et.gw[qi[1]] * (DIM == 3 ? et.gw[qi[2]] : 1.0);
          double    J[DIM][DIM], Ji[DIM][DIM];
          q1_jacobian<DIM>(X, xi, J);
          const double det = det_inv<DIM>(J, Ji);
          double       x[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            x[d] = 0;
#pragma unroll
          for (int v = 0; v < (1 << DIM); ++v)
            {
              double wv = 1;
#pragma unroll
              for (int e = 0; e < DIM; ++e)
                wv *= ((v >> e) & 1) ? xi[e] : 1.0 - xi[e];
#pragma unroll
              for (int d = 0; d < DIM; ++d)
                x[d] += wv * X[v][d];
            }
          double uh = 0, gr[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            gr[d] = 0;
          for (int a = 0; a < nd; ++a)
            {
              const int ai[3] = {a % p1, (a / p1) % p1, DIM == 3 ? a / (p1 * p1) : 0};
              const int gx = cx * p + ai[0], gy = cy * p + ai[1], gz = DIM == 3 ? cz * p + ai[2] : 0;
              if (is_boundary_node(m, gx, gy, gz))
                continue; // the FE function is zero on Dirichlet nodes
              const double ua = u[gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz)];
              double       phi = 1, dphi[DIM];
#pragma unroll
              for (int d = 0; d < DIM; ++d)
                dphi[d] = 1;
#pragma unroll
              for (int d = 0; d < DIM; ++d)
                {
                  const double sv = et.phi[qi[d]][ai[d]];
                  phi *= sv;
#pragma unroll
                  for (int j = 0; j < DIM; ++j)
                    dphi[j] *= j == d ? et.dphi[qi[d]][ai[d]] : sv;
                }
              uh += ua * phi;
#pragma unroll
              for (int j = 0; j < DIM; ++j)
                gr[j] += ua * dphi[j];
            }
          double ue = tv, ge[DIM];
#pragma unroll
          for (int i = 0; i < DIM; ++i)
            {
              ue *= sin(k2 * x[i]);
              ge[i] = k2 * tv;
#pragma unroll
              for (int j = 0; j < DIM; ++j)
                ge[i] *= i == j ? cos(k2 * x[j]) : sin(k2 * x[j]);
            }
          const double e   = uh - ue;
          const double JxW = fabs(det) * w;
          s2 += JxW * e * e;
          s8 = fmax(s8, fabs(e));
#pragma unroll
          for (int i = 0; i < DIM; ++i)
            {
              double gp = 0;
#pragma unroll
              for (int j = 0; j < DIM; ++j)
                gp += Ji[j][i] * gr[j];
              sh += JxW * (gp - ge[i]) * (gp - ge[i]);
            }
        }
      cl2[cell] = s2;
      ch1[cell] = sh;
      cl8[cell] = s8;
    }

    // out = {sum a, sum b, max c} over n cells; one block, fixed order
    __global__ void
    err_reduce_kernel(long long n, const double *__restrict__ a, const double *__restrict__ b,
                      const double *__restrict__ c, double *__restrict__ out)
    {
      __shared__ double sa[1024], sb[1024], sc[1024];
      double            x = 0, y = 0, z = 0;
      for (long long i = threadIdx.x; i < n; i += blockDim.x)
        {
          x += a[i];
          y += b[i];
          z = fmax(z, c[i]);
        }
      sa[threadIdx.x] = x;
      sb[threadIdx.x] = y;
      sc[threadIdx.x] = z;
      __syncthreads();
      for (int h = blockDim.x / 2; h > 0; h >>= 1)
        {
          if (threadIdx.x < h)
            {
              sa[threadIdx.x] += sa[threadIdx.x + h];
              sb[threadIdx.x] += sb[threadIdx.x + h];
              sc[threadIdx.x] = fmax(sc[threadIdx.x], sc[threadIdx.x + h]);
            }
          __syncthreads();
        }
      if (threadIdx.x == 0)
        {
          out[0] = sa[0];
          out[1] = sb[0];
          out[2] = sc[0];
        }
    }

    // ------------------------------------------------- adjoint gradient
    // g[c] += scale * kappa_c * sum_j lam_j^T K_c (sum_i T(j,i) V_i) on the
    // cell's dofs, K_c the cell stiffness with unit coefficient (Dirichlet
    // dofs excluded): the derivative of lam^T (T (x) K(kappa)) V with respect
    // to log kappa_c. One thread per cell, FP64.
    template <int DIM, int P, bool CART>
    __global__ void
    grad_contract_kernel(const MeshView m, const __grid_constant__ Cart1D<double> c1,
                         const __grid_constant__ QTab<double> qt, const __grid_constant__ TimeMats<double> Tm,
                         const double *__restrict__ lam, const double *__restrict__ V, double scale,
                         double *__restrict__ g)
    {
      constexpr int   P1   = P + 1;
      constexpr int   ND   = Tens<P1, DIM>::ND;
      const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (cell >= m.ncells)
        return;
      const int cx = int(cell % m.n[0]), cy = int((cell / m.n[0]) % m.n[1]),
                cz = DIM == 3 ? int(cell / ((long long)m.n[0] * m.n[1])) : 0;
      long long idx[ND];
      bool      fr[ND];
#pragma unroll
      for (int q = 0; q < ND; ++q)
        {
          const int gx = cx * P + q % P1, gy = cy * P + (q / P1) % P1, gz = DIM == 3 ? cz * P + q / (P1 * P1) : 0;
          idx[q]       = gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz);
          fr[q]        = !is_boundary_node(m, gx, gy, gz);
        }
      MeshView mu   = m;
      mu.coeff_mode = 0; // unit coefficient inside the cell kernels
      double acc    = 0;
      for (int j = 0; j < Tm.nt_out; ++j)
        {
          double w[ND], z[ND], out[ND];
#pragma unroll
          for (int q = 0; q < ND; ++q)
            {
              double s = 0;
              for (int i = 0; i < Tm.nt_in; ++i)
                s += Tm.A[j * Tm.nt_in + i] * (fr[q] ? V[i * m.N + idx[q]] : 0.0);
              w[q] = s;
              z[q] = 0;
            }
          if constexpr (CART)
            op_detail::cart_apply<DIM, P>(c1, w, z, out);
          else
            op_detail::general_apply<DIM, P>(mu, qt, cx, cy, cz, cell, w, z, out);
#pragma unroll
          for (int q = 0; q < ND; ++q)
            if (fr[q])
              acc += lam[j * m.N + idx[q]] * out[q];
        }
      const double kap = m.coeff_mode == 1 ? m.coeff64[cell] : 1.0;
      g[cell] += scale * kap * acc;
    }

    void
    grad_contract(const Mesh &mesh, const tfe::Mat &T, const double *lam, const double *V, double scale, double *g,
                  cudaStream_t s)
    {
      const MeshView  &m = mesh.v;
      TimeMats<double> tm{};
      tm.nt_out = T.m;
      tm.nt_in  = T.n;
      for (int k = 0; k < T.m * T.n; ++k)
        tm.A[k] = T.a[k];
      Cart1D<double> c1{};
      {
        const FETables &t = host_tables();
        const int       n = m.p + 1;
        for (int d = 0; d < 3; ++d)
          for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
              {
                c1.M[d][a * n + b] = t.M1[m.p][a][b] * m.h[d];
                c1.K[d][a * n + b] = t.K1[m.p][a][b] / m.h[d];
              }
      }
      const QTab<double> qt = make_qtab<double>(m.p);
      const unsigned     nb = unsigned((m.ncells + 127) / 128);
#define STMG_GC(D, PP)                                                                                   \
  if (m.dim == D && m.p == PP)                                                                           \
    {                                                                                                    \
      if (m.box)                                                                                         \
        grad_contract_kernel<D, PP, true><<<nb, 128, 0, s>>>(m, c1, qt, tm, lam, V, scale, g);           \
      else                                                                                               \
        grad_contract_kernel<D, PP, false><<<nb, 128, 0, s>>>(m, c1, qt, tm, lam, V, scale, g);          \
      count_launch();                                                                                    \
      STMG_CUDA(cudaGetLastError());                                                                     \
      return;                                                                                            \
    }
      STMG_GC(2, 1) STMG_GC(2, 2) STMG_GC(2, 3) STMG_GC(3, 1) STMG_GC(3, 2) STMG_GC(3, 3)
#undef STMG_GC
      throw Error(STMG_ERR_UNSUPPORTED, "gradient: dim/degree not supported");
    }

    // ------------------------------------------------- dense tail helpers
    // Device FP64 matrices, column-major: M(i, j) = m[i + j * rows].
    struct DMat
    {
      long long      rows = 0, cols = 0;
      DevBuf<double> m;
      DMat() = default;
      DMat(long long r, long long c)
        : rows(r)
        , cols(c)
        , m(std::size_t(r * c))
      {}
    };

    // C = A B (+ C if acc), 32 x 32 tiles through shared memory
    __global__ void
    dgemm_kernel(long long n, long long k, long long m, const double *__restrict__ A, const double *__restrict__ B,
                 double *__restrict__ C, int acc)
    {
      __shared__ double As[32][33], Bs[32][33];
      const int       tx = threadIdx.x & 31, ty = threadIdx.x >> 5; // 32 x 8 threads
      const long long i0 = blockIdx.x * 32ll, j0 = blockIdx.y * 32ll;
      double          c[4] = {0, 0, 0, 0};
      for (long long p0 = 0; p0 < k; p0 += 32)
        {
          for (int r = ty; r < 32; r += 8)
            {
              const long long i = i0 + tx, p = p0 + r; // A(i, p): column p, row i
              As[r][tx]         = (i < n && p < k) ? A[i + p * n] : 0.0;
              const long long pp = p0 + tx, j = j0 + r; // B(pp, j)
              Bs[r][tx]          = (pp < k && j < m) ? B[pp + j * k] : 0.0;
            }
          __syncthreads();
#pragma unroll 8
          for (int q = 0; q < 32; ++q)
            {
              const double av = As[q][tx];
#pragma unroll
              for (int u = 0; u < 4; ++u)
                c[u] += av * Bs[ty + 8 * u][q];
            }
          __syncthreads();
        }
      const long long i = i0 + tx;
      if (i < n)
#pragma unroll
        for (int u = 0; u < 4; ++u)
          {
            const long long j = j0 + ty + 8 * u;
            if (j < m)
              C[i + j * n] = (acc ? C[i + j * n] : 0.0) + c[u];
          }
    }

    DMat
    dmul(const DMat &A, const DMat &B, cudaStream_t s)
    {
      STMG_REQUIRE(A.cols == B.rows, STMG_ERR_SHAPE, "gmg: dense tail shapes");
      DMat      C(A.rows, B.cols);
      const dim3 grid(unsigned((A.rows + 31) / 32), unsigned((B.cols + 31) / 32));
      dgemm_kernel<<<grid, 256, 0, s>>>(A.rows, A.cols, B.cols, A.m.ptr, B.m.ptr, C.m.ptr, 0);
      STMG_CUDA(cudaGetLastError());
      return C;
    }

    // y = a x + b y (+ c on the diagonal), elementwise over an n x n matrix
    __global__ void
    dcombine_kernel(long long n, double a, const double *__restrict__ x, double b, double *__restrict__ y, double diag)
    {
      const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (i >= n * n)
        return;
      y[i] = a * x[i] + b * y[i] + (i / n == i % n ? diag : 0.0);
    }

    void
    dcombine(double a, const DMat &x, double b, DMat &y, double diag, cudaStream_t s)
    {
      const long long n = y.rows;
      dcombine_kernel<<<unsigned((n * n + 255) / 256), 256, 0, s>>>(n, a, x.m.ptr, b, y.m.ptr, diag);
      STMG_CUDA(cudaGetLastError());
    }

    // matrix of a linear map on device FP64 vectors, applied to the columns
    // of the identity (column j of the result = map(e_j))
    template <typename F>
    DMat
    dense_of(long long n_out, long long n_in, F &&apply, cudaStream_t s)
    {
      DMat I(n_in, n_in), Y(n_out, n_in);
      STMG_CUDA(cudaMemsetAsync(I.m.ptr, 0, sizeof(double) * n_in * n_in, s));
      dcombine_kernel<<<unsigned((n_in * n_in + 255) / 256), 256, 0, s>>>(n_in, 0.0, I.m.ptr, 0.0, I.m.ptr, 1.0);
      STMG_CUDA(cudaGetLastError());
      for (long long j = 0; j < n_in; ++j)
        apply(I.m.ptr + j * n_in, Y.m.ptr + j * n_out);
      return Y;
    }

    // row-major copy of a column-major matrix in the V-cycle's type
    template <typename T>
    __global__ void
    to_rowmajor_kernel(long long n, const double *__restrict__ cm, T *__restrict__ rm)
    {
      const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (e >= n * n)
        return;
      const long long r = e / n, c = e % n;
      rm[e]             = T(cm[r + c * n]);
    }

    // y = C x with C in FP64 and FP64 accumulation whatever the vectors'
    // type (the coarse-grid map stays FP64 inside an FP32 V-cycle); one warp
    // per row, fixed reduction order
    template <typename T>
    __global__ void
    dense_matvec_kernel(int n, const double *__restrict__ C, const T *__restrict__ x, T *__restrict__ y)
    {
      const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
      if (row >= n)
        return;
      double acc = 0.0;
      for (int j = lane; j < n; j += 32)
        acc += C[(long long)row * n + j] * double(x[j]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0)
        y[row] = T(acc);
    }

    // ------------------------------------------------- right-hand side
    // VectorTools::create_right_hand_side with QGauss(p+1) for the
    // manufactured sources of tests/include/exact_solution.h:53-75 (heat)
    // and 164-184 (wave): one thread per node gathers its cells' integrals.
    template <int DIM, int P>
    __global__ void
    manufactured_rhs_kernel(const MeshView m, const __grid_constant__ QTab<double> qt, double t, double f, int wave,
                            double *__restrict__ out)
    {
      constexpr int   P1   = P + 1;
      const long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (node >= m.N)
        return;
      const int g[3] = {int(node % m.nn[0]), int((node / m.nn[0]) % m.nn[1]), int(node / ((long long)m.nn[0] * m.nn[1]))};
      if (is_boundary_node(m, g[0], g[1], g[2]))
        {
          out[node] = 0.0;
          return;
        }
      const double tf = wave ? std::pow(2.0, DIM) * (PI * f) * (PI * f) * sin(2 * PI * f * t)
                             : DIM * 4 * PI * PI * f * f * sin(2 * PI * f * t) + 2 * PI * f * cos(2 * PI * f * t);
      int lo[3], hi[3];
      for (int d = 0; d < 3; ++d)
        {
          if (d >= DIM)
            {
              lo[d] = hi[d] = 0;
              continue;
            }
          hi[d] = min(g[d] / P, m.n[d] - 1);
          lo[d] = (g[d] % P == 0 && g[d] > 0) ? g[d] / P - 1 : hi[d];
        }
      double acc = 0;
      for (int cz = lo[2]; cz <= hi[2]; ++cz)
        for (int cy = lo[1]; cy <= hi[1]; ++cy)
          for (int cx = lo[0]; cx <= hi[0]; ++cx)
            {
              double X[1 << DIM][DIM];
              load_corners<DIM>(m, cx, cy, cz, X);
              const int a[3] = {g[0] - cx * P, g[1] - cy * P, DIM == 3 ? g[2] - cz * P : 0};
              const int nq   = DIM == 3 ? P1 * P1 * P1 : P1 * P1;
              for (int q = 0; q < nq; ++q)
                {
                  const int qi[3] = {q % P1, (q / P1) % P1, q / (P1 * P1)};
                  double    xi[3] = {qt.gx[qi[0]], qt.gx[qi[1]], DIM == 3 ? qt.gx[qi[2]] : 0.0};
                  double    J[DIM][DIM], Ji[DIM][DIM];
                  q1_jacobian<DIM>(X, xi, J);
                  const double det = det_inv<DIM>(J, Ji);
                  double       w = 1, phi = 1, val = tf;
                  for (int d = 0; d < DIM; ++d)
                    {
                      w *= qt.gw[qi[d]];
                      phi *= qt.S[qi[d] * P1 + a[d]];
                      // physical coordinate of the point (Q1 map)
                      double x = 0;
                      for (int v = 0; v < (1 << DIM); ++v)
                        {
                          double wv = 1;
                          for (int e = 0; e < DIM; ++e)
                            wv *= ((v >> e) & 1) ? xi[e] : 1.0 - xi[e];
                          x += wv * X[v][d];
                        }
                      val *= sin(2 * PI * f * x);
                    }
                  acc += fabs(det) * w * phi * val;
                }
            }
      out[node] = acc;
    }

    // dst (+)= sum_j C(i,j) src_j over blocks, src/dst possibly offset
    __global__ void
    block_combine_kernel(long long N, int n_out, int n_in, const __grid_constant__ TimeMats<double> C,
                         const double *__restrict__ src, double *__restrict__ dst)
    {
      const long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (node >= N)
        return;
      for (int i = 0; i < n_out; ++i)
        {
          double acc = dst[i * N + node];
          for (int j = 0; j < n_in; ++j)
            if (C.A[i * n_in + j] != 0.0)
              acc += C.A[i * n_in + j] * src[j * N + node];
          dst[i * N + node] = acc;
        }
    }

    void
    block_combine(long long N, const tfe::Mat &C, const double *src, double *dst, cudaStream_t s)
    {
      TimeMats<double> tm;
      std::memset(&tm, 0, sizeof(tm));
      tm.nt_out = C.m;
      tm.nt_in  = C.n;
      for (int i = 0; i < C.m * C.n; ++i)
        tm.A[i] = C.a[i];
      block_combine_kernel<<<unsigned((N + 255) / 256), 256, 0, s>>>(N, C.m, C.n, tm, src, dst);
      count_launch();
      STMG_CUDA(cudaGetLastError());
    }

    template <typename T>
    T *
    as(DevBuf<unsigned char> &b)
    {
      return reinterpret_cast<T *>(b.ptr);
    }
  } // namespace

  // ------------------------------------------------------------- meshes
  std::vector<std::unique_ptr<Mesh>>
  build_meshes(const SolverConfig &c)
  {
    const int dim = c.dim, R = c.refine, p = c.degree;
    int       nf[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d)
      nf[d] = c.subdiv[d] << R;
    std::vector<std::unique_ptr<Mesh>> out;
    for (int s = 0; s <= R; ++s)
      {
        const int f     = 1 << (R - s);
        int       n[3]  = {1, 1, 1};
        int       nv[3] = {1, 1, 1}, nvf[3] = {1, 1, 1};
        for (int d = 0; d < dim; ++d)
          {
            n[d]   = nf[d] / f;
            nv[d]  = n[d] + 1;
            nvf[d] = nf[d] + 1;
          }
        std::vector<double> vert;
        if (!c.fine_vertices.empty())
          {
            vert.resize(std::size_t(nv[0]) * nv[1] * nv[2] * dim);
            for (int k = 0; k < nv[2]; ++k)
              for (int j = 0; j < nv[1]; ++j)
                for (int i = 0; i < nv[0]; ++i)
                  {
                    const std::size_t v  = i + std::size_t(nv[0]) * (j + std::size_t(nv[1]) * k);
                    const std::size_t vf = std::size_t(i) * f + std::size_t(nvf[0]) * (std::size_t(j) * f + std::size_t(nvf[1]) * std::size_t(k) * f);
                    for (int d = 0; d < dim; ++d)
                      vert[v * dim + d] = c.fine_vertices[vf * dim + d];
                  }
          }
        int                 mode = 0;
        std::vector<double> coeff;
        if (!c.fine_coeff.empty())
          {
            if (f == 1)
              {
                mode  = 1;
                coeff = c.fine_coeff;
              }
            else
              {
                // the fine per-cell field sampled at this level's quadrature
                // points: a point lies in fine sub-cell min(floor(xi f), f-1)
                mode                 = 2;
                const FETables &t    = host_tables();
                const int       p1   = p + 1;
                const long long ncel = (long long)n[0] * n[1] * n[2];
                const int       nq   = dim == 3 ? p1 * p1 * p1 : p1 * p1;
                coeff.resize(ncel * nq);
                for (long long cc = 0; cc < ncel; ++cc)
                  {
                    const int ci[3] = {int(cc % n[0]), int((cc / n[0]) % n[1]), int(cc / ((long long)n[0] * n[1]))};
                    for (int q = 0; q < nq; ++q)
                      {
                        const int qi[3] = {q % p1, (q / p1) % p1, q / (p1 * p1)};
                        int       fi[3] = {0, 0, 0};
                        for (int d = 0; d < dim; ++d)
                          fi[d] = ci[d] * f + std::min(int(std::floor(t.gx[p][qi[d]] * f)), f - 1);
                        coeff[cc * nq + q] = c.fine_coeff[fi[0] + std::size_t(nf[0]) * (fi[1] + std::size_t(nf[1]) * fi[2])];
                      }
                  }
              }
          }
        out.push_back(make_mesh(dim, n, p, c.lo, c.hi, vert.empty() ? nullptr : vert.data(), mode,
                                coeff.empty() ? nullptr : coeff.data()));
      }
    return out;
  }

  // ---------------------------------------------------------------- GMG
  GMG::GMG(const SolverConfig &c, std::vector<std::unique_ptr<Mesh>> &meshes, Blas &b, bool transpose_time)
    : dtype(c.mg_dtype)
    , cfg(c)
    , blas(b)
  {
    const auto type   = tfe::Type(c.time_type);
    const int  lowest = type == tfe::DG ? 0 : 1;
    int        k_min  = c.fe_degree_min < 0 ? c.time_degree - 1 : c.fe_degree_min;
    k_min             = std::clamp(k_min, lowest, c.time_degree);
    int n_min         = c.n_steps_min < 0 ? c.n_steps / 2 : c.n_steps_min;
    n_min             = std::clamp(n_min, 1, c.n_steps);
    const int n_sp    = int(meshes.size());
    seq               = tfe::mg_sequence(n_sp, c.time_degree, k_min, c.n_steps, n_min);
    const auto sp     = tfe::space_levels(seq, n_sp);
    const auto w      = tfe::level_weights(type, c.problem == 2, c.time_degree, c.tau, c.n_steps, seq);
    const int  L      = int(seq.size()) + 1;
    levels.resize(L);
    int r = c.time_degree, ns = c.n_steps;
    for (int l = L - 1; l >= 0; --l)
      {
        if (l < L - 1)
          {
            if (seq[l] == tfe::K)
              --r;
            else if (seq[l] == tfe::TAU)
              ns /= 2;
          }
        Level &lv  = levels[l];
        lv.mesh    = meshes[sp[l]].get();
        lv.r       = r;
        lv.n_steps = ns;
        lv.nt      = (type == tfe::DG ? r + 1 : r) * ns;
        lv.A       = w[l][0];
        lv.B       = w[l][1];
        if (transpose_time)
          for (tfe::Mat *M : {&lv.A, &lv.B})
            {
              tfe::Mat t(M->n, M->m);
              for (int i = 0; i < M->m; ++i)
                for (int j = 0; j < M->n; ++j)
                  t(j, i) = (*M)(i, j);
              *M = t;
            }
      }
    const std::size_t elem = dtype == STMG_F64 ? 8 : 4;
    for (int l = 0; l < L; ++l)
      {
        Level &lv = levels[l];
        lv.op     = std::make_unique<StOperator>(lv.mesh, lv.nt, lv.nt, lv.A.a.data(), lv.B.a.data(), dtype);
        lv.vanka  = std::make_unique<Vanka>(lv.mesh, lv.nt, lv.A.a.data(), lv.B.a.data(), dtype,
                                           dtype == STMG_F64 ? STMG_F64 : c.vanka_storage);
        if (l > 0)
          lv.to_coarser = make_transfer(l, dtype);
        const std::size_t bytes = std::size_t(lv.size()) * elem;
        lv.sol.alloc(bytes);
        lv.def.alloc(bytes);
        lv.t.alloc(bytes);
        lv.r_.alloc(bytes);
        lv.z.alloc(bytes);
      }
    const char *ng = std::getenv("STMG_NO_GRAPH");
    use_graph      = !(ng && ng[0] == '1');
    cudaStream_t s = nullptr;
    for (int l = 1; l < L; ++l)
      levels[l].omega = dtype == STMG_F64 ? estimate_relaxation<double>(l, s) : estimate_relaxation<float>(l, s);
    STMG_CUDA(cudaDeviceSynchronize());
    build_tail();
  }

  std::unique_ptr<Transfer>
  GMG::make_transfer(int l, int dt) const
  {
    const Level &lv   = levels[l];
    const Level &co   = levels[l - 1];
    const auto   type = tfe::Type(cfg.time_type);
    if (seq[l - 1] == tfe::NONE)
      return std::make_unique<HTransfer>(lv.mesh, co.mesh, lv.nt, dt);
    const tfe::Mat P = seq[l - 1] == tfe::K ? tfe::projection(type, lv.r - 1, lv.r, lv.n_steps)
                                            : tfe::prolongation(type, lv.r, lv.n_steps);
    STMG_REQUIRE(P.m == lv.nt && P.n == co.nt, STMG_ERR_SHAPE, "gmg: time transfer shape");
    return std::make_unique<TTransfer>(lv.mesh, lv.nt, co.nt, P.a.data(), nullptr, dt);
  }

  // The levels 0..tail as one matrix. Per level, with W = omega P_vanka,
  // M = I - W A and m sweeps, smoothing from zero is S = sum_{k<m} M^k W and
  // post-smoothing maps x to M^m x + S d, so (Multigrid::level_v_step)
  //   C_0 = S_0,  C_l = M_l^m (S_l + Pro_l C_{l-1} Res_l (I - A_l S_l)) + S_l.
  // A, P_vanka, Pro and Res are read off the FP64 kernels column by column;
  // the products run as FP64 GEMMs on the device.
  void
  GMG::build_tail()
  {
    const char *e = std::getenv("STMG_DENSE_TAIL");
    if (e && e[0] == '0')
      return;
    int t = -1;
    for (int l = 0; l < int(levels.size()); ++l)
      {
        if (levels[l].size() > DENSE_TAIL_MAX)
          break;
        t = l;
      }
    if (t < 0)
      return;
    cudaStream_t s = nullptr;
    DMat         C;
    for (int l = 0; l <= t; ++l)
      {
        Level          &lv = levels[l];
        const long long n  = lv.size();
        StOperator      op(lv.mesh, lv.nt, lv.nt, lv.A.a.data(), lv.B.a.data(), STMG_F64);
        Vanka           vk(lv.mesh, lv.nt, lv.A.a.data(), lv.B.a.data(), STMG_F64, STMG_F64);
        const DMat      A = dense_of(n, n, [&](const double *x, double *y) { op.apply(false, x, y, false, s); }, s);
        DMat            W = dense_of(n, n, [&](const double *x, double *y) { vk.apply(x, y, s); }, s);
        dcombine(0.0, W, lv.omega, W, 0.0, s); // W = omega P_vanka
        DMat M = dmul(W, A, s);
        dcombine(0.0, M, -1.0, M, 1.0, s); // M = I - W A
        // binary powering: (M^a, S_a) with S_{a+b} = S_a + M^a S_b
        const unsigned m = steps(l) * unsigned(cfg.smoothing_steps);
        STMG_REQUIRE(m > 0, STMG_ERR_ARG, "gmg: zero smoothing steps");
        DMat Mp = std::move(M), Sp = std::move(W), Mm, S;
        bool have = false;
        for (unsigned bits = m;;)
          {
            if (bits & 1u)
              {
                if (!have)
                  {
                    Mm = DMat(n, n);
                    S  = DMat(n, n);
                    STMG_CUDA(cudaMemcpyAsync(Mm.m.ptr, Mp.m.ptr, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, s));
                    STMG_CUDA(cudaMemcpyAsync(S.m.ptr, Sp.m.ptr, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, s));
                    have = true;
                  }
                else
                  {
                    const DMat MS = dmul(Mm, Sp, s);
                    dcombine(1.0, MS, 1.0, S, 0.0, s);
                    Mm = dmul(Mm, Mp, s);
                  }
              }
            bits >>= 1;
            if (!bits)
              break;
            const DMat MS = dmul(Mp, Sp, s);
            dcombine(1.0, MS, 1.0, Sp, 0.0, s);
            Mp = dmul(Mp, Mp, s);
          }
        if (l == 0)
          {
            C = std::move(S);
            continue;
          }
        const long long nc = levels[l - 1].size();
        auto            tr = make_transfer(l, STMG_F64);
        const DMat      Pro = dense_of(
          n, nc,
          [&](const double *x, double *y) {
            fill<double>(n, 0.0, y, s);
            tr->prolongate_add(x, y, s);
          },
          s);
        const DMat Res = dense_of(
          nc, n,
          [&](const double *x, double *y) {
            fill<double>(nc, 0.0, y, s);
            tr->restrict_add(x, y, s);
          },
          s);
        DMat IAS = dmul(A, S, s);
        dcombine(0.0, IAS, -1.0, IAS, 1.0, s); // I - A S
        DMat X = dmul(Pro, dmul(C, dmul(Res, IAS, s), s), s);
        dcombine(1.0, S, 1.0, X, 0.0, s);
        C = dmul(Mm, X, s);
        dcombine(1.0, S, 1.0, C, 0.0, s);
        STMG_CUDA(cudaStreamSynchronize(s));
      }
    const long long n = levels[t].size();
    tail_mat.alloc(std::size_t(n * n) * 8);
    const unsigned nb = unsigned((n * n + 255) / 256);
    to_rowmajor_kernel<double><<<nb, 256, 0, s>>>(n, C.m.ptr, reinterpret_cast<double *>(tail_mat.ptr));
    STMG_CUDA(cudaGetLastError());
    STMG_CUDA(cudaStreamSynchronize(s));
    tail = t;
  }

  std::vector<double>
  GMG::omegas() const
  {
    std::vector<double> o;
    for (auto &l : levels)
      o.push_back(l.omega);
    return o;
  }

  unsigned
  GMG::steps(int l) const
  {
    // MGSmootherPrecondition with variable = true doubles the sweeps per
    // coarser level (gmg.h:558,726)
    return 1u << (levels.size() - 1 - l);
  }

  // PreconditionRelaxation::step: x += omega P (b - A x)
  template <typename T>
  void
  GMG::relax_step(int l, T *x, const T *b, cudaStream_t s)
  {
    Level &lv = levels[l];
    lv.op->apply_ex(false, x, as<T>(lv.r_), -1.0, 0.0, b, s); // r = b - A x
    lv.vanka->apply_ex(as<T>(lv.r_), x, lv.omega, 1.0, s);    // x += omega P r
  }

  // zero_start: MGSmootherPrecondition::apply (first sweep is
  // PreconditionRelaxation::vmult, x = omega P b); otherwise ::smooth.
  template <typename T>
  void
  GMG::smooth(int l, T *x, const T *b, bool zero_start, cudaStream_t s)
  {
    Level   &lv = levels[l];
    unsigned k  = steps(l) * unsigned(cfg.smoothing_steps);
    if (zero_start)
      {
        lv.vanka->apply_ex(b, x, lv.omega, 0.0, s); // x = omega P b
        --k;
      }
    for (unsigned i = 0; i < k; ++i)
      relax_step<T>(l, x, b, s);
  }

  // Multigrid::level_v_step (deal.II multigrid.templates.h)
  template <typename T>
  void
  GMG::vstep(int l, cudaStream_t s)
  {
    Level &lv = levels[l];
    if (l == tail)
      {
        const long long n = lv.size();
        dense_matvec_kernel<T><<<unsigned((n + 7) / 8), 256, 0, s>>>(int(n), as<double>(tail_mat), as<T>(lv.def),
                                                                     as<T>(lv.sol));
        count_launch();
        STMG_CUDA(cudaGetLastError());
        return;
      }
    if (l == 0)
      {
        // MGCoarseGridApplySmoother: smooth from zero (its first sweep
        // reduces to x = omega P b since A 0 = 0)
        smooth<T>(0, as<T>(lv.sol), as<T>(lv.def), true, s);
        return;
      }
    smooth<T>(l, as<T>(lv.sol), as<T>(lv.def), true, s);
    lv.op->apply_ex(false, as<T>(lv.sol), as<T>(lv.t), -1.0, 0.0, as<T>(lv.def), s); // t = d - A x
    Level &co = levels[l - 1];
    fill<T>(co.size(), T(0), as<T>(co.def), s);
    lv.to_coarser->restrict_add(as<T>(lv.t), as<T>(co.def), s);
    vstep<T>(l - 1, s);
    lv.to_coarser->prolongate_add(as<T>(co.sol), as<T>(lv.sol), s);
    smooth<T>(l, as<T>(lv.sol), as<T>(lv.def), false, s);
  }

  // The V-cycle below the FP64/FP32 boundary works on the levels' own
  // buffers only, so it is captured once into a CUDA graph and replayed.
  template <typename T>
  void
  GMG::cycle(cudaStream_t s)
  {
    const int top = int(levels.size()) - 1;
    if (!use_graph)
      return vstep<T>(top, s);
    if (!graph)
      {
        STMG_CUDA(cudaStreamSynchronize(s));
        if (!cap)
          STMG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        vstep<T>(top, cap); // warm-up: kernel attributes and occupancy caches
        STMG_CUDA(cudaStreamSynchronize(cap));
        const long long l0 = launch_count();
        cudaGraph_t     g  = nullptr;
        STMG_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        vstep<T>(top, cap);
        STMG_CUDA(cudaStreamEndCapture(cap, &g));
        graph_nodes = launch_count() - l0;
        add_launches(-graph_nodes); // captured, not run
        STMG_CUDA(cudaGraphInstantiate(&graph, g, 0));
        STMG_CUDA(cudaGraphDestroy(g));
      }
    STMG_CUDA(cudaGraphLaunch(graph, s));
    add_launches(graph_nodes);
  }

  GMG::~GMG()
  {
    if (graph)
      cudaGraphExecDestroy(graph);
    if (cap)
      cudaStreamDestroy(cap);
  }

  void
  GMG::vmult(double *dst, const double *src, cudaStream_t s, double scale)
  {
    // The V-cycle is linear: with scale a power of two, the cycle runs on
    // scale * src and its result is multiplied by 1 / scale, both exact, so
    // dst is the same to the last bit while the cycle's vectors keep a
    // moderate size in its own precision.
    NvtxScope       range("gmg");
    Level          &top = levels.back();
    const long long n   = top.size();
    if (dtype == STMG_F64)
      {
        convert<double, double>(n, src, as<double>(top.def), s, scale);
        cycle<double>(s);
        convert<double, double>(n, as<double>(top.sol), dst, s, 1.0 / scale);
      }
    else
      {
        convert<float, double>(n, src, as<float>(top.def), s, scale);
        cycle<float>(s);
        convert<double, float>(n, as<float>(top.sol), dst, s, 1.0 / scale);
      }
  }

  // GMG::estimate_relaxation (gmg.h:792-844): power iteration with
  // PreconditionChebyshev's start vector (all ones, entry 0 zero), 20 steps,
  // max = 1.2 lambda, omega = 2 / (lambda + 1.2 lambda).
  template <typename T>
  double
  GMG::estimate_relaxation(int l, cudaStream_t s)
  {
    Level          &lv = levels[l];
    const long long n  = lv.size();
    T              *x = as<T>(lv.sol), *y = as<T>(lv.t), *z = as<T>(lv.z);
    fill<T>(n, T(1), x, s);
    STMG_CUDA(cudaMemsetAsync(x, 0, sizeof(T), s));
    double nrm = std::sqrt(blas.dot<T>(n, x, x, s));
    axpby<T>(n, T(0), x, T(1.0 / nrm), x, s);
    double ev = 0;
    for (int it = 0; it < 20; ++it)
      {
        lv.op->apply(false, x, y, false, s);
        lv.vanka->apply(y, z, s);
        ev  = blas.dot<T>(n, x, z, s);
        nrm = std::sqrt(blas.dot<T>(n, z, z, s));
        STMG_REQUIRE(std::isfinite(nrm) && nrm > 0, STMG_ERR_NONFINITE, "gmg: power iteration broke down");
        axpby<T>(n, T(1.0 / nrm), z, T(0), x, s);
      }
    ev = std::abs(ev);
    return 2.0 / (ev + 1.2 * ev);
  }

  // -------------------------------------------------------------- FGMRES
  FGMRES::FGMRES(long long n_, int basis_, Blas &b)
    : n(n_)
    , basis(basis_)
    , blas(b)
  {
    STMG_REQUIRE(basis >= 2 && basis <= MAX_DOTS, STMG_ERR_ARG, "fgmres: restart length 2..32");
    V.resize(basis);
    Z.resize(basis);
    for (int i = 0; i < basis; ++i)
      {
        V[i].alloc(n);
        Z[i].alloc(n);
      }
    aux.alloc(n);
  }

  template <typename Aop, typename Pop>
  int
  FGMRES::solve(Aop &&A, Pop &&P, double *x, const double *b, double abs_tol, double reduce, int max_iter,
                cudaStream_t s)
  {
    // Iteration k checks the residual of the k-dimensional flexible Krylov
    // solution; a restart cycle uses at most basis-1 directions (deal.II
    // SolverFGMRES); ReductionControl: converged if res <= abs_tol or
    // res <= reduce * initial residual.
    int    it          = 0;
    double reduced_tol = -1;
    bool   first       = true;
    // second Gram-Schmidt pass: off until a norm check asks for it, then on
    // for the rest of this solve (deal.II's iterated_gram_schmidt)
    bool   reorth      = false;
    std::vector<const double *> vp(basis), zp(basis);
    for (int i = 0; i < basis; ++i)
      {
        vp[i] = V[i].ptr;
        zp[i] = Z[i].ptr;
      }
    while (true)
      {
        A(aux.ptr, x);
        sub_from<double>(n, b, aux.ptr, s);
        const double beta = std::sqrt(blas.dot<double>(n, aux.ptr, aux.ptr, s));
        STMG_REQUIRE(std::isfinite(beta), STMG_ERR_NONFINITE, "fgmres: non-finite residual");
        if (first)
          {
            reduced_tol      = beta * reduce;
            initial_residual = beta;
            first            = false;
          }
        last_residual = beta;
        if (beta <= reduced_tol || beta <= abs_tol)
          return it;
        STMG_REQUIRE(it < max_iter, STMG_ERR_NOCONV, "fgmres: iteration limit reached");
        std::vector<std::vector<double>> H(basis + 1, std::vector<double>(basis, 0.0));
        std::vector<double>              cs(basis), sn(basis), g(basis + 1, 0.0);
        // V[i] holds the i-th basis vector divided by sc[i]: a new direction
        // keeps the orthogonalised w itself (buffer swap, no normalising pass)
        std::vector<double> sc(basis, 1.0);
        g[0] = beta;
        axpby<double>(n, 1.0 / beta, aux.ptr, 0.0, V[0].ptr, s);
        int  used = 0;
        bool done = false;
        for (int j = 0; j + 1 < basis; ++j)
          {
            // V[j] has norm 1 / sc[j] (up to rounding); the preconditioner
            // gets it scaled by the power of two nearest sc[j], so the FP32
            // V-cycle sees a vector of norm in [1/2, 2) however far the
            // products of the subdiagonal norms drift over a restart cycle
            P(Z[j].ptr, V[j].ptr, std::ldexp(1.0, std::ilogb(sc[j] * 1.4142135623730951)));
            A(aux.ptr, Z[j].ptr);
            // classical Gram-Schmidt as deal.II's iterated_gram_schmidt: one
            // pass over the basis for h = V^T w, one for w -= V h and |w|^2.
            // Every fifth inner iteration |w|^2 before the pass comes with h
            // (w dotted with itself); if the pass leaves less than
            // 10 sqrt(eps) of that norm, a second pass runs now and in every
            // later iteration of this solve.
            // With the stored scales: h_i = sc_i (V[i] . w), w -= sum_i (h_i sc_i) V[i].
            // The coefficients h_i sc_i stay on the device between the two
            // passes (Blas::gs_pass): one host wait per pass.
            const bool consider = !reorth && j % 5 == 4;
            std::vector<double> h(j + 2), h2(j + 1);
            double hn2 = blas.gs_pass<double>(n, j + 1, vp.data(), sc.data(), aux.ptr, consider, h.data(), s);
            for (int i = 0; i <= j; ++i)
              H[i][j] = h[i];
            if (consider && !(std::sqrt(hn2) > 10.0 * std::sqrt(h[j + 1]) * std::sqrt(DBL_EPSILON)))
              reorth = true;
            if (reorth)
              {
                hn2 = blas.gs_pass<double>(n, j + 1, vp.data(), sc.data(), aux.ptr, false, h2.data(), s);
                for (int i = 0; i <= j; ++i)
                  H[i][j] += h2[i];
              }
            const double hn = std::sqrt(hn2);
            H[j + 1][j]     = hn;
            if (hn != 0.0)
              {
                std::swap(V[j + 1], aux);
                vp[j + 1] = V[j + 1].ptr;
                sc[j + 1] = 1.0 / hn;
              }
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
            STMG_REQUIRE(std::isfinite(res), STMG_ERR_NONFINITE, "fgmres: non-finite residual");
            last_residual = res;
            if (res <= reduced_tol || res <= abs_tol)
              {
                done = true;
                break;
              }
            STMG_REQUIRE(it < max_iter, STMG_ERR_NOCONV, "fgmres: iteration limit reached");
          }
        std::vector<double> y(used);
        for (int i = used - 1; i >= 0; --i)
          {
            double acc = g[i];
            for (int k = i + 1; k < used; ++k)
              acc -= H[i][k] * y[k];
            y[i] = acc / H[i][i];
          }
        blas.combine<double>(n, 1.0, used, y.data(), zp.data(), x, s);
        if (done)
          return it;
      }
  }

  // --------------------------------------------------------- slab solver
  SlabSolver::SlabSolver(const SolverConfig &c)
    : cfg(c)
  {
    STMG_REQUIRE(c.problem == 1 || c.problem == 2, STMG_ERR_ARG, "solver: problem must be heat (1) or wave (2)");
    STMG_REQUIRE(c.time_type == 1 || c.time_type == 2, STMG_ERR_ARG, "solver: time type must be CGP (1) or DG (2)");
    meshes = build_meshes(c);
    gmg    = std::make_unique<GMG>(c, meshes, blas);
    Mesh *fine = meshes.back().get();
    N          = fine->v.N;
    const auto type = tfe::Type(c.time_type);
    auto       w1a  = tfe::slab_weights(type, c.time_degree, c.tau, 1);
    for (int i = 0; i < 4; ++i)
      w1[i] = w1a[i];
    ni = w1[0].m;
    nb = ni * c.n_steps;
    tfe::Mat lhsK, lhsM, rK, rM, rV(nb, 1);
    if (c.problem == 2)
      {
        auto ww = tfe::wave_weights(type, w1[0], w1[1], w1[2], w1[3], c.n_steps);
        lhsK = ww[0], lhsM = ww[1], rK = ww[2], rM = ww[3], rV = ww[4];
        const tfe::Mat Ai = tfe::inverse(w1[0]);
        AixB              = tfe::mul(Ai, w1[1]);
        AixG              = tfe::mul(Ai, w1[2]);
        AixZ              = tfe::mul(Ai, w1[3]);
        for (auto &e : (type == tfe::DG ? AixG : AixZ).a)
          e = -e;
      }
    else
      {
        auto wn = tfe::slab_weights(type, c.time_degree, c.tau, c.n_steps);
        lhsK    = wn[0];
        lhsM    = wn[1];
        rK      = type == tfe::CGP ? wn[2] : tfe::Mat(nb, 1);
        rM      = type == tfe::CGP ? wn[3] : wn[2];
      }
    lhsK_ = lhsK;
    rK_   = rK;
    A64   = std::make_unique<StOperator>(fine, nb, nb, lhsK.a.data(), lhsM.a.data(), STMG_F64);
    rhs64 = std::make_unique<StOperator>(fine, nb, 1, rK.a.data(), rM.a.data(), STMG_F64);
    if (c.problem == 2)
      {
        tfe::Mat zero(nb, 1);
        rhsv64 = std::make_unique<StOperator>(fine, nb, 1, zero.a.data(), rV.a.data(), STMG_F64);
      }
    const double one = 1.0, zero1 = 0.0;
    mass64 = std::make_unique<StOperator>(fine, 1, 1, &zero1, &one, STMG_F64);
    gmres  = std::make_unique<FGMRES>(N * nb, c.restart, blas);
    x.alloc(N * nb);
    v.alloc(N * nb);
    rhs.alloc(N * nb);
    prev_x.alloc(N);
    prev_v.alloc(N);
    F.alloc(N);
    STMG_CUDA(cudaMemset(x.ptr, 0, N * nb * 8));
    STMG_CUDA(cudaMemset(v.ptr, 0, N * nb * 8));
    // node coordinates (Q1 map of the owning cell at the Lobatto points)
    const MeshView &m  = fine->v;
    const FETables &tb = host_tables();
    node_x.resize(N * m.dim);
    const int p = m.p;
    for (long long i = 0; i < N; ++i)
      {
        const long long gi[3] = {i % m.nn[0], (i / m.nn[0]) % m.nn[1], i / ((long long)m.nn[0] * m.nn[1])};
        int             ce[3] = {0, 0, 0};
        double          xi[3] = {0, 0, 0};
        for (int d = 0; d < m.dim; ++d)
          {
            ce[d] = std::min(int(gi[d] / p), m.n[d] - 1);
            xi[d] = tb.xs[p][gi[d] - ce[d] * p];
          }
        for (int d = 0; d < m.dim; ++d)
          {
            double acc = 0;
            for (int vtx = 0; vtx < (1 << m.dim); ++vtx)
              {
                double wv = 1;
                for (int e = 0; e < m.dim; ++e)
                  wv *= ((vtx >> e) & 1) ? xi[e] : 1.0 - xi[e];
                const long long vi = (ce[0] + (vtx & 1)) +
                                     (long long)(m.n[0] + 1) * ((ce[1] + ((vtx >> 1) & 1)) +
                                                                (m.dim == 3 ? (long long)(m.n[1] + 1) * (ce[2] + ((vtx >> 2) & 1)) : 0));
                acc += wv * fine->vert_h[vi * m.dim + d];
              }
            node_x[i * m.dim + d] = acc;
          }
      }
    Mf.alloc(N);
    fsrc.alloc(N);
    if (c.rhs_mode == 1)
      {
        STMG_REQUIRE((long long)c.f_nodal.size() == N, STMG_ERR_SHAPE, "solver: nodal source has wrong size");
        set_source(c.f_nodal.data());
      }
    set_initial(nullptr, nullptr);
  }

  void
  SlabSolver::set_source(const double *f_nodal)
  {
    STMG_REQUIRE(cfg.rhs_mode == 1, STMG_ERR_ARG, "solver: set_source needs rhs_mode 1");
    STMG_CUDA(cudaMemcpy(fsrc.ptr, f_nodal, N * sizeof(double), cudaMemcpyHostToDevice));
    mass64->apply(false, fsrc.ptr, Mf.ptr, false, nullptr);
    STMG_CUDA(cudaStreamSynchronize(nullptr));
  }

  void
  SlabSolver::set_initial(const double *u0, const double *v0)
  {
    const MeshView     &m = meshes.back()->v;
    std::vector<double> hu(N, 0.0), hv(N, 0.0);
    const double        f = cfg.frequency;
    for (long long i = 0; i < N; ++i)
      {
        const long long gi[3] = {i % m.nn[0], (i / m.nn[0]) % m.nn[1], i / ((long long)m.nn[0] * m.nn[1])};
        bool            bd    = false;
        for (int d = 0; d < m.dim; ++d)
          bd = bd || gi[d] == 0 || gi[d] == m.nn[d] - 1;
        if (bd)
          continue;
        double su = 0, sv = 2 * PI * f; // u(0) = sin(0) ... = 0, v(0) = 2 pi f prod sin
        for (int d = 0; d < m.dim; ++d)
          sv *= std::sin(2 * PI * f * node_x[i * m.dim + d]);
        hu[i] = u0 ? u0[i] : su;
        hv[i] = v0 ? v0[i] : sv;
      }
    wait_snapshot_host();
    STMG_CUDA(cudaMemset(x.ptr, 0, N * nb * 8));
    STMG_CUDA(cudaMemset(v.ptr, 0, N * nb * 8));
    STMG_CUDA(cudaMemcpy(x.ptr + (nb - 1) * N, hu.data(), N * 8, cudaMemcpyHostToDevice));
    if (cfg.problem == 2)
      STMG_CUDA(cudaMemcpy(v.ptr + (nb - 1) * N, hv.data(), N * 8, cudaMemcpyHostToDevice));
    time     = 0;
    err_l2sq = err_h1sq = err_l8 = 0;
  }

  void
  SlabSolver::force(double t, double *out, cudaStream_t s)
  {
    const MeshView &m = meshes.back()->v;
    if (cfg.rhs_mode == 1)
      {
        STMG_CUDA(cudaMemcpyAsync(out, Mf.ptr, N * 8, cudaMemcpyDeviceToDevice, s));
        return;
      }
    if (cfg.rhs_mode == 2)
      {
        STMG_CUDA(cudaMemsetAsync(out, 0, N * 8, s));
        return;
      }
    const unsigned nbk  = unsigned((N + 127) / 128);
    const int      wave = cfg.problem == 2;
#define STMG_RHS(D, PP)                                                                                  \
  if (m.dim == D && m.p == PP)                                                                           \
    {                                                                                                    \
      manufactured_rhs_kernel<D, PP><<<nbk, 128, 0, s>>>(m, make_qtab<double>(PP), t, cfg.frequency, wave, out); \
      STMG_CUDA(cudaGetLastError());                                                                     \
      return;                                                                                            \
    }
    STMG_RHS(2, 1) STMG_RHS(2, 2) STMG_RHS(2, 3) STMG_RHS(2, 4) STMG_RHS(2, 5) STMG_RHS(3, 1) STMG_RHS(3, 2) STMG_RHS(3, 3)
#undef STMG_RHS
    throw Error(STMG_ERR_UNSUPPORTED, "solver: manufactured source for this dim/degree");
      count_launch();
  }

  void
  SlabSolver::system_vmult(double *dst, const double *src, cudaStream_t s)
  {
    A64->apply(false, src, dst, false, s);
  }

  int
  SlabSolver::solve(double *xv, const double *b, cudaStream_t s)
  {
    auto Aop = [&](double *dst, const double *src) {
      NvtxScope r("vmult");
      A64->apply(false, src, dst, false, s);
    };
    auto Pop = [&](double *dst, const double *src, double scale) { gmg->vmult(dst, src, s, scale); };
    return gmres->solve(Aop, Pop, xv, b, cfg.abs_tol, cfg.tol, cfg.max_iter, s);
  }

  void
  SlabSolver::run(int n_slabs, int *its, cudaStream_t s)
  {
    wait_snapshot(s);
    const auto                type = tfe::Type(cfg.time_type);
    const std::vector<double> tq   = tfe::basis_points(type, cfg.time_degree);
    for (int slab = 0; slab < n_slabs; ++slab)
      {
        NvtxScope step_range("step");
        STMG_CUDA(cudaMemcpyAsync(prev_x.ptr, x.ptr + (nb - 1) * N, N * 8, cudaMemcpyDeviceToDevice, s));
        if (cfg.problem == 2)
          STMG_CUDA(cudaMemcpyAsync(prev_v.ptr, v.ptr + (nb - 1) * N, N * 8, cudaMemcpyDeviceToDevice, s));
        // rhs (time_integrators.h:163-170 / 248-252)
        rhs64->apply(false, prev_x.ptr, rhs.ptr, false, s);
        if (cfg.problem == 2)
          rhsv64->apply(false, prev_v.ptr, rhs.ptr, true, s);
        // assemble_force (time_integrators.h:60-87)
        for (int it = 0; it < cfg.n_steps; ++it)
          for (int j = 0; j < int(tq.size()); ++j)
            {
              const double tt = time + cfg.tau * it + cfg.tau * tq[j];
              if (cfg.rhs_mode == 2)
                continue;
              force(tt, F.ptr, s);
              if (type == tfe::DG)
                axpby<double>(N, w1[0](j, j), F.ptr, 1.0, rhs.ptr + (j + it * ni) * N, s);
              else if (j == 0)
                for (int i = 0; i < w1[2].m; ++i)
                  axpby<double>(N, -w1[2](i, 0), F.ptr, 1.0, rhs.ptr + (i + it * ni) * N, s);
              else
                axpby<double>(N, w1[0](j - 1, j - 1), F.ptr, 1.0, rhs.ptr + (j - 1 + it * ni) * N, s);
            }
        // initial guess (time_integrators.h:96-104)
        for (int b = 0; b < nb; ++b)
          {
            if (cfg.extrapolate)
              STMG_CUDA(cudaMemcpyAsync(x.ptr + b * N, prev_x.ptr, N * 8, cudaMemcpyDeviceToDevice, s));
            else
              STMG_CUDA(cudaMemsetAsync(x.ptr + b * N, 0, N * 8, s));
          }
        const int k = solve(x.ptr, rhs.ptr, s);
        if (its)
          its[slab] = k;
        if (cfg.problem == 2)
          {
            // velocity recovery (time_integrators.h:263-279)
            STMG_CUDA(cudaMemsetAsync(v.ptr, 0, N * nb * 8, s));
            const int ntd = AixB.m;
            for (int it = 0; it < cfg.n_steps; ++it)
              {
                const double *pu = it == 0 ? prev_x.ptr : x.ptr + (it * ntd - 1) * N;
                block_combine(N, AixB, x.ptr + it * ntd * N, v.ptr + it * ntd * N, s);
                if (type == tfe::DG)
                  block_combine(N, AixG, pu, v.ptr + it * ntd * N, s);
                else
                  {
                    // the previous step's last velocity block; it does not
                    // overlap the blocks written for this step
                    const double *pv = it == 0 ? prev_v.ptr : v.ptr + (it * ntd - 1) * N;
                    block_combine(N, AixG, pv, v.ptr + it * ntd * N, s);
                    block_combine(N, AixZ, pu, v.ptr + it * ntd * N, s);
                  }
              }
          }
        if (cfg.rhs_mode == 0)
          accumulate_errors(tq, s);
        time += cfg.n_steps * cfg.tau;
      }
    STMG_CUDA(cudaStreamSynchronize(s));
  }

  // ErrorCalculator::evaluate_error (exact_solution.h:217-299): per step and
  // QGauss(r+1) time point the FE function in time (Lagrange basis over the
  // step's time dofs; cGP takes the previous value as its first node), then
  // the space integrals; sums tau w_q |e|^2 (L2, H1) and the largest |e|.
  void
  SlabSolver::accumulate_errors(const std::vector<double> &tq, cudaStream_t s)
  {
    const auto      type = tfe::Type(cfg.time_type);
    const MeshView &m    = meshes.back()->v;
    std::vector<double> eq, ew, sx, sw;
    tfe::gauss(cfg.time_degree + 1, eq, ew);
    const int nq = cfg.time_degree + 1;
    tfe::gauss(nq, sx, sw);
    ErrTab et{};
    et.nq = nq;
    et.p1 = m.p + 1;
    {
      const FETables     &t = host_tables();
      std::vector<double> xs(t.xs[m.p], t.xs[m.p] + m.p + 1);
      for (int q = 0; q < nq; ++q)
        {
          et.gx[q] = sx[q];
          et.gw[q] = sw[q];
          for (int a = 0; a <= m.p; ++a)
            {
              et.phi[q][a] = tfe::lagrange(xs, a, sx[q]);
              // derivative of the Lagrange polynomial: sum over the dropped factor
              double dv = 0;
              for (int k = 0; k <= m.p; ++k)
                {
                  if (k == a)
                    continue;
                  double term = 1.0 / (xs[a] - xs[k]);
                  for (int l = 0; l <= m.p; ++l)
                    if (l != a && l != k)
                      term *= (sx[q] - xs[l]) / (xs[a] - xs[l]);
                  dv += term;
                }
              et.dphi[q][a] = dv;
            }
        }
    }
    if (!err_buf.ptr)
      {
        err_buf.alloc(std::size_t(3) * m.ncells + 3);
        err_num.alloc(N);
      }
    double *cl2 = err_buf.ptr, *ch1 = cl2 + m.ncells, *cl8 = ch1 + m.ncells, *out = cl8 + m.ncells;
    for (int it = 0; it < cfg.n_steps; ++it)
      for (std::size_t q = 0; q < eq.size(); ++q)
        {
          const double tt = time + cfg.tau * it + eq[q] * cfg.tau;
          STMG_CUDA(cudaMemsetAsync(err_num.ptr, 0, N * 8, s));
          const double *pu = it == 0 ? prev_x.ptr : x.ptr + (ni * it - 1) * N;
          for (std::size_t i = 0; i < tq.size(); ++i)
            {
              const double b = tfe::lagrange(tq, int(i), eq[q]);
              if (b == 0.0)
                continue;
              const double *src = type == tfe::DG ? x.ptr + (ni * it + i) * N : (i == 0 ? pu : x.ptr + (ni * it + i - 1) * N);
              axpby<double>(N, b, src, 1.0, err_num.ptr, s);
            }
          const unsigned nbk = unsigned((m.ncells + 127) / 128);
          if (m.dim == 2)
            err_cell_kernel<2><<<nbk, 128, 0, s>>>(m, et, err_num.ptr, tt, cfg.frequency, cl2, ch1, cl8);
          else
            err_cell_kernel<3><<<nbk, 128, 0, s>>>(m, et, err_num.ptr, tt, cfg.frequency, cl2, ch1, cl8);
          count_launch();
          STMG_CUDA(cudaGetLastError());
          err_reduce_kernel<<<1, 1024, 0, s>>>(m.ncells, cl2, ch1, cl8, out);
          count_launch();
          STMG_CUDA(cudaGetLastError());
          double h[3];
          STMG_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s));
          STMG_CUDA(cudaStreamSynchronize(s));
          err_l2sq += cfg.tau * ew[q] * h[0];
          err_h1sq += cfg.tau * ew[q] * h[1];
          err_l8 = std::max(err_l8, h[2]);
        }
  }

  double
  SlabSolver::gradient(int n_slabs, const double *obs, int checkpoint_every, double *grad, int *its_fwd, int *its_adj,
                       cudaStream_t s)
  {
    STMG_REQUIRE(cfg.problem == 1, STMG_ERR_UNSUPPORTED, "gradient: heat problems only");
    STMG_REQUIRE(n_slabs >= 1 && obs && grad, STMG_ERR_ARG, "gradient: bad arguments");
    wait_snapshot(s);
    Mesh           &fine = *meshes.back();
    STMG_REQUIRE(fine.v.coeff_mode != 2, STMG_ERR_UNSUPPORTED, "gradient: needs a coefficient per cell");
    const long long n    = N * nb;
    const int       k    = checkpoint_every > 0 ? checkpoint_every
                                                : std::max(1, int(std::ceil(std::sqrt(double(n_slabs)))));
    const int       nseg = (n_slabs + k - 1) / k;
    if (!gmgT)
      gmgT = std::make_unique<GMG>(cfg, meshes, blas, true);
    DevBuf<double> O(n), d(n), lam(n), lam_next(n), radj(n), g(fine.v.ncells), ck(std::size_t(nseg) * N),
      U(std::size_t(k) * n), e(N);
    std::vector<double> ck_time(nseg);
    STMG_CUDA(cudaMemsetAsync(g.ptr, 0, fine.v.ncells * 8, s));
    auto load_obs = [&](int slab) {
      STMG_CUDA(cudaMemcpyAsync(O.ptr, obs + std::size_t(slab) * n, n * 8, cudaMemcpyHostToDevice, s));
    };
    auto set_state = [&](const double *u_end, double t) {
      STMG_CUDA(cudaMemcpyAsync(x.ptr + (nb - 1) * N, u_end, N * 8, cudaMemcpyDeviceToDevice, s));
      time = t;
    };
    // forward: checkpoints (end value of the previous slab) and the misfit
    double J = 0;
    for (int slab = 0; slab < n_slabs; ++slab)
      {
        if (slab % k == 0)
          {
            STMG_CUDA(cudaMemcpyAsync(ck.ptr + std::size_t(slab / k) * N, x.ptr + (nb - 1) * N, N * 8,
                                      cudaMemcpyDeviceToDevice, s));
            ck_time[slab / k] = time;
          }
        int it = 0;
        run(1, &it, s);
        if (its_fwd)
          its_fwd[slab] = it;
        load_obs(slab);
        STMG_CUDA(cudaMemcpyAsync(d.ptr, x.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
        axpby<double>(n, -1.0, O.ptr, 1.0, d.ptr, s);
        J += 0.5 * blas.dot<double>(n, d.ptr, d.ptr, s);
      }
    // state after the forward run, restored at the end
    DevBuf<double> x_end(n);
    STMG_CUDA(cudaMemcpyAsync(x_end.ptr, x.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
    const double t_end = time;
    auto         AT    = [&](double *dst, const double *src) {
      NvtxScope r("Tvmult");
      A64->apply(true, src, dst, false, s);
    };
    auto         PT    = [&](double *dst, const double *src, double scale) { gmgT->vmult(dst, src, s, scale); };
    bool         have_next = false;
    for (int seg = nseg - 1; seg >= 0; --seg)
      {
        const int s0 = seg * k, s1 = std::min(n_slabs, s0 + k);
        // recompute the segment's slabs from its checkpoint
        set_state(ck.ptr + std::size_t(seg) * N, ck_time[seg]);
        for (int slab = s0; slab < s1; ++slab)
          {
            run(1, nullptr, s);
            STMG_CUDA(cudaMemcpyAsync(U.ptr + std::size_t(slab - s0) * n, x.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
          }
        for (int slab = s1 - 1; slab >= s0; --slab)
          {
            const double *Us = U.ptr + std::size_t(slab - s0) * n;
            // adjoint rhs: U_s - O_s + E^T R^T lambda_{s+1}
            load_obs(slab);
            STMG_CUDA(cudaMemcpyAsync(radj.ptr, Us, n * 8, cudaMemcpyDeviceToDevice, s));
            axpby<double>(n, -1.0, O.ptr, 1.0, radj.ptr, s);
            if (have_next)
              rhs64->apply(true, lam_next.ptr, radj.ptr + (nb - 1) * N, true, s);
            STMG_CUDA(cudaMemsetAsync(lam.ptr, 0, n * 8, s));
            const int it = gmres->solve(AT, PT, lam.ptr, radj.ptr, cfg.abs_tol, cfg.tol, cfg.max_iter, s);
            if (its_adj)
              its_adj[slab] = it;
            // gradient: lambda_s^T (rK (x) K_c) e(U_{s-1}) - lambda_s^T (Alpha (x) K_c) U_s
            grad_contract(fine, lhsK_, lam.ptr, Us, -1.0, g.ptr, s);
            const double *prev = slab == s0 ? ck.ptr + std::size_t(seg) * N
                                            : U.ptr + std::size_t(slab - 1 - s0) * n + (nb - 1) * N;
            grad_contract(fine, rK_, lam.ptr, prev, 1.0, g.ptr, s);
            std::swap(lam.ptr, lam_next.ptr);
            have_next = true;
          }
      }
    STMG_CUDA(cudaMemcpyAsync(x.ptr, x_end.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
    time = t_end;
    STMG_CUDA(cudaMemcpyAsync(grad, g.ptr, fine.v.ncells * 8, cudaMemcpyDeviceToHost, s));
    STMG_CUDA(cudaStreamSynchronize(s));
    return J;
  }

  void
  SlabSolver::download(double *u, double *vv) const
  {
    if (u)
      STMG_CUDA(cudaMemcpy(u, x.ptr, N * nb * 8, cudaMemcpyDeviceToHost));
    if (vv)
      STMG_CUDA(cudaMemcpy(vv, v.ptr, N * nb * 8, cudaMemcpyDeviceToHost));
  }

  SlabSolver::AsyncCopy::~AsyncCopy()
  {
    // best effort at teardown: no exceptions out of a destructor
    if (stream)
      {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
      }
    for (cudaEvent_t e : {ready, snapped, copied})
      if (e)
        cudaEventDestroy(e);
  }

  void
  SlabSolver::download_async(double *u, double *vv, cudaStream_t s)
  {
    if (!acopy.stream)
      {
        // non-blocking: the legacy default stream must not wait for it
        STMG_CUDA(cudaStreamCreateWithFlags(&acopy.stream, cudaStreamNonBlocking));
        STMG_CUDA(cudaEventCreateWithFlags(&acopy.ready, cudaEventDisableTiming));
        STMG_CUDA(cudaEventCreateWithFlags(&acopy.snapped, cudaEventDisableTiming));
        STMG_CUDA(cudaEventCreateWithFlags(&acopy.copied, cudaEventDisableTiming));
      }
    const std::size_t n = std::size_t(N) * nb;
    if (u && stage_u.n < n)
      stage_u.alloc(n);
    if (vv && stage_v.n < n)
      stage_v.alloc(n);
    // device snapshot after the work queued on s, then the host copies; the
    // copy stream is in order, so a previous host copy out of the staging
    // buffers has finished before they are overwritten
    STMG_CUDA(cudaEventRecord(acopy.ready, s));
    STMG_CUDA(cudaStreamWaitEvent(acopy.stream, acopy.ready, 0));
    if (u)
      STMG_CUDA(cudaMemcpyAsync(stage_u.ptr, x.ptr, n * 8, cudaMemcpyDeviceToDevice, acopy.stream));
    if (vv)
      STMG_CUDA(cudaMemcpyAsync(stage_v.ptr, v.ptr, n * 8, cudaMemcpyDeviceToDevice, acopy.stream));
    STMG_CUDA(cudaEventRecord(acopy.snapped, acopy.stream));
    if (u)
      STMG_CUDA(cudaMemcpyAsync(u, stage_u.ptr, n * 8, cudaMemcpyDeviceToHost, acopy.stream));
    if (vv)
      STMG_CUDA(cudaMemcpyAsync(vv, stage_v.ptr, n * 8, cudaMemcpyDeviceToHost, acopy.stream));
    STMG_CUDA(cudaEventRecord(acopy.copied, acopy.stream));
    acopy.pending = true;
  }

  void
  SlabSolver::wait_snapshot(cudaStream_t s)
  {
    if (acopy.pending)
      STMG_CUDA(cudaStreamWaitEvent(s, acopy.snapped, 0));
  }

  void
  SlabSolver::wait_snapshot_host()
  {
    if (acopy.pending)
      STMG_CUDA(cudaEventSynchronize(acopy.snapped));
  }

  void
  SlabSolver::download_wait()
  {
    if (acopy.pending)
      STMG_CUDA(cudaEventSynchronize(acopy.copied));
  }

} // namespace stmg
