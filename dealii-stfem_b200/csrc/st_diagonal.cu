// Diagonal of the space-time operator (SystemMatrix::get_matrix_diagonal and
// get_matrix_diagonal_inverse, tests/include/operators.h:188-215, over the
// diagonals of K and M that MatrixFreeOperator::compute_diagonal builds,
// operators.h:467-485).
//
// The spatial diagonals come from the operator kernels by probing: nodes
// whose coordinates agree modulo p+1 in every direction share no cell, so
// with e_c the indicator of one such class, (K e_c)_i = K_ii for every i in
// the class. (p+1)^dim applies of K and of M give both diagonals exactly (up
// to the kernels' rounding). Constrained (Dirichlet) rows get 1, the value
// deal.II's matrix-free diagonal gives constrained dofs.
#include <cmath>
#include <limits>

#include "kernels_common.cuh"
#include "st_operator.h"

namespace stmg
{
  namespace
  {
    __device__ __forceinline__ void
    node_coords(const MeshView &m, long long i, int (&g)[3])
    {
      g[0] = int(i % m.nn[0]);
      g[1] = int((i / m.nn[0]) % m.nn[1]);
      g[2] = int(i / ((long long)m.nn[0] * m.nn[1]));
    }

    __device__ __forceinline__ int
    node_class(const MeshView &m, const int (&g)[3])
    {
      const int q = m.p + 1;
      int       c = g[0] % q;
      if (m.dim > 1)
        c += q * (g[1] % q);
      if (m.dim > 2)
        c += q * q * (g[2] % q);
      return c;
    }

    // e = indicator of the interior nodes of class c
    __global__ void
    probe_kernel(const MeshView m, int c, double *__restrict__ e)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m.N; i += (long long)gridDim.x * blockDim.x)
        {
          int g[3];
          node_coords(m, i, g);
          e[i] = (node_class(m, g) == c && !is_boundary_node(m, g[0], g[1], g[2])) ? 1.0 : 0.0;
        }
    }

    // d_i = (A e)_i for the nodes of class c; constrained rows 1
    __global__ void
    gather_kernel(const MeshView m, int c, const double *__restrict__ Ae, double *__restrict__ d)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m.N; i += (long long)gridDim.x * blockDim.x)
        {
          int g[3];
          node_coords(m, i, g);
          if (node_class(m, g) != c)
            continue;
          d[i] = is_boundary_node(m, g[0], g[1], g[2]) ? 1.0 : Ae[i];
        }
    }

    struct DiagCoef
    {
      double a[MAX_NT], b[MAX_NT]; // Alpha(i,i), Beta(i,i)
    };

    // block i: a_i dK + b_i dM (diagonal) or dK^+ / a_i + dM^+ / b_i
    // (inverse, with x^+ = 1/x if |x| > tol else 1), as the reference
    // composes the space-time blocks
    template <typename T>
    __global__ void
    compose_kernel(long long N, int nt, const double *__restrict__ dK, const double *__restrict__ dM,
                   const __grid_constant__ DiagCoef c, int inverse, double tol, T *__restrict__ dst)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        {
          const double k = dK[i], mm = dM[i];
          for (int j = 0; j < nt; ++j)
            {
              double v;
              if (inverse)
                {
                  const double ki = std::fabs(k) > tol ? 1.0 / k : 1.0;
                  const double mi = std::fabs(mm) > tol ? 1.0 / mm : 1.0;
                  v               = ki / c.a[j] + mi / c.b[j];
                }
              else
                v = c.a[j] * k + c.b[j] * mm;
              dst[j * N + i] = T(v);
            }
        }
    }

    unsigned
    grid_n(long long n)
    {
      const long long b = (n + 255) / 256;
      return unsigned(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
    }
  } // namespace

  void
  spatial_diagonals(Mesh *mesh, double *dK, double *dM, cudaStream_t s)
  {
    const MeshView &m  = mesh->v;
    const double    one = 1.0, zero = 0.0;
    StOperator      K(mesh, 1, 1, &one, &zero, STMG_F64), M(mesh, 1, 1, &zero, &one, STMG_F64);
    DevBuf<double>  e(m.N), Ae(m.N);
    int             classes = 1;
    for (int d = 0; d < m.dim; ++d)
      classes *= m.p + 1;
    for (int c = 0; c < classes; ++c)
      {
        probe_kernel<<<grid_n(m.N), 256, 0, s>>>(m, c, e.ptr);
        count_launch();
        STMG_CUDA(cudaGetLastError());
        K.apply(false, e.ptr, Ae.ptr, false, s);
        gather_kernel<<<grid_n(m.N), 256, 0, s>>>(m, c, Ae.ptr, dK);
        count_launch();
        STMG_CUDA(cudaGetLastError());
        M.apply(false, e.ptr, Ae.ptr, false, s);
        gather_kernel<<<grid_n(m.N), 256, 0, s>>>(m, c, Ae.ptr, dM);
        count_launch();
        STMG_CUDA(cudaGetLastError());
      }
    STMG_CUDA(cudaStreamSynchronize(s));
  }

  void
  StOperator::diagonal(bool inverse, void *dst, cudaStream_t s) const
  {
    STMG_REQUIRE(nt_in == nt_out, STMG_ERR_SHAPE, "operator: the diagonal needs a square time coupling");
    STMG_REQUIRE(dst, STMG_ERR_ARG, "operator: null vector");
    const long long N = mesh->v.N;
    if (!diag_K.ptr)
      {
        diag_K.alloc(N);
        diag_M.alloc(N);
        spatial_diagonals(mesh, diag_K.ptr, diag_M.ptr, s);
      }
    DiagCoef c{};
    for (int j = 0; j < nt_out; ++j)
      {
        c.a[j] = A[j * nt_in + j];
        c.b[j] = B[j * nt_in + j];
      }
    // MatrixFreeOperator::compute_diagonal's tolerance: sqrt of the
    // operator's Number epsilon
    const double tol = dtype == STMG_F64 ? std::sqrt(std::numeric_limits<double>::epsilon())
                                         : std::sqrt(double(std::numeric_limits<float>::epsilon()));
    if (dtype == STMG_F64)
      compose_kernel<double><<<grid_n(N), 256, 0, s>>>(N, nt_out, diag_K.ptr, diag_M.ptr, c, inverse ? 1 : 0, tol,
                                                      static_cast<double *>(dst));
    else
      compose_kernel<float><<<grid_n(N), 256, 0, s>>>(N, nt_out, diag_K.ptr, diag_M.ptr, c, inverse ? 1 : 0, tol,
                                                     static_cast<float *>(dst));
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }
} // namespace stmg
