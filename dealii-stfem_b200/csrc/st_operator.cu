// Fused space-time operator dst_j = sum_i A(j,i) K src_i + B(j,i) M src_i
// (the reference's SystemMatrix over two MatrixFreeOperator objects,
// tests/include/operators.h:71-256 and 355-562), one pass over the cells for
// all time blocks at once.
//
// One CTA per tile of cells:
//  A. stage the tile's node brick of every input time block in shared
//     memory (Dirichlet nodes read as zero);
//  B. one thread per (cell, output time dof j): mix the inputs in time at
//     the nodes, a_j = sum_i A(j,i) kappa u_i and b_j = sum_i B(j,i) u_i, and
//     form K a_j + M b_j by register-resident sum factorisation (exact 1-D
//     matrices on cartesian cells, QGauss(p+1) with the Q1 geometry at every
//     quadrature point otherwise);
//  C. gather the cell results per brick node in a fixed order; tile-interior
//     nodes are final and go to dst, brick-shell nodes go to the tile's
//     face slots, summed by the fix-up kernel in a fixed tile order.
// The result is deterministic (no atomics) and dst is written exactly once.
#include <algorithm>
#include <cstring>

#include "kernels_common.cuh"
#include "st_operator.h"

namespace stmg
{
  namespace
  {
    template <int DIM, int P, typename T>
    __device__ __forceinline__ void
    cart_apply(const Cart1D<T> &c, T *a, T *b, T *out)
    {
      constexpr int P1 = P + 1;
      constexpr int ND = Tens<P1, DIM>::ND;
      if constexpr (DIM == 2)
        {
          // K a + M b = Kx (My a) + Mx (Ky a + My b)
          T s[ND];
          sweep<P1, 2, 1, false, false>(c.M[1], a, s);
          sweep<P1, 2, 1, false, false>(c.K[1], a, a);
          sweep<P1, 2, 1, true, false>(c.M[1], b, a);
          sweep<P1, 2, 0, false, false>(c.K[0], s, out);
          sweep<P1, 2, 0, true, false>(c.M[0], a, out);
        }
      else
        {
          // K a + M b = Kx (My Mz a) + Mx (Ky Mz a + My (Kz a + Mz b))
          T s[ND], u[ND];
          sweep<P1, 3, 2, false, false>(c.M[2], a, s);
          sweep<P1, 3, 2, false, false>(c.K[2], a, a);
          sweep<P1, 3, 2, true, false>(c.M[2], b, a);
          sweep<P1, 3, 1, false, false>(c.M[1], s, u);
          sweep<P1, 3, 1, false, false>(c.K[1], s, b);
          sweep<P1, 3, 1, true, false>(c.M[1], a, b);
          sweep<P1, 3, 0, false, false>(c.K[0], u, out);
          sweep<P1, 3, 0, true, false>(c.M[0], b, out);
        }
    }

    // K a + M b on a Q1-mapped cell with QGauss(p+1) and a coefficient per
    // cell or per quadrature point.
    template <int DIM, int P, typename T>
    __device__ __forceinline__ void
    general_apply(const MeshView &m, const QTab<T> &qt, int cx, int cy, int cz, long long cell, T *a, T *b, T *out)
    {
      constexpr int P1 = P + 1;
      constexpr int ND = Tens<P1, DIM>::ND;
      // values at the quadrature points
      sweep<P1, DIM, 0, false, false>(qt.S, a, a);
      sweep<P1, DIM, 1, false, false>(qt.S, a, a);
      sweep<P1, DIM, 0, false, false>(qt.S, b, b);
      sweep<P1, DIM, 1, false, false>(qt.S, b, b);
      if constexpr (DIM == 3)
        {
          sweep<P1, DIM, 2, false, false>(qt.S, a, a);
          sweep<P1, DIM, 2, false, false>(qt.S, b, b);
        }
      // reference gradients by collocation
      T g0[ND], g1[ND], g2[DIM == 3 ? ND : 1];
      sweep<P1, DIM, 0, false, false>(qt.Dq, a, g0);
      sweep<P1, DIM, 1, false, false>(qt.Dq, a, g1);
      if constexpr (DIM == 3)
        sweep<P1, DIM, 2, false, false>(qt.Dq, a, g2);
      T X[1 << DIM][DIM];
      load_corners<DIM>(m, cx, cy, cz, X);
      const T *cq    = nullptr;
      T        kcell = T(1);
      if constexpr (sizeof(T) == 8)
        {
          if (m.coeff_mode == 1)
            kcell = T(m.coeff64[cell]);
          else if (m.coeff_mode == 2)
            cq = reinterpret_cast<const T *>(m.coeff64) + cell * ND;
        }
      else
        {
          if (m.coeff_mode == 1)
            kcell = T(m.coeff32[cell]);
          else if (m.coeff_mode == 2)
            cq = reinterpret_cast<const T *>(m.coeff32) + cell * ND;
        }
#pragma unroll
      for (int q = 0; q < ND; ++q)
        {
          const int qx = q % P1, qy = (q / P1) % P1, qz = q / (P1 * P1);
          T         xi[3] = {qt.gx[qx], qt.gx[qy], DIM == 3 ? qt.gx[qz] : T(0)};
          T         J[DIM][DIM], Ji[DIM][DIM];
          q1_jacobian<DIM>(X, xi, J);
          const T det = det_inv<DIM>(J, Ji);
          T       w   = qt.gw[qx] * qt.gw[qy];
          if constexpr (DIM == 3)
            w *= qt.gw[qz];
          const T JxW = fabs(det) * w;
          const T k   = (cq ? cq[q] : kcell) * JxW;
          // physical gradient Ji^T g, flux = k Ji (Ji^T g)
          T gr[DIM] = {g0[q], g1[q]};
          if constexpr (DIM == 3)
            gr[2] = g2[q];
          T ph[DIM];
#pragma unroll
          for (int i = 0; i < DIM; ++i)
            {
              T s = T(0);
#pragma unroll
              for (int d = 0; d < DIM; ++d)
                s += Ji[d][i] * gr[d];
              ph[i] = k * s;
            }
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            {
              T s = T(0);
#pragma unroll
              for (int i = 0; i < DIM; ++i)
                s += Ji[d][i] * ph[i];
              gr[d] = s;
            }
          g0[q] = gr[0];
          g1[q] = gr[1];
          if constexpr (DIM == 3)
            g2[q] = gr[2];
          b[q] *= JxW;
        }
      // integrate: collocation derivatives transposed, then S^T
      sweep<P1, DIM, 0, true, true>(qt.Dq, g0, b);
      sweep<P1, DIM, 1, true, true>(qt.Dq, g1, b);
      if constexpr (DIM == 3)
        sweep<P1, DIM, 2, true, true>(qt.Dq, g2, b);
      sweep<P1, DIM, 0, false, true>(qt.S, b, b);
      sweep<P1, DIM, 1, false, true>(qt.S, b, b);
      if constexpr (DIM == 3)
        sweep<P1, DIM, 2, false, true>(qt.S, b, out);
      else
#pragma unroll
        for (int q = 0; q < ND; ++q)
          out[q] = b[q];
    }

    template <int DIM, int P, typename T, bool CART>
    __global__ void __launch_bounds__(256)
    st_apply_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeMats<T> tm,
                    const __grid_constant__ Cart1D<T> c1, const __grid_constant__ QTab<T> qt,
                    const T *__restrict__ src, T *__restrict__ dst, T *__restrict__ shell, int add)
    {
      constexpr int P1 = P + 1;
      constexpr int ND = Tens<P1, DIM>::ND;
      extern __shared__ __align__(16) unsigned char smem_raw[];
      T *brick = reinterpret_cast<T *>(smem_raw);

      int t[3], c0[3], tc[3], e[3];
      tile_extents<DIM>(m, tl, blockIdx.x, t, c0, tc, e);
      const int       nb      = e[0] * e[1] * e[2];
      const int       nbmax   = tl.E[0] * tl.E[1] * tl.E[2];
      T              *cellbuf = brick + (long long)tm.nt_in * nbmax;
      const long long N       = m.N;

      // A. brick of every input block
      for (int idx = threadIdx.x; idx < tm.nt_in * nb; idx += blockDim.x)
        {
          const int i = idx / nb, r = idx % nb;
          const int bx = r % e[0], by = (r / e[0]) % e[1], bz = r / (e[0] * e[1]);
          const int gx = c0[0] * P + bx, gy = c0[1] * P + by, gz = c0[2] * P + bz;
          T         v  = T(0);
          if (!is_boundary_node(m, gx, gy, gz))
            v = src[i * N + gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz)];
          brick[i * nb + r] = v;
        }
      __syncthreads();

      // B. per (cell, output time dof)
      const int ncell = tc[0] * tc[1] * tc[2];
      for (int w = threadIdx.x; w < ncell * tm.nt_out; w += blockDim.x)
        {
          const int lc = w / tm.nt_out, j = w % tm.nt_out;
          const int lx = lc % tc[0], ly = (lc / tc[0]) % tc[1], lz = lc / (tc[0] * tc[1]);
          const int cx = c0[0] + lx, cy = c0[1] + ly, cz = c0[2] + lz;
          const long long cell = cx + (long long)m.n[0] * (cy + (long long)m.n[1] * cz);
          T kap = T(1);
          if (CART && m.coeff_mode == 1)
            kap = sizeof(T) == 8 ? T(m.coeff64[cell]) : T(m.coeff32[cell]);
          T a[ND], b[ND];
#pragma unroll
          for (int q = 0; q < ND; ++q)
            a[q] = b[q] = T(0);
          for (int i = 0; i < tm.nt_in; ++i)
            {
              const T al = tm.A[j * tm.nt_in + i] * kap, be = tm.B[j * tm.nt_in + i];
              if (al == T(0) && be == T(0))
                continue;
              const T *br = brick + i * nb + lx * P + e[0] * (ly * P + e[1] * (lz * P));
#pragma unroll
              for (int q = 0; q < ND; ++q)
                {
                  const int qx = q % P1, qy = (q / P1) % P1, qz = q / (P1 * P1);
                  const T   u  = br[qx + e[0] * (qy + e[1] * qz)];
                  a[q] += al * u;
                  b[q] += be * u;
                }
            }
          T out[ND];
          if constexpr (CART)
            cart_apply<DIM, P>(c1, a, b, out);
          else
            general_apply<DIM, P>(m, qt, cx, cy, cz, cell, a, b, out);
          T *cb = cellbuf + (long long)(lc * tm.nt_out + j) * ND;
#pragma unroll
          for (int q = 0; q < ND; ++q)
            cb[q] = out[q];
        }
      __syncthreads();

      // C. gather per brick node and write
      for (int idx = threadIdx.x; idx < tm.nt_out * nb; idx += blockDim.x)
        {
          const int j = idx / nb, r = idx % nb;
          const int b3[3] = {r % e[0], (r / e[0]) % e[1], r / (e[0] * e[1])};
          int       lc0[3], nlc[3];
#pragma unroll
          for (int d = 0; d < 3; ++d)
            {
              if (d >= DIM)
                {
                  lc0[d] = 0;
                  nlc[d] = 1;
                  continue;
                }
              const int q = b3[d] / P, rem = b3[d] % P;
              if (rem == 0 && q > 0 && q < tc[d])
                lc0[d] = q - 1, nlc[d] = 2;
              else
                lc0[d] = min(q, tc[d] - 1), nlc[d] = 1;
            }
          T s = T(0);
          for (int kz = 0; kz < nlc[2]; ++kz)
            for (int ky = 0; ky < nlc[1]; ++ky)
              for (int kx = 0; kx < nlc[0]; ++kx)
                {
                  const int cx = lc0[0] + kx, cy = lc0[1] + ky, cz = lc0[2] + kz;
                  const int lc = cx + tc[0] * (cy + tc[1] * cz);
                  const int ax = b3[0] - cx * P, ay = b3[1] - cy * P, az = DIM == 3 ? b3[2] - cz * P : 0;
                  s += cellbuf[(long long)(lc * tm.nt_out + j) * ND + ax + P1 * (ay + P1 * az)];
                }
          bool interior = b3[0] > 0 && b3[0] < e[0] - 1 && b3[1] > 0 && b3[1] < e[1] - 1;
          if (DIM == 3)
            interior = interior && b3[2] > 0 && b3[2] < e[2] - 1;
          if (interior)
            {
              const long long g = (c0[0] * P + b3[0]) + (long long)m.nn[0] * ((c0[1] * P + b3[1]) +
                                                                                 (long long)m.nn[1] * (c0[2] * P + b3[2]));
              T *d = dst + j * N + g;
              *d   = add ? *d + s : s;
            }
          else
            shell[((long long)blockIdx.x * tm.nt_out + j) * tl.tile_stride + shell_slot<DIM>(tl, e, b3[0], b3[1], b3[2])] = s;
        }
    }

    // Fix-up: nodes on tile boundaries (and Dirichlet nodes) get the sum of
    // their tiles' shell contributions in fixed order.
    template <int DIM, typename T>
    __global__ void
    shell_fixup_kernel(const MeshView m, const Tiling tl, int nt, const T *__restrict__ shell, T *__restrict__ dst, int add)
    {
      const long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (node >= m.N)
        return;
      const int g[3] = {int(node % m.nn[0]), int((node / m.nn[0]) % m.nn[1]), int(node / ((long long)m.nn[0] * m.nn[1]))};
      const bool bd = is_boundary_node(m, g[0], g[1], g[2]);
      bool       on = false;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        on = on || (g[d] % (tl.T[d] * m.p) == 0);
      if (!bd && !on)
        return;
      for (int j = 0; j < nt; ++j)
        {
          T *d = dst + j * m.N + node;
          if (bd)
            {
              if (!add)
                *d = T(0);
              continue;
            }
          const T s = shell_sum<DIM, T>(m, tl, shell, nt, j, g);
          *d        = add ? *d + s : s;
        }
    }

    template <int DIM, int P, typename T>
    void
    launch_dp(const StOperator &op, bool transpose, const T *src, T *dst, T *shell, bool add, cudaStream_t s)
    {
      const TimeMats<T> &tm   = transpose ? op.tmT<T>() : op.tm<T>();
      const MeshView    &m    = op.mesh->v;
      const Tiling      &tl   = transpose ? op.tilingT : op.tiling;
      const std::size_t  smem = op.smem_bytes(tl, tm.nt_in, tm.nt_out, sizeof(T));
      auto               kern = m.cartesian ? st_apply_kernel<DIM, P, T, true> : st_apply_kernel<DIM, P, T, false>;
      STMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      kern<<<unsigned(tl.n_tiles), 256, smem, s>>>(m, tl, tm, op.cart<T>(), op.qtab<T>(), src, dst, shell, add ? 1 : 0);
      count_launch();
      STMG_CUDA(cudaGetLastError());
      const unsigned nb = unsigned((m.N + 255) / 256);
      shell_fixup_kernel<DIM, T><<<nb, 256, 0, s>>>(m, tl, tm.nt_out, shell, dst, add ? 1 : 0);
      count_launch();
      STMG_CUDA(cudaGetLastError());
    }

    template <typename T>
    void
    launch(const StOperator &op, bool transpose, const T *src, T *dst, T *shell, bool add, cudaStream_t s)
    {
      const int dim = op.mesh->v.dim, p = op.mesh->v.p;
#define STMG_CASE(D, PP)                                                                                 \
  if (dim == D && p == PP)                                                                               \
    return launch_dp<D, PP, T>(op, transpose, src, dst, shell, add, s);
      STMG_CASE(2, 1) STMG_CASE(2, 2) STMG_CASE(2, 3) STMG_CASE(2, 4) STMG_CASE(2, 5)
      STMG_CASE(3, 1) STMG_CASE(3, 2) STMG_CASE(3, 3) STMG_CASE(3, 4)
#undef STMG_CASE
      throw Error(STMG_ERR_UNSUPPORTED, "operator: unsupported dim/degree");
    }

    template <typename T>
    void
    fill_mats(TimeMats<T> &tm, int nt_out, int nt_in, const std::vector<double> &A, const std::vector<double> &B,
              bool transpose)
    {
      std::memset(&tm, 0, sizeof(tm));
      tm.nt_out = transpose ? nt_in : nt_out;
      tm.nt_in  = transpose ? nt_out : nt_in;
      for (int j = 0; j < nt_out; ++j)
        for (int i = 0; i < nt_in; ++i)
          {
            const int k = transpose ? i * nt_out + j : j * nt_in + i;
            tm.A[k]     = T(A[j * nt_in + i]);
            tm.B[k]     = T(B[j * nt_in + i]);
          }
    }

    template <typename T>
    Cart1D<T>
    make_cart(const MeshView &m)
    {
      Cart1D<T>       c{};
      const FETables &t = host_tables();
      const int       n = m.p + 1;
      for (int d = 0; d < 3; ++d)
        for (int a = 0; a < n; ++a)
          for (int b = 0; b < n; ++b)
            {
              c.M[d][a * n + b] = T(t.M1[m.p][a][b] * m.h[d]);
              c.K[d][a * n + b] = T(t.K1[m.p][a][b] / m.h[d]);
            }
      return c;
    }
  } // namespace

  std::size_t
  StOperator::smem_bytes(const Tiling &tl, int nt_in_, int nt_out_, std::size_t elem) const
  {
    const int nd = mesh->nd;
    return elem * (std::size_t(nt_in_) * tl.E[0] * tl.E[1] * tl.E[2] +
                   std::size_t(tl.T[0]) * tl.T[1] * tl.T[2] * nt_out_ * nd);
  }

  Tiling
  StOperator::choose_tiling(int nt_in_, int nt_out_) const
  {
    const MeshView  &m     = mesh->v;
    const std::size_t elem = dtype == STMG_F64 ? 8 : 4;
    const std::size_t budget = 100 * 1024;
    static const int cand3[][3] = {{8, 8, 4}, {8, 4, 4}, {4, 4, 4}, {4, 4, 2}, {4, 2, 2}, {2, 2, 2}, {2, 2, 1}, {2, 1, 1}, {1, 1, 1}};
    static const int cand2[][3] = {{16, 16, 1}, {16, 8, 1}, {8, 8, 1}, {8, 4, 1}, {4, 4, 1}, {4, 2, 1}, {2, 2, 1}, {2, 1, 1}, {1, 1, 1}};
    const int(*cand)[3] = m.dim == 3 ? cand3 : cand2;
    for (int k = 0; k < 9; ++k)
      {
        Tiling t = make_tiling(m, cand[k]);
        if (smem_bytes(t, nt_in_, nt_out_, elem) <= budget)
          return t;
      }
    throw Error(STMG_ERR_UNSUPPORTED, "operator: time blocks do not fit in shared memory");
  }

  StOperator::StOperator(Mesh *mesh_, int nt_out_, int nt_in_, const double *A_, const double *B_, int dtype_)
    : mesh(mesh_)
    , nt_out(nt_out_)
    , nt_in(nt_in_)
    , dtype(dtype_)
  {
    STMG_REQUIRE(nt_out >= 1 && nt_out <= MAX_NT && nt_in >= 1 && nt_in <= MAX_NT, STMG_ERR_ARG,
                 "operator: time dimensions must be 1..16");
    STMG_REQUIRE(dtype == STMG_F64 || dtype == STMG_F32, STMG_ERR_ARG, "operator: dtype must be F64 or F32");
    A.assign(A_, A_ + nt_out * nt_in);
    B.assign(B_, B_ + nt_out * nt_in);
    fill_mats(tm64, nt_out, nt_in, A, B, false);
    fill_mats(tm32, nt_out, nt_in, A, B, false);
    fill_mats(tmT64, nt_out, nt_in, A, B, true);
    fill_mats(tmT32, nt_out, nt_in, A, B, true);
    cart64 = make_cart<double>(mesh->v);
    cart32 = make_cart<float>(mesh->v);
    qtab64 = make_qtab<double>(mesh->v.p);
    qtab32 = make_qtab<float>(mesh->v.p);
    tiling  = choose_tiling(nt_in, nt_out);
    tilingT = choose_tiling(nt_out, nt_in);
    const std::size_t elem = dtype == STMG_F64 ? 8 : 4;
    const std::size_t n1   = std::size_t(tiling.n_tiles) * nt_out * tiling.tile_stride;
    const std::size_t n2   = std::size_t(tilingT.n_tiles) * nt_in * tilingT.tile_stride;
    shell.alloc(std::max(n1, n2) * elem);
  }

  void
  StOperator::apply(bool transpose, const void *src, void *dst, bool add, cudaStream_t s) const
  {
    STMG_REQUIRE(src && dst, STMG_ERR_ARG, "operator: null vector");
    if (dtype == STMG_F64)
      launch<double>(*this, transpose, static_cast<const double *>(src), static_cast<double *>(dst),
                     reinterpret_cast<double *>(shell.ptr), add, s);
    else
      launch<float>(*this, transpose, static_cast<const float *>(src), static_cast<float *>(dst),
                    reinterpret_cast<float *>(shell.ptr), add, s);
  }
} // namespace stmg
