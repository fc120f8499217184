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
#include <mutex>
#include <string>

#include "st_operator.h"
#include "tile_ops.cuh"

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

    // K a + M b on an axis-parallel box cell (Jacobian diag(h)) with a
    // coefficient per quadrature point: general_apply with the geometry
    // folded into per-direction constants.
    template <int DIM, int P, typename T>
    __device__ __forceinline__ void
    box_apply(const MeshView &m, const QTab<T> &qt, long long cell, T *a, T *b, T *out)
    {
      constexpr int P1 = P + 1;
      constexpr int ND = Tens<P1, DIM>::ND;
      sweep<P1, DIM, 0, false, false>(qt.S, a, a);
      sweep<P1, DIM, 1, false, false>(qt.S, a, a);
      sweep<P1, DIM, 0, false, false>(qt.S, b, b);
      sweep<P1, DIM, 1, false, false>(qt.S, b, b);
      if constexpr (DIM == 3)
        {
          sweep<P1, DIM, 2, false, false>(qt.S, a, a);
          sweep<P1, DIM, 2, false, false>(qt.S, b, b);
        }
      T g0[ND], g1[ND], g2[DIM == 3 ? ND : 1];
      sweep<P1, DIM, 0, false, false>(qt.Dq, a, g0);
      sweep<P1, DIM, 1, false, false>(qt.Dq, a, g1);
      if constexpr (DIM == 3)
        sweep<P1, DIM, 2, false, false>(qt.Dq, a, g2);
      T det = T(m.h[0]) * T(m.h[1]);
      if constexpr (DIM == 3)
        det *= T(m.h[2]);
      const T ih0 = T(1) / (T(m.h[0]) * T(m.h[0])), ih1 = T(1) / (T(m.h[1]) * T(m.h[1]));
      const T ih2 = DIM == 3 ? T(1) / (T(m.h[2]) * T(m.h[2])) : T(0);
      const T *cq = m.coeff_mode == 2 ? (sizeof(T) == 8 ? reinterpret_cast<const T *>(m.coeff64)
                                                         : reinterpret_cast<const T *>(m.coeff32)) +
                                          cell * ND
                                      : nullptr;
      const T kcell = m.coeff_mode == 1 ? (sizeof(T) == 8 ? T(m.coeff64[cell]) : T(m.coeff32[cell])) : T(1);
#pragma unroll
      for (int q = 0; q < ND; ++q)
        {
          const int qx = q % P1, qy = (q / P1) % P1, qz = q / (P1 * P1);
          T         w  = qt.gw[qx] * qt.gw[qy];
          if constexpr (DIM == 3)
            w *= qt.gw[qz];
          const T JxW = det * w;
          const T k   = (cq ? cq[q] : kcell) * JxW;
          g0[q] *= k * ih0;
          g1[q] *= k * ih1;
          if constexpr (DIM == 3)
            g2[q] *= k * ih2;
          b[q] *= JxW;
        }
      sweep<P1, DIM, 0, true, true>(qt.Dq, g0, b);
      sweep<P1, DIM, 1, true, true>(qt.Dq, g1, b);
      if constexpr (DIM == 3)
        sweep<P1, DIM, 2, true, true>(qt.Dq, g2, b);
      sweep<P1, DIM, 0, false, true>(qt.S, b, b);
      if constexpr (DIM == 3)
        {
          sweep<P1, DIM, 1, false, true>(qt.S, b, b);
          sweep<P1, DIM, 2, false, true>(qt.S, b, out);
        }
      else
        sweep<P1, DIM, 1, false, true>(qt.S, b, out);
    }

    // MODE 1: cartesian cells, coefficient per cell (cart_apply); 2: box
    // cells, coefficient per quadrature point (box_apply); 0: general
    template <int DIM, int P, typename T, int MODE, int TX, int TY, int TZ>
    __global__ void __launch_bounds__(256, (sizeof(T) == 4 && MODE == 1) ? 2 : 1)
    st_apply_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeMats<T> tm,
                    const __grid_constant__ Cart1D<T> c1, const __grid_constant__ QTab<T> qt,
                    const T *__restrict__ src, T *__restrict__ dst, T *__restrict__ shell, const OutMode<T> om)
    {
      using S          = TileShape<DIM, P, TX, TY, TZ>;
      constexpr int ND = S::ND;
      extern __shared__ __align__(16) unsigned char smem_raw[];
      const int nbuf    = max(tm.nt_in, tm.nt_out) * S::NB;
      T        *bricks[2] = {reinterpret_cast<T *>(smem_raw), reinterpret_cast<T *>(smem_raw) + nbuf};
      T        *cellbuf   = bricks[1] + nbuf;
      long long tile      = blockIdx.x;
      int       t[3], c0[3], tc[3], e[3];
      if (tile < tl.n_tiles)
        {
          tile_extents<DIM>(m, tl, tile, t, c0, tc, e);
          load_brick<S>(bricks[0], src, m, tm.nt_in, c0, e);
        }
      cp_async_commit();
      for (int buf = 0; tile < tl.n_tiles; tile += gridDim.x, buf ^= 1)
        {
          tile_extents<DIM>(m, tl, tile, t, c0, tc, e);
          const long long next = tile + gridDim.x;
          if (next < tl.n_tiles)
            {
              int nt3[3], nc0[3], ntc[3], ne[3];
              tile_extents<DIM>(m, tl, next, nt3, nc0, ntc, ne);
              load_brick<S>(bricks[buf ^ 1], src, m, tm.nt_in, nc0, ne);
            }
          cp_async_commit();
          cp_async_wait<1>();
          __syncthreads();

          // B. per (output time dof, cell): K a_j + M b_j into cellbuf
          const T *brick = bricks[buf];
          for (int w = threadIdx.x; w < tm.nt_out * S::TC; w += blockDim.x)
            {
              const int j = w / S::TC, lc = w - j * S::TC;
              const int lx = lc % TX, ly = (lc / TX) % TY, lz = lc / (TX * TY);
              if (lx >= tc[0] || ly >= tc[1] || lz >= tc[2])
                continue;
              const int cx = c0[0] + lx, cy = c0[1] + ly, cz = c0[2] + lz;
              const long long cell = cx + (long long)m.n[0] * (cy + (long long)m.n[1] * cz);
              T kap = T(1);
              if (MODE == 1 && m.coeff_mode == 1)
                kap = sizeof(T) == 8 ? T(m.coeff64[cell]) : T(m.coeff32[cell]);
              T a[ND], b[ND];
#pragma unroll
              for (int q = 0; q < ND; ++q)
                a[q] = b[q] = T(0);
              const T *br0 = brick + lx * P + S::E0 * (ly * P + S::E1 * (lz * P));
              for (int i = 0; i < tm.nt_in; ++i)
                {
                  const T  al = tm.A[j * tm.nt_in + i] * kap, be = tm.B[j * tm.nt_in + i];
                  const T *br = br0 + i * S::NB;
                  if (al != T(0))
#pragma unroll
                    for (int q = 0; q < ND; ++q)
                      a[q] += al * br[S::offset(q)];
                  if (be != T(0))
#pragma unroll
                    for (int q = 0; q < ND; ++q)
                      b[q] += be * br[S::offset(q)];
                }
              T out[ND];
              if constexpr (MODE == 1)
                cart_apply<DIM, P>(c1, a, b, out);
              else if constexpr (MODE == 2)
                box_apply<DIM, P>(m, qt, cell, a, b, out);
              else
                general_apply<DIM, P>(m, qt, cx, cy, cz, cell, a, b, out);
              T *cb = cellbuf + (j * S::TC + lc) * ND;
#pragma unroll
              for (int q = 0; q < ND; ++q)
                cb[q] = out[q];
            }
          __syncthreads();
          // C. coloured scatter into the output brick (the current input
          // brick's buffer, no longer read), D. write out
          T *ob = bricks[buf];
          scatter_cells<S, DIM, T>(cellbuf, ob, tm.nt_out, tc);
          write_brick<S, DIM, T, false>(ob, m, tl, tile, tm.nt_out, c0, e, dst, shell, om);
          __syncthreads();
        }
      cp_async_wait<0>();
    }

    // compile-time tile shape per (dim, degree, precision); the fallback
    // shape serves time dimensions whose bricks do not fit the main one
    template <int DIM, int P, typename T, bool BIG>
    struct OpShape
    {
      static constexpr int TX = DIM == 2 ? (P <= 2 ? (BIG ? 16 : 4) : (P <= 4 ? (BIG ? 8 : 2) : (BIG ? 4 : 1)))
                                         : (P == 1 ? (BIG ? 8 : 2) : (P == 2 ? (BIG ? (sizeof(T) == 4 ? 8 : 4) : 2) : (BIG ? 4 : 1)));
      static constexpr int TY = DIM == 2 ? TX : (P == 1 ? TX : (P == 2 ? (BIG ? 4 : 2) : (BIG ? (P == 3 ? 4 : 2) : 1)));
      static constexpr int TZ = DIM == 2 ? 1 : (P == 1 ? TX : (P == 2 ? (BIG ? 4 : 2) : (BIG ? 2 : 1)));
    };

    template <int DIM, int P, typename T, bool BIG>
    void
    launch_shape(const StOperator &op, const TimeMats<T> &tm, const T *src, T *dst, T *shell, const OutMode<T> &om,
                 const Tiling &tl, std::size_t smem, cudaStream_t s)
    {
      using Sh = OpShape<DIM, P, T, BIG>;
      const MeshView &m    = op.mesh->v;
      auto            kern = m.cartesian ? st_apply_kernel<DIM, P, T, 1, Sh::TX, Sh::TY, Sh::TZ>
                             : (m.box ? st_apply_kernel<DIM, P, T, 2, Sh::TX, Sh::TY, Sh::TZ>
                                      : st_apply_kernel<DIM, P, T, 0, Sh::TX, Sh::TY, Sh::TZ>);
      const unsigned  grid = persistent_grid(reinterpret_cast<const void *>(kern), 256, smem, tl.n_tiles);
      kern<<<grid, 256, smem, s>>>(m, tl, tm, op.cart<T>(), op.qtab<T>(), src, dst, shell, om);
      count_launch();
      STMG_CUDA(cudaGetLastError());
      if (tl.n_tiles > 1)
        launch_plane_fixup<DIM, T, false>(m, tl, tm.nt_out, shell, dst, om, s);
    }

    template <int DIM, int P, typename T>
    void
    launch_dp(const StOperator &op, bool transpose, const T *src, T *dst, T *shell, const OutMode<T> &om,
              cudaStream_t s)
    {
      const TimeMats<T> &tm  = transpose ? op.tmT<T>() : op.tm<T>();
      const bool         big = transpose ? op.bigT : op.big;
      const Tiling      &tl  = transpose ? op.tilingT : op.tiling;
      const std::size_t  smem = op.smem_bytes(transpose ? op.shpT : op.shp, tm.nt_in, tm.nt_out, sizeof(T));
      if (big)
        launch_shape<DIM, P, T, true>(op, tm, src, dst, shell, om, tl, smem, s);
      else
        launch_shape<DIM, P, T, false>(op, tm, src, dst, shell, om, tl, smem, s);
    }

    template <typename T>
    void
    launch(const StOperator &op, bool transpose, const T *src, T *dst, T *shell, const OutMode<T> &om, cudaStream_t s)
    {
      const int dim = op.mesh->v.dim, p = op.mesh->v.p;
#define STMG_CASE(D, PP)                                                                                 \
  if (dim == D && p == PP)                                                                               \
    return launch_dp<D, PP, T>(op, transpose, src, dst, shell, om, s);
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

  namespace
  {
    template <typename T>
    void
    shape_of(int dim, int p, bool big, int *T3)
    {
#define STMG_SH(D, PP)                                                                                   \
  if (dim == D && p == PP)                                                                               \
    {                                                                                                    \
      if (big)                                                                                           \
        T3[0] = OpShape<D, PP, T, true>::TX, T3[1] = OpShape<D, PP, T, true>::TY, T3[2] = OpShape<D, PP, T, true>::TZ; \
      else                                                                                               \
        T3[0] = OpShape<D, PP, T, false>::TX, T3[1] = OpShape<D, PP, T, false>::TY, T3[2] = OpShape<D, PP, T, false>::TZ; \
      return;                                                                                            \
    }
      STMG_SH(2, 1) STMG_SH(2, 2) STMG_SH(2, 3) STMG_SH(2, 4) STMG_SH(2, 5)
      STMG_SH(3, 1) STMG_SH(3, 2) STMG_SH(3, 3) STMG_SH(3, 4)
#undef STMG_SH
      throw Error(STMG_ERR_UNSUPPORTED, "operator: unsupported dim/degree");
    }
  } // namespace

  std::size_t
  StOperator::smem_bytes(const int *shape, int nt_in_, int nt_out_, std::size_t elem) const
  {
    // two bricks (each holding the larger of the input and output blocks)
    // and the per-cell results, for the compile-time tile shape
    const int         p = mesh->v.p, dim = mesh->v.dim;
    const std::size_t nb = std::size_t(shape[0] * p + 1) * (shape[1] * p + 1) * (dim == 3 ? shape[2] * p + 1 : 1);
    const std::size_t tc = std::size_t(shape[0]) * shape[1] * (dim == 3 ? shape[2] : 1);
    return elem * (2 * std::size_t(std::max(nt_in_, nt_out_)) * nb + tc * nt_out_ * mesh->nd);
  }

  Tiling
  StOperator::choose_tiling(int nt_in_, int nt_out_, bool &big_out, int *shape) const
  {
    const std::size_t elem   = dtype == STMG_F64 ? 8 : 4;
    const std::size_t budget = 200 * 1024;
    for (bool big : {true, false})
      {
        int T3[3];
        if (dtype == STMG_F64)
          shape_of<double>(mesh->v.dim, mesh->v.p, big, T3);
        else
          shape_of<float>(mesh->v.dim, mesh->v.p, big, T3);
        if (smem_bytes(T3, nt_in_, nt_out_, elem) <= budget)
          {
            // on small meshes the big tiles leave SMs idle: prefer the small
            // shape when the big one yields fewer than two tiles per SM
            if (big && make_tiling(mesh->v, T3).n_tiles < 2ll * sm_count())
              {
                int t3[3];
                if (dtype == STMG_F64)
                  shape_of<double>(mesh->v.dim, mesh->v.p, false, t3);
                else
                  shape_of<float>(mesh->v.dim, mesh->v.p, false, t3);
                if (smem_bytes(t3, nt_in_, nt_out_, elem) <= budget)
                  continue;
              }
            big_out = big;
            for (int d = 0; d < 3; ++d)
              shape[d] = T3[d];
            return make_tiling(mesh->v, T3);
          }
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
    tiling  = choose_tiling(nt_in, nt_out, big, shp);
    tilingT = choose_tiling(nt_out, nt_in, bigT, shpT);
    const std::size_t elem = dtype == STMG_F64 ? 8 : 4;
    const std::size_t n1   = std::size_t(tiling.n_tiles) * nt_out * tiling.tile_stride;
    const std::size_t n2   = std::size_t(tilingT.n_tiles) * nt_in * tilingT.tile_stride;
    shell.alloc(std::max(n1, n2) * elem);
  }

  void
  StOperator::apply(bool transpose, const void *src, void *dst, bool add, cudaStream_t s) const
  {
    apply_ex(transpose, src, dst, 1.0, add ? 1.0 : 0.0, nullptr, s);
  }

  void
  StOperator::apply_ex(bool transpose, const void *src, void *dst, double alpha, double beta, const void *rhs,
                       cudaStream_t s) const
  {
    STMG_REQUIRE(src && dst, STMG_ERR_ARG, "operator: null vector");
    if (dtype == STMG_F64)
      {
        const OutMode<double> om{alpha, beta, static_cast<const double *>(rhs)};
        launch<double>(*this, transpose, static_cast<const double *>(src), static_cast<double *>(dst),
                       reinterpret_cast<double *>(shell.ptr), om, s);
      }
    else
      {
        const OutMode<float> om{float(alpha), float(beta), static_cast<const float *>(rhs)};
        launch<float>(*this, transpose, static_cast<const float *>(src), static_cast<float *>(dst),
                      reinterpret_cast<float *>(shell.ptr), om, s);
      }
  }
} // namespace stmg

// ---------------------------------------------------------------------------
// Operator apply that allocates no device memory. The only scratch the
// apply needs, the tiles' face slots, lives in one fixed array of this file's
// device image, so every GPU that loads the library holds these bytes until
// the process exits. Calls share the array: two calls whose kernels overlap
// on the GPU (different streams, or different host threads on one device)
// race on it. Nothing in it has to start at zero: every face slot the fix-up
// reads is written by its tile earlier in the same call.
namespace stmg
{
  constexpr std::size_t NOALLOC_SCRATCH_BYTES = std::size_t(16) << 20; // 16 MiB

  static __device__ __align__(256) unsigned char noalloc_scratch[NOALLOC_SCRATCH_BYTES];

  namespace
  {
    constexpr int MAX_DEVICES = 64;
    std::mutex    scratch_mutex;
    void         *scratch_device_ptr[MAX_DEVICES] = {};

    // Device address of noalloc_scratch on the current device, looked up on
    // the first call per device (host code must not pass the array's name
    // to a kernel: on the host it is only a stand-in for the symbol).
    void *
    scratch_address()
    {
      int dev = 0;
      STMG_CUDA(cudaGetDevice(&dev));
      STMG_REQUIRE(dev >= 0 && dev < MAX_DEVICES, STMG_ERR_CUDA, "op_vmult_box_noalloc: device ordinal out of range");
      std::lock_guard<std::mutex> lock(scratch_mutex);
      if (!scratch_device_ptr[dev])
        {
          void             *p = nullptr;
          const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
          if (e != cudaSuccess || !p)
            throw Error(STMG_ERR_CUDA, std::string("op_vmult_box_noalloc: cudaGetSymbolAddress of the scratch array: ") +
                                         cudaGetErrorString(e));
          scratch_device_ptr[dev] = p;
        }
      return scratch_device_ptr[dev];
    }

    // the tiling StOperator::choose_tiling picks for these sizes
    template <typename T>
    Tiling
    box_tiling(const MeshView &m, int nd, int nt_in, int nt_out, bool &big_out)
    {
      const std::size_t budget = 200 * 1024;
      auto              smem   = [&](const int *sh) {
        const std::size_t nb = std::size_t(sh[0] * m.p + 1) * (sh[1] * m.p + 1) * (m.dim == 3 ? sh[2] * m.p + 1 : 1);
        const std::size_t tc = std::size_t(sh[0]) * sh[1] * (m.dim == 3 ? sh[2] : 1);
        return sizeof(T) * (2 * std::size_t(std::max(nt_in, nt_out)) * nb + tc * nt_out * nd);
      };
      int big_sh[3], small_sh[3];
      shape_of<T>(m.dim, m.p, true, big_sh);
      shape_of<T>(m.dim, m.p, false, small_sh);
      const bool big_fits = smem(big_sh) <= budget, small_fits = smem(small_sh) <= budget;
      if (big_fits && !(make_tiling(m, big_sh).n_tiles < 2ll * sm_count() && small_fits))
        {
          big_out = true;
          return make_tiling(m, big_sh);
        }
      STMG_REQUIRE(small_fits, STMG_ERR_UNSUPPORTED, "operator: time blocks do not fit in shared memory");
      big_out = false;
      return make_tiling(m, small_sh);
    }

    template <int DIM, int P, typename T, bool BIG>
    void
    launch_box(const MeshView &m, const Tiling &tl, const TimeMats<T> &tm, const Cart1D<T> &c1, const QTab<T> &qt,
               const T *src, T *dst, T *shell, cudaStream_t s)
    {
      using Sh = OpShape<DIM, P, T, BIG>;
      using S  = TileShape<DIM, P, Sh::TX, Sh::TY, Sh::TZ>;
      const std::size_t smem = sizeof(T) * (2 * std::size_t(std::max(tm.nt_in, tm.nt_out)) * S::NB +
                                            std::size_t(S::TC) * tm.nt_out * S::ND);
      auto              kern = st_apply_kernel<DIM, P, T, 1, Sh::TX, Sh::TY, Sh::TZ>;
      const unsigned    grid = persistent_grid(reinterpret_cast<const void *>(kern), 256, smem, tl.n_tiles);
      const OutMode<T>  om{T(1), T(0), nullptr};
      kern<<<grid, 256, smem, s>>>(m, tl, tm, c1, qt, src, dst, shell, om);
      count_launch();
      STMG_CUDA(cudaGetLastError());
      if (tl.n_tiles > 1)
        launch_plane_fixup<DIM, T, false>(m, tl, tm.nt_out, shell, dst, om, s);
    }

    template <typename T>
    void
    box_apply(const MeshView &m, int nd, const double *A, const double *B, int nt_out, int nt_in, const T *src, T *dst,
              cudaStream_t s)
    {
      bool         big = true;
      const Tiling tl  = box_tiling<T>(m, nd, nt_in, nt_out, big);
      const std::size_t need = tl.n_tiles > 1 ? std::size_t(tl.n_tiles) * nt_out * tl.tile_stride * sizeof(T) : 0;
      if (need > NOALLOC_SCRATCH_BYTES)
        throw Error(STMG_ERR_SHAPE, "op_vmult_box_noalloc: this mesh needs " + std::to_string(need) +
                                      " bytes of tile scratch, more than the fixed " +
                                      std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes; use stmg_op_create instead");
      T *shell = static_cast<T *>(scratch_address());
      TimeMats<T> tm{};
      tm.nt_out = nt_out;
      tm.nt_in  = nt_in;
      for (int k = 0; k < nt_out * nt_in; ++k)
        {
          tm.A[k] = T(A[k]);
          tm.B[k] = T(B[k]);
        }
      const Cart1D<T> c1 = make_cart<T>(m);
      const QTab<T>   qt = make_qtab<T>(m.p);
#define STMG_BOX(D, PP)                                                                                  \
  if (m.dim == D && m.p == PP)                                                                           \
    return big ? launch_box<D, PP, T, true>(m, tl, tm, c1, qt, src, dst, shell, s)                       \
               : launch_box<D, PP, T, false>(m, tl, tm, c1, qt, src, dst, shell, s);
      STMG_BOX(2, 1) STMG_BOX(2, 2) STMG_BOX(2, 3) STMG_BOX(2, 4) STMG_BOX(2, 5)
      STMG_BOX(3, 1) STMG_BOX(3, 2) STMG_BOX(3, 3) STMG_BOX(3, 4)
#undef STMG_BOX
      throw Error(STMG_ERR_UNSUPPORTED, "op_vmult_box_noalloc: unsupported dim/degree");
    }
  } // namespace

  void
  op_vmult_box_noalloc(int dim, const int *n_cells, int degree, const double *lo, const double *hi, const void *coeff,
                       int nt_out, int nt_in, const double *A, const double *B, int dtype, const void *src, void *dst,
                       cudaStream_t s)
  {
    STMG_REQUIRE(n_cells && lo && hi && A && B && src && dst, STMG_ERR_ARG, "op_vmult_box_noalloc: null argument");
    STMG_REQUIRE(dim == 2 || dim == 3, STMG_ERR_ARG, "op_vmult_box_noalloc: dim must be 2 or 3");
    STMG_REQUIRE(degree >= 1 && degree <= MAX_P && (dim == 2 || degree <= 4), STMG_ERR_UNSUPPORTED,
                 "op_vmult_box_noalloc: degree must be 1..5 (3-D: 1..4)");
    STMG_REQUIRE(nt_out >= 1 && nt_out <= MAX_NT && nt_in >= 1 && nt_in <= MAX_NT, STMG_ERR_ARG,
                 "op_vmult_box_noalloc: time dimensions must be 1..16");
    STMG_REQUIRE(dtype == STMG_F64 || dtype == STMG_F32, STMG_ERR_ARG, "op_vmult_box_noalloc: dtype must be F64 or F32");
    // the view make_mesh builds for a uniform box (no vertex array needed)
    MeshView m{};
    m.dim    = dim;
    m.p      = degree;
    m.N      = 1;
    m.ncells = 1;
    for (int d = 0; d < 3; ++d)
      {
        STMG_REQUIRE(d >= dim || (n_cells[d] >= 1 && hi[d] > lo[d]), STMG_ERR_ARG,
                     "op_vmult_box_noalloc: cell counts and box extents must be positive");
        m.n[d]  = d < dim ? n_cells[d] : 1;
        m.nn[d] = d < dim ? n_cells[d] * degree + 1 : 1;
        m.h[d]  = d < dim ? (hi[d] - lo[d]) / n_cells[d] : 1.0;
        if (d < dim)
          {
            m.N *= m.nn[d];
            m.ncells *= m.n[d];
          }
      }
    m.cartesian  = 1;
    m.vert       = nullptr;
    m.coeff_mode = coeff ? 1 : 0;
    m.coeff64    = dtype == STMG_F64 ? static_cast<const double *>(coeff) : nullptr;
    m.coeff32    = dtype == STMG_F32 ? static_cast<const float *>(coeff) : nullptr;
    int nd = 1;
    for (int d = 0; d < dim; ++d)
      nd *= degree + 1;
    if (dtype == STMG_F64)
      box_apply<double>(m, nd, A, B, nt_out, nt_in, static_cast<const double *>(src), static_cast<double *>(dst), s);
    else
      box_apply<float>(m, nd, A, B, nt_out, nt_in, static_cast<const float *>(src), static_cast<float *>(dst), s);
  }
} // namespace stmg
