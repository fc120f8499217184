// Space-time operator kernels (see st_operator.cu for the method),
// instantiated per (dimension, degree) by st_apply_d<D>p<P>.cu.
#pragma once

#include "async_copy.cuh"
#include "kernels_common.cuh"
#include "tile_ops.cuh"

namespace stmg
{
  // everything one operator launch needs (host side)
  template <typename T>
  struct OpLaunch
  {
    MeshView     m;
    Tiling       tl;
    TimeMats<T>  tm;
    Cart1D<T>    c1;
    QTab<T>      qt;
    const T     *src;
    T           *dst;
    T           *shell;
    OutMode<T>   om;
    bool         big;
    cudaStream_t s;
    bool         tiny = false; // 3-D degree 2: tiles of 2x2x2 cells, phase B by planes (small meshes)
  };

  // shared memory of the operator kernel for a tile shape: two input bricks
  // (time values of a node contiguous, padded to ntp) and the per-cell results
  inline int
  op_ntp(int nt_in)
  {
    return nt_in <= 2 ? nt_in : (nt_in + 3) / 4 * 4;
  }

  inline std::size_t
  op_smem_bytes(int dim, int p, const int *shape, int nt_in, int nt_out, std::size_t elem)
  {
    const std::size_t nb = std::size_t(shape[0] * p + 1) * (shape[1] * p + 1) * (dim == 3 ? shape[2] * p + 1 : 1);
    const std::size_t tc = std::size_t(shape[0]) * shape[1] * (dim == 3 ? shape[2] : 1);
    std::size_t       nd = 1;
    for (int d = 0; d < dim; ++d)
      nd *= p + 1;
    return elem * (2 * std::size_t(op_ntp(nt_in)) * nb + tc * nt_out * nd);
  }

  template <int DIM, int P, typename T>
  void op_launch_dp(const OpLaunch<T> &L);

  namespace op_detail
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

    // K a + M b on a cartesian cell with two live arrays: one pass per
    // direction over the 1-D pencils, each pencil updated in place,
    //   z: a <- Mz a,  b <- Mz b + Kz a
    //   y: a <- My a,  b <- My b + Ky a
    //   x:             b <- Mx b + Kx a
    // (= Kx My Mz a + Mx Ky Mz a + Mx My Kz a + Mx My Mz b); result in b.
    template <int DIM, int P, typename T>
    __device__ __forceinline__ void
    cart_apply_pencils(const Cart1D<T> &c, T *a, T *b)
    {
      constexpr int P1 = P + 1;
      auto pass = [&](int d, int base, int stride, bool keep_a) {
        T va[P1], vb[P1];
#pragma unroll
        for (int k = 0; k < P1; ++k)
          {
            va[k] = a[base + k * stride];
            vb[k] = b[base + k * stride];
          }
#pragma unroll
        for (int i = 0; i < P1; ++i)
          {
            T ma = T(0), sb = T(0);
#pragma unroll
            for (int k = 0; k < P1; ++k)
              {
                const T mik = c.M[d][i * P1 + k];
                if (keep_a)
                  ma += mik * va[k];
                sb += mik * vb[k] + c.K[d][i * P1 + k] * va[k];
              }
            if (keep_a)
              a[base + i * stride] = ma;
            b[base + i * stride] = sb;
          }
      };
      if constexpr (DIM == 3)
        {
#pragma unroll
          for (int o = 0; o < P1 * P1; ++o)
            pass(2, o, P1 * P1, true);
#pragma unroll
          for (int z = 0; z < P1; ++z)
#pragma unroll
            for (int x = 0; x < P1; ++x)
              pass(1, x + z * P1 * P1, P1, true);
#pragma unroll
          for (int r = 0; r < P1 * P1; ++r)
            pass(0, r * P1, 1, false);
        }
      else
        {
#pragma unroll
          for (int x = 0; x < P1; ++x)
            pass(1, x, P1, true);
#pragma unroll
          for (int y = 0; y < P1; ++y)
            pass(0, y * P1, 1, false);
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
      T det = T(m.h[0]) * T(m.h[1]);
      if constexpr (DIM == 3)
        det *= T(m.h[2]);
      const T *cq = m.coeff_mode == 2 ? (sizeof(T) == 8 ? reinterpret_cast<const T *>(m.coeff64)
                                                         : reinterpret_cast<const T *>(m.coeff32)) +
                                          cell * ND
                                      : nullptr;
      const T kcell = m.coeff_mode == 1 ? (sizeof(T) == 8 ? T(m.coeff64[cell]) : T(m.coeff32[cell])) : T(1);
      // coefficient x JxW at the quadrature points (kept in a), mass part in b
      T kw[ND];
#pragma unroll
      for (int q = 0; q < ND; ++q)
        {
          const int qx = q % P1, qy = (q / P1) % P1, qz = q / (P1 * P1);
          T         w  = qt.gw[qx] * qt.gw[qy];
          if constexpr (DIM == 3)
            w *= qt.gw[qz];
          const T JxW = det * w;
          kw[q]       = (cq ? cq[q] : kcell) * JxW;
          b[q] *= JxW;
        }
      // one gradient component at a time: b += Dq_d^T (k JxW / h_d^2 Dq_d a)
      T g[ND];
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        {
          const T ih = T(1) / (T(m.h[d]) * T(m.h[d]));
          if (d == 0)
            sweep<P1, DIM, 0, false, false>(qt.Dq, a, g);
          else if (d == 1)
            sweep<P1, DIM, 1, false, false>(qt.Dq, a, g);
          else
            sweep<P1, DIM, DIM == 3 ? 2 : 1, false, false>(qt.Dq, a, g);
#pragma unroll
          for (int q = 0; q < ND; ++q)
            g[q] *= kw[q] * ih;
          if (d == 0)
            sweep<P1, DIM, 0, true, true>(qt.Dq, g, b);
          else if (d == 1)
            sweep<P1, DIM, 1, true, true>(qt.Dq, g, b);
          else
            sweep<P1, DIM, DIM == 3 ? 2 : 1, true, true>(qt.Dq, g, b);
        }
      sweep<P1, DIM, 0, false, true>(qt.S, b, b);
      if constexpr (DIM == 3)
        {
          sweep<P1, DIM, 1, false, true>(qt.S, b, b);
          sweep<P1, DIM, 2, false, true>(qt.S, b, out);
        }
      else
        sweep<P1, DIM, 1, false, true>(qt.S, b, out);
    }

    // Phase B for 3-D cells of degree 3 by planes. The per-thread form
    // keeps five 64-value arrays live per (cell, time dof) item and spills;
    // here a group of P1 = 4 consecutive lanes takes one item, lane pz
    // holding the item's P1 x P1 values in the plane z = pz. Sweeps along x
    // and y stay in the lane's registers, sweeps along z gather the plane
    // values of the group by shuffles. w holds the lane's row (or column)
    // of the 1-D matrix: out[xy] (+)= sum_k w[k] in_k[xy], in_k the value of
    // the group's lane k.
    template <int P1, bool ADD, typename T>
    __device__ __forceinline__ void
    zsweep(const T (&w)[P1], const T *in, T *out, int gbase)
    {
#pragma unroll
      for (int xy = 0; xy < P1 * P1; ++xy)
        {
          T v[P1];
#pragma unroll
          for (int k = 0; k < P1; ++k)
            v[k] = __shfl_sync(0xffffffffu, in[xy], gbase + k);
          T acc = ADD ? out[xy] : T(0);
#pragma unroll
          for (int k = 0; k < P1; ++k)
            acc += w[k] * v[k];
          out[xy] = acc;
        }
    }

    // K a + M b of one item by planes (lane pz of the group at gbase):
    // MODE 1 the separable Cartesian form (kappa already in a), MODE 2 the
    // box cell with a coefficient per cell or quadrature point, MODE 0 the
    // Q1-mapped cell. a and b hold the plane's nodal values on entry; the
    // result is left in b.
    template <int P, typename T, int MODE>
    __device__ __forceinline__ void
    planes_apply(const MeshView &m, const QTab<T> &qt, const Cart1D<T> &c1, int cx, int cy, int cz, long long cell,
                 int pz, int gbase, T *a, T *b)
    {
      constexpr int P1 = P + 1;
      constexpr int PL = P1 * P1;
      if constexpr (MODE == 1)
        {
          // (a, b) <- (M_d a, M_d b + K_d a) along z, y, then x (a dropped)
          T mz[P1], kz[P1];
#pragma unroll
          for (int k = 0; k < P1; ++k)
            {
              mz[k] = c1.M[2][pz * P1 + k];
              kz[k] = c1.K[2][pz * P1 + k];
            }
#pragma unroll
          for (int xy = 0; xy < PL; ++xy)
            {
              T va[P1], vb[P1];
#pragma unroll
              for (int k = 0; k < P1; ++k)
                {
                  va[k] = __shfl_sync(0xffffffffu, a[xy], gbase + k);
                  vb[k] = __shfl_sync(0xffffffffu, b[xy], gbase + k);
                }
              T ma = T(0), sb = T(0);
#pragma unroll
              for (int k = 0; k < P1; ++k)
                {
                  ma += mz[k] * va[k];
                  sb += mz[k] * vb[k] + kz[k] * va[k];
                }
              a[xy] = ma;
              b[xy] = sb;
            }
#pragma unroll
          for (int d = 1; d >= 0; --d)
            {
              const int stride = d == 0 ? 1 : P1;
#pragma unroll
              for (int o = 0; o < P1; ++o)
                {
                  const int base = d == 0 ? o * P1 : o;
                  T         va[P1], vb[P1];
#pragma unroll
                  for (int k = 0; k < P1; ++k)
                    {
                      va[k] = a[base + k * stride];
                      vb[k] = b[base + k * stride];
                    }
#pragma unroll
                  for (int i = 0; i < P1; ++i)
                    {
                      T ma = T(0), sb = T(0);
#pragma unroll
                      for (int k = 0; k < P1; ++k)
                        {
                          const T mik = c1.M[d][i * P1 + k];
                          if (d == 1)
                            ma += mik * va[k];
                          sb += mik * vb[k] + c1.K[d][i * P1 + k] * va[k];
                        }
                      if (d == 1)
                        a[base + i * stride] = ma;
                      b[base + i * stride] = sb;
                    }
                }
            }
        }
      else
        {
          T sr[P1], sc[P1], dr[P1], dc[P1];
#pragma unroll
          for (int k = 0; k < P1; ++k)
            {
              sr[k] = qt.S[pz * P1 + k];
              sc[k] = qt.S[k * P1 + pz];
              dr[k] = qt.Dq[pz * P1 + k];
              dc[k] = qt.Dq[k * P1 + pz];
            }
          // values at the quadrature points (plane pz is now qz = pz)
          sweep<P1, 2, 0, false, false>(qt.S, a, a);
          sweep<P1, 2, 1, false, false>(qt.S, a, a);
          zsweep<P1, false>(sr, a, a, gbase);
          sweep<P1, 2, 0, false, false>(qt.S, b, b);
          sweep<P1, 2, 1, false, false>(qt.S, b, b);
          zsweep<P1, false>(sr, b, b, gbase);
          // reference gradients by collocation
          T g0[PL], g1[PL], g2[PL];
          sweep<P1, 2, 0, false, false>(qt.Dq, a, g0);
          sweep<P1, 2, 1, false, false>(qt.Dq, a, g1);
          zsweep<P1, false>(dr, a, g2, gbase);
          const T *cq    = nullptr;
          T        kcell = T(1);
          if constexpr (sizeof(T) == 8)
            {
              if (m.coeff_mode == 1)
                kcell = T(m.coeff64[cell]);
              else if (m.coeff_mode == 2)
                cq = reinterpret_cast<const T *>(m.coeff64) + cell * (PL * P1) + pz * PL;
            }
          else
            {
              if (m.coeff_mode == 1)
                kcell = T(m.coeff32[cell]);
              else if (m.coeff_mode == 2)
                cq = reinterpret_cast<const T *>(m.coeff32) + cell * (PL * P1) + pz * PL;
            }
          const T wz = qt.gw[pz];
          if constexpr (MODE == 2)
            {
              const T det = T(m.h[0]) * T(m.h[1]) * T(m.h[2]);
              const T ih0 = T(1) / (T(m.h[0]) * T(m.h[0])), ih1 = T(1) / (T(m.h[1]) * T(m.h[1])),
                      ih2 = T(1) / (T(m.h[2]) * T(m.h[2]));
#pragma unroll
              for (int xy = 0; xy < PL; ++xy)
                {
                  const int qx = xy % P1, qy = xy / P1;
                  const T   JxW = det * (qt.gw[qx] * qt.gw[qy] * wz);
                  const T   kw  = (cq ? cq[xy] : kcell) * JxW;
                  g0[xy] *= kw * ih0;
                  g1[xy] *= kw * ih1;
                  g2[xy] *= kw * ih2;
                  b[xy] *= JxW;
                }
            }
          else
            {
              const T gz = qt.gx[pz];
              T       X[8][3];
              load_corners<3>(m, cx, cy, cz, X);
#pragma unroll
              for (int xy = 0; xy < PL; ++xy)
                {
                  const int qx = xy % P1, qy = xy / P1;
                  T         xi[3] = {qt.gx[qx], qt.gx[qy], gz};
                  T         J[3][3], Ji[3][3];
                  q1_jacobian<3>(X, xi, J);
                  const T det = det_inv<3>(J, Ji);
                  const T JxW = fabs(det) * (qt.gw[qx] * qt.gw[qy] * wz);
                  const T k   = (cq ? cq[xy] : kcell) * JxW;
                  // physical gradient Ji^T g, flux = k Ji (Ji^T g)
                  const T gr[3] = {g0[xy], g1[xy], g2[xy]};
                  T       ph[3];
#pragma unroll
                  for (int i = 0; i < 3; ++i)
                    ph[i] = k * (Ji[0][i] * gr[0] + Ji[1][i] * gr[1] + Ji[2][i] * gr[2]);
                  g0[xy] = Ji[0][0] * ph[0] + Ji[0][1] * ph[1] + Ji[0][2] * ph[2];
                  g1[xy] = Ji[1][0] * ph[0] + Ji[1][1] * ph[1] + Ji[1][2] * ph[2];
                  g2[xy] = Ji[2][0] * ph[0] + Ji[2][1] * ph[1] + Ji[2][2] * ph[2];
                  b[xy] *= JxW;
                }
            }
          // integrate: collocation derivatives transposed, then S^T
          sweep<P1, 2, 0, true, true>(qt.Dq, g0, b);
          sweep<P1, 2, 1, true, true>(qt.Dq, g1, b);
          zsweep<P1, true>(dc, g2, b, gbase);
          sweep<P1, 2, 0, false, true>(qt.S, b, b);
          sweep<P1, 2, 1, false, true>(qt.S, b, b);
          zsweep<P1, false>(sc, b, b, gbase);
        }
    }

    // compile-time tile shape per (dim, degree, precision); the fallback
    // shape serves time dimensions whose bricks do not fit the main one
    template <int DIM, int P, typename T, bool BIG>
    struct OpShape
    {
      static constexpr int TX = DIM == 2 ? (P <= 2 ? (BIG ? 16 : 4) : (P <= 4 ? (BIG ? 8 : 2) : (BIG ? 4 : 1)))
                                         : (P == 1 ? (BIG ? 8 : 2) : (P == 2 ? (BIG ? 8 : 4) : (BIG ? 4 : 1)));
      static constexpr int TY = DIM == 2 ? TX : (P == 1 ? TX : (P == 2 ? 4 : (BIG ? (P == 3 ? 4 : 2) : 1)));
      static constexpr int TZ = DIM == 2 ? 1 : (P == 1 ? TX : (P == 2 ? (BIG ? 4 : 2) : (BIG ? 2 : 1)));
    };


    // One CTA per tile of cells (persistent over tiles):
    //  A. the tile's input brick, all time values of a node contiguous, is
    //     staged by cp.async one tile ahead (Dirichlet and out-of-mesh nodes
    //     zero); warps walk brick rows, lanes cover (node, time) pairs;
    //  B. one thread per (output time dof j, cell): a_j = sum_i A(j,i) kappa
    //     u_i and b_j = sum_i B(j,i) u_i at the cell's nodes (one vector load
    //     per node), then K a_j + M b_j by register sum factorisation, into
    //     the per-cell result buffer;
    //  C. one thread per (j, brick node): the sum over the node's cells in a
    //     fixed order; tile-interior nodes go to dst, shell nodes to the
    //     tile's face slots (or constrained writes when one tile covers the
    //     mesh).
    // NTPC: 1 or 2 time values per node, or 4 for multiples of four.
    template <int DIM, int P, typename T, int MODE, int TX, int TY, int TZ, int NTPC, bool PL = false>
    __global__ void __launch_bounds__(256, (MODE == 1 || (sizeof(T) == 4 && MODE == 2)) ? 2 : 1)
    st_apply_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeMats<T> tm,
                    const __grid_constant__ Cart1D<T> c1, const __grid_constant__ QTab<T> qt,
                    const T *__restrict__ src, T *__restrict__ dst, T *__restrict__ shell, const OutMode<T> om)
    {
      using S          = TileShape<DIM, P, TX, TY, TZ>;
      constexpr int ND = S::ND;
      constexpr int P1 = P + 1;
      constexpr int NW = 8; // warps per CTA
      // 3-D degree 3, and degree 2 where PL asks for it (the small tiles of
      // small meshes, whose per-thread cell chains would be the critical
      // path): phase B by planes (see planes_apply)
      constexpr bool PLANES = DIM == 3 && (P == 3 || PL);
      extern __shared__ __align__(16) unsigned char smem_raw[];
      const int nti = tm.nt_in, nto = tm.nt_out;
      const int ntp = NTPC == 4 ? (nti + 3) / 4 * 4 : NTPC;
      T        *bricks[2] = {reinterpret_cast<T *>(smem_raw), reinterpret_cast<T *>(smem_raw) + S::NB * ntp};
      T        *cellbuf   = bricks[1] + S::NB * ntp; // [TC][nto][ND]
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      // brick load lanes: (node along x, time value)
      const int npl = 32 / ntp, lnode = lane / ntp, li = lane - lnode * ntp;
      const int n_tiles = int(tl.n_tiles);

      // padded time slots are never loaded: keep them zero
      for (int idx = threadIdx.x; idx < 2 * S::NB * ntp; idx += blockDim.x)
        bricks[0][idx] = T(0);
      __syncthreads();

      auto load = [&](int tile, T *brick) {
        const int t0 = tile % tl.ntiles[0], t1 = (tile / tl.ntiles[0]) % tl.ntiles[1],
                  t2 = tile / (tl.ntiles[0] * tl.ntiles[1]);
        const int gx0 = t0 * tl.T[0] * P, gy0 = t1 * tl.T[1] * P, gz0 = t2 * tl.T[2] * P;
        const int ex = min(tl.T[0], m.n[0] - t0 * tl.T[0]) * P + 1;
        const int ey = DIM > 1 ? min(tl.T[1], m.n[1] - t1 * tl.T[1]) * P + 1 : 1;
        const int ez = DIM == 3 ? min(tl.T[2], m.n[2] - t2 * tl.T[2]) * P + 1 : 1;
        if (lnode >= npl || li >= nti)
          return;
        for (int row = warp; row < S::E1 * S::E2; row += NW)
          {
            const int  bz = row / S::E1, by = row - bz * S::E1;
            const int  gy = gy0 + by, gz = gz0 + bz;
            bool       rok = by < ey && bz < ez && gy > 0 && gy < m.nn[1] - 1;
            if (DIM == 3)
              rok = rok && gz > 0 && gz < m.nn[2] - 1;
            const T   *grow = src + li * m.N + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz);
            T         *srow = brick + (long long)row * S::E0 * ntp + li;
            for (int bx = lnode; bx < S::E0; bx += npl)
              {
                const int  gx = gx0 + bx;
                const bool ok = rok && bx < ex && gx > 0 && gx < m.nn[0] - 1;
                cp_async_small<sizeof(T)>(srow + bx * ntp, ok ? grow + gx : src, ok);
              }
          }
      };

      int tile = blockIdx.x;
      if (tile < n_tiles)
        load(tile, bricks[0]);
      cp_async_commit();
      for (int buf = 0; tile < n_tiles; tile += gridDim.x, buf ^= 1)
        {
          if (tile + int(gridDim.x) < n_tiles)
            load(tile + gridDim.x, bricks[buf ^ 1]);
          cp_async_commit();
          cp_async_wait<1>();
          __syncthreads();
          int t[3], c0[3], tc[3], e[3];
          tile_extents<DIM>(m, tl, tile, t, c0, tc, e);

          // B. per (output time dof, cell)
          const T *brick = bricks[buf];
          if constexpr (PLANES)
            {
              // groups of P1 lanes per item; every lane of a warp runs each
              // pass (the z sweeps shuffle across the warp), lanes without an
              // item work on the tile's first cell and store nothing
              constexpr int IPW = 32 / P1;
              const int     grp = lane / P1, pz = lane - grp * P1, gbase = grp * P1;
              for (int w0 = warp * IPW; w0 < nto * S::TC; w0 += NW * IPW)
                {
                  const int w  = w0 + grp;
                  int       lc = w / nto, j = w - lc * nto;
                  int       lx = lc % TX, ly = (lc / TX) % TY, lz = lc / (TX * TY);
                  // (lanes past the last full group, for P1 not dividing 32,
                  // join the shuffles but hold no item)
                  const bool item = grp < IPW && w < nto * S::TC && lx < tc[0] && ly < tc[1] && lz < tc[2];
                  if (!item)
                    lc = j = lx = ly = lz = 0;
                  const int       cx = c0[0] + lx, cy = c0[1] + ly, cz = c0[2] + lz;
                  const long long cell = cx + (long long)m.n[0] * (cy + (long long)m.n[1] * cz);
                  T               kap  = T(1);
                  if (MODE == 1 && m.coeff_mode == 1)
                    kap = sizeof(T) == 8 ? T(m.coeff64[cell]) : T(m.coeff32[cell]);
                  T a[P1 * P1], b[P1 * P1];
#pragma unroll
                  for (int q = 0; q < P1 * P1; ++q)
                    a[q] = b[q] = T(0);
                  const T *brp = brick + (lx * P + S::E0 * (ly * P + S::E1 * (lz * P + pz))) * ntp;
                  for (int i0 = 0; i0 < ntp; i0 += NTPC)
                    {
                      T al[NTPC], be[NTPC];
#pragma unroll
                      for (int u = 0; u < NTPC; ++u)
                        {
                          const int i = i0 + u;
                          al[u]       = i < nti ? tm.A[j * nti + i] * kap : T(0);
                          be[u]       = i < nti ? tm.B[j * nti + i] : T(0);
                        }
#pragma unroll
                      for (int q = 0; q < P1 * P1; ++q)
                        {
                          const T *x = brp + ((q % P1) + S::E0 * (q / P1)) * ntp + i0;
#pragma unroll
                          for (int u = 0; u < NTPC; ++u)
                            {
                              const T xv = x[u];
                              a[q] += al[u] * xv;
                              b[q] += be[u] * xv;
                            }
                        }
                    }
                  planes_apply<P, T, MODE>(m, qt, c1, cx, cy, cz, cell, pz, gbase, a, b);
                  if (item)
                    {
                      T *cb = cellbuf + (lc * nto + j) * ND + pz * P1 * P1;
#pragma unroll
                      for (int q = 0; q < P1 * P1; ++q)
                        cb[q] = b[q];
                    }
                }
            }
          else
          for (int w = threadIdx.x; w < nto * S::TC; w += blockDim.x)
            {
              // consecutive threads take the time dofs of one cell: they
              // share the cell's brick reads (broadcast) and write
              // consecutive per-cell results
              const int lc = w / nto, j = w - lc * nto;
              const int lx = lc % TX, ly = (lc / TX) % TY, lz = lc / (TX * TY);
              if (lx >= tc[0] || ly >= tc[1] || lz >= tc[2])
                continue;
              const int       cx = c0[0] + lx, cy = c0[1] + ly, cz = c0[2] + lz;
              const long long cell = cx + (long long)m.n[0] * (cy + (long long)m.n[1] * cz);
              T               kap  = T(1);
              if (MODE == 1 && m.coeff_mode == 1)
                kap = sizeof(T) == 8 ? T(m.coeff64[cell]) : T(m.coeff32[cell]);
              T a[ND], b[ND];
#pragma unroll
              for (int q = 0; q < ND; ++q)
                a[q] = b[q] = T(0);
              const T *br0 = brick + (lx * P + S::E0 * (ly * P + S::E1 * (lz * P))) * ntp;
              for (int i0 = 0; i0 < ntp; i0 += NTPC)
                {
                  T al[NTPC], be[NTPC];
#pragma unroll
                  for (int u = 0; u < NTPC; ++u)
                    {
                      const int i = i0 + u;
                      al[u]       = i < nti ? tm.A[j * nti + i] * kap : T(0);
                      be[u]       = i < nti ? tm.B[j * nti + i] : T(0);
                    }
#pragma unroll
                  for (int q = 0; q < ND; ++q)
                    {
                      const T *x = br0 + S::offset(q) * ntp + i0;
                      T        xv[NTPC];
                      if constexpr (NTPC == 4 && sizeof(T) == 4)
                        {
                          const float4 v = *reinterpret_cast<const float4 *>(x);
                          xv[0] = v.x, xv[1] = v.y, xv[2] = v.z, xv[NTPC - 1] = v.w;
                        }
                      else if constexpr (NTPC >= 2)
                        {
#pragma unroll
                          for (int u = 0; u < NTPC; u += 2)
                            {
                              if constexpr (sizeof(T) == 8)
                                {
                                  const double2 v = *reinterpret_cast<const double2 *>(x + u);
                                  xv[u] = v.x, xv[u + 1] = v.y;
                                }
                              else
                                {
                                  const float2 v = *reinterpret_cast<const float2 *>(x + u);
                                  xv[u] = v.x, xv[u + 1] = v.y;
                                }
                            }
                        }
                      else
                        xv[0] = x[0];
#pragma unroll
                      for (int u = 0; u < NTPC; ++u)
                        {
                          a[q] += al[u] * xv[u];
                          b[q] += be[u] * xv[u];
                        }
                    }
                }
              T *cb = cellbuf + (lc * nto + j) * ND;
              if constexpr (MODE == 1 && sizeof(T) == 8)
                {
                  // FP64: two live arrays keep the kernel at two CTAs per SM
                  cart_apply_pencils<DIM, P>(c1, a, b); // result in b
#pragma unroll
                  for (int q = 0; q < ND; ++q)
                    cb[q] = b[q];
                }
              else
                {
                  T out[ND];
                  if constexpr (MODE == 1)
                    cart_apply<DIM, P>(c1, a, b, out);
                  else if constexpr (MODE == 2)
                    box_apply<DIM, P>(m, qt, cell, a, b, out);
                  else
                    general_apply<DIM, P>(m, qt, cx, cy, cz, cell, a, b, out);
#pragma unroll
                  for (int q = 0; q < ND; ++q)
                    cb[q] = out[q];
                }
            }
          __syncthreads();

          // C. per (j, brick node): sum over the node's cells, write out.
          // A node on a cell face also belongs to the next cell along that
          // direction: offsets to the second candidate per direction, and
          // lane (x) constants for the tile, row (y, z) constants per row.
          int  lx_base[2], lx_dx[2], lx_two[2];
          bool lx_in[2];
#pragma unroll
          for (int h = 0; h < 2; ++h)
            {
              const int  bx   = lane + 32 * h;
              const bool face = bx % P == 0 && bx > 0;
              const int  cx0  = face ? bx / P - 1 : bx / P;
              const int  ax0  = face ? P : bx % P;
              lx_base[h]      = cx0 * nto * ND + ax0;
              lx_dx[h]        = nto * ND - ax0;
              lx_two[h]       = face && bx / P < tc[0];
              lx_in[h]        = bx > 0 && bx < e[0] - 1;
            }
          for (int row = warp; row < S::E1 * S::E2; row += NW)
            {
              const int bz = row / S::E1, by = row - bz * S::E1;
              if (by >= e[1] || bz >= e[2])
                continue;
              const bool fy = by % P == 0 && by > 0;
              const int  cy0 = fy ? by / P - 1 : by / P, ay0 = fy ? P : by % P;
              const bool ty  = fy && by / P < tc[1];
              const int  dy  = TX * nto * ND - P1 * ay0;
              int        cz0 = 0, az0 = 0, dz = 0;
              bool       tz  = false;
              if (DIM == 3)
                {
                  const bool fz = bz % P == 0 && bz > 0;
                  cz0           = fz ? bz / P - 1 : bz / P;
                  az0           = fz ? P : bz % P;
                  tz            = fz && bz / P < tc[2];
                  dz            = TX * TY * nto * ND - P1 * P1 * az0;
                }
              const T   *cbr = cellbuf + TX * (cy0 + TY * cz0) * nto * ND + P1 * (ay0 + P1 * az0);
              const long long grow = c0[0] * P + (long long)m.nn[0] * ((c0[1] * P + by) + (long long)m.nn[1] * (c0[2] * P + bz));
              const bool yzin = by > 0 && by < e[1] - 1 && (DIM < 3 || (bz > 0 && bz < e[2] - 1));
              // shell slot of this row: x faces by (y, z); y and z faces by x
              long long rslot = 0;
              if (!yzin)
                {
                  if (by == 0)
                    rslot = tl.face_off[2] + (long long)tl.E[0] * bz;
                  else if (by == e[1] - 1 || DIM == 2)
                    rslot = tl.face_off[3] + (long long)tl.E[0] * bz;
                  else if (bz == 0)
                    rslot = tl.face_off[4] + (long long)tl.E[0] * by;
                  else
                    rslot = tl.face_off[5] + (long long)tl.E[0] * by;
                }
              const long long xslot = by + (long long)tl.E[1] * bz;
#pragma unroll
              for (int h = 0; h < (S::E0 + 31) / 32; ++h)
                {
                  const int bx = lane + 32 * h;
                  if (bx >= e[0])
                    break;
                  const T  *c    = cbr + lx_base[h];
                  const int dx   = lx_dx[h];
                  const bool two = lx_two[h];
                  const long long slot = bx == 0 ? tl.face_off[0] + xslot
                                                 : (bx == e[0] - 1 ? tl.face_off[1] + xslot : rslot + bx);
                  const bool inner = yzin && lx_in[h];
                  const T   *cj    = c;
                  long long  gj    = grow + bx; // index into dst and rhs
                  T         *sj    = shell + (long long)tile * nto * tl.tile_stride + slot;
                  // four time dofs at a time, their dst / rhs loads issued
                  // before their stores (OutMode::write_n)
                  for (int j0 = 0; j0 < nto; j0 += 4, gj += 4 * m.N)
                    {
                      const int cnt = min(4, nto - j0);
                      T         sv[4];
#pragma unroll
                      for (int jj = 0; jj < 4; ++jj, cj += ND, sj += tl.tile_stride)
                        {
                          if (jj >= cnt)
                            break;
                          T s = cj[0];
                          if (two)
                            s += cj[dx];
                          if (ty)
                            {
                              s += cj[dy];
                              if (two)
                                s += cj[dy + dx];
                            }
                          if (tz)
                            {
                              s += cj[dz];
                              if (two)
                                s += cj[dz + dx];
                              if (ty)
                                {
                                  s += cj[dz + dy];
                                  if (two)
                                    s += cj[dz + dy + dx];
                                }
                            }
                          sv[jj] = s;
                          if (!inner && tl.n_tiles != 1)
                            *sj = s;
                        }
                      if (inner)
                        om.write_n(dst, gj, m.N, sv, cnt);
                      else if (tl.n_tiles == 1)
                        om.template write_constrained_n<4>(dst, gj, m.N, cnt);
                    }
                }
            }
          __syncthreads();
        }
      cp_async_wait<0>();
    }
  } // namespace op_detail

  template <int DIM, int P, typename T, int MODE, bool BIG, int NTPC>
  void
  op_launch_variant(const OpLaunch<T> &L)
  {
    using Sh  = op_detail::OpShape<DIM, P, T, BIG>;
    auto kern = op_detail::st_apply_kernel<DIM, P, T, MODE, Sh::TX, Sh::TY, Sh::TZ, NTPC>;
    int  shape[3] = {Sh::TX, Sh::TY, Sh::TZ};
    if constexpr (DIM == 3 && P == 2)
      if (L.tiny)
        {
          kern  = op_detail::st_apply_kernel<DIM, P, T, MODE, 2, 2, 2, NTPC, true>;
          shape[0] = shape[1] = shape[2] = 2;
        }
    const std::size_t smem = op_smem_bytes(DIM, P, shape, L.tm.nt_in, L.tm.nt_out, sizeof(T));
    const unsigned grid = persistent_grid(reinterpret_cast<const void *>(kern), 256, smem, L.tl.n_tiles);
    kern<<<grid, 256, smem, L.s>>>(L.m, L.tl, L.tm, L.c1, L.qt, L.src, L.dst, L.shell, L.om);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    if (L.tl.n_tiles > 1)
      launch_plane_fixup<DIM, T, false>(L.m, L.tl, L.tm.nt_out, L.shell, L.dst, L.om, L.s);
  }

  template <int DIM, int P, typename T, int MODE, bool BIG>
  void
  op_launch_nt(const OpLaunch<T> &L)
  {
    const int nti = L.tm.nt_in;
    if (nti == 1)
      return op_launch_variant<DIM, P, T, MODE, BIG, 1>(L);
    if (nti == 2)
      return op_launch_variant<DIM, P, T, MODE, BIG, 2>(L);
    return op_launch_variant<DIM, P, T, MODE, BIG, 4>(L);
  }

  template <int DIM, int P, typename T, int MODE>
  void
  op_launch_mode(const OpLaunch<T> &L)
  {
    if (L.big)
      op_launch_nt<DIM, P, T, MODE, true>(L);
    else
      op_launch_nt<DIM, P, T, MODE, false>(L);
  }

  // the dispatch every st_apply_d<D>p<P>.cu instantiates
  template <int DIM, int P, typename T>
  void
  op_launch_impl(const OpLaunch<T> &L)
  {
    if (L.m.cartesian)
      op_launch_mode<DIM, P, T, 1>(L);
    else if (L.m.box)
      op_launch_mode<DIM, P, T, 2>(L);
    else
      op_launch_mode<DIM, P, T, 0>(L);
  }
} // namespace stmg
