// Vanka apply kernels (see vanka.cu for the method); instantiated per
// spatial dimension by vanka_apply_2d.cu and vanka_apply_3d.cu.
#pragma once

#include <cuda_bf16.h>

#include "tile_ops.cuh"
#include "vanka.h"

namespace stmg
{
  namespace vanka_detail
  {
    template <typename TS>
    __device__ __forceinline__ float
    load_s(const TS *p)
    {
      if constexpr (std::is_same_v<TS, __nv_bfloat16>)
        return __bfloat162float(*p);
      else
        return float(*p);
    }

    // --------------------------------------------------------------- apply
    // small dense solve (mu A + B) z = y with partial pivoting, in registers
    template <int NT, typename T>
    __device__ __forceinline__ void
    mode_solve(const TimeMats<T> &tm, T mu, const T *y, T *z, int nt)
    {
      constexpr int N = NT > 0 ? NT : MAX_NT;
      T             A[N][N + 1];
      const int     n = NT > 0 ? NT : nt;
#pragma unroll
      for (int i = 0; i < N; ++i)
        {
          if (i >= n)
            break;
#pragma unroll
          for (int j = 0; j < N; ++j)
            {
              if (j >= n)
                break;
              A[i][j] = mu * tm.A[i * n + j] + tm.B[i * n + j];
            }
          A[i][N] = y[i];
        }
#pragma unroll
      for (int k = 0; k < N; ++k)
        {
          if (k >= n)
            break;
          int piv = k;
#pragma unroll
          for (int i = k + 1; i < N; ++i)
            if (i < n && fabs(A[i][k]) > fabs(A[piv][k]))
              piv = i;
          if (piv != k)
#pragma unroll
            for (int j = 0; j <= N; ++j)
              {
                const T tmp = A[k][j];
                A[k][j]     = A[piv][j];
                A[piv][j]   = tmp;
              }
          const T d = T(1) / A[k][k];
#pragma unroll
          for (int i = k + 1; i < N; ++i)
            {
              if (i >= n)
                break;
              const T f = A[i][k] * d;
#pragma unroll
              for (int j = k + 1; j < N; ++j)
                if (j < n)
                  A[i][j] -= f * A[k][j];
              A[i][N] -= f * A[k][N];
            }
        }
#pragma unroll
      for (int i = N - 1; i >= 0; --i)
        {
          if (i >= n)
            continue;
          T s = A[i][N];
#pragma unroll
          for (int j = i + 1; j < N; ++j)
            if (j < n)
              s -= A[i][j] * z[j];
          z[i] = s / A[i][i];
        }
    }

    // Per cell the setup stores one record: V as [mode][dof] in the storage
    // type, padded to 16 bytes, then mu (nd values of the compute type),
    // padded to 16 bytes; rec_bytes = record stride. Records stream through
    // shared memory in chunks of `chunk` cells (cp.async, double buffered).
    template <int DIM, int P, typename T, typename TS, int NT, int TX, int TY, int TZ>
    __global__ void __launch_bounds__(256, 2)
    vanka_apply_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeMats<T> tm,
                       const unsigned char *__restrict__ rec, int rec_bytes, int mu_off, int chunk,
                       const T *__restrict__ src, T *__restrict__ dst, T *__restrict__ shell, const OutMode<T> om)
    {
      using S          = TileShape<DIM, P, TX, TY, TZ>;
      constexpr int ND = S::ND;
      constexpr int NA = NT > 0 ? NT : MAX_NT;
      extern __shared__ __align__(16) unsigned char vk_smem[];
      const int      nt      = tm.nt_out;
      unsigned char *recs[2] = {vk_smem, vk_smem + (long long)chunk * rec_bytes};
      T             *bricks[2];
      bricks[0]     = reinterpret_cast<T *>(vk_smem + 2ll * chunk * rec_bytes);
      bricks[1]     = bricks[0] + nt * S::NB;
      T *zbuf       = bricks[1] + nt * S::NB;
      T *obuf       = zbuf + chunk * nt * ND;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
      const int r16  = rec_bytes / 16;
      const int nch  = (S::TC + chunk - 1) / chunk;

      auto issue = [&](long long tl_i, int chk, int rb, int bb) {
        int tt[3], cc0[3], ttc[3], ee[3];
        tile_extents<DIM>(m, tl, tl_i, tt, cc0, ttc, ee);
        if (chk == 0)
          load_brick<S>(bricks[bb], src, m, nt, cc0, ee);
        const int first = chk * chunk;
        for (int c = warp; c < chunk; c += nw)
          {
            const int lc = first + c;
            const int lx = lc % TX, ly = (lc / TX) % TY, lz = lc / (TX * TY);
            if (lc >= S::TC || lx >= ttc[0] || ly >= ttc[1] || lz >= ttc[2])
              continue;
            const long long cell = (cc0[0] + lx) + (long long)m.n[0] * ((cc0[1] + ly) + (long long)m.n[1] * (cc0[2] + lz));
            const unsigned char *g = rec + cell * rec_bytes;
            unsigned char       *d = recs[rb] + (long long)c * rec_bytes;
            for (int q = lane; q < r16; q += 32)
              cp_async16(d + 16 * q, g + 16 * q);
          }
      };

      long long tile = blockIdx.x;
      int       ch   = 0;
      if (tile < tl.n_tiles)
        issue(tile, 0, 0, 0);
      cp_async_commit();
      int rb = 0, bb = 0;
      int t[3], c0[3], tc[3], e[3];
      while (tile < tl.n_tiles)
        {
          tile_extents<DIM>(m, tl, tile, t, c0, tc, e);
          long long ntile = tile;
          int       nchk  = ch + 1;
          if (nchk >= nch)
            {
              ntile = tile + gridDim.x;
              nchk  = 0;
            }
          if (ntile < tl.n_tiles)
            issue(ntile, nchk, rb ^ 1, nchk == 0 ? bb ^ 1 : bb);
          cp_async_commit();
          cp_async_wait<1>();
          __syncthreads();

          const T  *brick = bricks[bb];
          const int first = ch * chunk;
          // B1: per (cell, mode): y = V^T x, z = (mu A + B)^{-1} y
          for (int w = threadIdx.x; w < chunk * ND; w += blockDim.x)
            {
              const int c = w / ND, mm = w - c * ND;
              const int lc = first + c;
              const int lx = lc % TX, ly = (lc / TX) % TY, lz = lc / (TX * TY);
              if (lc >= S::TC || lx >= tc[0] || ly >= tc[1] || lz >= tc[2])
                continue;
              const unsigned char *r   = recs[rb] + (long long)c * rec_bytes;
              const TS            *col = reinterpret_cast<const TS *>(r) + mm * ND;
              const T              mu  = reinterpret_cast<const T *>(r + mu_off)[mm];
              T                    y[NA], z[NA];
#pragma unroll
              for (int i = 0; i < NA; ++i)
                y[i] = T(0);
              const T *br = brick + lx * P + S::E0 * (ly * P + S::E1 * (lz * P));
#pragma unroll
              for (int a = 0; a < ND; ++a)
                {
                  T va;
                  if constexpr (sizeof(T) == 8)
                    va = T(col[a]);
                  else
                    va = load_s(col + a);
                  const T *bp = br + S::offset(a);
#pragma unroll
                  for (int i = 0; i < NA; ++i)
                    if (NT > 0 || i < nt)
                      y[i] += va * bp[i * S::NB];
                }
              mode_solve<NT, T>(tm, mu, y, z, nt);
              T *zb = zbuf + c * nt * ND + mm;
#pragma unroll
              for (int i = 0; i < NA; ++i)
                if (NT > 0 || i < nt)
                  zb[i * ND] = z[i];
            }
          __syncthreads();
          // B2: per (cell, dof): out = V z
          for (int w = threadIdx.x; w < chunk * ND; w += blockDim.x)
            {
              const int c = w / ND, a = w - c * ND;
              const int lc = first + c;
              const int lx = lc % TX, ly = (lc / TX) % TY, lz = lc / (TX * TY);
              if (lc >= S::TC || lx >= tc[0] || ly >= tc[1] || lz >= tc[2])
                continue;
              const TS *vr = reinterpret_cast<const TS *>(recs[rb] + (long long)c * rec_bytes) + a;
              const T  *zb = zbuf + c * nt * ND;
              T         o[NA];
#pragma unroll
              for (int i = 0; i < NA; ++i)
                o[i] = T(0);
#pragma unroll 9
              for (int mm = 0; mm < ND; ++mm)
                {
                  T vm;
                  if constexpr (sizeof(T) == 8)
                    vm = T(vr[mm * ND]);
                  else
                    vm = load_s(vr + mm * ND);
#pragma unroll
                  for (int i = 0; i < NA; ++i)
                    if (NT > 0 || i < nt)
                      o[i] += vm * zb[i * ND + mm];
                }
#pragma unroll
              for (int i = 0; i < NA; ++i)
                if (NT > 0 || i < nt)
                  obuf[(i * S::TC + lc) * ND + a] = o[i];
            }
          __syncthreads();
          if (ch == nch - 1)
            {
              // C/D: coloured scatter into the output brick (this tile's input
              // brick buffer, no longer read), then write with 1/valence
              T *ob = bricks[bb];
              scatter_cells<S, DIM, T>(obuf, ob, nt, tc);
              write_brick<S, DIM, T, true>(ob, m, tl, tile, nt, c0, e, dst, shell, om);
              __syncthreads();
              bb ^= 1;
            }
          rb ^= 1;
          tile = ntile;
          ch   = nchk;
        }
      cp_async_wait<0>();
    }

    // compile-time tile shapes of the Vanka apply (main and fallback)
    template <int DIM, int P, bool BIG>
    struct VkShape
    {
      static constexpr int TX = DIM == 2 ? (P <= 2 ? (BIG ? 8 : 2) : (P <= 4 ? (BIG ? 4 : 1) : (BIG ? 2 : 1)))
                                         : (P == 1 ? (BIG ? 8 : 2) : (P == 2 ? (BIG ? 4 : 2) : (BIG ? 2 : 1)));
      static constexpr int TY = TX;
      static constexpr int TZ = DIM == 2 ? 1 : (P == 1 ? (BIG ? 4 : 2) : TX);
    };

    template <int DIM, int P, typename T, typename TS, int NT, bool BIG>
    void
    launch_apply3(const Vanka &vk, const T *src, T *dst, const OutMode<T> &om, cudaStream_t s)
    {
      using Sh = VkShape<DIM, P, BIG>;
      const MeshView   &m    = vk.mesh->v;
      const Tiling     &tl   = vk.tiling;
      const std::size_t smem = vk.smem_bytes(vk.shape);
      auto              kern = vanka_apply_kernel<DIM, P, T, TS, NT, Sh::TX, Sh::TY, Sh::TZ>;
      const unsigned    grid = persistent_grid(reinterpret_cast<const void *>(kern), 256, smem, tl.n_tiles);
      const TimeMats<T> &tm  = vk.tmats<T>();
      kern<<<grid, 256, smem, s>>>(m, tl, tm, vk.V.ptr, vk.rec_bytes, vk.mu_off, vk.chunk, src, dst,
                                   reinterpret_cast<T *>(vk.shell.ptr), om);
      count_launch();
      STMG_CUDA(cudaGetLastError());
      if (tl.n_tiles > 1)
        launch_plane_fixup<DIM, T, true>(m, tl, vk.nt, reinterpret_cast<T *>(vk.shell.ptr), dst, om, s);
    }

    template <int DIM, int P, typename T, typename TS, int NT>
    void
    launch_apply_nt(const Vanka &vk, const T *src, T *dst, const OutMode<T> &om, cudaStream_t s)
    {
      if (vk.big)
        launch_apply3<DIM, P, T, TS, NT, true>(vk, src, dst, om, s);
      else
        launch_apply3<DIM, P, T, TS, NT, false>(vk, src, dst, om, s);
    }

    template <int DIM, int P, typename T, typename TS>
    void
    launch_apply2(const Vanka &vk, const T *src, T *dst, const OutMode<T> &om, cudaStream_t s)
    {
      switch (vk.nt)
        {
          case 2:
            return launch_apply_nt<DIM, P, T, TS, 2>(vk, src, dst, om, s);
          case 3:
            return launch_apply_nt<DIM, P, T, TS, 3>(vk, src, dst, om, s);
          case 4:
            return launch_apply_nt<DIM, P, T, TS, 4>(vk, src, dst, om, s);
          default:
            return launch_apply_nt<DIM, P, T, TS, 0>(vk, src, dst, om, s);
        }
    }

    template <int DIM, int P>
    void
    launch_apply1(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s)
    {
      const OutMode<double> o64{alpha, beta, nullptr};
      const OutMode<float>  o32{float(alpha), float(beta), nullptr};
      if (vk.compute == STMG_F64)
        return launch_apply2<DIM, P, double, double>(vk, static_cast<const double *>(src), static_cast<double *>(dst),
                                                     o64, s);
      if (vk.storage == STMG_BF16)
        return launch_apply2<DIM, P, float, __nv_bfloat16>(vk, static_cast<const float *>(src),
                                                           static_cast<float *>(dst), o32, s);
      return launch_apply2<DIM, P, float, float>(vk, static_cast<const float *>(src), static_cast<float *>(dst), o32, s);
    }
  } // namespace vanka_detail

  // compile-time Vanka tile shape for (dim, degree, main/fallback)
  inline void
  vanka_shape(int dim, int p, bool big, int *T3)
  {
#define STMG_VS(D, PP)                                                                                   \
  if (dim == D && p == PP)                                                                               \
    {                                                                                                    \
      if (big)                                                                                           \
        T3[0] = vanka_detail::VkShape<D, PP, true>::TX, T3[1] = vanka_detail::VkShape<D, PP, true>::TY,   \
        T3[2] = vanka_detail::VkShape<D, PP, true>::TZ;                                                  \
      else                                                                                               \
        T3[0] = vanka_detail::VkShape<D, PP, false>::TX, T3[1] = vanka_detail::VkShape<D, PP, false>::TY, \
        T3[2] = vanka_detail::VkShape<D, PP, false>::TZ;                                                 \
      return;                                                                                            \
    }
    STMG_VS(2, 1) STMG_VS(2, 2) STMG_VS(2, 3) STMG_VS(2, 4) STMG_VS(2, 5) STMG_VS(3, 1) STMG_VS(3, 2) STMG_VS(3, 3)
#undef STMG_VS
    throw Error(STMG_ERR_UNSUPPORTED, "vanka: unsupported dim/degree");
  }
} // namespace stmg
