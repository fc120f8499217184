// Vanka apply kernels (see vanka.cu for the method); instantiated per
// spatial dimension by vanka_apply_2d.cu and vanka_apply_3d.cu.
#pragma once

#include <cuda_bf16.h>

#include "kernels_common.cuh"
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

    __device__ __forceinline__ int
    valence_of(const MeshView &m, const int (&g)[3])
    {
      int v = 1;
      for (int d = 0; d < m.dim; ++d)
        if (g[d] % m.p == 0 && g[d] > 0 && g[d] < m.nn[d] - 1)
          v *= 2;
      return v;
    }

    template <int DIM, int P, typename T, typename TS, int NT>
    __global__ void __launch_bounds__(256)
    vanka_apply_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeMats<T> tm,
                       const TS *__restrict__ V, const T *__restrict__ mu, const T *__restrict__ src,
                       T *__restrict__ dst, T *__restrict__ shell)
    {
      constexpr int P1 = P + 1;
      constexpr int ND = Tens<P1, DIM>::ND;
      constexpr int NA = NT > 0 ? NT : MAX_NT;
      extern __shared__ __align__(16) unsigned char vk_smem[];
      T        *brick = reinterpret_cast<T *>(vk_smem);
      const int nt    = tm.nt_out;

      int t[3], c0[3], tc[3], e[3];
      tile_extents<DIM>(m, tl, blockIdx.x, t, c0, tc, e);
      const int       nb    = e[0] * e[1] * e[2];
      const int       nbmax = tl.E[0] * tl.E[1] * tl.E[2];
      const int       tcmax = tl.T[0] * tl.T[1] * tl.T[2];
      T              *zbuf  = brick + (long long)nt * nbmax;
      T              *obuf  = zbuf + (long long)tcmax * nt * ND;
      const long long N     = m.N;

      for (int idx = threadIdx.x; idx < nt * nb; idx += blockDim.x)
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

      const int ncell = tc[0] * tc[1] * tc[2];
      // B1: per (cell, mode): y = V^T x, z = (mu A + B)^{-1} y
      for (int w = threadIdx.x; w < ncell * ND; w += blockDim.x)
        {
          const int lc = w / ND, mm = w % ND;
          const int lx = lc % tc[0], ly = (lc / tc[0]) % tc[1], lz = lc / (tc[0] * tc[1]);
          const long long cell = (c0[0] + lx) + (long long)m.n[0] * ((c0[1] + ly) + (long long)m.n[1] * (c0[2] + lz));
          const TS *col = V + (cell * ND + mm) * ND;
          T         y[NA], z[NA];
#pragma unroll
          for (int i = 0; i < NA; ++i)
            y[i] = T(0);
          const T *br = brick + lx * P + e[0] * (ly * P + e[1] * (lz * P));
#pragma unroll
          for (int a = 0; a < ND; ++a)
            {
              const int ax = a % P1, ay = (a / P1) % P1, az = a / (P1 * P1);
              T         va;
              if constexpr (sizeof(T) == 8)
                va = T(col[a]);
              else
                va = load_s(col + a);
              const T *bp = br + ax + e[0] * (ay + e[1] * az);
#pragma unroll
              for (int i = 0; i < NA; ++i)
                if (NT > 0 || i < nt)
                  y[i] += va * bp[i * nb];
            }
          mode_solve<NT, T>(tm, mu[cell * ND + mm], y, z, nt);
          T *zb = zbuf + (long long)lc * nt * ND + mm;
#pragma unroll
          for (int i = 0; i < NA; ++i)
            if (NT > 0 || i < nt)
              zb[i * ND] = z[i];
        }
      __syncthreads();
      // B2: per (cell, node): out = V z
      for (int w = threadIdx.x; w < ncell * ND; w += blockDim.x)
        {
          const int lc = w / ND, a = w % ND;
          const int lx = lc % tc[0], ly = (lc / tc[0]) % tc[1], lz = lc / (tc[0] * tc[1]);
          const long long cell = (c0[0] + lx) + (long long)m.n[0] * ((c0[1] + ly) + (long long)m.n[1] * (c0[2] + lz));
          const TS *row = V + cell * ND * ND + a;
          const T  *zb  = zbuf + (long long)lc * nt * ND;
          T         o[NA];
#pragma unroll
          for (int i = 0; i < NA; ++i)
            o[i] = T(0);
#pragma unroll 4
          for (int mm = 0; mm < ND; ++mm)
            {
              T vm;
              if constexpr (sizeof(T) == 8)
                vm = T(row[mm * ND]);
              else
                vm = load_s(row + mm * ND);
#pragma unroll
              for (int i = 0; i < NA; ++i)
                if (NT > 0 || i < nt)
                  o[i] += vm * zb[i * ND + mm];
            }
          T *ob = obuf + (long long)lc * nt * ND + a;
#pragma unroll
          for (int i = 0; i < NA; ++i)
            if (NT > 0 || i < nt)
              ob[i * ND] = o[i];
        }
      __syncthreads();
      // C: gather per brick node, weight 1/valence where complete
      for (int idx = threadIdx.x; idx < nt * nb; idx += blockDim.x)
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
                  s += obuf[((long long)lc * nt + j) * ND + ax + P1 * (ay + P1 * az)];
                }
          bool interior = b3[0] > 0 && b3[0] < e[0] - 1 && b3[1] > 0 && b3[1] < e[1] - 1;
          if (DIM == 3)
            interior = interior && b3[2] > 0 && b3[2] < e[2] - 1;
          if (interior)
            {
              const int       g[3] = {c0[0] * P + b3[0], c0[1] * P + b3[1], c0[2] * P + b3[2]};
              const long long gi   = g[0] + (long long)m.nn[0] * (g[1] + (long long)m.nn[1] * g[2]);
              dst[j * N + gi]      = s / T(valence_of(m, g));
            }
          else
            shell[((long long)blockIdx.x * nt + j) * tl.tile_stride + shell_slot<DIM>(tl, e, b3[0], b3[1], b3[2])] = s;
        }
    }

    template <int DIM, typename T>
    __global__ void
    vanka_fixup_kernel(const MeshView m, const Tiling tl, int nt, const T *__restrict__ shell, T *__restrict__ dst)
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
      const T w = T(1) / T(valence_of(m, g));
      for (int j = 0; j < nt; ++j)
        dst[j * m.N + node] = bd ? T(0) : shell_sum<DIM, T>(m, tl, shell, nt, j, g) * w;
    }
    template <int DIM, int P, typename T, typename TS, int NT>
    void
    launch_apply3(const Vanka &vk, const T *src, T *dst, cudaStream_t s)
    {
      const MeshView &m    = vk.mesh->v;
      const Tiling   &tl   = vk.tiling;
      const std::size_t smem = vk.smem_bytes(tl);
      auto kern = vanka_apply_kernel<DIM, P, T, TS, NT>;
      STMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      const TimeMats<T> &tm = vk.tmats<T>();
      kern<<<unsigned(tl.n_tiles), 256, smem, s>>>(m, tl, tm, reinterpret_cast<const TS *>(vk.V.ptr),
                                                   reinterpret_cast<const T *>(vk.mu.ptr), src, dst,
                                                   reinterpret_cast<T *>(vk.shell.ptr));
      count_launch();
      STMG_CUDA(cudaGetLastError());
      vanka_fixup_kernel<DIM, T><<<unsigned((m.N + 255) / 256), 256, 0, s>>>(m, tl, vk.nt, reinterpret_cast<T *>(vk.shell.ptr), dst);
      count_launch();
      STMG_CUDA(cudaGetLastError());
    }

    template <int DIM, int P, typename T, typename TS>
    void
    launch_apply2(const Vanka &vk, const T *src, T *dst, cudaStream_t s)
    {
      switch (vk.nt)
        {
          case 2:
            return launch_apply3<DIM, P, T, TS, 2>(vk, src, dst, s);
          case 3:
            return launch_apply3<DIM, P, T, TS, 3>(vk, src, dst, s);
          case 4:
            return launch_apply3<DIM, P, T, TS, 4>(vk, src, dst, s);
          default:
            return launch_apply3<DIM, P, T, TS, 0>(vk, src, dst, s);
        }
    }

    template <int DIM, int P>
    void
    launch_apply1(const Vanka &vk, const void *src, void *dst, cudaStream_t s)
    {
      if (vk.compute == STMG_F64)
        return launch_apply2<DIM, P, double, double>(vk, static_cast<const double *>(src), static_cast<double *>(dst), s);
      if (vk.storage == STMG_BF16)
        return launch_apply2<DIM, P, float, __nv_bfloat16>(vk, static_cast<const float *>(src), static_cast<float *>(dst), s);
      return launch_apply2<DIM, P, float, float>(vk, static_cast<const float *>(src), static_cast<float *>(dst), s);
    }
  } // namespace vanka_detail
} // namespace stmg
