// Vanka apply kernels (see vanka.cu for the method); instantiated per
// spatial dimension by vanka_apply_2d.cu and vanka_apply_3d.cu.
#pragma once

#include <cuda_bf16.h>

#include <type_traits>

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

    // ------------------------------------------------ streamed FP32 apply
    // (mu A + B) z = y for one mode in registers: Gaussian elimination with
    // partial pivoting where the pivot row is brought up by compare-and-swap
    // with static indices, so nothing is spilled to local memory.
    template <int NT>
    __device__ __forceinline__ void
    mode_solve_reg(const TimeMats<float> &tm, float mu, const float (&y)[NT], float (&z)[NT])
    {
      float A[NT][NT + 1];
#pragma unroll
      for (int i = 0; i < NT; ++i)
        {
#pragma unroll
          for (int j = 0; j < NT; ++j)
            A[i][j] = fmaf(mu, tm.A[i * NT + j], tm.B[i * NT + j]);
          A[i][NT] = y[i];
        }
#pragma unroll
      for (int k = 0; k < NT; ++k)
        {
#pragma unroll
          for (int i = k + 1; i < NT; ++i)
            {
              const bool sw = fabsf(A[i][k]) > fabsf(A[k][k]);
#pragma unroll
              for (int j = k; j <= NT; ++j)
                {
                  const float a = A[k][j], b = A[i][j];
                  A[k][j]       = sw ? b : a;
                  A[i][j]       = sw ? a : b;
                }
            }
          const float d = __frcp_rn(A[k][k]);
          A[k][k]       = d; // the back substitution multiplies by it
#pragma unroll
          for (int i = k + 1; i < NT; ++i)
            {
              const float f = A[i][k] * d;
#pragma unroll
              for (int j = k + 1; j <= NT; ++j)
                A[i][j] -= f * A[k][j];
            }
        }
#pragma unroll
      for (int i = NT - 1; i >= 0; --i)
        {
          float s = A[i][NT];
#pragma unroll
          for (int j = i + 1; j < NT; ++j)
            s -= A[i][j] * z[j];
          z[i] = s * A[i][i];
        }
    }

    // (mu A + B) z = y through the eigenbasis of B^{-1} A (see TimeEig):
    // w = G y, then per real eigenvalue w_k /= mu a_k + 1 and per complex pair
    // the 2x2 block [[mu a + 1, mu b], [-mu b, mu a + 1]] inverted, z = S w.
    template <int NT>
    __device__ __forceinline__ void
    mode_solve_eig(const TimeEig &te, float mu, const float (&y)[NT], float (&z)[NT])
    {
      float w[NT];
#pragma unroll
      for (int i = 0; i < NT; ++i)
        {
          float s = 0.0f;
#pragma unroll
          for (int j = 0; j < NT; ++j)
            s = fmaf(te.G[i * NT + j], y[j], s);
          w[i] = s;
        }
#pragma unroll
      for (int k = 0; k < NT; ++k)
        {
          const float d = fmaf(mu, te.a[k], 1.0f);
          if (te.kind[k] == 1)
            w[k] *= __frcp_rn(d);
          else if (te.kind[k] == 2 && k + 1 < NT)
            {
              const float e = mu * te.b[k], inv = __frcp_rn(fmaf(d, d, e * e));
              const float u = w[k], v = w[k + 1];
              w[k]          = inv * fmaf(d, u, -e * v);
              w[k + 1]      = inv * fmaf(e, u, d * v);
            }
        }
#pragma unroll
      for (int i = 0; i < NT; ++i)
        {
          float s = 0.0f;
#pragma unroll
          for (int j = 0; j < NT; ++j)
            s = fmaf(te.S[i * NT + j], w[j], s);
          z[i] = s;
        }
    }

    // NT time values of one node, stored contiguously (NTP = padded count)
    template <int NT>
    struct TimeVec
    {
      static constexpr int NTP = NT == 3 ? 4 : NT;
      __device__ __forceinline__ static void
      load(const float *p, float (&v)[NT])
      {
        if constexpr (NTP == 4)
          {
            const float4 q = *reinterpret_cast<const float4 *>(p);
            v[0]           = q.x;
            v[1]           = q.y;
            v[2]           = q.z;
            if constexpr (NT == 4)
              v[3] = q.w;
          }
        else if constexpr (NTP == 2)
          {
            const float2 q = *reinterpret_cast<const float2 *>(p);
            v[0]           = q.x;
            v[1]           = q.y;
          }
        else
          v[0] = *p;
      }
      __device__ __forceinline__ static void
      store(float *p, const float (&v)[NT])
      {
        if constexpr (NTP == 4)
          *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], NT == 4 ? v[NT - 1] : 0.0f);
        else if constexpr (NTP == 2)
          *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
        else
          *p = v[0];
      }
    };

    constexpr int VK_STAGES = 3; // record ring depth (colour phases in flight)

    // Tile geometry in 32-bit integers (tile counts stay far below 2^31).
    struct TileGeo
    {
      int c0[3], tc[3], e[3];
    };

    template <int DIM, int P>
    __device__ __forceinline__ TileGeo
    tile_geo(const MeshView &m, const Tiling &tl, int tile)
    {
      TileGeo   g;
      const int t[3] = {tile % tl.ntiles[0], (tile / tl.ntiles[0]) % tl.ntiles[1], tile / (tl.ntiles[0] * tl.ntiles[1])};
#pragma unroll
      for (int d = 0; d < 3; ++d)
        {
          g.c0[d] = t[d] * tl.T[d];
          g.tc[d] = d < DIM ? min(tl.T[d], m.n[d] - g.c0[d]) : 1;
          g.e[d]  = d < DIM ? g.tc[d] * P + 1 : 1;
        }
      return g;
    }

    // Streamed apply: the tile's cells are visited colour by colour (cells of
    // one colour share no node), one warp per cell: modes over the lanes for
    // y = V x and the n_t x n_t solves, dofs over the lanes for V^T z, which
    // is added straight into the shared output brick (fixed order, no
    // atomics). Records are stored in (tile, colour, cell) order, so each
    // colour phase reads one contiguous block; blocks stream through a
    // VK_STAGES ring of cp.async groups, one group per colour phase, the next
    // tile's input brick riding in the group of its first phase. Bricks keep
    // the time values of a node together (one vector load per node) and are
    // moved by brick rows: each warp covers 32 / E0 rows per step.
    template <int DIM, int P, typename TS, int NT, int TX, int TY, int TZ>
    __global__ void __launch_bounds__(256, 2)
    vanka_stream_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeMats<float> tm,
                        const __grid_constant__ TimeEig te, const unsigned char *__restrict__ rec, int rec_bytes,
                        int mu_off, int cpc, const float *__restrict__ src, float *__restrict__ dst,
                        float *__restrict__ shell, const OutMode<float> om)
    {
      using S           = TileShape<DIM, P, TX, TY, TZ>;
      using TV          = TimeVec<NT>;
      constexpr int ND  = S::ND;
      constexpr int NTP = TV::NTP;
      constexpr int NC  = 1 << DIM;
      constexpr int CPC = ((TX + 1) / 2) * ((TY + 1) / 2) * (DIM == 3 ? (TZ + 1) / 2 : 1);
      constexpr int RPW = 32 / S::E0;                    // brick rows per warp step
      constexpr int ROWS = NT * S::E1 * S::E2;          // rows of one brick (all time dofs)
      constexpr int NW   = 8;                            // warps per CTA
      static_assert(S::E0 <= 32, "brick rows wider than a warp");
      extern __shared__ __align__(16) unsigned char vk_smem[];
      __shared__ int col_n[NC], col_pre[NC], col_cell[NC][CPC];
      const int       warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int       lrow = lane / S::E0, lx = lane - lrow * S::E0;
      const long long stage_bytes = (long long)cpc * rec_bytes;
      float          *bin0 = reinterpret_cast<float *>(vk_smem + VK_STAGES * stage_bytes);
      float          *bout = bin0 + 2 * S::NB * NTP;
      float          *zb   = bout + S::NB * NTP + warp * ND * NTP;
      const long long tcr  = (long long)tl.T[0] * tl.T[1] * tl.T[2];
      const int       my_tiles = int(blockIdx.x) < tl.n_tiles ? int((tl.n_tiles - 1 - blockIdx.x) / gridDim.x) + 1 : 0;
      const int       phases   = my_tiles * NC;

      // per colour: cell count, first record slot, local cell coordinates
      if (threadIdx.x < NC)
        {
          const int col = threadIdx.x;
          int       cnt[3], n = 1, pre = 0;
          for (int c = 0; c <= col; ++c)
            {
              int nc = 1;
#pragma unroll
              for (int d = 0; d < 3; ++d)
                {
                  const int o = (c >> d) & 1;
                  cnt[d]      = d < DIM ? (tl.T[d] - o + 1) / 2 : (o ? 0 : 1);
                  nc *= cnt[d];
                }
              if (c < col)
                pre += nc;
              else
                n = nc;
            }
          col_n[col]   = n;
          col_pre[col] = pre;
          for (int idx = 0; idx < n && idx < CPC; ++idx)
            {
              const int ix = idx % cnt[0], iy = (idx / cnt[0]) % cnt[1], iz = idx / (cnt[0] * cnt[1]);
              const int cx = 2 * ix + (col & 1), cy = 2 * iy + ((col >> 1) & 1), cz = 2 * iz + ((col >> 2) & 1);
              col_cell[col][idx] = cx | (cy << 8) | (cz << 16);
            }
        }
      for (int idx = threadIdx.x; idx < S::NB * NTP; idx += blockDim.x)
        bout[idx] = 0.0f;
      __syncthreads();

      auto issue = [&](int k) {
        if (k < phases)
          {
            const int            tile = blockIdx.x + (k / NC) * gridDim.x;
            const int            col  = k % NC;
            const unsigned char *g    = rec + (tile * tcr + col_pre[col]) * rec_bytes;
            unsigned char       *d    = vk_smem + (k % VK_STAGES) * stage_bytes;
            const int            q16  = col_n[col] * (rec_bytes / 16);
            for (int q = threadIdx.x; q < q16; q += blockDim.x)
              cp_async16(d + 16 * q, g + 16 * q);
            if (col == 0)
              {
                const TileGeo tg  = tile_geo<DIM, P>(m, tl, tile);
                float        *bi  = bin0 + ((k / NC) & 1) * S::NB * NTP;
                const int     gx  = tg.c0[0] * P + lx;
                const bool    okx = lx < tg.e[0] && gx > 0 && gx < m.nn[0] - 1;
                for (int rb = warp * RPW; rb < ROWS; rb += NW * RPW)
                  {
                    const int row = rb + lrow;
                    if (lrow >= RPW || row >= ROWS)
                      continue;
                    const int  i = row / (S::E1 * S::E2), rem = row - i * (S::E1 * S::E2);
                    const int  bz = rem / S::E1, by = rem - bz * S::E1;
                    const int  gy = tg.c0[1] * P + by, gz = tg.c0[2] * P + bz;
                    bool       ok = okx && by < tg.e[1] && bz < tg.e[2] && gy > 0 && gy < m.nn[1] - 1;
                    if (DIM == 3)
                      ok = ok && gz > 0 && gz < m.nn[2] - 1;
                    const float *gp = ok ? src + i * m.N + gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz) : src;
                    cp_async_small<4>(bi + ((bz * S::E1 + by) * S::E0 + lx) * NTP + i, gp, ok);
                  }
              }
          }
        cp_async_commit();
      };

#pragma unroll
      for (int k = 0; k < VK_STAGES - 1; ++k)
        issue(k);

      TileGeo tg{};
      for (int k = 0; k < phases; ++k)
        {
          cp_async_wait<VK_STAGES - 2>();
          __syncthreads(); // phase k's records visible; phase k-1 done (its stage and output adds)
          issue(k + VK_STAGES - 1);

          const int tile = blockIdx.x + (k / NC) * gridDim.x;
          const int col  = k % NC;
          if (col == 0)
            tg = tile_geo<DIM, P>(m, tl, tile);
          const int            n   = col_n[col];
          const unsigned char *stg = vk_smem + (k % VK_STAGES) * stage_bytes;
          const float         *bi  = bin0 + ((k / NC) & 1) * S::NB * NTP;
          for (int idx = warp; idx < n; idx += NW)
            {
              const int cl = col_cell[col][idx];
              const int cx = cl & 255, cy = (cl >> 8) & 255, cz = cl >> 16;
              if (cx >= tg.tc[0] || cy >= tg.tc[1] || cz >= tg.tc[2])
                continue;
              const unsigned char *r    = stg + idx * rec_bytes;
              const TS            *V    = reinterpret_cast<const TS *>(r);
              const float         *mu   = reinterpret_cast<const float *>(r + mu_off);
              const int            base = cx * P + S::E0 * (cy * P + S::E1 * (cz * P));
              // y = V x per mode, then the mode's time solve
              for (int mm = lane; mm < ND; mm += 32)
                {
                  float     y[NT];
                  const TS *vr = V + mm * ND;
                  if constexpr (NT == 4)
                    {
                      // packed FP32 pairs: two FFMA2 per node
                      float2 y01 = make_float2(0.0f, 0.0f), y23 = y01;
#pragma unroll
                      for (int a = 0; a < ND; ++a)
                        {
                          const float  v  = load_s(vr + a);
                          const float4 x  = *reinterpret_cast<const float4 *>(bi + (base + S::offset(a)) * NTP);
                          const float2 vv = make_float2(v, v);
                          y01             = __ffma2_rn(vv, make_float2(x.x, x.y), y01);
                          y23             = __ffma2_rn(vv, make_float2(x.z, x.w), y23);
                        }
                      y[0] = y01.x;
                      y[1] = y01.y;
                      y[2] = y23.x;
                      y[NT - 1] = y23.y;
                    }
                  else
                    {
#pragma unroll
                      for (int i = 0; i < NT; ++i)
                        y[i] = 0.0f;
#pragma unroll
                      for (int a = 0; a < ND; ++a)
                        {
                          const float v = load_s(vr + a);
                          float       x[NT];
                          TV::load(bi + (base + S::offset(a)) * NTP, x);
#pragma unroll
                          for (int i = 0; i < NT; ++i)
                            y[i] = fmaf(v, x[i], y[i]);
                        }
                    }
                  float z[NT];
                  if (te.use)
                    mode_solve_eig<NT>(te, mu[mm], y, z);
                  else
                    mode_solve_reg<NT>(tm, mu[mm], y, z);
                  TV::store(zb + mm * NTP, z);
                }
              __syncwarp();
              // out = V^T z per dof, added into the output brick
              for (int a = lane; a < ND; a += 32)
                {
                  float o[NT];
                  if constexpr (NT == 4)
                    {
                      float2 o01 = make_float2(0.0f, 0.0f), o23 = o01;
#pragma unroll 9
                      for (int mm = 0; mm < ND; ++mm)
                        {
                          const float  v  = load_s(V + mm * ND + a);
                          const float4 z  = *reinterpret_cast<const float4 *>(zb + mm * NTP);
                          const float2 vv = make_float2(v, v);
                          o01             = __ffma2_rn(vv, make_float2(z.x, z.y), o01);
                          o23             = __ffma2_rn(vv, make_float2(z.z, z.w), o23);
                        }
                      o[0] = o01.x;
                      o[1] = o01.y;
                      o[2] = o23.x;
                      o[NT - 1] = o23.y;
                    }
                  else
                    {
#pragma unroll
                      for (int i = 0; i < NT; ++i)
                        o[i] = 0.0f;
#pragma unroll 9
                      for (int mm = 0; mm < ND; ++mm)
                        {
                          const float v = load_s(V + mm * ND + a);
                          float       z[NT];
                          TV::load(zb + mm * NTP, z);
#pragma unroll
                          for (int i = 0; i < NT; ++i)
                            o[i] = fmaf(v, z[i], o[i]);
                        }
                    }
                  float *ob = bout + (base + S::offset(a)) * NTP;
                  float  cur[NT];
                  TV::load(ob, cur);
#pragma unroll
                  for (int i = 0; i < NT; ++i)
                    cur[i] += o[i];
                  TV::store(ob, cur);
                }
              __syncwarp();
            }
          if (col == NC - 1)
            {
              __syncthreads();
              // the tile's output: interior nodes -> dst (1/valence), shell
              // nodes -> face slots (or constrained writes for one tile);
              // warps walk (y, z) rows, lanes x, the time dofs innermost
              const int  gx  = tg.c0[0] * P + lx;
              const int  vx  = (gx % P == 0) ? 2 : 1;
              const bool inx = lx > 0 && lx < tg.e[0] - 1;
              for (int rb = warp * RPW; rb < S::E1 * S::E2; rb += NW * RPW)
                {
                  const int row = rb + lrow;
                  if (lrow >= RPW || row >= S::E1 * S::E2 || lx >= tg.e[0])
                    continue;
                  const int bz = row / S::E1, by = row - bz * S::E1;
                  if (by >= tg.e[1] || bz >= tg.e[2])
                    continue;
                  bool inte = inx && by > 0 && by < tg.e[1] - 1;
                  if (DIM == 3)
                    inte = inte && bz > 0 && bz < tg.e[2] - 1;
                  const int gy = tg.c0[1] * P + by, gz = tg.c0[2] * P + bz;
                  int       v  = vx * ((gy % P == 0) ? 2 : 1);
                  if (DIM == 3)
                    v *= (gz % P == 0) ? 2 : 1;
                  const float w = v == 1 ? 1.0f : (v == 2 ? 0.5f : (v == 4 ? 0.25f : 0.125f));
                  float       o[NT];
                  TV::load(bout + ((bz * S::E1 + by) * S::E0 + lx) * NTP, o);
                  const long long gi = gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz);
                  if (inte)
                    {
#pragma unroll
                      for (int j = 0; j < NT; ++j)
                        o[j] *= w;
                      om.write_n(dst, gi, m.N, o);
                    }
                  else if (tl.n_tiles == 1)
                    om.template write_constrained_n<NT>(dst, gi, m.N);
                  else
                    {
                      float *sj = shell + (long long)tile * NT * tl.tile_stride + shell_slot<DIM>(tl, tg.e, lx, by, bz);
#pragma unroll
                      for (int j = 0; j < NT; ++j, sj += tl.tile_stride)
                        *sj = o[j];
                    }
                }
              __syncthreads();
              for (int idx = threadIdx.x; idx < S::NB * NTP; idx += blockDim.x)
                bout[idx] = 0.0f;
            }
        }
      cp_async_wait<0>();
    }

    // ------------------------------------------------- row-record apply
    // Record streaming by the bulk copy engine: one cp.async.bulk (global ->
    // this CTA's shared memory, no multicast) per colour phase, completing on
    // an mbarrier. Waiting threads sleep in mbarrier.try_wait (suspend-time
    // hint) instead of polling, so they leave the issue slots to the warps
    // that compute. Every wait is bounded: after VR_WAIT_NS of global time the
    // kernel sets the fault flag, waits (bounded) for the copies it issued and
    // returns.
    constexpr int                VR_STAGES  = 3;             // fewest record stages (colour phases in flight - 1)
    constexpr int                VR_STAGES_MAX = 5;          // most record stages
    constexpr int                VR_WARPS   = 8;             // warps per CTA, a warp per cell
    constexpr unsigned           VR_SUSPEND = 20000;         // ns a waiting thread may sleep per try_wait
    constexpr unsigned long long VR_WAIT_NS = 2000000000ull; // give up a barrier phase after 2 s

    __device__ __forceinline__ unsigned
    smem_u32(const void *p)
    {
      return static_cast<unsigned>(__cvta_generic_to_shared(p));
    }

    __device__ __forceinline__ void
    mbar_init(unsigned bar, unsigned count)
    {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
    }

    __device__ __forceinline__ void
    mbar_expect_tx(unsigned bar, unsigned bytes)
    {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
    }

    __device__ __forceinline__ void
    mbar_arrive(unsigned bar)
    {
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
    }

    __device__ __forceinline__ unsigned long long
    global_ns()
    {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      return t;
    }

    // one try_wait: true if the phase of the given parity has completed; the
    // thread may sleep up to VR_SUSPEND ns waiting for it
    __device__ __forceinline__ bool
    mbar_try_wait(unsigned bar, unsigned parity)
    {
      unsigned done;
      asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                   "selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done)
                   : "r"(bar), "r"(parity), "r"(VR_SUSPEND)
                   : "memory");
      return done != 0;
    }

    // true once the phase of the given parity has completed, false after
    // VR_WAIT_NS
    __device__ __forceinline__ bool
    mbar_wait(unsigned bar, unsigned parity)
    {
      if (mbar_try_wait(bar, parity))
        return true;
      const unsigned long long t0 = global_ns();
      while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > VR_WAIT_NS)
          return false;
      return true;
    }

    // bytes (a multiple of 16, 16-byte aligned ends) global -> shared,
    // completing on bar
    __device__ __forceinline__ void
    bulk_copy_g2s(unsigned dst, const void *src, unsigned bytes, unsigned bar)
    {
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                   "l"(src), "r"(bytes), "r"(bar)
                   : "memory");
    }

    // orders this thread's earlier shared-memory accesses before later
    // bulk-copy writes to the same bytes
    __device__ __forceinline__ void
    fence_proxy_async_smem()
    {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }

    // entries a of a row held as 16-byte words (FP32) or 8-byte words (BF16)
    template <typename TS>
    struct RowWord
    {
      using W = std::conditional_t<sizeof(TS) == 4, float4, uint2>;
      static constexpr int PER = sizeof(W) / sizeof(TS); // entries per word
      __device__ __forceinline__ static float
      get(const W &w, int i)
      {
        if constexpr (sizeof(TS) == 4)
          return i == 0 ? w.x : (i == 1 ? w.y : (i == 2 ? w.z : w.w));
        else
          {
            const unsigned u = (i < 2) ? w.x : w.y;
            return (i & 1) ? __uint_as_float(u & 0xffff0000u) : __uint_as_float(u << 16);
          }
      }
    };

    // y (NTP values as pairs) += v * x (NTP values)
    template <int NTP>
    __device__ __forceinline__ void
    acc_time(float2 (&y)[(NTP + 1) / 2], float v, const float *x)
    {
      if constexpr (NTP == 4)
        {
          const float4 q  = *reinterpret_cast<const float4 *>(x);
          const float2 vv = make_float2(v, v);
          y[0]            = __ffma2_rn(vv, make_float2(q.x, q.y), y[0]);
          y[1]            = __ffma2_rn(vv, make_float2(q.z, q.w), y[1]);
        }
      else if constexpr (NTP == 2)
        y[0] = __ffma2_rn(make_float2(v, v), *reinterpret_cast<const float2 *>(x), y[0]);
      else
        y[0].x = fmaf(v, *x, y[0].x);
    }

    // 1 / d to about one ulp (the multifunction unit's reciprocal)
    __device__ __forceinline__ float
    rcp_approx(float d)
    {
      float r;
      asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
      return r;
    }

    // w = (mu Lambda + I)^{-1} y in the real block form of the eigenbasis of
    // Beta^{-1} Alpha (the G and S factors are applied to whole bricks): NR
    // real eigenvalues first, then complex pairs (a_k +- i b_k), each pair's
    // 2x2 block [[mu a + 1, mu b], [-mu b, mu a + 1]] inverted
    template <int NT, int NR>
    __device__ __forceinline__ void
    mode_scale(const TimeEig &te, float mu, float (&y)[NT])
    {
#pragma unroll
      for (int k = 0; k < NR; ++k)
        y[k] *= rcp_approx(fmaf(mu, te.a[k], 1.0f));
#pragma unroll
      for (int k = NR; k + 1 < NT; k += 2)
        {
          const float d = fmaf(mu, te.a[k], 1.0f), e = mu * te.b[k];
          const float inv = rcp_approx(fmaf(d, d, e * e));
          const float u = y[k], v = y[k + 1];
          y[k]          = inv * fmaf(d, u, -e * v);
          y[k + 1]      = inv * fmaf(e, u, d * v);
        }
    }

    // v (NT values) <- M v for a row-major NT x NT matrix M (kernel parameter)
    template <int NT>
    __device__ __forceinline__ void
    time_map(const float *M, float (&v)[NT])
    {
      float o[NT];
#pragma unroll
      for (int i = 0; i < NT; ++i)
        {
          float s = 0.0f;
#pragma unroll
          for (int j = 0; j < NT; ++j)
            s = fmaf(M[i * NT + j], v[j], s);
          o[i] = s;
        }
#pragma unroll
      for (int i = 0; i < NT; ++i)
        v[i] = o[i];
    }

    // A tile's output brick (accumulated in the eigenbasis) back through S
    // and out, as in the streamed apply: tile-interior nodes to dst through
    // the output mode, weighted by 1/valence; shell nodes to the tile's face
    // slots, or the constrained write when one tile covers the mesh. nw
    // warps walk brick rows, 32 / E0 rows per warp step.
    template <int DIM, int P, int NT, typename S>
    __device__ __forceinline__ void
    row_tile_output(const MeshView &m, const Tiling &tl, const TimeEig &te, const TileGeo &tg, int tile,
                    const float *bout, float *__restrict__ dst, float *__restrict__ shell, const OutMode<float> &om,
                    int nw)
    {
      using TV           = TimeVec<NT>;
      constexpr int NTP  = TV::NTP;
      constexpr int RPW  = 32 / S::E0;
      const int     warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int     lrow = lane / S::E0, lx = lane - lrow * S::E0;
      const int     gx   = tg.c0[0] * P + lx;
      const int     vx   = (gx % P == 0) ? 2 : 1;
      const bool    inx  = lx > 0 && lx < tg.e[0] - 1;
      for (int rb = warp * RPW; rb < S::E1 * S::E2; rb += nw * RPW)
        {
          const int row = rb + lrow;
          if (lrow >= RPW || row >= S::E1 * S::E2 || lx >= tg.e[0])
            continue;
          const int bz = row / S::E1, by = row - bz * S::E1;
          if (by >= tg.e[1] || bz >= tg.e[2])
            continue;
          bool inte = inx && by > 0 && by < tg.e[1] - 1;
          if (DIM == 3)
            inte = inte && bz > 0 && bz < tg.e[2] - 1;
          const int gy = tg.c0[1] * P + by, gz = tg.c0[2] * P + bz;
          int       v  = vx * ((gy % P == 0) ? 2 : 1);
          if (DIM == 3)
            v *= (gz % P == 0) ? 2 : 1;
          const float w = v == 1 ? 1.0f : (v == 2 ? 0.5f : (v == 4 ? 0.25f : 0.125f));
          float       o[NT];
          TV::load(bout + ((bz * S::E1 + by) * S::E0 + lx) * NTP, o);
          time_map<NT>(te.S, o);
          const long long gi = gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz);
          if (inte)
            {
#pragma unroll
              for (int jt = 0; jt < NT; ++jt)
                o[jt] *= w;
              om.write_n(dst, gi, m.N, o);
            }
          else if (tl.n_tiles == 1)
            om.template write_constrained_n<NT>(dst, gi, m.N);
          else
            {
              float *sj = shell + (long long)tile * NT * tl.tile_stride + shell_slot<DIM>(tl, tg.e, lx, by, bz);
#pragma unroll
              for (int jt = 0; jt < NT; ++jt, sj += tl.tile_stride)
                *sj = o[jt];
            }
        }
    }

    // Row-record apply: as the streamed apply (colour phases, records in
    // (tile, colour, cell) order, one warp per cell, one output brick per
    // tile), but
    //  * each colour phase's records arrive by one bulk copy on an mbarrier;
    //  * a record holds V by rows read as whole words, the FP32 row of mode m
    //    ending in its eigenvalue mu_m;
    //  * the time solves work in the eigenbasis with its two factors moved
    //    out of the cells: the input brick is mapped by G = S^{-1} Beta^{-1}
    //    once per tile and the tile's output by S when it is written, so a
    //    mode's solve is the scaling of mode_scale;
    //  * the time values of a node are added pairwise (FFMA2), the 27-term
    //    sums split into two chains.
    template <int DIM, int P, typename TS, int NT, int TX, int TY, int TZ, int STG>
    __global__ void __launch_bounds__(VR_WARPS * 32, 2)
    vanka_row_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeEig te,
                     const unsigned char *__restrict__ rec, int rec_bytes, int mu_off, int cpc,
                     const float *__restrict__ src, float *__restrict__ dst, float *__restrict__ shell,
                     const OutMode<float> om, int *__restrict__ fault)
    {
      using S           = TileShape<DIM, P, TX, TY, TZ>;
      using TV          = TimeVec<NT>;
      using RW          = RowWord<TS>;
      using W           = typename RW::W;
      constexpr int ND  = S::ND;
      constexpr int NTP = TV::NTP;
      constexpr int NA  = (NTP + 1) / 2; // accumulator pairs
      constexpr int NR  = NT % 2;        // real eigenvalues of Beta^{-1} Alpha
      constexpr int NC  = 1 << DIM;
      constexpr int CPC = ((TX + 1) / 2) * ((TY + 1) / 2) * (DIM == 3 ? (TZ + 1) / 2 : 1);
      constexpr int NW  = VR_WARPS;
      constexpr int RS  = vk_row_stride<TS>(ND); // row stride (entries)
      constexpr int RWD = RS / RW::PER;          // words per row
      constexpr int RPW = 32 / S::E0;            // brick rows per warp step
      constexpr int ROWS = NT * S::E1 * S::E2;   // rows of one input brick
      constexpr bool MU_IN_ROW = sizeof(TS) == 4;
      static_assert(ND <= 32, "row-record apply: at most 32 dofs per cell");
      static_assert(S::E0 <= 32, "brick rows wider than a warp");
      extern __shared__ __align__(16) unsigned char vk_smem[];
      __shared__ int                             col_n[NC], col_pre[NC], col_cell[NC][CPC];
      __shared__ __align__(8) unsigned long long bars[STG];
      const int       warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int       lrow = lane / S::E0, lx = lane - lrow * S::E0;
      const long long stage_bytes = (long long)cpc * rec_bytes;
      float          *bin0 = reinterpret_cast<float *>(vk_smem + STG * stage_bytes);
      float          *bout = bin0 + 2 * S::NB * NTP;
      float          *wb   = bout + S::NB * NTP + warp * ND * NTP;
      const long long tcr  = (long long)tl.T[0] * tl.T[1] * tl.T[2];
      const int       my_tiles = int(blockIdx.x) < tl.n_tiles ? int((tl.n_tiles - 1 - blockIdx.x) / gridDim.x) + 1 : 0;
      const int       phases   = my_tiles * NC;

      if (threadIdx.x < NC)
        {
          const int col = threadIdx.x;
          int       cnt[3], n = 1, pre = 0;
          for (int c = 0; c <= col; ++c)
            {
              int nc = 1;
#pragma unroll
              for (int d = 0; d < 3; ++d)
                {
                  const int o = (c >> d) & 1;
                  cnt[d]      = d < DIM ? (tl.T[d] - o + 1) / 2 : (o ? 0 : 1);
                  nc *= cnt[d];
                }
              if (c < col)
                pre += nc;
              else
                n = nc;
            }
          col_n[col]   = n;
          col_pre[col] = pre;
          for (int idx = 0; idx < n && idx < CPC; ++idx)
            {
              const int ix = idx % cnt[0], iy = (idx / cnt[0]) % cnt[1], iz = idx / (cnt[0] * cnt[1]);
              const int cx = 2 * ix + (col & 1), cy = 2 * iy + ((col >> 1) & 1), cz = 2 * iz + ((col >> 2) & 1);
              col_cell[col][idx] = cx | (cy << 8) | (cz << 16);
            }
        }
      if (threadIdx.x == 0)
        {
          for (int st = 0; st < STG; ++st)
            mbar_init(smem_u32(&bars[st]), 1);
          asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
      for (int idx = threadIdx.x; idx < S::NB * NTP; idx += blockDim.x)
        bout[idx] = 0.0f;
      __syncthreads();

      // phase k: the colour phase's records by one bulk copy (thread 0) and,
      // for a tile's first colour, the tile's input brick (cp.async group)
      auto issue = [&](int k) {
        if (k < phases)
          {
            const int tile = blockIdx.x + (k / NC) * gridDim.x;
            const int col  = k % NC;
            if (threadIdx.x == 0)
              {
                const unsigned bar   = smem_u32(&bars[k % STG]);
                const unsigned bytes = unsigned(col_n[col]) * unsigned(rec_bytes);
                if (bytes > 0)
                  {
                    fence_proxy_async_smem();
                    mbar_expect_tx(bar, bytes);
                    bulk_copy_g2s(smem_u32(vk_smem + (k % STG) * stage_bytes),
                                  rec + (tile * tcr + col_pre[col]) * rec_bytes, bytes, bar);
                  }
                else
                  mbar_arrive(bar);
              }
            if (col == 0)
              {
                const TileGeo tg  = tile_geo<DIM, P>(m, tl, tile);
                float        *bi  = bin0 + ((k / NC) & 1) * S::NB * NTP;
                const int     gx  = tg.c0[0] * P + lx;
                const bool    okx = lx < tg.e[0] && gx > 0 && gx < m.nn[0] - 1;
                for (int rb = warp * RPW; rb < ROWS; rb += NW * RPW)
                  {
                    const int row = rb + lrow;
                    if (lrow >= RPW || row >= ROWS)
                      continue;
                    const int i = row / (S::E1 * S::E2), rem = row - i * (S::E1 * S::E2);
                    const int bz = rem / S::E1, by = rem - bz * S::E1;
                    const int gy = tg.c0[1] * P + by, gz = tg.c0[2] * P + bz;
                    bool      ok = okx && by < tg.e[1] && bz < tg.e[2] && gy > 0 && gy < m.nn[1] - 1;
                    if (DIM == 3)
                      ok = ok && gz > 0 && gz < m.nn[2] - 1;
                    const float *gp = ok ? src + i * m.N + gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz) : src;
                    cp_async_small<4>(bi + ((bz * S::E1 + by) * S::E0 + lx) * NTP + i, gp, ok);
                  }
              }
          }
        cp_async_commit();
      };

#pragma unroll
      for (int k = 0; k < STG - 1; ++k)
        issue(k);

      TileGeo tg{};
      int     k = 0;
      for (; k < phases; ++k)
        {
          const bool arrived = mbar_wait(smem_u32(&bars[k % STG]), unsigned(k / STG) & 1u);
          cp_async_wait<STG - 2>();
          // phase k's records and brick visible; phase k-1 done (its stage free, its output adds made)
          if (__syncthreads_or(!arrived))
            break;
          issue(k + STG - 1);

          const int tile = blockIdx.x + (k / NC) * gridDim.x;
          const int col  = k % NC;
          float    *bi   = bin0 + ((k / NC) & 1) * S::NB * NTP;
          if (col == 0)
            {
              tg = tile_geo<DIM, P>(m, tl, tile);
              // the tile's input in the eigenbasis: x <- G x per node
              for (int nd = threadIdx.x; nd < S::NB; nd += blockDim.x)
                {
                  float v[NT];
                  TV::load(bi + nd * NTP, v);
                  time_map<NT>(te.G, v);
                  TV::store(bi + nd * NTP, v);
                }
              __syncthreads();
            }
          const int            n   = col_n[col];
          const unsigned char *stg = vk_smem + (k % STG) * stage_bytes;
          for (int idx = warp; idx < n; idx += NW)
            {
              const int cl = col_cell[col][idx];
              const int cx = cl & 255, cy = (cl >> 8) & 255, cz = cl >> 16;
              if (cx >= tg.tc[0] || cy >= tg.tc[1] || cz >= tg.tc[2])
                continue;
              const unsigned char *r     = stg + idx * rec_bytes;
              const TS            *V     = reinterpret_cast<const TS *>(r);
              const int            bbase = cx * P + S::E0 * (cy * P + S::E1 * (cz * P));

              // pass 1 (lane = mode): y = V x, then the mode's time solve
              {
                const int mm  = lane < ND ? lane : ND - 1;
                const W  *row = reinterpret_cast<const W *>(V + mm * RS);
                W         vw[RWD];
#pragma unroll
                for (int q = 0; q < RWD; ++q)
                  vw[q] = row[q];
                float2 ya[NA], yb[NA];
#pragma unroll
                for (int q = 0; q < NA; ++q)
                  ya[q] = yb[q] = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int a = 0; a < ND; ++a)
                  {
                    const float  v = RW::get(vw[a / RW::PER], a % RW::PER);
                    const float *x = bi + (bbase + S::offset(a)) * NTP;
                    if (a & 1)
                      acc_time<NTP>(yb, v, x);
                    else
                      acc_time<NTP>(ya, v, x);
                  }
                float mu;
                if constexpr (MU_IN_ROW)
                  mu = RW::get(vw[ND / RW::PER], ND % RW::PER);
                else
                  mu = reinterpret_cast<const float *>(r + mu_off)[mm];
                float y[NT];
#pragma unroll
                for (int i = 0; i < NT; ++i)
                  y[i] = (i & 1) ? ya[i / 2].y + yb[i / 2].y : ya[i / 2].x + yb[i / 2].x;
                mode_scale<NT, NR>(te, mu, y);
                if (lane < ND)
                  TV::store(wb + lane * NTP, y);
              }
              __syncwarp();
              // pass 2 (lane = dof): out = V^T w, added into the output brick
              {
                const int a = lane < ND ? lane : ND - 1;
                float2    oa[NA], ob[NA];
#pragma unroll
                for (int q = 0; q < NA; ++q)
                  oa[q] = ob[q] = make_float2(0.0f, 0.0f);
#pragma unroll 9
                for (int mm = 0; mm < ND; ++mm)
                  {
                    const float v = load_s(V + mm * RS + a);
                    if (mm & 1)
                      acc_time<NTP>(ob, v, wb + mm * NTP);
                    else
                      acc_time<NTP>(oa, v, wb + mm * NTP);
                  }
                if (lane < ND)
                  {
                    float *o = bout + (bbase + S::offset(a)) * NTP;
                    float  cur[NT];
                    TV::load(o, cur);
#pragma unroll
                    for (int i = 0; i < NT; ++i)
                      cur[i] += (i & 1) ? oa[i / 2].y + ob[i / 2].y : oa[i / 2].x + ob[i / 2].x;
                    TV::store(o, cur);
                  }
              }
              __syncwarp();
            }
          if (col == NC - 1)
            {
              __syncthreads();
              row_tile_output<DIM, P, NT, S>(m, tl, te, tg, tile, bout, dst, shell, om, NW);
              __syncthreads();
              for (int idx = threadIdx.x; idx < S::NB * NTP; idx += blockDim.x)
                bout[idx] = 0.0f;
            }
        }
      if (k < phases)
        {
          // a record copy did not arrive in time: flag it, wait (bounded) for
          // the copies this CTA issued and return
          if (threadIdx.x == 0)
            {
              atomicExch(fault, 1);
              const int last = min(phases, k + STG - 1);
              for (int j = k; j < last; ++j)
                mbar_wait(smem_u32(&bars[j % STG]), unsigned(j / STG) & 1u);
            }
          __syncthreads();
        }
      cp_async_wait<0>();
    }

    // Small-tile apply over the row records, for meshes whose colour-phase
    // tiles leave most SMs idle: tiles of 2^dim cells, one cell per colour,
    // whose 2^dim records arrive together, and one warp per cell for all of
    // them at once. Each cell's V^T w goes to a slot of its own; each brick
    // node then sums the slots of its cells in colour order, the order in
    // which the colour phases of vanka_row_kernel add them. A tile costs one
    // cell's latency instead of 2^dim phases of it. Records, input brick, G
    // and S maps, output modes and face slots as in vanka_row_kernel.
    template <int DIM, int P, typename TS, int NT>
    __global__ void __launch_bounds__(32 << DIM)
    vanka_slot_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeEig te,
                      const unsigned char *__restrict__ rec, int rec_bytes, int mu_off, const float *__restrict__ src,
                      float *__restrict__ dst, float *__restrict__ shell, const OutMode<float> om)
    {
      using S            = TileShape<DIM, P, 2, 2, 2>;
      using TV           = TimeVec<NT>;
      using RW           = RowWord<TS>;
      using W            = typename RW::W;
      constexpr int ND   = S::ND;
      constexpr int NTP  = TV::NTP;
      constexpr int NA   = (NTP + 1) / 2;
      constexpr int NR   = NT % 2;
      constexpr int NC   = 1 << DIM;
      constexpr int P1   = P + 1;
      constexpr int RS   = vk_row_stride<TS>(ND);
      constexpr int RWD  = RS / RW::PER;
      constexpr int RPW  = 32 / S::E0;
      constexpr int ROWS = NT * S::E1 * S::E2;
      constexpr bool MU_IN_ROW = sizeof(TS) == 4;
      static_assert(ND <= 32, "small-tile apply: at most 32 dofs per cell");
      static_assert(S::E0 <= 32, "brick rows wider than a warp");
      extern __shared__ __align__(16) unsigned char vk_smem[];
      // records [NC][rec_bytes] | brick [NB][NTP] (input, then output) |
      // slots [NC][ND][NTP] | mode values [NC][ND][NTP]
      float    *brick = reinterpret_cast<float *>(vk_smem + NC * rec_bytes);
      float    *slots = brick + S::NB * NTP;
      float    *wbuf  = slots + NC * ND * NTP;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int lrow = lane / S::E0, lx = lane - lrow * S::E0;
      const int cx = warp & 1, cy = (warp >> 1) & 1, cz = (warp >> 2) & 1; // this warp's cell (= colour)
      const int r16 = NC * rec_bytes / 16;

      for (int tile = blockIdx.x; tile < tl.n_tiles; tile += gridDim.x)
        {
          const TileGeo tg = tile_geo<DIM, P>(m, tl, tile);
          // the tile's records (slot c holds the cell of colour c) and its
          // input brick, one group of asynchronous copies
          const unsigned char *g = rec + (long long)tile * NC * rec_bytes;
          for (int q = threadIdx.x; q < r16; q += blockDim.x)
            cp_async16(vk_smem + 16 * q, g + 16 * q);
          {
            const int  gx  = tg.c0[0] * P + lx;
            const bool okx = lx < tg.e[0] && gx > 0 && gx < m.nn[0] - 1;
            for (int rb = warp * RPW; rb < ROWS; rb += NC * RPW)
              {
                const int row = rb + lrow;
                if (lrow >= RPW || row >= ROWS)
                  continue;
                const int i = row / (S::E1 * S::E2), rem = row - i * (S::E1 * S::E2);
                const int bz = rem / S::E1, by = rem - bz * S::E1;
                const int gy = tg.c0[1] * P + by, gz = tg.c0[2] * P + bz;
                bool      ok = okx && by < tg.e[1] && bz < tg.e[2] && gy > 0 && gy < m.nn[1] - 1;
                if (DIM == 3)
                  ok = ok && gz > 0 && gz < m.nn[2] - 1;
                const float *gp = ok ? src + i * m.N + gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz) : src;
                cp_async_small<4>(brick + ((bz * S::E1 + by) * S::E0 + lx) * NTP + i, gp, ok);
              }
          }
          cp_async_commit();
          cp_async_wait<0>();
          __syncthreads();
          // the input in the eigenbasis: x <- G x per node
          for (int nd = threadIdx.x; nd < S::NB; nd += blockDim.x)
            {
              float v[NT];
              TV::load(brick + nd * NTP, v);
              time_map<NT>(te.G, v);
              TV::store(brick + nd * NTP, v);
            }
          __syncthreads();
          const bool live = cx < tg.tc[0] && cy < tg.tc[1] && (DIM < 3 || cz < tg.tc[2]);
          if (live)
            {
              const unsigned char *r     = vk_smem + warp * rec_bytes;
              const TS            *V     = reinterpret_cast<const TS *>(r);
              const int            bbase = cx * P + S::E0 * (cy * P + S::E1 * (cz * P));
              float               *wb    = wbuf + warp * ND * NTP;
              // pass 1 (lane = mode): y = V x, then the mode's time solve
              {
                const int mm  = lane < ND ? lane : ND - 1;
                const W  *row = reinterpret_cast<const W *>(V + mm * RS);
                W         vw[RWD];
#pragma unroll
                for (int q = 0; q < RWD; ++q)
                  vw[q] = row[q];
                float2 ya[NA], yb[NA];
#pragma unroll
                for (int q = 0; q < NA; ++q)
                  ya[q] = yb[q] = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int a = 0; a < ND; ++a)
                  {
                    const float  v = RW::get(vw[a / RW::PER], a % RW::PER);
                    const float *x = brick + (bbase + S::offset(a)) * NTP;
                    if (a & 1)
                      acc_time<NTP>(yb, v, x);
                    else
                      acc_time<NTP>(ya, v, x);
                  }
                float mu;
                if constexpr (MU_IN_ROW)
                  mu = RW::get(vw[ND / RW::PER], ND % RW::PER);
                else
                  mu = reinterpret_cast<const float *>(r + mu_off)[mm];
                float y[NT];
#pragma unroll
                for (int i = 0; i < NT; ++i)
                  y[i] = (i & 1) ? ya[i / 2].y + yb[i / 2].y : ya[i / 2].x + yb[i / 2].x;
                mode_scale<NT, NR>(te, mu, y);
                if (lane < ND)
                  TV::store(wb + lane * NTP, y);
              }
              __syncwarp();
              // pass 2 (lane = dof): V^T w into this cell's slot
              {
                const int a = lane < ND ? lane : ND - 1;
                float2    oa[NA], ob[NA];
#pragma unroll
                for (int q = 0; q < NA; ++q)
                  oa[q] = ob[q] = make_float2(0.0f, 0.0f);
#pragma unroll 9
                for (int mm = 0; mm < ND; ++mm)
                  {
                    const float v = load_s(V + mm * RS + a);
                    if (mm & 1)
                      acc_time<NTP>(ob, v, wb + mm * NTP);
                    else
                      acc_time<NTP>(oa, v, wb + mm * NTP);
                  }
                if (lane < ND)
                  {
                    float o[NT];
#pragma unroll
                    for (int i = 0; i < NT; ++i)
                      o[i] = (i & 1) ? oa[i / 2].y + ob[i / 2].y : oa[i / 2].x + ob[i / 2].x;
                    TV::store(slots + (warp * ND + lane) * NTP, o);
                  }
              }
            }
          __syncthreads();
          // each brick node: the slots of its live cells in colour order
          // (into the brick buffer, whose input nobody reads any more)
          for (int nd = threadIdx.x; nd < S::NB; nd += blockDim.x)
            {
              const int bx = nd % S::E0, by = (nd / S::E0) % S::E1, bz = nd / (S::E0 * S::E1);
              float     acc[NT];
#pragma unroll
              for (int i = 0; i < NT; ++i)
                acc[i] = 0.0f;
#pragma unroll
              for (int c = 0; c < NC; ++c)
                {
                  const int ux = c & 1, uy = (c >> 1) & 1, uz = (c >> 2) & 1;
                  const int ax = bx - ux * P, ay = by - uy * P, az = bz - uz * P;
                  bool      in = ax >= 0 && ax <= P && ay >= 0 && ay <= P && ux < tg.tc[0] && uy < tg.tc[1];
                  if (DIM == 3)
                    in = in && az >= 0 && az <= P && uz < tg.tc[2];
                  if (in)
                    {
                      const int a = ax + P1 * (ay + (DIM == 3 ? P1 * az : 0));
                      float     o[NT];
                      TV::load(slots + (c * ND + a) * NTP, o);
#pragma unroll
                      for (int i = 0; i < NT; ++i)
                        acc[i] += o[i];
                    }
                }
              TV::store(brick + nd * NTP, acc);
            }
          __syncthreads();
          row_tile_output<DIM, P, NT, S>(m, tl, te, tg, tile, brick, dst, shell, om, NC);
          __syncthreads();
        }
      cp_async_wait<0>();
    }

    template <int DIM, int P, typename TS, int NT>
    void
    launch_slot(const Vanka &vk, const float *src, float *dst, const OutMode<float> &om, cudaStream_t s)
    {
      if constexpr (Tens<P + 1, DIM>::ND <= 32)
        {
          const MeshView   &m    = vk.mesh->v;
          const Tiling     &tl   = vk.tiling;
          const std::size_t smem = vk.smem_bytes(vk.shape);
          auto              kern = vanka_slot_kernel<DIM, P, TS, NT>;
          const unsigned    grid = persistent_grid(reinterpret_cast<const void *>(kern), 32 << DIM, smem, tl.n_tiles);
          kern<<<grid, 32 << DIM, smem, s>>>(m, tl, vk.teig, vk.V.ptr, vk.rec_bytes, vk.mu_off, src, dst,
                                             reinterpret_cast<float *>(vk.shell.ptr), om);
          count_launch();
          STMG_CUDA(cudaGetLastError());
          if (tl.n_tiles > 1)
            launch_plane_fixup<DIM, float, true>(m, tl, vk.nt, reinterpret_cast<float *>(vk.shell.ptr), dst, om, s);
        }
      else
        throw Error(STMG_ERR_UNSUPPORTED, "vanka: row records need at most 32 dofs per cell");
    }

    // ---------------------------------------------- tensor-core apply
    __device__ __forceinline__ void
    ldsm_x4(unsigned addr, unsigned (&r)[4])
    {
      asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                   : "r"(addr));
    }

    __device__ __forceinline__ void
    ldsm_x4_trans(unsigned addr, unsigned (&r)[4])
    {
      asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                   : "r"(addr));
    }

    // d += a b for one m16n8k16 tile, BF16 operands, FP32 accumulation
    __device__ __forceinline__ void
    mma_bf16_16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
    {
      asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                   "{%8, %9}, {%0, %1, %2, %3};\n"
                   : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                   : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }

    // two floats as packed BF16 (lo in the low half), rounded to nearest
    __device__ __forceinline__ unsigned
    pack_bf16(float lo, float hi)
    {
      const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
      return *reinterpret_cast<const unsigned *>(&v);
    }

    // the rounding residuals x - bf16(x) of a packed pair, packed again
    __device__ __forceinline__ unsigned
    pack_bf16_residual(float lo, float hi, unsigned h)
    {
      return pack_bf16(lo - __uint_as_float(h << 16), hi - __uint_as_float(h & 0xffff0000u));
    }

    // Tensor-core apply for BF16 records (row records of MmaRows<KT>, 3 or 4
    // time dofs): the streamed colour phases of the row-record apply with the
    // two per-cell products on the tensor cores, one warp per cell:
    //   pass 1  Y = V [x_hi | x_lo]  (m16n8k16, modes x 8 columns, K = dofs),
    //           x = G x_in split into two BF16 parts per node when the tile's
    //           brick arrives (x_hi + x_lo keeps ~16 significant bits), so
    //           Y's column pairs t and t+4 add to the FP32-accurate V x;
    //   scale   w = (mu Lambda + I)^{-1} y per mode (complex pairs first);
    //   pass 2  out = V^T [w_hi | w_lo], added into the output brick;
    // the tile's output is mapped back by S when it is written.
    // Fragment layouts (PTX ISA, mma.m16n8k16 .bf16): lane = 4 g + t holds
    // A(g, 2t..2t+1), A(g+8, ..), A(g, 2t+8..), A(g+8, 2t+8..); B(2t..2t+1, g),
    // B(2t+8..2t+9, g); C(g, 2t..2t+1), C(g+8, 2t..2t+1).
    template <int DIM, int P, int NT, int TX, int TY, int TZ, int STG>
    __global__ void __launch_bounds__(VR_WARPS * 32, 2)
    vanka_mma_kernel(const MeshView m, const Tiling tl, const __grid_constant__ TimeEig te,
                     const unsigned char *__restrict__ rec, int rec_bytes, int mu_off, int cpc,
                     const float *__restrict__ src, float *__restrict__ dst, float *__restrict__ shell,
                     const OutMode<float> om, int *__restrict__ fault)
    {
      using S           = TileShape<DIM, P, TX, TY, TZ>;
      using TV          = TimeVec<NT>;
      constexpr int ND  = S::ND;
      constexpr int NTP = 4;
      constexpr int KT  = ND <= 16 ? 16 : 32; // padded modes / dofs
      constexpr int NKT = KT / 16;            // m16n8k16 tiles per dimension
      constexpr int NR  = NT % 2;             // one real eigenvalue for odd n_t, last
      constexpr int NPT = NT - NR;            // time dofs in complex pairs
      constexpr int NC  = 1 << DIM;
      constexpr int CPC = ((TX + 1) / 2) * ((TY + 1) / 2) * (DIM == 3 ? (TZ + 1) / 2 : 1);
      constexpr int NW  = VR_WARPS;
      constexpr int RPW = 32 / S::E0;
      constexpr int ROWS = NT * S::E1 * S::E2;
      using MR          = MmaRows<KT>;
      static_assert(TV::NTP == 4, "tensor-core apply: 3 or 4 time dofs");
      static_assert(ND <= 32, "tensor-core apply: at most 32 dofs per cell");
      extern __shared__ __align__(16) unsigned char vk_smem[];
      __shared__ int                             col_n[NC], col_pre[NC], col_cell[NC][CPC];
      __shared__ __align__(8) unsigned long long bars[STG];
      const int       warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int       g = lane >> 2, t = lane & 3;
      const int       lrow = lane / S::E0, lx = lane - lrow * S::E0;
      const long long stage_bytes = (long long)cpc * rec_bytes;
      float          *bin0 = reinterpret_cast<float *>(vk_smem + STG * stage_bytes);
      float          *bout = bin0 + 2 * S::NB * NTP;
      unsigned char  *wbw  = reinterpret_cast<unsigned char *>(bout + S::NB * NTP) + warp * 32 * 16; // [32 modes][8 bf16]
      unsigned char  *zero = reinterpret_cast<unsigned char *>(bout + S::NB * NTP) + NW * 32 * 16;  // 128 zero bytes
      const long long tcr  = (long long)tl.T[0] * tl.T[1] * tl.T[2];
      const int       my_tiles = int(blockIdx.x) < tl.n_tiles ? int((tl.n_tiles - 1 - blockIdx.x) / gridDim.x) + 1 : 0;
      const int       phases   = my_tiles * NC;

      // brick offsets (cell-relative) of this lane's dofs: pass-1 B rows
      // d = 16 kt + 2t + {0, 1, 8, 9}; output rows d = g + 8 i
      int  boff[NKT][4], ooff[NKT * 2];
      bool bok[NKT][4], ook[NKT * 2];
#pragma unroll
      for (int kt = 0; kt < NKT; ++kt)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          {
            const int d  = 16 * kt + 2 * t + (q & 1) + 8 * (q >> 1);
            bok[kt][q]   = d < ND;
            boff[kt][q]  = S::offset(d < ND ? d : 0);
          }
#pragma unroll
      for (int i = 0; i < NKT * 2; ++i)
        {
          const int d = g + 8 * i;
          ook[i]      = d < ND;
          ooff[i]     = S::offset(d < ND ? d : 0);
        }

      if (threadIdx.x < NC)
        {
          const int col = threadIdx.x;
          int       cnt[3], n = 1, pre = 0;
          for (int c = 0; c <= col; ++c)
            {
              int nc = 1;
#pragma unroll
              for (int d = 0; d < 3; ++d)
                {
                  const int o = (c >> d) & 1;
                  cnt[d]      = d < DIM ? (tl.T[d] - o + 1) / 2 : (o ? 0 : 1);
                  nc *= cnt[d];
                }
              if (c < col)
                pre += nc;
              else
                n = nc;
            }
          col_n[col]   = n;
          col_pre[col] = pre;
          for (int idx = 0; idx < n && idx < CPC; ++idx)
            {
              const int ix = idx % cnt[0], iy = (idx / cnt[0]) % cnt[1], iz = idx / (cnt[0] * cnt[1]);
              const int cx = 2 * ix + (col & 1), cy = 2 * iy + ((col >> 1) & 1), cz = 2 * iz + ((col >> 2) & 1);
              col_cell[col][idx] = cx | (cy << 8) | (cz << 16);
            }
        }
      if (threadIdx.x == 0)
        {
          for (int st = 0; st < STG; ++st)
            mbar_init(smem_u32(&bars[st]), 1);
          asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
      for (int idx = threadIdx.x; idx < S::NB * NTP; idx += blockDim.x)
        bout[idx] = 0.0f;
      // the per-warp w buffers (rows of modes >= nd stay zero) and the zero block
      for (int idx = threadIdx.x; idx < (NW * 32 * 16 + 128) / 4; idx += blockDim.x)
        reinterpret_cast<unsigned *>(bout + S::NB * NTP)[idx] = 0u;
      __syncthreads();

      auto issue = [&](int k) {
        if (k < phases)
          {
            const int tile = blockIdx.x + (k / NC) * gridDim.x;
            const int col  = k % NC;
            if (threadIdx.x == 0)
              {
                const unsigned bar   = smem_u32(&bars[k % STG]);
                const unsigned bytes = unsigned(col_n[col]) * unsigned(rec_bytes);
                if (bytes > 0)
                  {
                    fence_proxy_async_smem();
                    mbar_expect_tx(bar, bytes);
                    bulk_copy_g2s(smem_u32(vk_smem + (k % STG) * stage_bytes),
                                  rec + (tile * tcr + col_pre[col]) * rec_bytes, bytes, bar);
                  }
                else
                  mbar_arrive(bar);
              }
            if (col == 0)
              {
                const TileGeo tg  = tile_geo<DIM, P>(m, tl, tile);
                float        *bi  = bin0 + ((k / NC) & 1) * S::NB * NTP;
                const int     gx  = tg.c0[0] * P + lx;
                const bool    okx = lx < tg.e[0] && gx > 0 && gx < m.nn[0] - 1;
                for (int rb = warp * RPW; rb < ROWS; rb += NW * RPW)
                  {
                    const int row = rb + lrow;
                    if (lrow >= RPW || row >= ROWS)
                      continue;
                    const int i = row / (S::E1 * S::E2), rem = row - i * (S::E1 * S::E2);
                    const int bz = rem / S::E1, by = rem - bz * S::E1;
                    const int gy = tg.c0[1] * P + by, gz = tg.c0[2] * P + bz;
                    bool      ok = okx && by < tg.e[1] && bz < tg.e[2] && gy > 0 && gy < m.nn[1] - 1;
                    if (DIM == 3)
                      ok = ok && gz > 0 && gz < m.nn[2] - 1;
                    const float *gp = ok ? src + i * m.N + gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz) : src;
                    cp_async_small<4>(bi + ((bz * S::E1 + by) * S::E0 + lx) * NTP + i, gp, ok);
                  }
              }
          }
        cp_async_commit();
      };

#pragma unroll
      for (int k = 0; k < STG - 1; ++k)
        issue(k);

      TileGeo tg{};
      int     k = 0;
      for (; k < phases; ++k)
        {
          const bool arrived = mbar_wait(smem_u32(&bars[k % STG]), unsigned(k / STG) & 1u);
          cp_async_wait<STG - 2>();
          if (__syncthreads_or(!arrived))
            break;
          issue(k + STG - 1);

          const int tile = blockIdx.x + (k / NC) * gridDim.x;
          const int col  = k % NC;
          float    *bi   = bin0 + ((k / NC) & 1) * S::NB * NTP;
          if (col == 0)
            {
              tg = tile_geo<DIM, P>(m, tl, tile);
              // the tile's input in the eigenbasis, split in BF16 parts: per
              // node 8 BF16 (G x rounded, then the rounding residuals) in
              // place of the node's four FP32 values
              for (int nd = threadIdx.x; nd < S::NB; nd += blockDim.x)
                {
                  float v[NT];
                  TV::load(bi + nd * NTP, v);
                  time_map<NT>(te.G, v);
                  float w4[4] = {v[0], NT > 1 ? v[1] : 0.0f, NT > 2 ? v[2] : 0.0f, NT > 3 ? v[NT - 1] : 0.0f};
                  if (NT == 3)
                    w4[3] = 0.0f;
                  const unsigned h0 = pack_bf16(w4[0], w4[1]), h1 = pack_bf16(w4[2], w4[3]);
                  const unsigned l0 = pack_bf16_residual(w4[0], w4[1], h0), l1 = pack_bf16_residual(w4[2], w4[3], h1);
                  *reinterpret_cast<uint4 *>(bi + nd * NTP) = make_uint4(h0, h1, l0, l1);
                }
              __syncthreads();
            }
          const int            n   = col_n[col];
          const unsigned char *stg = vk_smem + (k % STG) * stage_bytes;
          const unsigned short *xb = reinterpret_cast<const unsigned short *>(bi); // 8 BF16 per node
          for (int idx = warp; idx < n; idx += NW)
            {
              const int cl = col_cell[col][idx];
              const int cx = cl & 255, cy = (cl >> 8) & 255, cz = cl >> 16;
              if (cx >= tg.tc[0] || cy >= tg.tc[1] || cz >= tg.tc[2])
                continue;
              const unsigned char *r     = stg + idx * rec_bytes;
              const unsigned       rs    = smem_u32(r), zs = smem_u32(zero);
              const int            bbase = cx * P + S::E0 * (cy * P + S::E1 * (cz * P));

              // pass 1: Y = V X, modes x (4 hi + 4 lo columns)
              float y[NKT][4];
#pragma unroll
              for (int mt = 0; mt < NKT; ++mt)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                  y[mt][q] = 0.0f;
#pragma unroll
              for (int kt = 0; kt < NKT; ++kt)
                {
                  // B: X(d, g) for d = 16 kt + 2t + {0, 1, 8, 9}
                  unsigned short xv[4];
#pragma unroll
                  for (int q = 0; q < 4; ++q)
                    xv[q] = bok[kt][q] ? xb[(bbase + boff[kt][q]) * 8 + g] : (unsigned short)0;
                  const unsigned b0 = unsigned(xv[0]) | (unsigned(xv[1]) << 16);
                  const unsigned b1 = unsigned(xv[2]) | (unsigned(xv[3]) << 16);
#pragma unroll
                  for (int mt = 0; mt < NKT; ++mt)
                    {
                      // A: V rows 16 mt + 8 (j & 1) + r, dof chunk 2 kt + (j >> 1)
                      const int j = lane >> 3, rr = lane & 7;
                      const int mrow = 16 * mt + 8 * (j & 1) + rr;
                      const unsigned ad = mrow < ND ? rs + unsigned(MR::offset(mrow, 16 * kt + 8 * (j >> 1)))
                                                    : zs + unsigned(16 * rr);
                      unsigned a[4];
                      ldsm_x4(ad, a);
                      mma_bf16_16816(y[mt], a, b0, b1);
                    }
                }
              // columns t and t + 4 (lanes t and t ^ 2) add up: V x for times
              // 2 (t & 1), 2 (t & 1) + 1 of modes 16 mt + g (+ 8)
              const int tau = 2 * (t & 1);
#pragma unroll
              for (int mt = 0; mt < NKT; ++mt)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                  y[mt][q] += __shfl_xor_sync(0xffffffffu, y[mt][q], 2);
              // time solves: w = (mu Lambda + I)^{-1} y in the pair (tau, tau + 1)
              const float *mu = reinterpret_cast<const float *>(r + mu_off);
#pragma unroll
              for (int mt = 0; mt < NKT; ++mt)
#pragma unroll
                for (int hh = 0; hh < 2; ++hh)
                  {
                    const int   mode = 16 * mt + g + 8 * hh;
                    const float mm   = mu[mode < ND ? mode : 0];
                    float       u = y[mt][2 * hh], v = y[mt][2 * hh + 1];
                    if (tau + 1 < NPT)
                      {
                        const float d = fmaf(mm, te.a[tau], 1.0f), e = mm * te.b[tau];
                        const float inv = rcp_approx(fmaf(d, d, e * e));
                        const float wu = inv * fmaf(d, u, -e * v), wv = inv * fmaf(e, u, d * v);
                        u = wu;
                        v = wv;
                      }
                    else if (tau < NT)
                      {
                        u *= rcp_approx(fmaf(mm, te.a[tau], 1.0f));
                        v = 0.0f;
                      }
                    else
                      u = v = 0.0f;
                    // lanes t < 2 store the BF16 parts, lanes t >= 2 the residuals
                    if (mode < ND)
                      {
                        const unsigned h = pack_bf16(u, v);
                        const unsigned o = t < 2 ? h : pack_bf16_residual(u, v, h);
                        *reinterpret_cast<unsigned *>(wbw + mode * 16 + (t < 2 ? 0 : 8) + 2 * tau) = o;
                      }
                  }
              __syncwarp();

              // pass 2: out = V^T W, dofs x (4 hi + 4 lo columns)
              float o[NKT][4];
#pragma unroll
              for (int mt = 0; mt < NKT; ++mt)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                  o[mt][q] = 0.0f;
              const unsigned short *wb16 = reinterpret_cast<const unsigned short *>(wbw);
#pragma unroll
              for (int kt = 0; kt < NKT; ++kt)
                {
                  // B: W(mode, g) for mode = 16 kt + 2t + {0, 1, 8, 9}
                  const int      m0 = 16 * kt + 2 * t;
                  const unsigned b0 = unsigned(wb16[m0 * 8 + g]) | (unsigned(wb16[(m0 + 1) * 8 + g]) << 16);
                  const unsigned b1 = unsigned(wb16[(m0 + 8) * 8 + g]) | (unsigned(wb16[(m0 + 9) * 8 + g]) << 16);
#pragma unroll
                  for (int mt = 0; mt < NKT; ++mt)
                    {
                      // A = V^T: rows (modes) 16 kt + 8 (j >> 1) + r of V, dof chunk 2 mt + (j & 1), transposed
                      const int j = lane >> 3, rr = lane & 7;
                      const int mrow = 16 * kt + 8 * (j >> 1) + rr;
                      const unsigned ad = mrow < ND ? rs + unsigned(MR::offset(mrow, 16 * mt + 8 * (j & 1)))
                                                    : zs + unsigned(16 * rr);
                      unsigned a[4];
                      ldsm_x4_trans(ad, a);
                      mma_bf16_16816(o[mt], a, b0, b1);
                    }
                }
#pragma unroll
              for (int mt = 0; mt < NKT; ++mt)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                  o[mt][q] += __shfl_xor_sync(0xffffffffu, o[mt][q], 2);
              if (t < 2)
                {
#pragma unroll
                  for (int mt = 0; mt < NKT; ++mt)
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh)
                      {
                        const int i = 2 * mt + hh; // dof g + 8 i
                        if (!ook[i])
                          continue;
                        float2 *ob  = reinterpret_cast<float2 *>(bout + (bbase + ooff[i]) * NTP + tau);
                        float2  cur = *ob;
                        cur.x += o[mt][2 * hh];
                        cur.y += o[mt][2 * hh + 1];
                        *ob = cur;
                      }
                }
              __syncwarp();
            }
          if (col == NC - 1)
            {
              __syncthreads();
              const int  gx  = tg.c0[0] * P + lx;
              const int  vx  = (gx % P == 0) ? 2 : 1;
              const bool inx = lx > 0 && lx < tg.e[0] - 1;
              for (int rb = warp * RPW; rb < S::E1 * S::E2; rb += NW * RPW)
                {
                  const int row = rb + lrow;
                  if (lrow >= RPW || row >= S::E1 * S::E2 || lx >= tg.e[0])
                    continue;
                  const int bz = row / S::E1, by = row - bz * S::E1;
                  if (by >= tg.e[1] || bz >= tg.e[2])
                    continue;
                  bool inte = inx && by > 0 && by < tg.e[1] - 1;
                  if (DIM == 3)
                    inte = inte && bz > 0 && bz < tg.e[2] - 1;
                  const int gy = tg.c0[1] * P + by, gz = tg.c0[2] * P + bz;
                  int       v  = vx * ((gy % P == 0) ? 2 : 1);
                  if (DIM == 3)
                    v *= (gz % P == 0) ? 2 : 1;
                  const float w = v == 1 ? 1.0f : (v == 2 ? 0.5f : (v == 4 ? 0.25f : 0.125f));
                  float       ov[NT];
                  TV::load(bout + ((bz * S::E1 + by) * S::E0 + lx) * NTP, ov);
                  time_map<NT>(te.S, ov);
                  const long long gi = gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz);
                  if (inte)
                    {
#pragma unroll
                      for (int jt = 0; jt < NT; ++jt)
                        ov[jt] *= w;
                      om.write_n(dst, gi, m.N, ov);
                    }
                  else if (tl.n_tiles == 1)
                    om.template write_constrained_n<NT>(dst, gi, m.N);
                  else
                    {
                      float *sj = shell + (long long)tile * NT * tl.tile_stride + shell_slot<DIM>(tl, tg.e, lx, by, bz);
#pragma unroll
                      for (int jt = 0; jt < NT; ++jt, sj += tl.tile_stride)
                        *sj = ov[jt];
                    }
                }
              __syncthreads();
              for (int idx = threadIdx.x; idx < S::NB * NTP; idx += blockDim.x)
                bout[idx] = 0.0f;
            }
        }
      if (k < phases)
        {
          if (threadIdx.x == 0)
            {
              atomicExch(fault, 1);
              const int last = min(phases, k + STG - 1);
              for (int j = k; j < last; ++j)
                mbar_wait(smem_u32(&bars[j % STG]), unsigned(j / STG) & 1u);
            }
          __syncthreads();
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

    template <int DIM, int P, typename TS, int NT, bool BIG>
    void
    launch_stream(const Vanka &vk, const float *src, float *dst, const OutMode<float> &om, cudaStream_t s)
    {
      using Sh = VkShape<DIM, P, BIG>;
      const MeshView   &m    = vk.mesh->v;
      const Tiling     &tl   = vk.tiling;
      const std::size_t smem = vk.smem_bytes(vk.shape);
      auto              kern = vanka_stream_kernel<DIM, P, TS, NT, Sh::TX, Sh::TY, Sh::TZ>;
      const unsigned    grid = persistent_grid(reinterpret_cast<const void *>(kern), 256, smem, tl.n_tiles);
      kern<<<grid, 256, smem, s>>>(m, tl, vk.tmats<float>(), vk.teig, vk.V.ptr, vk.rec_bytes, vk.mu_off,
                                   vk.colour_cells, src, dst, reinterpret_cast<float *>(vk.shell.ptr), om);
      count_launch();
      STMG_CUDA(cudaGetLastError());
      if (tl.n_tiles > 1)
        launch_plane_fixup<DIM, float, true>(m, tl, vk.nt, reinterpret_cast<float *>(vk.shell.ptr), dst, om, s);
    }

    template <int DIM, int P, typename TS, int NT, bool BIG>
    void
    launch_row(const Vanka &vk, const float *src, float *dst, const OutMode<float> &om, cudaStream_t s)
    {
      using Sh = VkShape<DIM, P, BIG>;
      if constexpr (Tens<P + 1, DIM>::ND <= 32)
        {
          const MeshView   &m    = vk.mesh->v;
          const Tiling     &tl   = vk.tiling;
          const std::size_t smem = vk.smem_bytes(vk.shape);
          auto kern = vk.stages >= 5 ? vanka_row_kernel<DIM, P, TS, NT, Sh::TX, Sh::TY, Sh::TZ, 5>
                    : vk.stages == 4 ? vanka_row_kernel<DIM, P, TS, NT, Sh::TX, Sh::TY, Sh::TZ, 4>
                                     : vanka_row_kernel<DIM, P, TS, NT, Sh::TX, Sh::TY, Sh::TZ, 3>;
          const unsigned    grid = persistent_grid(reinterpret_cast<const void *>(kern), VR_WARPS * 32, smem, tl.n_tiles);
          kern<<<grid, VR_WARPS * 32, smem, s>>>(m, tl, vk.teig, vk.V.ptr, vk.rec_bytes, vk.mu_off, vk.colour_cells, src,
                                                 dst, reinterpret_cast<float *>(vk.shell.ptr), om,
                                                 vanka_fault_flag_device());
          count_launch();
          STMG_CUDA(cudaGetLastError());
          if (tl.n_tiles > 1)
            launch_plane_fixup<DIM, float, true>(m, tl, vk.nt, reinterpret_cast<float *>(vk.shell.ptr), dst, om, s);
        }
      else
        throw Error(STMG_ERR_UNSUPPORTED, "vanka: row records need at most 32 dofs per cell");
    }

    template <int DIM, int P, int NT, bool BIG>
    void
    launch_mma(const Vanka &vk, const float *src, float *dst, const OutMode<float> &om, cudaStream_t s)
    {
      using Sh = VkShape<DIM, P, BIG>;
      if constexpr (Tens<P + 1, DIM>::ND <= 32 && (NT == 3 || NT == 4))
        {
          const MeshView   &m    = vk.mesh->v;
          const Tiling     &tl   = vk.tiling;
          const std::size_t smem = vk.smem_bytes(vk.shape);
          auto kern = vk.stages >= 5 ? vanka_mma_kernel<DIM, P, NT, Sh::TX, Sh::TY, Sh::TZ, 5>
                    : vk.stages == 4 ? vanka_mma_kernel<DIM, P, NT, Sh::TX, Sh::TY, Sh::TZ, 4>
                                     : vanka_mma_kernel<DIM, P, NT, Sh::TX, Sh::TY, Sh::TZ, 3>;
          const unsigned    grid = persistent_grid(reinterpret_cast<const void *>(kern), VR_WARPS * 32, smem, tl.n_tiles);
          kern<<<grid, VR_WARPS * 32, smem, s>>>(m, tl, vk.teig_pf, vk.V.ptr, vk.rec_bytes, vk.mu_off, vk.colour_cells,
                                                 src, dst, reinterpret_cast<float *>(vk.shell.ptr), om,
                                                 vanka_fault_flag_device());
          count_launch();
          STMG_CUDA(cudaGetLastError());
          if (tl.n_tiles > 1)
            launch_plane_fixup<DIM, float, true>(m, tl, vk.nt, reinterpret_cast<float *>(vk.shell.ptr), dst, om, s);
        }
      else
        throw Error(STMG_ERR_UNSUPPORTED, "vanka: the tensor-core apply needs 3 or 4 time dofs and 32 dofs per cell");
    }

    template <int DIM, int P, typename TS, int NT>
    void
    launch_stream_nt(const Vanka &vk, const float *src, float *dst, const OutMode<float> &om, cudaStream_t s)
    {
      if constexpr (std::is_same_v<TS, __nv_bfloat16>)
        if (vk.mmarec)
          {
            if (vk.big)
              launch_mma<DIM, P, NT, true>(vk, src, dst, om, s);
            else
              launch_mma<DIM, P, NT, false>(vk, src, dst, om, s);
            return;
          }
      if (vk.slotrec)
        return launch_slot<DIM, P, TS, NT>(vk, src, dst, om, s);
      if (vk.rowrec)
        {
          if (vk.big)
            launch_row<DIM, P, TS, NT, true>(vk, src, dst, om, s);
          else
            launch_row<DIM, P, TS, NT, false>(vk, src, dst, om, s);
          return;
        }
      if (vk.big)
        launch_stream<DIM, P, TS, NT, true>(vk, src, dst, om, s);
      else
        launch_stream<DIM, P, TS, NT, false>(vk, src, dst, om, s);
    }

    template <int DIM, int P, typename TS>
    void
    launch_stream_any(const Vanka &vk, const float *src, float *dst, const OutMode<float> &om, cudaStream_t s)
    {
      switch (vk.nt)
        {
          case 1:
            return launch_stream_nt<DIM, P, TS, 1>(vk, src, dst, om, s);
          case 2:
            return launch_stream_nt<DIM, P, TS, 2>(vk, src, dst, om, s);
          case 3:
            return launch_stream_nt<DIM, P, TS, 3>(vk, src, dst, om, s);
          case 4:
            return launch_stream_nt<DIM, P, TS, 4>(vk, src, dst, om, s);
          default:
            throw Error(STMG_ERR_ARG, "vanka: streamed apply needs 1..4 time dofs");
        }
    }

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
      if (vk.streamed)
        {
          if (vk.storage == STMG_BF16)
            return launch_stream_any<DIM, P, __nv_bfloat16>(vk, static_cast<const float *>(src),
                                                             static_cast<float *>(dst), o32, s);
          return launch_stream_any<DIM, P, float>(vk, static_cast<const float *>(src), static_cast<float *>(dst), o32,
                                                  s);
        }
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
