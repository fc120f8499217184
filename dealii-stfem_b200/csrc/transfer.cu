// Multigrid transfers between space-time levels.
//  h: FE_Q(p) interpolation from a mesh to its 2x refinement, per time
//     block, and its transpose (deal.II's MGTwoLevelTransfer as wrapped by
//     MGTwoLevelBlockTransfer, tests/include/gmg.h:35-75); on a structured
//     mesh the global prolongation is the tensor product of 1-D stencils, so
//     both directions run tile by tile in shared memory, one direction at a
//     time (fixed summation order, Dirichlet nodes zero on both sides).
//  t: (P (x) I) over the time blocks (MGTwoLevelTransferST::prolongate_and_add
//     / restrict_and_add, gmg.h:121-135, via tensorproduct_add,
//     operators.h:46-58).
#include <cmath>
#include <cstring>

#include "async_copy.cuh"
#include "kernels_common.cuh"
#include "transfer.h"

namespace stmg
{
  namespace
  {
    template <typename T>
    __global__ void
    time_transfer_kernel(long long N, int n_out, int n_in, const __grid_constant__ TimeMats<T> P,
                         const T *__restrict__ src, T *__restrict__ dst)
    {
      const long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (node >= N)
        return;
      T x[MAX_NT];
      for (int j = 0; j < n_in; ++j)
        x[j] = src[j * N + node];
      for (int i = 0; i < n_out; ++i)
        {
          T acc = dst[i * N + node];
          for (int j = 0; j < n_in; ++j)
            {
              const T a = P.A[i * n_in + j];
              if (a != T(0))
                acc += a * x[j];
            }
          dst[i * N + node] = acc;
        }
    }

    // ---------------------------------------------------- tiled h transfer
    // coarse cells per tile and direction
    template <int DIM, int P, typename T>
    constexpr int h_tile_cells()
    {
      return DIM == 3 ? (P == 1 ? 8 : (P == 2 ? (sizeof(T) == 4 ? 4 : 2) : 2))
                      : (P <= 2 ? 32 / (2 * P) : (P == 3 ? 5 : (P == 4 ? 4 : 3)));
    }

    // dst[off] += v for the items of one pass of a CTA: each thread takes
    // items threadIdx.x + blockDim.x k, KB at a time, and has the KB loads of
    // dst in flight before it stores (one read-add-write per item, as in a
    // plain loop, without a global-memory round trip per item)
    template <int KB, typename T, typename Item>
    __device__ __forceinline__ void
    batched_add(int n, T *__restrict__ dst, const Item &item)
    {
      for (int base = threadIdx.x; base < n; base += KB * blockDim.x)
        {
          long long off[KB];
          T         v[KB], old[KB];
          bool      ok[KB];
#pragma unroll
          for (int k = 0; k < KB; ++k)
            {
              const int i = base + k * blockDim.x;
              ok[k]       = i < n && item(i, off[k], v[k]);
            }
#pragma unroll
          for (int k = 0; k < KB; ++k)
            old[k] = ok[k] ? dst[off[k]] : T(0);
#pragma unroll
          for (int k = 0; k < KB; ++k)
            if (ok[k])
              dst[off[k]] = old[k] + v[k];
        }
    }

    // Prolongation dst_f += P src_c, one CTA per tile of C^dim coarse cells
    // and time dof (blockIdx.y): the coarse block (P C + 1 nodes per
    // direction, Dirichlet nodes zero) is interpolated direction by direction
    // in shared memory (x, then y, then z) and the fine nodes the tile owns
    // are added to dst (Dirichlet nodes skipped). Fine nodes
    // [2PC t, 2PC (t+1)) belong to tile t; the last fine node to the last
    // tile.
    template <int DIM, int P, int C, typename T>
    __global__ void __launch_bounds__(256)
    h_prolongate_tiled(const MeshView fm, const MeshView cm, const __grid_constant__ HWeights<T> W,
                       const T *__restrict__ src, T *__restrict__ dst)
    {
      constexpr int LC = P * C + 1, LF = 2 * P * C + 1;
      constexpr int NZC = DIM == 3 ? LC : 1, NZF = DIM == 3 ? LF : 1;
      __shared__ T sc[NZC * LC * LC], s1[NZC * LC * LF], s2[NZC * LF * LF];
      const int ntx = (cm.n[0] + C - 1) / C, nty = (cm.n[1] + C - 1) / C;
      const int tile = blockIdx.x, j = blockIdx.y;
      const int t0 = tile % ntx, t1 = (tile / ntx) % nty, t2 = DIM == 3 ? tile / (ntx * nty) : 0;
      const int q0[3] = {t0 * C * P, t1 * C * P, t2 * C * P};        // first coarse node
      const int f0[3] = {2 * t0 * C * P, 2 * t1 * C * P, 2 * t2 * C * P}; // first fine node
      for (int i = threadIdx.x; i < NZC * LC * LC; i += blockDim.x)
        {
          const int x = i % LC, y = (i / LC) % LC, z = i / (LC * LC);
          const int g[3] = {q0[0] + x, q0[1] + y, DIM == 3 ? q0[2] + z : 0};
          bool      ok   = g[0] < cm.nn[0] && g[1] < cm.nn[1] && (DIM < 3 || g[2] < cm.nn[2]);
          ok             = ok && !is_boundary_node(cm, g[0], g[1], g[2]);
          cp_async_small<sizeof(T)>(sc + i,
                                    ok ? src + j * cm.N + g[0] + (long long)cm.nn[0] * (g[1] + (long long)cm.nn[1] * g[2])
                                       : src,
                                    ok);
        }
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      // x: sc[z][y][cx] -> s1[z][y][fx]
      for (int i = threadIdx.x; i < NZC * LC * LF; i += blockDim.x)
        {
          const int fx = i % LF, r = i / LF;
          const int cc = min(fx / (2 * P), C - 1), t = fx - 2 * P * cc;
          const T  *in = sc + r * LC + P * cc;
          T         v  = T(0);
#pragma unroll
          for (int b = 0; b <= P; ++b)
            v += W.w[t][b] * in[b];
          s1[i] = v;
        }
      __syncthreads();
      // y: s1[z][cy][fx] -> s2[z][fy][fx]
      for (int i = threadIdx.x; i < NZC * LF * LF; i += blockDim.x)
        {
          const int fx = i % LF, fy = (i / LF) % LF, z = i / (LF * LF);
          const int cc = min(fy / (2 * P), C - 1), t = fy - 2 * P * cc;
          const T  *in = s1 + (z * LC + P * cc) * LF + fx;
          T         v  = T(0);
#pragma unroll
          for (int b = 0; b <= P; ++b)
            v += W.w[t][b] * in[b * LF];
          s2[i] = v;
        }
      __syncthreads();
      // z (3-D): s2[cz][fy][fx] -> fine, added to dst
      batched_add<8>(NZF * LF * LF, dst, [&](int i, long long &off, T &v) {
        const int fx = i % LF, fy = (i / LF) % LF, fz = i / (LF * LF);
        const int g[3] = {f0[0] + fx, f0[1] + fy, DIM == 3 ? f0[2] + fz : 0};
        // owned: below the next tile's first node, or the mesh's last node
        bool own = (fx < LF - 1 || g[0] == fm.nn[0] - 1) && (fy < LF - 1 || g[1] == fm.nn[1] - 1);
        if (DIM == 3)
          own = own && (fz < LF - 1 || g[2] == fm.nn[2] - 1);
        own = own && g[0] < fm.nn[0] && g[1] < fm.nn[1] && (DIM < 3 || g[2] < fm.nn[2]);
        if (!own || is_boundary_node(fm, g[0], g[1], g[2]))
          return false;
        if constexpr (DIM == 3)
          {
            const int cc = min(fz / (2 * P), C - 1), t = fz - 2 * P * cc;
            const T  *in = s2 + (P * cc) * LF * LF + fy * LF + fx;
            v            = T(0);
#pragma unroll
            for (int b = 0; b <= P; ++b)
              v += W.w[t][b] * in[b * LF * LF];
          }
        else
          v = s2[i];
        off = j * fm.N + g[0] + (long long)fm.nn[0] * (g[1] + (long long)fm.nn[1] * g[2]);
        return true;
      });
    }

    // Restriction dst_c += P^T src_f, one CTA per tile of C^dim coarse cells
    // and time dof (blockIdx.y), owning coarse nodes [PC t, PC (t+1)) (the
    // last node to the last tile): the fine block [2P(C t - 1), 2P C (t+1)]
    // per direction (Dirichlet and outside nodes zero) is reduced direction
    // by direction. A coarse vertex collects the fine nodes of both
    // neighbouring coarse cells, the shared fine vertex once. Every pass runs
    // by rows: the fine block's rows over the warps with x over the lanes,
    // the coarse passes GQ rows per warp with the coarse x index over the
    // lanes (a lane's x and its weights fixed), so the index arithmetic is
    // per row, not per entry.
    template <int DIM, int P, int C, typename T>
    __global__ void __launch_bounds__(256)
    h_restrict_tiled(const MeshView fm, const MeshView cm, const __grid_constant__ HWeights<T> W,
                     const T *__restrict__ src, T *__restrict__ dst)
    {
      constexpr int LR = 2 * P * (C + 1) + 1, LQ = P * C + 1;
      constexpr int NZR = DIM == 3 ? LR : 1, NZQ = DIM == 3 ? LQ : 1;
      constexpr int NW = 8;        // warps (the launch has 256 threads)
      constexpr int GQ = 32 / LQ;  // coarse rows per warp step
      static_assert(LQ <= 32, "coarse tile rows wider than a warp");
      extern __shared__ __align__(16) unsigned char hr_smem[];
      T *sf = reinterpret_cast<T *>(hr_smem);
      T *s1 = sf + NZR * LR * LR;   // [z][y][qx]
      T *s2 = s1 + NZR * LR * LQ;   // [z][qy][qx]
      const int ntx = (cm.n[0] + C - 1) / C, nty = (cm.n[1] + C - 1) / C;
      const int tile = blockIdx.x, j = blockIdx.y;
      const int t0 = tile % ntx, t1 = (tile / ntx) % nty, t2 = DIM == 3 ? tile / (ntx * nty) : 0;
      const int q0[3] = {t0 * C * P, t1 * C * P, t2 * C * P};
      const int fo[3] = {2 * P * (t0 * C - 1), 2 * P * (t1 * C - 1), 2 * P * (t2 * C - 1)};
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int lsub = lane / LQ, lq = lane - lsub * LQ; // lane -> (row in the step, coarse x)
      const bool lact = lsub < GQ;
      // one direction of P^T: out[q] from in[f], stride s between fine entries
      auto reduce1 = [&](const T *in, int stride, int qx) {
        const int cl = qx / P, k = qx - P * cl; // coarse cell (local) and index in it
        T         v  = T(0);
        // the cell to the right of / containing the node: fine t = 0..2P
        const T *r = in + (2 * P * (cl + 1)) * stride;
#pragma unroll
        for (int t = 0; t <= 2 * P; ++t)
          v += W.w[t][k] * r[t * stride];
        if (k == 0)
          {
            // the cell to the left: fine t = 0..2P-1
            const T *l = in + (2 * P * cl) * stride;
#pragma unroll
            for (int t = 0; t < 2 * P; ++t)
              v += W.w[t][P] * l[t * stride];
          }
        return v;
      };
      // the fine block: rows (z, y) over the warps, x over the lanes
      // (asynchronous copies, zero fill outside the interior)
      for (int r = warp; r < NZR * LR; r += NW)
        {
          const int       z = r / LR, y = r - z * LR;
          const int       gy = fo[1] + y, gz = DIM == 3 ? fo[2] + z : 0;
          const bool      rin = gy > 0 && gy < fm.nn[1] - 1 && (DIM < 3 || (gz > 0 && gz < fm.nn[2] - 1));
          const long long roff = j * fm.N + (long long)fm.nn[0] * (gy + (long long)fm.nn[1] * gz);
#pragma unroll
          for (int x = lane; x < LR; x += 32)
            {
              const int  gx = fo[0] + x;
              const bool ok = rin && gx > 0 && gx < fm.nn[0] - 1;
              cp_async_small<sizeof(T)>(sf + r * LR + x, ok ? src + (roff + gx) : src, ok);
            }
        }
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      // x: sf[z][y][fx] -> s1[z][y][qx]
      for (int r0 = warp * GQ; r0 < NZR * LR; r0 += NW * GQ)
        {
          const int r = r0 + lsub;
          if (lact && r < NZR * LR)
            s1[r * LQ + lq] = reduce1(sf + r * LR, 1, lq);
        }
      __syncthreads();
      // y: s1[z][fy][qx] -> s2[z][qy][qx]
      for (int r0 = warp * GQ; r0 < NZR * LQ; r0 += NW * GQ)
        {
          const int r = r0 + lsub;
          if (lact && r < NZR * LQ)
            {
              const int z = r / LQ, qy = r - z * LQ;
              s2[r * LQ + lq] = reduce1(s1 + z * LR * LQ + lq, LQ, qy);
            }
        }
      __syncthreads();
      // z (3-D) and the owned coarse nodes added to dst: rows (qz, qy) GQ
      // per warp step, all of a lane's dst loads in flight before its stores
      constexpr int NRQ = NZQ * LQ;
      constexpr int KB  = (NRQ + NW * GQ - 1) / (NW * GQ);
      const int     g0  = q0[0] + lq;
      const bool    ownx = lq < LQ - 1 || g0 == cm.nn[0] - 1;
      const bool    inx  = g0 > 0 && g0 < cm.nn[0] - 1;
      long long     off[KB];
      T             v[KB], old[KB];
      bool          ok[KB];
#pragma unroll
      for (int kb = 0; kb < KB; ++kb)
        {
          const int r = warp * GQ + kb * NW * GQ + lsub;
          ok[kb]      = false;
          if (!lact || r >= NRQ || !ownx || !inx)
            continue;
          const int qz = DIM == 3 ? r / LQ : 0, qy = r - qz * LQ;
          const int g1 = q0[1] + qy, g2 = DIM == 3 ? q0[2] + qz : 0;
          bool      own = (qy < LQ - 1 || g1 == cm.nn[1] - 1) && g1 > 0 && g1 < cm.nn[1] - 1;
          if (DIM == 3)
            own = own && (qz < LQ - 1 || g2 == cm.nn[2] - 1) && g2 > 0 && g2 < cm.nn[2] - 1;
          if (!own)
            continue;
          v[kb]   = DIM == 3 ? reduce1(s2 + qy * LQ + lq, LQ * LQ, qz) : s2[r * LQ + lq];
          off[kb] = j * cm.N + g0 + (long long)cm.nn[0] * (g1 + (long long)cm.nn[1] * g2);
          ok[kb]  = true;
        }
#pragma unroll
      for (int kb = 0; kb < KB; ++kb)
        old[kb] = ok[kb] ? dst[off[kb]] : T(0);
#pragma unroll
      for (int kb = 0; kb < KB; ++kb)
        if (ok[kb])
          dst[off[kb]] = old[kb] + v[kb];
    }

    template <int DIM, int P, typename T>
    void
    h_tiled_launch(bool prolong, const MeshView &f, const MeshView &c, int nt, const HWeights<T> &W, const T *src,
                   T *dst, cudaStream_t s)
    {
      constexpr int C = h_tile_cells<DIM, P, T>();
      long long     tiles = 1;
      for (int d = 0; d < DIM; ++d)
        tiles *= (c.n[d] + C - 1) / C;
      const dim3 grid{unsigned(tiles), unsigned(nt), 1u};
      if (prolong)
        h_prolongate_tiled<DIM, P, C, T><<<grid, 256, 0, s>>>(f, c, W, src, dst);
      else
        {
          constexpr int LR = 2 * P * (C + 1) + 1, LQ = P * C + 1, NZR = DIM == 3 ? LR : 1;
          constexpr std::size_t smem = sizeof(T) * (std::size_t(NZR) * LR * LR + std::size_t(NZR) * LR * LQ +
                                                    std::size_t(NZR) * LQ * LQ);
          auto kern = h_restrict_tiled<DIM, P, C, T>;
          STMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
          kern<<<grid, 256, smem, s>>>(f, c, W, src, dst);
        }
      count_launch();
      STMG_CUDA(cudaGetLastError());
    }

    template <typename T>
    void
    h_tiled(bool prolong, const MeshView &f, const MeshView &c, int nt, const HWeights<T> &W, const T *src, T *dst,
            cudaStream_t s)
    {
#define STMG_HT(D, PP)                                                                                   \
  if (f.dim == D && f.p == PP)                                                                           \
    return h_tiled_launch<D, PP, T>(prolong, f, c, nt, W, src, dst, s);
      STMG_HT(2, 1) STMG_HT(2, 2) STMG_HT(2, 3) STMG_HT(2, 4) STMG_HT(2, 5)
      STMG_HT(3, 1) STMG_HT(3, 2) STMG_HT(3, 3) STMG_HT(3, 4)
#undef STMG_HT
      throw Error(STMG_ERR_UNSUPPORTED, "h-transfer: unsupported dim/degree");
    }
  } // namespace

  HTransfer::HTransfer(Mesh *fine_, Mesh *coarse_, int nt_, int dtype_)
    : fine(fine_)
    , coarse(coarse_)
    , nt(nt_)
    , dtype(dtype_)
  {
    const MeshView &f = fine->v, &c = coarse->v;
    STMG_REQUIRE(f.dim == c.dim && f.p == c.p, STMG_ERR_SHAPE, "h-transfer: meshes differ in dim or degree");
    for (int d = 0; d < f.dim; ++d)
      STMG_REQUIRE(f.n[d] == 2 * c.n[d], STMG_ERR_SHAPE, "h-transfer: fine mesh must be the 2x refinement");
    STMG_REQUIRE(nt >= 1 && nt <= MAX_NT, STMG_ERR_ARG, "h-transfer: time blocks 1..16");
    const FETables &t  = host_tables();
    const int       p  = f.p, p1 = p + 1;
    // 1-D weights of the coarse basis at the fine nodes of a coarse cell
    std::memset(&w64, 0, sizeof(w64));
    std::memset(&w32, 0, sizeof(w32));
    for (int tpos = 0; tpos <= 2 * p; ++tpos)
      {
        const int    half = tpos > p ? 1 : (tpos == p ? 1 : 0);
        const int    a    = tpos - half * p;
        const double xi   = 0.5 * (half + t.xs[p][a]);
        for (int b = 0; b < p1; ++b)
          {
            double v = 1.0;
            for (int k = 0; k < p1; ++k)
              if (k != b)
                v *= (xi - t.xs[p][k]) / (t.xs[p][b] - t.xs[p][k]);
            if (std::abs(v) < 1e-14)
              v = 0.0;
            w64.w[tpos][b] = v;
            w32.w[tpos][b] = float(v);
          }
      }
  }

  void
  HTransfer::prolongate_add(const void *src, void *dst, cudaStream_t s) const
  {
    const MeshView &f = fine->v, &c = coarse->v;
    if (dtype == STMG_F64)
      h_tiled<double>(true, f, c, nt, hw<double>(), static_cast<const double *>(src), static_cast<double *>(dst), s);
    else
      h_tiled<float>(true, f, c, nt, hw<float>(), static_cast<const float *>(src), static_cast<float *>(dst), s);
  }

  void
  HTransfer::restrict_add(const void *src, void *dst, cudaStream_t s) const
  {
    const MeshView &f = fine->v, &c = coarse->v;
    if (dtype == STMG_F64)
      h_tiled<double>(false, f, c, nt, hw<double>(), static_cast<const double *>(src), static_cast<double *>(dst), s);
    else
      h_tiled<float>(false, f, c, nt, hw<float>(), static_cast<const float *>(src), static_cast<float *>(dst), s);
  }

  TTransfer::TTransfer(Mesh *mesh_, int nt_fine_, int nt_coarse_, const double *P_, const double *R_, int dtype_)
    : mesh(mesh_)
    , nt_fine(nt_fine_)
    , nt_coarse(nt_coarse_)
    , dtype(dtype_)
  {
    STMG_REQUIRE(nt_fine >= 1 && nt_fine <= MAX_NT && nt_coarse >= 1 && nt_coarse <= MAX_NT, STMG_ERR_ARG,
                 "t-transfer: time blocks 1..16");
    std::memset(&P64, 0, sizeof(P64));
    std::memset(&R64, 0, sizeof(R64));
    std::memset(&P32, 0, sizeof(P32));
    std::memset(&R32, 0, sizeof(R32));
    for (int i = 0; i < nt_fine; ++i)
      for (int j = 0; j < nt_coarse; ++j)
        {
          P64.A[i * nt_coarse + j] = P_[i * nt_coarse + j];
          P32.A[i * nt_coarse + j] = float(P_[i * nt_coarse + j]);
          // restriction nt_coarse x nt_fine; transpose of P unless given
          const double r                  = R_ ? R_[j * nt_fine + i] : P_[i * nt_coarse + j];
          R64.A[j * nt_fine + i]          = r;
          R32.A[j * nt_fine + i]          = float(r);
        }
  }

  void
  TTransfer::prolongate_add(const void *src, void *dst, cudaStream_t s) const
  {
    const long long N  = mesh->v.N;
    const unsigned  nb = unsigned((N + 255) / 256);
    if (dtype == STMG_F64)
      time_transfer_kernel<double><<<nb, 256, 0, s>>>(N, nt_fine, nt_coarse, P64, static_cast<const double *>(src),
                                                      static_cast<double *>(dst));
    else
      time_transfer_kernel<float><<<nb, 256, 0, s>>>(N, nt_fine, nt_coarse, P32, static_cast<const float *>(src),
                                                     static_cast<float *>(dst));
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

  void
  TTransfer::restrict_add(const void *src, void *dst, cudaStream_t s) const
  {
    const long long N  = mesh->v.N;
    const unsigned  nb = unsigned((N + 255) / 256);
    if (dtype == STMG_F64)
      time_transfer_kernel<double><<<nb, 256, 0, s>>>(N, nt_coarse, nt_fine, R64, static_cast<const double *>(src),
                                                      static_cast<double *>(dst));
    else
      time_transfer_kernel<float><<<nb, 256, 0, s>>>(N, nt_coarse, nt_fine, R32, static_cast<const float *>(src),
                                                     static_cast<float *>(dst));
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }
} // namespace stmg
