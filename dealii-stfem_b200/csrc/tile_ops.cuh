// Tile phases shared by the cell-parallel kernels, with compile-time tile
// shapes so every brick index is a constant-stride expression:
//  load_brick    global -> shared brick of nt blocks (cp.async, Dirichlet and
//                out-of-mesh nodes zero-filled)
//  scatter_cells per-cell results -> shared output brick, cells processed in
//                2^dim colours (no two cells of a colour share a node), so the
//                sum at every node has a fixed order
//  write_brick   shared output brick -> dst (tile-interior nodes) and the
//                tile's shell slots (nodes shared with other tiles)
#pragma once

#include "async_copy.cuh"
#include "kernels_common.cuh"

namespace stmg
{
  template <int DIM, int P, int TX, int TY, int TZ>
  struct TileShape
  {
    static constexpr int P1 = P + 1;
    static constexpr int ND = Tens<P1, DIM>::ND;
    static constexpr int E0 = TX * P + 1;
    static constexpr int E1 = TY * P + 1;
    static constexpr int E2 = DIM == 3 ? TZ * P + 1 : 1;
    static constexpr int NB = E0 * E1 * E2;
    static constexpr int TC = TX * TY * (DIM == 3 ? TZ : 1);
    static constexpr int offset(int a)
    {
      return (a % P1) + E0 * (((a / P1) % P1) + E1 * (DIM == 3 ? a / (P1 * P1) : 0));
    }
  };

  template <typename S, typename T>
  __device__ __forceinline__ void
  load_brick(T *brick, const T *__restrict__ src, const MeshView &m, int nt, const int (&c0)[3], const int (&e)[3])
  {
    constexpr int P = S::P1 - 1;
    const long long N = m.N;
    for (int idx = threadIdx.x; idx < nt * S::NB; idx += blockDim.x)
      {
        const int i = idx / S::NB, r = idx - i * S::NB;
        const int bx = r % S::E0, by = (r / S::E0) % S::E1, bz = r / (S::E0 * S::E1);
        const int gx = c0[0] * P + bx, gy = c0[1] * P + by, gz = c0[2] * P + bz;
        bool      ok = bx < e[0] && by < e[1] && bz < e[2] && gx > 0 && gx < m.nn[0] - 1 && gy > 0 && gy < m.nn[1] - 1;
        if (m.dim == 3)
          ok = ok && gz > 0 && gz < m.nn[2] - 1;
        const T *g = ok ? src + i * N + gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz) : src;
        cp_async_small<sizeof(T)>(brick + idx, g, ok);
      }
  }

  // cellbuf[(j * TC + lc) * ND + a] -> ob[j * NB + brick offset]
  template <typename S, int DIM, typename T>
  __device__ __forceinline__ void
  scatter_cells(const T *cellbuf, T *ob, int nt, const int (&tc)[3])
  {
    constexpr int P  = S::P1 - 1;
    constexpr int TX = (S::E0 - 1) / P, TY = (S::E1 - 1) / P, TZ = DIM == 3 ? (S::E2 - 1) / P : 1;
    for (int idx = threadIdx.x; idx < nt * S::NB; idx += blockDim.x)
      ob[idx] = T(0);
    __syncthreads();
#pragma unroll 1
    for (int col = 0; col < (1 << DIM); ++col)
      {
        const int ox = col & 1, oy = (col >> 1) & 1, oz = (col >> 2) & 1;
        const int nx = (TX - ox + 1) / 2, ny = (TY - oy + 1) / 2, nz = DIM == 3 ? (TZ - oz + 1) / 2 : 1;
        const int items = nx * ny * nz * S::ND;
        for (int w = threadIdx.x; w < items; w += blockDim.x)
          {
            const int k = w / S::ND, a = w - k * S::ND;
            const int ix = k % nx, iy = (k / nx) % ny, iz = k / (nx * ny);
            const int lx = 2 * ix + ox, ly = 2 * iy + oy, lz = 2 * iz + oz;
            if (lx >= tc[0] || ly >= tc[1] || lz >= tc[2])
              continue;
            const int lc = lx + TX * (ly + TY * lz);
            const int bo = lx * P + S::E0 * (ly * P + S::E1 * lz * P) + (a % S::P1) +
                           S::E0 * (((a / S::P1) % S::P1) + S::E1 * (DIM == 3 ? a / (S::P1 * S::P1) : 0));
            for (int j = 0; j < nt; ++j)
              ob[j * S::NB + bo] += cellbuf[(j * S::TC + lc) * S::ND + a];
          }
        __syncthreads();
      }
  }

  // Writes the output brick: nodes inside the tile -> dst through om (with
  // 1/valence when `weighted`), nodes on the brick shell -> shell slots, or
  // constrained writes when one tile covers the mesh.
  template <typename S, int DIM, typename T, bool WEIGHTED>
  __device__ __forceinline__ void
  write_brick(const T *ob, const MeshView &m, const Tiling &tl, long long tile, int nt, const int (&c0)[3],
              const int (&e)[3], T *__restrict__ dst, T *__restrict__ shell, const OutMode<T> &om)
  {
    constexpr int P = S::P1 - 1;
    for (int idx = threadIdx.x; idx < nt * S::NB; idx += blockDim.x)
      {
        const int j = idx / S::NB, r = idx - j * S::NB;
        const int bx = r % S::E0, by = (r / S::E0) % S::E1, bz = r / (S::E0 * S::E1);
        if (bx >= e[0] || by >= e[1] || bz >= e[2])
          continue;
        const T   s    = ob[idx];
        bool      inte = bx > 0 && bx < e[0] - 1 && by > 0 && by < e[1] - 1;
        if (DIM == 3)
          inte = inte && bz > 0 && bz < e[2] - 1;
        const int       gx = c0[0] * P + bx, gy = c0[1] * P + by, gz = c0[2] * P + bz;
        const long long gi = j * m.N + gx + (long long)m.nn[0] * (gy + (long long)m.nn[1] * gz);
        if (inte)
          {
            if (WEIGHTED)
              {
                // valence: cells sharing the node (2 per interior cell face crossed)
                int v = 1;
                v *= (gx % P == 0) ? 2 : 1;
                v *= (gy % P == 0) ? 2 : 1;
                if (DIM == 3)
                  v *= (gz % P == 0) ? 2 : 1;
                om.write(dst, gi, s / T(v));
              }
            else
              om.write(dst, gi, s);
          }
        else if (tl.n_tiles == 1)
          om.write_constrained(dst, gi); // a single tile's shell is the Dirichlet boundary
        else
          shell[(tile * nt + j) * tl.tile_stride + shell_slot<DIM>(tl, e, bx, by, bz)] = s;
      }
  }
} // namespace stmg
