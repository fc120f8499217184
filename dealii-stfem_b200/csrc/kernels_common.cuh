// Device helpers shared by the cell-parallel kernels: register-resident
// tensor-product sweeps, Q1 geometry, node indexing and the tile shell.
#pragma once

#include "stmg_internal.h"

namespace stmg
{
  // Output combination of the cell-parallel kernels:
  //   dst = rhs + alpha s + beta dst   (rhs optional, beta = 0 ignores dst)
  // Constrained (Dirichlet) rows get rhs + beta dst.
  template <typename T>
  struct OutMode
  {
    T        alpha, beta;
    const T *rhs;
    __device__ __forceinline__ void
    write(T *dst, long long i, T s) const
    {
      T v = alpha * s;
      if (beta != T(0))
        v += beta * dst[i];
      if (rhs)
        v += rhs[i];
      dst[i] = v;
    }
    __device__ __forceinline__ void
    write_constrained(T *dst, long long i) const
    {
      T v = T(0);
      if (beta != T(0))
        v += beta * dst[i];
      if (rhs)
        v += rhs[i];
      dst[i] = v;
    }
  };

  template <int P1, int DIM>
  struct Tens
  {
    static constexpr int ND = DIM == 2 ? P1 * P1 : P1 * P1 * P1;
  };

  // out (+)= M along direction DIR of a P1^DIM tensor held in registers
  // (M row-major P1 x P1, transposed if TR). In-place use is allowed.
  template <int P1, int DIM, int DIR, bool ADD, bool TR, typename T, typename MT>
  __device__ __forceinline__ void
  sweep(const MT *__restrict__ M, const T *in, T *out)
  {
    constexpr int stride = DIR == 0 ? 1 : (DIR == 1 ? P1 : P1 * P1);
    constexpr int ND     = Tens<P1, DIM>::ND;
    constexpr int outer  = ND / (stride * P1);
#pragma unroll
    for (int o = 0; o < outer; ++o)
#pragma unroll
      for (int s = 0; s < stride; ++s)
        {
          const int base = o * stride * P1 + s;
          T         v[P1];
#pragma unroll
          for (int k = 0; k < P1; ++k)
            v[k] = in[base + k * stride];
#pragma unroll
          for (int i = 0; i < P1; ++i)
            {
              T acc = ADD ? out[base + i * stride] : T(0);
#pragma unroll
              for (int k = 0; k < P1; ++k)
                acc += T(TR ? M[k * P1 + i] : M[i * P1 + k]) * v[k];
              out[base + i * stride] = acc;
            }
        }
  }

  // Jacobian of the Q1 (bi/trilinear) map at reference point xi from the
  // cell's corner coordinates X[v][i], v bits = (x, y, z) upper side.
  template <int DIM, typename T>
  __device__ __forceinline__ void
  q1_jacobian(const T (&X)[1 << DIM][DIM], const T *xi, T (&J)[DIM][DIM])
  {
    if constexpr (DIM == 2)
      {
        const T x = xi[0], y = xi[1];
#pragma unroll
        for (int i = 0; i < 2; ++i)
          {
            J[i][0] = (T(1) - y) * (X[1][i] - X[0][i]) + y * (X[3][i] - X[2][i]);
            J[i][1] = (T(1) - x) * (X[2][i] - X[0][i]) + x * (X[3][i] - X[1][i]);
          }
      }
    else
      {
        const T x = xi[0], y = xi[1], z = xi[2];
#pragma unroll
        for (int i = 0; i < 3; ++i)
          {
            J[i][0] = (T(1) - y) * (T(1) - z) * (X[1][i] - X[0][i]) + y * (T(1) - z) * (X[3][i] - X[2][i]) +
                      (T(1) - y) * z * (X[5][i] - X[4][i]) + y * z * (X[7][i] - X[6][i]);
            J[i][1] = (T(1) - x) * (T(1) - z) * (X[2][i] - X[0][i]) + x * (T(1) - z) * (X[3][i] - X[1][i]) +
                      (T(1) - x) * z * (X[6][i] - X[4][i]) + x * z * (X[7][i] - X[5][i]);
            J[i][2] = (T(1) - x) * (T(1) - y) * (X[4][i] - X[0][i]) + x * (T(1) - y) * (X[5][i] - X[1][i]) +
                      (T(1) - x) * y * (X[6][i] - X[2][i]) + x * y * (X[7][i] - X[3][i]);
          }
      }
  }

  // determinant and inverse of a DIM x DIM matrix
  template <int DIM, typename T>
  __device__ __forceinline__ T
  det_inv(const T (&J)[DIM][DIM], T (&Ji)[DIM][DIM])
  {
    if constexpr (DIM == 2)
      {
        const T d  = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        const T id = T(1) / d;
        Ji[0][0]   = J[1][1] * id;
        Ji[0][1]   = -J[0][1] * id;
        Ji[1][0]   = -J[1][0] * id;
        Ji[1][1]   = J[0][0] * id;
        return d;
      }
    else
      {
        const T c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const T c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const T c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        const T d   = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        const T id  = T(1) / d;
        Ji[0][0]    = c00 * id;
        Ji[1][0]    = c01 * id;
        Ji[2][0]    = c02 * id;
        Ji[0][1]    = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
        Ji[1][1]    = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
        Ji[2][1]    = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
        Ji[0][2]    = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
        Ji[1][2]    = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
        Ji[2][2]    = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
        return d;
      }
  }

  // Corner coordinates of cell (cx, cy, cz).
  template <int DIM, typename T>
  __device__ __forceinline__ void
  load_corners(const MeshView &m, int cx, int cy, int cz, T (&X)[1 << DIM][DIM])
  {
    const long long nv0 = m.n[0] + 1, nv1 = m.n[1] + 1;
#pragma unroll
    for (int v = 0; v < (1 << DIM); ++v)
      {
        const long long vi = (cx + (v & 1)) + nv0 * ((cy + ((v >> 1) & 1)) + (DIM == 3 ? nv1 * (cz + ((v >> 2) & 1)) : 0));
#pragma unroll
        for (int i = 0; i < DIM; ++i)
          X[v][i] = T(m.vert[vi * DIM + i]);
      }
  }

  __device__ __forceinline__ bool
  is_boundary_node(const MeshView &m, int gx, int gy, int gz)
  {
    bool b = gx == 0 || gx == m.nn[0] - 1;
    if (m.dim > 1)
      b = b || gy == 0 || gy == m.nn[1] - 1;
    if (m.dim > 2)
      b = b || gz == 0 || gz == m.nn[2] - 1;
    return b;
  }

  // Canonical shell slot of brick node (bx,by,bz) of a tile with extents e:
  // x faces own their whole face, y faces the rest of theirs, z faces what
  // is left. Returns the offset inside one time dof's tile record.
  template <int DIM>
  __device__ __forceinline__ long long
  shell_slot(const Tiling &tl, const int (&e)[3], int bx, int by, int bz)
  {
    if (bx == 0)
      return tl.face_off[0] + by + (long long)tl.E[1] * bz;
    if (bx == e[0] - 1)
      return tl.face_off[1] + by + (long long)tl.E[1] * bz;
    if (by == 0)
      return tl.face_off[2] + bx + (long long)tl.E[0] * bz;
    if (by == e[1] - 1 || DIM == 2)
      return tl.face_off[3] + bx + (long long)tl.E[0] * bz;
    if (bz == 0)
      return tl.face_off[4] + bx + (long long)tl.E[0] * by;
    return tl.face_off[5] + bx + (long long)tl.E[0] * by;
  }

  template <int DIM>
  __device__ __forceinline__ void
  tile_extents(const MeshView &m, const Tiling &tl, long long tile, int (&t)[3], int (&c0)[3], int (&tc)[3],
               int (&e)[3])
  {
    t[0] = int(tile % tl.ntiles[0]);
    t[1] = int((tile / tl.ntiles[0]) % tl.ntiles[1]);
    t[2] = int(tile / ((long long)tl.ntiles[0] * tl.ntiles[1]));
#pragma unroll
    for (int d = 0; d < 3; ++d)
      {
        c0[d] = t[d] * tl.T[d];
        tc[d] = d < DIM ? min(tl.T[d], m.n[d] - c0[d]) : 1;
        e[d]  = d < DIM ? tc[d] * m.p + 1 : 1;
      }
  }

  // Sum of the shell contributions of all tiles containing global node g
  // for time dof j, in a fixed tile order (the deterministic fix-up).
  template <int DIM, typename T>
  __device__ __forceinline__ T
  shell_sum(const MeshView &m, const Tiling &tl, const T *__restrict__ shell, int nt, int j, const int (&g)[3])
  {
    int  cand_t[3][2], cand_l[3][2], nc[3];
    const int p = m.p;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      {
        if (d >= DIM)
          {
            cand_t[d][0] = 0;
            cand_l[d][0] = 0;
            nc[d]        = 1;
            continue;
          }
        const int span = tl.T[d] * p;
        if (g[d] % span == 0 && g[d] > 0 && g[d] < m.nn[d] - 1)
          {
            cand_t[d][0] = g[d] / span - 1;
            cand_l[d][0] = span;
            cand_t[d][1] = g[d] / span;
            cand_l[d][1] = 0;
            nc[d]        = 2;
          }
        else
          {
            cand_t[d][0] = min(g[d] / span, tl.ntiles[d] - 1);
            cand_l[d][0] = g[d] - cand_t[d][0] * span;
            nc[d]        = 1;
          }
      }
    T s = T(0);
    for (int iz = 0; iz < nc[2]; ++iz)
      for (int iy = 0; iy < nc[1]; ++iy)
        for (int ix = 0; ix < nc[0]; ++ix)
          {
            const int t[3] = {cand_t[0][ix], cand_t[1][iy], cand_t[2][iz]};
            int       e[3];
#pragma unroll
            for (int d = 0; d < 3; ++d)
              e[d] = d < DIM ? min(tl.T[d], m.n[d] - t[d] * tl.T[d]) * p + 1 : 1;
            const long long tile = t[0] + (long long)tl.ntiles[0] * (t[1] + (long long)tl.ntiles[1] * t[2]);
            const long long off  = shell_slot<DIM>(tl, e, cand_l[0][ix], cand_l[1][iy], cand_l[2][iz]);
            s += shell[(tile * nt + j) * tl.tile_stride + off];
          }
    return s;
  }
} // namespace stmg
