// Device helpers shared by the cell-parallel kernels: register-resident
// tensor-product sweeps, Q1 geometry, node indexing and the tile shell.
#pragma once

#include <algorithm>

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
    // dst[i + k stride] for k < n (n <= K), each as write() computes it,
    // with every load of dst and rhs issued before the first store (the
    // time blocks of a node would otherwise be n dependent round trips:
    // nothing tells the compiler the addresses differ)
    template <int K>
    __device__ __forceinline__ void
    write_n(T *dst, long long i, long long stride, const T (&s)[K], int n = K) const
    {
      T d[K], r[K];
#pragma unroll
      for (int k = 0; k < K; ++k)
        {
          d[k] = r[k] = T(0);
          if (k < n)
            {
              if (beta != T(0))
                d[k] = dst[i + k * stride];
              if (rhs)
                r[k] = rhs[i + k * stride];
            }
        }
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (k < n)
          {
            T v = alpha * s[k];
            if (beta != T(0))
              v += beta * d[k];
            if (rhs)
              v += r[k];
            dst[i + k * stride] = v;
          }
    }
    template <int K>
    __device__ __forceinline__ void
    write_constrained_n(T *dst, long long i, long long stride, int n = K) const
    {
      T d[K], r[K];
#pragma unroll
      for (int k = 0; k < K; ++k)
        {
          d[k] = r[k] = T(0);
          if (k < n)
            {
              if (beta != T(0))
                d[k] = dst[i + k * stride];
              if (rhs)
                r[k] = rhs[i + k * stride];
            }
        }
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (k < n)
          {
            T v = T(0);
            if (beta != T(0))
              v += beta * d[k];
            if (rhs)
              v += r[k];
            dst[i + k * stride] = v;
          }
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

  // Fix-up of the nodes the tiles share, visited by family: nodes on
  // interior x tile planes (owned by the tiles' x faces), then y planes
  // (minus x-plane nodes), then z planes (minus x- and y-plane nodes), then
  // the Dirichlet faces (each node once). One block takes a segment of one
  // row of one plane: the plane (and its family) comes from blockIdx.z, the
  // row from blockIdx.y, the position along the row from the thread, so no
  // node index is decoded by division; along y and z planes the rows run
  // along x (coalesced writes of dst).
  struct FixupRanges
  {
    int nxp, nyp, nzp, nfaces; // interior planes per direction, Dirichlet faces
    int rows, seg;             // grid extents: rows, row segments of FIXUP_THREADS
    int planes() const { return nxp + nyp + nzp + nfaces; }
  };

  constexpr int FIXUP_THREADS = 128;

  inline FixupRanges
  fixup_ranges(const MeshView &m, const Tiling &tl)
  {
    FixupRanges r;
    r.nxp    = tl.ntiles[0] - 1;
    r.nyp    = tl.ntiles[1] - 1;
    r.nzp    = m.dim == 3 ? tl.ntiles[2] - 1 : 0;
    r.nfaces = m.dim == 3 ? 6 : 4;
    r.rows   = std::max(m.nn[1], m.nn[2]);
    r.seg    = (std::max(m.nn[0], m.nn[1]) + FIXUP_THREADS - 1) / FIXUP_THREADS;
    return r;
  }

  // floor(g / span) for 0 <= g < 2^24 and the span's reciprocal rs
  __device__ __forceinline__ int
  div_span(int g, int span, float rs)
  {
    int q = __float2int_rd(float(g) * rs);
    if (q * span > g)
      --q;
    else if ((q + 1) * span <= g)
      ++q;
    return q;
  }

  template <int DIM, typename T, bool WEIGHTED>
  __global__ void __launch_bounds__(FIXUP_THREADS)
  plane_fixup_kernel(const MeshView m, const Tiling tl, int nt, const T *__restrict__ shell, T *__restrict__ dst,
                     const OutMode<T> om, const FixupRanges rg)
  {
    const int n0 = m.nn[0], n1 = m.nn[1], n2 = m.nn[2];
    const int span[3] = {tl.T[0] * m.p, tl.T[1] * m.p, tl.T[2] * m.p};
    int       pl = blockIdx.z, row = blockIdx.y, pos = blockIdx.x * FIXUP_THREADS + threadIdx.x;
    int       g[3];
    bool      boundary = false;
    if (pl < rg.nxp)
      {
        // x plane: rows z, positions y
        if (row >= n2 || pos >= n1)
          return;
        g[0] = (pl + 1) * span[0], g[1] = pos, g[2] = row;
      }
    else if ((pl -= rg.nxp) < rg.nyp)
      {
        // y plane: rows z, positions x
        if (row >= n2 || pos >= n0 || pos % span[0] == 0)
          return; // on an x plane or the x faces
        g[0] = pos, g[1] = (pl + 1) * span[1], g[2] = row;
      }
    else if ((pl -= rg.nyp) < rg.nzp)
      {
        // z plane: rows y, positions x
        if (row >= n1 || pos >= n0 || pos % span[0] == 0 || row % span[1] == 0)
          return;
        g[0] = pos, g[1] = row, g[2] = (pl + 1) * span[2];
      }
    else
      {
        // Dirichlet faces, each node once: x faces whole, y faces without
        // the x faces' nodes, z faces without both
        pl -= rg.nzp;
        boundary = true;
        const int f = pl >> 1, hi = pl & 1;
        if (f == 0)
          {
            if (row >= n2 || pos >= n1)
              return;
            g[0] = hi ? n0 - 1 : 0, g[1] = pos, g[2] = row;
          }
        else if (f == 1)
          {
            if (row >= n2 || pos < 1 || pos >= n0 - 1)
              return;
            g[0] = pos, g[1] = hi ? n1 - 1 : 0, g[2] = row;
          }
        else
          {
            if (row < 1 || row >= n1 - 1 || pos < 1 || pos >= n0 - 1)
              return;
            g[0] = pos, g[1] = row, g[2] = hi ? n2 - 1 : 0;
          }
      }
    const long long node = g[0] + (long long)n0 * (g[1] + (long long)n1 * g[2]);
    if (boundary)
      {
        for (int j0 = 0; j0 < nt; j0 += 4)
          om.template write_constrained_n<4>(dst, node + (long long)j0 * m.N, m.N, min(4, nt - j0));
        return;
      }
    if (is_boundary_node(m, g[0], g[1], g[2]))
      return; // visited as a boundary item
    T w = T(1);
    if (WEIGHTED)
      {
        int v = 1;
        for (int d = 0; d < DIM; ++d)
          if (g[d] % m.p == 0)
            v *= 2;
        w = T(1) / T(v);
      }
    // the tiles holding the node: per direction the tile and the node's
    // local index, a second tile where the node lies on a tile plane
    int tt0[3], ll0[3], two[3], ee0[3], ee1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      {
        if (d >= DIM)
          {
            tt0[d] = 0, ll0[d] = 0, two[d] = 0, ee0[d] = ee1[d] = 1;
            continue;
          }
        const int q = div_span(g[d], span[d], 1.0f / float(span[d]));
        two[d]      = q * span[d] == g[d]; // interior node on a tile plane (boundary nodes returned above)
        tt0[d]      = two[d] ? q - 1 : min(q, tl.ntiles[d] - 1);
        ll0[d]      = g[d] - tt0[d] * span[d];
        ee0[d]      = min(tl.T[d], m.n[d] - tt0[d] * tl.T[d]) * m.p + 1;
        ee1[d]      = two[d] ? min(tl.T[d], m.n[d] - (tt0[d] + 1) * tl.T[d]) * m.p + 1 : 1;
      }
    long long off[8];
    bool      ok[8];
#pragma unroll
    for (int c = 0; c < 8; ++c)
      {
        const int ix = c & 1, iy = (c >> 1) & 1, iz = (c >> 2) & 1;
        ok[c]        = !((ix && !two[0]) || (iy && !two[1]) || (iz && !two[2]));
        const int e[3] = {ix ? ee1[0] : ee0[0], iy ? ee1[1] : ee0[1], iz ? ee1[2] : ee0[2]};
        const long long tile = (tt0[0] + ix) + (long long)tl.ntiles[0] * ((tt0[1] + iy) + (long long)tl.ntiles[1] * (tt0[2] + iz));
        off[c] = ok[c] ? tile * nt * tl.tile_stride +
                           shell_slot<DIM>(tl, e, ix ? 0 : ll0[0], iy ? 0 : ll0[1], iz ? 0 : ll0[2])
                       : 0;
      }
    // four time dofs at a time with all their face-slot loads in flight
    // (each node's sum still runs over the tiles in the fixed order c)
    for (int j0 = 0; j0 < nt; j0 += 4)
      {
        T s[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (ok[c])
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
              if (j0 + jj < nt)
                s[jj] += shell[off[c] + (long long)(j0 + jj) * tl.tile_stride];
        T v[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
          v[jj] = s[jj] * w;
        om.template write_n<4>(dst, node + (long long)j0 * m.N, m.N, v, min(4, nt - j0));
      }
  }

  template <int DIM, typename T, bool WEIGHTED>
  inline void
  launch_plane_fixup(const MeshView &m, const Tiling &tl, int nt, const T *shell, T *dst, const OutMode<T> &om,
                     cudaStream_t s)
  {
    const FixupRanges rg = fixup_ranges(m, tl);
    if (rg.planes() <= 0)
      return;
    const dim3 grid(unsigned(rg.seg), unsigned(rg.rows), unsigned(rg.planes()));
    plane_fixup_kernel<DIM, T, WEIGHTED><<<grid, FIXUP_THREADS, 0, s>>>(m, tl, nt, shell, dst, om, rg);
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }
} // namespace stmg
