// Cell-patch space-time Vanka smoother (PreconditionVanka,
// tests/include/gmg.h:402-540).
//
// The reference inverts, per cell c, the patch matrix
//   B_c = Alpha (x) K_c + Beta (x) M_c,
// K_c, M_c being the assembled global matrices restricted to the cell's dofs
// (neighbour contributions included), and applies
//   dst = sum_c R_c^T diag(1/valence) B_c^{-1} R_c src.
// Here B_c^{-1} is applied in factored form. With the generalised
// eigendecomposition K_c V = M_c V diag(mu), V^T M_c V = I,
//   B_c^{-1} = (I (x) V) blockdiag_m (mu_m Alpha + Beta)^{-1} (I (x) V^T),
// which is the same operator, so a cell stores V (nd x nd) and mu (nd)
// instead of the (n_t nd)^2 inverse. Setup (FP64): patch assembly,
// Cholesky of M_c, cyclic Jacobi of L^{-1} K_c L^{-T}. Apply: one pass over
// the cells with the operator's tile / brick / shell scheme.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <complex>
#include <cstring>

#include <cuda_bf16.h>

#include "kernels_common.cuh"
#include "vanka.h"

#include <mutex>
#include "vanka_apply_impl.cuh"

namespace stmg
{
  namespace
  {
    template <typename TS>
    __device__ __forceinline__ TS
    to_storage(double v)
    {
      if constexpr (std::is_same_v<TS, __nv_bfloat16>)
        return __float2bfloat16_rn(float(v));
      else
        return TS(v);
    }

    // cells containing global node coordinate g along one direction
    __device__ __forceinline__ void
    cell_range(int g, int P, int n, int &lo, int &hi)
    {
      hi = min(g / P, n - 1);
      lo = (g % P == 0 && g > 0) ? g / P - 1 : g / P;
      lo = min(lo, n - 1);
    }

    // --------------------------------------------------------------- setup
    // One CTA per cell: assemble K_c, M_c, factor, write V (as [m][a]) and mu.
    // Record slot of cell cc in (tile, colour, cell) order: tiles of tl.T
    // cells, colour = parity of the local cell coordinates, cells of one
    // colour in lexicographic order of their half-coordinates.
    __device__ __forceinline__ long long
    record_slot(const Tiling &tl, int dim, const int (&cc)[3])
    {
      int       t[3], l[3];
      long long tile = 0, stride = 1, tc = 1;
      for (int d = 0; d < 3; ++d)
        {
          t[d] = cc[d] / tl.T[d];
          l[d] = cc[d] - t[d] * tl.T[d];
          tile += t[d] * stride;
          stride *= tl.ntiles[d];
          tc *= tl.T[d];
        }
      const int col = (l[0] & 1) | ((l[1] & 1) << 1) | ((l[2] & 1) << 2);
      int       prefix = 0;
      for (int c = 0; c < col; ++c)
        {
          int n = 1;
          for (int d = 0; d < 3; ++d)
            {
              const int o = (c >> d) & 1;
              n *= d < dim ? (tl.T[d] - o + 1) / 2 : (o ? 0 : 1);
            }
          prefix += n;
        }
      const int c0 = (tl.T[0] - (l[0] & 1) + 1) / 2, c1 = (tl.T[1] - (l[1] & 1) + 1) / 2;
      const int idx = (l[0] >> 1) + c0 * ((l[1] >> 1) + c1 * (l[2] >> 1));
      return tile * tc + prefix + idx;
    }

    template <int DIM, int P, bool CART, typename TS>
    __global__ void
    vanka_setup_kernel(const MeshView m, const double *__restrict__ Kref, const double *__restrict__ Mref,
                       const double *__restrict__ elemK, const double *__restrict__ elemM,
                       unsigned char *__restrict__ rec, int rec_bytes, int mu_off, int mu_double,
                       int *__restrict__ status, const Tiling tl, int tiled, int row_stride, int mu_stride,
                       int swz_kt)
    {
      constexpr int P1 = P + 1;
      constexpr int ND = Tens<P1, DIM>::ND;
      extern __shared__ double setup_smem[];
      double(*K)[ND + 1] = reinterpret_cast<double(*)[ND + 1]>(setup_smem);
      double(*M)[ND + 1] = reinterpret_cast<double(*)[ND + 1]>(setup_smem + ND * (ND + 1));
      double(*Q)[ND + 1] = reinterpret_cast<double(*)[ND + 1]>(setup_smem + 2 * ND * (ND + 1));
      double *rot        = setup_smem + 3 * ND * (ND + 1);
      const long long cell = blockIdx.x;
      const int cc[3] = {int(cell % m.n[0]), int((cell / m.n[0]) % m.n[1]), int(cell / ((long long)m.n[0] * m.n[1]))};
      const int tid = threadIdx.x, nth = blockDim.x;
      const long long slot = tiled ? record_slot(tl, DIM, cc) : cell;

      // 1. patch matrices: global K, M restricted to the cell's dofs
      for (int e = tid; e < ND * ND; e += nth)
        {
          const int a = e / ND, b = e % ND;
          const int la[3] = {a % P1, (a / P1) % P1, DIM == 3 ? a / (P1 * P1) : 0};
          const int lb[3] = {b % P1, (b / P1) % P1, DIM == 3 ? b / (P1 * P1) : 0};
          int       ga[3], gb[3];
          for (int d = 0; d < 3; ++d)
            {
              ga[d] = cc[d] * P + la[d];
              gb[d] = cc[d] * P + lb[d];
            }
          const bool bda = is_boundary_node(m, ga[0], ga[1], ga[2]);
          const bool bdb = is_boundary_node(m, gb[0], gb[1], gb[2]);
          double     kv = 0, mv = 0;
          if (bda || bdb)
            {
              // constrained rows/columns decouple; their diagonal value
              // never meets a nonzero input
              if (a == b)
                kv = mv = 1.0;
            }
          else
            {
              int lo[3], hi[3];
              for (int d = 0; d < 3; ++d)
                {
                  if (d >= DIM)
                    {
                      lo[d] = hi[d] = 0;
                      continue;
                    }
                  int l1, h1, l2, h2;
                  cell_range(ga[d], P, m.n[d], l1, h1);
                  cell_range(gb[d], P, m.n[d], l2, h2);
                  lo[d] = max(l1, l2);
                  hi[d] = min(h1, h2);
                }
              for (int ez = lo[2]; ez <= hi[2]; ++ez)
                for (int ey = lo[1]; ey <= hi[1]; ++ey)
                  for (int ex = lo[0]; ex <= hi[0]; ++ex)
                    {
                      const long long ec = ex + (long long)m.n[0] * (ey + (long long)m.n[1] * ez);
                      const int       ia = (ga[0] - ex * P) + P1 * ((ga[1] - ey * P) + P1 * (DIM == 3 ? ga[2] - ez * P : 0));
                      const int       ib = (gb[0] - ex * P) + P1 * ((gb[1] - ey * P) + P1 * (DIM == 3 ? gb[2] - ez * P : 0));
                      if constexpr (CART)
                        {
                          const double kap = m.coeff_mode == 1 ? m.coeff64[ec] : 1.0;
                          kv += kap * Kref[ia * ND + ib];
                          mv += Mref[ia * ND + ib];
                        }
                      else
                        {
                          kv += elemK[ec * ND * ND + ia * ND + ib];
                          mv += elemM[ec * ND * ND + ia * ND + ib];
                        }
                    }
            }
          K[a][b] = kv;
          M[a][b] = mv;
          Q[a][b] = a == b ? 1.0 : 0.0;
        }
      __syncthreads();

      // 2. Cholesky M = L L^T (lower triangle of M)
      for (int j = 0; j < ND; ++j)
        {
          if (tid == 0)
            {
              double s = M[j][j];
              for (int k = 0; k < j; ++k)
                s -= M[j][k] * M[j][k];
              if (!(s > 0))
                atomicExch(status, 1);
              M[j][j] = sqrt(fmax(s, 1e-300));
            }
          __syncthreads();
          for (int i = j + 1 + tid; i < ND; i += nth)
            {
              double s = M[i][j];
              for (int k = 0; k < j; ++k)
                s -= M[i][k] * M[j][k];
              M[i][j] = s / M[j][j];
            }
          __syncthreads();
        }
      // 3. K <- L^{-1} K L^{-T}: forward substitution on columns, then rows
      for (int col = tid; col < ND; col += nth)
        for (int i = 0; i < ND; ++i)
          {
            double s = K[i][col];
            for (int k = 0; k < i; ++k)
              s -= M[i][k] * K[k][col];
            K[i][col] = s / M[i][i];
          }
      __syncthreads();
      for (int row = tid; row < ND; row += nth)
        for (int i = 0; i < ND; ++i)
          {
            double s = K[row][i];
            for (int k = 0; k < i; ++k)
              s -= M[i][k] * K[row][k];
            K[row][i] = s / M[i][i];
          }
      __syncthreads();
      // symmetrise (rounding)
      for (int e = tid; e < ND * ND; e += nth)
        {
          const int a = e / ND, b = e % ND;
          if (a < b)
            {
              const double v = 0.5 * (K[a][b] + K[b][a]);
              K[a][b]        = v;
              K[b][a]        = v;
            }
        }
      __syncthreads();

      // 4. parallel cyclic Jacobi, K = Q diag(mu) Q^T: each round applies
      //    the m/2 disjoint rotations of a round-robin tournament (index 0
      //    fixed, the others rotating; an odd ND gets a dummy index ND), as
      //    K <- J^T (K J), Q <- Q J.
      constexpr int MJ = (ND % 2) ? ND + 1 : ND;
      constexpr int NP = MJ / 2;
      int    *rp = reinterpret_cast<int *>(rot + 4);
      double *rc = rot + 4 + NP, *rs = rc + NP;
      for (int sweep = 0; sweep < 40; ++sweep)
        {
          if (tid == 0)
            {
              double off = 0, dg = 0;
              for (int a = 0; a < ND; ++a)
                {
                  dg += K[a][a] * K[a][a];
                  for (int b = a + 1; b < ND; ++b)
                    off += K[a][b] * K[a][b];
                }
              rot[3] = (off <= 1e-30 * dg) ? 1.0 : 0.0;
            }
          __syncthreads();
          if (rot[3] != 0.0)
            break;
          for (int round = 0; round < MJ - 1; ++round)
            {
              for (int k = tid; k < NP; k += nth)
                {
                  const int ia = k, ib = MJ - 1 - k;
                  const int pa = ia == 0 ? 0 : ((ia - 1 + round) % (MJ - 1)) + 1;
                  const int pb = ((ib - 1 + round) % (MJ - 1)) + 1;
                  const int p  = min(pa, pb), q = max(pa, pb);
                  double    c = 1, sn = 0;
                  if (q < ND)
                    {
                      const double apq = K[p][q];
                      if (apq != 0.0)
                        {
                          const double th = (K[q][q] - K[p][p]) / (2.0 * apq);
                          const double t  = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                          c               = 1.0 / sqrt(t * t + 1.0);
                          sn              = t * c;
                        }
                    }
                  rp[2 * k]     = p;
                  rp[2 * k + 1] = q;
                  rc[k]         = c;
                  rs[k]         = sn;
                }
              __syncthreads();
              // columns: K <- K J, Q <- Q J (row i owned by one thread)
              for (int i = tid; i < ND; i += nth)
                for (int k = 0; k < NP; ++k)
                  {
                    const int q = rp[2 * k + 1];
                    if (q >= ND || rs[k] == 0.0)
                      continue;
                    const int    p = rp[2 * k];
                    const double c = rc[k], sn = rs[k];
                    const double kp = K[i][p], kq = K[i][q];
                    K[i][p]         = c * kp - sn * kq;
                    K[i][q]         = sn * kp + c * kq;
                    const double qp = Q[i][p], qq = Q[i][q];
                    Q[i][p]         = c * qp - sn * qq;
                    Q[i][q]         = sn * qp + c * qq;
                  }
              __syncthreads();
              // rows: K <- J^T K (pair k, column j)
              for (int e = tid; e < NP * ND; e += nth)
                {
                  const int k = e / ND, j = e % ND;
                  const int q = rp[2 * k + 1];
                  if (q >= ND || rs[k] == 0.0)
                    continue;
                  const int    p = rp[2 * k];
                  const double c = rc[k], sn = rs[k];
                  const double kp = K[p][j], kq = K[q][j];
                  K[p][j]         = c * kp - sn * kq;
                  K[q][j]         = sn * kp + c * kq;
                }
              __syncthreads();
            }
        }
      // 5. V = L^{-T} Q (back substitution per column), store as [m][a]
      for (int col = tid; col < ND; col += nth)
        {
          for (int i = ND - 1; i >= 0; --i)
            {
              double s = Q[i][col];
              for (int k = i + 1; k < ND; ++k)
                s -= M[k][i] * Q[k][col];
              Q[i][col] = s / M[i][i];
            }
          unsigned char *mr = rec + slot * rec_bytes + mu_off;
          if (mu_double)
            reinterpret_cast<double *>(mr)[col * mu_stride] = K[col][col];
          else
            reinterpret_cast<float *>(mr)[col * mu_stride] = float(K[col][col]);
        }
      __syncthreads();
      for (int e = tid; e < ND * ND; e += nth)
        {
          const int mm = e / ND, a = e % ND;
          if (swz_kt == 32)
            *reinterpret_cast<TS *>(rec + slot * rec_bytes + MmaRows<32>::offset(mm, a)) = to_storage<TS>(Q[a][mm]);
          else if (swz_kt == 16)
            *reinterpret_cast<TS *>(rec + slot * rec_bytes + MmaRows<16>::offset(mm, a)) = to_storage<TS>(Q[a][mm]);
          else
            reinterpret_cast<TS *>(rec + slot * rec_bytes)[mm * row_stride + a] = to_storage<TS>(Q[a][mm]);
        }
    }

    // Element matrices of every cell for the general (non-cartesian) path.
    template <int DIM, int P>
    __global__ void
    element_matrix_kernel(const MeshView m, const __grid_constant__ QTab<double> qt, double *__restrict__ Ke,
                          double *__restrict__ Me)
    {
      constexpr int P1 = P + 1;
      constexpr int ND = Tens<P1, DIM>::ND;
      const long long cell = blockIdx.x;
      const int cc[3] = {int(cell % m.n[0]), int((cell / m.n[0]) % m.n[1]), int(cell / ((long long)m.n[0] * m.n[1]))};
      __shared__ double G[ND][DIM * DIM], W[ND];
      double X[1 << DIM][DIM];
      load_corners<DIM>(m, cc[0], cc[1], cc[2], X);
      for (int q = threadIdx.x; q < ND; q += blockDim.x)
        {
          const int qx = q % P1, qy = (q / P1) % P1, qz = q / (P1 * P1);
          double    xi[3] = {qt.gx[qx], qt.gx[qy], DIM == 3 ? qt.gx[qz] : 0.0};
          double    J[DIM][DIM], Ji[DIM][DIM];
          q1_jacobian<DIM>(X, xi, J);
          const double det = det_inv<DIM>(J, Ji);
          double       w   = qt.gw[qx] * qt.gw[qy] * (DIM == 3 ? qt.gw[qz] : 1.0);
          const double JxW = fabs(det) * w;
          const double k = m.coeff_mode == 1 ? m.coeff64[cell] : (m.coeff_mode == 2 ? m.coeff64[cell * ND + q] : 1.0);
          for (int a = 0; a < DIM; ++a)
            for (int b = 0; b < DIM; ++b)
              {
                double s = 0;
                for (int i = 0; i < DIM; ++i)
                  s += Ji[a][i] * Ji[b][i];
                G[q][a * DIM + b] = k * JxW * s;
              }
          W[q] = JxW;
        }
      __syncthreads();
      // reference gradients of basis function a at point q via S, D tables:
      // phi_a(q) = prod S, d_j phi_a(q) = D in direction j
      for (int e = threadIdx.x; e < ND * ND; e += blockDim.x)
        {
          const int a = e / ND, b = e % ND;
          const int ai[3] = {a % P1, (a / P1) % P1, a / (P1 * P1)};
          const int bi[3] = {b % P1, (b / P1) % P1, b / (P1 * P1)};
          double    kv = 0, mv = 0;
          for (int q = 0; q < ND; ++q)
            {
              const int qi[3] = {q % P1, (q / P1) % P1, q / (P1 * P1)};
              double    pa = 1, pb = 1, ga[DIM], gb[DIM];
              for (int j = 0; j < DIM; ++j)
                ga[j] = gb[j] = 1;
              for (int d = 0; d < DIM; ++d)
                {
                  const double sa = qt.S[qi[d] * P1 + ai[d]], sb = qt.S[qi[d] * P1 + bi[d]];
                  // D = Dq S (collocation): d phi_a / d xi_d at q
                  double da = 0, db = 0;
                  for (int r = 0; r < P1; ++r)
                    {
                      da += qt.Dq[qi[d] * P1 + r] * qt.S[r * P1 + ai[d]];
                      db += qt.Dq[qi[d] * P1 + r] * qt.S[r * P1 + bi[d]];
                    }
                  pa *= sa;
                  pb *= sb;
                  for (int j = 0; j < DIM; ++j)
                    {
                      ga[j] *= (j == d) ? da : sa;
                      gb[j] *= (j == d) ? db : sb;
                    }
                }
              mv += W[q] * pa * pb;
              for (int i = 0; i < DIM; ++i)
                for (int j = 0; j < DIM; ++j)
                  kv += ga[i] * G[q][i * DIM + j] * gb[j];
            }
          Ke[cell * ND * ND + e] = kv;
          Me[cell * ND * ND + e] = mv;
        }
    }

  } // namespace

  // ------------------------------------------------------------------ host
  std::size_t
  Vanka::smem_bytes(const int *T3) const
  {
    const std::size_t elem = compute == STMG_F64 ? 8 : 4;
    const int         p = mesh->v.p, dim = mesh->v.dim;
    const std::size_t nb = std::size_t(T3[0] * p + 1) * (T3[1] * p + 1) * (dim == 3 ? T3[2] * p + 1 : 1);
    const std::size_t tc = std::size_t(T3[0]) * T3[1] * (dim == 3 ? T3[2] : 1);
    if (streamed)
      {
        const std::size_t ntp = nt == 3 ? 4 : nt;
        if (slotrec)
          return (std::size_t(1) << dim) * (rec_bytes + 4 * 2 * std::size_t(mesh->nd) * ntp) + 4 * nb * ntp;
        if (mmarec)
          return std::size_t(stages) * colour_cells * rec_bytes + 4 * 3 * nb * ntp +
                 vanka_detail::VR_WARPS * 32 * 16 + 128;
        if (rowrec)
          return std::size_t(stages) * colour_cells * rec_bytes +
                 4 * (3 * nb * ntp + vanka_detail::VR_WARPS * std::size_t(mesh->nd) * ntp);
        return std::size_t(vanka_detail::VK_STAGES) * colour_cells * rec_bytes +
               4 * (3 * nb * ntp + 8 * std::size_t(mesh->nd) * ntp);
      }
    return 2ull * chunk * rec_bytes +
           elem * (2ull * nt * nb + std::size_t(chunk) * nt * mesh->nd + tc * nt * mesh->nd);
  }

  namespace
  {
    template <int DIM, int P>
    void
    run_setup(Vanka &vk)
    {
      constexpr int   ND = Tens<P + 1, DIM>::ND;
      const MeshView &m  = vk.mesh->v;
      DevBuf<int>     status(1);
      STMG_CUDA(cudaMemset(status.ptr, 0, sizeof(int)));
      DevBuf<double> Kref, Mref, eK, eM;
      const int      threads = ND <= 32 ? 32 : 64;
      if (m.cartesian)
        {
          // reference element matrices of the level's cell size (kappa = 1)
          const FETables     &t = host_tables();
          std::vector<double> k(ND * ND), mm(ND * ND);
          for (int a = 0; a < ND; ++a)
            for (int b = 0; b < ND; ++b)
              {
                const int ai[3] = {a % (P + 1), (a / (P + 1)) % (P + 1), a / ((P + 1) * (P + 1))};
                const int bi[3] = {b % (P + 1), (b / (P + 1)) % (P + 1), b / ((P + 1) * (P + 1))};
                double    mv = 1, kv = 0;
                for (int d = 0; d < DIM; ++d)
                  mv *= t.M1[P][ai[d]][bi[d]] * m.h[d];
                for (int j = 0; j < DIM; ++j)
                  {
                    double term = 1;
                    for (int d = 0; d < DIM; ++d)
                      term *= d == j ? t.K1[P][ai[d]][bi[d]] / m.h[d] : t.M1[P][ai[d]][bi[d]] * m.h[d];
                    kv += term;
                  }
                k[a * ND + b]  = kv;
                mm[a * ND + b] = mv;
              }
          Kref.upload(k);
          Mref.upload(mm);
        }
      else
        {
          eK.alloc(m.ncells * ND * ND);
          eM.alloc(m.ncells * ND * ND);
          element_matrix_kernel<DIM, P><<<unsigned(m.ncells), 64>>>(m, make_qtab<double>(P), eK.ptr, eM.ptr);
          count_launch();
          STMG_CUDA(cudaGetLastError());
        }
      const std::size_t smem = (3ull * ND * (ND + 1) + 4 + 3 * ((ND + 1) / 2 + 1)) * sizeof(double);
      auto go = [&](auto *Vp) {
        using TS  = std::remove_pointer_t<decltype(Vp)>;
        auto kern = m.cartesian ? vanka_setup_kernel<DIM, P, true, TS> : vanka_setup_kernel<DIM, P, false, TS>;
        STMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        (void)Vp;
        kern<<<unsigned(m.ncells), threads, smem>>>(m, Kref.ptr, Mref.ptr, eK.ptr, eM.ptr, vk.V.ptr, vk.rec_bytes,
                                                    vk.mu_off, vk.compute == STMG_F64 ? 1 : 0, status.ptr, vk.tiling,
                                                    vk.streamed ? 1 : 0, vk.row_stride, vk.mu_stride,
                                                    vk.mmarec ? vk.mma_kt : 0);
        count_launch();
        STMG_CUDA(cudaGetLastError());
      };
      if (vk.storage == STMG_F64)
        go(reinterpret_cast<double *>(vk.V.ptr));
      else if (vk.storage == STMG_F32)
        go(reinterpret_cast<float *>(vk.V.ptr));
      else
        go(reinterpret_cast<__nv_bfloat16 *>(vk.V.ptr));
      STMG_CUDA(cudaDeviceSynchronize());
      int st = 0;
      STMG_CUDA(cudaMemcpy(&st, status.ptr, sizeof(int), cudaMemcpyDeviceToHost));
      STMG_REQUIRE(st == 0, STMG_ERR_NONFINITE, "vanka setup: patch mass matrix not positive definite");
    }

  } // namespace

  namespace
  {
    using cplx = std::complex<double>;

    // x = M^{-1} y for a small complex matrix (Gaussian elimination with
    // partial pivoting); false if singular
    bool
    csolve(int n, std::vector<cplx> M, std::vector<cplx> &x)
    {
      for (int k = 0; k < n; ++k)
        {
          int piv = k;
          for (int i = k + 1; i < n; ++i)
            if (std::abs(M[i * n + k]) > std::abs(M[piv * n + k]))
              piv = i;
          if (std::abs(M[piv * n + k]) < 1e-300)
            return false;
          if (piv != k)
            {
              for (int j = 0; j < n; ++j)
                std::swap(M[k * n + j], M[piv * n + j]);
              std::swap(x[k], x[piv]);
            }
          for (int i = k + 1; i < n; ++i)
            {
              const cplx f = M[i * n + k] / M[k * n + k];
              for (int j = k; j < n; ++j)
                M[i * n + j] -= f * M[k * n + j];
              x[i] -= f * x[k];
            }
        }
      for (int i = n - 1; i >= 0; --i)
        {
          cplx s = x[i];
          for (int j = i + 1; j < n; ++j)
            s -= M[i * n + j] * x[j];
          x[i] = s / M[i * n + i];
        }
      return true;
    }

    // Real eigen-decomposition of C = Beta^{-1} Alpha for n <= 4: the
    // characteristic polynomial (Faddeev-LeVerrier), its roots by
    // Durand-Kerner iteration polished by Newton, eigenvectors by inverse
    // iteration on the shifted matrix; accepted when C S = S Lambda holds to
    // 1e-10 and S is well conditioned.
    TimeEig
    time_eigen(int n, const double *A, const double *B)
    {
      TimeEig te{};
      te.nt = n;
      if (n < 1 || n > 4)
        return te;
      // C = B^{-1} A
      std::vector<cplx> Bc(n * n), C(n * n);
      for (int i = 0; i < n * n; ++i)
        Bc[i] = B[i];
      for (int j = 0; j < n; ++j)
        {
          std::vector<cplx> col(n);
          for (int i = 0; i < n; ++i)
            col[i] = A[i * n + j];
          if (!csolve(n, Bc, col))
            return te;
          for (int i = 0; i < n; ++i)
            C[i * n + j] = col[i];
        }
      // characteristic polynomial p(x) = x^n + c[1] x^{n-1} + ... + c[n]
      std::vector<double> c(n + 1, 0.0);
      c[0] = 1;
      std::vector<double> Mk(n * n, 0.0), AM(n * n);
      for (int k = 1; k <= n; ++k)
        {
          // M_k = C M_{k-1} + c_{k-1} I, c_k = -tr(C M_k) / k
          std::vector<double> Mn(n * n, 0.0);
          for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
              {
                double s = 0;
                for (int l = 0; l < n; ++l)
                  s += C[i * n + l].real() * Mk[l * n + j];
                Mn[i * n + j] = s + (i == j ? c[k - 1] : 0.0);
              }
          double tr = 0;
          for (int i = 0; i < n; ++i)
            for (int l = 0; l < n; ++l)
              tr += C[i * n + l].real() * Mn[l * n + i];
          c[k] = -tr / k;
          Mk   = Mn;
        }
      auto peval = [&](cplx x) {
        cplx v = 1;
        for (int k = 1; k <= n; ++k)
          v = v * x + c[k];
        return v;
      };
      auto pder = [&](cplx x) {
        cplx v = double(n);
        for (int k = 1; k < n; ++k)
          v = v * x + double(n - k) * c[k];
        return v;
      };
      double rad = 0;
      for (int k = 1; k <= n; ++k)
        rad = std::max(rad, std::abs(c[k]));
      rad = 1 + rad;
      std::vector<cplx> r(n);
      for (int k = 0; k < n; ++k)
        r[k] = std::polar(rad * 0.9, 0.4 + 2 * 3.14159265358979323846 * k / n);
      for (int it = 0; it < 500; ++it)
        {
          double moved = 0;
          for (int k = 0; k < n; ++k)
            {
              cplx den = 1;
              for (int j = 0; j < n; ++j)
                if (j != k)
                  den *= r[k] - r[j];
              const cplx d = peval(r[k]) / den;
              r[k] -= d;
              moved = std::max(moved, std::abs(d));
            }
          if (moved < 1e-15 * rad)
            break;
        }
      for (int k = 0; k < n; ++k)
        for (int it = 0; it < 3; ++it)
          {
            const cplx dp = pder(r[k]);
            if (std::abs(dp) > 0)
              r[k] -= peval(r[k]) / dp;
          }
      // order: real roots, then complex pairs (positive imaginary part first)
      std::vector<cplx> lam;
      for (int k = 0; k < n; ++k)
        if (std::abs(r[k].imag()) <= 1e-10 * (1 + std::abs(r[k])))
          lam.push_back(cplx(r[k].real(), 0.0));
      for (int k = 0; k < n; ++k)
        if (r[k].imag() > 1e-10 * (1 + std::abs(r[k])))
          {
            lam.push_back(r[k]);
            lam.push_back(std::conj(r[k]));
          }
      if (int(lam.size()) != n)
        return te;
      // distinct eigenvalues only
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
          if (std::abs(lam[i] - lam[j]) < 1e-8 * (1 + std::abs(lam[i])))
            return te;
      // eigenvectors by inverse iteration; real matrix Sr in the real block form
      std::vector<double> Sr(n * n, 0.0);
      for (int k = 0; k < n; ++k)
        {
          const bool pair = lam[k].imag() > 0;
          if (lam[k].imag() < 0)
            continue; // filled with its partner
          const cplx sh = lam[k] + cplx(1e-9 * (1 + std::abs(lam[k])), 1e-9 * (1 + std::abs(lam[k])));
          std::vector<cplx> M(n * n), v(n, cplx(1.0, 0.5));
          for (int i = 0; i < n * n; ++i)
            M[i] = C[i] - (i / n == i % n ? sh : cplx(0));
          for (int it = 0; it < 3; ++it)
            {
              if (!csolve(n, M, v))
                return te;
              double nv = 0;
              for (auto &e : v)
                nv = std::max(nv, std::abs(e));
              for (auto &e : v)
                e /= nv;
            }
          for (int i = 0; i < n; ++i)
            {
              Sr[i * n + k] = v[i].real();
              if (pair)
                Sr[i * n + k + 1] = v[i].imag();
            }
          te.kind[k] = pair ? 2 : 1;
          te.a[k]    = float(lam[k].real());
          te.b[k]    = float(lam[k].imag());
          if (pair)
            {
              te.kind[k + 1] = 3;
              te.a[k + 1]    = te.a[k];
              te.b[k + 1]    = te.b[k];
            }
        }
      // residual of C Sr = Sr Lambda_r
      double res = 0, cn = 0;
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
          {
            double cs = 0;
            for (int l = 0; l < n; ++l)
              cs += C[i * n + l].real() * Sr[l * n + k];
            double sl;
            if (te.kind[k] == 1)
              sl = Sr[i * n + k] * lam[k].real();
            else if (te.kind[k] == 2)
              sl = lam[k].real() * Sr[i * n + k] - lam[k].imag() * Sr[i * n + k + 1];
            else // second column of a pair: lam[k - 1] carries the positive imaginary part
              sl = lam[k - 1].imag() * Sr[i * n + k - 1] + lam[k - 1].real() * Sr[i * n + k];
            res = std::max(res, std::abs(cs - sl));
            cn  = std::max(cn, std::abs(C[i * n + k]));
          }
      if (res > 1e-10 * (1 + cn))
        return te;
      // G = Sr^{-1} B^{-1}; condition estimate from |Sr| |Sr^{-1}|
      std::vector<cplx> Src(n * n);
      for (int i = 0; i < n * n; ++i)
        Src[i] = Sr[i];
      double ninv = 0, ns = 0;
      std::vector<double> Sinv(n * n);
      for (int j = 0; j < n; ++j)
        {
          std::vector<cplx> e(n, 0.0);
          e[j] = 1;
          if (!csolve(n, Src, e))
            return te;
          for (int i = 0; i < n; ++i)
            Sinv[i * n + j] = e[i].real();
        }
      for (int i = 0; i < n * n; ++i)
        {
          ninv = std::max(ninv, std::abs(Sinv[i]));
          ns   = std::max(ns, std::abs(Sr[i]));
        }
      if (ns * ninv * n > 1e5)
        return te;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          {
            // G = Sinv B^{-1}: solve B^T g_row = Sinv_row
            te.S[i * n + j] = float(Sr[i * n + j]);
          }
      std::vector<cplx> BT(n * n);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          BT[i * n + j] = B[j * n + i];
      for (int i = 0; i < n; ++i)
        {
          std::vector<cplx> row(n);
          for (int j = 0; j < n; ++j)
            row[j] = Sinv[i * n + j];
          if (!csolve(n, BT, row))
            return te;
          for (int j = 0; j < n; ++j)
            te.G[i * n + j] = float(row[j].real());
        }
      te.use = 1;
      return te;
    }
  } // namespace

  Vanka::Vanka(Mesh *mesh_, int nt_, const double *A, const double *B, int compute_, int storage_)
    : mesh(mesh_)
    , nt(nt_)
    , compute(compute_)
    , storage(storage_)
  {
    STMG_REQUIRE(nt >= 1 && nt <= MAX_NT, STMG_ERR_ARG, "vanka: time dofs must be 1..16");
    STMG_REQUIRE(compute == STMG_F64 || compute == STMG_F32, STMG_ERR_ARG, "vanka: compute type F64 or F32");
    STMG_REQUIRE(compute == STMG_F32 ? (storage == STMG_F32 || storage == STMG_BF16) : storage == STMG_F64,
                 STMG_ERR_ARG, "vanka: storage F32/BF16 with F32 compute, F64 with F64 compute");
    const int dim = mesh->v.dim, p = mesh->v.p;
    STMG_REQUIRE(!(dim == 3 && p > 3), STMG_ERR_UNSUPPORTED, "vanka: 3-D degree up to 3");
    std::memset(&tm64, 0, sizeof(tm64));
    std::memset(&tm32, 0, sizeof(tm32));
    tm64.nt_out = tm64.nt_in = tm32.nt_out = tm32.nt_in = nt;
    for (int i = 0; i < nt * nt; ++i)
      {
        tm64.A[i] = A[i];
        tm64.B[i] = B[i];
        tm32.A[i] = float(A[i]);
        tm32.B[i] = float(B[i]);
      }
    {
      const char *e = std::getenv("STMG_VANKA_EIG");
      if (!(e && e[0] == '0'))
        teig = time_eigen(nt, A, B);
      teig.nt = nt;
    }
    const std::size_t nd   = mesh->nd;
    const std::size_t elem = storage == STMG_F64 ? 8 : (storage == STMG_F32 ? 4 : 2);
    auto              pad  = [](std::size_t b) { return (b + 15) / 16 * 16; };
    // compile-time tile shape: the streamed apply takes the main shape when
    // two CTAs per SM fit, else the fallback; the other apply also sizes its
    // record chunk within a shared-memory budget. 3-D cells of degree 3 and
    // up take the chunked apply: their records (16.6 KB and more) leave the
    // streamed ring room for one cell per colour phase, one busy warp per CTA.
    streamed = compute == STMG_F32 && nt <= 4 && !(dim == 3 && p >= 3);
    {
      const char *e = std::getenv("STMG_VANKA_ROWREC");
      // the row-record kernel is built for the eigenvalue pattern of the
      // dG / cGP time matrices: one real eigenvalue for odd n_t, none for even
      int nreal = 0;
      for (int k = 0; k < nt; ++k)
        nreal += teig.kind[k] == 1 ? 1 : 0;
      rowrec = streamed && teig.use && nd <= 32 && nreal == nt % 2 && !(e && e[0] == '0');
    }
    {
      // the small-tile apply where the colour-phase tiles would leave SMs
      // idle (STMG_VANKA_SLOT=0 / 1 turns it off / on for every row-record
      // mesh)
      const char *e = std::getenv("STMG_VANKA_SLOT");
      int         sh[3];
      vanka_shape(dim, p, true, sh);
      const bool few = make_tiling(mesh->v, sh).n_tiles < sm_count();
      slotrec        = rowrec && (e ? e[0] == '1' : few);
    }
    {
      // the tensor-core apply: BF16 storage, 3 or 4 time dofs (one brick word
      // of four FP32 per node)
      const char *e = std::getenv("STMG_VANKA_MMA");
      mmarec = rowrec && !slotrec && storage == STMG_BF16 && (nt == 3 || nt == 4) && !(e && e[0] == '0');
    }
    if (mmarec)
      {
        mma_kt     = nd <= 16 ? 16 : 32;
        row_stride = mma_kt;
        mu_off     = int(pad(nd * mma_kt * 2));
        mu_stride  = 1;
        rec_bytes  = int(pad(mu_off + nd * 4));
        // eigenbasis with the complex pairs first, the real eigenvalue last
        const int nr = nt % 2, np2 = nt - nr;
        int       order[MAX_NT];
        for (int k = 0; k < nt; ++k)
          order[k] = k < np2 ? k + nr : k - np2; // new index k <- old index order[k]
        teig_pf     = teig;
        for (int k = 0; k < nt; ++k)
          {
            const int o       = order[k];
            teig_pf.kind[k]   = teig.kind[o];
            teig_pf.a[k]      = teig.a[o];
            teig_pf.b[k]      = teig.b[o];
            for (int j = 0; j < nt; ++j)
              {
                teig_pf.G[k * nt + j] = teig.G[o * nt + j]; // rows of G
                teig_pf.S[j * nt + k] = teig.S[j * nt + o]; // columns of S
              }
          }
      }
    else if (rowrec)
      {
        row_stride = storage == STMG_F32 ? vk_row_stride<float>(int(nd)) : vk_row_stride<__nv_bfloat16>(int(nd));
        if (storage == STMG_F32)
          {
            // mu in the row after the mode's entries
            mu_off    = int(nd * 4);
            mu_stride = row_stride;
            rec_bytes = int(nd * row_stride * 4);
          }
        else
          {
            mu_off    = int(pad(nd * row_stride * elem));
            mu_stride = 1;
            rec_bytes = int(pad(mu_off + nd * 4));
          }
      }
    else
      {
        row_stride = int(nd);
        mu_stride  = 1;
        mu_off     = int(pad(nd * nd * elem));
        rec_bytes  = int(pad(mu_off + nd * (compute == STMG_F64 ? 8 : 4)));
      }
    bool ok = false;
    if (slotrec)
      {
        shape[0] = shape[1] = 2;
        shape[2]            = dim == 3 ? 2 : 1;
        tiling              = make_tiling(mesh->v, shape);
        colour_cells        = 1;
        big                 = false;
        ok                  = smem_bytes(shape) <= 200 * 1024;
        slotrec             = ok;
      }
    for (bool b : {true, false})
      {
        if (!streamed || ok)
          break;
        vanka_shape(dim, p, b, shape);
        tiling       = make_tiling(mesh->v, shape);
        colour_cells = 1;
        for (int c = 0; c < (1 << dim); ++c)
          {
            int n = 1;
            for (int d = 0; d < dim; ++d)
              n *= (tiling.T[d] - ((c >> d) & 1) + 1) / 2;
            colour_cells = std::max(colour_cells, n);
          }
        if (smem_bytes(shape) <= (b ? 110 : 200) * 1024)
          {
            ok  = true;
            big = b;
            // deeper record pipelines while two CTAs per SM still fit
            if (rowrec)
              while (stages < vanka_detail::VR_STAGES_MAX)
                {
                  ++stages;
                  if (smem_bytes(shape) > (b ? 110 : 200) * 1024)
                    {
                      --stages;
                      break;
                    }
                }
          }
      }
    if (!ok)
      {
        streamed = false;
        STMG_REQUIRE(!rowrec, STMG_ERR_UNSUPPORTED, "vanka: row records do not fit in shared memory");
      }
    for (bool b : {true, false})
      {
        if (ok)
          break;
        vanka_shape(dim, p, b, shape);
        for (int ch : {8, 4, 2, 1})
          {
            chunk = ch;
            // big tiles only where they give every SM two tiles or more
            if (smem_bytes(shape) <= (b ? 112 : 200) * 1024 &&
                (!b || make_tiling(mesh->v, shape).n_tiles >= 2ll * sm_count()))
              {
                ok     = true;
                big    = b;
                tiling = make_tiling(mesh->v, shape);
                break;
              }
          }
      }
    STMG_REQUIRE(ok, STMG_ERR_UNSUPPORTED, "vanka: does not fit in shared memory");
    const long long slots =
      streamed ? tiling.n_tiles * (long long)tiling.T[0] * tiling.T[1] * tiling.T[2] : mesh->v.ncells;
    V.alloc(std::size_t(slots) * rec_bytes);
    // record padding (and the slots of cells beyond a partial tile) is read
    // by whole-row and whole-phase copies: keep it zero
    STMG_CUDA(cudaMemset(V.ptr, 0, std::size_t(slots) * rec_bytes));
#define STMG_SETUP(D, PP)                                                                                \
  if (dim == D && p == PP)                                                                               \
    run_setup<D, PP>(*this);
    STMG_SETUP(2, 1) STMG_SETUP(2, 2) STMG_SETUP(2, 3) STMG_SETUP(2, 4) STMG_SETUP(2, 5)
    STMG_SETUP(3, 1) STMG_SETUP(3, 2) STMG_SETUP(3, 3)
#undef STMG_SETUP
    shell.alloc(std::size_t(tiling.n_tiles) * nt * tiling.tile_stride * (compute == STMG_F64 ? 8 : 4));
  }

  void
  Vanka::apply(const void *src, void *dst, cudaStream_t s) const
  {
    apply_ex(src, dst, 1.0, 0.0, s);
  }

  namespace
  {
    std::mutex fault_mutex;
    int       *fault_host = nullptr, *fault_dev = nullptr;

    void
    fault_alloc()
    {
      std::lock_guard<std::mutex> lock(fault_mutex);
      if (!fault_host)
        {
          STMG_CUDA(cudaHostAlloc(&fault_host, sizeof(int), cudaHostAllocMapped));
          *fault_host = 0;
          STMG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&fault_dev), fault_host, 0));
        }
    }
  } // namespace

  int *
  vanka_fault_flag_device()
  {
    fault_alloc();
    return fault_dev;
  }

  void
  vanka_check_fault()
  {
    if (fault_host && *reinterpret_cast<volatile int *>(fault_host))
      throw Error(STMG_ERR_CUDA, "vanka: a record copy to shared memory did not complete in time (kernel gave up)");
  }

  void
  Vanka::apply_ex(const void *src, void *dst, double alpha, double beta, cudaStream_t s) const
  {
    STMG_REQUIRE(src && dst, STMG_ERR_ARG, "vanka: null vector");
    vanka_check_fault();
    if (mesh->v.dim == 2)
      return vanka_apply_2d(*this, src, dst, alpha, beta, s);
    return vanka_apply_3d(*this, src, dst, alpha, beta, s);
  }
} // namespace stmg
