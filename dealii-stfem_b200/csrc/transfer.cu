// Multigrid transfers between space-time levels.
//  h: FE_Q(p) interpolation from a mesh to its 2x refinement, per time
//     block, and its transpose (deal.II's MGTwoLevelTransfer as wrapped by
//     MGTwoLevelBlockTransfer, tests/include/gmg.h:35-75); on a structured
//     mesh the global prolongation is the tensor product of 1-D stencils, so
//     both directions run in gather form (one thread per output node, fixed
//     summation order, Dirichlet nodes zero on both sides).
//  t: (P (x) I) over the time blocks (MGTwoLevelTransferST::prolongate_and_add
//     / restrict_and_add, gmg.h:121-135, via tensorproduct_add,
//     operators.h:46-58).
#include <cmath>
#include <cstring>

#include "kernels_common.cuh"
#include "transfer.h"

namespace stmg
{
  namespace
  {
    template <typename T>
    __global__ void
    h_prolongate_kernel(const MeshView fm, const MeshView cm, int nt, const int *__restrict__ start,
                        const double *__restrict__ w, const T *__restrict__ src, T *__restrict__ dst)
    {
      const long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (node >= fm.N)
        return;
      const int g[3] = {int(node % fm.nn[0]), int((node / fm.nn[0]) % fm.nn[1]), int(node / ((long long)fm.nn[0] * fm.nn[1]))};
      if (is_boundary_node(fm, g[0], g[1], g[2]))
        return;
      const int p1 = fm.p + 1;
      // 1-D stencils: coarse nodes start[d][g_d] .. +p with weights
      int    s[3], cnt[3];
      const double *wd[3];
      long long off = 0;
      for (int d = 0; d < 3; ++d)
        {
          if (d < fm.dim)
            {
              s[d]   = start[off + g[d]];
              wd[d]  = w + (off + g[d]) * p1;
              cnt[d] = p1;
              off += fm.nn[d];
            }
          else
            {
              s[d]   = 0;
              wd[d]  = nullptr;
              cnt[d] = 1;
            }
        }
      for (int j = 0; j < nt; ++j)
        {
          T acc = T(0);
          for (int kz = 0; kz < cnt[2]; ++kz)
            {
              const double wz = wd[2] ? wd[2][kz] : 1.0;
              if (wz == 0.0)
                continue;
              for (int ky = 0; ky < cnt[1]; ++ky)
                {
                  const double wy = wd[1][ky] * wz;
                  if (wy == 0.0)
                    continue;
                  for (int kx = 0; kx < cnt[0]; ++kx)
                    {
                      const double wx = wd[0][kx] * wy;
                      if (wx == 0.0)
                        continue;
                      const int cx = s[0] + kx, cy = s[1] + ky, cz = s[2] + kz;
                      if (is_boundary_node(cm, cx, cy, cz))
                        continue;
                      acc += T(wx) * src[j * cm.N + cx + (long long)cm.nn[0] * (cy + (long long)cm.nn[1] * cz)];
                    }
                }
            }
          dst[j * fm.N + node] += acc;
        }
    }

    template <typename T>
    __global__ void
    h_restrict_kernel(const MeshView fm, const MeshView cm, int nt, int maxr, const int *__restrict__ cnt,
                      const int *__restrict__ fidx, const double *__restrict__ w, const T *__restrict__ src,
                      T *__restrict__ dst)
    {
      const long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      if (node >= cm.N)
        return;
      const int c[3] = {int(node % cm.nn[0]), int((node / cm.nn[0]) % cm.nn[1]), int(node / ((long long)cm.nn[0] * cm.nn[1]))};
      if (is_boundary_node(cm, c[0], c[1], c[2]))
        return;
      int           n[3];
      const int    *f[3];
      const double *wd[3];
      long long     off = 0;
      for (int d = 0; d < 3; ++d)
        {
          if (d < cm.dim)
            {
              n[d]  = cnt[off + c[d]];
              f[d]  = fidx + (off + c[d]) * maxr;
              wd[d] = w + (off + c[d]) * maxr;
              off += cm.nn[d];
            }
          else
            {
              n[d]  = 1;
              f[d]  = nullptr;
              wd[d] = nullptr;
            }
        }
      for (int j = 0; j < nt; ++j)
        {
          T acc = T(0);
          for (int kz = 0; kz < n[2]; ++kz)
            {
              const int    fz = f[2] ? f[2][kz] : 0;
              const double wz = wd[2] ? wd[2][kz] : 1.0;
              for (int ky = 0; ky < n[1]; ++ky)
                {
                  const int    fy = f[1][ky];
                  const double wy = wd[1][ky] * wz;
                  for (int kx = 0; kx < n[0]; ++kx)
                    {
                      const int fx = f[0][kx];
                      if (is_boundary_node(fm, fx, fy, fz))
                        continue;
                      acc += T(wd[0][kx] * wy) * src[j * fm.N + fx + (long long)fm.nn[0] * (fy + (long long)fm.nn[1] * fz)];
                    }
                }
            }
          dst[j * cm.N + node] += acc;
        }
    }

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
    maxr                = 4 * p + 1;
    std::vector<int>    start, cnt, fidx;
    std::vector<double> w, rw;
    for (int d = 0; d < f.dim; ++d)
      {
        // coarse node -> list of (fine node, weight)
        std::vector<std::vector<std::pair<int, double>>> col(c.nn[d]);
        for (int g = 0; g < f.nn[d]; ++g)
          {
            const int    fc = std::min(g / p, f.n[d] - 1);
            const int    a  = g - fc * p;
            const int    cc = fc / 2;
            const double xi = 0.5 * ((fc % 2) + t.xs[p][a]);
            start.push_back(cc * p);
            for (int b = 0; b < p1; ++b)
              {
                double v = 1.0;
                for (int k = 0; k < p1; ++k)
                  if (k != b)
                    v *= (xi - t.xs[p][k]) / (t.xs[p][b] - t.xs[p][k]);
                if (std::abs(v) < 1e-14)
                  v = 0.0;
                w.push_back(v);
                if (v != 0.0)
                  col[cc * p + b].emplace_back(g, v);
              }
          }
        for (int i = 0; i < c.nn[d]; ++i)
          {
            STMG_REQUIRE(int(col[i].size()) <= maxr, STMG_ERR_SHAPE, "h-transfer: stencil overflow");
            cnt.push_back(int(col[i].size()));
            for (int k = 0; k < maxr; ++k)
              {
                fidx.push_back(k < int(col[i].size()) ? col[i][k].first : 0);
                rw.push_back(k < int(col[i].size()) ? col[i][k].second : 0.0);
              }
          }
      }
    p_start.upload(start);
    p_w.upload(w);
    r_cnt.upload(cnt);
    r_f.upload(fidx);
    r_w.upload(rw);
  }

  void
  HTransfer::prolongate_add(const void *src, void *dst, cudaStream_t s) const
  {
    const MeshView &f = fine->v, &c = coarse->v;
    const unsigned  nb = unsigned((f.N + 255) / 256);
    if (dtype == STMG_F64)
      h_prolongate_kernel<double><<<nb, 256, 0, s>>>(f, c, nt, p_start.ptr, p_w.ptr, static_cast<const double *>(src),
                                                     static_cast<double *>(dst));
    else
      h_prolongate_kernel<float><<<nb, 256, 0, s>>>(f, c, nt, p_start.ptr, p_w.ptr, static_cast<const float *>(src),
                                                    static_cast<float *>(dst));
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

  void
  HTransfer::restrict_add(const void *src, void *dst, cudaStream_t s) const
  {
    const MeshView &f = fine->v, &c = coarse->v;
    const unsigned  nb = unsigned((c.N + 255) / 256);
    if (dtype == STMG_F64)
      h_restrict_kernel<double><<<nb, 256, 0, s>>>(f, c, nt, maxr, r_cnt.ptr, r_f.ptr, r_w.ptr,
                                                   static_cast<const double *>(src), static_cast<double *>(dst));
    else
      h_restrict_kernel<float><<<nb, 256, 0, s>>>(f, c, nt, maxr, r_cnt.ptr, r_f.ptr, r_w.ptr,
                                                  static_cast<const float *>(src), static_cast<float *>(dst));
    count_launch();
    STMG_CUDA(cudaGetLastError());
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
