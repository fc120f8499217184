// Host objects behind stmg_transfer_t: h-transfer between a mesh and its
// 2x refinement, and the time transfer (P (x) I) on one mesh.
#pragma once

#include "stmg_internal.h"

namespace stmg
{
  class Transfer
  {
  public:
    virtual ~Transfer() = default;
    // dst_fine += P src_coarse
    virtual void prolongate_add(const void *src, void *dst, cudaStream_t s) const = 0;
    // dst_coarse += R src_fine
    virtual void restrict_add(const void *src, void *dst, cudaStream_t s) const = 0;
  };

  class HTransfer final : public Transfer
  {
  public:
    HTransfer(Mesh *fine, Mesh *coarse, int nt, int dtype);
    void prolongate_add(const void *src, void *dst, cudaStream_t s) const override;
    void restrict_add(const void *src, void *dst, cudaStream_t s) const override;

    Mesh          *fine, *coarse;
    int            nt, dtype, maxr = 0;
    DevBuf<int>    p_start, r_cnt, r_f;
    DevBuf<double> p_w, r_w;
  };

  class TTransfer final : public Transfer
  {
  public:
    // P: nt_fine x nt_coarse; R: nt_coarse x nt_fine or null for P^T
    TTransfer(Mesh *mesh, int nt_fine, int nt_coarse, const double *P, const double *R, int dtype);
    void prolongate_add(const void *src, void *dst, cudaStream_t s) const override;
    void restrict_add(const void *src, void *dst, cudaStream_t s) const override;

    Mesh            *mesh;
    int              nt_fine, nt_coarse, dtype;
    TimeMats<double> P64, R64;
    TimeMats<float>  P32, R32;
  };
} // namespace stmg
