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

  // 1-D weights of the coarse cell's Lagrange basis at the fine nodes inside
  // it: w[t][b], t = 0..2P (fine position, (fine cell half) * P + local
  // index), b = 0..P (coarse local node). Kernel parameter.
  template <typename T>
  struct HWeights
  {
    T w[2 * MAX_P + 1][MAX_P + 1];
  };

  class HTransfer final : public Transfer
  {
  public:
    HTransfer(Mesh *fine, Mesh *coarse, int nt, int dtype);
    void prolongate_add(const void *src, void *dst, cudaStream_t s) const override;
    void restrict_add(const void *src, void *dst, cudaStream_t s) const override;

    Mesh          *fine, *coarse;
    int            nt, dtype;
    HWeights<double> w64;
    HWeights<float>  w32;
    template <typename T>
    const HWeights<T> &hw() const
    {
      if constexpr (sizeof(T) == 8)
        return w64;
      else
        return w32;
    }
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
