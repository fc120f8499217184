// Host object behind stmg_vanka_t: the cell-patch space-time Vanka
// smoother in factored form (PreconditionVanka, tests/include/gmg.h:402-540).
#pragma once

#include "stmg_internal.h"

namespace stmg
{
  class Vanka
  {
  public:
    // compute: STMG_F32 (storage F32 or BF16) or STMG_F64 (storage F64).
    // A, B: host nt x nt time matrices of the level (Alpha, Beta).
    Vanka(Mesh *mesh, int nt, const double *A, const double *B, int compute, int storage);

    // dst = sum_c R_c^T diag(1/valence) B_c^{-1} R_c src (dst overwritten)
    void apply(const void *src, void *dst, cudaStream_t s) const;

    std::size_t smem_bytes(const Tiling &tl) const;
    template <typename T>
    const TimeMats<T> &tmats() const
    {
      if constexpr (sizeof(T) == 8)
        return tm64;
      else
        return tm32;
    }
    std::size_t inverse_bytes() const { return V.n + mu.n; }

    Mesh                 *mesh;
    int                   nt, compute, storage;
    Tiling                tiling;
    DevBuf<unsigned char> V;     // per cell, V as [mode][dof] in the storage type
    DevBuf<unsigned char> mu;    // per cell eigenvalues in the compute type
    DevBuf<unsigned char> shell; // tile face slots (scratch)
    TimeMats<double>      tm64;
    TimeMats<float>       tm32;
  };

  void vanka_apply_2d(const Vanka &vk, const void *src, void *dst, cudaStream_t s);
  void vanka_apply_3d(const Vanka &vk, const void *src, void *dst, cudaStream_t s);
} // namespace stmg
