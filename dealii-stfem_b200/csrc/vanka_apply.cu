// Vanka apply dispatch by dimension and degree; the kernels of each
// (dimension, degree) are instantiated in their own vanka_apply_d*p*.cu so
// they compile in parallel.
#include "vanka.h"

namespace stmg
{
  void
  vanka_apply_2d(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s)
  {
    switch (vk.mesh->v.p)
      {
        case 1:
          return vanka_apply_dp<2, 1>(vk, src, dst, alpha, beta, s);
        case 2:
          return vanka_apply_dp<2, 2>(vk, src, dst, alpha, beta, s);
        case 3:
          return vanka_apply_dp<2, 3>(vk, src, dst, alpha, beta, s);
        case 4:
          return vanka_apply_dp<2, 4>(vk, src, dst, alpha, beta, s);
        case 5:
          return vanka_apply_dp<2, 5>(vk, src, dst, alpha, beta, s);
      }
    throw Error(STMG_ERR_UNSUPPORTED, "vanka: unsupported degree");
  }

  void
  vanka_apply_3d(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s)
  {
    switch (vk.mesh->v.p)
      {
        case 1:
          return vanka_apply_dp<3, 1>(vk, src, dst, alpha, beta, s);
        case 2:
          return vanka_apply_dp<3, 2>(vk, src, dst, alpha, beta, s);
        case 3:
          return vanka_apply_dp<3, 3>(vk, src, dst, alpha, beta, s);
      }
    throw Error(STMG_ERR_UNSUPPORTED, "vanka: unsupported degree");
  }
} // namespace stmg
