// Vanka apply for 3-D meshes (degrees 1, 2, 3).
#include "vanka_apply_impl.cuh"

namespace stmg
{
  void
  vanka_apply_3d(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s)
  {
    const int p = vk.mesh->v.p;
    if (p == 1)
      return vanka_detail::launch_apply1<3, 1>(vk, src, dst, alpha, beta, s);
    if (p == 2)
      return vanka_detail::launch_apply1<3, 2>(vk, src, dst, alpha, beta, s);
    if (p == 3)
      return vanka_detail::launch_apply1<3, 3>(vk, src, dst, alpha, beta, s);
    throw Error(STMG_ERR_UNSUPPORTED, "vanka: unsupported degree");
  }
} // namespace stmg
