// Vanka apply for 2-D meshes (degrees 1 to 5).
#include "vanka_apply_impl.cuh"

namespace stmg
{
  void
  vanka_apply_2d(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s)
  {
    const int p = vk.mesh->v.p;
    if (p == 1)
      return vanka_detail::launch_apply1<2, 1>(vk, src, dst, alpha, beta, s);
    if (p == 2)
      return vanka_detail::launch_apply1<2, 2>(vk, src, dst, alpha, beta, s);
    if (p == 3)
      return vanka_detail::launch_apply1<2, 3>(vk, src, dst, alpha, beta, s);
    if (p == 4)
      return vanka_detail::launch_apply1<2, 4>(vk, src, dst, alpha, beta, s);
    if (p == 5)
      return vanka_detail::launch_apply1<2, 5>(vk, src, dst, alpha, beta, s);
    throw Error(STMG_ERR_UNSUPPORTED, "vanka: unsupported degree");
  }
} // namespace stmg
