// Vanka apply kernels for 2-D meshes of degree 1.
#include "vanka_apply_impl.cuh"

namespace stmg
{
  template <>
  void
  vanka_apply_dp<2, 1>(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s)
  {
    vanka_detail::launch_apply1<2, 1>(vk, src, dst, alpha, beta, s);
  }
} // namespace stmg
