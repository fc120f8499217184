// Space-time operator kernels for 2-D meshes of degree 1.
#include "op_apply_impl.cuh"

namespace stmg
{
  template <>
  void
  op_launch_dp<2, 1, float>(const OpLaunch<float> &L)
  {
    op_launch_impl<2, 1, float>(L);
  }

  template <>
  void
  op_launch_dp<2, 1, double>(const OpLaunch<double> &L)
  {
    op_launch_impl<2, 1, double>(L);
  }
} // namespace stmg
