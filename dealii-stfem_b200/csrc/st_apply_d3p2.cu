// Space-time operator kernels for 3-D meshes of degree 2.
#include "op_apply_impl.cuh"

namespace stmg
{
  template <>
  void
  op_launch_dp<3, 2, float>(const OpLaunch<float> &L)
  {
    op_launch_impl<3, 2, float>(L);
  }

  template <>
  void
  op_launch_dp<3, 2, double>(const OpLaunch<double> &L)
  {
    op_launch_impl<3, 2, double>(L);
  }
} // namespace stmg
