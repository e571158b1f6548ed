// Euler-gravity tendency kernels fused with the linear vertical operator
// (IMEX ARK23 stages): compile-time node counts for the hot orders, the
// runtime-Nq kernel otherwise.
#include "atb_tendency.cuh"
namespace atb {
template <int VK>
static tend_launch_fn pick_fused_vk(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EG, 3, VK, 3, true>;
    case 4: return tend_launch<LAW_EG, 3, VK, 4, true>;
    case 5: return tend_launch<LAW_EG, 3, VK, 5, true>;
    case 6: return tend_launch<LAW_EG, 3, VK, 6, true>;
    case 7: return tend_launch<LAW_EG, 3, VK, 7, true>;
    case 8: return tend_launch<LAW_EG, 3, VK, 8, true>;
  }
  return tend_launch<LAW_EG, 3, VK, 0, true>;
}
tend_launch_fn pick_launcher_fused(int dim, int vk, int nq) {
  if (dim != 3) return nullptr;
  if (vk == VK_EC) return pick_fused_vk<VK_EC>(nq);
  if (vk == VK_EC32) return pick_fused_vk<VK_EC32>(nq);
  return nullptr;
}
}  // namespace atb
