// Euler-gravity tendency kernels fused with the linear vertical operator
// (IMEX ARK23 stages): compile-time node counts for the hot orders, the
// runtime-Nq kernel otherwise; with both operators' surface flux Rusanov, a
// kernel with that flux built in (the other fluxes' code is not carried).
#include "atb_tendency.cuh"
namespace atb {
template <int VK, int SF>
static tend_launch_fn pick_fused_vk(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EG, 3, VK, 3, true, SF>;
    case 4: return tend_launch<LAW_EG, 3, VK, 4, true, SF>;
    case 5: return tend_launch<LAW_EG, 3, VK, 5, true, SF>;
    case 6: return tend_launch<LAW_EG, 3, VK, 6, true, SF>;
    case 7: return tend_launch<LAW_EG, 3, VK, 7, true, SF>;
    case 8: return tend_launch<LAW_EG, 3, VK, 8, true, SF>;
  }
  return tend_launch<LAW_EG, 3, VK, 0, true, SF>;
}
tend_launch_fn pick_launcher_fused(int dim, int vk, int nq, int sflux, int lin_sflux) {
  if (dim != 3) return nullptr;
  const bool rus = sflux == F_RUSANOV && lin_sflux == F_RUSANOV;
  if (vk == VK_EC) return rus ? pick_fused_vk<VK_EC, F_RUSANOV>(nq) : pick_fused_vk<VK_EC, -1>(nq);
  if (vk == VK_EC32) return rus ? pick_fused_vk<VK_EC32, F_RUSANOV>(nq) : pick_fused_vk<VK_EC32, -1>(nq);
  return nullptr;
}
}  // namespace atb
