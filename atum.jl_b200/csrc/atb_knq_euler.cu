// Compile-time node-count specialisations of the tendency kernel (hot
// configurations; the runtime-Nq kernel covers everything else).
#include "atb_tendency.cuh"
namespace atb {
tend_launch_fn pick_nq_euler_2_vk_ec(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EULER, 2, VK_EC, 3>;
    case 4: return tend_launch<LAW_EULER, 2, VK_EC, 4>;
    case 5: return tend_launch<LAW_EULER, 2, VK_EC, 5>;
    case 6: return tend_launch<LAW_EULER, 2, VK_EC, 6>;
    case 7: return tend_launch<LAW_EULER, 2, VK_EC, 7>;
    case 8: return tend_launch<LAW_EULER, 2, VK_EC, 8>;
  }
  return nullptr;
}
tend_launch_fn pick_nq_euler_3_vk_ec(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EULER, 3, VK_EC, 3>;
    case 4: return tend_launch<LAW_EULER, 3, VK_EC, 4>;
    case 5: return tend_launch<LAW_EULER, 3, VK_EC, 5>;
    case 6: return tend_launch<LAW_EULER, 3, VK_EC, 6>;
    case 7: return tend_launch<LAW_EULER, 3, VK_EC, 7>;
    case 8: return tend_launch<LAW_EULER, 3, VK_EC, 8>;
  }
  return nullptr;
}
}  // namespace atb
