// Compile-time node-count specialisations of the FP32-flux Kennedy-Gruber
// tendency kernel for 3-D Euler-gravity.
#include "atb_tendency.cuh"
namespace atb {
tend_launch_fn pick_nq_eg_3_vk_kg32(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EG, 3, VK_KG32, 3>;
    case 4: return tend_launch<LAW_EG, 3, VK_KG32, 4>;
    case 5: return tend_launch<LAW_EG, 3, VK_KG32, 5>;
    case 6: return tend_launch<LAW_EG, 3, VK_KG32, 6>;
    case 7: return tend_launch<LAW_EG, 3, VK_KG32, 7>;
    case 8: return tend_launch<LAW_EG, 3, VK_KG32, 8>;
  }
  return nullptr;
}
}  // namespace atb
