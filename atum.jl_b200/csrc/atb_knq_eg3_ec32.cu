// Compile-time node-count specialisations of the tendency kernel, FP32-flux
// precision form of the entropy-conservative volume term.
#include "atb_tendency.cuh"
namespace atb {
tend_launch_fn pick_nq_eg_3_vk_ec32(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EG, 3, VK_EC32, 3>;
    case 4: return tend_launch<LAW_EG, 3, VK_EC32, 4>;
    case 5: return tend_launch<LAW_EG, 3, VK_EC32, 5>;
    case 6: return tend_launch<LAW_EG, 3, VK_EC32, 6>;
    case 7: return tend_launch<LAW_EG, 3, VK_EC32, 7>;
    case 8: return tend_launch<LAW_EG, 3, VK_EC32, 8>;
  }
  return nullptr;
}
}  // namespace atb
