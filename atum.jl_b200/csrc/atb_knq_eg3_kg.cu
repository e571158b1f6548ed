// Compile-time node-count specialisations of the tendency kernel (hot
// configurations; the runtime-Nq kernel covers everything else).
#include "atb_tendency.cuh"
namespace atb {
tend_launch_fn pick_nq_eg_3_vk_kg(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EG, 3, VK_KG, 3>;
    case 4: return tend_launch<LAW_EG, 3, VK_KG, 4>;
    case 5: return tend_launch<LAW_EG, 3, VK_KG, 5>;
    case 6: return tend_launch<LAW_EG, 3, VK_KG, 6>;
    case 7: return tend_launch<LAW_EG, 3, VK_KG, 7>;
    case 8: return tend_launch<LAW_EG, 3, VK_KG, 8>;
  }
  return nullptr;
}
}  // namespace atb
