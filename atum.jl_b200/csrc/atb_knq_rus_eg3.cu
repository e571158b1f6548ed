// Compile-time node-count specialisations of the tendency kernel with the
// Rusanov surface flux built in (the kernel carries no other numerical flux:
// a smaller instruction stream), for the hot explicit configurations.
#include "atb_tendency.cuh"
namespace atb {
tend_launch_fn pick_rus_eg_3_ec(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EG, 3, VK_EC, 3, false, F_RUSANOV>;
    case 4: return tend_launch<LAW_EG, 3, VK_EC, 4, false, F_RUSANOV>;
    case 5: return tend_launch<LAW_EG, 3, VK_EC, 5, false, F_RUSANOV>;
    case 6: return tend_launch<LAW_EG, 3, VK_EC, 6, false, F_RUSANOV>;
    case 7: return tend_launch<LAW_EG, 3, VK_EC, 7, false, F_RUSANOV>;
    case 8: return tend_launch<LAW_EG, 3, VK_EC, 8, false, F_RUSANOV>;
  }
  return nullptr;
}
tend_launch_fn pick_rus_eg_3_ec32(int nq) {
  switch (nq) {
    case 3: return tend_launch<LAW_EG, 3, VK_EC32, 3, false, F_RUSANOV>;
    case 4: return tend_launch<LAW_EG, 3, VK_EC32, 4, false, F_RUSANOV>;
    case 5: return tend_launch<LAW_EG, 3, VK_EC32, 5, false, F_RUSANOV>;
    case 6: return tend_launch<LAW_EG, 3, VK_EC32, 6, false, F_RUSANOV>;
    case 7: return tend_launch<LAW_EG, 3, VK_EC32, 7, false, F_RUSANOV>;
    case 8: return tend_launch<LAW_EG, 3, VK_EC32, 8, false, F_RUSANOV>;
  }
  return nullptr;
}
}  // namespace atb
