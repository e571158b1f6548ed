// Tendency-kernel instantiations for LAW_EG with a runtime node count
// (one file per law so the instantiations compile in parallel).
#include "atb_tendency.cuh"
#include "atb_reduce.cuh"
namespace atb {
template <> tend_launch_fn pick_launcher<LAW_EG>(int dim, int vk) {
  if (dim == 1 && vk == VK_WEAK) return tend_launch<LAW_EG, 1, VK_WEAK, 0>;
  if (dim == 1 && vk == VK_CENTRAL) return tend_launch<LAW_EG, 1, VK_CENTRAL, 0>;
  if (dim == 1 && vk == VK_EC) return tend_launch<LAW_EG, 1, VK_EC, 0>;
  if (dim == 1 && vk == VK_KG) return tend_launch<LAW_EG, 1, VK_KG, 0>;
  if (dim == 2 && vk == VK_WEAK) return tend_launch<LAW_EG, 2, VK_WEAK, 0>;
  if (dim == 2 && vk == VK_CENTRAL) return tend_launch<LAW_EG, 2, VK_CENTRAL, 0>;
  if (dim == 2 && vk == VK_EC) return tend_launch<LAW_EG, 2, VK_EC, 0>;
  if (dim == 2 && vk == VK_KG) return tend_launch<LAW_EG, 2, VK_KG, 0>;
  if (dim == 3 && vk == VK_WEAK) return tend_launch<LAW_EG, 3, VK_WEAK, 0>;
  if (dim == 3 && vk == VK_CENTRAL) return tend_launch<LAW_EG, 3, VK_CENTRAL, 0>;
  if (dim == 3 && vk == VK_EC) return tend_launch<LAW_EG, 3, VK_EC, 0>;
  if (dim == 3 && vk == VK_KG) return tend_launch<LAW_EG, 3, VK_KG, 0>;
  if (dim == 1 && vk == VK_EC32) return tend_launch<LAW_EG, 1, VK_EC32, 0>;
  if (dim == 2 && vk == VK_EC32) return tend_launch<LAW_EG, 2, VK_EC32, 0>;
  if (dim == 3 && vk == VK_EC32) return tend_launch<LAW_EG, 3, VK_EC32, 0>;
  if (dim == 1 && vk == VK_KG32) return tend_launch<LAW_EG, 1, VK_KG32, 0>;
  if (dim == 2 && vk == VK_KG32) return tend_launch<LAW_EG, 2, VK_KG32, 0>;
  if (dim == 3 && vk == VK_KG32) return tend_launch<LAW_EG, 3, VK_KG32, 0>;
  return nullptr;
}
template <> red_launch_fn pick_reducer<LAW_EG>(int dim) {
  if (dim == 1) return red_launch<LAW_EG, 1>;
  if (dim == 2) return red_launch<LAW_EG, 2>;
  if (dim == 3) return red_launch<LAW_EG, 3>;
  return nullptr;
}
}  // namespace atb
