// Dispatch to the compile-time node-count specialisations (atb_knq_*.cu).
#include "atb_tendency.cuh"
namespace atb {
tend_launch_fn pick_nq_eg_2_vk_ec32(int nq);
tend_launch_fn pick_nq_euler_2_vk_ec32(int nq);
tend_launch_fn pick_nq_sw_2_vk_ec32(int nq);
tend_launch_fn pick_nq_eg_3_vk_ec32(int nq);
tend_launch_fn pick_nq_eg_3_vk_ec(int nq);
tend_launch_fn pick_nq_eg_3_vk_kg(int nq);
tend_launch_fn pick_nq_eg_3_vk_kg32(int nq);
tend_launch_fn pick_nq_eg_3_vk_weak(int nq);
tend_launch_fn pick_nq_eg_2_vk_ec(int nq);
tend_launch_fn pick_nq_leg_3_vk_weak(int nq);
tend_launch_fn pick_nq_leg_2_vk_weak(int nq);
tend_launch_fn pick_nq_euler_2_vk_ec(int nq);
tend_launch_fn pick_nq_euler_3_vk_ec(int nq);
tend_launch_fn pick_nq_sw_2_vk_ec(int nq);
tend_launch_fn pick_rus_eg_3_ec(int nq);
tend_launch_fn pick_rus_eg_3_ec32(int nq);
tend_launch_fn pick_rus_euler_2_ec(int nq);
tend_launch_fn pick_rus_euler_2_ec32(int nq);
tend_launch_fn pick_rus_sw_2_ec(int nq);
tend_launch_fn pick_rus_sw_2_ec32(int nq);
tend_launch_fn pick_launcher_rusanov(int law, int dim, int vk, int nq) {
  if (law == LAW_EG && dim == 3 && vk == VK_EC) return pick_rus_eg_3_ec(nq);
  if (law == LAW_EG && dim == 3 && vk == VK_EC32) return pick_rus_eg_3_ec32(nq);
  if (law == LAW_EULER && dim == 2 && vk == VK_EC) return pick_rus_euler_2_ec(nq);
  if (law == LAW_EULER && dim == 2 && vk == VK_EC32) return pick_rus_euler_2_ec32(nq);
  if (law == LAW_SW && dim == 2 && vk == VK_EC) return pick_rus_sw_2_ec(nq);
  if (law == LAW_SW && dim == 2 && vk == VK_EC32) return pick_rus_sw_2_ec32(nq);
  return nullptr;
}
template <> tend_launch_fn pick_launcher_nq<LAW_ADV>(int dim, int vk, int nq) {
  (void)dim; (void)vk; (void)nq;
  return nullptr;
}
template <> tend_launch_fn pick_launcher_nq<LAW_EULER>(int dim, int vk, int nq) {
  if (dim == 2 && vk == VK_EC32) return pick_nq_euler_2_vk_ec32(nq);
  if (dim == 2 && vk == VK_EC) return pick_nq_euler_2_vk_ec(nq);
  if (dim == 3 && vk == VK_EC) return pick_nq_euler_3_vk_ec(nq);
  (void)dim; (void)vk; (void)nq;
  return nullptr;
}
template <> tend_launch_fn pick_launcher_nq<LAW_EG>(int dim, int vk, int nq) {
  if (dim == 2 && vk == VK_EC32) return pick_nq_eg_2_vk_ec32(nq);
  if (dim == 3 && vk == VK_EC32) return pick_nq_eg_3_vk_ec32(nq);
  if (dim == 3 && vk == VK_EC) return pick_nq_eg_3_vk_ec(nq);
  if (dim == 3 && vk == VK_KG) return pick_nq_eg_3_vk_kg(nq);
  if (dim == 3 && vk == VK_KG32) return pick_nq_eg_3_vk_kg32(nq);
  if (dim == 3 && vk == VK_WEAK) return pick_nq_eg_3_vk_weak(nq);
  if (dim == 2 && vk == VK_EC) return pick_nq_eg_2_vk_ec(nq);
  (void)dim; (void)vk; (void)nq;
  return nullptr;
}
template <> tend_launch_fn pick_launcher_nq<LAW_LEG>(int dim, int vk, int nq) {
  if (dim == 3 && vk == VK_WEAK) return pick_nq_leg_3_vk_weak(nq);
  if (dim == 2 && vk == VK_WEAK) return pick_nq_leg_2_vk_weak(nq);
  (void)dim; (void)vk; (void)nq;
  return nullptr;
}
template <> tend_launch_fn pick_launcher_nq<LAW_SW>(int dim, int vk, int nq) {
  if (dim == 2 && vk == VK_EC32) return pick_nq_sw_2_vk_ec32(nq);
  if (dim == 2 && vk == VK_EC) return pick_nq_sw_2_vk_ec(nq);
  (void)dim; (void)vk; (void)nq;
  return nullptr;
}
}  // namespace atb
