// Persistent variants of the hot tendency kernels (atb_op_set_persistent):
// a few CTAs walk every element tile with a grid stride.  Rusanov surface
// flux built in, compile-time node counts for N = 3..5.
#include "atb_tendency.cuh"
namespace atb {
template <int LAW, int DIM, int VK, bool FUSE>
static tend_launch_fn pick_persist_nq(int nq) {
  switch (nq) {
    case 4: return tend_launch<LAW, DIM, VK, 4, FUSE, F_RUSANOV, true>;
    case 5: return tend_launch<LAW, DIM, VK, 5, FUSE, F_RUSANOV, true>;
    case 6: return tend_launch<LAW, DIM, VK, 6, FUSE, F_RUSANOV, true>;
  }
  return nullptr;
}
tend_launch_fn pick_launcher_persistent(int law, int dim, int vk, int nq, int sflux, bool fused, int lin_sflux) {
  if (sflux != F_RUSANOV || (fused && lin_sflux != F_RUSANOV)) return nullptr;
  if (fused) return (law == LAW_EG && dim == 3 && vk == VK_EC) ? pick_persist_nq<LAW_EG, 3, VK_EC, true>(nq) : nullptr;
  if (law == LAW_EG && dim == 3 && vk == VK_EC) return pick_persist_nq<LAW_EG, 3, VK_EC, false>(nq);
  if (law == LAW_EULER && dim == 2 && vk == VK_EC) return pick_persist_nq<LAW_EULER, 2, VK_EC, false>(nq);
  if (law == LAW_SW && dim == 2 && vk == VK_EC) return pick_persist_nq<LAW_SW, 2, VK_EC, false>(nq);
  if (law == LAW_SW && dim == 2 && vk == VK_EC32) return pick_persist_nq<LAW_SW, 2, VK_EC32, false>(nq);
  return nullptr;
}
}  // namespace atb
