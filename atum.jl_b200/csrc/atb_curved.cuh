// Curved-element (cubed-sphere) DGSEM tendency kernels: host-side entry
// points (atb_curved.cu).
#pragma once
#include "atb_tendency.cuh"

namespace atb {

// dynamic shared memory of a curved-element launch of E elements (fuse: the
// fused ARK23 stage with the radial linear operator)
size_t curved_smem_bytes(int vk, int naux, int Nq, int E, bool fuse = false);
// the fused ARK23 stage kernel on curved elements (Euler-gravity EC / KG
// tendency + radial weak-form linear Euler-gravity operator, Rusanov faces);
// nullptr when there is none
tend_launch_fn pick_launcher_curved_fused(int vk, int sflux, int lin_sflux);
// launcher for (law, volume kind, surface flux) on curved 3-D elements;
// nullptr when there is none (Euler, Euler-gravity: weak, central, EC, KG; linear Euler-gravity:
// weak, central)
tend_launch_fn pick_launcher_curved(int law, int vk, int sflux);

}  // namespace atb
