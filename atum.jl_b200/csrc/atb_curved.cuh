// Curved-element (cubed-sphere) DGSEM tendency kernels: host-side entry
// points (atb_curved.cu).
#pragma once
#include "atb_tendency.cuh"

namespace atb {

// dynamic shared memory of a curved-element launch of E elements
size_t curved_smem_bytes(int vk, int naux, int Nq, int E);
// launcher for (law, volume kind, surface flux) on curved 3-D elements;
// nullptr when there is none (Euler, Euler-gravity: weak, central, EC, KG; linear Euler-gravity:
// weak, central)
tend_launch_fn pick_launcher_curved(int law, int vk, int sflux);

}  // namespace atb
