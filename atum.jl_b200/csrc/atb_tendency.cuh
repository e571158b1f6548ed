// Fused DGSEM tendency kernel: volume term + surface term + sources + the
// time-stepper's write-back, one CTA pass per batch of elements.
//
// Replaces, for one stage, the reference's chain
//   dq .*= a                                   src/odesolvers.jl:51
//   esvolumeterm_dir! x dim  (or volumeterm!)  src/dgsem.jl:470-561 (217-306)
//   surfaceterm!                               src/dgsem.jl:683-732
//   q .+= b dt dq                              src/odesolvers.jl:53
// which makes dim+3 passes over the state and synchronises the host after
// every stage (src/dgsem.jl:97), by one kernel that reads q (and dq) once and
// writes dq (and the next q) once.
//
// Mapping: one thread per LGL node, E elements per CTA (E * Np threads).  The
// element's state, aux and per-node derived quantities (velocity, pressure,
// b = rho/2p, or the physical flux rows for the weak / central forms) are
// staged in shared memory with coalesced loads (SoA: consecutive threads,
// consecutive addresses).  Each thread sums its tensor lines' two-point fluxes
// in registers; brick metrics are diagonal, so only row `dir` of each
// two-point flux is evaluated, and the pair with itself (whose contribution
// D[i][i] w_i/w_i - D[i][i] vanishes) is skipped.  Face tasks (2*dim faces x
// Nfp nodes per element) gather the neighbour trace straight from global
// memory (L2-resident), evaluate the numerical flux once per face node and
// lift it into a shared-memory slot; after one barrier every node subtracts
// the slots of the faces it lies on, in face order, so corner nodes need no
// atomics and the result is deterministic.
//
// Epilogues (runtime-uniform):
//   EPI_SET      out = T                         (increment = false)
//   EPI_ADD      out += T                        (increment = true)
//   EPI_LSRK     out = a*out + T; out2 = q + bdt*out   (2N-storage LSRK stage,
//                                                 out2 is a second state buffer)
//   EPI_SUBOUT2  out = T; out2 -= T              (ARK, split_rhs = false:
//                                                 im_K = L(Q), ex_K -= im_K)
//   EPI_RLSRK    out = T; out2 = a*out2 + T      (relaxation LSRK: k, dq)
#pragma once
#include "atb_physics.cuh"

namespace atb {

enum { VK_WEAK = 0, VK_CENTRAL = 1, VK_EC = 2, VK_KG = 3 };
enum { EPI_SET = 0, EPI_ADD = 1, EPI_LSRK = 2, EPI_SUBOUT2 = 3, EPI_RLSRK = 4 };

struct TendArgs {
  int K, Nq, Np, Nfp, E, naux;
  const double* ginv;  // K*3: 2/h_d per element
  const int* nbr;      // K*6: neighbour element, or -(boundary tag)
  const double* aux;   // naux * stride
  const double* tab;   // Cfd[Nq*Nq], Cw[Nq*Nq], lift_end
  LawP law;
  int dirs, sflux, epi;
  double a, bdt;
  size_t stride;  // K*Np
  const double* q[5];
  double* out[5];
  double* out2[5];
};

template <int LAW, int DIM, int VK> struct NPre {
  static constexpr int NS = NSt<LAW, DIM>::v;
  static constexpr int v = (VK == VK_EC || VK == VK_KG) ? ((LAW == LAW_SW) ? DIM + 1 : DIM + 5) : DIM * NS;
};
// upper bound of the aux components a kernel stages (compile time, so the
// per-thread aux arrays stay in registers)
template <int LAW, int DIM> struct NAuxMax {
  static constexpr int v = (LAW == LAW_EG || LAW == LAW_LEG) ? DIM + 3 : (LAW == LAW_SW) ? DIM + 1 : 1;
};
// values stored per node pair: row d of the symmetric two-point flux, plus
// b_avg * rho_log for the Euler-gravity EC fluctuation
template <int LAW, int DIM, int VK> struct NPairVals {
  static constexpr int v = NSt<LAW, DIM>::v + ((LAW == LAW_EG && VK == VK_EC) ? 1 : 0);
};

inline size_t tend_smem_bytes(int ns, int npre, int naux, int dim, int Nq, int Np, int Nfp, int E, int npv) {
  const int npl = Nq * (Nq - 1) / 2;
  size_t per = (size_t)(ns + naux + npre) * Np + (size_t)2 * dim * Nfp * ns;
  if (npv > 0) per += (size_t)Nfp * npl * npv;
  return sizeof(double) * (2 * (size_t)Nq * Nq + 2 + per * E) + 64 * sizeof(int);
}

// pair index of nodes a < b on a line of Nq nodes
__device__ __forceinline__ int pair_index(int a, int b, int Nq) { return a * Nq - a * (a + 1) / 2 + (b - a - 1); }

template <int LAW, int DIM, int VK>
__global__ void __launch_bounds__(512) tendency_kernel(const TendArgs A) {
  constexpr int NS = NSt<LAW, DIM>::v;
  constexpr int NPRE = NPre<LAW, DIM, VK>::v;
  constexpr int NAM = NAuxMax<LAW, DIM>::v;
  constexpr bool PAIRS = (VK == VK_EC || VK == VK_KG);
  constexpr int NPV = PAIRS ? NPairVals<LAW, DIM, VK>::v : 0;
  extern __shared__ double sm[];
  const int Nq = A.Nq, Np = A.Np, Nfp = A.Nfp, naux = A.naux;
  const int npl = Nq * (Nq - 1) / 2;
  const int slot = threadIdx.x / Np;
  const int node = threadIdx.x - slot * Np;
  const int e = blockIdx.x * A.E + slot;
  const bool act = (slot < A.E) && (e < A.K);
  const int tabn = 2 * Nq * Nq + 2;
  double* sC = sm;            // Cfd
  double* sW = sm + Nq * Nq;  // Cw
  const size_t slotsz = (size_t)(NS + naux + NPRE) * Np + (size_t)2 * DIM * Nfp * NS + (size_t)Nfp * npl * NPV;
  double* sq = sm + tabn + slot * slotsz;
  double* sa = sq + NS * Np;
  double* sp = sa + naux * Np;
  double* ss = sp + NPRE * Np;
  double* spv = ss + 2 * DIM * Nfp * NS;  // pair values
  int* spair = (int*)(sm + tabn + A.E * slotsz);
  for (int t = threadIdx.x; t < tabn; t += blockDim.x) sm[t] = A.tab[t];
  if (PAIRS && threadIdx.x < npl) {
    int p = threadIdx.x, a = 0;
    while (p >= Nq - 1 - a) { p -= Nq - 1 - a; ++a; }
    spair[threadIdx.x] = a | ((a + 1 + p) << 8);
  }
  const LawP& L = A.law;
  const size_t gid = (size_t)e * Np + node;
  double qn[NS], an[NAM], Pn[NPRE > 0 ? NPRE : 1];
#pragma unroll
  for (int k = 0; k < NAM; ++k) an[k] = 0.0;
  if (act) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      qn[s] = __ldg(A.q[s] + gid);
      sq[s * Np + node] = qn[s];
    }
#pragma unroll
    for (int k = 0; k < NAM; ++k)
      if (k < naux) {
        an[k] = __ldg(A.aux + k * A.stride + gid);
        sa[k * Np + node] = an[k];
      }
    if constexpr (PAIRS) {
      if constexpr (LAW == LAW_SW) {
#pragma unroll
        for (int c = 0; c < DIM; ++c) Pn[c] = qn[1 + c] / qn[0];
        Pn[DIM] = qn[DIM + 1] / qn[0];
      } else {
        precompute_euler<DIM>(L.gamma, qn, (LAW == LAW_EG) ? an[0] : 0.0, Pn);
      }
#pragma unroll
      for (int k = 0; k < NPRE; ++k) sp[k * Np + node] = Pn[k];
    } else {
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        if (!((A.dirs >> d) & 1)) continue;
        double f[NS];
        flux_dir<LAW, DIM>(L, d, qn, an, f);
#pragma unroll
        for (int s = 0; s < NS; ++s) sp[(d * NS + s) * Np + node] = f[s];
      }
    }
  }
  __syncthreads();

  double T[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) T[s] = 0.0;
  const int ijk[3] = {node % Nq, (node / Nq) % Nq, node / (Nq * Nq)};
  double gi[3] = {0, 0, 0};
  if (act) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) gi[d] = __ldg(A.ginv + 3 * e + d);
    if ((A.dirs >> (DIM - 1)) & 1) add_sources<LAW, DIM>(L, VK == VK_WEAK, qn, an, T);
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    if (!((A.dirs >> d) & 1)) continue;
    const int sd = (d == 0) ? 1 : (d == 1) ? Nq : Nq * Nq;
    const int id = ijk[d];
    const int base = node - id * sd;
    if constexpr (PAIRS) {
      // ---- phase A: each unordered pair of each line of direction d once
      if (act) {
        for (int t = node; t < Nfp * npl; t += Np) {
          const int line = t / npl, p = t - line * npl;
          const int lb = (d == 0) ? line * Nq : (d == 1) ? (line % Nq) + Nq * Nq * (line / Nq) : line;
          const int ab = spair[p];
          const int na = lb + (ab & 0xff) * sd, nb = lb + (ab >> 8) * sd;
          double f[NPV];
          if constexpr (LAW == LAW_SW) {
            double q1[NS], q2[NS], P1[DIM + 1], P2[DIM + 1];
#pragma unroll
            for (int s = 0; s < NS; ++s) { q1[s] = sq[s * Np + na]; q2[s] = sq[s * Np + nb]; }
#pragma unroll
            for (int k = 0; k < DIM + 1; ++k) { P1[k] = sp[k * Np + na]; P2[k] = sp[k * Np + nb]; }
            sw_ec_dir<DIM>(L.grav, 0, d, q1, P1, 0.0, q2, P2, 0.0, f);
          } else {
            double P1[NPRE], P2[NPRE];
#pragma unroll
            for (int k = 0; k < NPRE; ++k) { P1[k] = sp[k * Np + na]; P2[k] = sp[k * Np + nb]; }
            const double Phi1 = (LAW == LAW_EG) ? sa[na] : 0.0, Phi2 = (LAW == LAW_EG) ? sa[nb] : 0.0;
            if constexpr (VK == VK_EC) {
              double x;
              ec_sym_dir<LAW, DIM>(L.gamma, d, sq[na], P1, Phi1, sq[nb], P2, Phi2, f, &x);
              if constexpr (NPV > NS) f[NS] = x;
            } else {
              kg_dir<LAW_EULER, DIM>(d, sq[na], P1, 0.0, sq[nb], P2, 0.0, f);
            }
          }
          double* dst = spv + (size_t)t * NPV;
#pragma unroll
          for (int s = 0; s < NPV; ++s) dst[s] = f[s];
        }
      }
      __syncthreads();
      // ---- phase B: every node contracts its row, adding its own fluctuation
      if (act) {
        const int line = (d == 0) ? node / Nq : (d == 1) ? ijk[0] + Nq * ijk[2] : node % (Nq * Nq);
        const double* lp = spv + (size_t)line * npl * NPV;
        for (int m = 0; m < Nq; ++m) {
          if (m == id) continue;
          const int p = (m < id) ? pair_index(m, id, Nq) : pair_index(id, m, Nq);
          const double* fv = lp + p * NPV;
          double f[NS];
#pragma unroll
          for (int s = 0; s < NS; ++s) f[s] = fv[s];
          const int nn = base + m * sd;
          if constexpr (LAW == LAW_EG) {
            const double dPhi = an[0] - sa[nn];
            if constexpr (VK == VK_EC)
              f[1 + d] = f[1 + d] - fv[NS] * Pn[DIM + 4] * dPhi;  // alpha = b_avg rho_log / (2 b_own)
            else
              f[1 + d] = f[1 + d] - ((qn[0] + sq[nn]) / 2.0 / 2.0) * dPhi;
          }
          if constexpr (LAW == LAW_SW) {
            if (L.swtopo) f[1 + d] = f[1 + d] - L.grav * qn[0] * (an[0] - sa[nn]) / 2.0;
          }
          const double c = sC[id * Nq + m] * gi[d];
#pragma unroll
          for (int s = 0; s < NS; ++s) T[s] = T[s] + c * f[s];
        }
      }
      __syncthreads();  // the pair buffer is reused by the next direction
    } else if (act) {
      for (int m = 0; m < Nq; ++m) {
        const int nn = base + m * sd;
        if constexpr (VK == VK_WEAK) {
          const double c = sW[id * Nq + m] * gi[d];
#pragma unroll
          for (int s = 0; s < NS; ++s) T[s] = T[s] + c * sp[(d * NS + s) * Np + nn];
        } else {  // central
          if (m == id) continue;
          const double c = sC[id * Nq + m] * gi[d];
#pragma unroll
          for (int s = 0; s < NS; ++s)
            T[s] = T[s] + c * ((sp[(d * NS + s) * Np + node] + sp[(d * NS + s) * Np + nn]) / 2.0);
        }
      }
    }
  }

  // ------------------------------------------------------------ faces
  const double lift_end = sm[2 * Nq * Nq];
  if (act) {
    for (int t = node; t < 2 * DIM * Nfp; t += Np) {
      const int face = t / Nfp, j = t - face * Nfp;
      const int d = face >> 1, side = face & 1;
      if (!((A.dirs >> d) & 1)) continue;
      const int t0 = j % Nq, t1 = j / Nq;
      int fi0, fi1, fi2;
      if (d == 0) { fi0 = side ? Nq - 1 : 0; fi1 = t0; fi2 = t1; }
      else if (d == 1) { fi0 = t0; fi1 = side ? Nq - 1 : 0; fi2 = t1; }
      else { fi0 = t0; fi1 = t1; fi2 = side ? Nq - 1 : 0; }
      const int nm = fi0 + Nq * (fi1 + Nq * fi2);
      double qm[NS], qp[NS], am[NAM], ap[NAM];
#pragma unroll
      for (int s = 0; s < NS; ++s) qm[s] = sq[s * Np + nm];
#pragma unroll
      for (int k = 0; k < NAM; ++k) am[k] = (k < naux) ? sa[k * Np + nm] : 0.0;
      const int nb = __ldg(A.nbr + 6 * e + face);
      const double sgn = side ? 1.0 : -1.0;
      if (nb >= 0) {
        const int flip = (Nq - 1) * (side ? -1 : 1);
        const int pn = nm + flip * ((d == 0) ? 1 : (d == 1) ? Nq : Nq * Nq);
        const size_t pid = (size_t)nb * Np + pn;
#pragma unroll
        for (int s = 0; s < NS; ++s) qp[s] = __ldg(A.q[s] + pid);
#pragma unroll
        for (int k = 0; k < NAM; ++k) ap[k] = (k < naux) ? __ldg(A.aux + k * A.stride + pid) : 0.0;
      } else {
        boundary_state<LAW, DIM>(L, d, sgn, -nb, qm, qp);
#pragma unroll
        for (int k = 0; k < NAM; ++k) ap[k] = am[k];
      }
      double nf[NS];
      surface_flux<LAW, DIM>(L, A.sflux, d, sgn, qm, am, qp, ap, nf);
      const double lift = gi[d] * lift_end;
#pragma unroll
      for (int s = 0; s < NS; ++s) ss[(face * Nfp + j) * NS + s] = lift * nf[s];
    }
  }
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    if (!((A.dirs >> d) & 1)) continue;
    const int id = ijk[d];
    if (id != 0 && id != Nq - 1) continue;
    const int face = 2 * d + (id == Nq - 1 ? 1 : 0);
    const int j = (d == 0) ? ijk[1] + Nq * ijk[2] : (d == 1) ? ijk[0] + Nq * ijk[2] : ijk[0] + Nq * ijk[1];
#pragma unroll
    for (int s = 0; s < NS; ++s) T[s] = T[s] - ss[(face * Nfp + j) * NS + s];
  }

  // --------------------------------------------------------- epilogue
  switch (A.epi) {
    case EPI_SET:
#pragma unroll
      for (int s = 0; s < NS; ++s) A.out[s][gid] = T[s];
      break;
    case EPI_ADD:
#pragma unroll
      for (int s = 0; s < NS; ++s) A.out[s][gid] = A.out[s][gid] + T[s];
      break;
    case EPI_LSRK:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double dqn = A.a * A.out[s][gid] + T[s];
        A.out[s][gid] = dqn;
        A.out2[s][gid] = qn[s] + A.bdt * dqn;
      }
      break;
    case EPI_SUBOUT2:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        A.out[s][gid] = T[s];
        A.out2[s][gid] = A.out2[s][gid] - T[s];
      }
      break;
    case EPI_RLSRK:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        A.out[s][gid] = T[s];
        A.out2[s][gid] = A.a * A.out2[s][gid] + T[s];
      }
      break;
  }
}

// launcher signature used by the host dispatch table
typedef void (*tend_launch_fn)(const TendArgs& A, int grid, int block, size_t smem, cudaStream_t st);

template <int LAW, int DIM, int VK>
void tend_launch(const TendArgs& A, int grid, int block, size_t smem, cudaStream_t st) {
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaFuncSetAttribute(tendency_kernel<LAW, DIM, VK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = smem;
  }
  tendency_kernel<LAW, DIM, VK><<<grid, block, smem, st>>>(A);
}

template <int LAW> tend_launch_fn pick_launcher(int dim, int vk);

// per-node precomputed values and per-pair stored values, for the host
inline int npre_of(int law, int dim, int vk) {
  int ns = (law == LAW_ADV) ? 1 : dim + 2;
  if (vk == VK_EC || vk == VK_KG) return (law == LAW_SW) ? dim + 1 : dim + 5;
  return dim * ns;
}
inline int npv_of(int law, int dim, int vk) {
  int ns = (law == LAW_ADV) ? 1 : dim + 2;
  if (vk == VK_EC || vk == VK_KG) return ns + ((law == LAW_EG && vk == VK_EC) ? 1 : 0);
  return 0;
}

}  // namespace atb
