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
//   EPI_LSRK     out = a*out + T (out = T when a = 0); out2 = q + bdt*out
//                (2N-storage LSRK stage, out2 a second state buffer; with
//                dte set, bdt*dte[e] replaces bdt: per-instance steps)
//   EPI_SUBOUT2  out = T; out2 -= T              (ARK, split_rhs = false:
//                                                 im_K = L(Q), ex_K -= im_K)
//   EPI_RLSRK    out = T; out2 = a*out2 + T      (relaxation LSRK: k, dq)
//   EPI_ARK      IMEX stage of ARK23 with split_rhs = false, T = L(Q): with
//                E = out - T (explicit part, out holding N(Q)) and I = T,
//                every active accumulator j gets
//                acc_j = (accin_j or Q) + adt*(ca_j*E + cb_j*I)
//                -- the stage right-hand sides and the final update are
//                accumulated here, so E and I are never stored
#pragma once
#include "atb_generic.cuh"
#include "atb_physics.cuh"

namespace atb {

__device__ __forceinline__ void tend_cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// VK_EC32: the entropy-conservative volume flux in the FP32-flux precision
// form (mixed: balance-critical terms in FP64 adds/multiplies, the rest FP32)
// VK_KG32: the Kennedy-Gruber volume flux in the FP32-flux precision form
// (FP64 rho and p averages, FP32 velocities, energies and products)
enum { VK_WEAK = 0, VK_CENTRAL = 1, VK_EC = 2, VK_KG = 3, VK_EC32 = 4, VK_KG32 = 5 };
enum { EPI_SET = 0, EPI_ADD = 1, EPI_LSRK = 2, EPI_SUBOUT2 = 3, EPI_RLSRK = 4, EPI_ARK = 5 };

// neighbour-table encoding: relative offsets for interior faces, so an
// instance's rows move between element ranges unchanged; NBR_BOUNDARY + tag
// (tag = face number 1..6) on a non-periodic boundary face
constexpr int NBR_BOUNDARY = -2147483647 - 1;

struct TendArgs {
  int K, Nq, Np, Nfp, E, naux;
  const double* ginv;  // K*3: 2/h_d per element
  const int* nbr;      // K*6: neighbour element - e, or NBR_BOUNDARY + tag
  const double* aux;   // naux * stride
  const double* tab;   // Cfd[Nq*Nq], Cw[Nq*Nq], lift_end
  LawP law;
  int dirs, sflux, epi;
  double a, bdt;
  const double* dte;  // per-element time step (batched instances), or null
  // EPI_ARK accumulators (acc[j][0] null: inactive; accin[j][0] null: base Q)
  double* acc[3][5];
  const double* accin[3][5];
  double ca[3], cb[3], adt;
  // fused linear operator (tendency_kernel<..., FUSE = true>): the linear
  // Euler-gravity law, its surface flux and directions
  LawP lin_law;
  int lin_sflux, lin_dirs;
  int naux_nl;  // aux components the explicit operator's faces read (fused launches stage more)
  int pf;       // epilogue input fields prefetched into shared memory (0: read at the end)
  size_t stride;      // K*Np
  // curved elements (atb_curved.cu): D[i][m], metric terms G[(d*3 + c)*stride
  // + gid] = d xi_d / d x_c, M J per node, per face node (e*6 + face)*Nfp + j
  // the outward unit normal (3 values), faceMJ, and the neighbour's global
  // node index (-1 - tag on a boundary face)
  const double* Dmat;
  const double* G;
  const double* MJn;
  const double* fnrm;
  const double* fMJ;
  const int* fnb;
  const double* q[5];
  double* out[5];
  double* out2[5];
};

// Per-node values staged for the volume term:
//   EC (Euler / Euler-gravity): u (DIM), b = rho/2p, |u|^2, p/rho
//   KG: u (DIM), p, e = rho e / rho
//   EC (shallow water): u (DIM), theta
//   weak / central forms: the DIM physical flux rows (DIM * NS)
//   EC32 (Euler / Euler-gravity): FP64 p, b, p/rho, then FP32 u (DIM), |u|^2
//         packed two per double slot
//   EC32 (shallow water): FP32 u (DIM), theta, packed
template <int LAW, int DIM, int VK> struct NPre {
  static constexpr int NS = NSt<LAW, DIM>::v;
  static constexpr int v = (VK == VK_EC)     ? ((LAW == LAW_SW) ? DIM + 1 : DIM + 3)
                           : (VK == VK_KG)   ? DIM + 2
                           : (VK == VK_EC32) ? ((LAW == LAW_SW) ? (DIM + 2) / 2 : 3 + (DIM + 2) / 2)
                           : (VK == VK_KG32) ? 1 + (DIM + 2) / 2
                                             : DIM * NS;
};
// upper bound of the aux components a kernel stages (compile time, so the
// per-thread aux arrays stay in registers)
template <int LAW, int DIM> struct NAuxMax {
  static constexpr int v = (LAW == LAW_EG || LAW == LAW_LEG) ? DIM + 3 : (LAW == LAW_SW) ? DIM + 1 : 1;
};
// values stored per node pair: row d of the symmetric two-point flux, plus
// b_avg * rho_log for the Euler-gravity EC fluctuation; the stride is odd so
// that consecutive pairs fall in different shared-memory banks
template <int LAW, int DIM, int VK> struct NPairVals {
  static constexpr int v = NSt<LAW, DIM>::v + ((LAW == LAW_EG && (VK == VK_EC || VK == VK_EC32)) ? 1 : 0);
  static constexpr int stride = v | 1;
};

// cmp: the compact layout of the fused Euler-gravity stage (fused_compact_fits)
inline size_t tend_smem_bytes(int ns, int npre, int naux, int dim, int Nq, int Np, int Nfp, int E, int npvs,
                              bool fuse = false, int pf = 0, bool cmp = false) {
  const int npl = Nq * (Nq - 1) / 2;
  size_t per;
  if (cmp) {
    per = (size_t)(ns + 3 + npre) * Np + (size_t)Nfp * npl * npvs + (size_t)ns * Np;
  } else {
    per = (size_t)(ns + naux + npre) * Np + (size_t)2 * dim * Nfp * ns;
    if (npvs > 0) per += (size_t)Nfp * npl * npvs;
    if (fuse) per += (size_t)ns * Np + (size_t)2 * Nfp * ns;  // linear flux rows, linear face slots
  }
  per += (size_t)pf * ns * Np;  // prefetched epilogue inputs
  return sizeof(double) * (2 * (size_t)Nq * Nq + 2 + per * E) + 64 * sizeof(int);
}

__host__ __device__ constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// Compact shared-memory layout of the fused Euler-gravity ARK stage: three
// aux fields per node are staged (Phi, rho_ref, p_ref -- all that the volume
// term and the face fluxes read of other nodes; grad Phi enters only the
// linear operator's source, evaluated from registers before the face tasks),
// the explicit face slots reuse the per-node precomputed values' region, and
// the parked accumulators, the parked linear source and the linear face slots
// reuse the pair buffer once the volume term is done.  It applies when those
// regions are large enough (Nq >= 5 for the FP64 EC flux).
__host__ __device__ constexpr bool fused_compact_fits(int nq, int dim, int ns, int npre, int npvs) {
  return nq > 0 && npre * ipow(nq, dim) >= 2 * dim * ipow(nq, dim - 1) * ns &&
         ipow(nq, dim - 1) * (nq * (nq - 1) / 2) * npvs >= (ns + dim) * ipow(nq, dim) + 2 * ipow(nq, dim - 1) * ns;
}

// volume-term two-point fluxes on the staged per-node layouts (row d)
//
// EC flux: when both logarithmic means are on their series branch
// (u = ((a-b)/(a+b))^2 < 1e-2 for rho and for b, the common case between
// the nodes of an element of a resolved flow) every division of the flux
// shares ONE reciprocal, 1/((r1+r2)^2 (b1+b2)^2):
//   rho_log = (r1+r2)/2 * G(u_rho),  b_log = (b1+b2)/2 * G(u_b),
//   rho_avg/(2 b_avg) = (r1+r2)/2 / (b1+b2),
//   1/(2 (gamma-1) b_log) = F(u_b) / ((gamma-1) (b1+b2)),
// with F(u) = 1 + u/3 + u^2/5 + ... + u^7/15 (the reference's series, longer)
// and G = 1/F to the same order (truncation below 1e-17 relative for
// u < 1e-2).  Otherwise the general form below is used.  A wide series range
// keeps the pairs of a warp on one branch.
template <int LAW, int DIM, class T>
__device__ __forceinline__ void ec_vol(T gamma, T igm1, int d, T r1, const T* P1, T Phi1, T r2, const T* P2, T Phi2,
                                       T* f, T* xtra) {
  const T rho_avg = (r1 + r2) / T(2);
  T ua[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) ua[c] = (P1[c] + P2[c]) / T(2);
  const T b1 = P1[DIM], b2 = P2[DIM];
  const T b_avg = (b1 + b2) / T(2);
  const T u2_avg = (P1[DIM + 1] + P2[DIM + 1]) / T(2);
  const T rs = r1 + r2, rd = r1 - r2, bs = b1 + b2, bd = b1 - b2;
  const T rs2 = rs * rs, bs2 = bs * bs, rd2 = rd * rd, bd2 = bd * bd;
  T rho_log, pc, cterm;
  if (rd2 < T(1e-2) * rs2 && bd2 < T(1e-2) * bs2) {
    const T inv = T(1) / (rs2 * bs2);
    const T ur = rd2 * bs2 * inv, ub = bd2 * rs2 * inv;
    const T inv_bs = bs * rs2 * inv;  // 1 / (b1 + b2)
    rho_log = rho_avg * series_G(ur);
    pc = rho_avg * inv_bs;
    cterm = series_F(ub) * inv_bs * igm1;
  } else {
    rho_log = logavg_fast(r1, r2);
    const T b_log = logavg_fast(b1, b2);
    const T rinv = T(1) / (b_avg * b_log);  // shared by rho_avg/(2 b_avg) and 1/(2(gamma-1) b_log)
    pc = rho_avg * b_log * rinv / T(2);
    cterm = b_avg * rinv * igm1 / T(2);
  }
  (void)gamma;
  const T ud = ua[d];
  const T frd = ud * rho_log;
  f[0] = frd;
  T mu = T(0);
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    T m = ud * (ua[c] * rho_log);
    if (c == d) m = m + pc;
    f[1 + c] = m;
    mu = (c == 0) ? m * ua[c] : mu + m * ua[c];
  }
  T c1 = cterm - u2_avg / T(2);
  if (LAW == LAW_EG) c1 = c1 + (Phi1 + Phi2) / T(2);
  f[DIM + 1] = c1 * frd + mu;
  *xtra = b_avg * rho_log;
}

template <int DIM, class T>
__device__ __forceinline__ void kg_vol(int d, T r1, const T* P1, T r2, const T* P2, T* f) {
  const T rho_avg = (r1 + r2) / T(2);
  const T ud = (P1[d] + P2[d]) / T(2);
  const T p_avg = (P1[DIM] + P2[DIM]) / T(2);
  const T e_avg = (P1[DIM + 1] + P2[DIM + 1]) / T(2);
  const T frd = ud * rho_avg;
  f[0] = frd;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    T m = ud * (((P1[c] + P2[c]) / T(2)) * rho_avg);
    if (c == d) m = m + p_avg;
    f[1 + c] = m;
  }
  f[DIM + 1] = ud * (rho_avg * e_avg + p_avg);
}

// pair index of nodes a < b on a line of Nq nodes
__device__ __forceinline__ int pair_index(int a, int b, int Nq) { return a * Nq - a * (a + 1) / 2 + (b - a - 1); }

// one face-node task (face t / Nfp of direction D_, node t % Nfp): gather
// the neighbour trace (or the boundary state), evaluate the numerical flux and
// store it lifted into the face's shared-memory slot
// CMPA: the staged aux fields are the compact [Phi, rho_ref, p_ref]
// (components 0, DIM+1, DIM+2; the face fluxes read no others)
template <int LAW, int DIM, int NAM, int D_, bool F32S = false, bool CMPA = false>
__device__ __forceinline__ void face_task(const TendArgs& A, const LawP& L, int sflux, int naux, int Nq, int Np,
                                          int Nfp, int e, int t, const double* sq, const double* sa, double* ss,
                                          double gid, double lift_end) {
  constexpr int NS = NSt<LAW, DIM>::v;
  const int face = t / Nfp, j = t - face * Nfp;
  const int side = face & 1;
  if (!((A.dirs >> D_) & 1)) return;
  const int t0 = j % Nq, t1 = j / Nq;
  const int fix = side ? Nq - 1 : 0;
  const int nm = (D_ == 0) ? fix + Nq * (t0 + Nq * t1) : (D_ == 1) ? t0 + Nq * (fix + Nq * t1) : t0 + Nq * (t1 + Nq * fix);
  double qm[NS], qp[NS], am[NAM], ap[NAM];
#pragma unroll
  for (int s = 0; s < NS; ++s) qm[s] = sq[s * Np + nm];
#pragma unroll
  for (int k = 0; k < NAM; ++k) {
    if constexpr (CMPA) {
      const int c = (k == 0) ? 0 : (k == DIM + 1) ? 1 : (k == DIM + 2) ? 2 : -1;
      am[k] = (k < naux && c >= 0) ? sa[c * Np + nm] : 0.0;
    } else {
      am[k] = (k < naux) ? sa[k * Np + nm] : 0.0;
    }
  }
  // neighbour table entries are relative (neighbour element - e), or a
  // boundary tag offset by NBR_BOUNDARY
  const int nv = __ldg(A.nbr + 6 * e + face);
  const double sgn = side ? 1.0 : -1.0;
  if (nv > NBR_BOUNDARY + 64) {
    const int nb = e + nv;
    const int stride_d = (D_ == 0) ? 1 : (D_ == 1) ? Nq : Nq * Nq;
    const int pn = nm + (side ? -(Nq - 1) : (Nq - 1)) * stride_d;
    const size_t pid = (size_t)nb * Np + pn;
#pragma unroll
    for (int s = 0; s < NS; ++s) qp[s] = __ldg(A.q[s] + pid);
#pragma unroll
    for (int k = 0; k < NAM; ++k) ap[k] = (k < naux) ? __ldg(A.aux + k * A.stride + pid) : 0.0;
  } else {
    boundary_state<LAW, DIM>(L, D_, sgn, nv - NBR_BOUNDARY, qm, qp);
#pragma unroll
    for (int k = 0; k < NAM; ++k) ap[k] = am[k];
  }
  double nf[NS];
  bool done = false;
  if constexpr (F32S) done = surface_flux32<LAW, DIM>(L, sflux, D_, sgn, qm, am, qp, ap, nf);
  if (!done) surface_flux<LAW, DIM>(L, sflux, D_, sgn, qm, am, qp, ap, nf);
  const double lift = gid * lift_end;
#pragma unroll
  for (int s = 0; s < NS; ++s) ss[(face * Nfp + j) * NS + s] = lift * nf[s];
}

// NQ_ > 0: the node count per direction is a compile-time constant (index
// arithmetic folds, line loops unroll); NQ_ = 0 reads it from the arguments.
// CTA size limit of the fused kernels: 256 threads unless one element needs
// more; with the compact layout at Nq = 5 (125 nodes), one element per CTA of
// 128 threads, four CTAs per SM at the full 128-register budget (measured on
// B200: faster than five CTAs at 96 registers, whose spills cost more than
// the added warps gain).  cmp: the kernel uses the compact layout
// (fused_compact_fits).
__host__ __device__ constexpr int fused_max_threads(int nq, bool cmp = false) {
  return (nq == 0 || nq * nq * nq > 256) ? 512 : (cmp && nq == 5) ? 128 : 256;
}
__host__ __device__ constexpr int fused_min_blocks(int nq, bool cmp = false) {
  return (cmp && nq == 5) ? 4 : 512 / fused_max_threads(nq, cmp);
}

// Plain launches: up to 512 threads.  Fused launches (which carry the linear
// operator too): fused_max_threads, with enough resident CTAs requested that
// the register budget stays at 128 -- measured faster on B200 than the
// spill-free 156-register allocation, whose lower occupancy costs more.
//
// SF >= 0: the surface flux kind (of the explicit operator and, fused, of the
// linear one) is a compile-time constant, so the kernel carries one numerical
// flux instead of all of them; SF = -1 reads it from the arguments.
//
// PERSIST: a persistent launch -- fewer CTAs than tiles of E elements, each
// CTA walking the tiles (of every packed instance) with a grid stride and
// restaging shared memory for each; otherwise one CTA per tile.  The tile's
// work is the same code either way (tile_body).
template <int LAW, int DIM, int VK, int NQ_, bool FUSE = false, int SF = -1, bool PERSIST = false>
__global__ void __launch_bounds__(
    FUSE ? fused_max_threads(NQ_, LAW == LAW_EG && fused_compact_fits(NQ_, DIM, NSt<LAW, DIM>::v, NPre<LAW, DIM, VK>::v,
                                                                        NPairVals<LAW, DIM, VK>::stride))
         : 512,
    FUSE ? fused_min_blocks(NQ_, LAW == LAW_EG && fused_compact_fits(NQ_, DIM, NSt<LAW, DIM>::v, NPre<LAW, DIM, VK>::v,
                                                                       NPairVals<LAW, DIM, VK>::stride))
         : 1) tendency_kernel(const TendArgs A) {
  constexpr int NS = NSt<LAW, DIM>::v;
  constexpr int NPRE = NPre<LAW, DIM, VK>::v;
  constexpr int NAM = NAuxMax<LAW, DIM>::v;
  constexpr bool PAIRS = (VK == VK_EC || VK == VK_KG || VK == VK_EC32 || VK == VK_KG32);
  // FP32-flux form: the explicit operator's surface flux in FP32 too (the
  // fused linear operator keeps FP64, like the implicit solve)
  constexpr bool F32S = (VK == VK_EC32 || VK == VK_KG32);
  constexpr int PR_IDX = (VK == VK_EC32) ? 2 : DIM + 2;  // p/rho in the own-node values
  constexpr int NPV = PAIRS ? NPairVals<LAW, DIM, VK>::v : 0;
  constexpr int NPVS = PAIRS ? NPairVals<LAW, DIM, VK>::stride : 0;
  constexpr bool CQ = NQ_ > 0;
  // the fused kernel runs the ARK23 stage epilogue only
  const int epi = FUSE ? EPI_ARK : A.epi;
  const int sflux = SF >= 0 ? SF : A.sflux;
  const int lin_sflux = SF >= 0 ? SF : A.lin_sflux;
  extern __shared__ double sm[];
  const int Nq = CQ ? NQ_ : A.Nq;
  const int Np = CQ ? ipow(NQ_, DIM) : A.Np;
  const int Nfp = CQ ? ipow(NQ_, DIM - 1) : A.Nfp;
  const int naux = A.naux;
  const int npl = Nq * (Nq - 1) / 2;
  constexpr bool CMP = FUSE && LAW == LAW_EG && fused_compact_fits(NQ_, DIM, NS, NPRE, NPVS);
  const int slot = threadIdx.x / Np;
  const int node = threadIdx.x - slot * Np;
  const int tabn = 2 * Nq * Nq + 2;
  double* sC = sm;            // Cfd
  double* sW = sm + Nq * Nq;  // Cw
  const int naux_s = CMP ? 3 : naux;  // aux fields staged in shared memory
  const size_t slotsz =
      CMP ? (size_t)(NS + 3 + NPRE) * Np + (size_t)Nfp * npl * NPVS + (size_t)NS * Np + (size_t)A.pf * NS * Np
          : (size_t)(NS + naux + NPRE) * Np + (size_t)2 * DIM * Nfp * NS + (size_t)Nfp * npl * NPVS +
                (FUSE ? (size_t)NS * Np + (size_t)2 * Nfp * NS : 0) + (size_t)A.pf * NS * Np;
  double* sq = sm + tabn + slot * slotsz;
  double* sa = sq + NS * Np;
  double* sp = sa + naux_s * Np;
  // compact: the explicit face slots take the precomputed values' region
  double* ss = CMP ? sp : sp + NPRE * Np;
  double* spv = CMP ? sp + NPRE * Np : ss + 2 * DIM * Nfp * NS;  // pair values
  double* slf = spv + (size_t)Nfp * npl * NPVS;  // FUSE: linear vertical flux per node
  // FUSE: linear z-face slots (compact: in the pair buffer, after the parked
  // accumulators and the parked linear source)
  double* ssl = CMP ? spv + (size_t)(NS + DIM) * Np : slf + NS * Np;
  // prefetched epilogue inputs: the last A.pf*NS*Np doubles of the slot
  double* spf_in = sq + slotsz - (size_t)A.pf * NS * Np;
  int* spair = (int*)(sm + tabn + A.E * slotsz);
  for (int t = threadIdx.x; t < tabn; t += blockDim.x) sm[t] = A.tab[t];
  if (PAIRS && threadIdx.x < npl) {
    int p = threadIdx.x, a = 0;
    while (p >= Nq - 1 - a) { p -= Nq - 1 - a; ++a; }
    spair[threadIdx.x] = a | ((a + 1 + p) << 8);
  }
  const LawP& L = A.law;
  // everything above reads launch constants only; the state, aux and
  // accumulators below may come from the previous kernel of the stream
  pdl_wait();
  auto tile_body = [&](const int tile) {
  const int e = tile * A.E + slot;
  const bool act = (slot < A.E) && (e < A.K);
  const size_t gid = (size_t)e * Np + node;
  // Fused ARK stages: the epilogue's own-node inputs (the accumulators) are
  // copied into shared memory now, asynchronously, so their latency hides
  // behind the whole tendency; each thread later reads only what it copied.
  // (Plain kernels keep reading them at the end: the extra code costs them
  // registers, measured slower.)
  if (FUSE && A.pf > 0 && act) {
    int j = 0;
    auto pf5 = [&](const double* p0, const double* p1, const double* p2, const double* p3, const double* p4) {
      const double* P[5] = {p0, p1, p2, p3, p4};
#pragma unroll
      for (int s = 0; s < NS; ++s) tend_cp_async8(spf_in + (j * NS + s) * Np + node, P[s] + gid);
      ++j;
    };
    switch (epi) {
      case EPI_ADD: pf5(A.out[0], A.out[1], A.out[2], A.out[3], A.out[4]); break;
      case EPI_LSRK:
        if (A.a != 0.0) pf5(A.out[0], A.out[1], A.out[2], A.out[3], A.out[4]);
        break;
      case EPI_ARK:
        if (!FUSE) pf5(A.out[0], A.out[1], A.out[2], A.out[3], A.out[4]);
#pragma unroll
        for (int k = 0; k < 3; ++k)
          if (A.acc[k][0] && A.accin[k][0])
            pf5(A.accin[k][0], A.accin[k][1], A.accin[k][2], A.accin[k][3], A.accin[k][4]);
        break;
      case EPI_SUBOUT2:
      case EPI_RLSRK: pf5(A.out2[0], A.out2[1], A.out2[2], A.out2[3], A.out2[4]); break;
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
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
        if constexpr (CMP) {
          if (k == 0) sa[node] = an[k];
          if (k == DIM + 1) sa[Np + node] = an[k];
          if (k == DIM + 2) sa[2 * Np + node] = an[k];
        } else {
          sa[k * Np + node] = an[k];
        }
      }
    if constexpr (VK == VK_EC && LAW == LAW_SW) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) Pn[c] = qn[1 + c] / qn[0];
      Pn[DIM] = qn[DIM + 1] / qn[0];
    } else if constexpr (VK == VK_EC) {
      // one reciprocal of rho and one of p/rho per node
      const double rho = qn[0], rinv = 1.0 / rho;
#pragma unroll
      for (int c = 0; c < DIM; ++c) Pn[c] = qn[1 + c] * rinv;
      const double Phi = (LAW == LAW_EG) ? an[0] : 0.0;
      const double p = (L.gamma - 1.0) * (qn[DIM + 1] - dot<DIM>(qn + 1, Pn) / 2.0 - rho * Phi);
      const double pr = p * rinv;
      Pn[DIM] = 0.5 / pr;  // b = rho / (2 p)
      Pn[DIM + 1] = dot<DIM>(Pn, Pn);
      Pn[DIM + 2] = pr;
    } else if constexpr (VK == VK_KG) {
      const double rho = qn[0];
#pragma unroll
      for (int c = 0; c < DIM; ++c) Pn[c] = qn[1 + c] / rho;
      Pn[DIM] = pressure_eg<DIM>(L.gamma, qn, (LAW == LAW_EG) ? an[0] : 0.0);
      Pn[DIM + 1] = qn[DIM + 1] / rho;
    } else if constexpr (VK == VK_KG32) {
      const double rho = qn[0], rinv = 1.0 / rho;
      Pn[0] = pressure_eg<DIM>(L.gamma, qn, (LAW == LAW_EG) ? an[0] : 0.0);
      float* spf = (float*)(sp + Np);
      const float rinvf = (float)rinv;
#pragma unroll
      for (int c = 0; c < DIM; ++c) spf[c * Np + node] = (float)qn[1 + c] * rinvf;
      spf[DIM * Np + node] = (float)qn[DIM + 1] * rinvf;
    } else if constexpr (VK == VK_EC32 && LAW == LAW_SW) {
      float* spf = (float*)sp;
      const float hinv = 1.f / (float)qn[0];
#pragma unroll
      for (int c = 0; c < DIM; ++c) spf[c * Np + node] = (float)qn[1 + c] * hinv;
      spf[DIM * Np + node] = (float)qn[DIM + 1] * hinv;
    } else if constexpr (VK == VK_EC32) {
      const double rho = qn[0], rinv = 1.0 / rho;
      const double Phi = (LAW == LAW_EG) ? an[0] : 0.0;
      const double ke = 0.5 * dot<DIM>(qn + 1, qn + 1) * rinv;
      const double p = (L.gamma - 1.0) * (qn[DIM + 1] - ke - rho * Phi);
      const double pr = p * rinv;
      Pn[0] = p;
      Pn[1] = 0.5 / pr;
      Pn[2] = pr;
      float* spf = (float*)(sp + 3 * Np);
      const float rinvf = (float)rinv;
      float uu = 0.f;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const float u = (float)qn[1 + c] * rinvf;
        spf[c * Np + node] = u;
        uu += u * u;
      }
      spf[DIM * Np + node] = uu;
    }
    if constexpr (VK == VK_KG32) {
      sp[node] = Pn[0];
    } else if constexpr (VK == VK_EC32 && LAW != LAW_SW) {
#pragma unroll
      for (int k = 0; k < 3; ++k) sp[k * Np + node] = Pn[k];
    } else if constexpr (VK == VK_EC32) {
    } else if constexpr (PAIRS) {
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
  if constexpr (FUSE && LAW == LAW_EG) {
    // fused linear operator: its z flux rows, staged with the state (no
    // barrier of its own)
    if (act) {
      double f[NS];
      flux_dir<LAW_LEG, DIM>(A.lin_law, DIM - 1, qn, an, f);
#pragma unroll
      for (int s = 0; s < NS; ++s) slf[s * Np + node] = f[s];
    }
  }
  __syncthreads();

  double T[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) T[s] = 0.0;
  const double igm1 = 1.0 / (L.gamma - 1.0);
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
        // rolled: the instruction stream stays small (unrolling by two
        // interleaves the flux chains of a thread's pairs, but the larger
        // kernel body stalls on instruction fetch; measured 5% slower for
        // the fused ARK stage kernel on B200)
#pragma unroll 1
        for (int t = node; t < Nfp * npl; t += Np) {
          const int line = t / npl, p = t - line * npl;
          const int lb = (d == 0) ? line * Nq : (d == 1) ? (line % Nq) + Nq * Nq * (line / Nq) : line;
          const int ab = spair[p];
          const int na = lb + (ab & 0xff) * sd, nb = lb + (ab >> 8) * sd;
          double f[NS + 1];
          if constexpr (VK == VK_KG32) {
            const float* spf = (const float*)(sp + Np);
            float u1[DIM], u2[DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c) { u1[c] = spf[c * Np + na]; u2[c] = spf[c * Np + nb]; }
            kg_vol32<DIM>(d, sq[na], sp[na], u1, spf[DIM * Np + na], sq[nb], sp[nb], u2, spf[DIM * Np + nb], f);
            double* dst = spv + (size_t)t * NPVS;
#pragma unroll
            for (int s = 0; s < NPV; ++s) dst[s] = f[s];
            continue;
          }
          if constexpr (VK == VK_EC32) {
            if constexpr (LAW == LAW_SW) {
              const float* spf = (const float*)sp;
              float P1[DIM + 1], P2[DIM + 1];
              double q1[NS], q2[NS];
#pragma unroll
              for (int k = 0; k < DIM + 1; ++k) { P1[k] = spf[k * Np + na]; P2[k] = spf[k * Np + nb]; }
#pragma unroll
              for (int s = 0; s < NS; ++s) { q1[s] = sq[s * Np + na]; q2[s] = sq[s * Np + nb]; }
              sw_vol32<DIM>(L.grav, d, q1, P1, q2, P2, f);
            } else {
              const float* spf = (const float*)(sp + 3 * Np);
              float u1[DIM], u2[DIM];
#pragma unroll
              for (int c = 0; c < DIM; ++c) { u1[c] = spf[c * Np + na]; u2[c] = spf[c * Np + nb]; }
              const double Phi1 = (LAW == LAW_EG) ? sa[na] : 0.0, Phi2 = (LAW == LAW_EG) ? sa[nb] : 0.0;
              ec_vol32<LAW, DIM>((float)igm1, d, sq[na], sp[na], sp[Np + na], u1, spf[DIM * Np + na], Phi1, sq[nb],
                                 sp[nb], sp[Np + nb], u2, spf[DIM * Np + nb], Phi2, f, f + NS);
            }
            double* dst = spv + (size_t)t * NPVS;
#pragma unroll
            for (int s = 0; s < NPV; ++s) dst[s] = f[s];
            continue;
          }
          double P1[NPRE], P2[NPRE];
#pragma unroll
          for (int k = 0; k < NPRE; ++k) { P1[k] = sp[k * Np + na]; P2[k] = sp[k * Np + nb]; }
          if constexpr (LAW == LAW_SW) {
            double q1[NS], q2[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) { q1[s] = sq[s * Np + na]; q2[s] = sq[s * Np + nb]; }
            sw_ec_dir<DIM>(L.grav, 0, d, q1, P1, 0.0, q2, P2, 0.0, f);
          } else if constexpr (VK == VK_EC) {
            const double Phi1 = (LAW == LAW_EG) ? sa[na] : 0.0, Phi2 = (LAW == LAW_EG) ? sa[nb] : 0.0;
            ec_vol<LAW, DIM>(L.gamma, igm1, d, sq[na], P1, Phi1, sq[nb], P2, Phi2, f, f + NS);
          } else {
            kg_vol<DIM>(d, sq[na], P1, sq[nb], P2, f);
          }
          double* dst = spv + (size_t)t * NPVS;
#pragma unroll
          for (int s = 0; s < NPV; ++s) dst[s] = f[s];
        }
      }
      __syncthreads();
      // ---- phase B: every node contracts its row, adding its own fluctuation
      if (act) {
        const int line = (d == 0) ? node / Nq : (d == 1) ? ijk[0] + Nq * ijk[2] : node % (Nq * Nq);
        const double* lp = spv + (size_t)line * npl * NPVS;
        // the Nq - 1 partners m != id, without a skipped (divergent) iteration
#pragma unroll
        for (int k = 0; k < (CQ ? NQ_ - 1 : 7); ++k) {
          if (!CQ && k >= Nq - 1) break;
          const int m = k + (k >= id ? 1 : 0);
          const int p = (m < id) ? pair_index(m, id, Nq) : pair_index(id, m, Nq);
          const double* fv = lp + p * NPVS;
          double f[NS];
#pragma unroll
          for (int s = 0; s < NS; ++s) f[s] = fv[s];
          const int nn = base + m * sd;
          if constexpr (LAW == LAW_EG) {
            const double dPhi = an[0] - sa[nn];
            if constexpr (VK == VK_EC || VK == VK_EC32)
              f[1 + d] = f[1 + d] - fv[NS] * Pn[PR_IDX] * dPhi;  // alpha = b_avg rho_log / (2 b_own)
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
#pragma unroll
      for (int m = 0; m < (CQ ? NQ_ : 8); ++m) {
        if (!CQ && m >= Nq) break;
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

  constexpr int DZ = DIM - 1;
  // While the face tasks run (the register-heaviest part), the explicit
  // accumulators wait in the pair buffer (free after the last direction) and
  // the own-node state and aux are re-read from their staged copies
  // afterwards: nothing of this node's stays live in registers across them.
  constexpr bool PARK = PAIRS && CQ && ((size_t)ipow(NQ_ > 0 ? NQ_ : 1, DIM - 1) * ((NQ_ * (NQ_ - 1)) / 2) * NPVS >=
                                        (size_t)NS * ipow(NQ_ > 0 ? NQ_ : 1, DIM));
  if constexpr (PARK) {
    if (act) {
#pragma unroll
      for (int s = 0; s < NS; ++s) spv[s * Np + node] = T[s];
    }
  }
  // compact layout: the linear operator's source (it reads grad Phi, which is
  // not staged) is evaluated now, from registers, exactly as the linear
  // operator begins -- TL = 0, then its sources -- and parked with T; it only
  // touches the momentum components
  if constexpr (CMP) {
    if (act && ((A.lin_dirs >> (DIM - 1)) & 1)) {
      double tl[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) tl[s] = 0.0;
      add_sources<LAW_LEG, DIM>(A.lin_law, true, qn, an, tl);
#pragma unroll
      for (int k = 0; k < DIM; ++k) spv[(NS + k) * Np + node] = tl[1 + k];
    }
  }

  // ------------------------------------------------------------ faces
  // Face-node tasks of all elements of the CTA, spread over all its threads.
  // Where it costs little padding, each direction's 2*Nfp tasks are padded to
  // whole warps, so a warp only runs faces of one direction (the flux code is
  // not split between directions inside a warp); the direction is dispatched
  // to a compile-time constant so every state / normal index in the numerical
  // flux is static.
  {
    const double lift_end = sm[2 * Nq * Nq];
    const bool lin_faces = FUSE && LAW == LAW_EG && ((A.lin_dirs >> DZ) & 1);
    const int naux_nl = FUSE ? A.naux_nl : naux;
    // warp-aligned groups when that costs little padding (3-D N=3, 4, 7),
    // else dense (small faces would leave most lanes idle)
    const int fpad = ((2 * Nfp + 31) / 32) * 32;
    const int fp = (10 * fpad <= 13 * 2 * Nfp) ? fpad : 2 * Nfp;
    const int per_elem = (DIM + (lin_faces ? 1 : 0)) * fp;
    for (int v = threadIdx.x; v < A.E * per_elem; v += blockDim.x) {
      const int es = v / per_elem, r = v - es * per_elem;
      const int dd = r / fp, tt = r - dd * fp;
      const int ef = tile * A.E + es;
      if (tt >= 2 * Nfp || ef >= A.K) continue;
      double* const sqe = sm + tabn + es * slotsz;
      double* const sae = sqe + NS * Np;
      double* const spe = sae + naux_s * Np;
      double* const sse = CMP ? spe : spe + NPRE * Np;
      if constexpr (FUSE && LAW == LAW_EG) {
        if (dd == DIM) {
          // z faces of the linear operator (face numbers 2*DZ, 2*DZ + 1): the
          // slot pointer is shifted so those faces land in the linear slots
          double* const ssle = CMP ? spe + NPRE * Np + (size_t)(NS + DIM) * Np
                                   : sse + 2 * DIM * Nfp * NS + (size_t)Nfp * npl * NPVS + NS * Np;
          face_task<LAW_LEG, DIM, NAuxMax<LAW_LEG, DIM>::v, DZ, false, CMP>(
              A, A.lin_law, lin_sflux, naux, Nq, Np, Nfp, ef, 2 * DZ * Nfp + tt, sqe, sae,
              ssle - (size_t)2 * DZ * Nfp * NS, __ldg(A.ginv + 3 * ef + DZ), lift_end);
          continue;
        }
      }
      const int t = 2 * dd * Nfp + tt;
      switch (dd) {
        case 0: face_task<LAW, DIM, NAM, 0, F32S, CMP>(A, L, sflux, naux_nl, Nq, Np, Nfp, ef, t, sqe, sae, sse, __ldg(A.ginv + 3 * ef), lift_end); break;
        case 1: if constexpr (DIM > 1) face_task<LAW, DIM, NAM, 1, F32S, CMP>(A, L, sflux, naux_nl, Nq, Np, Nfp, ef, t, sqe, sae, sse, __ldg(A.ginv + 3 * ef + 1), lift_end); break;
        default: if constexpr (DIM > 2) face_task<LAW, DIM, NAM, 2, F32S, CMP>(A, L, sflux, naux_nl, Nq, Np, Nfp, ef, t, sqe, sae, sse, __ldg(A.ginv + 3 * ef + 2), lift_end); break;
      }
    }
  }
  __syncthreads();
  if (!act) return;
  if constexpr (PARK) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      T[s] = spv[s * Np + node];
      qn[s] = sq[s * Np + node];
    }
    // (compact layout: nothing after this point reads the aux fields)
    if constexpr (!CMP) {
#pragma unroll
      for (int k = 0; k < NAM; ++k)
        if (k < naux) an[k] = sa[k * Np + node];
    }
  }
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
  // fused linear operator: the weak-form linear Euler-gravity operator along
  // z, evaluated exactly as its own launch would: sources, then the D^T
  // contraction of the staged flux rows, then the z faces
  double TL[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) TL[s] = 0.0;
  if constexpr (FUSE && LAW == LAW_EG) {
    if ((A.lin_dirs >> DZ) & 1) {
      if constexpr (CMP) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) TL[1 + k] = spv[(NS + k) * Np + node];
      } else {
        add_sources<LAW_LEG, DIM>(A.lin_law, true, qn, an, TL);
      }
      const int sd = (DZ == 0) ? 1 : (DZ == 1) ? Nq : Nq * Nq;
      const int id = ijk[DZ];
      const int base = node - id * sd;
      const double gz = __ldg(A.ginv + 3 * e + DZ);
#pragma unroll
      for (int m = 0; m < (CQ ? NQ_ : 8); ++m) {
        if (!CQ && m >= Nq) break;
        const int nn = base + m * sd;
        const double c = sW[id * Nq + m] * gz;
#pragma unroll
        for (int s = 0; s < NS; ++s) TL[s] = TL[s] + c * slf[s * Np + nn];
      }
    }
    const int id = ijk[DZ];
    if (((A.lin_dirs >> DZ) & 1) && (id == 0 || id == Nq - 1)) {
      const int side = (id == Nq - 1) ? 1 : 0;
      const int j = (DZ == 0) ? ijk[1] + Nq * ijk[2] : (DZ == 1) ? ijk[0] + Nq * ijk[2] : ijk[0] + Nq * ijk[1];
#pragma unroll
      for (int s = 0; s < NS; ++s) TL[s] = TL[s] - ssl[(side * Nfp + j) * NS + s];
    }
  }

  // --------------------------------------------------------- epilogue
  const bool pfon = FUSE && A.pf > 0;
  if (pfon) asm volatile("cp.async.wait_all;\n" ::: "memory");
  // j-th prefetched field, state s (own node); the same order as issued
  auto pin = [&](int j, int s) { return spf_in[(j * NS + s) * Np + node]; };
  switch (epi) {
    case EPI_SET:
#pragma unroll
      for (int s = 0; s < NS; ++s) A.out[s][gid] = T[s];
      break;
    case EPI_ADD:
#pragma unroll
      for (int s = 0; s < NS; ++s) A.out[s][gid] = (pfon ? pin(0, s) : A.out[s][gid]) + T[s];
      break;
    case EPI_LSRK: {
      const double bdt = A.dte ? A.bdt * A.dte[e] : A.bdt;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        // first stage (a = 0): the previous increment is not read, so stale
        // or never-written increment storage cannot leak into the step
        const double dqn = (A.a != 0.0) ? A.a * (pfon ? pin(0, s) : A.out[s][gid]) + T[s] : T[s];
        A.out[s][gid] = dqn;
        A.out2[s][gid] = qn[s] + bdt * dqn;
      }
    } break;
    case EPI_ARK:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        // fused: T = N(Q), TL = L(Q); else out holds N(Q) and T = L(Q)
        const double E = FUSE ? T[s] - TL[s] : (pfon ? pin(0, s) : A.out[s][gid]) - T[s];
        const double I = FUSE ? TL[s] : T[s];
        int jj = FUSE ? 0 : 1;
#pragma unroll
        for (int j = 0; j < 3; ++j)
          if (A.acc[j][0]) {
            double base = qn[s];
            if (A.accin[j][0]) base = pfon ? pin(jj++, s) : A.accin[j][s][gid];
            A.acc[j][s][gid] = base + A.adt * (A.ca[j] * E + A.cb[j] * I);
          }
      }
      break;
    case EPI_SUBOUT2:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double o2 = pfon ? pin(0, s) : A.out2[s][gid];
        A.out[s][gid] = T[s];
        A.out2[s][gid] = o2 - T[s];
      }
      break;
    case EPI_RLSRK:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double o2 = pfon ? pin(0, s) : A.out2[s][gid];
        A.out[s][gid] = T[s];
        A.out2[s][gid] = A.a * o2 + T[s];
      }
      break;
  }
  };  // tile_body
  if constexpr (PERSIST) {
    const int ntiles = (A.K + A.E - 1) / A.E;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      tile_body(tile);
      __syncthreads();  // the next tile restages shared memory
    }
  } else {
    tile_body(blockIdx.x);
  }
  pdl_trigger();
}

// launcher signature used by the host dispatch table
typedef void (*tend_launch_fn)(const TendArgs& A, int grid, int block, size_t smem, cudaStream_t st);

template <int LAW, int DIM, int VK, int NQ_ = 0, bool FUSE = false, int SF = -1, bool PERSIST = false>
void tend_launch(const TendArgs& A, int grid, int block, size_t smem, cudaStream_t st) {
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    // on failure the launch below reports the error
    if (cudaFuncSetAttribute(tendency_kernel<LAW, DIM, VK, NQ_, FUSE, SF, PERSIST>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess)
      configured = smem;
  }
  launch_maybe_pdl(tendency_kernel<LAW, DIM, VK, NQ_, FUSE, SF, PERSIST>, dim3(grid), dim3(block), smem, st, A);
}

// persistent variants (atb_op_set_persistent) of the hot configurations: the
// explicit Rusanov kernels of 3-D Euler-gravity, 2-D Euler and 2-D shallow
// water (FP64 and FP32 flux) and the fused Euler-gravity ARK23 stage, for
// the orders N = 3..5; nullptr when there is none
tend_launch_fn pick_launcher_persistent(int law, int dim, int vk, int nq, int sflux, bool fused, int lin_sflux);

// Euler-gravity explicit tendency fused with the weak-form linear operator
// along z (ARK23 stages, split_rhs = false): 3-D, EC / FP32-flux EC volume
// flux; nullptr when there is no such kernel
// sflux / lin_sflux: the surface fluxes of the two operators (a kernel with
// the flux kind built in when both are Rusanov)
tend_launch_fn pick_launcher_fused(int dim, int vk, int nq, int sflux, int lin_sflux);

// generic (runtime Nq) launcher, and the compile-time-Nq specialisations
// that exist for (law, dim, vk, nq) -- nullptr when there is none
// the compile-time-Nq kernels with the Rusanov surface flux built in (hot
// explicit configurations), nullptr when there is none
tend_launch_fn pick_launcher_rusanov(int law, int dim, int vk, int nq);
template <int LAW> tend_launch_fn pick_launcher(int dim, int vk);
template <int LAW> tend_launch_fn pick_launcher_nq(int dim, int vk, int nq);

// per-node precomputed values and per-pair stored values, for the host
inline int npre_of(int law, int dim, int vk) {
  int ns = (law == LAW_ADV) ? 1 : dim + 2;
  if (vk == VK_EC32) return (law == LAW_SW) ? (dim + 2) / 2 : 3 + (dim + 2) / 2;
  if (vk == VK_KG32) return 1 + (dim + 2) / 2;
  if (vk == VK_EC) return (law == LAW_SW) ? dim + 1 : dim + 3;
  if (vk == VK_KG) return dim + 2;
  return dim * ns;
}
inline int npv_stride_of(int law, int dim, int vk) {
  int ns = (law == LAW_ADV) ? 1 : dim + 2;
  if (vk == VK_EC || vk == VK_KG || vk == VK_EC32 || vk == VK_KG32)
    return (ns + ((law == LAW_EG && (vk == VK_EC || vk == VK_EC32)) ? 1 : 0)) | 1;
  return 0;
}

}  // namespace atb
