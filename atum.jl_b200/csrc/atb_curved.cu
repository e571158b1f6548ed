// DGSEM tendency on curved hexahedra (cubed-sphere shells): per-node metric
// terms, per-face-node normals and face masses, neighbour traces through a
// node-level face map.
//
// Restates, for one stage, src/dgsem.jl:217-306 (volumeterm!, weak form),
// 470-561 (esvolumeterm_dir!, flux differencing: l_g = MJ g[dir, :] of both
// nodes of every pair, all three rows of the two-point flux contracted with
// them) and 683-732 (surfaceterm! with facenormal / faceMJ / faceix of a curved
// grid), with the same epilogues as the brick kernels (atb_tendency.cuh).
//
// Mapping: one thread per LGL node, E elements per CTA.  The element's state
// and aux, the per-node values the volume term reads of other nodes (weak
// form: the contravariant flux rows MJ g[dir, :] . F; flux differencing: the
// entropy-conservative / Kennedy-Gruber point values and MJ g) are staged in
// shared memory.  Face tasks evaluate the numerical flux once per face node,
// gather the neighbour trace from global memory and leave faceMJ * flux in a
// shared slot; every node then subtracts the slots of its faces in face order.
// Brick grids keep the specialised kernels (diagonal metrics, one flux row).
#include "atb_curved.cuh"

namespace atb {

namespace {

constexpr int CNS = 5;  // 3-D Euler / Euler-gravity / linear Euler-gravity states

// physical flux rows F[d][s], d = 0..2 (src/balancelaws/*.jl flux)
template <int LAW>
__device__ __forceinline__ void flux_rows(const LawP& L, const double* q, const double* aux, double (*F)[CNS]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) flux_dir<LAW, 3>(L, d, q, aux, F[d]);
}

// wavespeed(law, n, q, aux) for a general unit normal n
template <int LAW>
__device__ __forceinline__ double wavespeed_n(const LawP& L, const double* n, const double* q, const double* aux) {
  if constexpr (LAW == LAW_LEG) {
    return sqrt(L.gamma * aux[5] / aux[4]);  // sound speed of the reference state (aux: Phi, grad Phi, rho_ref, p_ref)
  } else {
    const double rho = q[0];
    double u[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = q[1 + c] / rho;
    const double p = pressure_eg<3>(L.gamma, q, LAW == LAW_EG ? aux[0] : 0.0);
    return fabs(dot<3>(n, u)) + sqrt(L.gamma * p / rho);
  }
}

// All three rows of the entropy-conservative two-point flux with the pair's
// averages, logarithmic means and reciprocal computed once (the same
// arithmetic as ec_sym_dir row by row, plus the Euler-gravity fluctuation
// -alpha (Phi1 - Phi2) with alpha = b_avg rho_log / (2 b1) on each row's own
// momentum entry).  P: u (3), p, b, |u|^2, e, p/rho.
template <int LAW>
__device__ __forceinline__ void ec_rows(double gamma, double r1, const double* P1, double Phi1, double r2,
                                        const double* P2, double Phi2, double (*F)[CNS]) {
  const double rho_avg = (r1 + r2) / 2.0;
  double ua[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) ua[c] = (P1[c] + P2[c]) / 2.0;
  const double b1 = P1[4], b2 = P2[4];
  const double b_avg = (b1 + b2) / 2.0;
  const double u2_avg = (P1[5] + P2[5]) / 2.0;
  const double rho_log = logavg_fast(r1, r2);
  const double b_log = logavg_fast(b1, b2);
  const double rinv = 1.0 / (b_avg * b_log);
  const double pc = rho_avg * b_log * rinv / 2.0;
  double c1 = b_avg * rinv / (2.0 * (gamma - 1.0)) - u2_avg / 2.0;
  if (LAW == LAW_EG) c1 = c1 + (Phi1 + Phi2) / 2.0;
  const double fl = (LAW == LAW_EG) ? (b_avg * rho_log / (2.0 * b1)) * (Phi1 - Phi2) : 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double ud = ua[d];
    const double frd = ud * rho_log;
    F[d][0] = frd;
    double mu = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double m = ud * (ua[c] * rho_log);
      if (c == d) m = m + pc;
      F[d][1 + c] = m;
      mu = (c == 0) ? m * ua[c] : mu + m * ua[c];
    }
    F[d][4] = c1 * frd + mu;
    if (LAW == LAW_EG) F[d][1 + d] = F[d][1 + d] - fl;
  }
}

// two-point volume flux rows (entropy conservative / Kennedy-Gruber /
// central) of the ordered pair (1 = own node, 2 = partner)
template <int LAW, int VK>
__device__ __forceinline__ void twopoint_rows(const LawP& L, const double* q1, const double* a1, const double* P1,
                                              const double* q2, const double* a2, const double* P2,
                                              double (*F)[CNS]) {
  if constexpr (VK == VK_EC) {
    const double Phi1 = (LAW == LAW_EG) ? a1[0] : 0.0, Phi2 = (LAW == LAW_EG) ? a2[0] : 0.0;
    ec_rows<LAW>(L.gamma, q1[0], P1, Phi1, q2[0], P2, Phi2, F);
  } else if constexpr (VK == VK_KG) {
    const double Phi1 = (LAW == LAW_EG) ? a1[0] : 0.0, Phi2 = (LAW == LAW_EG) ? a2[0] : 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) kg_dir<LAW, 3>(d, q1[0], P1, Phi1, q2[0], P2, Phi2, F[d]);
  } else {
    double G[3][CNS];
    flux_rows<LAW>(L, q1, a1, F);
    flux_rows<LAW>(L, q2, a2, G);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int s = 0; s < CNS; ++s) F[d][s] = (F[d][s] + G[d][s]) / 2.0;
  }
}

// The two-point flux of an ordered pair contracted with two direction
// vectors, f1 = sum_c l1_c F#[c][:] and f2 = sum_c l2_c F#[c][:], from one set
// of pair means.  For the entropy-conservative flux the contraction with l is
// (U = l . u_avg, f_rho = U rho_log):
//   [f_rho, f_rho u_avg + (p_c - fl) l, f_rho (c1 + |u_avg|^2) + p_c U]
// with p_c = rho_avg / (2 b_avg), c1 = 1/(2 (gamma-1) b_log) - |u|^2_avg / 2
// (+ Phi_avg), and fl = b_avg rho_log / (2 b1) (Phi1 - Phi2) the Euler-gravity
// fluctuation on the momentum; for Kennedy-Gruber
//   [U rho_avg, U rho_avg u_avg + (p_avg - rho_avg (Phi1 - Phi2) / 2) l,
//    U (rho_avg e_avg + p_avg)]
// -- the rows of ec_rows / kg_dir summed with the weights l, in fewer operations.
template <int LAW, int VK>
__device__ __forceinline__ void pair_contract(const LawP& L, const double* q1, const double* a1, const double* P1,
                                              const double* q2, const double* a2, const double* P2,
                                              const double* l1, const double* l2, double* f1, double* f2) {
  if constexpr (VK == VK_EC || VK == VK_KG) {
    const double r1 = q1[0], r2 = q2[0];
    const double Phi1 = (LAW == LAW_EG) ? a1[0] : 0.0, Phi2 = (LAW == LAW_EG) ? a2[0] : 0.0;
    const double rho_avg = (r1 + r2) / 2.0;
    double ua[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) ua[c] = (P1[c] + P2[c]) / 2.0;
    double rho_m, pc, c4;  // momentum / energy coefficients
    double fl = 0.0;
    if constexpr (VK == VK_EC) {
      const double b1 = P1[4], b2 = P2[4];
      const double b_avg = (b1 + b2) / 2.0;
      const double u2_avg = (P1[5] + P2[5]) / 2.0;
      // with both logarithmic means on their series branch (the common case
      // within an element) every division shares one reciprocal,
      // 1 / ((r1+r2)^2 (b1+b2)^2): rho_log = rho_avg G(u_rho),
      // rho_avg / (2 b_avg) = rho_avg / (b1+b2), 1 / (2 (gamma-1) b_log) =
      // F(u_b) / ((gamma-1) (b1+b2)) -- as the brick kernels' ec_vol
      const double rs = r1 + r2, rd = r1 - r2, bs = b1 + b2, bd = b1 - b2;
      const double rs2 = rs * rs, bs2 = bs * bs, rd2 = rd * rd, bd2 = bd * bd;
      double cterm;
      if (rd2 < 1e-2 * rs2 && bd2 < 1e-2 * bs2) {
        const double inv = 1.0 / (rs2 * bs2);
        const double ur = rd2 * bs2 * inv, ub = bd2 * rs2 * inv;
        const double inv_bs = bs * rs2 * inv;
        rho_m = rho_avg * series_G(ur);
        pc = rho_avg * inv_bs;
        cterm = series_F(ub) * inv_bs / (L.gamma - 1.0);
      } else {
        rho_m = logavg_fast(r1, r2);
        const double b_log = logavg_fast(b1, b2);
        const double rinv = 1.0 / (b_avg * b_log);
        pc = rho_avg * b_log * rinv / 2.0;
        cterm = b_avg * rinv / (2.0 * (L.gamma - 1.0));
      }
      double c1 = cterm - u2_avg / 2.0;
      if (LAW == LAW_EG) {
        c1 = c1 + (Phi1 + Phi2) / 2.0;
        // alpha = b_avg rho_log / (2 b1), with 1 / (2 b1) = p1 / rho1 from the
        // node's point values
        fl = (b_avg * rho_m * P1[7]) * (Phi1 - Phi2);
      }
      c4 = c1 + dot<3>(ua, ua);
    } else {
      rho_m = rho_avg;
      pc = (P1[3] + P2[3]) / 2.0;  // p_avg
      c4 = rho_avg * ((P1[6] + P2[6]) / 2.0) + pc;  // rho_avg e_avg + p_avg
      if (LAW == LAW_EG) fl = (rho_avg / 2.0) * (Phi1 - Phi2);
    }
    const double pm = pc - fl;
    const double U1 = dot<3>(l1, ua), U2 = dot<3>(l2, ua);
    const double fr1 = U1 * rho_m, fr2 = U2 * rho_m;
    f1[0] = fr1;
    f2[0] = fr2;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      f1[1 + k] = fr1 * ua[k] + pm * l1[k];
      f2[1 + k] = fr2 * ua[k] + pm * l2[k];
    }
    if constexpr (VK == VK_EC) {
      f1[4] = fr1 * c4 + pc * U1;
      f2[4] = fr2 * c4 + pc * U2;
    } else {
      f1[4] = U1 * c4;
      f2[4] = U2 * c4;
    }
  } else {
    double F[3][CNS];
    twopoint_rows<LAW, VK>(L, q1, a1, P1, q2, a2, P2, F);
#pragma unroll
    for (int s = 0; s < CNS; ++s) {
      f1[s] = l1[0] * F[0][s] + l1[1] * F[1][s] + l1[2] * F[2][s];
      f2[s] = l2[0] * F[0][s] + l2[1] * F[1][s] + l2[2] * F[2][s];
    }
  }
}

// boundarystate(law, problem, n, q-, aux-, tag) for a general normal
__device__ __forceinline__ void boundary_state_n(const LawP& L, const double* n, int tag, const double* qm,
                                                 double* qp) {
  if (L.bc == BC_REFLECT) {
    // rhou+ = rhou- - 2 (n . rhou-) n (experiment/euler_gravity/acousticwave.jl:17-22)
    const double nm = dot<3>(n, qm + 1);
    qp[0] = qm[0];
#pragma unroll
    for (int k = 0; k < 3; ++k) qp[1 + k] = qm[1 + k] - 2.0 * nm * n[k];
    qp[4] = qm[4];
  } else if (L.bc == BC_DIRICHLET) {
    const double* st = L.bc_state[tag == 1 ? 0 : 1];
#pragma unroll
    for (int s = 0; s < CNS; ++s) qp[s] = st[s];
  } else {
#pragma unroll
    for (int s = 0; s < CNS; ++s) qp[s] = qm[s];
  }
}

// Roe flux for a general unit normal (src/balancelaws/euler.jl:91-138,
// euler_gravity.jl:149-198): the average of the two sides' normal fluxes minus
// the Roe-averaged characteristic dissipation
template <int LAW>
__device__ __forceinline__ void roe_n(const LawP& L, const double* n, const double* qm, const double* am,
                                      const double* qp, const double* ap, double* nf) {
  const double g = L.gamma;
  const double Phi = (LAW == LAW_EG) ? am[0] : 0.0;
  double Fm[3][CNS], Fp[3][CNS];
  flux_rows<LAW>(L, qm, am, Fm);
  flux_rows<LAW>(L, qp, ap, Fp);
  const double rm = qm[0], rp = qp[0];
  double um[3], up[3], u[3], du[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) { um[c] = qm[1 + c] / rm; up[c] = qp[1 + c] / rp; }
  const double pm = pressure_eg<3>(g, qm, Phi), pp = pressure_eg<3>(g, qp, Phi);
  const double hm = qm[4] / rm + pm / rm, hp = qp[4] / rp + pp / rp;
  const double cm = sqrt(g * pm / rm), cp = sqrt(g * pp / rp);
  const double srm = sqrt(rm), srp = sqrt(rp);
  const double rho = sqrt(rm * rp);
#pragma unroll
  for (int c = 0; c < 3; ++c) { u[c] = roe_avg(srm, srp, um[c], up[c]); du[c] = up[c] - um[c]; }
  const double h = roe_avg(srm, srp, hm, hp);
  const double c = roe_avg(srm, srp, cm, cp);
  const double un = dot<3>(u, n);
  const double drho = rp - rm, dp = pp - pm;
  const double dun = dot<3>(du, n);
  const double cm2 = 1.0 / (c * c);
  const double w1 = fabs(un - c) * (dp - rho * c * dun) * cm2 / 2.0;
  const double w2 = fabs(un + c) * (dp + rho * c * dun) * cm2 / 2.0;
  const double w3 = fabs(un) * (drho - dp * cm2);
  const double w4 = fabs(un) * rho;
  double fpv[CNS];
  fpv[0] = (w1 + w2 + w3) / 2.0;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    fpv[1 + k] = (w1 * (u[k] - c * n[k]) + w2 * (u[k] + c * n[k]) + w3 * u[k] + w4 * (du[k] - dun * n[k])) / 2.0;
  const double ke = (LAW == LAW_EG) ? w3 * (dot<3>(u, u) / 2.0 + Phi) : w3 * dot<3>(u, u) / 2.0;
  fpv[4] = (w1 * (h - c * un) + w2 * (h + c * un) + ke + w4 * (dot<3>(u, du) - un * dun)) / 2.0;
#pragma unroll
  for (int s = 0; s < CNS; ++s) {
    double fn = (Fm[0][s] + Fp[0][s]) * n[0];
    fn = fn + (Fm[1][s] + Fp[1][s]) * n[1];
    fn = fn + (Fm[2][s] + Fp[2][s]) * n[2];
    nf[s] = fn / 2.0 - fpv[s];
  }
}

// matrix-dissipation flux for a general unit normal (src/balancelaws/euler.jl:
// 198-256, euler_gravity.jl:271-332): the entropy-conservative flux . n minus
// half the entropy-variable jump scaled by the eigen-decomposition of the
// averaged state
template <int LAW>
__device__ __forceinline__ void matrix_n(const LawP& L, const double* n, const double* qm, const double* am,
                                         const double* qp, const double* ap, double* nf) {
  const double g = L.gamma;
  const double Phim = (LAW == LAW_EG) ? am[0] : 0.0, Phip = (LAW == LAW_EG) ? ap[0] : 0.0;
  double Pm[NPreE<3>::v], Pp[NPreE<3>::v];
  precompute_euler<3>(g, qm, Phim, Pm);
  precompute_euler<3>(g, qp, Phip, Pp);
  double ec[CNS];
  {
    double F[3][CNS];
#pragma unroll
    for (int d = 0; d < 3; ++d) ec_dir<LAW, 3>(g, d, qm[0], Pm, Phim, qp[0], Pp, Phip, F[d]);
#pragma unroll
    for (int s = 0; s < CNS; ++s) {
      double fn = F[0][s] * n[0];
      fn = fn + F[1][s] * n[1];
      ec[s] = fn + F[2][s] * n[2];
    }
  }
  const double rm = qm[0], rp = qp[0];
  const double bm = Pm[4], bp = Pp[4];
  const double Phi_avg = (Phim + Phip) / 2.0;
  const double rho_log = logavg(rm, rp);
  const double b_log = logavg(bm, bp);
  double ua[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) ua[c] = (Pm[c] + Pp[c]) / 2.0;
  const double p_avg = ((rm + rp) / 2.0) / (2.0 * ((bm + bp) / 2.0));
  // the norms of the velocities (not their squares), as the reference has it
  const double u2_bar = 2.0 * sqrt(dot<3>(ua, ua)) - (sqrt(Pm[5]) + sqrt(Pp[5])) / 2.0;
  double h_bar = g / (2.0 * b_log * (g - 1.0)) + u2_bar / 2.0;
  if (LAW == LAW_EG) h_bar = h_bar + Phi_avg;
  const double c_bar = sqrt(g * p_avg / rho_log);
  double umc[3], upc[3], ut[3];
  const double un = dot<3>(ua, n);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    umc[k] = ua[k] - c_bar * n[k];
    upc[k] = ua[k] + c_bar * n[k];
    ut[k] = ua[k] - un * n[k];
  }
  double vm[CNS], vp[CNS], dv[CNS];
  entropyvars<LAW, 3>(L, qm, am, vm);
  entropyvars<LAW, 3>(L, qp, ap, vp);
#pragma unroll
  for (int s = 0; s < CNS; ++s) dv[s] = vp[s] - vm[s];
  const double l1 = fabs(un - c_bar) * rho_log / (2.0 * g);
  const double l2 = fabs(un) * rho_log * (g - 1.0) / g;
  const double l3 = fabs(un + c_bar) * rho_log / (2.0 * g);
  const double l4 = fabs(un) * p_avg;
  double k2 = u2_bar / 2.0;
  if (LAW == LAW_EG) k2 = k2 + Phi_avg;
  const double w1 = l1 * (dv[0] + dot<3>(umc, dv + 1) + (h_bar - c_bar * un) * dv[4]);
  const double w2 = l2 * (dv[0] + dot<3>(ua, dv + 1) + k2 * dv[4]);
  const double w3 = l3 * (dv[0] + dot<3>(upc, dv + 1) + (h_bar + c_bar * un) * dv[4]);
  const double ndv = dot<3>(n, dv + 1);
  double Dm[CNS];
  Dm[0] = w1 + w2 + w3;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    Dm[1 + k] = w1 * umc[k] + w2 * ua[k] + w3 * upc[k] + l4 * (dv[1 + k] - ndv * n[k] + dv[4] * ut[k]);
  Dm[4] = w1 * (h_bar - c_bar * un) + w2 * k2 + w3 * (h_bar + c_bar * un) +
          l4 * (dot<3>(ut, dv + 1) + dv[4] * (dot<3>(ua, ua) - un * un));
#pragma unroll
  for (int s = 0; s < CNS; ++s) nf[s] = ec[s] - Dm[s] / 2.0;
}

// numerical flux . n (src/numericalfluxes.jl:31-42 and the two-point fluxes
// used as surface fluxes), general unit normal
template <int LAW>
__device__ __forceinline__ void surface_flux_n(const LawP& L, int kind, const double* n, const double* qm,
                                               const double* am, const double* qp, const double* ap, double* nf) {
  if constexpr (LAW != LAW_LEG) {
    if (kind == F_ROE) {
      roe_n<LAW>(L, n, qm, am, qp, ap, nf);
      return;
    }
    if (kind == F_MATRIX) {
      matrix_n<LAW>(L, n, qm, am, qp, ap, nf);
      return;
    }
  }
  double F[3][CNS];
  if (LAW != LAW_LEG && (kind == F_EC || kind == F_KG)) {
    double Pm[NPreE<3>::v], Pp[NPreE<3>::v];
    precompute_euler<3>(L.gamma, qm, LAW == LAW_EG ? am[0] : 0.0, Pm);
    precompute_euler<3>(L.gamma, qp, LAW == LAW_EG ? ap[0] : 0.0, Pp);
    if (kind == F_EC)
      twopoint_rows<LAW, VK_EC>(L, qm, am, Pm, qp, ap, Pp, F);
    else
      twopoint_rows<LAW, VK_KG>(L, qm, am, Pm, qp, ap, Pp, F);
  } else {
    twopoint_rows<LAW, VK_CENTRAL>(L, qm, am, nullptr, qp, ap, nullptr, F);
  }
  double ws = 0.0;
  if (kind == F_RUSANOV) ws = dmax(wavespeed_n<LAW>(L, n, qm, am), wavespeed_n<LAW>(L, n, qp, ap));
#pragma unroll
  for (int s = 0; s < CNS; ++s) {
    double fn = F[0][s] * n[0];
    fn = fn + F[1][s] * n[1];
    fn = fn + F[2][s] * n[2];
    nf[s] = (kind == F_RUSANOV) ? fn - ws * (qp[s] - qm[s]) / 2.0 : fn;
  }
}

// per-node values staged for other nodes of the element: flux differencing
// stages the two-point flux's point values (NPreE) and MJ g (9); the weak
// form stages the contravariant flux rows (3 x NS)
template <int VK> struct CurvedX {
  static constexpr int v = (VK == VK_WEAK) ? 3 * CNS : NPreE<3>::v + 9;
};

// SF >= 0: the surface flux kind as a compile-time constant (the kernel then
// carries no other flux's code); SF < 0: the kind given at run time.
// FUSE: one IMEX ARK23 stage (split_rhs = false) of Euler-gravity with the
// weak-form linear Euler-gravity operator along the radial direction: the
// explicit tendency N(Q), the linear operator L(Q) (its contravariant radial
// flux rows staged beside the state, its faces in the same task loop, its
// source) and the EPI_ARK accumulation of N - L and L in one launch, so the
// state, aux fields and metric terms are read once per stage.  Per element
// shared memory then adds NS * Np (linear flux rows) and 2 * Nfp * NS (linear
// face slots); all six aux fields are staged.
template <int LAW, int VK, int SF, bool FUSE = false>
__global__ void __launch_bounds__(512) curved_kernel(const TendArgs A) {
  constexpr int NS = CNS;
  constexpr int NA = NAuxMax<LAW, 3>::v;
  constexpr int NX = CurvedX<VK>::v;
  extern __shared__ __align__(16) double smem[];
  const int Nq = A.Nq, Np = A.Np, Nfp = A.Nfp, E = A.E, na = A.naux;
  const int nqq = (Nq * Nq + 1) & ~1;
  double* sD = smem;  // D[i][m] = l_m'(xi_i)
  const size_t per = (size_t)(NS + na + NX) * Np + (size_t)6 * Nfp * NS +
                     (FUSE ? (size_t)NS * Np + (size_t)2 * Nfp * NS : 0);
  const int tid = threadIdx.x;
  const int el = tid / Np;
  const int node = tid - el * Np;
  const int e = blockIdx.x * E + el;
  const bool active = el < E && e < A.K;
  for (int i = tid; i < Nq * Nq; i += blockDim.x) sD[i] = A.Dmat[i];
  // the state, aux and accumulators below may come from the previous kernel
  // of the stream (programmatic dependent launch, launch_maybe_pdl)
  pdl_wait();
  double* base = smem + nqq + (size_t)(el < E ? el : 0) * per;
  double* sq = base;
  double* sa = sq + (size_t)NS * Np;
  double* sx = sa + (size_t)na * Np;
  // fused: linear radial flux rows after the face slots, then the linear face slots
  double* sxl = sx + (size_t)NX * Np + (size_t)6 * Nfp * NS;
  const size_t stride = A.stride;
  const size_t gid = (size_t)e * Np + node;
  double qn[NS], an[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) an[k] = 0.0;
  double MJ = 1.0, lg[3][3];
  if (active) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      qn[s] = A.q[s][gid];
      sq[s * Np + node] = qn[s];
    }
    for (int k = 0; k < na && k < NA; ++k) {
      an[k] = A.aux[(size_t)k * stride + gid];
      sa[k * Np + node] = an[k];
    }
    MJ = A.MJn[gid];
    // metric terms of the active directions only (the radial linear operator
    // of the IMEX stages reads a third of them)
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int c = 0; c < 3; ++c) lg[d][c] = ((A.dirs >> d) & 1) ? A.G[((size_t)d * 3 + c) * stride + gid] : 0.0;
    if constexpr (FUSE) {
      // the linear operator's contravariant radial flux rows (its volume
      // term's staged values: MJ g[3, :] . F_lin), as the weak-form kernel
      double F[3][NS];
      flux_rows<LAW_LEG>(A.lin_law, qn, an, F);
#pragma unroll
      for (int s2 = 0; s2 < NS; ++s2) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) acc = acc + lg[2][c] * F[c][s2];
        sxl[s2 * Np + node] = acc * MJ;
      }
    }
    if constexpr (VK == VK_WEAK) {
      double F[3][NS];
      flux_rows<LAW>(A.law, qn, an, F);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (!((A.dirs >> d) & 1)) continue;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          double acc = 0.0;
#pragma unroll
          for (int c = 0; c < 3; ++c) acc = acc + lg[d][c] * F[c][s];
          sx[(d * NS + s) * Np + node] = acc * MJ;
        }
      }
    } else {
      double P[NPreE<3>::v];
      precompute_euler<3>(A.law.gamma, qn, LAW == LAW_EG ? an[0] : 0.0, P);
#pragma unroll
      for (int k = 0; k < NPreE<3>::v; ++k) sx[k * Np + node] = P[k];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          lg[d][c] = MJ * lg[d][c];
          sx[(NPreE<3>::v + d * 3 + c) * Np + node] = lg[d][c];
        }
    }
  }
  __syncthreads();

  // ---------------------------------------------------------- face tasks
  const int ntask = E * 6 * Nfp;
  for (int t = tid; t < ntask; t += blockDim.x) {
    const int fe = t / (6 * Nfp);
    const int r = t - fe * 6 * Nfp;
    const int face = r / Nfp, j = r - face * Nfp;
    const int k = face >> 1, side = face & 1;
    const int eg = blockIdx.x * E + fe;
    if (eg >= A.K || !((A.dirs >> k) & 1)) continue;
    // face node j: tangential dimensions in increasing order, first fastest
    const int t0 = j % Nq, t1 = j / Nq;
    const int ek = side ? Nq - 1 : 0;
    const int fn = (k == 0) ? ek + Nq * (t0 + Nq * t1) : (k == 1) ? t0 + Nq * (ek + Nq * t1) : t0 + Nq * (t1 + Nq * ek);
    double* fb = smem + nqq + (size_t)fe * per;
    const double* fq = fb;
    const double* fa = fb + (size_t)NS * Np;
    double* slot = fb + (size_t)(NS + na + NX) * Np;
    const size_t fj = ((size_t)eg * 6 + face) * Nfp + j;
    double n[3], qm[NS], am[NA], qp[NS], ap[NA];
#pragma unroll
    for (int c = 0; c < 3; ++c) n[c] = A.fnrm[fj * 3 + c];
#pragma unroll
    for (int s = 0; s < NS; ++s) qm[s] = fq[s * Np + fn];
#pragma unroll
    for (int c = 0; c < NA; ++c) am[c] = ap[c] = 0.0;
    for (int c = 0; c < na && c < NA; ++c) am[c] = fa[c * Np + fn];
    const int nb = A.fnb[fj];
    if (nb >= 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s) qp[s] = A.q[s][nb];
      for (int c = 0; c < na && c < NA; ++c) ap[c] = A.aux[(size_t)c * stride + nb];
    } else {
      boundary_state_n(A.law, n, -1 - nb, qm, qp);
#pragma unroll
      for (int c = 0; c < NA; ++c) ap[c] = am[c];
    }
    double nf[NS];
    surface_flux_n<LAW>(A.law, SF >= 0 ? SF : A.sflux, n, qm, am, qp, ap, nf);
    const double fm = A.fMJ[fj];
#pragma unroll
    for (int s = 0; s < NS; ++s) slot[(face * Nfp + j) * NS + s] = fm * nf[s];
    if constexpr (FUSE) {
      if (k == 2) {  // the linear operator's radial faces
        double* sl = fb + (size_t)(NS + na + NX) * Np + (size_t)6 * Nfp * NS + (size_t)NS * Np;
        if (nb < 0) boundary_state_n(A.lin_law, n, -1 - nb, qm, qp);
        surface_flux_n<LAW_LEG>(A.lin_law, A.lin_sflux, n, qm, am, qp, ap, nf);
#pragma unroll
        for (int s = 0; s < NS; ++s) sl[(side * Nfp + j) * NS + s] = fm * nf[s];
      }
    }
  }
  __syncthreads();
  if (!active) return;

  // ------------------------------------------------------------- volume
  const double MJI = 1.0 / MJ;
  int ijk[3] = {node % Nq, (node / Nq) % Nq, node / (Nq * Nq)};
  double T[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) T[s] = -0.0;
  if ((A.dirs >> 2) & 1) add_sources<LAW, 3>(A.law, VK == VK_WEAK, qn, an, T);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!((A.dirs >> d) & 1)) continue;
    const int i = ijk[d];
    const int step = (d == 0) ? 1 : (d == 1) ? Nq : Nq * Nq;
    const int n0 = node - i * step;
    if constexpr (VK == VK_WEAK) {
      for (int m = 0; m < Nq; ++m) {
        const double Dm = sD[m * Nq + i] * MJI;
        const int nn = n0 + m * step;
#pragma unroll
        for (int s = 0; s < NS; ++s) T[s] = T[s] + Dm * sx[(d * NS + s) * Np + nn];
      }
    } else {
      double P1[NPreE<3>::v];
#pragma unroll
      for (int k = 0; k < NPreE<3>::v; ++k) P1[k] = sx[k * Np + node];
      for (int m = 0; m < Nq; ++m) {
        if (m == i) continue;  // -D_ii lg_i F + F lg_i D_ii: no contribution
        const int nn = n0 + m * step;
        double q2[NS], a2[NA], P2[NPreE<3>::v], lm[3];
#pragma unroll
        for (int s = 0; s < NS; ++s) q2[s] = sq[s * Np + nn];
#pragma unroll
        for (int c = 0; c < NA; ++c) a2[c] = 0.0;
        for (int c = 0; c < na && c < NA; ++c) a2[c] = sa[c * Np + nn];
#pragma unroll
        for (int k = 0; k < NPreE<3>::v; ++k) P2[k] = sx[k * Np + nn];
#pragma unroll
        for (int c = 0; c < 3; ++c) lm[c] = sx[(NPreE<3>::v + d * 3 + c) * Np + nn];
        double f1[NS], f2[NS];
        pair_contract<LAW, VK>(A.law, qn, an, P1, q2, a2, P2, lg[d], lm, f1, f2);
        const double Ddn = MJI * sD[i * Nq + m], Dnd = MJI * sD[m * Nq + i];
#pragma unroll
        for (int s = 0; s < NS; ++s) T[s] = T[s] - Ddn * f1[s] + Dnd * f2[s];
      }
    }
  }
  // ------------------------------------------------------------ surface
  const double* slot = sx + (size_t)NX * Np;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (!((A.dirs >> k) & 1)) continue;
    const int id = ijk[k];
    if (id != 0 && id != Nq - 1) continue;
    const int side = (id == Nq - 1) ? 1 : 0;
    const int j = (k == 0) ? ijk[1] + Nq * ijk[2] : (k == 1) ? ijk[0] + Nq * ijk[2] : ijk[0] + Nq * ijk[1];
    const int face = 2 * k + side;
#pragma unroll
    for (int s = 0; s < NS; ++s) T[s] = T[s] - slot[(face * Nfp + j) * NS + s] * MJI;
  }
  // fused: the linear operator L(Q) along the radial direction (the weak-form
  // kernel's sums in its order: source, D^T of the staged rows, faces)
  double TL[NS];
  if constexpr (FUSE) {
#pragma unroll
    for (int s = 0; s < NS; ++s) TL[s] = -0.0;
    add_sources<LAW_LEG, 3>(A.lin_law, true, qn, an, TL);
    const int i = ijk[2];
    const int n0 = node - i * Nq * Nq;
    for (int m = 0; m < Nq; ++m) {
      const double Dm = sD[m * Nq + i] * MJI;
      const int nn = n0 + m * Nq * Nq;
#pragma unroll
      for (int s = 0; s < NS; ++s) TL[s] = TL[s] + Dm * sxl[s * Np + nn];
    }
    if (i == 0 || i == Nq - 1) {
      const double* sl = sxl + (size_t)NS * Np;
      const int side = (i == Nq - 1) ? 1 : 0;
      const int j = ijk[0] + Nq * ijk[1];
#pragma unroll
      for (int s = 0; s < NS; ++s) TL[s] = TL[s] - sl[(side * Nfp + j) * NS + s] * MJI;
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double Ex = T[s] - TL[s];
#pragma unroll
      for (int jj = 0; jj < 3; ++jj)
        if (A.acc[jj][0]) {
          const double b0 = A.accin[jj][0] ? A.accin[jj][s][gid] : qn[s];
          A.acc[jj][s][gid] = b0 + A.adt * (A.ca[jj] * Ex + A.cb[jj] * TL[s]);
        }
    }
    return;
  }

  // ----------------------------------------------------------- epilogue
  switch (A.epi) {
    case EPI_SET:
#pragma unroll
      for (int s = 0; s < NS; ++s) A.out[s][gid] = T[s];
      break;
    case EPI_ADD:
#pragma unroll
      for (int s = 0; s < NS; ++s) A.out[s][gid] = A.out[s][gid] + T[s];
      break;
    case EPI_LSRK: {
      const double bdt = A.dte ? A.bdt * A.dte[e] : A.bdt;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double dqn = (A.a != 0.0) ? A.a * A.out[s][gid] + T[s] : T[s];
        A.out[s][gid] = dqn;
        A.out2[s][gid] = qn[s] + bdt * dqn;
      }
    } break;
    case EPI_ARK:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        // out holds N(Q), T = L(Q)
        const double Ex = A.out[s][gid] - T[s];
#pragma unroll
        for (int jj = 0; jj < 3; ++jj)
          if (A.acc[jj][0]) {
            const double b0 = A.accin[jj][0] ? A.accin[jj][s][gid] : qn[s];
            A.acc[jj][s][gid] = b0 + A.adt * (A.ca[jj] * Ex + A.cb[jj] * T[s]);
          }
      }
      break;
    case EPI_SUBOUT2:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double o2 = A.out2[s][gid];
        A.out[s][gid] = T[s];
        A.out2[s][gid] = o2 - T[s];
      }
      break;
    case EPI_RLSRK:
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double o2 = A.out2[s][gid];
        A.out[s][gid] = T[s];
        A.out2[s][gid] = A.a * o2 + T[s];
      }
      break;
  }
  pdl_trigger();
}

template <int LAW, int VK, int SF, bool FUSE = false>
void curved_launch(const TendArgs& A, int grid, int block, size_t smem, cudaStream_t st) {
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    if (cudaFuncSetAttribute(curved_kernel<LAW, VK, SF, FUSE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) == cudaSuccess)
      configured = smem;
  }
  launch_maybe_pdl(curved_kernel<LAW, VK, SF, FUSE>, dim3(grid), dim3(block), smem, st, A);
}

}  // namespace

size_t curved_smem_bytes(int vk, int naux, int Nq, int E, bool fuse) {
  const int Np = Nq * Nq * Nq, Nfp = Nq * Nq;
  const int nx = (vk == VK_WEAK) ? 3 * CNS : NPreE<3>::v + 9;
  size_t per = (size_t)(CNS + naux + nx) * Np + (size_t)6 * Nfp * CNS;
  if (fuse) per += (size_t)CNS * Np + (size_t)2 * Nfp * CNS;
  return sizeof(double) * ((size_t)((Nq * Nq + 1) & ~1) + per * E);
}

tend_launch_fn pick_launcher_curved_fused(int vk, int sflux, int lin_sflux) {
  // Euler-gravity with the EC or KG volume flux and the Rusanov flux on both
  // operators' faces (the sphere experiments); nullptr otherwise
  if (sflux != F_RUSANOV || lin_sflux != F_RUSANOV) return nullptr;
  if (vk == VK_EC) return curved_launch<LAW_EG, VK_EC, F_RUSANOV, true>;
  if (vk == VK_KG) return curved_launch<LAW_EG, VK_KG, F_RUSANOV, true>;
  return nullptr;
}

tend_launch_fn pick_launcher_curved(int law, int vk, int sflux) {
  // Rusanov (the sphere experiments' surface flux) built in; every other
  // surface flux through the run-time kind
  const bool rus = sflux == F_RUSANOV;
  switch (law) {
    case LAW_EULER:
      if (vk == VK_WEAK) return rus ? curved_launch<LAW_EULER, VK_WEAK, F_RUSANOV> : curved_launch<LAW_EULER, VK_WEAK, -1>;
      if (vk == VK_EC) return rus ? curved_launch<LAW_EULER, VK_EC, F_RUSANOV> : curved_launch<LAW_EULER, VK_EC, -1>;
      if (vk == VK_KG) return rus ? curved_launch<LAW_EULER, VK_KG, F_RUSANOV> : curved_launch<LAW_EULER, VK_KG, -1>;
      if (vk == VK_CENTRAL) return curved_launch<LAW_EULER, VK_CENTRAL, -1>;
      break;
    case LAW_EG:
      if (vk == VK_WEAK) return rus ? curved_launch<LAW_EG, VK_WEAK, F_RUSANOV> : curved_launch<LAW_EG, VK_WEAK, -1>;
      if (vk == VK_EC) return rus ? curved_launch<LAW_EG, VK_EC, F_RUSANOV> : curved_launch<LAW_EG, VK_EC, -1>;
      if (vk == VK_KG) return rus ? curved_launch<LAW_EG, VK_KG, F_RUSANOV> : curved_launch<LAW_EG, VK_KG, -1>;
      if (vk == VK_CENTRAL) return curved_launch<LAW_EG, VK_CENTRAL, -1>;
      break;
    case LAW_LEG:
      if (vk == VK_WEAK) return rus ? curved_launch<LAW_LEG, VK_WEAK, F_RUSANOV> : curved_launch<LAW_LEG, VK_WEAK, -1>;
      if (vk == VK_CENTRAL) return curved_launch<LAW_LEG, VK_CENTRAL, -1>;
      break;
  }
  return nullptr;
}

}  // namespace atb
