// Device physics of the balance laws and numerical fluxes (sm_100a).
//
// Semantics follow the reference's pointwise functions; the code is shaped
// for the device: every flux is evaluated for ONE coordinate direction d at a
// time (brick metrics are diagonal, so the flux-differencing contraction only
// needs the d-th row of the two-point flux), and per-node quantities that the
// reference recomputes per pair (velocity, pressure, b = rho/2p) are computed
// once per node and passed in.  Values are identical to the reference's up to
// floating-point rounding.
//
//   flux / wavespeed / pressure   src/balancelaws/*.jl
//   logavg, avg, roe_avg          src/numericalfluxes.jl:8-23
//   two-point EC / KG             src/balancelaws/euler.jl:140-196,
//                                 euler_gravity.jl:200-269, shallow_water.jl:112-136
//   Rusanov / default surface     src/numericalfluxes.jl:27-42
//   Roe                           euler.jl:91-138, euler_gravity.jl:149-198, shallow_water.jl:68-110
//   Matrix dissipation            euler.jl:198-256, euler_gravity.jl:271-332
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace atb {

enum { LAW_ADV = 0, LAW_EULER = 1, LAW_EG = 2, LAW_LEG = 3, LAW_SW = 4 };
enum { F_CENTRAL = 0, F_RUSANOV = 1, F_EC = 2, F_KG = 3, F_ROE = 4, F_MATRIX = 5 };
enum { BC_COPY = 0, BC_REFLECT = 1, BC_INFLOW_ZERO = 2, BC_DIRICHLET = 3 };
enum { SRC_NONE = 0, SRC_CORIOLIS = 1 };

struct LawP {
  int kind, dim, ns, naux;
  double gamma, grav;
  double adv_u[3];
  double omega[3];
  double bc_state[2][5];
  int pde, bc, src, swtopo;
};

template <int LAW, int DIM> struct NSt { static constexpr int v = (LAW == LAW_ADV) ? 1 : DIM + 2; };

template <class T> __device__ __forceinline__ T dmax(T a, T b) { return a < b ? b : a; }
__device__ __forceinline__ double dlog(double x) { return log(x); }
__device__ __forceinline__ float dlog(float x) { return logf(x); }
__device__ __forceinline__ double dsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dsqrt(float x) { return sqrtf(x); }
template <class T> __device__ __forceinline__ T eps_of();
template <> __device__ __forceinline__ double eps_of<double>() { return 2.220446049250313e-16; }
template <> __device__ __forceinline__ float eps_of<float>() { return 1.1920929e-7f; }

// logarithmic mean (a+b)/(2F), F = log(zeta)/(2f), f = (zeta-1)/(zeta+1),
// series in u = f^2 below eps (src/numericalfluxes.jl:9-21).  Rearranged as
// (a+b) f / log(zeta): numerator and denominator both come from the same
// rounded zeta, so the result is accurate to a few ulps near the branch.
template <class T> __device__ __forceinline__ T logavg(T a, T b) {
  T zeta = a / b;
  T zm = zeta - T(1), zp = zeta + T(1);
  T f = zm / zp;
  T u = f * f;
  if (u < eps_of<T>()) {
    T F = T(1) + u * (T(1) / T(3) + u * (T(1) / T(5) + u * (T(1) / T(7) + u * (T(1) / T(9)))));
    return (a + b) / (T(2) * F);
  }
  return (a + b) * f / dlog(zeta);
}

// Logarithmic mean for the flux-differencing volume term: the reference's
// series, extended to eight terms, is used below u = f^2 = ((a-b)/(a+b))^2 <
// 1e-2 (truncation error below u^8/17 < 1e-17 relative), so log() is
// evaluated only for values more than ~20% apart; above the threshold
// (a - b) / log(a / b) is accurate to a few ulps because |log(a/b)| > 0.2.
// (Same function as the reference's logavg to FP64 rounding; the threshold
// follows Ranocha et al., "Efficient implementation of modern entropy stable
// and kinetic energy preserving DG methods", 2022.)
template <class T> __device__ __forceinline__ T logavg_fast(T a, T b) {
  const T s = a + b, d = a - b;
  if (d * d < T(1e-2) * (s * s)) {
    // eight series terms: truncation under 1e-17 relative below u = 1e-2
    const T f = d / s;
    const T u = f * f;
    const T F = T(1) + u * (T(1) / T(3) + u * (T(1) / T(5) + u * (T(1) / T(7) + u * (T(1) / T(9) +
                u * (T(1) / T(11) + u * (T(1) / T(13) + u * (T(1) / T(15))))))));
    return s / (T(2) * F);
  }
  return d / dlog(a / b);
}

template <class T> __device__ __forceinline__ T roe_avg(T srm, T srp, T sm, T sp) {
  return (srm * sm + srp * sp) / (srm + srp);
}

// ------------------------------------------------------------ point state
template <int DIM, class T> __device__ __forceinline__ T dot(const T* a, const T* b) {
  T s = a[0] * b[0];
#pragma unroll
  for (int d = 1; d < DIM; ++d) s = s + a[d] * b[d];
  return s;
}

// pressure of Euler / EulerGravity (Phi = 0 for plain Euler)
template <int DIM, class T> __device__ __forceinline__ T pressure_eg(T gamma, const T* q, T Phi) {
  return (gamma - T(1)) * (q[DIM + 1] - dot<DIM>(q + 1, q + 1) / (T(2) * q[0]) - q[0] * Phi);
}

// physical flux, direction d: f[s] = F[d][s]
template <int LAW, int DIM, class T>
__device__ __forceinline__ void flux_dir(const LawP& L, int d, const T* q, const T* aux, T* f) {
  if constexpr (LAW == LAW_ADV) {
    f[0] = T(L.adv_u[d]) * q[0];
  } else if constexpr (LAW == LAW_EULER || LAW == LAW_EG) {
    T Phi = (LAW == LAW_EG) ? aux[0] : T(0);
    T rho = q[0];
    T p = pressure_eg<DIM>(T(L.gamma), q, Phi);
    T dp = p;
    if (LAW == LAW_EG && L.pde) dp = dp - aux[DIM + 2];
    T ud = q[1 + d] / rho;
    f[0] = q[1 + d];
#pragma unroll
    for (int c = 0; c < DIM; ++c) f[1 + c] = q[1 + d] * (q[1 + c] / rho);  // rhou_d u_c
    f[1 + d] = f[1 + d] + dp;
    f[DIM + 1] = ud * (q[DIM + 1] + p);
  } else if constexpr (LAW == LAW_LEG) {
    T Phi = aux[0];
    T g = T(L.gamma);
    T p = (g - T(1)) * (q[DIM + 1] - q[0] * Phi);
    T ref_rho = aux[DIM + 1], ref_p = aux[DIM + 2];
    T ref_rhoe = ref_p / (g - T(1)) + ref_rho * Phi;
    f[0] = q[1 + d];
#pragma unroll
    for (int c = 0; c < DIM; ++c) f[1 + c] = T(0);
    f[1 + d] = p;
    f[DIM + 1] = ((ref_rhoe + ref_p) / ref_rho) * q[1 + d];
  } else {  // shallow water
    T rho = q[0];
    T p = T(L.grav) * (rho * rho) / T(2);
#pragma unroll
    for (int c = 0; c < DIM; ++c) f[1 + c] = q[1 + d] * (q[1 + c] / rho);
    f[0] = q[1 + d];
    f[1 + d] = f[1 + d] + p;
    f[DIM + 1] = (q[1 + d] / rho) * q[DIM + 1];
  }
}

// wavespeed for normal n = sgn * e_d
template <int LAW, int DIM, class T>
__device__ __forceinline__ T wavespeed_dir(const LawP& L, int d, const T* q, const T* aux) {
  if constexpr (LAW == LAW_ADV) {
    return fabs(T(L.adv_u[d]));
  } else if constexpr (LAW == LAW_EULER || LAW == LAW_EG) {
    T Phi = (LAW == LAW_EG) ? aux[0] : T(0);
    T p = pressure_eg<DIM>(T(L.gamma), q, Phi);
    return fabs(q[1 + d] / q[0]) + dsqrt(T(L.gamma) * p / q[0]);
  } else if constexpr (LAW == LAW_LEG) {
    return dsqrt(T(L.gamma) * aux[DIM + 2] / aux[DIM + 1]);
  } else {
    return fabs(q[1 + d] / q[0]) + dsqrt(T(L.grav) * q[0]);
  }
}

// ----------------------------------------------- two-point flux, dir d
// Per-node precomputed quantities for the entropy-conservative and
// Kennedy-Gruber fluxes of Euler / EulerGravity:
//   P[0..DIM-1] = u, P[DIM] = p, P[DIM+1] = b = rho/(2p), P[DIM+2] = |u|^2,
//   P[DIM+3] = e = rhoe/rho, P[DIM+4] = p/rho = 1/(2b)
template <int DIM> struct NPreE { static constexpr int v = DIM + 5; };

template <int DIM, class T>
__device__ __forceinline__ void precompute_euler(T gamma, const T* q, T Phi, T* P) {
  T rho = q[0];
#pragma unroll
  for (int c = 0; c < DIM; ++c) P[c] = q[1 + c] / rho;
  T p = pressure_eg<DIM>(gamma, q, Phi);
  P[DIM] = p;
  P[DIM + 1] = rho / (T(2) * p);
  P[DIM + 2] = dot<DIM>(P, P);
  P[DIM + 3] = q[DIM + 1] / rho;
  P[DIM + 4] = p / rho;
}

// EC two-point flux, row d (ordered pair: node 1 = own, node 2 = partner)
template <int LAW, int DIM, class T>
__device__ __forceinline__ void ec_dir(T gamma, int d, T r1, const T* P1, T Phi1, T r2, const T* P2, T Phi2,
                                       T* f) {
  T rho_avg = (r1 + r2) / T(2);
  T ua[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) ua[c] = (P1[c] + P2[c]) / T(2);
  T b1 = P1[DIM + 1], b2 = P2[DIM + 1];
  T b_avg = (b1 + b2) / T(2);
  T u2_avg = (P1[DIM + 2] + P2[DIM + 2]) / T(2);
  T rho_log = logavg(r1, r2);
  T b_log = logavg(b1, b2);
  T pc = rho_avg / (T(2) * b_avg);
  T ud = ua[d];
  T frd = ud * rho_log;
  f[0] = frd;
  T mu = T(0);
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    T m = ud * (ua[c] * rho_log);
    if (c == d) m = m + pc;
    f[1 + c] = m;
    mu = (c == 0) ? m * ua[c] : mu + m * ua[c];
  }
  T c1 = T(1) / (T(2) * (gamma - T(1)) * b_log) - u2_avg / T(2);
  if (LAW == LAW_EG) c1 = c1 + (Phi1 + Phi2) / T(2);
  f[DIM + 1] = c1 * frd + mu;
  if (LAW == LAW_EG) {
    T alpha = b_avg * rho_log / (T(2) * b1);
    f[1 + d] = f[1 + d] - alpha * (Phi1 - Phi2);
  }
}

// Symmetric part of the EC two-point flux, row d: everything except the
// Euler-gravity fluctuation -alpha (Phi1 - Phi2) on the momentum-d entry,
// alpha = b_avg rho_log / (2 b1).  Returns b_avg * rho_log in *xtra so that
// each node of the pair adds its own fluctuation with its own 1/(2 b).
// Per-node P: u (DIM), p, b, |u|^2, e, p/rho.
template <int LAW, int DIM, class T>
__device__ __forceinline__ void ec_sym_dir(T gamma, int d, T r1, const T* P1, T Phi1, T r2, const T* P2, T Phi2,
                                           T* f, T* xtra) {
  T rho_avg = (r1 + r2) / T(2);
  T ua[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) ua[c] = (P1[c] + P2[c]) / T(2);
  const T b1 = P1[DIM + 1], b2 = P2[DIM + 1];
  const T b_avg = (b1 + b2) / T(2);
  const T u2_avg = (P1[DIM + 2] + P2[DIM + 2]) / T(2);
  const T rho_log = logavg_fast(r1, r2);
  const T b_log = logavg_fast(b1, b2);
  // one reciprocal for rho_avg / (2 b_avg) and 1 / (2 (gamma-1) b_log)
  const T rinv = T(1) / (b_avg * b_log);
  const T pc = rho_avg * b_log * rinv / T(2);
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
  T c1 = b_avg * rinv / (T(2) * (gamma - T(1))) - u2_avg / T(2);
  if (LAW == LAW_EG) c1 = c1 + (Phi1 + Phi2) / T(2);
  f[DIM + 1] = c1 * frd + mu;
  *xtra = b_avg * rho_log;
}

// Kennedy-Gruber two-point flux, row d
template <int LAW, int DIM, class T>
__device__ __forceinline__ void kg_dir(int d, T r1, const T* P1, T Phi1, T r2, const T* P2, T Phi2, T* f) {
  T rho_avg = (r1 + r2) / T(2);
  T ud = (P1[d] + P2[d]) / T(2);
  T e_avg = (P1[DIM + 3] + P2[DIM + 3]) / T(2);
  T p_avg = (P1[DIM] + P2[DIM]) / T(2);
  T frd = ud * rho_avg;
  f[0] = frd;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    T m = ud * (((P1[c] + P2[c]) / T(2)) * rho_avg);
    if (c == d) m = m + p_avg;
    f[1 + c] = m;
  }
  if (LAW == LAW_EG) f[1 + d] = f[1 + d] - (rho_avg / T(2)) * (Phi1 - Phi2);
  f[DIM + 1] = ud * (rho_avg * e_avg + p_avg);
}

// shallow-water EC two-point flux, row d; P = [u (DIM), theta]; b = topography
template <int DIM, class T>
__device__ __forceinline__ void sw_ec_dir(T grav, int topo, int d, const T* q1, const T* P1, T b1, const T* q2,
                                          const T* P2, T b2, T* f) {
  T r1 = q1[0], r2 = q2[0];
  T rho_avg = (r1 + r2) / T(2);
  T rho2_avg = (r1 * r1 + r2 * r2) / T(2);
  T md = (q1[1 + d] + q2[1 + d]) / T(2);
  T th_avg = (P1[DIM] + P2[DIM]) / T(2);
  T pc = grav * (rho_avg * rho_avg - rho2_avg / T(2));
  if (topo) pc = pc - grav * r1 * (b1 - b2) / T(2);
  f[0] = md;
#pragma unroll
  for (int c = 0; c < DIM; ++c) f[1 + c] = md * ((P1[c] + P2[c]) / T(2));
  f[1 + d] = f[1 + d] + pc;
  f[DIM + 1] = md * th_avg;
}

// ------------------------------------------------------- entropy variables
template <int LAW, int DIM, class T>
__device__ __forceinline__ void entropyvars(const LawP& L, const T* q, const T* aux, T* v) {
  if constexpr (LAW == LAW_ADV) {
    v[0] = q[0];
  } else if constexpr (LAW == LAW_EULER || LAW == LAW_EG) {
    T g = T(L.gamma);
    T Phi = (LAW == LAW_EG) ? aux[0] : T(0);
    T rho = q[0];
    T p = pressure_eg<DIM>(g, q, Phi);
    T s = log(p / pow(rho, g));
    T b = rho / (T(2) * p);
    T u[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) u[c] = q[1 + c] / rho;
    T uu = dot<DIM>(u, u);
    v[0] = (LAW == LAW_EG) ? (g - s) / (g - T(1)) - (uu - T(2) * Phi) * b : (g - s) / (g - T(1)) - uu * b;
#pragma unroll
    for (int c = 0; c < DIM; ++c) v[1 + c] = (T(2) * b) * u[c];
    v[DIM + 1] = -(T(2) * b);
  } else if constexpr (LAW == LAW_SW) {
    T rho = q[0];
    v[0] = -dot<DIM>(q + 1, q + 1) / (T(2) * (rho * rho)) + T(L.grav) * rho;
    if (L.swtopo) v[0] = v[0] + T(L.grav) * aux[0];
#pragma unroll
    for (int c = 0; c < DIM; ++c) v[1 + c] = q[1 + c] / rho;
    v[DIM + 1] = T(0);
  } else {
#pragma unroll
    for (int s = 0; s < DIM + 2; ++s) v[s] = T(0);
  }
}

template <int LAW, int DIM, class T> __device__ __forceinline__ T entropy_fn(const LawP& L, const T* q, const T* aux) {
  if constexpr (LAW == LAW_ADV) {
    return q[0] * q[0] / T(2);
  } else if constexpr (LAW == LAW_EULER || LAW == LAW_EG) {
    T g = T(L.gamma);
    T Phi = (LAW == LAW_EG) ? aux[0] : T(0);
    T p = pressure_eg<DIM>(g, q, Phi);
    T s = log(p / pow(q[0], g));
    return (-q[0]) * s / (g - T(1));
  } else if constexpr (LAW == LAW_SW) {
    T rho = q[0];
    T e = dot<DIM>(q + 1, q + 1) / (T(2) * rho) + T(L.grav) * (rho * rho) / T(2);
    if (L.swtopo) e = e + T(L.grav) * rho * aux[0];
    return e;
  } else {
    return T(0);
  }
}

// ------------------------------------------------------------ boundaries
template <int LAW, int DIM, class T>
__device__ __forceinline__ void boundary_state(const LawP& L, int d, T sgn, int tag, const T* qm, T* qp) {
  constexpr int NS = NSt<LAW, DIM>::v;
  if (L.bc == BC_REFLECT && NS > 1) {
    // rhou+ = rhou- - 2 (n . rhou-) n with n = sgn e_d
#pragma unroll
    for (int s = 0; s < NS; ++s) qp[s] = qm[s];
    T nm = sgn * qm[1 + d];
    qp[1 + d] = qm[1 + d] - T(2) * nm * sgn;
  } else if (L.bc == BC_INFLOW_ZERO) {
    T un = sgn * T(L.adv_u[d]);
    // dot(u, n) over all components: the zero components add nothing
#pragma unroll
    for (int s = 0; s < NS; ++s) qp[s] = (un <= T(0)) ? T(0) : qm[s];
  } else if (L.bc == BC_DIRICHLET) {
    const double* st = L.bc_state[tag == 1 ? 0 : 1];
#pragma unroll
    for (int s = 0; s < NS; ++s) qp[s] = T(st[s]);
  } else {
#pragma unroll
    for (int s = 0; s < NS; ++s) qp[s] = qm[s];
  }
}

// Physical flux row d and wave speed of Euler / Euler-gravity / shallow water
// from one reciprocal 1/rho (the reference recomputes rho u_c / rho in every
// flux row and in the wave speed; the values agree to an ulp).
template <int LAW, int DIM, class T>
__device__ __forceinline__ T flux_ws_recip(const LawP& L, int d, const T* q, const T* aux, T* f) {
  const T rinv = T(1) / q[0];
  T u[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) u[c] = q[1 + c] * rinv;
  if constexpr (LAW == LAW_SW) {
    const T p = T(L.grav) * (q[0] * q[0]) / T(2);
    f[0] = q[1 + d];
#pragma unroll
    for (int c = 0; c < DIM; ++c) f[1 + c] = q[1 + d] * u[c];
    f[1 + d] = f[1 + d] + p;
    f[DIM + 1] = u[d] * q[DIM + 1];
    return fabs(u[d]) + dsqrt(T(L.grav) * q[0]);
  } else {
    const T Phi = (LAW == LAW_EG) ? aux[0] : T(0);
    const T g = T(L.gamma);
    const T p = (g - T(1)) * (q[DIM + 1] - dot<DIM>(q + 1, u) / T(2) - q[0] * Phi);
    T dp = p;
    if (LAW == LAW_EG && L.pde) dp = dp - aux[DIM + 2];
    f[0] = q[1 + d];
#pragma unroll
    for (int c = 0; c < DIM; ++c) f[1 + c] = q[1 + d] * u[c];
    f[1 + d] = f[1 + d] + dp;
    f[DIM + 1] = u[d] * (q[DIM + 1] + p);
    return fabs(u[d]) + dsqrt(g * p * rinv);
  }
}

// FP32-flux precision form of flux_ws_recip: the mass flux (a state value)
// and the pressure term stay FP64 -- the pressure difference across a face
// balances gravity / bathymetry in a resting state -- while the reciprocal
// of rho, the velocities, kinetic energy, advective products, the energy
// flux product and the wave speed are FP32.
template <int LAW, int DIM>
__device__ __forceinline__ double flux_ws_recip32(const LawP& L, int d, const double* q, const double* aux,
                                                  double* f) {
  const float rinv = 1.f / (float)q[0];
  float u[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) u[c] = (float)q[1 + c] * rinv;
  f[0] = q[1 + d];
  if constexpr (LAW == LAW_SW) {
    const double p = L.grav * (q[0] * q[0]) / 2.0;
#pragma unroll
    for (int c = 0; c < DIM; ++c) f[1 + c] = (double)((float)q[1 + d] * u[c]);
    f[1 + d] = f[1 + d] + p;
    f[DIM + 1] = (double)(u[d] * (float)q[DIM + 1]);
    return (double)(fabsf(u[d]) + sqrtf((float)L.grav * (float)q[0]));
  } else {
    const double Phi = (LAW == LAW_EG) ? aux[0] : 0.0;
    float ke = 0.f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) ke += (float)q[1 + c] * u[c];
    const double p = (L.gamma - 1.0) * (q[DIM + 1] - (double)(0.5f * ke) - q[0] * Phi);
    double dp = p;
    if (LAW == LAW_EG && L.pde) dp = dp - aux[DIM + 2];
#pragma unroll
    for (int c = 0; c < DIM; ++c) f[1 + c] = (double)((float)q[1 + d] * u[c]);
    f[1 + d] = f[1 + d] + dp;
    f[DIM + 1] = (double)(u[d] * (float)(q[DIM + 1] + p));
    return (double)(fabsf(u[d]) + sqrtf((float)L.gamma * (float)p * rinv));
  }
}

// ------------------------------------------------ FP32-flux two-point fluxes
// F(u) = atanh(sqrt u) / sqrt u = sum_k u^k / (2k+1) and G = 1 / F, eight
// terms each: below u = 1e-2 the truncation is under 1e-17 relative, so the
// series branch is as accurate as the logarithm it replaces there
template <class T> __device__ __forceinline__ T series_F(T u) {
  return T(1) + u * (T(1) / T(3) + u * (T(1) / T(5) + u * (T(1) / T(7) + u * (T(1) / T(9) +
         u * (T(1) / T(11) + u * (T(1) / T(13) + u * (T(1) / T(15))))))));
}
template <class T> __device__ __forceinline__ T series_G(T u) {
  return T(1) - u * (T(1) / T(3) + u * (T(4) / T(45) + u * (T(44) / T(945) + u * (T(428) / T(14175) +
         u * (T(10196) / T(467775) + u * (T(10719068) / T(638512875) + u * (T(25865068) / T(1915538625))))))));
}

// EC flux, row d, FP32-flux precision form.  Inputs: FP64 rho, p, b and the
// geopotential; FP32 velocities and |u|^2.  The pressure-like term is the
// FP64 average of the two pressures plus a second-order FP32 correction,
//   rho_avg / (2 b_avg) = p_avg - (p1 - p2)(b2 - b1) / (2 (b1 + b2)),
// and the logarithmic mean of rho is the FP64 average minus a small FP32
// series correction, so the hydrostatic balance between the pressure and
// gravity terms is carried in FP64 while every division, logarithm and
// advective product is FP32.  Returns FP64 row values and b_avg * rho_log.
template <int LAW, int DIM>
__device__ __forceinline__ void ec_vol32(float igm1, int d, double r1, double p1, double b1, const float* u1,
                                         float uu1, double Phi1, double r2, double p2, double b2,
                                         const float* u2, float uu2, double Phi2, double* f, double* xtra) {
  const double rho_avg = (r1 + r2) * 0.5, p_avg = (p1 + p2) * 0.5, b_avg = (b1 + b2) * 0.5;
  const float rs = (float)(r1 + r2), rd = (float)(r1 - r2);
  const float bs = (float)(b1 + b2), bd = (float)(b1 - b2);
  const float fr = rd / rs, fb = bd / bs;
  const float ur = fr * fr, ub = fb * fb;
  double rho_log;
  float cterm;
  if (ur < 1e-2f && ub < 1e-2f) {
    // 1 - G(u) = u/3 + 4u^2/45 + 44u^3/945 + ... (the terms of series_G)
    const float cr = ur * (1.f / 3.f + ur * (4.f / 45.f + ur * (44.f / 945.f + ur * (428.f / 14175.f +
                     ur * (10196.f / 467775.f + ur * (10719068.f / 638512875.f + ur * (25865068.f / 1915538625.f)))))));
    rho_log = rho_avg - rho_avg * (double)cr;
    cterm = series_F(ub) * igm1 / bs;  // 1 / (2 (gamma-1) b_log)
  } else {
    rho_log = logavg_fast(r1, r2);
    const float b_log = (ub < 1e-2f) ? 0.5f * bs * series_G(ub) : bd / logf((float)b1 / (float)b2);
    cterm = 0.5f * igm1 / b_log;
  }
  const double corr = (double)((float)(p1 - p2) * (float)(b2 - b1) / (2.f * bs));
  const double pc = p_avg - corr;
  float ua[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) ua[c] = 0.5f * (u1[c] + u2[c]);
  const float rl = (float)rho_log;
  const float ud = ua[d];
  const float frd = ud * rl;
  f[0] = (double)frd;
  float mu = 0.f;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const float m = ud * (ua[c] * rl);
    f[1 + c] = (double)m;
    mu += m * ua[c];
  }
  f[1 + d] += pc;
  mu += (float)pc * ud;
  float c1 = cterm - 0.25f * (uu1 + uu2);
  if (LAW == LAW_EG) c1 += (float)((Phi1 + Phi2) * 0.5);
  f[DIM + 1] = (double)(c1 * frd + mu);
  *xtra = b_avg * rho_log;
}

// shallow-water EC flux, row d, FP32-flux form: the pressure term
// g (rho_avg^2 - rho2_avg/2) = g rho1 rho2 / 2 stays FP64, advective products
// are FP32
template <int DIM>
__device__ __forceinline__ void sw_vol32(double grav, int d, const double* q1, const float* P1, const double* q2,
                                         const float* P2, double* f) {
  const double md = 0.5 * (q1[1 + d] + q2[1 + d]);
  const float mdf = (float)md;
  f[0] = md;
#pragma unroll
  for (int c = 0; c < DIM; ++c) f[1 + c] = (double)(mdf * (0.5f * (P1[c] + P2[c])));
  f[1 + d] += grav * q1[0] * q2[0] * 0.5;
  f[DIM + 1] = (double)(mdf * (0.5f * (P1[DIM] + P2[DIM])));
}

// Kennedy-Gruber flux, row d, FP32-flux precision form: the density and
// pressure averages -- the pressure term balances the FP64 gravity fluctuation
// of a hydrostatic state -- stay FP64; velocities, the specific energy and the
// advective products are FP32.
template <int DIM>
__device__ __forceinline__ void kg_vol32(int d, double r1, double p1, const float* u1, float e1, double r2, double p2,
                                         const float* u2, float e2, double* f) {
  const double rho_avg = (r1 + r2) * 0.5, p_avg = (p1 + p2) * 0.5;
  const float rf = (float)rho_avg;
  const float ud = 0.5f * (u1[d] + u2[d]);
  f[0] = (double)(ud * rf);
#pragma unroll
  for (int c = 0; c < DIM; ++c) f[1 + c] = (double)(ud * ((0.5f * (u1[c] + u2[c])) * rf));
  f[1 + d] = f[1 + d] + p_avg;
  const float e_avg = 0.5f * (e1 + e2);
  f[DIM + 1] = (double)(ud * (rf * e_avg)) + (double)ud * p_avg;
}

// Per-side values of the FP32-flux two-point fluxes, as the volume kernel
// stages them: FP64 pressure and b = rho / (2 p), FP32 velocity, |u|^2 and
// specific energy.
template <int DIM>
__device__ __forceinline__ void pre32(double gamma, const double* q, double Phi, double* p, double* b, float* u,
                                      float* uu, float* e) {
  const double rinv = 1.0 / q[0];
  const double ke = 0.5 * dot<DIM>(q + 1, q + 1) * rinv;
  *p = (gamma - 1.0) * (q[DIM + 1] - ke - q[0] * Phi);
  *b = 0.5 / (*p * rinv);
  const float rinvf = (float)rinv;
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    u[c] = (float)q[1 + c] * rinvf;
    s += u[c] * u[c];
  }
  *uu = s;
  *e = (float)q[DIM + 1] * rinvf;
}

// Roe dissipation (src/balancelaws/euler.jl:91-138, euler_gravity.jl:149-198;
// src/balancelaws/shallow_water.jl:68-110) in FP32 from FP64 jumps of the
// density, pressure (or height) and velocities, which vanish exactly where
// the state is continuous -- at rest the dissipation stays exactly zero.
// Returns the dissipation vector (the flux is central - it).
template <int LAW, int DIM>
__device__ __forceinline__ void roe_diss32(const LawP& L, int d, double sgn, const double* qm, const double* am,
                                           const double* qp, float* fpv) {
  float n[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) n[c] = (c == d) ? (float)sgn : 0.f;
  const float rm = (float)qm[0], rp = (float)qp[0];
  const float rim = 1.f / rm, rip = 1.f / rp;
  float um[DIM], up[DIM], u[DIM], du[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) { um[c] = (float)qm[1 + c] * rim; up[c] = (float)qp[1 + c] * rip; }
  const float srm = sqrtf(rm), srp = sqrtf(rp);
  const float rho = sqrtf(rm * rp);
#pragma unroll
  for (int c = 0; c < DIM; ++c) { u[c] = roe_avg(srm, srp, um[c], up[c]); du[c] = up[c] - um[c]; }
  const float drho = (float)(qp[0] - qm[0]);
  float c, dp, hm = 0.f, hp = 0.f, thm = 0.f, thp = 0.f;
  if constexpr (LAW == LAW_SW) {
    const double pm = L.grav * (qm[0] * qm[0]) / 2.0, pp = L.grav * (qp[0] * qp[0]) / 2.0;
    dp = (float)(pp - pm);
    thm = (float)qm[DIM + 1] * rim;
    thp = (float)qp[DIM + 1] * rip;
    c = roe_avg(srm, srp, sqrtf((float)L.grav * rm), sqrtf((float)L.grav * rp));
  } else {
    const double Phi = (LAW == LAW_EG) ? am[0] : 0.0;
    const double pm = pressure_eg<DIM>(L.gamma, qm, Phi), pp = pressure_eg<DIM>(L.gamma, qp, Phi);
    dp = (float)(pp - pm);
    const float g = (float)L.gamma;
    hm = ((float)qm[DIM + 1] + (float)pm) * rim;
    hp = ((float)qp[DIM + 1] + (float)pp) * rip;
    c = roe_avg(srm, srp, sqrtf(g * (float)pm * rim), sqrtf(g * (float)pp * rip));
  }
  const float un = dot<DIM>(u, n), dun = dot<DIM>(du, n);
  const float cm2 = 1.f / (c * c);
  const float w1 = fabsf(un - c) * (dp - rho * c * dun) * cm2 / 2.f;
  const float w2 = fabsf(un + c) * (dp + rho * c * dun) * cm2 / 2.f;
  const float w3 = fabsf(un) * (drho - dp * cm2);
  const float w4 = fabsf(un) * rho;
  fpv[0] = (w1 + w2 + w3) / 2.f;
#pragma unroll
  for (int k = 0; k < DIM; ++k)
    fpv[1 + k] = (w1 * (u[k] - c * n[k]) + w2 * (u[k] + c * n[k]) + w3 * u[k] + w4 * (du[k] - dun * n[k])) / 2.f;
  if constexpr (LAW == LAW_SW) {
    const float th = roe_avg(srm, srp, thm, thp);
    const float w5 = fabsf(un) * ((float)(qp[DIM + 1] - qm[DIM + 1]) - th * dp * cm2);
    fpv[DIM + 1] = ((w1 + w2) * th + w5) / 2.f;
  } else {
    const float h = roe_avg(srm, srp, hm, hp);
    float ke = w3 * dot<DIM>(u, u) / 2.f;
    if (LAW == LAW_EG) ke = w3 * (dot<DIM>(u, u) / 2.f + (float)am[0]);
    fpv[DIM + 1] = (w1 * (h - c * un) + w2 * (h + c * un) + ke + w4 * (dot<DIM>(u, du) - un * dun)) / 2.f;
  }
}

// Matrix dissipation (src/balancelaws/euler.jl:198-256, euler_gravity.jl:271-
// 332, including the reference's u2_bar quirk of norms at :219) in FP32 from
// the FP64 jump of the entropy variables.  Returns D (the flux is EC - D/2).
template <int LAW, int DIM>
__device__ __forceinline__ void matrix_diss32(const LawP& L, int d, double sgn, const double* qm, const double* am,
                                              const double* qp, const double* ap, double bm64, double bp64,
                                              const float* um, float uum, const float* up, float uup, float* Dm) {
  constexpr int NS = NSt<LAW, DIM>::v;
  const float g = (float)L.gamma;
  float n[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) n[c] = (c == d) ? (float)sgn : 0.f;
  const float Phi_avg = (LAW == LAW_EG) ? (float)((am[0] + ap[0]) / 2.0) : 0.f;
  const float rm = (float)qm[0], rp = (float)qp[0], bm = (float)bm64, bp = (float)bp64;
  const float rho_log = logavg(rm, rp);
  const float b_log = logavg(bm, bp);
  float ua[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) ua[c] = (um[c] + up[c]) / 2.f;
  const float p_avg = ((rm + rp) / 2.f) / (2.f * ((bm + bp) / 2.f));
  const float u2_bar = 2.f * sqrtf(dot<DIM>(ua, ua)) - (sqrtf(uum) + sqrtf(uup)) / 2.f;
  float h_bar = g / (2.f * b_log * (g - 1.f)) + u2_bar / 2.f;
  if (LAW == LAW_EG) h_bar += Phi_avg;
  const float c_bar = sqrtf(g * p_avg / rho_log);
  float umc[DIM], upc[DIM], ut[DIM];
  const float un = dot<DIM>(ua, n);
#pragma unroll
  for (int k = 0; k < DIM; ++k) {
    umc[k] = ua[k] - c_bar * n[k];
    upc[k] = ua[k] + c_bar * n[k];
    ut[k] = ua[k] - un * n[k];
  }
  double vm[NS], vp[NS];
  entropyvars<LAW, DIM>(L, qm, am, vm);
  entropyvars<LAW, DIM>(L, qp, ap, vp);
  double dv64[NS];
  float dv[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    dv64[s] = vp[s] - vm[s];
    dv[s] = (float)dv64[s];
  }
  const float l1 = fabsf(un - c_bar) * rho_log / (2.f * g);
  const float l2 = fabsf(un) * rho_log * (g - 1.f) / g;
  const float l3 = fabsf(un + c_bar) * rho_log / (2.f * g);
  const float l4 = fabsf(un) * p_avg;
  float k2 = u2_bar / 2.f;
  if (LAW == LAW_EG) k2 += Phi_avg;
  // the three projections of the entropy-variable jump cancel to a few
  // times their terms' size (the enthalpy-like h_bar times the jump of -2b
  // against the jump of the first entropy variable): summed in FP64
  auto proj = [&](const float* a, float hh) {
    double t = dv64[0] + (double)hh * dv64[DIM + 1];
#pragma unroll
    for (int k = 0; k < DIM; ++k) t += (double)a[k] * dv64[1 + k];
    return (float)t;
  };
  const float w1 = l1 * proj(umc, h_bar - c_bar * un);
  const float w2 = l2 * proj(ua, k2);
  const float w3 = l3 * proj(upc, h_bar + c_bar * un);
  const float ndv = dot<DIM>(n, dv + 1);
  Dm[0] = w1 + w2 + w3;
#pragma unroll
  for (int k = 0; k < DIM; ++k)
    Dm[1 + k] = w1 * umc[k] + w2 * ua[k] + w3 * upc[k] + l4 * (dv[1 + k] - ndv * n[k] + dv[DIM + 1] * ut[k]);
  Dm[DIM + 1] = w1 * (h_bar - c_bar * un) + w2 * k2 + w3 * (h_bar + c_bar * un) +
                l4 * (dot<DIM>(ut, dv + 1) + dv[DIM + 1] * (dot<DIM>(ua, ua) - un * un));
}

// Surface fluxes in the FP32-flux form.  Central / Rusanov: the two sides'
// fluxes from flux_ws_recip32, averaged in FP64; the dissipation is the FP64
// jump times an FP32 wave speed.  EC / KG: the volume term's FP32-flux
// two-point fluxes (ec_vol32 / kg_vol32 / sw_vol32) of the two face states.
// Roe: the central part as for Rusanov, the upwind dissipation from
// roe_diss32.  Matrix: the FP32-flux EC flux minus half of matrix_diss32.
template <int LAW, int DIM>
__device__ __forceinline__ bool surface_flux32(const LawP& L, int kind, int d, double sgn, const double* qm,
                                               const double* am, const double* qp, const double* ap, double* nf) {
  constexpr int NS = NSt<LAW, DIM>::v;
  if constexpr (LAW == LAW_EULER || LAW == LAW_EG) {
    if (kind == F_EC || kind == F_KG || kind == F_MATRIX) {
      const double Phim = (LAW == LAW_EG) ? am[0] : 0.0, Phip = (LAW == LAW_EG) ? ap[0] : 0.0;
      double pm, pp, bm, bp;
      float um[DIM], up[DIM], uum, uup, em, ep;
      pre32<DIM>(L.gamma, qm, Phim, &pm, &bm, um, &uum, &em);
      pre32<DIM>(L.gamma, qp, Phip, &pp, &bp, up, &uup, &ep);
      double f[NS + 1];
      if (kind == F_KG) {
        kg_vol32<DIM>(d, qm[0], pm, um, em, qp[0], pp, up, ep, f);
      } else {
        ec_vol32<LAW, DIM>((float)(1.0 / (L.gamma - 1.0)), d, qm[0], pm, bm, um, uum, Phim, qp[0], pp, bp, up,
                           uup, Phip, f, f + NS);
      }
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = f[s] * sgn;
      if (kind == F_MATRIX) {
        float Dm[NS];
        matrix_diss32<LAW, DIM>(L, d, sgn, qm, am, qp, ap, bm, bp, um, uum, up, uup, Dm);
#pragma unroll
        for (int s = 0; s < NS; ++s) nf[s] = nf[s] - (double)(Dm[s] / 2.f);
      }
      return true;
    }
  }
  if constexpr (LAW == LAW_SW) {
    if (kind == F_EC) {
      float Pm[DIM + 1], Pp[DIM + 1];
      const float him = 1.f / (float)qm[0], hip = 1.f / (float)qp[0];
#pragma unroll
      for (int c = 0; c < DIM; ++c) { Pm[c] = (float)qm[1 + c] * him; Pp[c] = (float)qp[1 + c] * hip; }
      Pm[DIM] = (float)qm[DIM + 1] * him;
      Pp[DIM] = (float)qp[DIM + 1] * hip;
      double f[NS];
      sw_vol32<DIM>(L.grav, d, qm, Pm, qp, Pp, f);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = f[s] * sgn;
      if (L.swtopo) {  // non-conservative surface term g h- (b+ - b-)/2 n, FP64 (balance)
        const double t = L.grav * qm[0] * (ap[0] - am[0]) / 2.0;
        nf[1 + d] = nf[1 + d] + t * sgn;
      }
      return true;
    }
  }
  if constexpr (LAW == LAW_EULER || LAW == LAW_EG || LAW == LAW_SW) {
    if (kind == F_ROE) {
      double fm[NS], fp[NS];
      flux_ws_recip32<LAW, DIM>(L, d, qm, am, fm);
      flux_ws_recip32<LAW, DIM>(L, d, qp, ap, fp);
      float fpv[NS];
      roe_diss32<LAW, DIM>(L, d, sgn, qm, am, qp, fpv);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = ((fm[s] + fp[s]) * sgn) / 2.0 - (double)fpv[s];
      if constexpr (LAW == LAW_SW) {
        if (L.swtopo) {  // non-conservative surface term g h- (b+ - b-)/2 n, FP64 (balance)
          const double t = L.grav * qm[0] * (ap[0] - am[0]) / 2.0;
          nf[1 + d] = nf[1 + d] + t * sgn;
        }
      }
      return true;
    }
  }
  if constexpr (LAW == LAW_EULER || LAW == LAW_EG || LAW == LAW_SW) {
    if (kind == F_CENTRAL || kind == F_RUSANOV) {
      double fm[NS], fp[NS];
      const double wm = flux_ws_recip32<LAW, DIM>(L, d, qm, am, fm);
      const double wp = flux_ws_recip32<LAW, DIM>(L, d, qp, ap, fp);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = ((fm[s] + fp[s]) / 2.0) * sgn;
      if (kind == F_RUSANOV) {
        const float ws = (float)dmax(wm, wp);
#pragma unroll
        for (int s = 0; s < NS; ++s) nf[s] = nf[s] - (double)(ws * (float)((qp[s] - qm[s]) / 2.0));
      }
      if constexpr (LAW == LAW_SW) {
        if (L.swtopo) {  // non-conservative surface term g h- (b+ - b-)/2 n, FP64 (balance)
          const double t = L.grav * qm[0] * (ap[0] - am[0]) / 2.0;
          nf[1 + d] = nf[1 + d] + t * sgn;
        }
      }
      return true;
    }
  }
  return false;
}

// ------------------------------------------------------------ surface flux
// normal n = sgn * e_d; nf = numerical flux . n (length NS)
template <int LAW, int DIM, class T>
__device__ __forceinline__ void surface_flux(const LawP& L, int kind, int d, T sgn, const T* qm, const T* am,
                                             const T* qp, const T* ap, T* nf) {
  constexpr int NS = NSt<LAW, DIM>::v;
  if constexpr (LAW == LAW_EULER || LAW == LAW_EG || LAW == LAW_SW) {
    if (kind == F_CENTRAL || kind == F_RUSANOV) {
      // src/numericalfluxes.jl:31-42 with one reciprocal per side
      T fm[NS], fp[NS];
      const T wm = flux_ws_recip<LAW, DIM>(L, d, qm, am, fm);
      const T wp = flux_ws_recip<LAW, DIM>(L, d, qp, ap, fp);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = ((fm[s] + fp[s]) / T(2)) * sgn;
      if (kind == F_RUSANOV) {
        const T ws = dmax(wm, wp);
#pragma unroll
        for (int s = 0; s < NS; ++s) nf[s] = nf[s] - ws * (qp[s] - qm[s]) / T(2);
      }
      if constexpr (LAW == LAW_SW) {
        if (L.swtopo) {  // non-conservative surface term g h- (b+ - b-)/2 n
          const T t = T(L.grav) * qm[0] * (ap[0] - am[0]) / T(2);
          nf[1 + d] = nf[1 + d] + t * sgn;
        }
      }
      return;
    }
  }
  if (kind == F_CENTRAL || kind == F_RUSANOV) {
    T fm[NS], fp[NS];
    flux_dir<LAW, DIM>(L, d, qm, am, fm);
    flux_dir<LAW, DIM>(L, d, qp, ap, fp);
#pragma unroll
    for (int s = 0; s < NS; ++s) nf[s] = ((fm[s] + fp[s]) / T(2)) * sgn;
    if (kind == F_RUSANOV) {
      T ws = dmax(wavespeed_dir<LAW, DIM>(L, d, qm, am), wavespeed_dir<LAW, DIM>(L, d, qp, ap));
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = nf[s] - ws * (qp[s] - qm[s]) / T(2);
    }
  } else if constexpr (LAW == LAW_EULER || LAW == LAW_EG) {
    const T g = T(L.gamma);
    if (kind == F_EC || kind == F_KG) {
      T Pm[NPreE<DIM>::v], Pp[NPreE<DIM>::v];
      T Phim = (LAW == LAW_EG) ? am[0] : T(0), Phip = (LAW == LAW_EG) ? ap[0] : T(0);
      precompute_euler<DIM>(g, qm, Phim, Pm);
      precompute_euler<DIM>(g, qp, Phip, Pp);
      T f[NS];
      if (kind == F_EC)
        ec_dir<LAW, DIM>(g, d, qm[0], Pm, Phim, qp[0], Pp, Phip, f);
      else
        kg_dir<LAW, DIM>(d, qm[0], Pm, Phim, qp[0], Pp, Phip, f);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = f[s] * sgn;
    } else if (kind == F_ROE) {
      T Phi = (LAW == LAW_EG) ? am[0] : T(0);
      T n[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) n[c] = (c == d) ? sgn : T(0);
      T fm[NS], fp[NS];
      flux_dir<LAW, DIM>(L, d, qm, am, fm);
      flux_dir<LAW, DIM>(L, d, qp, ap, fp);
      T rm = qm[0], rp = qp[0];
      T um[DIM], up[DIM], u[DIM], du[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) { um[c] = qm[1 + c] / rm; up[c] = qp[1 + c] / rp; }
      T pm = pressure_eg<DIM>(g, qm, Phi), pp = pressure_eg<DIM>(g, qp, Phi);
      T hm = qm[DIM + 1] / rm + pm / rm, hp = qp[DIM + 1] / rp + pp / rp;
      T cm = dsqrt(g * pm / rm), cp = dsqrt(g * pp / rp);
      T srm = dsqrt(rm), srp = dsqrt(rp);
      T rho = dsqrt(rm * rp);
#pragma unroll
      for (int c = 0; c < DIM; ++c) { u[c] = roe_avg(srm, srp, um[c], up[c]); du[c] = up[c] - um[c]; }
      T h = roe_avg(srm, srp, hm, hp);
      T c = roe_avg(srm, srp, cm, cp);
      T un = dot<DIM>(u, n);
      T drho = rp - rm, dp = pp - pm;
      T dun = dot<DIM>(du, n);
      T cm2 = T(1) / (c * c);
      T w1 = fabs(un - c) * (dp - rho * c * dun) * cm2 / T(2);
      T w2 = fabs(un + c) * (dp + rho * c * dun) * cm2 / T(2);
      T w3 = fabs(un) * (drho - dp * cm2);
      T w4 = fabs(un) * rho;
      T fpv[NS];
      fpv[0] = (w1 + w2 + w3) / T(2);
#pragma unroll
      for (int k = 0; k < DIM; ++k)
        fpv[1 + k] = (w1 * (u[k] - c * n[k]) + w2 * (u[k] + c * n[k]) + w3 * u[k] + w4 * (du[k] - dun * n[k])) / T(2);
      T ke = (LAW == LAW_EG) ? w3 * (dot<DIM>(u, u) / T(2) + Phi) : w3 * dot<DIM>(u, u) / T(2);
      fpv[DIM + 1] = (w1 * (h - c * un) + w2 * (h + c * un) + ke + w4 * (dot<DIM>(u, du) - un * dun)) / T(2);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = ((fm[s] + fp[s]) * sgn) / T(2) - fpv[s];
    } else {  // matrix dissipation
      T n[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) n[c] = (c == d) ? sgn : T(0);
      T Phim = (LAW == LAW_EG) ? am[0] : T(0), Phip = (LAW == LAW_EG) ? ap[0] : T(0);
      T Pm[NPreE<DIM>::v], Pp[NPreE<DIM>::v];
      precompute_euler<DIM>(g, qm, Phim, Pm);
      precompute_euler<DIM>(g, qp, Phip, Pp);
      T ec[NS];
      ec_dir<LAW, DIM>(g, d, qm[0], Pm, Phim, qp[0], Pp, Phip, ec);
      T rm = qm[0], rp = qp[0];
      T bm = Pm[DIM + 1], bp = Pp[DIM + 1];
      T Phi_avg = (Phim + Phip) / T(2);
      T rho_log = logavg(rm, rp);
      T b_log = logavg(bm, bp);
      T ua[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) ua[c] = (Pm[c] + Pp[c]) / T(2);
      T p_avg = ((rm + rp) / T(2)) / (T(2) * ((bm + bp) / T(2)));
      T u2_bar = T(2) * dsqrt(dot<DIM>(ua, ua)) - (dsqrt(Pm[DIM + 2]) + dsqrt(Pp[DIM + 2])) / T(2);
      T h_bar = g / (T(2) * b_log * (g - T(1))) + u2_bar / T(2);
      if (LAW == LAW_EG) h_bar = h_bar + Phi_avg;
      T c_bar = dsqrt(g * p_avg / rho_log);
      T umc[DIM], upc[DIM], ut[DIM];
      T un = dot<DIM>(ua, n);
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        umc[k] = ua[k] - c_bar * n[k];
        upc[k] = ua[k] + c_bar * n[k];
        ut[k] = ua[k] - un * n[k];
      }
      T vm[NS], vp[NS], dv[NS];
      entropyvars<LAW, DIM>(L, qm, am, vm);
      entropyvars<LAW, DIM>(L, qp, ap, vp);
#pragma unroll
      for (int s = 0; s < NS; ++s) dv[s] = vp[s] - vm[s];
      T l1 = fabs(un - c_bar) * rho_log / (T(2) * g);
      T l2 = fabs(un) * rho_log * (g - T(1)) / g;
      T l3 = fabs(un + c_bar) * rho_log / (T(2) * g);
      T l4 = fabs(un) * p_avg;
      T k2 = u2_bar / T(2);
      if (LAW == LAW_EG) k2 = k2 + Phi_avg;
      T w1 = l1 * (dv[0] + dot<DIM>(umc, dv + 1) + (h_bar - c_bar * un) * dv[DIM + 1]);
      T w2 = l2 * (dv[0] + dot<DIM>(ua, dv + 1) + k2 * dv[DIM + 1]);
      T w3 = l3 * (dv[0] + dot<DIM>(upc, dv + 1) + (h_bar + c_bar * un) * dv[DIM + 1]);
      T ndv = dot<DIM>(n, dv + 1);
      T Dm[NS];
      Dm[0] = w1 + w2 + w3;
#pragma unroll
      for (int k = 0; k < DIM; ++k)
        Dm[1 + k] = w1 * umc[k] + w2 * ua[k] + w3 * upc[k] + l4 * (dv[1 + k] - ndv * n[k] + dv[DIM + 1] * ut[k]);
      Dm[DIM + 1] = w1 * (h_bar - c_bar * un) + w2 * k2 + w3 * (h_bar + c_bar * un) +
                    l4 * (dot<DIM>(ut, dv + 1) + dv[DIM + 1] * (dot<DIM>(ua, ua) - un * un));
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = ec[s] * sgn - Dm[s] / T(2);
    }
  } else if constexpr (LAW == LAW_SW) {
    const T gg = T(L.grav);
    if (kind == F_EC) {
      T Pm[DIM + 1], Pp[DIM + 1];
#pragma unroll
      for (int c = 0; c < DIM; ++c) { Pm[c] = qm[1 + c] / qm[0]; Pp[c] = qp[1 + c] / qp[0]; }
      Pm[DIM] = qm[DIM + 1] / qm[0];
      Pp[DIM] = qp[DIM + 1] / qp[0];
      T f[NS];
      sw_ec_dir<DIM>(gg, 0, d, qm, Pm, T(0), qp, Pp, T(0), f);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = f[s] * sgn;
    } else {  // Roe
      T n[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) n[c] = (c == d) ? sgn : T(0);
      T fm[NS], fp[NS];
      flux_dir<LAW, DIM>(L, d, qm, am, fm);
      flux_dir<LAW, DIM>(L, d, qp, ap, fp);
      T rm = qm[0], rp = qp[0];
      T um[DIM], up[DIM], u[DIM], du[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) { um[c] = qm[1 + c] / rm; up[c] = qp[1 + c] / rp; }
      T thm = qm[DIM + 1] / rm, thp = qp[DIM + 1] / rp;
      T pm = gg * (rm * rm) / T(2), pp = gg * (rp * rp) / T(2);
      T cm = dsqrt(gg * rm), cp = dsqrt(gg * rp);
      T srm = dsqrt(rm), srp = dsqrt(rp);
      T rho = dsqrt(rm * rp);
#pragma unroll
      for (int c = 0; c < DIM; ++c) { u[c] = roe_avg(srm, srp, um[c], up[c]); du[c] = up[c] - um[c]; }
      T th = roe_avg(srm, srp, thm, thp);
      T c = roe_avg(srm, srp, cm, cp);
      T un = dot<DIM>(u, n);
      T drho = rp - rm, dp = pp - pm, dth = qp[DIM + 1] - qm[DIM + 1];
      T dun = dot<DIM>(du, n);
      T cm2 = T(1) / (c * c);
      T w1 = fabs(un - c) * (dp - rho * c * dun) * cm2 / T(2);
      T w2 = fabs(un + c) * (dp + rho * c * dun) * cm2 / T(2);
      T w3 = fabs(un) * (drho - dp * cm2);
      T w4 = fabs(un) * rho;
      T w5 = fabs(un) * (dth - th * dp * cm2);
      T fpv[NS];
      fpv[0] = (w1 + w2 + w3) / T(2);
#pragma unroll
      for (int k = 0; k < DIM; ++k)
        fpv[1 + k] = (w1 * (u[k] - c * n[k]) + w2 * (u[k] + c * n[k]) + w3 * u[k] + w4 * (du[k] - dun * n[k])) / T(2);
      fpv[DIM + 1] = ((w1 + w2) * th + w5) / T(2);
#pragma unroll
      for (int s = 0; s < NS; ++s) nf[s] = ((fm[s] + fp[s]) * sgn) / T(2) - fpv[s];
    }
  }
  if constexpr (LAW == LAW_SW) {
    if (L.swtopo) {  // non-conservative surface term g h- (b+ - b-)/2 n
      T t = T(L.grav) * qm[0] * (ap[0] - am[0]) / T(2);
      nf[1 + d] = nf[1 + d] + t * sgn;
    }
  }
}

// ---------------------------------------------------------------- sources
// law source! (linear_euler_gravity.jl:58-65), problem source! (Coriolis,
// experiment/euler_gravity/baroclinicwave.jl:27-34) and, in the weak form,
// nonconservative_term! (euler_gravity.jl:100-113; SW bathymetry extension).
template <int LAW, int DIM, class T>
__device__ __forceinline__ void add_sources(const LawP& L, bool weak, const T* q, const T* aux, T* dq) {
  if constexpr (LAW == LAW_LEG) {
#pragma unroll
    for (int k = 0; k < DIM; ++k) dq[1 + k] = dq[1 + k] - q[0] * aux[1 + k];
  }
  if constexpr (LAW != LAW_ADV) {
    if (L.src == SRC_CORIOLIS) {
      if constexpr (DIM == 3) {
        const T* m = q + 1;
        T ox = T(L.omega[0]), oy = T(L.omega[1]), oz = T(L.omega[2]);
        dq[1] = dq[1] - (oy * m[2] - oz * m[1]);
        dq[2] = dq[2] - (oz * m[0] - ox * m[2]);
        dq[3] = dq[3] - (ox * m[1] - oy * m[0]);
      } else if constexpr (DIM == 2) {  // f-plane, omega = (0, 0, f)
        T f = T(L.omega[2]);
        dq[1] = dq[1] - (-(f * q[2]));
        dq[2] = dq[2] - f * q[1];
      }
    }
  }
  if (weak) {
    if constexpr (LAW == LAW_EG) {
      T rho = q[0];
      if (L.pde) rho = rho - aux[DIM + 1];
#pragma unroll
      for (int k = 0; k < DIM; ++k) dq[1 + k] = dq[1 + k] - rho * aux[1 + k];
    }
    if constexpr (LAW == LAW_SW) {
      if (L.swtopo) {
        T gh = T(L.grav) * q[0];
#pragma unroll
        for (int k = 0; k < DIM; ++k) dq[1 + k] = dq[1 + k] - gh * aux[1 + k];
      }
    }
  }
}

}  // namespace atb
