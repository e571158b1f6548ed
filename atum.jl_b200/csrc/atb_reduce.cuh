// Deterministic FP64 reductions for the measures (src/measures.jl:6-33) and
// the relaxation-RK entropy terms (src/odesolvers.jl:108,116,125,129).
//
// Pass 1: each CTA (a grid-stride loop over nodes) reduces into NOUT partial
// values with a fixed-shape shared-memory tree and writes them to
// partials[blockIdx.x * NOUT + k].  Pass 2 (one CTA) sums the partials in a
// fixed order with Neumaier compensation.  The result does not depend on
// timing, so repeated calls are bitwise identical.
#pragma once
#include "atb_physics.cuh"

namespace atb {

enum { RED_L2 = 0, RED_LINF = 1, RED_ENTROPY = 2, RED_ENTPROD = 3, RED_NONFINITE = 4 };

struct RedArgs {
  int K, Nq, Np, naux, kind;
  const double* w;    // Nq LGL weights
  const double* J;    // K element Jacobians
  const double* aux;  // naux * stride
  LawP law;
  size_t stride;
  const double* p[5];  // state (first argument)
  const double* q[5];  // second argument (entropyproduct)
  double* partials;    // gridDim.x * 5
  const double* MJ;    // per-node M J (curved elements), or null
};

constexpr int RED_THREADS = 256;

__device__ __forceinline__ double node_mass(const RedArgs& R, int dim, size_t i) {
  if (R.MJ) return R.MJ[i];
  const int e = (int)(i / R.Np), n = (int)(i - (size_t)e * R.Np), Nq = R.Nq;
  double w = R.w[n % Nq];
  if (dim > 1) w = w * R.w[(n / Nq) % Nq];
  if (dim > 2) w = w * R.w[n / (Nq * Nq)];
  return w * R.J[e];
}

template <int LAW, int DIM>
__global__ void __launch_bounds__(RED_THREADS) reduce_kernel(const RedArgs R) {
  constexpr int NS = NSt<LAW, DIM>::v;
  __shared__ double red[5][RED_THREADS];
  double acc[5] = {0, 0, 0, 0, 0};
  const size_t n = R.stride;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double qp[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qp[s] = R.p[s][i];
    if (R.kind == RED_L2) {
      const double mj = node_mass(R, DIM, i);
#pragma unroll
      for (int s = 0; s < NS; ++s) acc[s] += mj * (qp[s] * qp[s]);
    } else if (R.kind == RED_LINF) {
#pragma unroll
      for (int s = 0; s < NS; ++s) acc[s] = fmax(acc[s], fabs(qp[s]));
    } else if (R.kind == RED_NONFINITE) {
#pragma unroll
      for (int s = 0; s < NS; ++s) acc[0] += isfinite(qp[s]) ? 0.0 : 1.0;
    } else {
      double an[8];
      for (int k = 0; k < R.naux && k < 8; ++k) an[k] = R.aux[k * n + i];
      const double mj = node_mass(R, DIM, i);
      if (R.kind == RED_ENTROPY) {
        acc[0] += mj * entropy_fn<LAW, DIM>(R.law, qp, an);
      } else {
        double v[NS];
        entropyvars<LAW, DIM>(R.law, qp, an, v);
        double d = v[0] * R.q[0][i];
#pragma unroll
        for (int s = 1; s < NS; ++s) d = d + v[s] * R.q[s][i];
        acc[0] += mj * d;
      }
    }
  }
  for (int k = 0; k < 5; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int h = RED_THREADS / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      for (int k = 0; k < 5; ++k) {
        double a = red[k][threadIdx.x], b = red[k][threadIdx.x + h];
        red[k][threadIdx.x] = (R.kind == RED_LINF) ? fmax(a, b) : a + b;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < 5) R.partials[blockIdx.x * 5 + threadIdx.x] = red[threadIdx.x][0];
}

typedef void (*red_launch_fn)(const RedArgs& R, int grid, cudaStream_t st);

template <int LAW, int DIM> void red_launch(const RedArgs& R, int grid, cudaStream_t st) {
  reduce_kernel<LAW, DIM><<<grid, RED_THREADS, 0, st>>>(R);
}

template <int LAW> red_launch_fn pick_reducer(int dim);

}  // namespace atb
