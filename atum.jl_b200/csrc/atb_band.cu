// Batched vertical banded solve for the IMEX implicit stage (the solve of
// I - dt a_ii L_vert, src/odesolvers.jl:351-356), fast path for a factor
// shared by every vertical column.
//
// Structure: the unknowns of a vertical line, ordered (element, node, state),
// give a band of half-width bw = Nq*ns - 1 = BW1 - 1, so row i of element ev
// couples only to the BW1 unknowns of elements ev-1, ev (forward) or ev, ev+1
// (backward).  One thread owns one line; its window of solution values is two
// register arrays (previous / current element) with every index known at
// compile time, so the inner products are fully unrolled FMAs with no local
// memory.  The factor block of one element (BW1 rows x 2*BW1 padded columns,
// 16*BW1^2 bytes) is the same for all lines of the CTA: it is staged into
// shared memory with cp.async, double-buffered so the copy of element ev+1
// overlaps the arithmetic of element ev, and read back as warp broadcasts.
// The ARK right-hand side q + dt sum_k (a_k ex_k + b_k im_k) is formed on the
// fly as each row is reached (src/odesolvers.jl:346-349), so Qhat never
// exists in memory.
#include "atb_generic.cuh"

namespace atb {

void launch_band_solve_generic(const BandSolve& B, cudaStream_t st);

namespace {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int BLK, int LPB>
__device__ __forceinline__ void stage_block(double* dst, const double* src) {
  // BLK doubles, 16-byte chunks spread over the CTA's threads
#pragma unroll 4
  for (int c = threadIdx.x; c < BLK / 2; c += LPB) cp_async16(dst + 2 * c, src + 2 * c);
}

template <int NQ, int NS, int LPB>
__global__ void __launch_bounds__(LPB) band_solve_shared_kernel(const BandSolve B) {
  constexpr int BW1 = NQ * NS;
  constexpr int BW = BW1 - 1;
  constexpr int WP = 2 * BW1;  // padded row stride (2*bw + 1 entries + 1 pad)
  constexpr int BLK = BW1 * WP;
  extern __shared__ __align__(16) double sband[];
  auto sbuf = [&](int b) { return sband + b * BLK; };
  const LineMap& M = B.M;
  const int line = blockIdx.x * LPB + threadIdx.x;
  const bool act = line < M.nlines;
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  const int hn = act ? line % nh : 0;
  const int e0 = act ? M.e0[line] : 0;
  const double* __restrict__ band = B.band;
  const int npairs = B.npairs;

  // ------------------------------------------------------------ forward
  stage_block<BLK, LPB>(sbuf(0), band);
  cp_async_commit();
  if (KV > 1) stage_block<BLK, LPB>(sbuf(1), band + BLK);
  cp_async_commit();
  double prev[BW1], cur[BW1];
#pragma unroll
  for (int j = 0; j < BW1; ++j) prev[j] = 0.0;
  for (int ev = 0; ev < KV; ++ev) {
    cp_async_wait1();
    __syncthreads();
    const double* Lb = sbuf(ev & 1);
    if (act) {
      const size_t eoff = (size_t)(e0 + ev * M.estep) * Np + hn;
#pragma unroll
      for (int i = 0; i < BW1; ++i) {
        const int s = i % NS, kv = i / NS;
        const size_t g = eoff + (size_t)nh * kv;
        double acc = B.q[s][g];
#pragma unroll
        for (int k = 0; k < 2; ++k)
          if (k < npairs) acc = acc + B.dt * (B.a[k] * B.ex[k][s][g] + B.b[k] * B.im[k][s][g]);
        const double* row = Lb + i * WP;
#pragma unroll
        for (int j = i + 1; j < BW1; ++j) acc = acc - row[j - i - 1] * prev[j];
#pragma unroll
        for (int j = 0; j < i; ++j) acc = acc - row[j - i + BW] * cur[j];
        cur[i] = acc;
        B.out[s][g] = acc;
      }
#pragma unroll
      for (int j = 0; j < BW1; ++j) prev[j] = cur[j];
    }
    __syncthreads();
    if (ev + 2 < KV) stage_block<BLK, LPB>(sbuf(ev & 1), band + (size_t)(ev + 2) * BLK);
    cp_async_commit();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();

  // ----------------------------------------------------------- backward
  stage_block<BLK, LPB>(sbuf(0), band + (size_t)(KV - 1) * BLK);
  cp_async_commit();
  if (KV > 1) stage_block<BLK, LPB>(sbuf(1), band + (size_t)(KV - 2) * BLK);
  cp_async_commit();
  double nxt[BW1];
#pragma unroll
  for (int j = 0; j < BW1; ++j) nxt[j] = 0.0;
  for (int t = 0; t < KV; ++t) {
    const int ev = KV - 1 - t;
    cp_async_wait1();
    __syncthreads();
    const double* Ub = sbuf(t & 1);
    if (act) {
      const size_t eoff = (size_t)(e0 + ev * M.estep) * Np + hn;
#pragma unroll
      for (int i = BW1 - 1; i >= 0; --i) {
        const int s = i % NS, kv = i / NS;
        const size_t g = eoff + (size_t)nh * kv;
        double acc = B.out[s][g];
        const double* row = Ub + i * WP;
#pragma unroll
        for (int j = i + 1; j < BW1; ++j) acc = acc - row[j - i + BW] * cur[j];
#pragma unroll
        for (int j = 0; j < i; ++j) acc = acc - row[2 * BW1 - 1 + j - i] * nxt[j];
        const double x = acc / row[BW];
        cur[i] = x;
        B.out[s][g] = x;
      }
#pragma unroll
      for (int j = 0; j < BW1; ++j) nxt[j] = cur[j];
    }
    __syncthreads();
    if (ev - 2 >= 0) stage_block<BLK, LPB>(sbuf(t & 1), band + (size_t)(ev - 2) * BLK);
    cp_async_commit();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ------------------------------------------------- block-parallel form
// From the shared LU factor, per element block e (BW1 x BW1):
//   Li_e = L_ee^-1,  G_e = L_ee^-1 L_e,e-1,  Ui_e = U_ee^-1,  H_e = U_ee^-1 U_e,e+1
// so that   y_e = Li_e b_e - G_e y_e-1,   x_e = Ui_e y_e - H_e x_e+1.
// Each of the BW1 rows of a block is then an independent pair of length-BW1
// dot products: the solve runs one thread per (row, line) instead of one per
// line, with only the element recurrence left sequential.
// Layout: blk[e][4][BW1][BW1] = Li, G, Ui, H (row-major).
__global__ void block_prep_kernel(const double* band, int KV, int BW1, double* blk) {
  // one CTA per element, one thread per column of the inverses
  const int e = blockIdx.x, c = threadIdx.x;
  const int bw = BW1 - 1, rs = 2 * BW1;
  auto F = [&](int i, int j) -> double {  // factor entry (i, j) of the line
    const int off = j - i + bw;
    return (off < 0 || off > 2 * bw) ? 0.0 : band[(size_t)i * rs + off];
  };
  double* Li = blk + (size_t)e * 4 * BW1 * BW1;
  double* G = Li + BW1 * BW1;
  double* Ui = G + BW1 * BW1;
  double* H = Ui + BW1 * BW1;
  const int r0 = e * BW1;
  if (c < BW1) {
    // column c of L_ee^-1 (unit lower triangular): forward substitution
    for (int i = 0; i < BW1; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) v -= F(r0 + i, r0 + k) * Li[k * BW1 + c];
      Li[i * BW1 + c] = v;
    }
    // column c of U_ee^-1: back substitution
    for (int i = BW1 - 1; i >= 0; --i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = i + 1; k < BW1; ++k) v -= F(r0 + i, r0 + k) * Ui[k * BW1 + c];
      Ui[i * BW1 + c] = v / F(r0 + i, r0 + i);
    }
  }
  __syncthreads();
  if (c < BW1) {
    // G = Li * L_e,e-1 ; H = Ui * U_e,e+1 (column c)
    for (int i = 0; i < BW1; ++i) {
      double g = 0.0, h = 0.0;
      for (int k = 0; k < BW1; ++k) {
        if (e > 0) g += Li[i * BW1 + k] * F(r0 + k, r0 - BW1 + c);
        if (e < KV - 1) h += Ui[i * BW1 + k] * F(r0 + k, r0 + BW1 + c);
      }
      G[i * BW1 + c] = g;
      H[i * BW1 + c] = h;
    }
  }
}

// One thread per (node kv of the element column, line l): it owns the NS rows
// kv*NS .. kv*NS+NS-1 of every element block of its line.  Per element it
// reads the line's right-hand-side / previous-solution vectors (2*BW1 values,
// shared by its NS rows) and its NS rows of the two matrices (warp-uniform
// addresses -> broadcasts, two doubles per load), and issues NS*2*BW1 FMAs.
// Warps hold 32 lines at the same kv, so the global accesses of a state
// component are consecutive addresses.
template <int NQ, int NS, int LPB>
__global__ void __launch_bounds__(NQ * LPB) band_solve_block_kernel(const BandSolve B, const double* blk) {
  constexpr int BW1 = NQ * NS;
  constexpr int MAT = BW1 * BW1;
  extern __shared__ __align__(16) double sm[];
  // smat(b): [Li|G] or [Ui|H], double-buffered (arithmetic, not a pointer
  // array: a runtime-indexed local array would live in local memory)
  auto smat = [&](int b) { return sm + b * 2 * MAT; };
  double* ys = sm + 4 * MAT;             // [2][BW1][LPB]
  double* bs = ys + 2 * BW1 * LPB;       // [BW1][LPB]
  const LineMap& M = B.M;
  const int l = threadIdx.x % LPB, kv = threadIdx.x / LPB;
  const int line = blockIdx.x * LPB + l;
  const bool act = line < M.nlines;
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  const int hn = act ? line % nh : 0;
  const int e0 = act ? M.e0[line] : 0;
  const int nthr = NQ * LPB;
  auto stage = [&](double* dst, const double* src) {
    for (int c = threadIdx.x; c < MAT; c += nthr) cp_async16(dst + 2 * c, src + 2 * c);  // 2*MAT doubles
  };
  auto gidx = [&](int ev) { return (size_t)(e0 + ev * M.estep) * Np + hn + (size_t)nh * kv; };
  // y_e = A_e v_e - C_e w_e-1 for this thread's NS rows (A, C row-major BW1 x BW1)
  auto block_rows = [&](const double* Am, const double* Cm, const double* v, const double* w, double* out) {
#pragma unroll
    for (int s = 0; s < NS; ++s) out[s] = 0.0;
    double acc2[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) acc2[s] = 0.0;
#pragma unroll
    for (int k = 0; k < BW1; ++k) {
      const double vk = v[k * LPB + l], wk = w[k * LPB + l];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int row = kv * NS + s;
        out[s] += Am[row * BW1 + k] * vk;
        acc2[s] += Cm[row * BW1 + k] * wk;
      }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) out[s] -= acc2[s];
  };
  // ------------------------------------------------------------ forward
  stage(smat(0), blk);
  cp_async_commit();
  if (KV > 1) stage(smat(1), blk + (size_t)4 * MAT);
  cp_async_commit();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    ys[(kv * NS + s) * LPB + l] = 0.0;  // y_{-1} = 0
    ys[BW1 * LPB + (kv * NS + s) * LPB + l] = 0.0;
  }
  double bnext[NS];
  auto rhs = [&](int ev, double* b) {
    const size_t g = gidx(ev);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      double v = 0.0;
      if (act) {
        v = B.q[s][g];
        // static pair index: the kernel-parameter pointer tables stay in the
        // constant bank instead of being copied to local memory
#pragma unroll
        for (int k = 0; k < 2; ++k)
          if (k < B.npairs) v = v + B.dt * (B.a[k] * B.ex[k][s][g] + B.b[k] * B.im[k][s][g]);
      }
      b[s] = v;
    }
  };
  rhs(0, bnext);
  for (int ev = 0; ev < KV; ++ev) {
#pragma unroll
    for (int s = 0; s < NS; ++s) bs[(kv * NS + s) * LPB + l] = bnext[s];
    if (ev + 1 < KV) rhs(ev + 1, bnext);
    cp_async_wait1();
    __syncthreads();
    double y[NS];
    block_rows(smat(ev & 1), smat(ev & 1) + MAT, bs, ys + ((ev + 1) & 1) * BW1 * LPB, y);
    const size_t g = gidx(ev);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      ys[(ev & 1) * BW1 * LPB + (kv * NS + s) * LPB + l] = y[s];
      if (act) B.out[s][g] = y[s];
    }
    __syncthreads();
    if (ev + 2 < KV) stage(smat(ev & 1), blk + (size_t)(ev + 2) * 4 * MAT);
    cp_async_commit();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  // ----------------------------------------------------------- backward
  stage(smat(0), blk + (size_t)(KV - 1) * 4 * MAT + 2 * MAT);
  cp_async_commit();
  if (KV > 1) stage(smat(1), blk + (size_t)(KV - 2) * 4 * MAT + 2 * MAT);
  cp_async_commit();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    ys[(kv * NS + s) * LPB + l] = 0.0;
    ys[BW1 * LPB + (kv * NS + s) * LPB + l] = 0.0;
  }
  double ynext[NS];
  auto yload = [&](int ev, double* yv) {
    const size_t g = gidx(ev);
#pragma unroll
    for (int s = 0; s < NS; ++s) yv[s] = act ? B.out[s][g] : 0.0;
  };
  yload(KV - 1, ynext);
  for (int t = 0; t < KV; ++t) {
    const int ev = KV - 1 - t;
#pragma unroll
    for (int s = 0; s < NS; ++s) bs[(kv * NS + s) * LPB + l] = ynext[s];
    if (ev > 0) yload(ev - 1, ynext);
    cp_async_wait1();
    __syncthreads();
    double x[NS];
    block_rows(smat(t & 1), smat(t & 1) + MAT, bs, ys + ((t + 1) & 1) * BW1 * LPB, x);
    const size_t g = gidx(ev);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      ys[(t & 1) * BW1 * LPB + (kv * NS + s) * LPB + l] = x[s];
      if (act) B.out[s][g] = x[s];
    }
    __syncthreads();
    if (ev - 2 >= 0) stage(smat(t & 1), blk + (size_t)(ev - 2) * 4 * MAT + 2 * MAT);
    cp_async_commit();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

typedef void (*solve_fn)(const BandSolve&, cudaStream_t);

template <int NQ, int NS> void solve_launch(const BandSolve& B, cudaStream_t st) {
  constexpr int LPB = 32;
  constexpr size_t smem = sizeof(double) * 2 * (NQ * NS) * (2 * NQ * NS);
  static bool configured = false;
  if (!configured && smem > 48 * 1024) {
    cudaFuncSetAttribute(band_solve_shared_kernel<NQ, NS, LPB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  }
  configured = true;
  band_solve_shared_kernel<NQ, NS, LPB><<<(B.M.nlines + LPB - 1) / LPB, LPB, smem, st>>>(B);
}

template <int NS> solve_fn pick_nq(int nq) {
  switch (nq) {
    case 2: return solve_launch<2, NS>;
    case 3: return solve_launch<3, NS>;
    case 4: return solve_launch<4, NS>;
    case 5: return solve_launch<5, NS>;
    case 6: return solve_launch<6, NS>;
    case 7: return solve_launch<7, NS>;
    case 8: return solve_launch<8, NS>;
  }
  return nullptr;
}


template <int NQ, int NS> void block_launch(const BandSolve& B, cudaStream_t st) {
  constexpr int BW1 = NQ * NS;
  constexpr int LPB = 32;
  constexpr size_t smem = sizeof(double) * (4 * BW1 * BW1 + 3 * BW1 * LPB);
  static bool configured = false;
  if (!configured && smem > 48 * 1024)
    cudaFuncSetAttribute(band_solve_block_kernel<NQ, NS, LPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  configured = true;
  band_solve_block_kernel<NQ, NS, LPB><<<(B.M.nlines + LPB - 1) / LPB, NQ * LPB, smem, st>>>(B, B.blk);
}

template <int NS> solve_fn pick_block(int nq) {
  switch (nq) {
    case 2: return block_launch<2, NS>;
    case 3: return block_launch<3, NS>;
    case 4: return block_launch<4, NS>;
    case 5: return block_launch<5, NS>;
    case 6: return block_launch<6, NS>;
    case 7: return block_launch<7, NS>;
    case 8: return block_launch<8, NS>;
  }
  return nullptr;
}

}  // namespace

void launch_block_prep(const double* band, int KV, int BW1, double* blk, cudaStream_t st) {
  block_prep_kernel<<<KV, ((BW1 + 31) / 32) * 32, 0, st>>>(band, KV, BW1, blk);
}


// Dispatch: the block-parallel form when the factor is shared and its
// per-element inverses were prepared, else the register-window substitution
// (shared factor), else the generic per-line kernel.
void launch_band_solve(const BandSolve& B, cudaStream_t st) {
  solve_fn f = nullptr;
  if (B.ld == 1 && B.blk) {
    if (B.M.ns == 1) f = pick_block<1>(B.M.Nq);
    if (B.M.ns == 4) f = pick_block<4>(B.M.Nq);
    if (B.M.ns == 5) f = pick_block<5>(B.M.Nq);
  }
  if (!f && B.ld == 1) {
    if (B.M.ns == 1) f = pick_nq<1>(B.M.Nq);
    if (B.M.ns == 4) f = pick_nq<4>(B.M.Nq);
    if (B.M.ns == 5) f = pick_nq<5>(B.M.Nq);
  }
  if (f)
    f(B, st);
  else
    launch_band_solve_generic(B, st);
}

}  // namespace atb
