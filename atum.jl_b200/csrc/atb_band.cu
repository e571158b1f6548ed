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
  double* sbuf[2] = {sband, sband + BLK};
  const LineMap& M = B.M;
  const int line = blockIdx.x * LPB + threadIdx.x;
  const bool act = line < M.nlines;
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  const int hn = act ? line % nh : 0;
  const int e0 = act ? M.e0[line] : 0;
  const double* __restrict__ band = B.band;
  const int npairs = B.npairs;

  // ------------------------------------------------------------ forward
  stage_block<BLK, LPB>(sbuf[0], band);
  cp_async_commit();
  if (KV > 1) stage_block<BLK, LPB>(sbuf[1], band + BLK);
  cp_async_commit();
  double prev[BW1], cur[BW1];
#pragma unroll
  for (int j = 0; j < BW1; ++j) prev[j] = 0.0;
  for (int ev = 0; ev < KV; ++ev) {
    cp_async_wait1();
    __syncthreads();
    const double* Lb = sbuf[ev & 1];
    if (act) {
      const size_t eoff = (size_t)(e0 + ev * M.estep) * Np + hn;
#pragma unroll
      for (int i = 0; i < BW1; ++i) {
        const int s = i % NS, kv = i / NS;
        const size_t g = eoff + (size_t)nh * kv;
        double acc = B.q[s][g];
        for (int k = 0; k < npairs; ++k) acc = acc + B.dt * (B.a[k] * B.ex[k][s][g] + B.b[k] * B.im[k][s][g]);
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
    if (ev + 2 < KV) stage_block<BLK, LPB>(sbuf[ev & 1], band + (size_t)(ev + 2) * BLK);
    cp_async_commit();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();

  // ----------------------------------------------------------- backward
  stage_block<BLK, LPB>(sbuf[0], band + (size_t)(KV - 1) * BLK);
  cp_async_commit();
  if (KV > 1) stage_block<BLK, LPB>(sbuf[1], band + (size_t)(KV - 2) * BLK);
  cp_async_commit();
  double nxt[BW1];
#pragma unroll
  for (int j = 0; j < BW1; ++j) nxt[j] = 0.0;
  for (int t = 0; t < KV; ++t) {
    const int ev = KV - 1 - t;
    cp_async_wait1();
    __syncthreads();
    const double* Ub = sbuf[t & 1];
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
    if (ev - 2 >= 0) stage_block<BLK, LPB>(sbuf[t & 1], band + (size_t)(ev - 2) * BLK);
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

template <int NQ, int NS, int LPB>
__global__ void __launch_bounds__(NQ * NS * LPB) band_solve_block_kernel(const BandSolve B, const double* blk) {
  constexpr int BW1 = NQ * NS;
  constexpr int MAT = BW1 * BW1;
  extern __shared__ __align__(16) double sm[];
  double* smat[2] = {sm, sm + 2 * MAT};          // [Li|G] or [Ui|H], double-buffered
  double* ys = sm + 4 * MAT;                     // [2][BW1][LPB]
  double* bs = ys + 2 * BW1 * LPB;               // [BW1][LPB]
  const LineMap& M = B.M;
  const int l = threadIdx.x % LPB, r = threadIdx.x / LPB;
  const int line = blockIdx.x * LPB + l;
  const bool act = line < M.nlines;
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  const int hn = act ? line % nh : 0;
  const int e0 = act ? M.e0[line] : 0;
  const int s = r % NS, kv = r / NS;
  const int nthr = BW1 * LPB;
  auto stage = [&](double* dst, const double* src) {
    for (int c = threadIdx.x; c < MAT; c += nthr) cp_async16(dst + 2 * c, src + 2 * c);  // 2*MAT doubles
  };
  // ------------------------------------------------------------ forward
  stage(smat[0], blk);
  cp_async_commit();
  if (KV > 1) stage(smat[1], blk + (size_t)4 * MAT);
  cp_async_commit();
  ys[r * LPB + l] = 0.0;  // y_{-1} = 0 (buffer 1 is "previous" for ev = 0)
  ys[BW1 * LPB + r * LPB + l] = 0.0;
  for (int ev = 0; ev < KV; ++ev) {
    const size_t g = (size_t)(e0 + ev * M.estep) * Np + hn + (size_t)nh * kv;
    double b = 0.0;
    if (act) {
      b = B.q[s][g];
      for (int k = 0; k < B.npairs; ++k) b = b + B.dt * (B.a[k] * B.ex[k][s][g] + B.b[k] * B.im[k][s][g]);
    }
    bs[r * LPB + l] = b;
    cp_async_wait1();
    __syncthreads();
    const double* Li = smat[ev & 1] + r * BW1;
    const double* G = Li + MAT;
    const double* yprev = ys + ((ev + 1) & 1) * BW1 * LPB;
    double z0 = 0.0, z1 = 0.0, w0 = 0.0, w1 = 0.0;
#pragma unroll
    for (int k = 0; k < BW1; k += 2) {
      z0 += Li[k] * bs[k * LPB + l];
      w0 += G[k] * yprev[k * LPB + l];
      if (k + 1 < BW1) {
        z1 += Li[k + 1] * bs[(k + 1) * LPB + l];
        w1 += G[k + 1] * yprev[(k + 1) * LPB + l];
      }
    }
    const double y = (z0 + z1) - (w0 + w1);
    ys[(ev & 1) * BW1 * LPB + r * LPB + l] = y;
    if (act) B.out[s][g] = y;
    __syncthreads();
    if (ev + 2 < KV) stage(smat[ev & 1], blk + (size_t)(ev + 2) * 4 * MAT);
    cp_async_commit();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  // ----------------------------------------------------------- backward
  stage(smat[0], blk + (size_t)(KV - 1) * 4 * MAT + 2 * MAT);
  cp_async_commit();
  if (KV > 1) stage(smat[1], blk + (size_t)(KV - 2) * 4 * MAT + 2 * MAT);
  cp_async_commit();
  ys[r * LPB + l] = 0.0;
  ys[BW1 * LPB + r * LPB + l] = 0.0;
  for (int t = 0; t < KV; ++t) {
    const int ev = KV - 1 - t;
    const size_t g = (size_t)(e0 + ev * M.estep) * Np + hn + (size_t)nh * kv;
    bs[r * LPB + l] = act ? B.out[s][g] : 0.0;
    cp_async_wait1();
    __syncthreads();
    const double* Ui = smat[t & 1] + r * BW1;
    const double* H = Ui + MAT;
    const double* xnext = ys + ((t + 1) & 1) * BW1 * LPB;
    double z0 = 0.0, z1 = 0.0, w0 = 0.0, w1 = 0.0;
#pragma unroll
    for (int k = 0; k < BW1; k += 2) {
      z0 += Ui[k] * bs[k * LPB + l];
      w0 += H[k] * xnext[k * LPB + l];
      if (k + 1 < BW1) {
        z1 += Ui[k + 1] * bs[(k + 1) * LPB + l];
        w1 += H[k + 1] * xnext[(k + 1) * LPB + l];
      }
    }
    const double x = (z0 + z1) - (w0 + w1);
    ys[(t & 1) * BW1 * LPB + r * LPB + l] = x;
    __syncthreads();  // every row has read its y before any row overwrites it
    if (act) B.out[s][g] = x;
    if (ev - 2 >= 0) stage(smat[t & 1], blk + (size_t)(ev - 2) * 4 * MAT + 2 * MAT);
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
  constexpr int LPB = (BW1 >= 20) ? 8 : 32;
  constexpr size_t smem = sizeof(double) * (4 * BW1 * BW1 + 3 * BW1 * LPB);
  static bool configured = false;
  if (!configured && smem > 48 * 1024)
    cudaFuncSetAttribute(band_solve_block_kernel<NQ, NS, LPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  configured = true;
  band_solve_block_kernel<NQ, NS, LPB><<<(B.M.nlines + LPB - 1) / LPB, BW1 * LPB, smem, st>>>(B, B.blk);
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
