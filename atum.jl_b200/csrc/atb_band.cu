// Batched vertical banded solve for the IMEX implicit stage (the solve of
// I - dt a_ii L_vert, src/odesolvers.jl:351-356), fast paths for a factor
// shared by every vertical column.
//
// Structure: the unknowns of a vertical line, ordered (element, node, state),
// give a band of half-width bw = Nq*ns - 1 = BW1 - 1, so row i of element ev
// couples only to the BW1 unknowns of elements ev-1, ev (forward) or ev, ev+1
// (backward).  The ARK right-hand side q + dt sum_k (a_k ex_k + b_k im_k) is
// formed on the fly as each row is reached (src/odesolvers.jl:346-349), so
// Qhat never exists in memory.  Kernels, in the order launch_band_solve
// prefers them:
//   band_solve_warp_kernel   block recurrence on the FP64 matrix unit, one
//                            warp per 8 lines, nonzero tiles only (ARK stages
//                            whose right-hand side is given whole)
//   band_solve_mma_kernel    the same over dense blocks, one warp per 8 rows
//   band_solve_rows_kernel   one-state laws
//   band_solve_shared_kernel substitution over the shared factor (below)
// and launch_band_solve_generic (atb_generic.cu) for a factor per line.
//
// band_solve_shared_kernel: one thread owns one line; its window of solution
// values is two register arrays (previous / current element) with every index
// known at compile time, so the inner products are fully unrolled FMAs with no
// local memory.  The factor block of one element (BW1 rows x 2*BW1 padded
// columns, 16*BW1^2 bytes) is the same for all lines of the CTA: it is staged
// into shared memory with cp.async, double-buffered so the copy of element
// ev+1 overlaps the arithmetic of element ev, and read back as warp broadcasts.
#include "atb_generic.cuh"

#include <cstdlib>
#include <type_traits>
#include <utility>

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


// Row-parallel form of the block recurrence: one thread per (row, line),
// rows = the BW1 unknowns (node kv, state s) of one element of a vertical line,
// lines fastest within a warp (LPB lines of a CTA -> consecutive horizontal
// nodes -> coalesced field accesses).  Per element step a thread forms one row
// of A_e v - C_e w (2*BW1 FMAs) from the staged blocks (two distinct rows per
// warp -> broadcasts) and the line's vectors in shared memory; the CTA holds
// BW1*LPB threads, so a step is short and many warps hide the latency of the
// sequential element chain.  Field pointers are selected once per thread with
// compile-time indices (a runtime-indexed kernel-parameter array would be
// copied to local memory).
template <int NQ, int NS, int LPB>
__global__ void __launch_bounds__(NQ * NS * LPB) band_solve_rows_kernel(const BandSolve B, const double* blk) {
  constexpr int BW1 = NQ * NS;
  constexpr int MAT = BW1 * BW1;
  constexpr int NT = BW1 * LPB;
  extern __shared__ __align__(16) double sm[];
  auto smat = [&](int b) { return sm + b * 2 * MAT; };
  double* vb = sm + 4 * MAT;       // [BW1][LPB]: right-hand side (forward) / y (backward)
  double* wb = vb + BW1 * LPB;     // [2][BW1][LPB]: previous element's result
  const LineMap& M = B.M;
  const int l = threadIdx.x % LPB, row = threadIdx.x / LPB;
  const int kv = row / NS, s = row - kv * NS;
  const int line = blockIdx.x * LPB + l;
  const bool act = line < M.nlines;
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  const int hn = act ? line % nh : 0;
  const int e0 = act ? M.e0[line] : 0;
  const double *pq = B.q[0], *pe0 = B.ex[0][0], *pi0 = B.im[0][0], *pe1 = B.ex[1][0], *pi1 = B.im[1][0];
  double* po = B.out[0];
#pragma unroll
  for (int c = 1; c < NS; ++c)
    if (c == s) {
      pq = B.q[c];
      pe0 = B.ex[0][c];
      pi0 = B.im[0][c];
      pe1 = B.ex[1][c];
      pi1 = B.im[1][c];
      po = B.out[c];
    }
  const int npairs = B.npairs;
  const double dt = B.dt, a0 = B.a[0], b0 = B.b[0], a1 = B.a[1], b1 = B.b[1];
  auto gidx = [&](int ev) { return (size_t)(e0 + ev * M.estep) * Np + hn + (size_t)nh * kv; };
  auto stage = [&](double* dst, const double* src) {
    for (int c = threadIdx.x; c < MAT; c += NT) cp_async16(dst + 2 * c, src + 2 * c);  // 2*MAT doubles
  };
  auto rhs = [&](int ev) {
    if (!act) return 0.0;
    const size_t g = gidx(ev);
    double v = pq[g];
    if (npairs > 0) v = v + dt * (a0 * pe0[g] + b0 * pi0[g]);
    if (npairs > 1) v = v + dt * (a1 * pe1[g] + b1 * pi1[g]);
    return v;
  };
  // y = A v - C w for this thread's row (same summation order as the
  // register-window form: two sums, then their difference)
  auto row_dot = [&](const double* Am, const double* Cm, const double* w) {
    double acc = 0.0, acc2 = 0.0;
#pragma unroll
    for (int k = 0; k < BW1; ++k) {
      acc += Am[row * BW1 + k] * vb[k * LPB + l];
      acc2 += Cm[row * BW1 + k] * w[k * LPB + l];
    }
    return acc - acc2;
  };
  // ------------------------------------------------------------ forward
  stage(smat(0), blk);
  cp_async_commit();
  if (KV > 1) stage(smat(1), blk + (size_t)4 * MAT);
  cp_async_commit();
  wb[row * LPB + l] = 0.0;  // y_{-1} = 0
  wb[BW1 * LPB + row * LPB + l] = 0.0;
  double bnext = rhs(0);
  for (int ev = 0; ev < KV; ++ev) {
    vb[row * LPB + l] = bnext;
    if (ev + 1 < KV) bnext = rhs(ev + 1);
    cp_async_wait1();
    __syncthreads();
    const double y = row_dot(smat(ev & 1), smat(ev & 1) + MAT, wb + ((ev + 1) & 1) * BW1 * LPB);
    wb[(ev & 1) * BW1 * LPB + row * LPB + l] = y;
    if (act) po[gidx(ev)] = y;
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
  wb[row * LPB + l] = 0.0;  // x_{KV} = 0
  wb[BW1 * LPB + row * LPB + l] = 0.0;
  // this thread wrote y_e at exactly the address it reads back
  double ynext = act ? po[gidx(KV - 1)] : 0.0;
  for (int t = 0; t < KV; ++t) {
    const int ev = KV - 1 - t;
    vb[row * LPB + l] = ynext;
    if (ev > 0) ynext = act ? po[gidx(ev - 1)] : 0.0;
    cp_async_wait1();
    __syncthreads();
    const double x = row_dot(smat(t & 1), smat(t & 1) + MAT, wb + ((t + 1) & 1) * BW1 * LPB);
    wb[(t & 1) * BW1 * LPB + row * LPB + l] = x;
    if (act) po[gidx(ev)] = x;
    __syncthreads();
    if (t + 2 < KV) stage(smat(t & 1), blk + (size_t)(KV - 3 - t) * 4 * MAT + 2 * MAT);
    cp_async_commit();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <int NQ, int NS>
void rows_launch(const BandSolve& B, cudaStream_t st) {
  constexpr int BW1 = NQ * NS;
  constexpr int LPB = 16;
  constexpr size_t smem = sizeof(double) * (4 * BW1 * BW1 + 3 * BW1 * LPB);
  static bool configured = false;
  if (!configured && smem > 48 * 1024)
    cudaFuncSetAttribute(band_solve_rows_kernel<NQ, NS, LPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  configured = true;
  band_solve_rows_kernel<NQ, NS, LPB><<<(B.M.nlines + LPB - 1) / LPB, BW1 * LPB, smem, st>>>(B, B.blk);
}

template <int NS> solve_fn pick_rows(int nq) {
  switch (nq) {
    case 2: return rows_launch<2, NS>;
    case 3: return rows_launch<3, NS>;
    case 4: return rows_launch<4, NS>;
    case 5: return rows_launch<5, NS>;
    case 6: return rows_launch<6, NS>;
    case 7: return rows_launch<7, NS>;
    case 8: return rows_launch<8, NS>;
  }
  return nullptr;
}

// FP64 matrix-unit form of the block recurrence (mma.sync m8n8k4 f64; the
// tcgen05 tensor cores have no FP64 kind).  A CTA owns LPC = 8*NT lines and
// one warp per 8-row tile of the BW1 element rows; per element step a warp
// computes its rows of Y = A_e V - C_e W for all LPC lines as KT x NT x 2
// matrix-unit operations: A_e / C_e fragments come straight from the
// (L1/L2-resident) block inverses into registers, prefetched one element ahead,
// V (right-hand side) and W (previous element's result) are B fragments read
// from shared memory (double-buffered, one barrier per element).  Rows are
// padded to MT*8 and the reduction dimension to KT*4 with zeros.
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NQ, int NS, int NT, int D>
__global__ void __launch_bounds__(32 * ((NQ * NS + 7) / 8)) band_solve_mma_kernel(const BandSolve B, const double* blk) {
  constexpr int BW1 = NQ * NS;
  constexpr int MAT = BW1 * BW1;
  constexpr int MT = (BW1 + 7) / 8;  // warps
  constexpr int KT = (BW1 + 3) / 4;
  constexpr int KP = 4 * KT;
  constexpr int LPC = 8 * NT;
  constexpr int NTH = 32 * MT;
  constexpr int NL = NQ * LPC;       // loader threads: one per (node kv, line)
  // row stride of V / W: 4 doubles of padding put the 4 rows of a B fragment
  // on distinct bank groups (2 wavefronts per fragment load, the minimum)
  constexpr int LDV = LPC + 4;
  extern __shared__ __align__(16) double sm[];
  double* Vb = sm;                  // [2][KP][LDV]
  double* Wb = sm + 2 * KP * LDV;   // [2][KP][LDV]
  double* R = sm + 4 * KP * LDV;    // [D][5][NS][NL]: raw right-hand-side fields in flight
  const LineMap& M = B.M;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  const int line0 = blockIdx.x * LPC;
  for (int i = threadIdx.x; i < 4 * KP * LDV; i += NTH) sm[i] = 0.0;
  // ---- this thread's output rows: row = 8*warp + g, lines 8*nt + 2*tq + {0,1}
  const int orow = 8 * warp + g;
  const bool orow_ok = orow < BW1;
  const int okv = orow_ok ? orow / NS : 0, os = orow_ok ? orow - okv * NS : 0;
  double* po = B.out[0];
#pragma unroll
  for (int c = 1; c < NS; ++c)
    if (c == os) po = B.out[c];
  size_t obase[NT][2];
  bool oact[NT][2];
  const size_t ostep = (size_t)M.estep * Np;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int line = line0 + 8 * nt + 2 * tq + i;
      oact[nt][i] = orow_ok && line < M.nlines;
      const int ln = oact[nt][i] ? line : 0;
      obase[nt][i] = (size_t)M.e0[ln] * Np + ln % nh + (size_t)nh * okv;
    }
  // ---- loader: thread lt < NL owns node lkv of line ll for every state
  const int lt = threadIdx.x;
  const bool ld_ok = lt < NL;
  const int lkv = ld_ok ? lt / LPC : 0, ll = ld_ok ? lt - lkv * LPC : 0;
  const int lline = line0 + ll;
  const bool lact = ld_ok && lline < M.nlines;
  const size_t lbase = lact ? (size_t)M.e0[lline] * Np + lline % nh + (size_t)nh * lkv : 0;
  const size_t lstep = (size_t)M.estep * Np;
  const int npairs = B.npairs;
  const double dt = B.dt, a0 = B.a[0], b0 = B.b[0], a1 = B.a[1], b1 = B.b[1];
  auto rslot = [&](int slot, int f, int s) { return R + ((slot * 5 + f) * NS + s) * NL + lt; };
  // raw fields of element ev into ring slot ev % D (the issuing thread is the
  // only reader of what it copies: no barrier between copy and use)
  auto issue_fwd = [&](int ev) {
    if (lact && ev < KV) {
      const size_t gi = lbase + (size_t)ev * lstep;
      const int slot = ev % D;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        cp_async8(rslot(slot, 0, s), B.q[s] + gi);
        if (npairs > 0) {
          cp_async8(rslot(slot, 1, s), B.ex[0][s] + gi);
          cp_async8(rslot(slot, 2, s), B.im[0][s] + gi);
        }
        if (npairs > 1) {
          cp_async8(rslot(slot, 3, s), B.ex[1][s] + gi);
          cp_async8(rslot(slot, 4, s), B.im[1][s] + gi);
        }
      }
    }
    cp_async_commit();
  };
  auto combine_fwd = [&](int ev, int buf) {
    if (!ld_ok) return;
    const int slot = ev % D;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      double x = 0.0;
      if (lact) {
        x = *rslot(slot, 0, s);
        if (npairs > 0) x = x + dt * (a0 * *rslot(slot, 1, s) + b0 * *rslot(slot, 2, s));
        if (npairs > 1) x = x + dt * (a1 * *rslot(slot, 3, s) + b1 * *rslot(slot, 4, s));
      }
      Vb[(buf * KP + lkv * NS + s) * LDV + ll] = x;
    }
  };
  auto issue_bwd = [&](int ev) {
    if (lact && ev >= 0) {
      const size_t gi = lbase + (size_t)ev * lstep;
      const int slot = ev % D;
#pragma unroll
      for (int s = 0; s < NS; ++s) cp_async8(rslot(slot, 0, s), B.out[s] + gi);
    }
    cp_async_commit();
  };
  auto combine_bwd = [&](int ev, int buf) {
    if (!ld_ok) return;
    const int slot = ev % D;
#pragma unroll
    for (int s = 0; s < NS; ++s) Vb[(buf * KP + lkv * NS + s) * LDV + ll] = lact ? *rslot(slot, 0, s) : 0.0;
  };
  // ---- A / C fragments: row 8*warp + g, column 4*kt + tq of a BW1 x BW1 block
  auto frag = [&](const double* m, double* f) {
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const int c = 4 * kt + tq;
      f[kt] = (orow_ok && c < BW1) ? __ldg(m + orow * BW1 + c) : 0.0;
    }
  };
  auto step = [&](int buf, const double* fa, const double* fc, int ev) {
    double acc[NT][2], acc2[NT][2];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc2[nt][0] = acc2[nt][1] = 0.0;
    const double* V = Vb + buf * KP * LDV;
    const double* Wp = Wb + (buf ^ 1) * KP * LDV;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int k = 4 * kt + tq, n = 8 * nt + g;
        dmma_8x8x4(acc[nt][0], acc[nt][1], fa[kt], V[k * LDV + n]);
        dmma_8x8x4(acc2[nt][0], acc2[nt][1], fc[kt], Wp[k * LDV + n]);
      }
    double* W = Wb + buf * KP * LDV;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double y = acc[nt][i] - acc2[nt][i];
        if (orow_ok) W[orow * LDV + 8 * nt + 2 * tq + i] = y;
        if (oact[nt][i]) po[obase[nt][i] + (size_t)ev * ostep] = y;
      }
  };
  __syncthreads();
  // ------------------------------------------------------------ forward
  double fa[KT], fc[KT], na[KT], nc[KT];
#pragma unroll
  for (int j = 0; j < D; ++j) issue_fwd(j);
  frag(blk, fa);
  frag(blk + MAT, fc);
  cp_async_wait<D - 1>();
  combine_fwd(0, 0);
  __syncthreads();
  for (int ev = 0; ev < KV; ++ev) {
    const int buf = ev & 1;
    issue_fwd(ev + D);
    if (ev + 1 < KV) {
      frag(blk + (size_t)(ev + 1) * 4 * MAT, na);
      frag(blk + (size_t)(ev + 1) * 4 * MAT + MAT, nc);
    }
    step(buf, fa, fc, ev);
    if (ev + 1 < KV) {
      cp_async_wait<D - 1>();
      combine_fwd(ev + 1, buf ^ 1);
    }
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) { fa[kt] = na[kt]; fc[kt] = nc[kt]; }
    __syncthreads();
  }
  cp_async_wait<0>();
  __syncthreads();
  // ----------------------------------------------------------- backward
  // step t uses buffer parity (KV + t) & 1; x_{KV} = 0
  for (int i = threadIdx.x; i < KP * LDV; i += NTH) Wb[((KV & 1) ^ 1) * KP * LDV + i] = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j) issue_bwd(KV - 1 - j);
  frag(blk + (size_t)(KV - 1) * 4 * MAT + 2 * MAT, fa);
  frag(blk + (size_t)(KV - 1) * 4 * MAT + 3 * MAT, fc);
  cp_async_wait<D - 1>();
  combine_bwd(KV - 1, KV & 1);
  __syncthreads();
  for (int t = 0; t < KV; ++t) {
    const int ev = KV - 1 - t;
    const int buf = (KV + t) & 1;
    issue_bwd(ev - D);
    if (ev > 0) {
      frag(blk + (size_t)(ev - 1) * 4 * MAT + 2 * MAT, na);
      frag(blk + (size_t)(ev - 1) * 4 * MAT + 3 * MAT, nc);
    }
    step(buf, fa, fc, ev);
    if (ev > 0) {
      cp_async_wait<D - 1>();
      combine_bwd(ev - 1, buf ^ 1);
    }
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) { fa[kt] = na[kt]; fc[kt] = nc[kt]; }
    __syncthreads();
  }
  cp_async_wait<0>();
}

template <int NQ, int NS>
void mma_launch(const BandSolve& B, cudaStream_t st) {
  constexpr int BW1 = NQ * NS;
  constexpr int NT = 2;
  constexpr int D = 3;
  constexpr int KP = 4 * ((BW1 + 3) / 4);
  constexpr int LPC = 8 * NT;
  constexpr int NTH = 32 * ((BW1 + 7) / 8);
  static_assert(NQ * LPC <= NTH, "the right-hand-side loader needs NQ*LPC threads");
  constexpr size_t smem = sizeof(double) * (4 * KP * (LPC + 4) + D * 5 * NS * NQ * LPC);
  static bool configured = false;
  if (!configured && smem > 48 * 1024)
    cudaFuncSetAttribute(band_solve_mma_kernel<NQ, NS, NT, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  configured = true;
  band_solve_mma_kernel<NQ, NS, NT, D><<<(B.M.nlines + LPC - 1) / LPC, NTH, smem, st>>>(B, B.blk);
}

// ---------------------------------------------- warp-owned block recurrence
// The same recurrence (y_e = Li_e b_e - G_e y_e-1, x_e = Ui_e y_e - H_e x_e+1)
// with one warp per 8 lines computing EVERY row of the block: the element-to-
// element dependency stays inside the warp, so the sequential chain carries
// no CTA barrier.  The blocks' zero structure is exploited tile by tile:
// Li is lower and Ui upper triangular, and since DG elements couple only
// through their face nodes, L_e,e-1 (U_e,e+1) is nonzero only in the last
// (first) Ns columns, so G_e (H_e) is too -- the product with the previous
// element's result needs only its face node, one or two m8n8k4 steps instead
// of KT.  Only the nonzero 8x4 tiles are stored (frag_prep_kernel, in
// matrix-unit fragment order: one 256-byte run per tile, one double per
// lane), copied per element into a shared ring by the CTA with contiguous
// 16-byte cp.async two elements ahead, and read with conflict-free 8-byte
// loads.  The host checks the structure once (warp_solve_structure_ok) and
// uses band_solve_mma_kernel when it does not hold.  Skipped tiles are exact
// zeros and every accumulator adds its tiles in the same order, so the
// results equal band_solve_mma_kernel's bit for bit.  Right-hand sides with
// no ARK pairs only (q given whole); the other forms use band_solve_mma_kernel.
struct TileRange {
  int lo, hi;  // reduction steps kt = lo .. hi (inclusive) of a row tile
};
__host__ __device__ constexpr int imin_c(int a, int b) { return a < b ? a : b; }
// pass 0: Li (mat 0), -G (mat 1); pass 1: Ui (mat 0), -H (mat 1); row tile mt
__host__ __device__ constexpr TileRange tile_range(int BW1, int NS, int pass, int mat, int mt) {
  const int KT = (BW1 + 3) / 4;
  if (pass == 0) return mat == 0 ? TileRange{0, imin_c(KT - 1, 2 * mt + 1)} : TileRange{(BW1 - NS) / 4, KT - 1};
  return mat == 0 ? TileRange{2 * mt, KT - 1} : TileRange{0, imin_c(KT - 1, (NS - 1) / 4)};
}
// tiles stored before (mat, mt) within one pass (mat-major, then mt); (2, 0) = all
__host__ __device__ constexpr int tile_off(int BW1, int NS, int pass, int mat, int mt) {
  const int MT = (BW1 + 7) / 8;
  int n = 0;
  for (int m = 0; m < 2; ++m)
    for (int t = 0; t < MT; ++t) {
      if (m == mat && t == mt) return n;
      const TileRange r = tile_range(BW1, NS, pass, m, t);
      n += r.hi - r.lo + 1;
    }
  return n;
}
__host__ __device__ constexpr int pass_tiles(int BW1, int NS, int pass) { return tile_off(BW1, NS, pass, 2, 0); }

template <int BW1, int NS>
struct WarpSolveShape {
  static constexpr int MT = (BW1 + 7) / 8;   // row tiles
  static constexpr int KT = (BW1 + 3) / 4;   // reduction steps
  static constexpr int KP = 4 * KT;          // reduction length (zero rows past BW1)
  static constexpr int RW = (KP > 8 * MT) ? KP : 8 * MT;  // rows of a result buffer
  static constexpr int LD = 12;              // row stride of [row][line] buffers: conflict-free B fragments
  static constexpr int T0 = pass_tiles(BW1, NS, 0), T1 = pass_tiles(BW1, NS, 1);
  static constexpr int FR = 32 * (T0 > T1 ? T0 : T1);     // doubles of one ring slot
  static constexpr int RS = 3;                            // ring depth (elements in flight)
  static constexpr int WBUF = RS * KP * LD + 2 * RW * LD;  // per warp: RHS ring + 2 result buffers
};

// frag[(e * (T0 + T1) + pass * T0 + tile_off(pass, mat, mt) + kt - lo) * 32 + lane]
//   = M[8 mt + lane / 4][4 kt + lane % 4]   (zero outside BW1 x BW1)
// with M = Li_e, -G_e (pass 0) or Ui_e, -H_e (pass 1) for mat = 0, 1.
__global__ void frag_prep_kernel(const double* blk, int KV, int BW1, int NS, double* frag) {
  const int MT = (BW1 + 7) / 8;
  const int T0 = pass_tiles(BW1, NS, 0), T1 = pass_tiles(BW1, NS, 1);
  const size_t n = (size_t)KV * (T0 + T1) * 32;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int lane = (int)(i % 32);
    const size_t tix = i / 32;
    const int e = (int)(tix / (T0 + T1));
    int t = (int)(tix - (size_t)e * (T0 + T1));
    const int pass = t < T0 ? 0 : 1;
    if (pass) t -= T0;
    int mat = 0, mt = 0, kt = 0;
    for (int m = 0; m < 2; ++m)
      for (int r = 0; r < MT; ++r) {
        const TileRange tr = tile_range(BW1, NS, pass, m, r);
        const int o = tile_off(BW1, NS, pass, m, r);
        if (t >= o && t < o + tr.hi - tr.lo + 1) {
          mat = m;
          mt = r;
          kt = tr.lo + t - o;
        }
      }
    const int row = 8 * mt + lane / 4, col = 4 * kt + lane % 4;
    double v = 0.0;
    if (row < BW1 && col < BW1) {
      const double* m = blk + ((size_t)e * 4 + 2 * pass + mat) * BW1 * BW1;
      v = m[row * BW1 + col];
      if (mat == 1) v = -v;
    }
    frag[i] = v;
  }
}

// f(integral_constant<int, 0>) ... f(integral_constant<int, N-1>): loop
// indices that are constant expressions inside the body
template <class Fn, int... I>
__device__ __forceinline__ void static_for_impl(Fn& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class Fn>
__device__ __forceinline__ void static_for(Fn&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

__device__ __forceinline__ void cp_async16g(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

template <int NQ, int NS, int NW>
__global__ void __launch_bounds__(32 * NW) band_solve_warp_kernel(const BandSolve B) {
  constexpr int BW1 = NQ * NS;
  using S = WarpSolveShape<BW1, NS>;
  constexpr int MT = S::MT, KT = S::KT, KP = S::KP, RW = S::RW, LD = S::LD, FR = S::FR, RS = S::RS;
  constexpr int T0 = S::T0, T1 = S::T1;
  constexpr int JT = (BW1 + 3) / 4;  // RHS rows per lane per element (4 rows x 8 lines per pass)
  extern __shared__ __align__(16) double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tq = lane & 3;
  double* Fr = sm;                                   // [RS][FR], shared by the CTA's warps
  double* ring = sm + RS * FR + warp * S::WBUF;      // [RS][KP][LD]: right-hand sides
  double* Wb = ring + RS * KP * LD;                  // [2][RW][LD]: results of the last two elements
  const LineMap& M = B.M;
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  const size_t lstep = (size_t)M.estep * Np;
  const int line0 = (blockIdx.x * NW + warp) * 8;
  for (int i = lane; i < S::WBUF; i += 32) ring[i] = 0.0;
  // ---- RHS loader: lane owns line (lane & 7) and rows 4j + (lane >> 3)
  const int ll = lane & 7;
  const bool lact = line0 + ll < M.nlines;
  const size_t lb = lact ? (size_t)M.e0[line0 + ll] * Np + (line0 + ll) % nh : 0;
  size_t roff[JT];
  int rsel[JT];
#pragma unroll
  for (int j = 0; j < JT; ++j) {
    const int row = 4 * j + (lane >> 3);
    rsel[j] = (lact && row < BW1) ? row % NS : -1;
    roff[j] = lb + (row < BW1 ? (size_t)nh * (row / NS) : 0);
  }
  auto field = [&](auto f, int s) {
    auto p = f[0];
#pragma unroll
    for (int c = 1; c < NS; ++c)
      if (c == s) p = f[c];
    return p;
  };
  const double* src[JT];
#pragma unroll
  for (int j = 0; j < JT; ++j) src[j] = field(B.q, rsel[j] < 0 ? 0 : rsel[j]) + roff[j];
  // ---- outputs: rows 8 mt + g, lines 2 tq + i (null: padding row or no line)
  double* dst[MT][2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int line = line0 + 2 * tq + i;
    const bool act = line < M.nlines;
    const size_t ob = act ? (size_t)M.e0[line] * Np + line % nh : 0;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      const int row = 8 * mt + g;
      dst[mt][i] = (act && row < BW1) ? field(B.out, row % NS) + (size_t)nh * (row / NS) + ob : nullptr;
    }
  }
  // element ev of pass P (its tiles and this warp's RHS) into ring slot
  // ev % RS; evoff = ev * (element step in the fields)
  auto issue = [&](auto passc, int ev, int slot, size_t evoff) {
    constexpr int P = decltype(passc)::value;
    if (ev >= 0 && ev < KV) {
      constexpr int n16 = (P ? T1 : T0) * 16;
      const double* gf = B.frag + ((size_t)ev * (T0 + T1) + (P ? T0 : 0)) * 32 + 2 * threadIdx.x;
      double* sf = Fr + slot * FR + 2 * threadIdx.x;
#pragma unroll
      for (int c = 0; c < n16; c += 32 * NW)
        if (c + (int)threadIdx.x < n16) cp_async16g(sf + 2 * c, gf + 2 * c);
      double* sr = ring + slot * KP * LD + (lane >> 3) * LD + ll;
#pragma unroll
      for (int j = 0; j < JT; ++j)
        if (rsel[j] >= 0) cp_async8(sr + 4 * j * LD, src[j] + evoff);
    }
    cp_async_commit();
  };
  auto step = [&](auto passc, int slot, size_t evoff, int par) {
    constexpr int P = decltype(passc)::value;
    const double* F = Fr + slot * FR + lane;
    const double* V = ring + slot * KP * LD;
    const double* Wp = Wb + (par ^ 1) * RW * LD;
    double* Wn = Wb + par * RW * LD;
    constexpr TileRange cr = tile_range(BW1, NS, P, 1, 0);  // the same for every row tile
    double bv[KT], bw[KT];
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      bv[kt] = V[(4 * kt + tq) * LD + g];
      bw[kt] = (kt >= cr.lo && kt <= cr.hi) ? Wp[(4 * kt + tq) * LD + g] : 0.0;
    }
    double aA[MT][2], aC[MT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      aA[mt][0] = aA[mt][1] = aC[mt][0] = aC[mt][1] = 0.0;
    }
    // reduction step outermost: consecutive matrix-unit operations feed
    // different accumulators (a dependent one waits the full latency); each
    // accumulator still adds its tiles in ascending kt.  The coupling
    // product (previous element) first: its operands are the ones produced
    // last.  Tile offsets are constant expressions (static_for indices).
    static_for<KT>([&](auto ktc) {
      constexpr int kt = decltype(ktc)::value;
      static_for<MT>([&](auto mtc) {
        constexpr int mt = decltype(mtc)::value;
        constexpr TileRange rc = tile_range(BW1, NS, P, 1, mt);
        if constexpr (kt >= rc.lo && kt <= rc.hi) {
          constexpr int off = (tile_off(BW1, NS, P, 1, mt) + kt - rc.lo) * 32;
          dmma_8x8x4(aC[mt][0], aC[mt][1], F[off], bw[kt]);
        }
      });
    });
    static_for<KT>([&](auto ktc) {
      constexpr int kt = decltype(ktc)::value;
      static_for<MT>([&](auto mtc) {
        constexpr int mt = decltype(mtc)::value;
        constexpr TileRange ra = tile_range(BW1, NS, P, 0, mt);
        if constexpr (kt >= ra.lo && kt <= ra.hi) {
          constexpr int off = (tile_off(BW1, NS, P, 0, mt) + kt - ra.lo) * 32;
          dmma_8x8x4(aA[mt][0], aA[mt][1], F[off], bv[kt]);
        }
      });
    });
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      const int row = 8 * mt + g;
      const double y0 = aA[mt][0] + aC[mt][0], y1 = aA[mt][1] + aC[mt][1];
      *reinterpret_cast<double2*>(Wn + row * LD + 2 * tq) = make_double2(y0, y1);
      if (dst[mt][0]) dst[mt][0][evoff] = y0;
      if (dst[mt][1]) dst[mt][1][evoff] = y1;
    }
  };
  const std::integral_constant<int, 0> fwd{};
  const std::integral_constant<int, 1> bwd{};
  // the right-hand side may come from the previous kernel of the stream
  pdl_wait();
  __syncthreads();
  // ------------------------------------------------------------ forward
  // slot: ev % RS; the refill of slot (ev + 2) % RS = (ev - 1) % RS follows
  // the barrier that ends every warp's use of it and this warp's step ev
  issue(fwd, 0, 0, 0);
  issue(fwd, 1, 1, lstep);
  {
    int slot = 0;
    size_t evoff = 0;
    for (int ev = 0; ev < KV; ++ev) {
      cp_async_wait<1>();
      __syncthreads();  // element ev in place; every warp is past element ev-1
      step(fwd, slot, evoff, ev & 1);
      const int s2 = slot == 0 ? RS - 1 : slot - 1;
      issue(fwd, ev + 2, s2, evoff + 2 * lstep);
      slot = slot == RS - 1 ? 0 : slot + 1;
      evoff += lstep;
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // the forward results are written (the backward pass reads them)
  // ----------------------------------------------------------- backward
#pragma unroll
  for (int j = 0; j < JT; ++j) src[j] = field(B.out, rsel[j] < 0 ? 0 : rsel[j]) + roff[j];
  // x_KV = 0: the buffer read first holds zeros
  for (int i = lane; i < RW * LD; i += 32) Wb[((KV & 1) ^ 1) * RW * LD + i] = 0.0;
  // slot: (KV - 1 - ev) % RS, i.e. the step count t % RS
  issue(bwd, KV - 1, 0, (size_t)(KV - 1) * lstep);
  issue(bwd, KV - 2, 1, (size_t)(KV - 2) * lstep);
  {
    int slot = 0;
    size_t evoff = (size_t)(KV - 1) * lstep;
    for (int t = 0; t < KV; ++t) {
      const int ev = KV - 1 - t;
      cp_async_wait<1>();
      __syncthreads();
      step(bwd, slot, evoff, (KV + t) & 1);
      const int s2 = slot == 0 ? RS - 1 : slot - 1;
      issue(bwd, ev - 2, s2, evoff - 2 * lstep);
      slot = slot == RS - 1 ? 0 : slot + 1;
      evoff -= lstep;
    }
  }
  cp_async_wait<0>();
  pdl_trigger();
}

template <int NQ, int NS, int NW>
constexpr size_t warp_solve_smem() {
  using S = WarpSolveShape<NQ * NS, NS>;
  return sizeof(double) * ((size_t)S::RS * S::FR + (size_t)NW * S::WBUF);
}

constexpr size_t kWarpSolveSmemMax = 227 * 1024;

template <int NQ, int NS, int NW>
void warp_launch_nw(const BandSolve& B, cudaStream_t st) {
  constexpr size_t smem = warp_solve_smem<NQ, NS, NW>();
  static bool configured = false;
  if (!configured && smem > 48 * 1024)
    cudaFuncSetAttribute(band_solve_warp_kernel<NQ, NS, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  configured = true;
  const int warps = (B.M.nlines + 7) / 8;
  launch_maybe_pdl(band_solve_warp_kernel<NQ, NS, NW>, dim3((warps + NW - 1) / NW), dim3(32 * NW), smem, st, B);
}

// Warps per CTA: the element steps are bound by the issue rate of each SM, so
// the time goes with the warps the busiest SM runs in total, ceil(CTAs / SMs)
// x NW; among counts within 2% of each other, CTAs on every SM, then more
// warps resident at once (latency hiding), then more warps per CTA (each copy
// of the tiles shared by more lines).
inline int pick_nw(int warps, int nsm, const size_t smem[4]) {
  static const int cand[4] = {2, 3, 4, 6};
  int best = -1;
  long best_load = 0;
  int best_sms = 0, best_res = 0;
  for (int i = 0; i < 4; ++i) {
    if (smem[i] > kWarpSolveSmemMax) continue;
    const int nw = cand[i];
    const long ctas = (warps + nw - 1) / nw;
    int cps = (int)((228 * 1024) / (smem[i] + 1024));
    if (cps > 2048 / (32 * nw)) cps = 2048 / (32 * nw);
    if (cps < 1) continue;
    const long per_sm = (ctas + nsm - 1) / nsm;
    const long load = per_sm * nw;
    const int sms = (int)(ctas < nsm ? ctas : nsm);
    const int res = (int)((per_sm < cps ? per_sm : cps) * nw);
    const bool better = best < 0 || 50 * load < 49 * best_load;
    const bool close = best >= 0 && 50 * load <= 51 * best_load && 50 * best_load <= 51 * load;
    if (better || (close && (sms > best_sms || (sms == best_sms && res >= best_res)))) {
      best = nw;
      best_load = load;
      best_sms = sms;
      best_res = res;
    }
  }
  return best;
}

template <int NQ, int NS>
bool warp_launch(const BandSolve& B, cudaStream_t st) {
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
  }
  const size_t smem[4] = {warp_solve_smem<NQ, NS, 2>(), warp_solve_smem<NQ, NS, 3>(), warp_solve_smem<NQ, NS, 4>(),
                          warp_solve_smem<NQ, NS, 6>()};
  switch (pick_nw((B.M.nlines + 7) / 8, nsm, smem)) {
    case 2: warp_launch_nw<NQ, NS, 2>(B, st); return true;
    case 3: warp_launch_nw<NQ, NS, 3>(B, st); return true;
    case 4: warp_launch_nw<NQ, NS, 4>(B, st); return true;
    case 6: warp_launch_nw<NQ, NS, 6>(B, st); return true;
  }
  return false;
}

typedef bool (*warp_fn)(const BandSolve&, cudaStream_t);
template <int NS> warp_fn pick_warp(int nq) {
  switch (nq) {
    case 2: return warp_launch<2, NS>;
    case 3: return warp_launch<3, NS>;
    case 4: return warp_launch<4, NS>;
    case 5: return warp_launch<5, NS>;
    case 6: return warp_launch<6, NS>;
    case 7: return warp_launch<7, NS>;
    case 8: return warp_launch<8, NS>;
  }
  return nullptr;
}

template <int NS> solve_fn pick_mma(int nq) {
  switch (nq) {
    case 2: return mma_launch<2, NS>;
    case 3: return mma_launch<3, NS>;
    case 4: return mma_launch<4, NS>;
    case 5: return mma_launch<5, NS>;
    case 6: return mma_launch<6, NS>;
    case 7: return mma_launch<7, NS>;
    case 8: return mma_launch<8, NS>;
  }
  return nullptr;
}

}  // namespace

void launch_block_prep(const double* band, int KV, int BW1, double* blk, cudaStream_t st) {
  block_prep_kernel<<<KV, ((BW1 + 31) / 32) * 32, 0, st>>>(band, KV, BW1, blk);
}

size_t frag_doubles(int KV, int BW1, int NS) {
  return (size_t)KV * (pass_tiles(BW1, NS, 0) + pass_tiles(BW1, NS, 1)) * 32;
}

void launch_frag_prep(const double* blk, int KV, int BW1, int NS, double* frag, cudaStream_t st) {
  const size_t n = frag_doubles(KV, BW1, NS);
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  frag_prep_kernel<<<blocks, 256, 0, st>>>(blk, KV, BW1, NS, frag);
}

bool warp_solve_structure_ok(const double* blk_host, int KV, int BW1, int NS) {
  // every nonzero of Li, G, Ui, H lies inside the stored tiles of its row tile
  const int MT = (BW1 + 7) / 8;
  for (int e = 0; e < KV; ++e)
    for (int pass = 0; pass < 2; ++pass)
      for (int mat = 0; mat < 2; ++mat) {
        const double* m = blk_host + ((size_t)e * 4 + 2 * pass + mat) * BW1 * BW1;
        for (int mt = 0; mt < MT; ++mt) {
          const TileRange r = tile_range(BW1, NS, pass, mat, mt);
          for (int row = 8 * mt; row < 8 * mt + 8 && row < BW1; ++row)
            for (int col = 0; col < BW1; ++col)
              if ((col < 4 * r.lo || col > 4 * r.hi + 3) && m[row * BW1 + col] != 0.0) return false;
        }
      }
  return true;
}


// Dispatch: the block-parallel form when the factor is shared and its
// per-element inverses were prepared, else the register-window substitution
// (shared factor), else the generic per-line kernel.
namespace {

// ------------------------------------------------ per-line factors
// Vertical lines whose factors differ (curved grids: every column of a sphere
// has its own metric terms).  One thread per line, the factor in the
// line-fastest layout band[(r * W + k) * nlines + line] (coalesced across the
// threads of a warp), the element-block recurrence with compile-time block
// size BW1 = NQ * NS so that the previous / next block's values and the
// current block's live in registers.  Sums run in the generic kernel's order
// (increasing column), so the results are the generic kernel's; with SPARSE
// the entries that the face-node coupling makes zero (the sub-diagonal block
// of L outside its face rows and columns, the super-diagonal block of U
// likewise; launch_band_lines_structure checks every line at setup) are not
// read, which halves the bytes of a solve.
// one row of the forward (FWD) or backward pass, then the next: compile-time
// row indices keep every block value in a register
template <int NQ, int NS, bool SPARSE, bool FWD, int I>
__device__ __forceinline__ void lines_rows(const BandSolve& B, const double* __restrict__ row0, size_t ld,
                                           size_t eoff, int nh, bool has_nb, const double (&nb)[NQ * NS],
                                           double (&cur)[NQ * NS]) {
  constexpr int BW1 = NQ * NS;
  constexpr int BW = BW1 - 1;
  constexpr int W = 2 * BW + 1;
  if constexpr (I >= 0 && I < BW1) {
    constexpr int s = I % NS, kv = I / NS;
    const size_t g = eoff + (size_t)nh * kv;
    const double* row = row0 + (size_t)I * W * ld;
    if constexpr (FWD) {
      double acc = B.q[s][g];
#pragma unroll
      for (int k = 0; k < 2; ++k)
        if (k < B.npairs) acc = acc + B.dt * (B.a[k] * B.ex[k][s][g] + B.b[k] * B.im[k][s][g]);
      if (has_nb) {
#pragma unroll
        for (int jp = I + 1; jp < BW1; ++jp) {
          if (SPARSE && !(I < NS && jp >= BW1 - NS)) continue;
          acc = acc - row[(size_t)(jp - I - 1) * ld] * nb[jp];
        }
      }
#pragma unroll
      for (int jp = 0; jp < I; ++jp) acc = acc - row[(size_t)(jp - I + BW) * ld] * cur[jp];
      cur[I] = acc;
      B.out[s][g] = acc;
      lines_rows<NQ, NS, SPARSE, FWD, I + 1>(B, row0, ld, eoff, nh, has_nb, nb, cur);
    } else {
      double acc = B.out[s][g];
#pragma unroll
      for (int jp = I + 1; jp < BW1; ++jp) acc = acc - row[(size_t)(jp - I + BW) * ld] * cur[jp];
      if (has_nb) {
#pragma unroll
        for (int jp = 0; jp < I; ++jp) {
          if (SPARSE && !(I >= BW1 - NS && jp < NS)) continue;
          acc = acc - row[(size_t)(2 * BW1 - 1 + jp - I) * ld] * nb[jp];
        }
      }
      cur[I] = acc / row[(size_t)BW * ld];
      B.out[s][g] = cur[I];
      lines_rows<NQ, NS, SPARSE, FWD, I - 1>(B, row0, ld, eoff, nh, has_nb, nb, cur);
    }
  }
}

template <int NQ, int NS, bool SPARSE>
__global__ void __launch_bounds__(64) band_solve_lines_kernel(const BandSolve B) {
  constexpr int BW1 = NQ * NS;
  constexpr int BW = BW1 - 1;
  constexpr int W = 2 * BW + 1;
  const LineMap& M = B.M;
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= M.nlines) return;
  const size_t ld = (size_t)M.nlines;
  const double* __restrict__ band = B.band + line;
  const int hn = line % M.nh;
  const int e0 = M.e0[line];
  const int KV = M.KV, nh = M.nh, Np = M.Np;
  double nb[BW1], cur[BW1];
#pragma unroll
  for (int j = 0; j < BW1; ++j) nb[j] = cur[j] = 0.0;
  // the right-hand side may come from the previous kernel of the stream
  // (programmatic dependent launch, launch_maybe_pdl)
  pdl_wait();
  // forward: L y = rhs (unit diagonal)
  for (int ev = 0; ev < KV; ++ev) {
    const size_t eoff = (size_t)(e0 + ev * M.estep) * Np + hn;
    lines_rows<NQ, NS, SPARSE, true, 0>(B, band + (size_t)ev * BW1 * W * ld, ld, eoff, nh, ev > 0, nb, cur);
#pragma unroll
    for (int j = 0; j < BW1; ++j) nb[j] = cur[j];
  }
  // backward: U x = y
#pragma unroll
  for (int j = 0; j < BW1; ++j) nb[j] = 0.0;
  for (int ev = KV - 1; ev >= 0; --ev) {
    const size_t eoff = (size_t)(e0 + ev * M.estep) * Np + hn;
    lines_rows<NQ, NS, SPARSE, false, BW1 - 1>(B, band + (size_t)ev * BW1 * W * ld, ld, eoff, nh, ev < KV - 1, nb,
                                               cur);
#pragma unroll
    for (int j = 0; j < BW1; ++j) nb[j] = cur[j];
  }
  pdl_trigger();
}

typedef void (*lines_fn)(const BandSolve& B, cudaStream_t st);
template <int NQ, int NS, bool SPARSE> void lines_launch(const BandSolve& B, cudaStream_t st) {
  launch_maybe_pdl(band_solve_lines_kernel<NQ, NS, SPARSE>, dim3((B.M.nlines + 63) / 64), dim3(64), 0, st, B);
}
template <int NS, bool SPARSE> lines_fn pick_lines_sp(int nq) {
  switch (nq) {
    case 2: return lines_launch<2, NS, SPARSE>;
    case 3: return lines_launch<3, NS, SPARSE>;
    case 4: return lines_launch<4, NS, SPARSE>;
    case 5: return lines_launch<5, NS, SPARSE>;
    case 6: return lines_launch<6, NS, SPARSE>;
    case 7: return lines_launch<7, NS, SPARSE>;
    case 8: return lines_launch<8, NS, SPARSE>;
  }
  return nullptr;
}
template <int NS> lines_fn pick_lines(int nq, bool sparse) {
  return sparse ? pick_lines_sp<NS, true>(nq) : pick_lines_sp<NS, false>(nq);
}

__global__ void band_lines_structure_kernel(const LineMap M, const double* band, int* count) {
  const int BW1 = M.Nq * M.ns, BW = BW1 - 1, W = 2 * BW + 1, NS = M.ns;
  const size_t total = (size_t)M.nlines * M.nunk * W;
  int bad = 0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const size_t rk = t / M.nlines;
    const int r = (int)(rk / W), k = (int)(rk - (size_t)r * W);
    const int i = r % BW1;
    bool skip = false;
    if (k <= BW1 - 2 - i) {  // previous element block, column jp = k + i + 1
      const int jp = k + i + 1;
      skip = !(i < NS && jp >= BW1 - NS);
    } else if (k >= 2 * BW1 - 1 - i) {  // next element block, column jp = k + i - (2 BW1 - 1)
      const int jp = k + i - (2 * BW1 - 1);
      skip = !(i >= BW1 - NS && jp < NS);
    }
    if (skip && band[t] != 0.0) bad = 1;
  }
  if (bad) atomicAdd(count, 1);
}

}  // namespace

void launch_band_lines_structure(const LineMap& M, const double* band, int* count, cudaStream_t st) {
  band_lines_structure_kernel<<<148 * 8, 256, 0, st>>>(M, band, count);
}

bool pdl_enabled() {
  static const int on = [] {
    const char* e = std::getenv("ATB_PDL");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return on != 0;
}

void launch_band_solve(const BandSolve& B, cudaStream_t st) {
  if (B.ld > 1 && B.ld == B.M.nlines && B.npairs <= 2 && (B.M.ns == 4 || B.M.ns == 5)) {
    lines_fn f = B.M.ns == 4 ? pick_lines<4>(B.M.Nq, B.lines_sparse != 0) : pick_lines<5>(B.M.Nq, B.lines_sparse != 0);
    if (f) {
      f(B, st);
      return;
    }
  }
  if (B.ld == 1 && B.frag && B.npairs == 0 && (B.M.ns == 4 || B.M.ns == 5)) {
    warp_fn w = B.M.ns == 4 ? pick_warp<4>(B.M.Nq) : pick_warp<5>(B.M.Nq);
    if (w && w(B, st)) return;
  }
  solve_fn f = nullptr;
  if (B.ld == 1 && B.blk) {
    if (B.M.ns == 1) f = pick_rows<1>(B.M.Nq);
    if (B.M.ns == 4) f = pick_mma<4>(B.M.Nq);
    if (B.M.ns == 5) f = pick_mma<5>(B.M.Nq);
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
