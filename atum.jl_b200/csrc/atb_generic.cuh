// Law-independent kernels: stage linear combinations, the vertical-column
// banded operator (probe assembly, no-pivot LU, batched solve fused with the
// ARK right-hand-side combination), reduction finalisation and the FP64 probe.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include <utility>

namespace atb {

// out = base + dt * sum_k (a_k X_k + b_k Y_k), accumulated in k order like
// `Qhat .+= dt .* (a .* ex_K[k] .+ at .* im_K[k])` (src/odesolvers.jl:346-349)
// and the final update (src/odesolvers.jl:382-384).
struct LinComb {
  int ns, npairs;
  size_t n;
  double dt;
  double a[3], b[3];
  const double* base[5];
  const double* X[3][5];
  const double* Y[3][5];
  double* out[5];
};
void launch_lincomb(const LinComb& C, cudaStream_t st);

// out = x + c * y  (per component)
struct Axpy {
  int ns;
  size_t n;
  double c;
  const double* x[5];
  const double* y[5];
  double* out[5];
};
void launch_axpy(const Axpy& A, cudaStream_t st);
// number of differing 32-bit words of two device arrays, added to *count
void launch_count_diff(const void* a, const void* b, size_t nwords, unsigned long long* count, cudaStream_t st);

// Vertical lines of nodes: line l = eh * nh + hn (horizontal element stack eh,
// horizontal node hn); unknown u = (ev * Nq + kv) * ns + s.
struct LineMap {
  int nlines, nunk, bw, Nq, ns, nh, KV, Np;
  int stacked, KH;
  size_t stride;
  const int* e0;  // nlines: element index of the bottom element of the stack
  int estep;      // element index step between vertically adjacent elements
};

void launch_probe_fill(const LineMap& M, int color, double* const* P, cudaStream_t st);
// probed band layout (one matrix per line): band[(r * W + (j - r + bw)) * nlines + line]
void launch_band_extract(const LineMap& M, int color, const double* const* LP, double* band, cudaStream_t st);
// line 0's band (one line) plus a count of lines differing from it bitwise
void launch_band_extract_first(const LineMap& M, int color, const double* const* LP, double* band1, int* ndiff,
                               cudaStream_t st);
void launch_band_compare(const LineMap& M, const double* band, int* ndiff, cudaStream_t st);
// copy line 0 into a compact matrix with padded row stride rs = 2*(bw+1)
void launch_band_compact(const LineMap& M, const double* band, double* out, cudaStream_t st);
// M = I + scale*A then no-pivot LU in place; entry (i, j) at
// band[(i * rs + (j - i + bw)) * ld + line], nl matrices
void launch_band_factor(int n, int bw, int nl, double* band, int rs, int ld, double scale, cudaStream_t st);

struct BandSolve {
  LineMap M;
  const double* band;
  int ld;  // 1 when every column shares the factor (compact, row stride 2*(bw+1)), else nlines
  // right-hand side: q + dt * sum_k (a_k ex_k + b_k im_k)
  int npairs;
  double dt, a[2], b[2];
  const double* q[5];
  const double* ex[2][5];
  const double* im[2][5];
  double* out[5];
  const double* blk;  // per-element [L^-1 | G | U^-1 | H] blocks (shared factor), or null
  const double* frag; // the same blocks in matrix-unit fragment order (launch_frag_prep), or null
  // per-line factors (ld = nlines): 1 when every line's factor couples
  // neighbouring elements through face nodes only (launch_band_lines_structure)
  int lines_sparse;
};
void launch_band_solve(const BandSolve& B, cudaStream_t st);
// number of entries of the per-line factors (ld = nlines) outside the
// face-node coupling structure that are not zero, added to *count
void launch_band_lines_structure(const LineMap& M, const double* band, int* count, cudaStream_t st);
void launch_block_prep(const double* band, int KV, int BW1, double* blk, cudaStream_t st);
// the per-element tiles of the warp-owned solve (band_solve_warp_kernel)
size_t frag_doubles(int KV, int BW1, int NS);
void launch_frag_prep(const double* blk, int KV, int BW1, int NS, double* frag, cudaStream_t st);
// whether the blocks (host copy of blk) have the zero structure those tiles assume
bool warp_solve_structure_ok(const double* blk_host, int KV, int BW1, int NS);

void launch_red_finish(const double* partials, int nblocks, int linf, double* out5, cudaStream_t st);
double probe_fp64_tflops(cudaStream_t st);

// ---------------------------------------------- programmatic dependent launch
// The stage kernels and the banded solve are launched with programmatic
// stream serialization: a kernel's grid may start while the previous kernel
// of its stream drains, runs its prologue (constant tables, pointers, buffer
// zeroing: nothing the previous kernel writes), and waits in pdl_wait() for
// the previous grid's completion and memory flush before its first dependent
// read.  Every such kernel calls pdl_trigger() after its last store, so a
// dependent grid launches only once all of its CTAs have done their work (a
// waiting dependent never holds resources one of them needs; triggering at
// the start, with dependents resident and waiting early, measured slower).  Both instructions are no-ops in
// a kernel launched without the attribute.  ATB_PDL=0 in the environment
// launches ordinarily.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
bool pdl_enabled();
template <typename... KArgs, typename... Args>
cudaError_t launch_maybe_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                             Args&&... args) {
  if (!pdl_enabled()) {
    kern<<<grid, block, smem, st>>>(args...);
    return cudaSuccess;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace atb
