// LSRK54 time stepping that allocates nothing (atb_lsrk54_step_noalloc).
//
// Who needs it: callers that cannot call cudaMalloc around a time step --
// a host application whose device memory is owned by its own pool allocator
// (a Julia or PyTorch process running its caching allocator at its memory
// limit), or a latency-critical loop that must not pay the device-wide
// synchronisation a cudaMalloc/cudaFree pair can cause.  They create the
// DGSEM operator once (atb_op_create allocates), then step it here as often
// as they like without any further allocation: the two scratch fields of the
// 2N-storage scheme (the stage increment dq and the second state buffer of
// the fused stage kernel) live in the file-scope array below.
//
// The array holds ATB_NOALLOC_MAX_DOFS doubles for each of the two fields
// (8 MiB in total); every GPU that loads the library keeps it until the
// process exits.  All calls share it, so calls that overlap on the GPU (two
// streams, two host threads, two devices' worth of work queued on one device)
// race on it; serialise them.  Its contents persist between calls; dq must
// start at zero and is cleared at the start of every call.
#include "../../include/atum_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

struct atb_op;
int atb_detail_fail(int code, const char* msg);
int atb_detail_op_device(const atb_op* op);
int atb_detail_lsrk54_steps(atb_op* op, double* const* q, double* dqbuf, double* qbbuf, double dt, int nsteps,
                            cudaStream_t st);

static __device__ __align__(256) double g_lsrk_noalloc_scratch[2 * (size_t)ATB_NOALLOC_MAX_DOFS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
int scratch_on_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return atb_detail_fail(ATB_ERR_CUDA, "atb_lsrk54_step_noalloc: no usable current device");
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_lsrk_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return atb_detail_fail(ATB_ERR_CUDA, "atb_lsrk54_step_noalloc: cudaGetSymbolAddress of the scratch failed");
    }
    g_scratch[dev] = static_cast<double*>(p);
  }
  *out = g_scratch[dev];
  return ATB_OK;
}
}  // namespace

extern "C" int atb_lsrk54_step_noalloc(atb_op* op, double* const* q, double dt, int nsteps, void* stream) {
  if (!op || !q || nsteps < 0) return atb_detail_fail(ATB_ERR_INVALID, "atb_lsrk54_step_noalloc: bad argument");
  if (!std::isfinite(dt)) return atb_detail_fail(ATB_ERR_INVALID, "atb_lsrk54_step_noalloc: dt is not finite");
  // the scratch address is per device: with another device current it would
  // point into memory the op's kernels cannot use
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return atb_detail_fail(ATB_ERR_CUDA, "atb_lsrk54_step_noalloc: no usable current device");
  }
  if (dev != atb_detail_op_device(op))
    return atb_detail_fail(ATB_ERR_INVALID,
                           "atb_lsrk54_step_noalloc: the current device is not the one the operator was created on");
  int ns = 0, K = 0, Np = 0;
  int rc = atb_op_dims(op, &ns, &K, &Np);
  if (rc) return rc;
  const size_t n = (size_t)ns * K * Np;
  if (n > (size_t)ATB_NOALLOC_MAX_DOFS)
    return atb_detail_fail(ATB_ERR_INVALID,
                           "atb_lsrk54_step_noalloc: the state has more DOFs than ATB_NOALLOC_MAX_DOFS "
                           "(use atb_solver_create / atb_solver_step, which allocate their scratch)");
  double* scratch = nullptr;
  if ((rc = scratch_on_current_device(&scratch))) return rc;
  double* dq = scratch;
  double* qb = scratch + (size_t)ATB_NOALLOC_MAX_DOFS;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(dq, 0, n * sizeof(double), st) != cudaSuccess) {
    cudaGetLastError();
    return atb_detail_fail(ATB_ERR_CUDA, "atb_lsrk54_step_noalloc: clearing dq failed");
  }
  return atb_detail_lsrk54_steps(op, q, dq, qb, dt, nsteps, st);
}
