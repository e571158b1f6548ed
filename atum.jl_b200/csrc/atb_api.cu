// Host side of the C ABI (include/atum_b200.h): operator and solver objects,
// brick geometry, kernel dispatch and the time-stepping drivers.
//
// There is no CPU compute path: every operator application, stage update,
// banded solve and reduction runs on the GPU; the host only sequences launches
// (and, for the relaxation RK, runs the scalar trust-region Newton on device
// reductions).
#include "../../include/atum_b200.h"
#include "atb_generic.cuh"
#include "atb_reduce.cuh"
#include "atb_tendency.cuh"
#include "atb_curved.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace atb;

namespace atb {
template <> tend_launch_fn pick_launcher<LAW_ADV>(int, int);
template <> tend_launch_fn pick_launcher<LAW_EULER>(int, int);
template <> tend_launch_fn pick_launcher<LAW_EG>(int, int);
template <> tend_launch_fn pick_launcher<LAW_LEG>(int, int);
template <> tend_launch_fn pick_launcher<LAW_SW>(int, int);
template <> tend_launch_fn pick_launcher_nq<LAW_ADV>(int, int, int);
template <> tend_launch_fn pick_launcher_nq<LAW_EULER>(int, int, int);
template <> tend_launch_fn pick_launcher_nq<LAW_EG>(int, int, int);
template <> tend_launch_fn pick_launcher_nq<LAW_LEG>(int, int, int);
template <> tend_launch_fn pick_launcher_nq<LAW_SW>(int, int, int);
template <> red_launch_fn pick_reducer<LAW_ADV>(int);
template <> red_launch_fn pick_reducer<LAW_EULER>(int);
template <> red_launch_fn pick_reducer<LAW_EG>(int);
template <> red_launch_fn pick_reducer<LAW_LEG>(int);
template <> red_launch_fn pick_reducer<LAW_SW>(int);
}  // namespace atb

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t _e = (call);                                                                       \
    if (_e != cudaSuccess) return fail(ATB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));    \
  } while (0)

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ATB_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return ATB_OK;
}

template <class T> int dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(ATB_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
  }
  return ATB_OK;
}

// ------------------------------------------------------------ profiling
constexpr int NPROF = 5;
struct Prof {
  bool on = false;
  long launches_total = 0;
  long n[NPROF] = {0, 0, 0, 0, 0};
  double ms[NPROF] = {0, 0, 0, 0, 0};
  std::vector<cudaEvent_t> pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  void resolve() {
    for (auto& p : pending) {
      cudaEventSynchronize(p.second.second);
      float t = 0;
      cudaEventElapsedTime(&t, p.second.first, p.second.second);
      ms[p.first] += t;
      n[p.first] += 1;
      pool.push_back(p.second.first);
      pool.push_back(p.second.second);
    }
    pending.clear();
  }
};
Prof g_prof;

// brackets one launch: construct before, call done() after
struct ProfScope {
  int k;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  ProfScope(int kclass, cudaStream_t s) : k(kclass), st(s) {
    g_prof.launches_total++;
    if (g_prof.on) {
      a = g_prof.get();
      cudaEventRecord(a, st);
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEvent_t b = g_prof.get();
      cudaEventRecord(b, st);
      g_prof.pending.push_back({k, {a, b}});
    }
  }
};

}  // namespace

struct atb_op {
  LawP law{};
  int dim = 0, N = 0, Nq = 0, Np = 0, Nfp = 0, K = 0, Kd[3] = {1, 1, 1}, ns = 0, naux = 0;
  int vk = 0, dirs = 0, sflux = 0, precision = 0, stacked = 0;
  int naux_used = 0;  // leading aux components the tendency kernel stages
  atb_op_desc kind{};  // instance 0's descriptor (kind checks of later placements)
  int ninst = 1;      // instances packed into this operator
  int K_active = 0;   // elements the tendency launches cover (a prefix of K)
  int device = -1;    // the CUDA device current at creation (its memory holds every buffer)
  std::vector<int> inst_off;  // first element of each instance, then K
  std::vector<int> col_e0;    // bottom element of every vertical column
  bool cols_uniform = true;   // every instance has the same element counts
  int npre = 0, npv = 0;
  // page-locked geometry staging of pools: a ring of kGeoRing areas, each
  // reused once the copies out of it have run, so a placement waits only for
  // the copies of the placement kGeoRing before it
  static constexpr int kGeoRing = 8;
  void* h_geo[kGeoRing] = {};
  size_t geo_bytes[kGeoRing] = {};
  cudaEvent_t geo_ev[kGeoRing] = {};  // last copy out of h_geo[i]
  int geo_turn = 0;
  std::vector<double> w, D;
  double* d_ginv = nullptr;
  int* d_nbr = nullptr;
  double* d_aux = nullptr;
  double* d_tab = nullptr;
  double* d_w = nullptr;
  double* d_J = nullptr;
  double* d_partials = nullptr;
  double* d_red = nullptr;
  double* h_red = nullptr;
  int red_blocks = 0;
  tend_launch_fn launch = nullptr;
  red_launch_fn reducer = nullptr;
  int prof_class = ATB_PROF_TEND;
  int E = 1;
  size_t smem = 0;
  int persist_ctas = 0;  // > 0: persistent launches of at most this many CTAs (brick kernels)
  tend_launch_fn launch_persist = nullptr;  // the persistent variant of `launch`
  // curved elements (atb_op_create_curved): per-node metrics and M J, per
  // face node normals, face masses and neighbour nodes, the D matrix
  bool curved = false;
  double* d_D = nullptr;
  double* d_G = nullptr;
  double* d_MJn = nullptr;
  double* d_fnrm = nullptr;
  double* d_fMJ = nullptr;
  int* d_fnb = nullptr;
  size_t stride() const { return (size_t)K * Np; }
};

namespace {

// CTA size of a tendency launch: E elements of Np nodes, rounded up to whole
// warps (the face tasks are spread over warp-aligned groups)
int cta_threads(int E, int Np) { return ((E * Np + 31) / 32) * 32; }

size_t op_smem(const atb_op* op, int E, int pf = 0) {
  if (op->curved) return curved_smem_bytes(op->vk, op->naux_used, op->Nq, E);
  return tend_smem_bytes(op->ns, op->npre, op->naux_used, op->dim, op->Nq, op->Np, op->Nfp, E, op->npv, false, pf);
}

void fill_args(const atb_op* op, TendArgs& A) {
  A.K = op->K_active;
  A.Nq = op->Nq;
  A.Np = op->Np;
  A.Nfp = op->Nfp;
  A.E = op->E;
  A.naux = op->naux_used;
  A.ginv = op->d_ginv;
  A.nbr = op->d_nbr;
  A.aux = op->d_aux;
  A.tab = op->d_tab;
  A.law = op->law;
  A.dirs = op->dirs;
  A.sflux = op->sflux;
  A.stride = op->stride();
  A.a = 0;
  A.bdt = 0;
  A.dte = nullptr;
  for (int j = 0; j < 3; ++j) {
    for (int c = 0; c < 5; ++c) { A.acc[j][c] = nullptr; A.accin[j][c] = nullptr; }
    A.ca[j] = A.cb[j] = 0.0;
  }
  A.adt = 0.0;
  A.lin_law = LawP{};
  A.lin_sflux = 0;
  A.lin_dirs = 0;
  A.naux_nl = op->naux_used;
  A.pf = 0;
  A.Dmat = op->d_D;
  A.G = op->d_G;
  A.MJn = op->d_MJn;
  A.fnrm = op->d_fnrm;
  A.fMJ = op->d_fMJ;
  A.fnb = op->d_fnb;
}

// EPI_ARK accumulators of one stage (see atb_tendency.cuh)
struct ArkAcc {
  double* acc[3][5];
  const double* accin[3][5];
  double ca[3], cb[3], adt;
};

// one tendency launch: epi with input q, outputs out/out2
int run_tendency(atb_op* op, int epi, const double* const* q, double* const* out, double* const* out2, double a,
                 double bdt, cudaStream_t st, const double* dte = nullptr, const ArkAcc* ark = nullptr) {
  TendArgs A;
  fill_args(op, A);
  A.epi = epi;
  A.a = a;
  A.bdt = bdt;
  A.dte = dte;
  if (ark) {
    for (int j = 0; j < 3; ++j) {
      for (int c = 0; c < 5; ++c) { A.acc[j][c] = ark->acc[j][c]; A.accin[j][c] = ark->accin[j][c]; }
      A.ca[j] = ark->ca[j];
      A.cb[j] = ark->cb[j];
    }
    A.adt = ark->adt;
  }
  for (int s = 0; s < 5; ++s) {
    A.q[s] = q[s < op->ns ? s : 0];
    A.out[s] = out ? out[s < op->ns ? s : 0] : nullptr;
    A.out2[s] = out2 ? out2[s < op->ns ? s : 0] : nullptr;
  }
  const size_t smem = op->smem;  // plain kernels: no epilogue prefetch (A.pf = 0)
  int grid = (op->K_active + op->E - 1) / op->E;
  if (grid == 0) return ATB_OK;
  tend_launch_fn fn = op->launch;
  if (op->persist_ctas > 0) {
    fn = op->launch_persist;
    if (grid > op->persist_ctas) grid = op->persist_ctas;
  }
  {
    ProfScope ps(op->prof_class, st);
    fn(A, grid, cta_threads(op->E, op->Np), smem, st);
  }
  return check_launch("tendency");
}

void field_ptrs(double* base, int ns, size_t stride, double** p) {
  for (int s = 0; s < 5; ++s) p[s] = base + (size_t)(s < ns ? s : 0) * stride;
}

int reduce(atb_op* op, int kind, const double* const* p, const double* const* q, double* out5, cudaStream_t st) {
  RedArgs R;
  R.K = op->K;
  R.Nq = op->Nq;
  R.Np = op->Np;
  R.naux = op->naux;
  R.kind = kind;
  R.w = op->d_w;
  R.J = op->d_J;
  R.aux = op->d_aux;
  R.law = op->law;
  R.stride = op->stride();
  for (int s = 0; s < 5; ++s) {
    R.p[s] = p[s < op->ns ? s : 0];
    R.q[s] = q ? q[s < op->ns ? s : 0] : R.p[s];
  }
  R.partials = op->d_partials;
  R.MJ = op->d_MJn;  // curved elements: per-node M J (null: weights x element Jacobian)
  {
    ProfScope ps(ATB_PROF_REDUCE, st);
    op->reducer(R, op->red_blocks, st);
  }
  int rc = check_launch("reduce");
  if (rc) return rc;
  {
    ProfScope ps(ATB_PROF_REDUCE, st);
    launch_red_finish(op->d_partials, op->red_blocks, kind == RED_LINF, op->d_red, st);
  }
  rc = check_launch("reduce finish");
  if (rc) return rc;
  CK(cudaMemcpyAsync(op->h_red, op->d_red, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int k = 0; k < 5; ++k) out5[k] = op->h_red[k];
  return ATB_OK;
}

}  // namespace

// =================================================================== op
extern "C" int atb_version(void) { return 1; }
extern "C" const char* atb_last_error(void) { return g_err.c_str(); }
extern "C" int atb_device_count(int* n) {
  CK(cudaGetDeviceCount(n));
  return ATB_OK;
}

extern "C" int atb_op_destroy(atb_op* op) {
  if (!op) return ATB_OK;
  cudaFree(op->d_ginv);
  cudaFree(op->d_nbr);
  cudaFree(op->d_aux);
  cudaFree(op->d_tab);
  cudaFree(op->d_w);
  cudaFree(op->d_J);
  cudaFree(op->d_partials);
  cudaFree(op->d_red);
  cudaFree(op->d_D);
  cudaFree(op->d_G);
  cudaFree(op->d_MJn);
  cudaFree(op->d_fnrm);
  cudaFree(op->d_fMJ);
  cudaFree(op->d_fnb);
  if (op->h_red) cudaFreeHost(op->h_red);
  for (int i = 0; i < atb_op::kGeoRing; ++i) {
    if (op->geo_ev[i]) {
      cudaEventSynchronize(op->geo_ev[i]);
      cudaEventDestroy(op->geo_ev[i]);
    }
    if (op->h_geo[i]) cudaFreeHost(op->h_geo[i]);
  }
  delete op;
  return ATB_OK;
}

namespace {

// element number of per-dimension indices idx in one instance's ordering
int elem_index(const atb_op_desc* d, const int* idx) {
  if (d->stacked) {
    int ev = idx[d->dim - 1], eh = 0, m = 1;
    for (int k = 0; k < d->dim - 1; ++k) { eh += idx[k] * m; m *= d->K[k]; }
    return eh * d->K[d->dim - 1] + ev;
  }
  int e = 0, m = 1;
  for (int k = 0; k < d->dim; ++k) { e += idx[k] * m; m *= d->K[k]; }
  return e;
}

bool same_kind(const atb_op_desc* a, const atb_op_desc* b) {
  bool ok = a->law == b->law && a->dim == b->dim && a->N == b->N && a->volume_form == b->volume_form &&
            a->volume_flux == b->volume_flux && a->surface_flux == b->surface_flux && a->directions == b->directions &&
            a->gamma == b->gamma && a->grav == b->grav && a->sphere == b->sphere &&
            a->pde_level_balance == b->pde_level_balance && a->bc_kind == b->bc_kind &&
            a->source_kind == b->source_kind && a->sw_topography == b->sw_topography && a->naux == b->naux &&
            a->precision == b->precision;
  for (int k = 0; k < 3; ++k) ok = ok && a->adv_u[k] == b->adv_u[k] && a->omega[k] == b->omega[k];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 5; ++j) ok = ok && a->bc_state[i][j] == b->bc_state[i][j];
  return ok;
}

// Geometry of one instance whose elements start at `off` in the packed
// ordering: 2/h per dimension, Jacobian determinant, neighbour table
// (neighbour element minus own element, or NBR_BOUNDARY + face number on a
// non-periodic boundary: the same wherever the instance sits), and the bottom
// element of every vertical column.  Outputs hold the instance's own elements
// only (element off + e at index e).
int instance_geometry(const atb_op_desc* di, int off, double* ginv, double* J, int* nbr, std::vector<int>* col_e0) {
  const int dim = di->dim;
  int Kd[3] = {1, 1, 1};
  for (int k = 0; k < dim; ++k) Kd[k] = di->K[k];
  if (col_e0) {
    // vertical columns (last dimension), horizontal element index fastest
    int KH = 1;
    for (int k = 0; k < dim - 1; ++k) KH *= Kd[k];
    for (int eh = 0; eh < KH; ++eh) {
      int ci[3] = {0, 0, 0}, r = eh;
      for (int k = 0; k < dim - 1; ++k) { ci[k] = r % Kd[k]; r /= Kd[k]; }
      col_e0->push_back(off + elem_index(di, ci));
    }
  }
  int idx[3];
  for (idx[2] = 0; idx[2] < Kd[2]; ++idx[2])
    for (idx[1] = 0; idx[1] < Kd[1]; ++idx[1])
      for (idx[0] = 0; idx[0] < Kd[0]; ++idx[0]) {
        const int e = elem_index(di, idx);
        double Je = 1.0;
        for (int k = 0; k < 3; ++k) ginv[e * 3 + k] = 0.0;
        for (int k = 0; k < dim; ++k) {
          const double h = di->vertices[k][idx[k] + 1] - di->vertices[k][idx[k]];
          if (!(h > 0)) return ATB_ERR_INVALID;
          ginv[e * 3 + k] = 2.0 / h;
          Je *= h / 2;
        }
        J[e] = Je;
        for (int k = 0; k < 3; ++k)
          for (int f = 0; f < 2; ++f) {
            const int face = 2 * k + f;
            if (k >= dim) { nbr[e * 6 + face] = NBR_BOUNDARY + face + 1; continue; }
            int nb[3] = {idx[0], idx[1], idx[2]};
            nb[k] += f ? 1 : -1;
            if (nb[k] < 0 || nb[k] >= Kd[k]) {
              if (di->periodic[k]) {
                nb[k] = (nb[k] + Kd[k]) % Kd[k];
              } else {
                nbr[e * 6 + face] = NBR_BOUNDARY + face + 1;  // boundary tag = face number
                continue;
              }
            }
            nbr[e * 6 + face] = elem_index(di, nb) - e;  // relative: position independent
          }
      }
  return ATB_OK;
}

// One operator over n instances that share their law, order, fluxes,
// precision and problem kinds: their elements are concatenated (instance i
// owns elements [off_i, off_i + K_i)) and every neighbour index is offset, so
// the tendency kernel -- which only sees an element list -- advances all of
// them in one launch (the instances never couple).
int op_create_impl(const atb_op_desc* descs, int n, const double* const* aux_hosts, atb_op** out,
                   bool zero_aux = false) {
  if (!descs || !out || n < 1) return fail(ATB_ERR_INVALID, "null argument");
  *out = nullptr;
  const atb_op_desc* d = &descs[0];
  if (d->dim < 1 || d->dim > 3) return fail(ATB_ERR_INVALID, "dim must be 1..3");
  if (d->N < 1 || d->N > 7) return fail(ATB_ERR_INVALID, "polynomial order N must be 1..7");
  if (d->law < 0 || d->law > 4) return fail(ATB_ERR_INVALID, "unknown law %d", d->law);
  if (d->precision != ATB_PREC_FP64 && d->precision != ATB_PREC_FP32FLUX)
    return fail(ATB_ERR_INVALID, "unknown precision %d", d->precision);
  if (!d->lgl_weights || !d->lgl_D) return fail(ATB_ERR_INVALID, "LGL tables missing");
  if (d->naux < 0 || d->naux > 8) return fail(ATB_ERR_INVALID, "naux must be 0..8");
  if ((d->directions & ((1 << d->dim) - 1)) == 0 || (d->directions >> d->dim))
    return fail(ATB_ERR_INVALID, "directions must be a non-empty subset of 1:dim");
  for (int i = 0; i < n; ++i) {
    if (i > 0 && !same_kind(d, &descs[i]))
      return fail(ATB_ERR_INVALID, "batched instance %d differs from instance 0 in law, order, fluxes, "
                                   "precision or problem kinds", i);
    if (descs[i].naux > 0 && !zero_aux && (!aux_hosts || !aux_hosts[i]))
      return fail(ATB_ERR_INVALID, "aux fields missing");
    for (int k = 0; k < d->dim; ++k) {
      if (descs[i].K[k] < 1) return fail(ATB_ERR_INVALID, "K[%d] must be >= 1", k);
      if (!descs[i].vertices[k]) return fail(ATB_ERR_INVALID, "vertex vector %d missing", k);
    }
  }
  int vk = VK_WEAK;
  if (d->volume_form == 1) {
    switch (d->volume_flux) {
      case ATB_FLUX_CENTRAL: vk = VK_CENTRAL; break;
      case ATB_FLUX_EC: vk = (d->precision == ATB_PREC_FP32FLUX) ? VK_EC32 : VK_EC; break;
      case ATB_FLUX_KG: vk = (d->precision == ATB_PREC_FP32FLUX) ? VK_KG32 : VK_KG; break;
      default: return fail(ATB_ERR_INVALID, "no two-point volume flux %d", d->volume_flux);
    }
  }
  if (d->precision == ATB_PREC_FP32FLUX &&
      !((vk == VK_EC32 && (d->law == LAW_EULER || d->law == LAW_EG || d->law == LAW_SW)) ||
        (vk == VK_KG32 && (d->law == LAW_EULER || d->law == LAW_EG))))
    return fail(ATB_ERR_INVALID,
                "the FP32-flux form exists for the flux-differencing volume term with the entropy-conservative "
                "flux (Euler, Euler-gravity, shallow water) or the Kennedy-Gruber flux (Euler, Euler-gravity)");
  tend_launch_fn fn = nullptr;
  red_launch_fn rf = nullptr;
  // a compile-time node-count specialisation when one exists, else the
  // runtime-Nq kernel
  const int nq = d->N + 1;
  switch (d->law) {
    case LAW_ADV: fn = pick_launcher_nq<LAW_ADV>(d->dim, vk, nq); if (!fn) fn = pick_launcher<LAW_ADV>(d->dim, vk); rf = pick_reducer<LAW_ADV>(d->dim); break;
    case LAW_EULER: fn = pick_launcher_nq<LAW_EULER>(d->dim, vk, nq); if (!fn) fn = pick_launcher<LAW_EULER>(d->dim, vk); rf = pick_reducer<LAW_EULER>(d->dim); break;
    case LAW_EG: fn = pick_launcher_nq<LAW_EG>(d->dim, vk, nq); if (!fn) fn = pick_launcher<LAW_EG>(d->dim, vk); rf = pick_reducer<LAW_EG>(d->dim); break;
    case LAW_LEG: fn = pick_launcher_nq<LAW_LEG>(d->dim, vk, nq); if (!fn) fn = pick_launcher<LAW_LEG>(d->dim, vk); rf = pick_reducer<LAW_LEG>(d->dim); break;
    case LAW_SW: fn = pick_launcher_nq<LAW_SW>(d->dim, vk, nq); if (!fn) fn = pick_launcher<LAW_SW>(d->dim, vk); rf = pick_reducer<LAW_SW>(d->dim); break;
  }
  if (!fn) return fail(ATB_ERR_INVALID, "unsupported (law %d, volume flux %d) combination", d->law, d->volume_flux);
  const int sf = d->surface_flux;
  if (sf == ATB_FLUX_RUSANOV) {
    // the kernel with the surface flux built in, where one is compiled
    if (tend_launch_fn fr = pick_launcher_rusanov(d->law, d->dim, vk, nq)) fn = fr;
  }
  bool sf_ok = sf == ATB_FLUX_CENTRAL || sf == ATB_FLUX_RUSANOV;
  if (d->law == LAW_EULER || d->law == LAW_EG) sf_ok = sf_ok || (sf >= ATB_FLUX_EC && sf <= ATB_FLUX_MATRIX);
  if (d->law == LAW_SW) sf_ok = sf_ok || sf == ATB_FLUX_EC || sf == ATB_FLUX_ROE;
  if (!sf_ok) return fail(ATB_ERR_INVALID, "no surface flux %d for law %d", sf, d->law);
  if (d->law == LAW_SW && d->sw_topography && d->naux < 1 + d->dim)
    return fail(ATB_ERR_INVALID, "shallow-water topography needs aux = [b, grad b]");
  if ((d->law == LAW_EG || d->law == LAW_LEG) && d->naux < 1 + d->dim)
    return fail(ATB_ERR_INVALID, "Euler-gravity laws need aux = [Phi, grad Phi, ...]");
  if ((d->law == LAW_LEG || (d->law == LAW_EG && d->pde_level_balance)) && d->naux < 3 + d->dim)
    return fail(ATB_ERR_INVALID, "this law needs the reference state in aux");

  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(ATB_ERR_CUDA, "no usable CUDA device");
  }
  atb_op* op = new atb_op();
  op->device = dev;
  op->launch = fn;
  op->reducer = rf;
  op->dim = d->dim;
  op->N = d->N;
  op->Nq = d->N + 1;
  op->Np = 1;
  for (int k = 0; k < d->dim; ++k) op->Np *= op->Nq;
  op->Nfp = op->Np / op->Nq;
  op->ninst = n;
  op->K = 0;
  std::vector<int> offs(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    int Ki = 1;
    for (int k = 0; k < d->dim; ++k) Ki *= descs[i].K[k];
    offs[i + 1] = offs[i] + Ki;
  }
  op->K = offs[n];
  op->K_active = op->K;
  op->kind = *d;
  op->inst_off = offs;
  for (int k = 0; k < 3; ++k) op->Kd[k] = k < d->dim ? d->K[k] : 1;  // instance 0
  for (int i = 1; i < n; ++i)
    for (int k = 0; k < d->dim; ++k) op->cols_uniform = op->cols_uniform && descs[i].K[k] == d->K[k];
  op->ns = (d->law == LAW_ADV) ? 1 : d->dim + 2;
  op->naux = d->naux;
  op->vk = vk;
  op->dirs = d->directions;
  op->sflux = sf;
  op->precision = d->precision;
  op->stacked = d->stacked;
  LawP& L = op->law;
  L.kind = d->law;
  L.dim = d->dim;
  L.ns = op->ns;
  L.naux = d->naux;
  L.gamma = d->gamma;
  L.grav = d->grav;
  for (int k = 0; k < 3; ++k) { L.adv_u[k] = d->adv_u[k]; L.omega[k] = d->omega[k]; }
  std::memcpy(L.bc_state, d->bc_state, sizeof(L.bc_state));
  L.pde = d->pde_level_balance;
  L.bc = d->bc_kind;
  L.src = d->source_kind;
  L.swtopo = d->sw_topography;

  const int Nq = op->Nq, Np = op->Np, K = op->K, dim = op->dim;
  op->w.assign(d->lgl_weights, d->lgl_weights + Nq);
  op->D.assign(d->lgl_D, d->lgl_D + Nq * Nq);
  // tables: Cfd[i][m] = D[m][i] w_m / w_i - D[i][m] (0 on the diagonal),
  //         Cw[i][m]  = D[m][i] w_m / w_i, lift_end = 1 / w_0
  std::vector<double> tab(2 * Nq * Nq + 2, 0.0);
  for (int i = 0; i < Nq; ++i)
    for (int m = 0; m < Nq; ++m) {
      double cw = op->D[m * Nq + i] * op->w[m] / op->w[i];
      tab[i * Nq + m] = (i == m) ? 0.0 : cw - op->D[i * Nq + m];
      tab[Nq * Nq + i * Nq + m] = cw;
    }
  tab[2 * Nq * Nq] = 1.0 / op->w[0];
  // geometry, instance by instance
  std::vector<double> ginv((size_t)K * 3, 0.0), J(K, 1.0);
  std::vector<int> nbr((size_t)K * 6, 0);
  for (int inst = 0; inst < n; ++inst) {
    const int rc = instance_geometry(&descs[inst], offs[inst], ginv.data() + (size_t)offs[inst] * 3,
                                     J.data() + offs[inst], nbr.data() + (size_t)offs[inst] * 6, &op->col_e0);
    if (rc) {
      delete op;
      return fail(rc, "vertex vectors of instance %d are not increasing", inst);
    }
  }
  // aux components the kernels read: Euler-gravity needs Phi (fluxes, wave
  // speeds), grad Phi for the weak form's non-conservative term, and the
  // reference state under pde_level_balance; the linear law needs all of
  // them; shallow-water bathymetry needs b (and grad b in the weak form)
  int nu = 0;
  if (d->law == LAW_EG) nu = d->pde_level_balance ? dim + 3 : (vk == VK_WEAK ? dim + 1 : 1);
  if (d->law == LAW_LEG) nu = dim + 3;
  if (d->law == LAW_SW && d->sw_topography) nu = (vk == VK_WEAK) ? dim + 1 : 1;
  op->naux_used = std::min(nu, op->naux);
  // launch shape: E elements per CTA, ~128 threads (>= 1 element; the
  // shape the autotuner picks on B200 for most orders); the
  // autotuner (atb_op_autotune) may pick another E
  op->npre = npre_of(d->law, dim, vk);
  op->npv = npv_stride_of(d->law, dim, vk);
  op->E = std::max(1, 128 / Np);
  while (op->E > 1 && op_smem(op, op->E) > 100 * 1024) --op->E;
  op->smem = op_smem(op, op->E);
  if (op->smem > 227 * 1024) {
    const size_t smem = op->smem;
    delete op;
    return fail(ATB_ERR_INVALID, "element too large for shared memory (%zu bytes)", smem);
  }
  op->red_blocks = 148 * 4;
  int rc;
  if ((rc = dalloc(&op->d_ginv, ginv.size())) || (rc = dalloc(&op->d_nbr, nbr.size())) ||
      (rc = dalloc(&op->d_tab, tab.size())) || (rc = dalloc(&op->d_w, (size_t)Nq)) || (rc = dalloc(&op->d_J, (size_t)K)) ||
      (rc = dalloc(&op->d_aux, (size_t)std::max(1, op->naux) * K * Np)) ||
      (rc = dalloc(&op->d_partials, (size_t)op->red_blocks * 5)) || (rc = dalloc(&op->d_red, 5))) {
    atb_op_destroy(op);
    return rc;
  }
  if (cudaMallocHost((void**)&op->h_red, 5 * sizeof(double)) != cudaSuccess) {
    op->h_red = nullptr;
    atb_op_destroy(op);
    return fail(ATB_ERR_NOMEM, "cudaMallocHost failed");
  }
  cudaError_t e1 = cudaMemcpy(op->d_ginv, ginv.data(), ginv.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaError_t e2 = cudaMemcpy(op->d_nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaError_t e3 = cudaMemcpy(op->d_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaError_t e4 = cudaMemcpy(op->d_w, op->w.data(), Nq * sizeof(double), cudaMemcpyHostToDevice);
  cudaError_t e5 = cudaMemcpy(op->d_J, J.data(), K * sizeof(double), cudaMemcpyHostToDevice);
  cudaError_t e6 = cudaSuccess;
  // aux: component-major over the concatenated elements
  if (zero_aux) e6 = cudaMemset(op->d_aux, 0, (size_t)std::max(1, op->naux) * K * Np * sizeof(double));
  for (int k = 0; k < op->naux && e6 == cudaSuccess && !zero_aux; ++k)
    for (int inst = 0; inst < n && e6 == cudaSuccess; ++inst) {
      const size_t Ki = (size_t)(offs[inst + 1] - offs[inst]);
      e6 = cudaMemcpy(op->d_aux + (size_t)k * K * Np + (size_t)offs[inst] * Np, aux_hosts[inst] + (size_t)k * Ki * Np,
                      Ki * Np * sizeof(double), cudaMemcpyHostToDevice);
    }
  if (e1 || e2 || e3 || e4 || e5 || e6) {
    atb_op_destroy(op);
    return fail(ATB_ERR_CUDA, "uploading operator tables failed");
  }
  *out = op;
  return ATB_OK;
}

}  // namespace

extern "C" int atb_op_create(const atb_op_desc* d, const double* aux_host, atb_op** out) {
  const double* aux[1] = {aux_host};
  // no aux values given: start from zeros, to be filled by atb_op_set_aux
  return op_create_impl(d, 1, aux, out, d && d->naux > 0 && !aux_host);
}

extern "C" int atb_op_set_aux(atb_op* op, const double* aux, void* stream) {
  if (!op || (!aux && op->naux > 0)) return fail(ATB_ERR_INVALID, "null argument");
  if (op->naux == 0) return ATB_OK;
  // host or device source: unified addressing picks the direction
  CK(cudaMemcpyAsync(op->d_aux, aux, (size_t)op->naux * op->stride() * sizeof(double), cudaMemcpyDefault,
                     (cudaStream_t)stream));
  return ATB_OK;
}

extern "C" int atb_op_create_curved(const atb_op_desc* d, const double* aux_host, const atb_curved_geometry* geo,
                                    atb_op** out) {
  if (!d || !geo || !out || !geo->metric || !geo->mj || !geo->normals || !geo->face_mj || !geo->nbr_node ||
      !geo->btag)
    return fail(ATB_ERR_INVALID, "null argument");
  *out = nullptr;
  if (d->dim != 3 || !d->stacked) return fail(ATB_ERR_INVALID, "curved elements: 3-D, stacked ordering");
  if (d->law != LAW_EULER && d->law != LAW_EG && d->law != LAW_LEG)
    return fail(ATB_ERR_INVALID, "curved elements: Euler, Euler-gravity or linear Euler-gravity");
  if (d->precision != ATB_PREC_FP64) return fail(ATB_ERR_INVALID, "curved elements: FP64");
  const int sf = d->surface_flux;
  if (!(sf == ATB_FLUX_CENTRAL || sf == ATB_FLUX_RUSANOV ||
        (d->law != LAW_LEG && sf >= ATB_FLUX_EC && sf <= ATB_FLUX_MATRIX)))
    return fail(ATB_ERR_INVALID, "curved elements: no surface flux %d for law %d", sf, d->law);
  if (d->bc_kind != ATB_BC_COPY && d->bc_kind != ATB_BC_REFLECT && d->bc_kind != ATB_BC_DIRICHLET)
    return fail(ATB_ERR_INVALID, "curved elements: boundary state copy, reflect or Dirichlet");
  atb_op* op = nullptr;
  int rc = op_create_impl(d, 1, &aux_host, &op, d->naux > 0 && !aux_host);
  if (rc) return rc;
  tend_launch_fn fn = pick_launcher_curved(d->law, op->vk, sf);
  if (!fn) {
    atb_op_destroy(op);
    return fail(ATB_ERR_INVALID, "curved elements: no kernel for law %d, volume flux %d", d->law, d->volume_flux);
  }
  const int Nq = op->Nq, Np = op->Np, Nfp = op->Nfp, K = op->K;
  const size_t KN = (size_t)K * Np, KF = (size_t)K * 6 * Nfp;
  if (KN > (size_t)2147483647) {
    atb_op_destroy(op);
    return fail(ATB_ERR_INVALID, "curved elements: too many nodes");
  }
  // neighbour nodes -> int (-1 - tag on a boundary face), checked
  std::vector<int> fnb(KF);
  for (size_t i = 0; i < KF; ++i) {
    const long long v = geo->nbr_node[i];
    const int tag = geo->btag[i / ((size_t)6 * Nfp) * 6 + (i / Nfp) % 6];
    if (v >= 0 && v < (long long)KN && tag == 0) {
      fnb[i] = (int)v;
    } else if (v < 0 && tag > 0) {
      fnb[i] = -1 - tag;
    } else {
      atb_op_destroy(op);
      return fail(ATB_ERR_INVALID, "curved elements: face node %zu has neighbour %lld with boundary tag %d", i, v,
                  tag);
    }
  }
  for (size_t i = 0; i < KN; ++i)
    if (!(geo->mj[i] > 0)) {
      atb_op_destroy(op);
      return fail(ATB_ERR_INVALID, "curved elements: M J must be positive");
    }
  op->curved = true;
  op->launch = fn;
  // aux the kernels read: Phi (fluxes, wave speeds), grad Phi (weak-form
  // gravity), the reference state (linear law; pde_level_balance)
  int nu = 0;
  if (d->law == LAW_EG) nu = d->pde_level_balance ? 6 : (op->vk == VK_WEAK ? 4 : 1);
  if (d->law == LAW_LEG) nu = 6;
  op->naux_used = std::min(nu, op->naux);
  op->E = std::max(1, 128 / Np);
  while (op->E > 1 && op_smem(op, op->E) > 100 * 1024) --op->E;
  op->smem = op_smem(op, op->E);
  if (op->smem > 227 * 1024 || cta_threads(op->E, Np) > 512) {
    atb_op_destroy(op);
    return fail(ATB_ERR_INVALID, "curved elements: element too large for one CTA");
  }
  if ((rc = dalloc(&op->d_D, (size_t)Nq * Nq)) || (rc = dalloc(&op->d_G, 9 * KN)) || (rc = dalloc(&op->d_MJn, KN)) ||
      (rc = dalloc(&op->d_fnrm, 3 * KF)) || (rc = dalloc(&op->d_fMJ, KF)) || (rc = dalloc(&op->d_fnb, KF))) {
    atb_op_destroy(op);
    return rc;
  }
  cudaError_t e[6] = {
      cudaMemcpy(op->d_D, op->D.data(), (size_t)Nq * Nq * sizeof(double), cudaMemcpyHostToDevice),
      cudaMemcpy(op->d_G, geo->metric, 9 * KN * sizeof(double), cudaMemcpyHostToDevice),
      cudaMemcpy(op->d_MJn, geo->mj, KN * sizeof(double), cudaMemcpyHostToDevice),
      cudaMemcpy(op->d_fnrm, geo->normals, 3 * KF * sizeof(double), cudaMemcpyHostToDevice),
      cudaMemcpy(op->d_fMJ, geo->face_mj, KF * sizeof(double), cudaMemcpyHostToDevice),
      cudaMemcpy(op->d_fnb, fnb.data(), KF * sizeof(int), cudaMemcpyHostToDevice)};
  for (int i = 0; i < 6; ++i)
    if (e[i] != cudaSuccess) {
      atb_op_destroy(op);
      return fail(ATB_ERR_CUDA, "uploading the curved geometry failed");
    }
  *out = op;
  return ATB_OK;
}

extern "C" int atb_op_create_batch(const atb_op_desc* descs, int n, const double* const* aux_hosts, atb_op** out) {
  return op_create_impl(descs, n, aux_hosts, out);
}

extern "C" int atb_op_create_pool(const atb_op_desc* kind, int capacity_elements, atb_op** out) {
  if (!kind || !out) return fail(ATB_ERR_INVALID, "null argument");
  if (capacity_elements < 1) return fail(ATB_ERR_INVALID, "capacity must be >= 1 element");
  // placeholder geometry: one row of unit elements along the first dimension
  atb_op_desc d = *kind;
  std::vector<double> v((size_t)capacity_elements + 1), u(2);
  for (int i = 0; i <= capacity_elements; ++i) v[i] = i;
  u[0] = 0;
  u[1] = 1;
  d.K[0] = capacity_elements;
  d.vertices[0] = v.data();
  for (int k = 1; k < 3; ++k) { d.K[k] = 1; d.vertices[k] = u.data(); }
  d.stacked = 0;
  const int rc = op_create_impl(&d, 1, nullptr, out, /*zero_aux=*/true);
  if (rc) return rc;
  (*out)->K_active = 0;
  (*out)->col_e0.clear();
  for (int i = 0; i < atb_op::kGeoRing; ++i)
    if (cudaEventCreateWithFlags(&(*out)->geo_ev[i], cudaEventDisableTiming) != cudaSuccess) {
      atb_op_destroy(*out);
      *out = nullptr;
      return fail(ATB_ERR_CUDA, "event creation failed");
    }
  (*out)->cols_uniform = false;  // placements have their own grids: no banded solve
  return ATB_OK;
}

extern "C" int atb_op_place_instance(atb_op* op, int first_element, const atb_op_desc* desc, const double* aux_host,
                                     void* stream) {
  if (!op || !desc) return fail(ATB_ERR_INVALID, "null argument");
  if (!same_kind(&op->kind, desc))
    return fail(ATB_ERR_INVALID, "placed instance differs from the pool in law, order, fluxes, precision or "
                                 "problem kinds");
  int Ki = 1;
  for (int k = 0; k < desc->dim; ++k) {
    if (desc->K[k] < 1 || !desc->vertices[k]) return fail(ATB_ERR_INVALID, "bad grid of placed instance");
    Ki *= desc->K[k];
  }
  if (first_element < 0 || (long)first_element + Ki > op->K)
    return fail(ATB_ERR_INVALID, "placement [%d, %ld) outside the pool's %d elements", first_element,
                (long)first_element + Ki, op->K);
  if (op->naux > 0 && !aux_host) return fail(ATB_ERR_INVALID, "aux fields missing");
  if (!op->geo_ev[0]) return fail(ATB_ERR_INVALID, "instances are placed into pools (atb_op_create_pool)");
  cudaStream_t st = (cudaStream_t)stream;
  // geometry through the next page-locked staging area of the ring: no
  // pageable copy that could block the caller behind queued work, and a wait
  // only for the copies of the placement kGeoRing placements ago (the copy
  // stream also carries every placement's aux and state)
  const int gi = op->geo_turn;
  op->geo_turn = (gi + 1) % atb_op::kGeoRing;
  const size_t gbytes = (size_t)Ki * (4 * sizeof(double) + 6 * sizeof(int));
  CK(cudaEventSynchronize(op->geo_ev[gi]));
  if (op->geo_bytes[gi] < gbytes) {
    if (op->h_geo[gi]) {
      cudaFreeHost(op->h_geo[gi]);
      op->h_geo[gi] = nullptr;
    }
    const size_t want = std::max(gbytes, (size_t)1 << 20);
    if (cudaHostAlloc(&op->h_geo[gi], want, cudaHostAllocDefault) != cudaSuccess) {
      op->h_geo[gi] = nullptr;
      op->geo_bytes[gi] = 0;
      return fail(ATB_ERR_NOMEM, "page-locked geometry staging of %zu bytes failed", want);
    }
    op->geo_bytes[gi] = want;
  }
  double* ginv = (double*)op->h_geo[gi];
  double* J = ginv + (size_t)Ki * 3;
  int* nbr = (int*)(J + Ki);
  if (instance_geometry(desc, first_element, ginv, J, nbr, nullptr))
    return fail(ATB_ERR_INVALID, "vertex vectors of the placed instance are not increasing");
  CK(cudaMemcpyAsync(op->d_ginv + (size_t)first_element * 3, ginv, (size_t)Ki * 3 * sizeof(double),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(op->d_J + first_element, J, (size_t)Ki * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(op->d_nbr + (size_t)first_element * 6, nbr, (size_t)Ki * 6 * sizeof(int),
                     cudaMemcpyHostToDevice, st));
  CK(cudaEventRecord(op->geo_ev[gi], st));
  // aux from host or device memory (unified addressing picks the direction):
  // a pageable host source is staged before the call returns; a page-locked
  // or device one is read later and must outlive the copies
  const size_t n = (size_t)Ki * op->Np;
  for (int k = 0; k < op->naux; ++k)
    CK(cudaMemcpyAsync(op->d_aux + (size_t)k * op->stride() + (size_t)first_element * op->Np, aux_host + k * n,
                       n * sizeof(double), cudaMemcpyDefault, st));
  return ATB_OK;
}

extern "C" int atb_op_move_instance(atb_op* op, int dst_first, int src_first, int n_elements, void* scratch,
                                    void* stream) {
  if (!op) return fail(ATB_ERR_INVALID, "null argument");
  const int Ki = n_elements;
  if (Ki < 0 || dst_first < 0 || src_first < 0 || (long)dst_first + Ki > op->K || (long)src_first + Ki > op->K)
    return fail(ATB_ERR_INVALID, "move outside the pool's %d elements", op->K);
  if (dst_first == src_first || Ki == 0) return ATB_OK;
  const bool overlap = std::abs(dst_first - src_first) < Ki;
  if (overlap && !scratch) return fail(ATB_ERR_INVALID, "overlapping move needs scratch");
  cudaStream_t st = (cudaStream_t)stream;
  // every per-element table is position independent (relative neighbours):
  // a move is a device copy of rows, through scratch when the ranges overlap
  auto move = [&](void* dst, const void* src, size_t bytes) -> int {
    if (overlap) {
      CK(cudaMemcpyAsync(scratch, src, bytes, cudaMemcpyDeviceToDevice, st));
      CK(cudaMemcpyAsync(dst, scratch, bytes, cudaMemcpyDeviceToDevice, st));
    } else {
      CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st));
    }
    return ATB_OK;
  };
  int rc;
  const size_t n = (size_t)Ki * op->Np;
  for (int k = 0; k < op->naux; ++k)
    if ((rc = move(op->d_aux + (size_t)k * op->stride() + (size_t)dst_first * op->Np,
                   op->d_aux + (size_t)k * op->stride() + (size_t)src_first * op->Np, n * sizeof(double))))
      return rc;
  if ((rc = move(op->d_ginv + (size_t)dst_first * 3, op->d_ginv + (size_t)src_first * 3, (size_t)Ki * 3 * sizeof(double))))
    return rc;
  if ((rc = move(op->d_J + dst_first, op->d_J + src_first, (size_t)Ki * sizeof(double)))) return rc;
  return move(op->d_nbr + (size_t)dst_first * 6, op->d_nbr + (size_t)src_first * 6, (size_t)Ki * 6 * sizeof(int));
}

extern "C" int atb_op_set_active_elements(atb_op* op, int n_elements) {
  if (!op || n_elements < 0 || n_elements > op->K) return fail(ATB_ERR_INVALID, "bad active element count");
  op->K_active = n_elements;
  return ATB_OK;
}

extern "C" int atb_op_autotune(atb_op* op, const double* const* q, double* scratch, void* stream, int* chosen) {
  // times one application per candidate E (elements per CTA) and keeps the
  // fastest; results do not depend on E (each node's arithmetic is the same)
  if (!op || !q || !scratch) return fail(ATB_ERR_INVALID, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  double* out[5];
  for (int s = 0; s < 5; ++s) out[s] = scratch + (size_t)(s < op->ns ? s : 0) * op->stride();
  const int E0 = op->E;
  int best = E0;
  float best_ms = 1e30f;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  for (int E = 1; cta_threads(E, op->Np) <= 512 && E <= 16; ++E) {
    if (op_smem(op, E) > 200 * 1024) break;
    op->E = E;
    op->smem = op_smem(op, E);
    int rc = run_tendency(op, EPI_SET, q, out, nullptr, 0, 0, st);  // warm-up
    if (rc) { op->E = E0; op->smem = op_smem(op, E0); cudaEventDestroy(a); cudaEventDestroy(b); return rc; }
    CK(cudaEventRecord(a, st));
    for (int r = 0; r < 5; ++r) run_tendency(op, EPI_SET, q, out, nullptr, 0, 0, st);
    CK(cudaEventRecord(b, st));
    CK(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best_ms) { best_ms = ms; best = E; }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  op->E = best;
  op->smem = op_smem(op, best);
  if (chosen) *chosen = best;
  return check_launch("autotune");
}

extern "C" int atb_op_set_persistent(atb_op* op, int ctas) {
  if (!op || ctas < 0) return fail(ATB_ERR_INVALID, "bad argument");
  if (ctas > 0) {
    tend_launch_fn fn = op->curved ? nullptr
                                   : pick_launcher_persistent(op->law.kind, op->dim, op->vk, op->Nq, op->sflux, false, 0);
    if (!fn)
      return fail(ATB_ERR_INVALID, "no persistent kernel for this operator (brick, Rusanov surface flux, N = 3..5: "
                                   "3-D Euler-gravity EC, 2-D Euler EC, 2-D shallow water EC / FP32-flux EC)");
    op->launch_persist = fn;
  }
  op->persist_ctas = ctas;
  return ATB_OK;
}

extern "C" int atb_op_set_launch(atb_op* op, int elements_per_cta) {
  if (!op || elements_per_cta < 1 || cta_threads(elements_per_cta, op->Np) > 512 ||
      op_smem(op, elements_per_cta) > 227 * 1024)
    return fail(ATB_ERR_INVALID, "bad elements per CTA");
  op->E = elements_per_cta;
  op->smem = op_smem(op, elements_per_cta);
  return ATB_OK;
}

extern "C" int atb_op_dims(const atb_op* op, int* ns, int* K, int* Np) {
  if (!op) return fail(ATB_ERR_INVALID, "null op");
  if (ns) *ns = op->ns;
  if (K) *K = op->K;
  if (Np) *Np = op->Np;
  return ATB_OK;
}

extern "C" int atb_op_apply(atb_op* op, double* const* dq, const double* const* q, double time, int increment,
                            void* stream) {
  (void)time;  // no time-dependent boundary or source kinds
  if (!op || !dq || !q) return fail(ATB_ERR_INVALID, "null argument");
  return run_tendency(op, increment ? EPI_ADD : EPI_SET, q, dq, nullptr, 0, 0, (cudaStream_t)stream);
}

extern "C" int atb_weightednorm(atb_op* op, const double* const* q, double p, double* comp, double* total,
                                void* stream) {
  if (!op || !q) return fail(ATB_ERR_INVALID, "null argument");
  const bool inf = std::isinf(p);
  if (!inf && p != 2) return fail(ATB_ERR_INVALID, "weightednorm supports p = 2 and p = Inf");
  double r[5];
  int rc = reduce(op, inf ? RED_LINF : RED_L2, q, nullptr, r, (cudaStream_t)stream);
  if (rc) return rc;
  double tot = 0, m = 0;
  for (int s = 0; s < op->ns; ++s) {
    double v = inf ? r[s] : std::sqrt(r[s]);
    if (comp) comp[s] = v;
    tot += v * v;
    m = std::max(m, v);
  }
  if (total) *total = inf ? m : std::sqrt(tot);
  return ATB_OK;
}

extern "C" int atb_entropyintegral(atb_op* op, const double* const* q, double* out, void* stream) {
  if (!op || !q || !out) return fail(ATB_ERR_INVALID, "null argument");
  double r[5];
  int rc = reduce(op, RED_ENTROPY, q, nullptr, r, (cudaStream_t)stream);
  *out = r[0];
  return rc;
}

extern "C" int atb_entropyproduct(atb_op* op, const double* const* p, const double* const* q, double* out,
                                  void* stream) {
  if (!op || !p || !q || !out) return fail(ATB_ERR_INVALID, "null argument");
  double r[5];
  int rc = reduce(op, RED_ENTPROD, p, q, r, (cudaStream_t)stream);
  *out = r[0];
  return rc;
}

extern "C" int atb_check_finite(atb_op* op, const double* const* q, void* stream) {
  if (!op || !q) return fail(ATB_ERR_INVALID, "null argument");
  double r[5];
  int rc = reduce(op, RED_NONFINITE, q, nullptr, r, (cudaStream_t)stream);
  if (rc) return rc;
  if (r[0] != 0) return fail(ATB_ERR_NONFINITE, "%g non-finite values in state", r[0]);
  return ATB_OK;
}

extern "C" int atb_profile_enable(int on) {
  g_prof.on = on != 0;
  return ATB_OK;
}
extern "C" int atb_profile_reset(void) {
  g_prof.resolve();
  for (int k = 0; k < NPROF; ++k) { g_prof.n[k] = 0; g_prof.ms[k] = 0; }
  return ATB_OK;
}
extern "C" int atb_profile_read(int kclass, long* launches, double* total_ms) {
  if (kclass < 0 || kclass >= NPROF) return fail(ATB_ERR_INVALID, "profile class %d", kclass);
  g_prof.resolve();
  if (launches) *launches = g_prof.n[kclass];
  if (total_ms) *total_ms = g_prof.ms[kclass];
  return ATB_OK;
}
extern "C" int atb_launch_count(long* n) {
  if (!n) return fail(ATB_ERR_INVALID, "null argument");
  *n = g_prof.launches_total;
  return ATB_OK;
}

extern "C" int atb_probe_fp64_peak(double* tflops, void* stream) {
  if (!tflops) return fail(ATB_ERR_INVALID, "null argument");
  *tflops = probe_fp64_tflops((cudaStream_t)stream);
  return check_launch("fp64 probe");
}

// =============================================================== solvers
struct atb_solver {
  int kind = 0;
  atb_op* rhs = nullptr;
  atb_op* lin = nullptr;
  atb_op* any = nullptr;
  double dt = 0, time = 0, gamma_r = 1;
  int split_rhs = 1;
  int ns = 0;
  size_t stride = 0;
  std::vector<double> rka, rkb, rkc, rkb_full;
  double exa[3][3], ima[3][3], exb[3], imb[3], exc[3], imc[3];
  double* dq = nullptr;  // LSRK: dq; RLSRK: dq
  double* qB = nullptr;  // LSRK double buffer; RLSRK: q0
  double* kb = nullptr;  // RLSRK: k
  double* Qs = nullptr;  // ARK: 2 stage states
  double* exK = nullptr; // ARK: 3
  double* imK = nullptr; // ARK: 3
  // banded operator
  LineMap M{};
  int* d_e0 = nullptr;
  double* band = nullptr;
  double* blk = nullptr;
  double* frag = nullptr;
  int ld = 0;
  // ARK23 stages fused into one kernel per stage (explicit tendency + linear
  // operator), when the two operators allow it (atb_solver_fuse)
  tend_launch_fn fused = nullptr;
  bool fuse_on = false;
  int lines_sparse = 0;  // per-line factors couple elements through face nodes only
  // per-element time steps (LSRK over packed instances), or null; owned by
  // the solver (atb_solver_set_instance_dt) or by the caller
  double* d_dte = nullptr;
  bool own_dte = false;
  // after_stage (src/odesolvers.jl:10-11,23): host callback between stages
  atb_stage_callback stage_cb = nullptr;
  void* stage_user = nullptr;
  atb_exchange_callback xchg_cb = nullptr;  // before every tendency of a new state
  void* xchg_user = nullptr;
};

namespace {

void solver_free(atb_solver* s) {
  cudaFree(s->dq);
  cudaFree(s->qB);
  cudaFree(s->kb);
  cudaFree(s->Qs);
  cudaFree(s->exK);
  cudaFree(s->imK);
  cudaFree(s->d_e0);
  cudaFree(s->band);
  cudaFree(s->blk);
  cudaFree(s->frag);
  if (s->own_dte) cudaFree(s->d_dte);
  delete s;
}

void coeffs_lsrk54(atb_solver* s) {
  // Carpenter-Kennedy LSRK(5,4) (src/odesolvers.jl:148-174), rationals rounded once
  s->rka = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
            -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
  s->rkb = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
            1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
            2277821191437.0 / 14882151754819.0};
  s->rkc = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
            2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};
}

void coeffs_lsrk144(atb_solver* s) {
  // Niegemann-Diehl-Busch LSRK(14,4) (src/odesolvers.jl:176-229)
  s->rka = {0, -0.7188012108672410, -0.7785331173421570, -0.0053282796654044, -0.8552979934029281,
            -3.9564138245774565, -1.5780575380587385, -2.0837094552574054, -0.7483334182761610,
            -0.7032861106563359, 0.0013917096117681, -0.0932075369637460, -0.9514200470875948,
            -7.1151571693922548};
  s->rkb = {0.0367762454319673, 0.3136296607553959, 0.1531848691869027, 0.0030097086818182,
            0.3326293790646110, 0.2440251405350864, 0.3718879239592277, 0.6204126221582444,
            0.1524043173028741, 0.0760894927419266, 0.0077604214040978, 0.0024647284755382,
            0.0780348340049386, 5.5059777270269628};
  s->rkc = {0, 0.0367762454319673, 0.1249685262725025, 0.2446177702277698, 0.2476149531070420,
            0.2969311120382472, 0.3978149645802642, 0.5270854589440328, 0.6981269994175695,
            0.8190890835352128, 0.8527059887098624, 0.8604711817462826, 0.8627060376969976,
            0.8734213127600976};
}

int copy_field(double* const* dst, const double* const* src, int ns, size_t n, cudaStream_t st) {
  for (int s = 0; s < ns; ++s)
    CK(cudaMemcpyAsync(dst[s], src[s], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return ATB_OK;
}

int build_band(atb_solver* s, cudaStream_t st) {
  atb_op* L = s->lin;
  const int dim = L->dim, Nq = L->Nq, ns = L->ns;
  if (!(L->dirs == (1 << (dim - 1))))
    return fail(ATB_ERR_INVALID, "the implicit operator must act along the last dimension only");
  LineMap& M = s->M;
  M.Nq = Nq;
  M.ns = ns;
  M.Np = L->Np;
  M.nh = L->Np / Nq;
  if (!L->cols_uniform)
    return fail(ATB_ERR_INVALID, "packed instances of an implicit operator must share their element counts");
  M.KV = L->Kd[dim - 1];
  M.KH = L->K / M.KV;
  M.nlines = M.KH * M.nh;
  M.nunk = M.KV * Nq * ns;
  M.bw = Nq * ns - 1;
  M.stride = L->stride();
  M.stacked = L->stacked;
  if (M.bw >= 64) return fail(ATB_ERR_INVALID, "banded bandwidth too large");
  // element index of the bottom element of each horizontal stack
  std::vector<int> e0(M.nlines);
  for (int eh = 0; eh < M.KH; ++eh)
    for (int hn = 0; hn < M.nh; ++hn) e0[eh * M.nh + hn] = L->col_e0[eh];
  // vertical neighbours: next element in a stacked instance, next layer
  // (the instance's horizontal count) otherwise
  M.estep = L->stacked ? 1 : M.KH / L->ninst;
  int rc;
  if ((rc = dalloc(&s->d_e0, (size_t)M.nlines))) return rc;
  CK(cudaMemcpy(s->d_e0, e0.data(), e0.size() * sizeof(int), cudaMemcpyHostToDevice));
  M.e0 = s->d_e0;
  const int W = 2 * M.bw + 1;
  double *P = nullptr, *LP = nullptr;
  const size_t fsz = (size_t)ns * M.stride;
  if ((rc = dalloc(&P, fsz))) return rc;
  if ((rc = dalloc(&LP, fsz))) { cudaFree(P); return rc; }
  double *pp[5], *lp[5];
  field_ptrs(P, ns, M.stride, pp);
  field_ptrs(LP, ns, M.stride, lp);
  auto probe_all = [&](auto&& extract) -> int {
    CK(cudaMemsetAsync(P, 0, fsz * sizeof(double), st));
    int r = ATB_OK;
    for (int c = 0; c < W && r == ATB_OK; ++c) {
      launch_probe_fill(M, c, pp, st);
      r = run_tendency(L, EPI_SET, pp, lp, nullptr, 0, 0, st);
      if (!r) extract(c);
    }
    return r;
  };
  // pass 1: line 0's band, and whether every column's probed operator is
  // bitwise the same (horizontally uniform problems) -> one shared factor
  double* one = nullptr;
  int* d_nd = nullptr;
  const size_t rs = 2 * (size_t)(M.bw + 1);
  double* band1 = nullptr;
  if ((rc = dalloc(&band1, (size_t)M.nunk * W)) || (rc = dalloc(&d_nd, 1))) {
    cudaFree(P); cudaFree(LP); cudaFree(band1);
    return rc;
  }
  CK(cudaMemsetAsync(band1, 0, (size_t)M.nunk * W * sizeof(double), st));
  CK(cudaMemsetAsync(d_nd, 0, sizeof(int), st));
  rc = probe_all([&](int c) { launch_band_extract_first(M, c, lp, band1, d_nd, st); });
  int nd = 1;
  if (!rc) {
    CK(cudaMemcpyAsync(&nd, d_nd, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  cudaFree(d_nd);
  const double scale = -s->dt * s->ima[2][2];  // M = I - dt a_ii L (src/odesolvers.jl:264-268)
  if (!rc && nd == 0) {
    cudaFree(P);
    cudaFree(LP);
    if ((rc = dalloc(&one, (size_t)M.nunk * rs))) { cudaFree(band1); return rc; }
    LineMap M1 = M;
    M1.nlines = 1;  // band1 holds one line
    launch_band_compact(M1, band1, one, st);
    launch_band_factor(M.nunk, M.bw, 1, one, (int)rs, 1, scale, st);
    CK(cudaStreamSynchronize(st));
    cudaFree(band1);
    s->band = one;
    s->ld = 1;
    // per-element inverses for the block-parallel solve
    const int BW1 = M.bw + 1;
    if ((rc = dalloc(&s->blk, (size_t)M.KV * 4 * BW1 * BW1))) return rc;
    launch_block_prep(s->band, M.KV, BW1, s->blk, st);
    // the tile-sparse warp-owned solve, when the blocks have its zero structure
    // (vertical coupling through face nodes only); ATB_BAND_DENSE=1 in the
    // environment keeps the dense-block kernel (the tests compare the two)
    std::vector<double> hblk((size_t)M.KV * 4 * BW1 * BW1);
    CK(cudaMemcpyAsync(hblk.data(), s->blk, hblk.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const char* dense = std::getenv("ATB_BAND_DENSE");
    if (!(dense && dense[0] == '1') && warp_solve_structure_ok(hblk.data(), M.KV, BW1, M.ns)) {
      if ((rc = dalloc(&s->frag, frag_doubles(M.KV, BW1, M.ns)))) return rc;
      launch_frag_prep(s->blk, M.KV, BW1, M.ns, s->frag, st);
    }
    CK(cudaStreamSynchronize(st));
  } else if (!rc) {
    // pass 2: columns differ -> one band and one factor per line
    cudaFree(band1);
    const size_t bandn = (size_t)M.nlines * M.nunk * W;
    if ((rc = dalloc(&s->band, bandn))) { cudaFree(P); cudaFree(LP); return rc; }
    CK(cudaMemsetAsync(s->band, 0, bandn * sizeof(double), st));
    rc = probe_all([&](int c) { launch_band_extract(M, c, lp, s->band, st); });
    cudaFree(P);
    cudaFree(LP);
    if (rc) return rc;
    launch_band_factor(M.nunk, M.bw, M.nlines, s->band, W, M.nlines, scale, st);
    s->ld = M.nlines;
    // the face-node coupling structure of every line's factor lets the solve
    // skip the zero blocks (ATB_BAND_DENSE=1 keeps the full band)
    int* d_bad = nullptr;
    if ((rc = dalloc(&d_bad, 1))) return rc;
    CK(cudaMemsetAsync(d_bad, 0, sizeof(int), st));
    launch_band_lines_structure(M, s->band, d_bad, st);
    int bad = 1;
    CK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    cudaFree(d_bad);
    const char* dense = std::getenv("ATB_BAND_DENSE");
    s->lines_sparse = (bad == 0 && !(dense && dense[0] == '1')) ? 1 : 0;
  } else {
    cudaFree(P);
    cudaFree(LP);
    cudaFree(band1);
    return rc;
  }
  if ((rc = check_launch("band factor"))) return rc;
  return ATB_OK;
}

// ------------------------------------------------------------ one step
// after_stage: the stage's launches are enqueued on st; the callback runs on
// the host and orders its own device work on st (or synchronises)
int call_stage(atb_solver* s, double ex_time, double im_time, double* const* qs) {
  double* p[5];
  for (int c = 0; c < 5; ++c) p[c] = qs[c < s->ns ? c : 0];
  const int r = s->stage_cb(ex_time, im_time, p, s->stage_user);
  if (r != 0) return fail(ATB_ERR_CALLBACK, "stage callback returned %d", r);
  return ATB_OK;
}

// the exchange hook: the state every tendency of the next launch reads,
// before that launch is enqueued (a sharded run fills its ghost elements)
int call_exchange(atb_solver* s, double* const* qs) {
  if (!s->xchg_cb) return ATB_OK;
  double* p[5];
  for (int c = 0; c < 5; ++c) p[c] = qs[c < s->ns ? c : 0];
  const int r = s->xchg_cb(p, s->xchg_user);
  if (r != 0) return fail(ATB_ERR_CALLBACK, "exchange callback returned %d", r);
  return ATB_OK;
}

// LSRK stages with a stage callback: the stage kernel writes the new state to
// qB and it is copied back into q before the callback, so the callback always
// sees (and may change) the caller's q, and the next stage starts from it.
// The arithmetic is that of lsrk_steps.
int lsrk_steps_cb(atb_solver* s, double* const* q, int nsteps, cudaStream_t st) {
  atb_op* op = s->rhs;
  double *dq[5], *qb[5], *cur[5];
  field_ptrs(s->dq, s->ns, s->stride, dq);
  field_ptrs(s->qB, s->ns, s->stride, qb);
  for (int k = 0; k < 5; ++k) cur[k] = q[k < s->ns ? k : 0];
  for (int n = 0; n < nsteps; ++n) {
    for (size_t i = 0; i < s->rka.size(); ++i) {
      int rc = call_exchange(s, cur);
      if (rc) return rc;
      rc = s->d_dte ? run_tendency(op, EPI_LSRK, cur, dq, qb, s->rka[i], s->rkb[i], st, s->d_dte)
                    : run_tendency(op, EPI_LSRK, cur, dq, qb, s->rka[i], s->rkb[i] * s->dt, st);
      if (rc) return rc;
      if ((rc = copy_field(q, qb, s->ns, (size_t)op->K_active * op->Np, st))) return rc;
      const double t = s->time + s->rkc[i] * s->dt;
      if ((rc = call_stage(s, t, t, q))) return rc;
    }
    s->time += s->dt;
  }
  return ATB_OK;
}

int lsrk_steps(atb_solver* s, double* const* q, int nsteps, cudaStream_t st) {
  if (s->stage_cb) return lsrk_steps_cb(s, q, nsteps, st);
  atb_op* op = s->rhs;
  double *dq[5], *qb[5], *cur[5], *oth[5];
  field_ptrs(s->dq, s->ns, s->stride, dq);
  field_ptrs(s->qB, s->ns, s->stride, qb);
  for (int k = 0; k < 5; ++k) { cur[k] = q[k < s->ns ? k : 0]; oth[k] = qb[k]; }
  bool in_user = true;
  for (int n = 0; n < nsteps; ++n) {
    for (size_t st_ = 0; st_ < s->rka.size(); ++st_) {
      int rc = call_exchange(s, cur);
      if (rc) return rc;
      rc = s->d_dte ? run_tendency(op, EPI_LSRK, cur, dq, oth, s->rka[st_], s->rkb[st_], st, s->d_dte)
                    : run_tendency(op, EPI_LSRK, cur, dq, oth, s->rka[st_], s->rkb[st_] * s->dt, st);
      if (rc) return rc;
      for (int k = 0; k < 5; ++k) std::swap(cur[k], oth[k]);
      in_user = !in_user;
    }
    s->time += s->dt;
  }
  // an odd number of stages leaves the state in qB: copy back the active
  // elements (the kernel writes no others)
  if (!in_user) return copy_field(q, cur, s->ns, (size_t)op->K_active * op->Np, st);
  return ATB_OK;
}

int rlsrk_step(atb_solver* s, double* const* q, cudaStream_t st) {
  atb_op* op = s->rhs;
  double *dq[5], *q0[5], *k[5];
  field_ptrs(s->dq, s->ns, s->stride, dq);
  field_ptrs(s->qB, s->ns, s->stride, q0);
  field_ptrs(s->kb, s->ns, s->stride, k);
  int rc = copy_field(q0, q, s->ns, s->stride, st);
  if (rc) return rc;
  double eta0 = 0, deta = -0.0;
  if ((rc = atb_entropyintegral(op, q0, &eta0, st))) return rc;
  for (size_t i = 0; i < s->rka.size(); ++i) {
    if ((rc = call_exchange(s, q))) return rc;
    if ((rc = run_tendency(op, EPI_RLSRK, q, k, dq, s->rka[i], 0, st))) return rc;
    double ep = 0;
    if ((rc = atb_entropyproduct(op, q, k, &ep, st))) return rc;
    deta = deta + s->rkb_full[i] * s->dt * ep;
    Axpy A{};
    A.ns = s->ns;
    A.n = s->stride;
    A.c = s->rkb[i] * s->dt;
    for (int c = 0; c < 5; ++c) { A.x[c] = q[c < s->ns ? c : 0]; A.y[c] = dq[c]; A.out[c] = q[c < s->ns ? c : 0]; }
    {
      ProfScope ps(ATB_PROF_COMBINE, st);
      launch_axpy(A, st);
    }
    if ((rc = check_launch("axpy"))) return rc;
    if (s->stage_cb) {
      const double t = s->time + s->rkc[i] * s->dt;
      if ((rc = call_stage(s, t, t, q))) return rc;
    }
  }
  // k = q - q0
  {
    Axpy A{};
    A.ns = s->ns;
    A.n = s->stride;
    A.c = -1.0;
    for (int c = 0; c < 5; ++c) { A.x[c] = q[c < s->ns ? c : 0]; A.y[c] = q0[c]; A.out[c] = k[c]; }
    ProfScope ps(ATB_PROF_COMBINE, st);
    launch_axpy(A, st);
  }
  auto setq = [&](double g) {
    Axpy A{};
    A.ns = s->ns;
    A.n = s->stride;
    A.c = g;
    for (int c = 0; c < 5; ++c) { A.x[c] = q0[c]; A.y[c] = k[c]; A.out[c] = q[c < s->ns ? c : 0]; }
    {
      ProfScope ps(ATB_PROF_COMBINE, st);
      launch_axpy(A, st);
    }
    return check_launch("axpy");
  };
  auto resid = [&](double g, double* r) {
    int e = setq(g);
    if (e) return e;
    double eta = 0;
    e = atb_entropyintegral(op, q, &eta, st);
    *r = eta - eta0 - g * deta;
    return e;
  };
  auto jac = [&](double g, double* J) {
    int e = setq(g);
    if (e) return e;
    double ep = 0;
    e = atb_entropyproduct(op, q, k, &ep, st);
    *J = ep - deta;
    return e;
  };
  // NLsolve trust region (autoscale, factor 1, eta 1e-4, ftol 10 eps, xtol 0)
  const double ftol = 10 * 2.220446049250313e-16;
  double g = s->gamma_r, r = 0;
  if ((rc = resid(g, &r))) return rc;
  if (!(std::fabs(r) <= ftol)) {
    double J = 0;
    if ((rc = jac(g, &J))) return rc;
    double Dsc = std::fabs(J) > 0 ? std::fabs(J) : 1.0;
    double delta = std::fabs(Dsc * g) > 0 ? std::fabs(Dsc * g) : 1.0;
    for (int it = 0; it < 1000; ++it) {
      if (!(J != 0) || !std::isfinite(J)) break;
      double p = -r / J;
      if (std::fabs(Dsc * p) > delta) p = (p > 0 ? delta : -delta) / Dsc;
      double gn = g + p, rn = 0;
      if ((rc = resid(gn, &rn))) return rc;
      double rp = r + J * p;
      double rho = (r * r - rn * rn) / (r * r - rp * rp);
      bool conv = false;
      if (rho > 1e-4) {
        g = gn;
        r = rn;
        if ((rc = jac(g, &J))) return rc;
        Dsc = std::max(0.1 * Dsc, std::fabs(J));
        conv = (p == 0) || std::fabs(r) <= ftol;
      }
      double np_ = std::fabs(Dsc * p);
      if (rho < 0.1)
        delta = delta / 2;
      else if (rho >= 0.9)
        delta = 2 * np_;
      else if (rho >= 0.5)
        delta = std::max(delta, 2 * np_);
      if (conv || !(delta > 0)) break;
    }
  }
  s->gamma_r = g;
  if ((rc = setq(g))) return rc;
  s->time += s->dt;
  return ATB_OK;
}

// ARK23 with split_rhs = false and the banded implicit solve, accumulated:
// stage i's linear-operator launch (EPI_ARK) turns N(Q_i) and L(Q_i) into the
// stage's explicit / implicit tendencies in registers and adds them straight
// into the right-hand sides of the later stages and into the final update, so
// no stage tendency is ever stored, the banded solve reads one ready
// right-hand side, and no separate combination kernel runs.  The additions
// happen in the same order as in ark_step, so the results are identical.
// one fused ARK stage launch: explicit tendency and linear operator of Q in
// one pass, EPI_ARK accumulation (atb_tendency.cuh, FUSE = true)
int run_fused(atb_solver* s, double* const* Q, const ArkAcc& ark, cudaStream_t st) {
  atb_op* op = s->rhs;
  TendArgs A;
  fill_args(op, A);
  const int naux = op->dim + 3;  // [Phi, grad Phi, rho_ref, p_ref] staged for both operators
  A.naux = naux;
  int E = op->E;
  if (op->curved) {
    // curved elements: the explicit operator's launch shape, no prefetch
    while (E > 1 && curved_smem_bytes(op->vk, naux, op->Nq, E, true) > 200 * 1024) --E;
    const size_t bytes = curved_smem_bytes(op->vk, naux, op->Nq, E, true);
    if (bytes > 227 * 1024) return fail(ATB_ERR_INVALID, "element too large for the fused curved ARK stage kernel");
    A.E = E;
    A.pf = 0;
    A.epi = EPI_ARK;
    A.lin_law = s->lin->law;
    A.lin_sflux = s->lin->sflux;
    A.lin_dirs = s->lin->dirs;
    for (int j = 0; j < 3; ++j) {
      for (int c = 0; c < 5; ++c) { A.acc[j][c] = ark.acc[j][c]; A.accin[j][c] = ark.accin[j][c]; }
      A.ca[j] = ark.ca[j];
      A.cb[j] = ark.cb[j];
    }
    A.adt = ark.adt;
    for (int c = 0; c < 5; ++c) {
      A.q[c] = Q[c];
      A.out[c] = Q[c];  // not read by the fused epilogue
      A.out2[c] = nullptr;
    }
    const int grid = (op->K_active + E - 1) / E;
    if (grid == 0) return ATB_OK;
    {
      ProfScope ps(ATB_PROF_TEND, st);
      s->fused(A, grid, cta_threads(E, op->Np), bytes, st);
    }
    return check_launch("fused curved ARK stage");
  }
  int pf = 0;
  for (int j = 0; j < 3; ++j) pf += (ark.acc[j][0] && ark.accin[j][0]) ? 1 : 0;
  // the compact layout of the Nq-specialised kernels (atb_tendency.cuh)
  const bool cmp = op->Nq >= 3 && op->Nq <= 8 && fused_compact_fits(op->Nq, op->dim, op->ns, op->npre, op->npv);
  auto bytes = [&](int e) {
    return tend_smem_bytes(op->ns, op->npre, naux, op->dim, op->Nq, op->Np, op->Nfp, e, op->npv, true, pf, cmp);
  };
  // fused kernels are compiled for fused_max_threads per CTA
  const int maxthr = fused_max_threads(op->Nq, cmp);
  while (E > 1 && (cta_threads(E, op->Np) > maxthr || bytes(E) > 100 * 1024)) --E;
  if (cta_threads(E, op->Np) > maxthr) return fail(ATB_ERR_INVALID, "element too large for the fused ARK stage kernel");
  if (pf && bytes(E) > 227 * 1024) {
    pf = 0;  // no room: the epilogue reads its accumulators directly
  }
  A.E = E;
  A.pf = pf;
  A.epi = EPI_ARK;
  A.lin_law = s->lin->law;
  A.lin_sflux = s->lin->sflux;
  A.lin_dirs = s->lin->dirs;
  for (int j = 0; j < 3; ++j) {
    for (int c = 0; c < 5; ++c) { A.acc[j][c] = ark.acc[j][c]; A.accin[j][c] = ark.accin[j][c]; }
    A.ca[j] = ark.ca[j];
    A.cb[j] = ark.cb[j];
  }
  A.adt = ark.adt;
  for (int c = 0; c < 5; ++c) {
    A.q[c] = Q[c];
    A.out[c] = Q[c];  // not read by the fused epilogue
    A.out2[c] = nullptr;
  }
  int grid = (op->K_active + E - 1) / E;
  if (grid == 0) return ATB_OK;
  tend_launch_fn fn = s->fused;
  if (op->persist_ctas > 0) {
    // the persistent fused stage kernel, where one is compiled
    if (tend_launch_fn fp = pick_launcher_persistent(op->law.kind, op->dim, op->vk, op->Nq, op->sflux, true,
                                                     s->lin->sflux)) {
      fn = fp;
      if (grid > op->persist_ctas) grid = op->persist_ctas;
    }
  }
  {
    ProfScope ps(ATB_PROF_TEND, st);
    fn(A, grid, cta_threads(E, op->Np), bytes(E), st);
  }
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess)
    return fail(ATB_ERR_CUDA, "fused ARK stage launch (%d elements of %d nodes per CTA, %zu bytes of shared memory): %s",
                E, op->Np, bytes(E), cudaGetErrorString(le));
  return ATB_OK;
}

int ark_step_accumulated(atb_solver* s, double* const* q, cudaStream_t st) {
  const int ns = s->ns;
  const size_t n = s->stride;
  double *N[5], *R1[5], *R2[5], *F[5];
  field_ptrs(s->exK, ns, n, N);
  field_ptrs(s->imK, ns, n, R1);
  field_ptrs(s->imK + (size_t)ns * n, ns, n, R2);
  field_ptrs(s->imK + (size_t)2 * ns * n, ns, n, F);
  double* qq[5];
  for (int k = 0; k < 5; ++k) qq[k] = q[k < ns ? k : 0];
  auto acc_clear = [](ArkAcc& a) {
    for (int j = 0; j < 3; ++j) {
      for (int c = 0; c < 5; ++c) { a.acc[j][c] = nullptr; a.accin[j][c] = nullptr; }
      a.ca[j] = a.cb[j] = 0.0;
    }
  };
  auto set = [&](ArkAcc& a, int j, double* const* dst, double* const* src, double ca, double cb) {
    for (int c = 0; c < 5; ++c) {
      a.acc[j][c] = dst[c];
      a.accin[j][c] = src ? src[c] : nullptr;
    }
    a.ca[j] = ca;
    a.cb[j] = cb;
  };
  auto solve = [&](double* const* R, double* const* Qout) -> int {
    BandSolve B{};
    B.M = s->M;
    B.band = s->band;
    B.blk = s->blk;
    B.frag = s->frag;
    B.ld = s->ld;
    B.lines_sparse = s->lines_sparse;
    B.npairs = 0;
    B.dt = s->dt;
    for (int c = 0; c < 5; ++c) { B.q[c] = R[c]; B.out[c] = Qout[c]; }
    {
      ProfScope ps(ATB_PROF_BAND, st);
      launch_band_solve(B, st);
    }
    return check_launch("band solve");
  };
  int rc;
  ArkAcc a;
  // one stage: N(Q) then L(Q) with the accumulation, or both in one launch
  auto stage = [&](double* const* Q) -> int {
    int r;
    if ((r = call_exchange(s, Q))) return r;
    if (s->fuse_on) return run_fused(s, Q, a, st);
    if ((r = run_tendency(s->rhs, EPI_SET, Q, N, nullptr, 0, 0, st))) return r;
    return run_tendency(s->lin, EPI_ARK, Q, N, nullptr, 0, 0, st, nullptr, &a);
  };
  // stage 1 (Q = q): R1, R2, F from q
  acc_clear(a);
  a.adt = s->dt;
  set(a, 0, R1, nullptr, s->exa[1][0], s->ima[1][0]);
  set(a, 1, R2, nullptr, s->exa[2][0], s->ima[2][0]);
  set(a, 2, F, nullptr, s->exb[0], s->imb[0]);
  if ((rc = stage(qq))) return rc;
  // stage 2.  The solves run in place (Q1 over R1, Q2 over R2): every band
  // kernel reads an element's right-hand side before it writes that element's
  // solution, and the step then touches four state-sized arrays plus the aux
  // fields instead of six -- at C2 107 MB, inside the 126 MB L2
  if ((rc = solve(R1, R1))) return rc;
  acc_clear(a);
  a.adt = s->dt;
  set(a, 0, R2, R2, s->exa[2][1], s->ima[2][1]);
  set(a, 1, F, F, s->exb[1], s->imb[1]);
  if ((rc = stage(R1))) return rc;
  if (s->stage_cb && (rc = call_stage(s, s->time + s->exc[1] * s->dt, s->time + s->imc[1] * s->dt, R1))) return rc;
  // stage 3 and the update of q
  if ((rc = solve(R2, R2))) return rc;
  acc_clear(a);
  a.adt = s->dt;
  set(a, 0, qq, F, s->exb[2], s->imb[2]);
  if ((rc = stage(R2))) return rc;
  // (the final update of q is accumulated by this stage's launch, so a
  // callback that looks at q here already sees the step's result)
  if (s->stage_cb && (rc = call_stage(s, s->time + s->exc[2] * s->dt, s->time + s->imc[2] * s->dt, R2))) return rc;
  s->time += s->dt;
  return ATB_OK;
}

int ark_step(atb_solver* s, double* const* q, cudaStream_t st) {
  if (s->rhs && s->lin && !s->split_rhs && s->band) return ark_step_accumulated(s, q, st);
  const int ns = s->ns;
  const size_t n = s->stride;
  double *Q[3][5], *ex[3][5], *im[3][5];
  for (int k = 0; k < 5; ++k) Q[0][k] = q[k < ns ? k : 0];
  field_ptrs(s->Qs, ns, n, Q[1]);
  field_ptrs(s->Qs + (size_t)ns * n, ns, n, Q[2]);
  for (int i = 0; i < 3; ++i) {
    field_ptrs(s->exK + (size_t)i * ns * n, ns, n, ex[i]);
    field_ptrs(s->imK + (size_t)i * ns * n, ns, n, im[i]);
  }
  auto eval = [&](int i) -> int {
    int rc;
    if ((rc = call_exchange(s, Q[i]))) return rc;
    if (s->rhs) {
      if ((rc = run_tendency(s->rhs, EPI_SET, Q[i], ex[i], nullptr, 0, 0, st))) return rc;
    } else {
      for (int c = 0; c < ns; ++c) CK(cudaMemsetAsync(ex[i][c], 0, n * sizeof(double), st));
    }
    if (s->lin) {
      if (!s->split_rhs)
        rc = run_tendency(s->lin, EPI_SUBOUT2, Q[i], im[i], ex[i], 0, 0, st);
      else
        rc = run_tendency(s->lin, EPI_SET, Q[i], im[i], nullptr, 0, 0, st);
      if (rc) return rc;
    } else {
      for (int c = 0; c < ns; ++c) CK(cudaMemsetAsync(im[i][c], 0, n * sizeof(double), st));
    }
    return ATB_OK;
  };
  int rc = eval(0);
  if (rc) return rc;
  for (int i = 1; i < 3; ++i) {
    if (s->lin) {
      BandSolve B{};
      B.M = s->M;
      B.band = s->band;
      B.blk = s->blk;
      B.frag = s->frag;
      B.ld = s->ld;
      B.lines_sparse = s->lines_sparse;
      B.npairs = i;
      B.dt = s->dt;
      for (int k = 0; k < i; ++k) {
        B.a[k] = s->exa[i][k];
        B.b[k] = s->ima[i][k];
        for (int c = 0; c < 5; ++c) { B.ex[k][c] = ex[k][c]; B.im[k][c] = im[k][c]; }
      }
      for (int c = 0; c < 5; ++c) { B.q[c] = q[c < ns ? c : 0]; B.out[c] = Q[i][c]; }
      {
        ProfScope ps(ATB_PROF_BAND, st);
        launch_band_solve(B, st);
      }
      if ((rc = check_launch("band solve"))) return rc;
    } else {
      LinComb C{};
      C.ns = ns;
      C.n = n;
      C.npairs = i;
      C.dt = s->dt;
      for (int k = 0; k < i; ++k) {
        C.a[k] = s->exa[i][k];
        C.b[k] = s->ima[i][k];
        for (int c = 0; c < 5; ++c) { C.X[k][c] = ex[k][c]; C.Y[k][c] = im[k][c]; }
      }
      for (int c = 0; c < 5; ++c) { C.base[c] = q[c < ns ? c : 0]; C.out[c] = Q[i][c]; }
      {
        ProfScope ps(ATB_PROF_COMBINE, st);
        launch_lincomb(C, st);
      }
      if ((rc = check_launch("lincomb"))) return rc;
    }
    if ((rc = eval(i))) return rc;
    if (s->stage_cb &&
        (rc = call_stage(s, s->time + s->exc[i] * s->dt, s->time + s->imc[i] * s->dt, Q[i])))
      return rc;
  }
  LinComb C{};
  C.ns = ns;
  C.n = n;
  C.npairs = 3;
  C.dt = s->dt;
  for (int k = 0; k < 3; ++k) {
    C.a[k] = s->exb[k];
    C.b[k] = s->imb[k];
    for (int c = 0; c < 5; ++c) { C.X[k][c] = ex[k][c]; C.Y[k][c] = im[k][c]; }
  }
  for (int c = 0; c < 5; ++c) { C.base[c] = q[c < ns ? c : 0]; C.out[c] = q[c < ns ? c : 0]; }
  {
    ProfScope ps(ATB_PROF_COMBINE, st);
    launch_lincomb(C, st);
  }
  if ((rc = check_launch("lincomb"))) return rc;
  s->time += s->dt;
  return ATB_OK;
}

int do_steps(atb_solver* s, double* const* q, int nsteps, cudaStream_t st) {
  if (s->kind <= ATB_LSRK144) return lsrk_steps(s, q, nsteps, st);
  for (int i = 0; i < nsteps; ++i) {
    int rc = (s->kind <= ATB_RLSRK144) ? rlsrk_step(s, q, st) : ark_step(s, q, st);
    if (rc) return rc;
  }
  return ATB_OK;
}

}  // namespace

int fusion_check(atb_solver* s, cudaStream_t st);

extern "C" int atb_solver_create(int kind, atb_op* rhs, atb_op* linrhs, double dt, double t0, int split_rhs,
                                 int paperversion, atb_solver** out) {
  if (!out) return fail(ATB_ERR_INVALID, "null argument");
  *out = nullptr;
  if (kind < ATB_LSRK54 || kind > ATB_ARK23) return fail(ATB_ERR_INVALID, "unknown solver kind %d", kind);
  if (!std::isfinite(dt) || !(dt > 0.0)) return fail(ATB_ERR_INVALID, "dt must be finite and positive (got %g)", dt);
  if (!std::isfinite(t0)) return fail(ATB_ERR_INVALID, "t0 must be finite");
  if (kind != ATB_ARK23 && (!rhs || linrhs)) return fail(ATB_ERR_INVALID, "explicit solvers take rhs only");
  if (kind == ATB_ARK23 && !rhs && !linrhs) return fail(ATB_ERR_INVALID, "ARK23 needs rhs or linrhs");
  atb_op* any = rhs ? rhs : linrhs;
  if (rhs && linrhs && (rhs->ns != linrhs->ns || rhs->K != linrhs->K || rhs->Np != linrhs->Np))
    return fail(ATB_ERR_INVALID, "rhs and linrhs act on different fields");
  atb_solver* s = new atb_solver();
  s->kind = kind;
  s->rhs = rhs;
  s->lin = linrhs;
  s->any = any;
  s->dt = dt;
  s->time = t0;
  s->split_rhs = split_rhs;
  if (linrhs) linrhs->prof_class = ATB_PROF_TEND_LIN;
  s->ns = any->ns;
  s->stride = any->stride();
  const size_t fsz = (size_t)s->ns * s->stride;
  int rc = ATB_OK;
  if (kind <= ATB_RLSRK144) {
    if (kind == ATB_LSRK54 || kind == ATB_RLSRK54)
      coeffs_lsrk54(s);
    else
      coeffs_lsrk144(s);
    if ((rc = dalloc(&s->dq, fsz)) || (rc = dalloc(&s->qB, fsz))) { solver_free(s); return rc; }
    cudaMemset(s->dq, 0, fsz * sizeof(double));
    if (kind >= ATB_RLSRK54) {
      if ((rc = dalloc(&s->kb, fsz))) { solver_free(s); return rc; }
      const size_t nst = s->rkb.size();
      s->rkb_full.assign(nst, 0.0);
      s->rkb_full[nst - 1] = s->rkb[nst - 1];
      for (int i = (int)nst - 2; i >= 0; --i) s->rkb_full[i] = s->rka[i + 1] * s->rkb_full[i + 1] + s->rkb[i];
    }
  } else {
    // ARK23, Giraldo-Kelly-Constantinescu 2013 (src/odesolvers.jl:284-309)
    const double r2 = std::sqrt(2.0);
    const double a32 = paperversion ? (3 + 2 * r2) / 6 : 0.5;
    const double exa[3][3] = {{0, 0, 0}, {2 - r2, 0, 0}, {1 - a32, a32, 0}};
    const double ima[3][3] = {{0, 0, 0}, {1 - 1 / r2, 1 - 1 / r2, 0}, {1 / (2 * r2), 1 / (2 * r2), 1 - 1 / r2}};
    const double exb[3] = {1 / (2 * r2), 1 / (2 * r2), 1 - 1 / r2};
    const double exc[3] = {0, 2 - r2, 1};
    std::memcpy(s->exa, exa, sizeof(exa));
    std::memcpy(s->ima, ima, sizeof(ima));
    std::memcpy(s->exb, exb, sizeof(exb));
    std::memcpy(s->imb, exb, sizeof(exb));
    std::memcpy(s->exc, exc, sizeof(exc));
    std::memcpy(s->imc, exc, sizeof(exc));
    // the accumulated stages (rhs and linrhs, split_rhs = false) keep one
    // explicit-tendency buffer and solve in place (no stage states); the
    // general path keeps all three stages' tendencies and two stage states
    const bool accumulated = rhs && linrhs && !split_rhs;
    const size_t nex = accumulated ? 1 : 3, nqs = accumulated ? 0 : 2;
    if ((rc = dalloc(&s->Qs, nqs * fsz)) || (rc = dalloc(&s->exK, nex * fsz)) || (rc = dalloc(&s->imK, 3 * fsz))) {
      solver_free(s);
      return rc;
    }
    if (linrhs && (rc = build_band(s, 0))) {
      solver_free(s);
      return rc;
    }
    if ((rc = fusion_check(s, 0))) {
      solver_free(s);
      return rc;
    }
    s->fuse_on = s->fused != nullptr;
  }
  if ((rc = check_launch("solver create"))) { solver_free(s); return rc; }
  *out = s;
  return ATB_OK;
}

extern "C" int atb_solver_destroy(atb_solver* s) {
  if (s) solver_free(s);
  return ATB_OK;
}

extern "C" int atb_solver_step(atb_solver* s, double* const* q, int nsteps, void* stream) {
  if (!s || !q || nsteps < 0) return fail(ATB_ERR_INVALID, "bad argument");
  return do_steps(s, q, nsteps, (cudaStream_t)stream);
}

extern "C" int atb_solve(atb_solver* s, double* const* q, double timeend, int adjust_final, int* steps_out,
                         void* stream) {
  if (!s || !q) return fail(ATB_ERR_INVALID, "bad argument");
  if (!std::isfinite(timeend)) return fail(ATB_ERR_INVALID, "timeend must be finite");
  int step = 0;
  bool finalstep = false;
  while (true) {
    ++step;
    const double time = s->time;
    if (time + s->dt >= timeend) {
      if (adjust_final) s->dt = timeend - time;
      finalstep = true;
    } else if (!(time + s->dt > time)) {
      // a step that does not advance the clock (dt <= 0, or below the clock's
      // resolution) would never reach timeend
      return fail(ATB_ERR_INVALID, "solve: dt = %g does not advance time %g towards timeend %g", s->dt, time,
                  timeend);
    }
    int rc = do_steps(s, q, 1, (cudaStream_t)stream);
    if (rc) return rc;
    if (finalstep) break;
  }
  if (steps_out) *steps_out = step;
  return ATB_OK;
}

extern "C" int atb_solver_get(const atb_solver* s, double* time, double* dt, double* gamma) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  if (time) *time = s->time;
  if (dt) *dt = s->dt;
  if (gamma) *gamma = s->gamma_r;
  return ATB_OK;
}

extern "C" int atb_solver_set_state(atb_solver* s, double time, double gamma) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  if (!std::isfinite(time) || !std::isfinite(gamma)) return fail(ATB_ERR_INVALID, "non-finite solver state");
  s->time = time;
  s->gamma_r = gamma;
  return ATB_OK;
}

extern "C" int atb_solver_set_dt(atb_solver* s, double dt) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  if (!std::isfinite(dt) || dt < 0.0) return fail(ATB_ERR_INVALID, "dt must be finite and non-negative (got %g)", dt);
  if (s->kind == ATB_ARK23 && s->lin && dt != s->dt)
    return fail(ATB_ERR_INVALID, "ARK23 factors I - dt a L for a fixed dt");
  s->dt = dt;
  return ATB_OK;
}

// Can the explicit and the linear operator of this ARK23 solver run as one
// kernel per stage?  Euler-gravity (3-D, EC or FP32-flux EC volume flux; on
// curved elements EC or KG with Rusanov faces) with the weak-form linear
// Euler-gravity operator along z (the radial direction) only, on the same grid
// (bitwise identical metrics and neighbours, curved geometry included) with
// the same leading aux fields [Phi, grad Phi, rho_ref, p_ref] (bitwise
// identical on the device).
int fusion_check(atb_solver* s, cudaStream_t st) {
  s->fused = nullptr;
  atb_op *R = s->rhs, *L = s->lin;
  if (s->kind != ATB_ARK23 || !R || !L || s->split_rhs || !s->band) return ATB_OK;
  if (R->law.kind != LAW_EG || L->law.kind != LAW_LEG || R->dim != 3 || L->vk != VK_WEAK) return ATB_OK;
  if (L->dirs != (1 << (R->dim - 1))) return ATB_OK;
  if (R->K != L->K || R->Np != L->Np || R->stacked != L->stacked) return ATB_OK;
  if (R->curved != L->curved) return ATB_OK;
  const int na = R->dim + 3;
  if (R->naux < na || L->naux < na) return ATB_OK;
  tend_launch_fn f = R->curved ? pick_launcher_curved_fused(R->vk, R->sflux, L->sflux)
                               : pick_launcher_fused(R->dim, R->vk, R->Nq, R->sflux, L->sflux);
  if (!f) return ATB_OK;
  unsigned long long* d_cnt = nullptr;
  int rc;
  if ((rc = dalloc(&d_cnt, 1))) return rc;
  CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st));
  const size_t K = (size_t)R->K, n = R->stride();
  launch_count_diff(R->d_ginv, L->d_ginv, K * 3 * 2, d_cnt, st);
  launch_count_diff(R->d_J, L->d_J, K * 2, d_cnt, st);
  launch_count_diff(R->d_nbr, L->d_nbr, K * 6, d_cnt, st);
  if (R->curved) {
    // the same curved geometry: metric terms, M J, face normals, masses and map
    const size_t KF = K * 6 * R->Nfp;
    launch_count_diff(R->d_G, L->d_G, 9 * n * 2, d_cnt, st);
    launch_count_diff(R->d_MJn, L->d_MJn, n * 2, d_cnt, st);
    launch_count_diff(R->d_fnrm, L->d_fnrm, 3 * KF * 2, d_cnt, st);
    launch_count_diff(R->d_fMJ, L->d_fMJ, KF * 2, d_cnt, st);
    launch_count_diff(R->d_fnb, L->d_fnb, KF, d_cnt, st);
  }
  for (int k = 0; k < na; ++k) launch_count_diff(R->d_aux + (size_t)k * n, L->d_aux + (size_t)k * n, n * 2, d_cnt, st);
  unsigned long long cnt = 1;
  cudaError_t e1 = cudaMemcpyAsync(&cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  cudaFree(d_cnt);
  if (e1 != cudaSuccess || e2 != cudaSuccess) return fail(ATB_ERR_CUDA, "fusion check failed");
  if (cnt == 0) s->fused = f;
  return ATB_OK;
}

extern "C" int atb_solver_fuse(atb_solver* s, int enable) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  if (enable && !s->fused)
    return fail(ATB_ERR_INVALID, "this solver's operators cannot run as one kernel per stage");
  s->fuse_on = enable && s->fused;
  return ATB_OK;
}

extern "C" int atb_solver_set_instance_dt(atb_solver* s, const double* dt_host) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  if (s->kind != ATB_LSRK54 && s->kind != ATB_LSRK144)
    return fail(ATB_ERR_INVALID, "per-instance time steps exist for the LSRK solvers");
  if (!dt_host) {
    if (s->own_dte) cudaFree(s->d_dte);
    s->d_dte = nullptr;
    s->own_dte = false;
    return ATB_OK;
  }
  atb_op* op = s->rhs;
  for (int i = 0; i < op->ninst; ++i)
    if (!(dt_host[i] >= 0) || !std::isfinite(dt_host[i]))
      return fail(ATB_ERR_INVALID, "time step of instance %d must be finite and >= 0", i);
  std::vector<double> dte((size_t)op->K);
  for (int i = 0; i < op->ninst; ++i)
    for (int e = op->inst_off[i]; e < op->inst_off[i + 1]; ++e) dte[e] = dt_host[i];
  int rc;
  if (!s->own_dte) s->d_dte = nullptr;
  if (!s->d_dte && (rc = dalloc(&s->d_dte, (size_t)op->K))) return rc;
  s->own_dte = true;
  CK(cudaMemcpy(s->d_dte, dte.data(), dte.size() * sizeof(double), cudaMemcpyHostToDevice));
  return ATB_OK;
}

extern "C" int atb_solver_set_exchange_callback(atb_solver* s, atb_exchange_callback cb, void* user) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  s->xchg_cb = cb;
  s->xchg_user = cb ? user : nullptr;
  return ATB_OK;
}

extern "C" int atb_solver_set_stage_callback(atb_solver* s, atb_stage_callback cb, void* user) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  s->stage_cb = cb;
  s->stage_user = cb ? user : nullptr;
  return ATB_OK;
}

extern "C" int atb_solver_set_element_dt(atb_solver* s, const double* dte_device) {
  if (!s) return fail(ATB_ERR_INVALID, "null solver");
  if (s->kind != ATB_LSRK54 && s->kind != ATB_LSRK144)
    return fail(ATB_ERR_INVALID, "per-element time steps exist for the LSRK solvers");
  if (s->d_dte && s->own_dte) cudaFree(s->d_dte);
  s->d_dte = const_cast<double*>(dte_device);
  s->own_dte = false;
  return ATB_OK;
}

extern "C" int atb_op_set_active(atb_op* op, int n_instances) {
  if (!op || n_instances < 0 || n_instances > op->ninst) return fail(ATB_ERR_INVALID, "bad active instance count");
  op->K_active = op->inst_off[n_instances];
  return ATB_OK;
}

extern "C" int atb_op_set_instance_aux(atb_op* op, int i, const double* aux_host, void* stream) {
  if (!op || i < 0 || i >= op->ninst) return fail(ATB_ERR_INVALID, "bad instance");
  if (op->naux == 0) return ATB_OK;
  if (!aux_host) return fail(ATB_ERR_INVALID, "aux fields missing");
  const size_t Ki = (size_t)(op->inst_off[i + 1] - op->inst_off[i]), n = Ki * op->Np;
  for (int k = 0; k < op->naux; ++k)
    CK(cudaMemcpyAsync(op->d_aux + (size_t)k * op->stride() + (size_t)op->inst_off[i] * op->Np, aux_host + k * n,
                       n * sizeof(double), cudaMemcpyHostToDevice, (cudaStream_t)stream));
  return ATB_OK;
}

extern "C" int atb_op_copy_instance_aux(atb_op* op, int dst, int src, void* stream) {
  if (!op || dst < 0 || src < 0 || dst >= op->ninst || src >= op->ninst) return fail(ATB_ERR_INVALID, "bad instance");
  const int Kd = op->inst_off[dst + 1] - op->inst_off[dst], Ks = op->inst_off[src + 1] - op->inst_off[src];
  if (Kd != Ks) return fail(ATB_ERR_INVALID, "instances %d and %d differ in size", dst, src);
  if (dst == src || op->naux == 0) return ATB_OK;
  const size_t n = (size_t)Kd * op->Np;
  for (int k = 0; k < op->naux; ++k)
    CK(cudaMemcpyAsync(op->d_aux + (size_t)k * op->stride() + (size_t)op->inst_off[dst] * op->Np,
                       op->d_aux + (size_t)k * op->stride() + (size_t)op->inst_off[src] * op->Np, n * sizeof(double),
                       cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return ATB_OK;
}

extern "C" int atb_op_instances(const atb_op* op, int* n, int* first_elements) {
  if (!op || !n) return fail(ATB_ERR_INVALID, "null argument");
  *n = op->ninst;
  if (first_elements)
    for (int i = 0; i <= op->ninst; ++i) first_elements[i] = op->inst_off[i];
  return ATB_OK;
}

// ------------------------------------------- helpers for atb_noalloc.cu
// LSRK(5,4) stages of `op` with caller-provided device scratch (dq and the
// second state buffer): launches only, no allocation of any kind.
int atb_detail_fail(int code, const char* msg) { return fail(code, "%s", msg); }
int atb_detail_op_device(const atb_op* op) { return op->device; }

int atb_detail_lsrk54_steps(atb_op* op, double* const* q, double* dqbuf, double* qbbuf, double dt, int nsteps,
                            cudaStream_t st) {
  static const double rka[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                                -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
  static const double rkb[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                                1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                                2277821191437.0 / 14882151754819.0};
  const int ns = op->ns;
  const size_t n = op->stride();
  double *dq[5], *cur[5], *oth[5];
  for (int k = 0; k < 5; ++k) {
    const int c = k < ns ? k : 0;
    dq[k] = dqbuf + (size_t)c * n;
    cur[k] = q[c];
    oth[k] = qbbuf + (size_t)c * n;
  }
  bool in_user = true;
  // the same launches as the allocating path (run_tendency): the active
  // element prefix only, nothing at all when it is empty
  const int grid = (op->K_active + op->E - 1) / op->E;
  if (grid == 0) return ATB_OK;
  for (int step = 0; step < nsteps; ++step)
    for (int i = 0; i < 5; ++i) {
      TendArgs A;
      fill_args(op, A);
      A.epi = EPI_LSRK;
      A.a = rka[i];
      A.bdt = rkb[i] * dt;
      for (int k = 0; k < 5; ++k) { A.q[k] = cur[k]; A.out[k] = dq[k]; A.out2[k] = oth[k]; }
      {
        ProfScope ps(op->prof_class, st);
        op->launch(A, grid, cta_threads(op->E, op->Np), op->smem, st);
      }
      const int rc = check_launch("tendency (no-alloc LSRK54)");
      if (rc) return rc;
      for (int k = 0; k < 5; ++k) std::swap(cur[k], oth[k]);
      in_user = !in_user;
    }
  // after an odd number of stages the state is in the scratch buffer: copy
  // back the active elements only (rows beyond them were never written)
  if (!in_user)
    for (int s = 0; s < ns; ++s)
      CK(cudaMemcpyAsync(q[s], cur[s], (size_t)op->K_active * op->Np * sizeof(double), cudaMemcpyDeviceToDevice,
                         st));
  return ATB_OK;
}
