// TEST INFRASTRUCTURE — CPU oracle, not the product (see oracle.h).
//
// Restates, operation for operation:
//   src/dgsem.jl:38-56    DGSEM construction (MJ, MJI, faceMJ)
//   src/dgsem.jl:59-98    operator call (volume launch(es) + surface)
//   src/dgsem.jl:217-306  volumeterm!            (WeakForm)
//   src/dgsem.jl:308-468  esvolumeterm!          (:naive)
//   src/dgsem.jl:470-561  esvolumeterm_dir!      (:per_dir, default)
//   src/dgsem.jl:563-681  esvolumeterm_dir_symmetric!
//   src/dgsem.jl:683-732  surfaceterm!
//   src/odesolvers.jl     solve!, LSRK, RLSRK, ARK23
//   src/measures.jl       weightednorm, entropyintegral, entropyproduct
//   src/bandedsystem.jl   probe assembly of the vertical banded operator
// and the Bennu 0.3 pieces the reference calls (un-vendored, version
// unpinned; restated from their published algorithms): Legendre-Gauss-Lobatto
// nodes/weights (Newton on q = L_{N+1} - L_{N-1}), the barycentric derivative
// matrix with negative-sum diagonal, the affine brick grid (points, metrics
// g = d(xi)/dx and J, face normals/Jacobians, face index maps, boundary tags =
// face number), StackedOrdering, and a no-pivot batched banded LU.
#include "oracle.h"
#include "physics.hpp"

#include <cstring>
#include <cstdio>
#include <vector>
#include <memory>
#include <thread>

using namespace orc;

namespace {

int g_threads = 1;

// static split of [0, n) over g_threads std::threads (element loops only:
// every element writes only its own nodes, so the split is race-free and the
// results do not depend on the thread count)
template <class F> void par_for(int n, F f) {
  int T = std::max(1, std::min(g_threads, n));
  if (T == 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([=, &f]() {
      int a = (int)((long)n * t / T), b = (int)((long)n * (t + 1) / T);
      for (int i = a; i < b; ++i) f(i);
    });
  for (auto& x : th) x.join();
}

// ------------------------------------------------------------------ LGL
void lgl_nodes_weights(int N, std::vector<double>& x, std::vector<double>& w) {
  x.assign(N + 1, 0.0);
  w.assign(N + 1, 0.0);
  auto qeval = [N](double xx, double& q, double& dq, double& LN) {
    double Lm2 = 1.0, Lm1 = xx, dLm2 = 0.0, dLm1 = 1.0, L = 0, dL = 0;
    for (int k = 2; k <= N; ++k) {
      L = (2.0 * k - 1.0) / k * xx * Lm1 - (k - 1.0) / k * Lm2;
      dL = dLm2 + (2.0 * k - 1.0) * Lm1;
      Lm2 = Lm1; Lm1 = L; dLm2 = dLm1; dLm1 = dL;
    }
    // now Lm1 = L_N, Lm2 = L_{N-1}
    double LN1 = (2.0 * N + 1.0) / (N + 1.0) * xx * Lm1 - N / (N + 1.0) * Lm2;
    double dLN1 = dLm2 + (2.0 * N + 1.0) * Lm1;
    q = LN1 - Lm2;
    dq = dLN1 - dLm2;
    LN = Lm1;
  };
  if (N == 1) {
    x[0] = -1; x[1] = 1; w[0] = 1; w[1] = 1;
    return;
  }
  x[0] = -1.0; x[N] = 1.0;
  w[0] = w[N] = 2.0 / (N * (N + 1.0));
  for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
    const double pi = 3.14159265358979323846;
    double xx = -std::cos((j + 0.25) * pi / N - 3.0 / (8.0 * N * pi * (j + 0.25)));
    double q, dq, LN;
    for (int it = 0; it < 100; ++it) {
      qeval(xx, q, dq, LN);
      double delta = -q / dq;
      xx += delta;
      if (std::fabs(delta) <= 4 * 2.220446049250313e-16 * std::fabs(xx)) break;
    }
    qeval(xx, q, dq, LN);
    x[j] = xx;
    w[j] = 2.0 / (N * (N + 1.0) * LN * LN);
    x[N - j] = -xx;
    w[N - j] = w[j];
  }
  if (N % 2 == 0) {
    double q, dq, LN;
    qeval(0.0, q, dq, LN);
    x[N / 2] = 0.0;
    w[N / 2] = 2.0 / (N * (N + 1.0) * LN * LN);
  }
}

// D[i][j] = l_j'(x_i), barycentric form with negative-sum diagonal.
std::vector<double> derivative_matrix(const std::vector<double>& x) {
  const int n = (int)x.size();
  std::vector<double> bw(n, 1.0), D(n * n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k)
      if (k != j) bw[j] *= (x[j] - x[k]);
  for (int j = 0; j < n; ++j) bw[j] = 1.0 / bw[j];
  for (int i = 0; i < n; ++i) {
    double s = 0;
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      D[i * n + j] = (bw[j] / bw[i]) / (x[i] - x[j]);
      s += D[i * n + j];
    }
    D[i * n + i] = -s;
  }
  return D;
}

// --------------------------------------------------------------- operator
struct Op {
  Law law;
  int dim, N, Nq, Np, Nfp, K, Kd[3], periodic[3], stacked;
  int volume_form, volume_flux, fd_kernel, surface_flux;
  int dirs[3], ndirs;
  std::vector<double> xi, wq, D;
  std::vector<int> eidx;        // K x 3 per-dim element index
  std::vector<double> h;        // K x 3
  std::vector<double> Jel;      // K
  std::vector<double> MJ, MJI;  // K*Np
  std::vector<double> aux;      // naux*K*Np
  std::vector<int> nbr;         // K x 6 neighbour element (or -1)
  std::vector<int> btag;        // K x 6
  std::vector<int> face_node;   // 6 x Nfp node index
  std::vector<double> face_w;   // 6 x Nfp face weight
  std::vector<double> points;   // dim x K x Np
  std::vector<double> v[3];
  // curved elements (orc_op_set_curved): per-node metric terms
  // G[((dir*3 + c)*K + e)*Np + n] = d xi_dir / d x_c, per-face-node outward
  // unit normals fn[((e*6 + f)*Nfp + j)*3 + c], face mass faceMJ[(e*6 + f)*Nfp + j]
  // and the neighbour's global node index fnb (-1 on a boundary face)
  bool curved = false;
  std::vector<double> G, fn, fMJ;
  std::vector<long long> fnb;

  int elem_of(const int* idx) const {
    if (stacked) {
      // StackedOrdering{CartesianOrdering}: vertical (last dim) fastest,
      // horizontal stacks in Cartesian order.
      int ev = idx[dim - 1], eh = 0, m = 1;
      for (int d = 0; d < dim - 1; ++d) { eh += idx[d] * m; m *= Kd[d]; }
      return eh * Kd[dim - 1] + ev;
    }
    int e = 0, m = 1;
    for (int d = 0; d < dim; ++d) { e += idx[d] * m; m *= Kd[d]; }
    return e;
  }
  bool has_dir(int d) const {
    for (int k = 0; k < ndirs; ++k)
      if (dirs[k] == d) return true;
    return false;
  }
  // ndindex of node
  void node_idx(int n, int* ijk) const {
    ijk[0] = n % Nq;
    ijk[1] = (n / Nq) % Nq;
    ijk[2] = n / (Nq * Nq);
  }
  double g(int e, int dir, int d) const { return dir == d ? 2.0 / h[e * 3 + d] : 0.0; }
  // metric term of node id = e*Np + n (src/dgsem.jl:38-56 metrics(grid))
  double gn(size_t id, int dir, int d) const {
    return curved ? G[((size_t)dir * 3 + d) * (size_t)K * Np + id] : g((int)(id / Np), dir, d);
  }
};

void op_build(Op& o, const orc_desc* d, const double* aux) {
  Law& L = o.law;
  L.kind = d->law;
  L.dim = d->dim;
  L.ns = (d->law == ADVECTION) ? 1 : d->dim + 2;
  L.naux = d->naux;
  L.gamma = d->gamma;
  L.grav = d->grav;
  for (int k = 0; k < 3; ++k) { L.adv_u[k] = d->adv_u[k]; L.omega[k] = d->omega[k]; }
  L.sphere = d->sphere;
  L.pde_level_balance = d->pde_level_balance;
  L.bc_kind = d->bc_kind;
  std::memcpy(L.bc_state, d->bc_state, sizeof(L.bc_state));
  L.source_kind = d->source_kind;
  L.sw_topography = d->sw_topography;

  o.dim = d->dim;
  o.N = d->N;
  o.Nq = d->N + 1;
  o.Np = 1;
  for (int k = 0; k < o.dim; ++k) o.Np *= o.Nq;
  o.Nfp = o.Np / o.Nq;
  o.K = 1;
  for (int k = 0; k < 3; ++k) {
    o.Kd[k] = k < o.dim ? d->K[k] : 1;
    o.periodic[k] = k < o.dim ? d->periodic[k] : 0;
    o.K *= o.Kd[k];
    if (k < o.dim) o.v[k].assign(d->v[k], d->v[k] + d->K[k] + 1);
  }
  o.stacked = d->stacked;
  o.volume_form = d->volume_form;
  o.volume_flux = d->volume_flux;
  o.fd_kernel = d->fd_kernel;
  o.surface_flux = d->surface_flux;
  o.ndirs = 0;
  for (int k = 0; k < o.dim; ++k)
    if (d->directions & (1 << k)) o.dirs[o.ndirs++] = k;

  lgl_nodes_weights(o.N, o.xi, o.wq);
  o.D = derivative_matrix(o.xi);
  const int Nq = o.Nq, Np = o.Np, K = o.K, dim = o.dim;

  o.eidx.assign(K * 3, 0);
  o.h.assign(K * 3, 1.0);
  o.Jel.assign(K, 1.0);
  o.nbr.assign(K * 6, -1);
  o.btag.assign(K * 6, 0);
  // enumerate per-dim indices and map to element number
  int idx[3];
  for (idx[2] = 0; idx[2] < o.Kd[2]; ++idx[2])
    for (idx[1] = 0; idx[1] < o.Kd[1]; ++idx[1])
      for (idx[0] = 0; idx[0] < o.Kd[0]; ++idx[0]) {
        int e = o.elem_of(idx);
        double J = 1.0;
        for (int k = 0; k < 3; ++k) {
          o.eidx[e * 3 + k] = idx[k];
          if (k < dim) {
            o.h[e * 3 + k] = o.v[k][idx[k] + 1] - o.v[k][idx[k]];
            J *= o.h[e * 3 + k] / 2;
          }
        }
        o.Jel[e] = J;
        for (int k = 0; k < dim; ++k)
          for (int f = 0; f < 2; ++f) {
            int nb[3] = {idx[0], idx[1], idx[2]};
            nb[k] += f ? 1 : -1;
            bool bnd = false;
            if (nb[k] < 0 || nb[k] >= o.Kd[k]) {
              if (o.periodic[k])
                nb[k] = (nb[k] + o.Kd[k]) % o.Kd[k];
              else
                bnd = true;
            }
            if (bnd) {
              o.btag[e * 6 + 2 * k + f] = 2 * k + f + 1;
              o.nbr[e * 6 + 2 * k + f] = -1;
            } else {
              o.nbr[e * 6 + 2 * k + f] = o.elem_of(nb);
            }
          }
      }
  // mass
  o.MJ.assign((size_t)K * Np, 0.0);
  o.MJI.assign((size_t)K * Np, 0.0);
  for (int e = 0; e < K; ++e)
    for (int n = 0; n < Np; ++n) {
      int ijk[3];
      o.node_idx(n, ijk);
      double w = o.wq[ijk[0]];
      for (int k = 1; k < dim; ++k) w = w * o.wq[ijk[k]];
      o.MJ[(size_t)e * Np + n] = w * o.Jel[e];
      o.MJI[(size_t)e * Np + n] = 1.0 / o.MJ[(size_t)e * Np + n];
    }
  // faces: node tables and weights; face node j enumerates the tangential
  // dims in increasing order, first fastest.
  o.face_node.assign(6 * o.Nfp, 0);
  o.face_w.assign(6 * o.Nfp, 1.0);
  for (int k = 0; k < dim; ++k)
    for (int f = 0; f < 2; ++f)
      for (int j = 0; j < o.Nfp; ++j) {
        int t[2] = {j % Nq, j / Nq};
        int ijk[3] = {0, 0, 0}, c = 0;
        double w = 1.0;
        bool first = true;
        for (int dd = 0; dd < dim; ++dd) {
          if (dd == k) {
            ijk[dd] = f ? Nq - 1 : 0;
          } else {
            ijk[dd] = t[c++];
            w = first ? o.wq[ijk[dd]] : w * o.wq[ijk[dd]];
            first = false;
          }
        }
        o.face_node[(2 * k + f) * o.Nfp + j] = ijk[0] + Nq * (ijk[1] + Nq * ijk[2]);
        o.face_w[(2 * k + f) * o.Nfp + j] = w;
      }
  // points
  o.points.assign((size_t)dim * K * Np, 0.0);
  for (int e = 0; e < K; ++e)
    for (int n = 0; n < Np; ++n) {
      int ijk[3];
      o.node_idx(n, ijk);
      for (int k = 0; k < dim; ++k) {
        double v0 = o.v[k][o.eidx[e * 3 + k]], v1 = o.v[k][o.eidx[e * 3 + k] + 1];
        double xi = o.xi[ijk[k]];
        o.points[((size_t)k * K + e) * Np + n] = (v0 * (1 - xi) + v1 * (1 + xi)) / 2;
      }
    }
  o.aux.assign((size_t)L.naux * K * Np, 0.0);
  if (aux && L.naux) std::memcpy(o.aux.data(), aux, sizeof(double) * L.naux * K * Np);
}

inline void gather(const double* x, int ns, size_t stride, size_t id, double* out) {
  for (int s = 0; s < ns; ++s) out[s] = x[s * stride + id];
}

// ----------------------------------------------------- WeakForm volume
void volume_weak(const Op& o, double* dq, const double* q, bool increment) {
  const Law& L = o.law;
  const int Nq = o.Nq, Np = o.Np, S = L.ns, A = L.naux, dim = o.dim;
  const size_t st = (size_t)o.K * Np;
  const bool srcdir = o.has_dir(dim - 1);
  par_for(o.K, [&](int e) {
    std::vector<double> lF((size_t)Np * 3 * 5);
    for (int n = 0; n < Np; ++n) {
      size_t id = (size_t)e * Np + n;
      double qn[5], an[8], F[3][5];
      gather(q, S, st, id, qn);
      gather(o.aux.data(), A, st, id, an);
      flux(L, qn, an, F);
      double MJ = o.MJ[id];
      for (int s = 0; s < S; ++s)
        for (int dd = 0; dd < o.ndirs; ++dd) {
          int dir = o.dirs[dd];
          double acc = 0;
          for (int c = 0; c < dim; ++c) acc = acc + o.gn(id, dir, c) * F[c][s];
          lF[((size_t)n * 3 + dd) * 5 + s] = acc * MJ;
        }
    }
    for (int n = 0; n < Np; ++n) {
      size_t id = (size_t)e * Np + n;
      int ijk[3];
      o.node_idx(n, ijk);
      double qn[5], an[8], dqn[5];
      gather(q, S, st, id, qn);
      gather(o.aux.data(), A, st, id, an);
      for (int s = 0; s < S; ++s) dqn[s] = -0.0;
      if (srcdir) {
        law_source(L, dqn, qn, an);
        problem_source(L, dqn, qn, an);
        nonconservative_term(L, dqn, qn, an);
      }
      double MJI = o.MJI[id];
      for (int m = 0; m < Nq; ++m) {
        double Dm[3];
        for (int k = 0; k < 3; ++k) Dm[k] = (k < dim ? o.D[m * Nq + ijk[k]] : 0.0) * MJI;
        for (int s = 0; s < S; ++s)
          for (int dd = 0; dd < o.ndirs; ++dd) {
            int dir = o.dirs[dd];
            int t[3] = {ijk[0], ijk[1], ijk[2]};
            t[dir] = m;
            int nn = t[0] + Nq * (t[1] + Nq * t[2]);
            dqn[s] = dqn[s] + Dm[dir] * lF[((size_t)nn * 3 + dd) * 5 + s];
          }
      }
      for (int s = 0; s < S; ++s) dq[s * st + id] = increment ? dq[s * st + id] + dqn[s] : dqn[s];
    }
    });
}

// -------------------------------------------- flux differencing, per dir
void volume_fd_dir(const Op& o, int dir, double* dq, const double* q, bool increment, bool symmetric) {
  const Law& L = o.law;
  const int Nq = o.Nq, Np = o.Np, S = L.ns, A = L.naux, dim = o.dim;
  const size_t st = (size_t)o.K * Np;
  const bool srcdir = (dir == dim - 1);
  par_for(o.K, [&](int e) {
    for (int n = 0; n < Np; ++n) {
      size_t id = (size_t)e * Np + n;
      int ijk[3];
      o.node_idx(n, ijk);
      double q1[5], a1[8], d1[5], d2[5];
      gather(q, S, st, id, q1);
      gather(o.aux.data(), A, st, id, a1);
      for (int s = 0; s < S; ++s) d1[s] = d2[s] = -0.0;
      if (srcdir) {
        law_source(L, d1, q1, a1);
        problem_source(L, d1, q1, a1);
      }
      double MJI = o.MJI[id];
      double lg_i[3];
      for (int c = 0; c < dim; ++c) lg_i[c] = o.MJ[id] * o.gn(id, dir, c);
      const int id_ = ijk[dir];
      for (int pass = 0; pass < (symmetric ? 2 : 1); ++pass) {
        double* acc = pass ? d2 : d1;
        for (int mm = 0; mm < Nq; ++mm) {
          int m = pass ? Nq - 1 - mm : mm;
          int t[3] = {ijk[0], ijk[1], ijk[2]};
          t[dir] = m;
          size_t ild = (size_t)e * Np + t[0] + Nq * (t[1] + Nq * t[2]);
          double q2[5], a2[8], F[3][5];
          gather(q, S, st, ild, q2);
          gather(o.aux.data(), A, st, ild, a2);
          twopointflux(o.volume_flux, L, q1, a1, q2, a2, F);
          double lg_n[3];
          for (int c = 0; c < dim; ++c) lg_n[c] = o.MJ[ild] * o.gn(ild, dir, c);
          for (int s = 0; s < S; ++s) {
            double Ddn = MJI * o.D[id_ * Nq + m];
            double Dnd = MJI * o.D[m * Nq + id_];
            for (int c = 0; c < dim; ++c) {
              if (symmetric) {
                acc[s] = acc[s] - Ddn * lg_i[c] * F[c][s] / 2;
                acc[s] = acc[s] + F[c][s] * lg_n[c] * Dnd / 2;
              } else {
                acc[s] = acc[s] - Ddn * lg_i[c] * F[c][s];
                acc[s] = acc[s] + F[c][s] * lg_n[c] * Dnd;
              }
            }
          }
        }
      }
      for (int s = 0; s < S; ++s) {
        double v = symmetric ? d1[s] + d2[s] : d1[s];
        dq[s * st + id] = increment ? dq[s * st + id] + v : v;
      }
    }
    });
}

// ------------------------------------- flux differencing, naive schedule
// esvolumeterm! (src/dgsem.jl:308-468): all directions interleaved per n.
// The reference loads only aux components 1..dim into its pencils
// (src/dgsem.jl:358-360); the restatement loads all of them (same results
// for every flux that reads only the geopotential).
void volume_fd_naive(const Op& o, double* dq, const double* q, bool increment) {
  const Law& L = o.law;
  const int Nq = o.Nq, Np = o.Np, S = L.ns, A = L.naux, dim = o.dim;
  const size_t st = (size_t)o.K * Np;
  par_for(o.K, [&](int e) {
    for (int n = 0; n < Np; ++n) {
      size_t id = (size_t)e * Np + n;
      int ijk[3];
      o.node_idx(n, ijk);
      double q1[5], a1[8], dqn[5];
      gather(q, S, st, id, q1);
      gather(o.aux.data(), A, st, id, a1);
      for (int s = 0; s < S; ++s) dqn[s] = -0.0;
      law_source(L, dqn, q1, a1);
      problem_source(L, dqn, q1, a1);
      double MJI = 1 / o.MJ[id];
      for (int m = 0; m < Nq; ++m) {
        for (int dir = 0; dir < dim; ++dir) {
          int t[3] = {ijk[0], ijk[1], ijk[2]};
          t[dir] = m;
          size_t ild = (size_t)e * Np + t[0] + Nq * (t[1] + Nq * t[2]);
          double q2[5], a2[8], F[3][5];
          gather(q, S, st, ild, q2);
          gather(o.aux.data(), A, st, ild, a2);
          twopointflux(o.volume_flux, L, q1, a1, q2, a2, F);
          int ii = ijk[dir];
          for (int s = 0; s < S; ++s) {
            double Din = MJI * o.D[ii * Nq + m];
            double Dni = MJI * o.D[m * Nq + ii];
            for (int c = 0; c < dim; ++c) {
              double lgi = o.MJ[id] * o.gn(id, dir, c), lgn = o.MJ[ild] * o.gn(ild, dir, c);
              dqn[s] = dqn[s] - Din * lgi * F[c][s];
              dqn[s] = dqn[s] + F[c][s] * lgn * Dni;
            }
          }
        }
      }
      for (int s = 0; s < S; ++s) dq[s * st + id] = increment ? dq[s * st + id] + dqn[s] : dqn[s];
    }
    });
}

// ------------------------------------------------------------ surface
void surface(const Op& o, double* dq, const double* q) {
  const Law& L = o.law;
  const int Nq = o.Nq, Np = o.Np, S = L.ns, A = L.naux, dim = o.dim;
  const size_t st = (size_t)o.K * Np;
  if (o.curved) {
    // surfaceterm! (src/dgsem.jl:683-732) with facenormal / faceMJ / faceix
    // of a curved grid: per-face-node normal and face mass, neighbour node
    // from the face map
    par_for(o.K, [&](int e) {
      for (int dd = 0; dd < o.ndirs; ++dd) {
        const int k = o.dirs[dd];
        for (int f = 0; f < 2; ++f) {
          const int face = 2 * k + f;
          const int tag = o.btag[e * 6 + face];
          for (int j = 0; j < o.Nfp; ++j) {
            const size_t fj = ((size_t)e * 6 + face) * o.Nfp + j;
            const int nm = o.face_node[face * o.Nfp + j];
            const size_t idm = (size_t)e * Np + nm;
            const double* nvec = &o.fn[fj * 3];
            double qm[5], am[8], qp[5], ap[8], nf[5];
            gather(o.aux.data(), A, st, idm, am);
            gather(q, S, st, idm, qm);
            if (tag == 0) {
              const size_t idp = (size_t)o.fnb[fj];
              gather(q, S, st, idp, qp);
              gather(o.aux.data(), A, st, idp, ap);
            } else {
              boundarystate(L, nvec, qm, am, tag, qp, ap);
            }
            surfaceflux(o.surface_flux, L, nvec, qm, am, qp, ap, nf);
            for (int s = 0; s < S; ++s) dq[s * st + idm] = dq[s * st + idm] - o.fMJ[fj] * nf[s] * o.MJI[idm];
          }
        }
      }
    });
    return;
  }
  par_for(o.K, [&](int e) {
    for (int dd = 0; dd < o.ndirs; ++dd) {
      int k = o.dirs[dd];
      double fJ = 1.0;
      bool first = true;
      for (int c = 0; c < dim; ++c)
        if (c != k) { fJ = first ? o.h[e * 3 + c] / 2 : fJ * (o.h[e * 3 + c] / 2); first = false; }
      for (int f = 0; f < 2; ++f) {
        int face = 2 * k + f;
        int tag = o.btag[e * 6 + face];
        int enb = o.nbr[e * 6 + face];
        double nvec[3] = {0, 0, 0};
        nvec[k] = f ? 1.0 : -1.0;
        for (int j = 0; j < o.Nfp; ++j) {
          int nm = o.face_node[face * o.Nfp + j];
          size_t idm = (size_t)e * Np + nm;
          double fMJ = o.face_w[face * o.Nfp + j] * fJ;
          double qm[5], am[8], qp[5], ap[8], nf[5];
          gather(o.aux.data(), A, st, idm, am);
          gather(q, S, st, idm, qm);
          if (tag == 0) {
            int np_ = o.face_node[(2 * k + (1 - f)) * o.Nfp + j];
            size_t idp = (size_t)enb * Np + np_;
            gather(q, S, st, idp, qp);
            gather(o.aux.data(), A, st, idp, ap);
          } else {
            boundarystate(L, nvec, qm, am, tag, qp, ap);
          }
          surfaceflux(o.surface_flux, L, nvec, qm, am, qp, ap, nf);
          for (int s = 0; s < S; ++s) dq[s * st + idm] = dq[s * st + idm] - fMJ * nf[s] * o.MJI[idm];
        }
      }
    }
    });
  (void)Nq;
}

void op_apply(const Op& o, double* dq, const double* q, double t, bool increment) {
  (void)t;
  if (o.volume_form == 0) {
    volume_weak(o, dq, q, increment);
  } else if (o.fd_kernel == 2) {
    volume_fd_naive(o, dq, q, increment);
  } else {
    for (int dd = 0; dd < o.ndirs; ++dd)
      volume_fd_dir(o, o.dirs[dd], dq, q, dd == 0 ? increment : true, o.fd_kernel == 1);
  }
  surface(o, dq, q);
}

// -------------------------------------------------------------- measures
// Neumaier-compensated sum: the reference's `sum` reassociates (pairwise /
// SIMD blocks); a compensated sum is the order-independent stand-in.
struct Sum {
  double s = 0, c = 0;
  void add(double x) {
    double t = s + x;
    if (std::fabs(s) >= std::fabs(x))
      c += (s - t) + x;
    else
      c += (x - t) + s;
    s = t;
  }
  double value() const { return s + c; }
};
double weightednorm(const Op& o, const double* q, double p, double* comp) {
  const size_t st = (size_t)o.K * o.Np;
  double nn[5];
  for (int s = 0; s < o.law.ns; ++s) {
    double acc = 0;
    if (std::isinf(p)) {
      for (size_t i = 0; i < st; ++i) acc = std::max(acc, std::fabs(q[s * st + i]));
      nn[s] = acc;
    } else {
      for (size_t i = 0; i < st; ++i) acc += o.MJ[i] * std::pow(std::fabs(q[s * st + i]), p);
      nn[s] = std::pow(acc, 1.0 / p);
    }
    if (comp) comp[s] = nn[s];
  }
  if (std::isinf(p)) {
    double m = 0;
    for (int s = 0; s < o.law.ns; ++s) m = std::max(m, nn[s]);
    return m;
  }
  double acc = 0;
  for (int s = 0; s < o.law.ns; ++s) acc += std::pow(nn[s], p);
  return std::pow(acc, 1.0 / p);
}

double entropyintegral(const Op& o, const double* q) {
  const size_t st = (size_t)o.K * o.Np;
  Sum acc;
  for (size_t i = 0; i < st; ++i) {
    double qn[5], an[8];
    gather(q, o.law.ns, st, i, qn);
    gather(o.aux.data(), o.law.naux, st, i, an);
    acc.add(o.MJ[i] * entropy(o.law, qn, an));
  }
  return acc.value();
}

double entropyproduct(const Op& o, const double* p, const double* q) {
  const size_t st = (size_t)o.K * o.Np;
  Sum acc;
  for (size_t i = 0; i < st; ++i) {
    double pn[5], an[8], v[5];
    gather(p, o.law.ns, st, i, pn);
    gather(o.aux.data(), o.law.naux, st, i, an);
    entropyvariables(o.law, pn, an, v);
    double d = v[0] * q[i];
    for (int s = 1; s < o.law.ns; ++s) d = d + v[s] * q[s * st + i];
    acc.add(o.MJ[i] * d);
  }
  return acc.value();
}

// -------------------------------------------------------------- solvers
struct Solver {
  int kind = 0;
  Op* rhs = nullptr;
  Op* lin = nullptr;
  double dt = 0, time = 0, gamma_r = 1;
  size_t n = 0;
  std::vector<double> rka, rkb, rkc, rkb_full;
  std::vector<double> dq, q0, k;
  // ARK
  double exa[3][3], exb[3], exc[3], ima[3][3], imb[3], imc[3];
  int split_rhs = 0;
  std::vector<double> Qhat, Qs[2], exK[3], imK[3];
  // banded factor: nlines x nunk x (2bw+1)
  int bw = 0, nunk = 0, nlines = 0;
  std::vector<double> band;
  std::vector<size_t> line_map;  // nlines x nunk -> global index (state-major offset)
  // after_stage (src/odesolvers.jl:10-11,23): called after every stage
  orc_stage_cb stage_cb = nullptr;
  void* stage_user = nullptr;
};

void coeffs_lsrk54(Solver& s) {
  s.rka = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
           -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
  s.rkb = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
           1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
           2277821191437.0 / 14882151754819.0};
  s.rkc = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
           2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};
}
void coeffs_lsrk144(Solver& s) {
  s.rka = {0, -0.7188012108672410, -0.7785331173421570, -0.0053282796654044, -0.8552979934029281,
           -3.9564138245774565, -1.5780575380587385, -2.0837094552574054, -0.7483334182761610,
           -0.7032861106563359, 0.0013917096117681, -0.0932075369637460, -0.9514200470875948,
           -7.1151571693922548};
  s.rkb = {0.0367762454319673, 0.3136296607553959, 0.1531848691869027, 0.0030097086818182,
           0.3326293790646110, 0.2440251405350864, 0.3718879239592277, 0.6204126221582444,
           0.1524043173028741, 0.0760894927419266, 0.0077604214040978, 0.0024647284755382,
           0.0780348340049386, 5.5059777270269628};
  s.rkc = {0, 0.0367762454319673, 0.1249685262725025, 0.2446177702277698, 0.2476149531070420,
           0.2969311120382472, 0.3978149645802642, 0.5270854589440328, 0.6981269994175695,
           0.8190890835352128, 0.8527059887098624, 0.8604711817462826, 0.8627060376969976,
           0.8734213127600976};
}

void lsrk_step(Solver& s, double* q) {
  const size_t n = s.n;
  for (size_t st = 0; st < s.rka.size(); ++st) {
    double stagetime = s.time + s.rkc[st] * s.dt;
    for (size_t i = 0; i < n; ++i) s.dq[i] = s.dq[i] * s.rka[st];
    op_apply(*s.rhs, s.dq.data(), q, stagetime, true);
    double c = s.rkb[st] * s.dt;
    for (size_t i = 0; i < n; ++i) q[i] = q[i] + c * s.dq[i];
    if (s.stage_cb) s.stage_cb(stagetime, stagetime, q, s.stage_user);  // src/odesolvers.jl:54
  }
  s.time += s.dt;
}

void rlsrk_step(Solver& s, double* q) {
  const size_t n = s.n;
  const Op& o = *s.rhs;
  std::memcpy(s.q0.data(), q, n * sizeof(double));
  double eta0 = entropyintegral(o, s.q0.data());
  double deta = -0.0;
  for (size_t st = 0; st < s.rka.size(); ++st) {
    for (size_t i = 0; i < n; ++i) s.dq[i] = s.dq[i] * s.rka[st];
    double stagetime = s.time + s.rkc[st] * s.dt;
    op_apply(o, s.k.data(), q, stagetime, false);
    for (size_t i = 0; i < n; ++i) s.dq[i] = s.dq[i] + s.k[i];
    deta = deta + s.rkb_full[st] * s.dt * entropyproduct(o, q, s.k.data());
    double c = s.rkb[st] * s.dt;
    for (size_t i = 0; i < n; ++i) q[i] = q[i] + c * s.dq[i];
    if (s.stage_cb) s.stage_cb(stagetime, stagetime, q, s.stage_user);  // src/odesolvers.jl:119
  }
  for (size_t i = 0; i < n; ++i) s.k[i] = q[i] - s.q0[i];
  // nlsolve(r, dr, [gamma]; ftol = 10 eps) with NLsolve's default
  // trust-region method (autoscale, factor 1, eta 1e-4), restated for one
  // unknown:
  //   r(g) = eta(q0 + g k) - eta0 - g deta,  r'(g) = <v(q0 + g k), k> - deta
  // A step with actual/predicted reduction of r^2 above eta is accepted;
  // otherwise it is undone and the radius halves.  Stops when |r| <= ftol
  // after an accepted step, when an accepted step is zero (xtol = 0), or
  // after 1000 iterations.
  auto setq = [&](double g) {
    for (size_t i = 0; i < n; ++i) q[i] = s.q0[i] + g * s.k[i];
  };
  auto resid = [&](double g) {
    setq(g);
    return entropyintegral(o, q) - eta0 - g * deta;
  };
  auto jac = [&](double g) {
    setq(g);
    return entropyproduct(o, q, s.k.data()) - deta;
  };
  const double ftol = 10 * 2.220446049250313e-16;
  double g = s.gamma_r;
  double r = resid(g);
  if (!(std::fabs(r) <= ftol)) {
    double J = jac(g);
    double Dsc = std::fabs(J) > 0 ? std::fabs(J) : 1.0;
    double delta = std::fabs(Dsc * g) > 0 ? std::fabs(Dsc * g) : 1.0;
    for (int it = 0; it < 1000; ++it) {
      if (!(J != 0) || !std::isfinite(J)) break;
      double p = -r / J;
      if (std::fabs(Dsc * p) > delta) p = (p > 0 ? delta : -delta) / Dsc;
      double gn = g + p;
      double rn = resid(gn);
      double rp = r + J * p;
      double pred = r * r - rp * rp;
      double rho = (r * r - rn * rn) / pred;
      bool conv = false;
      if (rho > 1e-4) {
        g = gn;
        r = rn;
        J = jac(g);
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
  s.gamma_r = g;
  setq(g);
  s.time += s.dt;
}

// Banded operator: vertical lines of nodes, unknown u = (ev*Nq + kv)*Ns + s.
void ark_build_band(Solver& s) {
  Op& o = *s.lin;
  const int dim = o.dim, Nq = o.Nq, Np = o.Np, S = o.law.ns;
  const int KV = o.Kd[dim - 1];
  int KH = 1;
  for (int d = 0; d < dim - 1; ++d) KH *= o.Kd[d];
  const int nh = Np / Nq;  // horizontal nodes per element
  s.nlines = KH * nh;
  s.nunk = KV * Nq * S;
  s.bw = Nq * S - 1;
  const size_t st = (size_t)o.K * Np;
  s.line_map.assign((size_t)s.nlines * s.nunk, 0);
  for (int eh = 0; eh < KH; ++eh)
    for (int hn = 0; hn < nh; ++hn) {
      int line = eh * nh + hn;
      int idx[3] = {0, 0, 0}, r = eh;
      for (int d = 0; d < dim - 1; ++d) { idx[d] = r % o.Kd[d]; r /= o.Kd[d]; }
      for (int ev = 0; ev < KV; ++ev) {
        idx[dim - 1] = ev;
        int e = o.elem_of(idx);
        for (int kv = 0; kv < Nq; ++kv) {
          int node = hn + nh * kv;
          for (int sv = 0; sv < S; ++sv)
            s.line_map[(size_t)line * s.nunk + (ev * Nq + kv) * S + sv] = sv * st + (size_t)e * Np + node;
        }
      }
    }
  const int W = 2 * s.bw + 1;
  s.band.assign((size_t)s.nlines * s.nunk * W, 0.0);
  std::vector<double> P(st * S), LP(st * S);
  for (int c = 0; c < W; ++c) {
    std::fill(P.begin(), P.end(), 0.0);
    for (int l = 0; l < s.nlines; ++l)
      for (int u = c; u < s.nunk; u += W) P[s.line_map[(size_t)l * s.nunk + u]] = 1.0;
    op_apply(o, LP.data(), P.data(), 0.0, false);
    for (int l = 0; l < s.nlines; ++l)
      for (int r = 0; r < s.nunk; ++r) {
        int delta = ((c - r) % W + W) % W;
        int j = delta <= s.bw ? r + delta : r + delta - W;
        if (j < 0 || j >= s.nunk) continue;
        s.band[((size_t)l * s.nunk + r) * W + (j - r + s.bw)] = LP[s.line_map[(size_t)l * s.nunk + r]];
      }
  }
  // M = I - dt*a_ii*A  (src/odesolvers.jl:264-268), then no-pivot banded LU
  double fac = -s.dt * s.ima[2][2];
  for (size_t i = 0; i < s.band.size(); ++i) s.band[i] = s.band[i] * fac;
  for (int l = 0; l < s.nlines; ++l)
    for (int r = 0; r < s.nunk; ++r) s.band[((size_t)l * s.nunk + r) * W + s.bw] += 1.0;
  const int bw = s.bw, n = s.nunk;
  for (int l = 0; l < s.nlines; ++l) {
    double* B = s.band.data() + (size_t)l * n * W;
    auto at = [&](int i, int j) -> double& { return B[(size_t)i * W + (j - i + bw)]; };
    for (int kk = 0; kk < n; ++kk) {
      double piv = at(kk, kk);
      for (int i = kk + 1; i <= std::min(kk + bw, n - 1); ++i) {
        double lik = at(i, kk) / piv;
        at(i, kk) = lik;
        for (int j = kk + 1; j <= std::min(kk + bw, n - 1); ++j) at(i, j) = at(i, j) - lik * at(kk, j);
      }
    }
  }
}

void ark_solve_band(const Solver& s, double* x, const double* b) {
  const int bw = s.bw, n = s.nunk, W = 2 * bw + 1;
  par_for(s.nlines, [&](int l) {
    const double* B = s.band.data() + (size_t)l * n * W;
    const size_t* map = s.line_map.data() + (size_t)l * n;
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) {
      double acc = b[map[i]];
      for (int j = std::max(0, i - bw); j < i; ++j) acc = acc - B[(size_t)i * W + (j - i + bw)] * y[j];
      y[i] = acc;
    }
    for (int i = n - 1; i >= 0; --i) {
      double acc = y[i];
      for (int j = i + 1; j <= std::min(n - 1, i + bw); ++j) acc = acc - B[(size_t)i * W + (j - i + bw)] * y[j];
      y[i] = acc / B[(size_t)i * W + bw];
    }
    for (int i = 0; i < n; ++i) x[map[i]] = y[i];
    });
}

void ark_step(Solver& s, double* q) {
  const size_t n = s.n;
  double* Q[3] = {q, s.Qs[0].data(), s.Qs[1].data()};
  auto eval = [&](int i, double* Qi) {
    double ext = s.time + s.exc[i] * s.dt, imt = s.time + s.imc[i] * s.dt;
    if (s.rhs)
      op_apply(*s.rhs, s.exK[i].data(), Qi, ext, false);
    else
      std::fill(s.exK[i].begin(), s.exK[i].end(), 0.0);
    if (s.lin)
      op_apply(*s.lin, s.imK[i].data(), Qi, imt, false);
    else
      std::fill(s.imK[i].begin(), s.imK[i].end(), 0.0);
    if (!s.split_rhs)
      for (size_t j = 0; j < n; ++j) s.exK[i][j] = s.exK[i][j] - s.imK[i][j];
  };
  eval(0, Q[0]);
  for (int i = 1; i < 3; ++i) {
    std::memcpy(s.Qhat.data(), q, n * sizeof(double));
    for (int kk = 0; kk < i; ++kk) {
      double a = s.exa[i][kk], at = s.ima[i][kk];
      for (size_t j = 0; j < n; ++j) s.Qhat[j] = s.Qhat[j] + s.dt * (a * s.exK[kk][j] + at * s.imK[kk][j]);
    }
    if (s.lin)
      ark_solve_band(s, Q[i], s.Qhat.data());
    else
      std::memcpy(Q[i], s.Qhat.data(), n * sizeof(double));
    eval(i, Q[i]);
    // src/odesolvers.jl:378: after stages 2..s, with both stage times
    if (s.stage_cb) s.stage_cb(s.time + s.exc[i] * s.dt, s.time + s.imc[i] * s.dt, Q[i], s.stage_user);
  }
  for (int i = 0; i < 3; ++i)
    for (size_t j = 0; j < n; ++j) q[j] = q[j] + s.dt * (s.exb[i] * s.exK[i][j] + s.imb[i] * s.imK[i][j]);
  s.time += s.dt;
}

void solver_step(Solver& s, double* q) {
  if (s.kind <= 1)
    lsrk_step(s, q);
  else if (s.kind <= 3)
    rlsrk_step(s, q);
  else
    ark_step(s, q);
}

// --------------------------------------------------------- flop counter
struct Cnt {
  double v;
  static long c[6];
  Cnt() : v(0) {}
  Cnt(double x) : v(x) {}
};
long Cnt::c[6];
inline Cnt operator+(Cnt a, Cnt b) { Cnt::c[0]++; return Cnt(a.v + b.v); }
inline Cnt operator-(Cnt a, Cnt b) { Cnt::c[0]++; return Cnt(a.v - b.v); }
inline Cnt operator-(Cnt a) { return Cnt(-a.v); }
inline Cnt operator*(Cnt a, Cnt b) { Cnt::c[1]++; return Cnt(a.v * b.v); }
inline Cnt operator/(Cnt a, Cnt b) { Cnt::c[2]++; return Cnt(a.v / b.v); }
inline bool operator<(Cnt a, Cnt b) { return a.v < b.v; }
inline bool operator<=(Cnt a, Cnt b) { return a.v <= b.v; }
// found by argument-dependent lookup from the physics templates
inline Cnt sqrt(Cnt a) { Cnt::c[3]++; return Cnt(std::sqrt(a.v)); }
inline Cnt log(Cnt a) { Cnt::c[4]++; return Cnt(std::log(a.v)); }
inline Cnt pow(Cnt a, Cnt b) { Cnt::c[5]++; return Cnt(std::pow(a.v, b.v)); }
inline Cnt abs(Cnt a) { return Cnt(std::fabs(a.v)); }
}  // namespace

// ------------------------------------------------------------------ C API
extern "C" {

void* orc_op_create(const orc_desc* d, const double* aux) {
  Op* o = new Op();
  op_build(*o, d, aux);
  return o;
}
void orc_op_destroy(void* op) { delete (Op*)op; }
void orc_op_apply(void* op, double* dq, const double* q, double t, int increment) {
  op_apply(*(Op*)op, dq, q, t, increment != 0);
}
int orc_op_set_curved(void* op, const double* metric, const double* mj, const double* normals,
                      const double* face_mj, const long long* nbr_node, const int* btag, const double* points) {
  Op& o = *(Op*)op;
  if (o.dim != 3 || !metric || !mj || !normals || !face_mj || !nbr_node || !btag) return -1;
  const size_t KN = (size_t)o.K * o.Np, KF = (size_t)o.K * 6 * o.Nfp;
  o.curved = true;
  o.G.assign(metric, metric + 9 * KN);
  o.MJ.assign(mj, mj + KN);
  for (size_t i = 0; i < KN; ++i) o.MJI[i] = 1.0 / o.MJ[i];
  o.fn.assign(normals, normals + 3 * KF);
  o.fMJ.assign(face_mj, face_mj + KF);
  o.fnb.assign(nbr_node, nbr_node + KF);
  o.btag.assign(btag, btag + (size_t)o.K * 6);
  for (size_t i = 0; i < KF; ++i)
    if (o.fnb[i] >= (long long)KN || (o.fnb[i] < 0 && o.btag[i / (6 * o.Nfp) * 6 + (i / o.Nfp) % 6] == 0))
      return -1;
  if (points) o.points.assign(points, points + 3 * KN);
  return 0;
}
void orc_points(void* op, double* x) {
  Op* o = (Op*)op;
  std::memcpy(x, o->points.data(), o->points.size() * sizeof(double));
}
void orc_mj(void* op, double* mj) {
  Op* o = (Op*)op;
  std::memcpy(mj, o->MJ.data(), o->MJ.size() * sizeof(double));
}

void* orc_solver_create(int kind, void* rhs, void* linrhs, double dt, double t0, int split_rhs,
                        int paperversion) {
  Solver* s = new Solver();
  s->kind = kind;
  s->rhs = (Op*)rhs;
  s->lin = (Op*)linrhs;
  s->dt = dt;
  s->time = t0;
  Op* any = s->rhs ? s->rhs : s->lin;
  s->n = (size_t)any->law.ns * any->K * any->Np;
  if (kind == 0 || kind == 2) coeffs_lsrk54(*s);
  if (kind == 1 || kind == 3) coeffs_lsrk144(*s);
  if (kind <= 3) {
    s->dq.assign(s->n, 0.0);
    if (kind >= 2) {
      s->q0.assign(s->n, 0.0);
      s->k.assign(s->n, 0.0);
      size_t ns = s->rkb.size();
      s->rkb_full.assign(ns, 0.0);
      s->rkb_full[ns - 1] = s->rkb[ns - 1];
      for (int i = (int)ns - 2; i >= 0; --i) s->rkb_full[i] = s->rka[i + 1] * s->rkb_full[i + 1] + s->rkb[i];
      s->gamma_r = 1.0;
    }
  } else {
    // ARK23 (src/odesolvers.jl:284-309), Giraldo-Kelly-Constantinescu 2013
    const double r2 = std::sqrt(2.0);
    double a32 = paperversion ? (3 + 2 * r2) / 6 : 0.5;
    double exa[3][3] = {{0, 0, 0}, {2 - r2, 0, 0}, {1 - a32, a32, 0}};
    double ima[3][3] = {{0, 0, 0}, {1 - 1 / r2, 1 - 1 / r2, 0}, {1 / (2 * r2), 1 / (2 * r2), 1 - 1 / r2}};
    double exb[3] = {1 / (2 * r2), 1 / (2 * r2), 1 - 1 / r2};
    double exc[3] = {0, 2 - r2, 1};
    std::memcpy(s->exa, exa, sizeof(exa));
    std::memcpy(s->ima, ima, sizeof(ima));
    std::memcpy(s->exb, exb, sizeof(exb));
    std::memcpy(s->imb, exb, sizeof(exb));
    std::memcpy(s->exc, exc, sizeof(exc));
    std::memcpy(s->imc, exc, sizeof(exc));
    s->split_rhs = split_rhs;
    s->Qhat.assign(s->n, 0.0);
    for (int i = 0; i < 2; ++i) s->Qs[i].assign(s->n, 0.0);
    for (int i = 0; i < 3; ++i) { s->exK[i].assign(s->n, 0.0); s->imK[i].assign(s->n, 0.0); }
    if (s->lin) ark_build_band(*s);
  }
  return s;
}
void orc_solver_destroy(void* s) { delete (Solver*)s; }

int orc_solve(void* sv, double* q, double timeend, int adjust_final) {
  Solver& s = *(Solver*)sv;
  int step = 0;
  bool finalstep = false;
  while (true) {
    ++step;
    double time = s.time;
    if (time + s.dt >= timeend) {
      if (adjust_final) s.dt = timeend - time;
      finalstep = true;
    }
    solver_step(s, q);
    if (finalstep) break;
  }
  return step;
}
void orc_step(void* sv, double* q, int nsteps) {
  for (int i = 0; i < nsteps; ++i) solver_step(*(Solver*)sv, q);
}
void orc_set_stage_callback(void* sv, orc_stage_cb cb, void* user) {
  ((Solver*)sv)->stage_cb = cb;
  ((Solver*)sv)->stage_user = user;
}
double orc_solver_time(void* s) { return ((Solver*)s)->time; }
double orc_solver_dt(void* s) { return ((Solver*)s)->dt; }
double orc_solver_gamma(void* s) { return ((Solver*)s)->gamma_r; }

double orc_weightednorm(void* op, const double* q, double p, double* comp) {
  return weightednorm(*(Op*)op, q, p, comp);
}
double orc_entropyintegral(void* op, const double* q) { return entropyintegral(*(Op*)op, q); }
double orc_entropyproduct(void* op, const double* p, const double* q) {
  return entropyproduct(*(Op*)op, p, q);
}
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

void orc_count_flops(const orc_desc* d, int what, int kind, const double* q1, const double* a1,
                     const double* q2, const double* a2, const double* n, long* counts) {
  Op o;
  double vv[2] = {0, 1};
  orc_desc dd = *d;
  for (int k = 0; k < 3; ++k) { dd.v[k] = vv; dd.K[k] = 1; }
  op_build(o, &dd, nullptr);
  Cnt cq1[5], cq2[5], ca1[8], ca2[8], cn[3], F[3][5], nf[5];
  for (int s = 0; s < 5; ++s) { cq1[s] = Cnt(q1[s]); cq2[s] = Cnt(q2[s]); }
  for (int s = 0; s < 8; ++s) { ca1[s] = Cnt(a1[s]); ca2[s] = Cnt(a2[s]); }
  for (int s = 0; s < 3; ++s) cn[s] = Cnt(n[s]);
  for (int k = 0; k < 6; ++k) Cnt::c[k] = 0;
  if (what == 0) flux(o.law, cq1, ca1, F);
  if (what == 1) twopointflux(kind, o.law, cq1, ca1, cq2, ca2, F);
  if (what == 2) surfaceflux(kind, o.law, cn, cq1, ca1, cq2, ca2, nf);
  if (what == 3) nf[0] = wavespeed(o.law, cn, cq1, ca1);
  for (int k = 0; k < 6; ++k) counts[k] = Cnt::c[k];
}

}  // extern "C"
