/* TEST INFRASTRUCTURE — CPU oracle, not the product.
 *
 * C API of the CPU restatement of Atum.jl's DGSEM tendency + time stepping
 * (reference: src/dgsem.jl, src/odesolvers.jl, src/measures.jl,
 * src/bandedsystem.jl, src/balancelaws/*.jl) together with the parts of the
 * un-vendored Bennu 0.3 dependency the path needs (LGL cell, brick grid,
 * metrics, face maps, banded LU).  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only as the checker
 * or the timed CPU baseline: the product path never calls it.
 *
 * Field layout: SoA, state s of element e at node n is x[(s*K + e)*Np + n]
 * (the reference's StructArray components, each Np x K column-major).
 */
#ifndef ATUM_ORACLE_H
#define ATUM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int law;            /* 0 advection, 1 euler, 2 euler+gravity, 3 linear euler+gravity, 4 shallow water */
  int dim;            /* 1..3 */
  int N;              /* polynomial order, Nq = N+1 */
  int K[3];           /* elements per dimension */
  const double* v[3]; /* vertex coordinates per dimension (K[d]+1 each) */
  int periodic[3];
  int stacked;        /* 1: StackedOrdering (last dim fastest), 0: CartesianOrdering */
  int volume_form;    /* 0 WeakForm, 1 FluxDifferencingForm */
  int volume_flux;    /* flux kind for flux differencing */
  int fd_kernel;      /* 0 :per_dir, 1 :per_dir_symmetric, 2 :naive */
  int surface_flux;   /* 0 central 1 rusanov 2 ec 3 kg 4 roe 5 matrix */
  int directions;     /* bitmask, bit d -> direction d+1 */
  double gamma, grav;
  double adv_u[3];
  int sphere, pde_level_balance;
  int bc_kind;        /* 0 copy, 1 reflect, 2 inflow-zero, 3 dirichlet */
  double bc_state[2][5];
  int source_kind;    /* 0 none, 1 coriolis */
  double omega[3];
  int sw_topography;
  int naux;
} orc_desc;

void* orc_op_create(const orc_desc* d, const double* aux);
void orc_op_destroy(void* op);
void orc_op_apply(void* op, double* dq, const double* q, double t, int increment);
/* curved 3-D elements (a cubed-sphere shell): per-node metric terms
 * metric[((dir*3 + c)*K + e)*Np + n] = d xi_dir / d x_c, M J per node, per face
 * node (face f = 2*dir + side, face node j as the brick's face tables) the
 * outward unit normal normals[((e*6 + f)*Nfp + j)*3 + c], faceMJ, and the
 * neighbour's global node index e'*Np + n' (-1 with btag[e*6 + f] != 0 on a
 * boundary face); points (3 x K x Np) may be NULL.  Returns 0, or -1 on bad
 * input.  Replaces the brick geometry the descriptor built. */
int orc_op_set_curved(void* op, const double* metric, const double* mj, const double* normals,
                      const double* face_mj, const long long* nbr_node, const int* btag, const double* points);
void orc_points(void* op, double* x);   /* dim x K x Np */
void orc_mj(void* op, double* mj);      /* K x Np */

/* kind: 0 LSRK54, 1 LSRK144, 2 RLSRK54, 3 RLSRK144, 4 ARK23 (rhs may be NULL for ARK23) */
void* orc_solver_create(int kind, void* rhs, void* linrhs, double dt, double t0, int split_rhs,
                        int paperversion);
void orc_solver_destroy(void* s);
int orc_solve(void* s, double* q, double timeend, int adjust_final); /* returns steps taken */
void orc_step(void* s, double* q, int nsteps);
/* after_stage (src/odesolvers.jl:10-11,23,54,119,378): cb(ex_time, im_time,
 * stage state, user) after every LSRK / RLSRK stage (both times the stage
 * time, the state q) and after ARK23 stages 2 and 3 (the stage state Q_i);
 * NULL clears it */
typedef void (*orc_stage_cb)(double ex_time, double im_time, const double* q_stage, void* user);
void orc_set_stage_callback(void* s, orc_stage_cb cb, void* user);
double orc_solver_time(void* s);
double orc_solver_dt(void* s);
double orc_solver_gamma(void* s);

double orc_weightednorm(void* op, const double* q, double p, double* componentwise_out);
double orc_entropyintegral(void* op, const double* q);
double orc_entropyproduct(void* op, const double* p, const double* q);
void orc_set_threads(int n);

/* flop counter: what 0 = flux, 1 = twopointflux(kind), 2 = surfaceflux(kind), 3 = wavespeed.
 * counts[0..5] = add/sub, mul, div, sqrt, log, pow */
void orc_count_flops(const orc_desc* d, int what, int kind, const double* q1, const double* a1,
                     const double* q2, const double* a2, const double* n, long* counts);

#ifdef __cplusplus
}
#endif
#endif
