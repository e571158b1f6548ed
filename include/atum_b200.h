/*
 * atum_b200 — C ABI of the B200-native DGSEM tendency + time-stepping library
 * (libatumb200.so, sm_100a).
 *
 * Each entry point replaces one call of the reference Atum.jl path; the
 * reference location is given beside it (paths relative to the Atum.jl
 * repository).  All functions return an int status (ATB_OK = 0, negative on
 * error, message from atb_last_error()).  Nothing throws across the ABI.
 * Handles are not thread-safe; distinct handles may be used from distinct
 * threads.
 *
 * Field arguments are host arrays of Ns DEVICE pointers (the components of
 * the reference's StructArray fieldarray), each component holding K*Np
 * float64 values, node index i + Nq*(j + Nq*k) fastest, element slowest
 * (src/dgsem.jl:251, q[ijk, e]).  Streams are cudaStream_t passed as void*
 * (NULL = the legacy default stream).
 *
 * Devices: an operator lives on the CUDA device that was current when it was
 * created (every buffer it and its solvers allocate is that device's memory).
 * Every later call on it, or on a solver built from it, must run with that
 * device current; the library does not switch devices itself.
 * atb_lsrk54_step_noalloc checks this and returns ATB_ERR_INVALID otherwise.
 */
#ifndef ATUM_B200_H
#define ATUM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATB_OK 0
#define ATB_ERR_INVALID (-1)     /* bad argument / unsupported combination */
#define ATB_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define ATB_ERR_NOMEM (-3)       /* device allocation failed */
#define ATB_ERR_NONFINITE (-4)   /* NaN/Inf detected in a state */
#define ATB_ERR_BUDGET (-5)      /* serving: request exceeds the HBM budget */
#define ATB_ERR_TIMEOUT (-6)     /* bounded device wait expired */
#define ATB_ERR_CALLBACK (-7)    /* a stage callback returned nonzero */

/* law: src/balancelaws/{advection,euler,euler_gravity,linear_euler_gravity,shallow_water}.jl */
#define ATB_LAW_ADVECTION 0
#define ATB_LAW_EULER 1
#define ATB_LAW_EULER_GRAVITY 2
#define ATB_LAW_LINEAR_EULER_GRAVITY 3
#define ATB_LAW_SHALLOW_WATER 4
/* numerical fluxes: src/numericalfluxes.jl:25-47 */
#define ATB_FLUX_CENTRAL 0
#define ATB_FLUX_RUSANOV 1
#define ATB_FLUX_EC 2
#define ATB_FLUX_KG 3
#define ATB_FLUX_ROE 4
#define ATB_FLUX_MATRIX 5
/* boundarystate kinds (src/balancelaw.jl:21 and the reference's problem hooks) */
#define ATB_BC_COPY 0
#define ATB_BC_REFLECT 1
#define ATB_BC_INFLOW_ZERO 2
#define ATB_BC_DIRICHLET 3
/* problem source! kinds */
#define ATB_SRC_NONE 0
#define ATB_SRC_CORIOLIS 1
/* precision forms */
#define ATB_PREC_FP64 0
#define ATB_PREC_FP32FLUX 1
/* solvers: src/odesolvers.jl */
#define ATB_LSRK54 0
#define ATB_LSRK144 1
#define ATB_RLSRK54 2
#define ATB_RLSRK144 3
#define ATB_ARK23 4

typedef struct atb_op atb_op;
typedef struct atb_solver atb_solver;

/* DGSEM(; law, grid, surface_numericalflux, volume_form, directions, auxstate)
 * -- src/dgsem.jl:38-56.  The grid is Bennu's brickgrid (per-dimension vertex
 * vectors, periodicity, Cartesian or stacked ordering); the 1-D LGL tables are
 * the cell's nodes, weights and derivatives_1d(cell)[1] (row-major D[i][j] =
 * l_j'(x_i)). */
typedef struct {
  int law, dim, N;
  int K[3];
  const double* vertices[3]; /* host, K[d]+1 each */
  int periodic[3];
  int stacked;               /* StackedOrdering{CartesianOrdering} */
  int volume_form;           /* 0 WeakForm, 1 FluxDifferencingForm */
  int volume_flux;           /* two-point flux of the flux-differencing form */
  int fd_kernel;             /* 0 :per_dir, 1 :per_dir_symmetric, 2 :naive (same math) */
  int surface_flux;
  int directions;            /* bitmask, bit d = direction d+1 */
  double gamma, grav;
  double adv_u[3];
  int sphere, pde_level_balance;
  int bc_kind;
  double bc_state[2][5];     /* Dirichlet: tag 1 -> [0], others -> [1] */
  int source_kind;
  double omega[3];
  int sw_topography;         /* shallow-water bathymetry extension (aux = b, grad b) */
  int naux;
  int precision;             /* ATB_PREC_* */
  const double* lgl_nodes;   /* host, Nq */
  const double* lgl_weights; /* host, Nq */
  const double* lgl_D;       /* host, Nq*Nq */
} atb_op_desc;

int atb_version(void);
const char* atb_last_error(void);
int atb_device_count(int* n);

/* DGSEM construction (src/dgsem.jl:38-56); aux_host: naux*K*Np values in the
 * field layout, evaluated on the host like auxiliary.(law, points(grid)).
 * aux_host may be NULL: the aux fields then start at zero and are meant to be
 * filled by atb_op_set_aux. */
int atb_op_create(const atb_op_desc* desc, const double* aux_host, atb_op** out);
/* Replaces the aux fields (naux*K*Np values, component-major) from host or
 * device memory -- the reference evaluates auxiliary.(law, points(grid)) on
 * the device (src/dgsem.jl:47-49); a caller that does the same passes its
 * device array here.  Ordered on `stream`. */
int atb_op_set_aux(atb_op* op, const double* aux, void* stream);
int atb_op_destroy(atb_op* op);
int atb_op_dims(const atb_op* op, int* ns, int* K, int* Np);

/* Curved elements: DGSEM(; law, grid = cubedspheregrid(cell, vr, KH), ...)
 * (src/dgsem.jl:38-56 with Bennu's metrics(grid) / facemetrics(grid) of a
 * curved grid; experiment/euler_gravity/acousticwave.jl:90-99).  The
 * descriptor gives law, order, forms, fluxes, directions, constants and the
 * element counts K = {6*KH, KH, KV} with stacked = 1 (vertex vectors: any
 * increasing vectors of K[d]+1 values; they are not read for the geometry).
 * Host arrays, Np = Nq^3, Nfp = Nq^2, face f = 2*dir + side, face node j
 * enumerating the two tangential dimensions in increasing order, the lower
 * one fastest:
 *   metric[((dir*3 + c)*K + e)*Np + n]  d xi_dir / d x_c
 *   mj[e*Np + n]                        M J (LGL weights times the Jacobian)
 *   normals[((e*6 + f)*Nfp + j)*3 + c]  outward unit normal
 *   face_mj[(e*6 + f)*Nfp + j]          face weights times |J grad xi_dir|
 *   nbr_node[(e*6 + f)*Nfp + j]         the neighbour's node e'*Np + n', or
 *                                       -1 on a boundary face
 *   btag[e*6 + f]                       boundary tag (0 interior)
 * 3-D Euler, Euler-gravity (weak form; flux differencing with the central,
 * entropy-conservative or Kennedy-Gruber flux) and linear Euler-gravity (weak
 * form); surface fluxes central and Rusanov, and for the nonlinear laws also
 * entropy conservative, Kennedy-Gruber, Roe and matrix dissipation; FP64.
 * The operator works with every solver, ARK23's banded vertical solve
 * included (one band per vertical line of nodes). */
typedef struct {
  const double* metric;
  const double* mj;
  const double* normals;
  const double* face_mj;
  const long long* nbr_node;
  const int* btag;
} atb_curved_geometry;
int atb_op_create_curved(const atb_op_desc* desc, const double* aux_host, const atb_curved_geometry* geo,
                         atb_op** out);

/* Multi-instance batching (no reference counterpart; the reference builds one
 * DGSEM per problem, src/dgsem.jl:38-56, and steps each alone).  n instances
 * that share law, order, forms, fluxes, directions, precision, constants and
 * problem kinds -- grids may differ -- become one operator whose elements are
 * the instances' elements concatenated (instance i owns elements
 * [first_i, first_{i+1})); neighbour indices stay inside each instance, so
 * every instance's result is bitwise the one it gets alone.  Fields of the
 * packed operator are the instances' fields concatenated per component.
 * aux_hosts[i]: instance i's aux fields (naux*K_i*Np, component-major). */
int atb_op_create_batch(const atb_op_desc* descs, int n, const double* const* aux_hosts, atb_op** out);
/* instance count and the n+1 element offsets (first_elements may be NULL) */
int atb_op_instances(const atb_op* op, int* n, int* first_elements);
/* Serving support (no reference counterpart).  atb_op_set_active limits
 * tendency launches to the first n instances (elements [0, first_n)); the
 * others keep their state untouched by applications of the operator.  It
 * changes a host-side launch parameter, so a captured CUDA graph keeps the
 * value it was captured with.  atb_op_set_instance_aux replaces instance i's
 * aux fields (naux*K_i*Np host doubles, component-major) with copies ordered on
 * `stream`; atb_op_copy_instance_aux copies instance src's aux fields over
 * instance dst's (equal sizes) on `stream`. */
int atb_op_set_active(atb_op* op, int n_instances);
/* Element pools for serving (no reference counterpart).  atb_op_create_pool
 * makes an operator of `kind` (law, order, forms, fluxes, precision, problem
 * kinds and constants of the descriptor; its grid is ignored) with room for
 * capacity_elements elements and none active.  atb_op_place_instance writes
 * the geometry (metrics, neighbour table offset by first_element) and aux
 * fields of the instance `desc` (same kind, any grid) into elements
 * [first_element, first_element + K) with copies ordered on `stream` (the
 * geometry goes through the pool's own page-locked staging; aux_host may be
 * host or device memory: a pageable host source may be released on return, a
 * page-locked or device one must stay valid until the copies have run).  atb_op_set_active_elements sets how
 * many leading elements tendency launches cover; a caller keeps its placed
 * instances inside that prefix.  Pools have no banded solve (ARK23). */
int atb_op_create_pool(const atb_op_desc* kind, int capacity_elements, atb_op** out);
int atb_op_place_instance(atb_op* op, int first_element, const atb_op_desc* desc, const double* aux_host,
                          void* stream);
int atb_op_set_active_elements(atb_op* op, int n_elements);
/* Moves n_elements elements (their metrics, neighbour rows and aux fields)
 * from [src_first, +n) to [dst_first, +n) on the device, ordered on `stream`.
 * Neighbour rows are stored relative to their element, so a placed instance
 * moves unchanged.  Overlapping ranges go through `scratch`, device memory of
 * n_elements * (8*Np*naux + 56) bytes (may be NULL otherwise).  The state
 * fields are the caller's to move. */
int atb_op_move_instance(atb_op* op, int dst_first, int src_first, int n_elements, void* scratch, void* stream);
int atb_op_set_instance_aux(atb_op* op, int i, const double* aux_host, void* stream);
int atb_op_copy_instance_aux(atb_op* op, int dst, int src, void* stream);
/* Launch-shape tuning (no reference counterpart): times the tendency kernel
 * for every admissible elements-per-CTA count on state q (scratch: ns*K*Np
 * doubles of device memory, overwritten) and keeps the fastest; *chosen gets
 * it.  Results do not depend on the shape.  atb_op_set_launch sets it. */
int atb_op_autotune(atb_op* op, const double* const* q, double* scratch, void* stream, int* chosen);
int atb_op_set_launch(atb_op* op, int elements_per_cta);
/* Persistent launches (no reference counterpart): with ctas > 0 every tendency
 * launch of the operator (its fused ARK23 stages included) runs at most `ctas`
 * CTAs, each walking the element tiles -- across all packed instances,
 * whatever their sizes -- with a grid stride; 0 restores one CTA per tile.
 * Results do not depend on it.  Persistent kernels exist for brick operators
 * with the Rusanov surface flux at N = 3..5: 3-D Euler-gravity (EC volume
 * flux; with ARK23 also the fused stage), 2-D Euler (EC), 2-D shallow water
 * (EC, FP32-flux EC); ATB_ERR_INVALID otherwise. */
int atb_op_set_persistent(atb_op* op, int ctas);

/* (dg::DGSEM)(dq, q, time; increment) -- src/dgsem.jl:59-98 */
int atb_op_apply(atb_op* op, double* const* dq, const double* const* q, double time, int increment, void* stream);

/* LSRK54/LSRK144/RLSRK54/RLSRK144/ARK23 constructors -- src/odesolvers.jl:59-67,138-146,284-309.
 * rhs may be NULL for ARK23 (ARK23(nothing, linrhs, ...)); linrhs is NULL for the explicit kinds.
 * For ARK23 the constructor probes linrhs and factors I - dt a_ii L once per distinct
 * vertical column (src/bandedsystem.jl:1-15, src/odesolvers.jl:264-268).
 * dt must be finite and positive, t0 finite (ATB_ERR_INVALID otherwise). */
int atb_solver_create(int kind, atb_op* rhs, atb_op* linrhs, double dt, double t0, int split_rhs, int paperversion,
                      atb_solver** out);
int atb_solver_destroy(atb_solver* s);
/* dostep! repeated nsteps times -- src/odesolvers.jl:47-57,103-136,312-388 */
int atb_solver_step(atb_solver* s, double* const* q, int nsteps, void* stream);
/* solve!(q, timeend, solver; adjust_final) -- src/odesolvers.jl:9-26.  A step
 * that would not advance the clock towards timeend (dt <= 0 or below the
 * clock's resolution) is rejected with ATB_ERR_INVALID instead of looping. */
int atb_solve(atb_solver* s, double* const* q, double timeend, int adjust_final, int* steps_out, void* stream);
int atb_solver_get(const atb_solver* s, double* time, double* dt, double* gamma);
/* dt must be finite and >= 0 (solve! sets dt = timeend - time on its final step) */
int atb_solver_set_dt(atb_solver* s, double dt);
/* Checkpoint / resume (no reference counterpart: the reference writes only VTK
 * snapshots, experiment/euler_gravity/risingbubble.jl:81-95): restores the
 * clock and the last relaxation factor (the RLSRK Newton's starting point)
 * that atb_solver_get reported, so a solver rebuilt on the same operators and
 * dt continues a checkpointed run bit for bit.  Non-finite values are
 * rejected. */
int atb_solver_set_state(atb_solver* s, double time, double gamma);
/* Per-instance time steps for an LSRK solver over a packed operator (no
 * reference counterpart): dt_host holds one step per instance (host memory,
 * copied synchronously; 0 freezes an instance); NULL returns to the solver's
 * single dt.  The solver's own clock still advances by its dt; per-instance
 * times are the caller's bookkeeping.  atb_solver_set_element_dt instead hands
 * the solver a caller-owned device array of one time step per element (K
 * doubles), read by every later stage, so its contents may change between
 * steps without another call; NULL returns to the single dt. */
int atb_solver_set_instance_dt(atb_solver* s, const double* dt_host);
/* ARK23 kernel fusion (no reference counterpart): when the explicit operator is
 * 3-D Euler-gravity with an EC / FP32-flux EC volume flux and the implicit one
 * the weak-form linear Euler-gravity operator along z on the same grid and aux
 * fields (split_rhs = false), each stage runs both as one kernel; on by
 * default when possible.  enable = 0 runs them as two launches; enabling a
 * solver that cannot fuse is an error. */
int atb_solver_fuse(atb_solver* s, int enable);
int atb_solver_set_element_dt(atb_solver* s, const double* dte_device);

/* after_stage of solve!(q, timeend, solver; after_stage) -- src/odesolvers.jl:
 * 10-11,23, called at :54 (LSRK), :119 (RLSRK) and :378 (ARK).  With a
 * callback set, every atb_solver_step / atb_solve calls
 *   cb(ex_time, im_time, q_stage, user)
 * on the host after each stage's launches have been enqueued on the call's
 * stream: LSRK / RLSRK after every stage, with both times the stage time and
 * q_stage the caller's q (the callback may change it; the next stage starts
 * from it); ARK23 after stages 2 and 3, with the explicit and implicit stage
 * times and q_stage the solver's stage state Q_i (Ns device pointers, valid
 * during the call).  A callback that reads device memory from the host must
 * synchronise the stream first; device work it enqueues on that stream is
 * ordered before the next stage.  A nonzero return stops the step with
 * ATB_ERR_CALLBACK.  With the accumulated ARK23 path (split_rhs = 0 with a
 * banded solve) the step's update of q is already applied when the stage-3
 * callback runs.  NULL clears the callback.  (No counterpart in the C sense:
 * the reference passes a Julia closure.) */
typedef int (*atb_stage_callback)(double ex_time, double im_time, double* const* q_stage, void* user);
int atb_solver_set_stage_callback(atb_solver* s, atb_stage_callback cb, void* user);
/* Exchange hook (no reference counterpart; the element-slab sharding of one
 * problem over several GPUs, atum_b200.sharded): cb(state, user) runs on the
 * host before every tendency launch that reads a new state -- each LSRK /
 * RLSRK stage (the stage's input state) and each ARK23 stage (q, then the
 * stage states Q_2, Q_3 after their solves) -- with the Ns device pointers of
 * that state; it fills the state's ghost elements with work ordered on the
 * solver's stream.  A nonzero return stops the step with ATB_ERR_CALLBACK.
 * NULL clears it.  Not called by atb_lsrk54_step_noalloc. */
typedef int (*atb_exchange_callback)(double* const* state, void* user);
int atb_solver_set_exchange_callback(atb_solver* s, atb_exchange_callback cb, void* user);

/* measures -- src/measures.jl:6-33 (p = 2 or INFINITY); results to host memory */
int atb_weightednorm(atb_op* op, const double* const* q, double p, double* comp_host, double* total_host,
                     void* stream);
int atb_entropyintegral(atb_op* op, const double* const* q, double* out_host, void* stream);
int atb_entropyproduct(atb_op* op, const double* const* p, const double* const* q, double* out_host, void* stream);
/* NaN/Inf scan of a state: ATB_ERR_NONFINITE if any */
int atb_check_finite(atb_op* op, const double* const* q, void* stream);

/* device FP64 FMA throughput probe (measurement utility): runs a fixed FMA loop
 * on every SM and returns the achieved FP64 TFLOP/s. */
int atb_probe_fp64_peak(double* tflops, void* stream);

/* Launch profiling (measurement utility, no reference counterpart).  When
 * enabled, every kernel the library launches is bracketed by CUDA events on
 * its own stream; atb_profile_read resolves them (synchronising) and returns
 * launches and total milliseconds per kernel class:
 *   0 tendency of an explicit / nonlinear operator, 1 tendency of an implicit
 *   (linear) operator, 2 banded solve, 3 stage combinations, 4 reductions. */
#define ATB_PROF_TEND 0
#define ATB_PROF_TEND_LIN 1
#define ATB_PROF_BAND 2
#define ATB_PROF_COMBINE 3
#define ATB_PROF_REDUCE 4
int atb_profile_enable(int on);
int atb_profile_reset(void);
int atb_profile_read(int kclass, long* launches, double* total_ms);
/* number of kernels launched by the library since load (all classes) */
int atb_launch_count(long* n);

/* LSRK54 steps of an existing operator that allocate nothing.  No counterpart
 * in the reference: it is for callers that cannot call cudaMalloc around a time
 * step (an application whose device memory belongs to its own pool allocator,
 * or a latency-critical loop that must not pay cudaMalloc/cudaFree's implicit
 * synchronisation).  Same arithmetic as ATB_LSRK54 through atb_solver_step; the
 * stage increment and the second state buffer live in a library-owned static
 * device array of 2 * ATB_NOALLOC_MAX_DOFS doubles (8 MiB, held by every GPU that
 * loads the library until exit).  States with more than ATB_NOALLOC_MAX_DOFS
 * DOFs (ns*K*Np) are rejected with ATB_ERR_INVALID.  The first call on a device
 * looks up the array's device address for that device (cudaGetSymbolAddress);
 * make that first call before any stream capture.  All calls share the array:
 * calls that overlap on the GPU race on it and must be serialised by the caller;
 * the increment is cleared at the start of each call.  The call must run with
 * the operator's creating device current (the array's address differs per
 * device); otherwise, and for a non-finite dt, it returns ATB_ERR_INVALID.
 * Only the operator's active elements are stepped and written back. */
#define ATB_NOALLOC_MAX_DOFS 524288
int atb_lsrk54_step_noalloc(atb_op* op, double* const* q, double dt, int nsteps, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ATUM_B200_H */
