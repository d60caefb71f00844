/* ddhdg_b200 -- C ABI of the B200 (sm_100a) HDG hot path for the Van
 * Roosbroeck drift-diffusion system.
 *
 * The library replaces, for structured Cartesian meshes of segments, quads
 * and hexes, the per-Newton-step work that the reference (spiani/ddhdg) does
 * in
 *   NPSolver<dim,Problem>::assemble_system(reconstruct, thermo_eq, mt)
 *       include/np_solver.h:627-630, include/assembling_methods.template.h:10-89
 *   the per-cell worker assemble_system_one_cell<...>
 *       include/assembling_methods.template.h:2290-2748
 *   LocalCondenser::condense_ct_matrix   src/local_condenser.cpp:142-160
 *   copy_local_to_global                 src/np_solver.cpp:1293-1322
 *   the Newton loop private_run          src/np_solver.cpp:1452-1561
 *
 * Conventions
 *   - Every entry point returns an int status (DDHDG_OK == 0); no C++
 *     exception crosses the boundary.
 *   - Arrays are device pointers owned by the caller unless the name of the
 *     argument ends in _host.
 *   - Cells are numbered lexicographically (x fastest).  The degrees of
 *     freedom of cell c are contiguous: cell_state[c * Nc_all + ...] with the
 *     per-cell order [E_0..E_{d-1}, V, Wn_0.., n, Wp_0.., p] x (k+1)^d
 *     Gauss-Lobatto nodes (x fastest) -- the FESystem order of the
 *     reference's FE_DGQ spaces (src/np_solver.cpp:292-325).
 *   - Faces are numbered axis by axis (all x-normal faces, then y, then z),
 *     lexicographically inside each axis.  The full trace vector is
 *     trace_state[F][3][nf] (components V, n, p; (k+1)^(d-1) Gauss-Lobatto
 *     nodes of FE_FaceQ).  The restricted trace system (enabled components
 *     only) numbers dof (F, comp, m) as (F * ncomp + comp) * nf + m.
 *   - All physical quantities are already rescaled by the Adimensionalizer
 *     (include/adimensionalizer.h:28-262) except the band data and the SRH
 *     intrinsic density, which the kernels rescale like the reference.
 */
#ifndef DDHDG_B200_H
#define DDHDG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *ddhdg_stream_t; /* a cudaStream_t */

enum ddhdg_status
{
  DDHDG_OK             = 0,
  DDHDG_BAD_ARG        = 1,
  DDHDG_OOM            = 2,
  DDHDG_SINGULAR_PIVOT = 3, /* a local (cell) factorisation met a zero pivot */
  DDHDG_REFINE_STALLED = 4, /* mixed precision refinement did not converge */
  DDHDG_TIMEOUT        = 5,
  DDHDG_CUDA_ERROR     = 6,
  DDHDG_NOT_CONVERGED  = 7, /* Newton reached the iteration cap */
  DDHDG_SOLVER_ERROR   = 8, /* the global trace solve failed */
  DDHDG_NO_DEVICE      = 9
};

enum ddhdg_flux
{
  DDHDG_FLUX_USE_CELL  = 0, /* DDFluxType::use_cell */
  DDHDG_FLUX_USE_TRACE = 1, /* DDFluxType::use_trace */
  DDHDG_FLUX_QIU_SHI   = 2  /* DDFluxType::qiu_shi_stabilization */
};

enum ddhdg_bc
{
  DDHDG_BC_NONE      = 0,
  DDHDG_BC_DIRICHLET = 1,
  DDHDG_BC_NEUMANN   = 2
};

/* Problem description (host memory; copied to the device by
 * ddhdg_ctx_create).  Mirrors Ddhdg::Problem (include/problem.h:13-46) with
 * the solver parameters (include/np_solver_parameters.h:261-404). */
typedef struct ddhdg_problem_desc
{
  int    dim;    /* 1, 2 or 3 */
  int    degree; /* polynomial degree k of V, n and p (cell and trace) */
  int    n[3];   /* cells per axis */
  double origin[3];
  double h[3];   /* cell size per axis in mesh units */

  int enabled[3]; /* V, n, p */
  int flux;       /* enum ddhdg_flux */
  int phi_linearize;
  /* bit 0: consistent sign of the E coupling in the cell drift terms;
   * bit 1: recombination derivatives scaled by the doping magnitude.
   * 0 reproduces the reference's Jacobian exactly. */
  int jacobian_fix;
  int precision; /* 0: FP64, 1: FP32 local factorisation + FP64 residuals */

  double eps;         /* rescaled permittivity */
  double mu_n, mu_p;  /* rescaled mobilities */
  double temperature; /* kelvin (constant over the device) */
  double thermal_voltage_rescale;
  double V_rescale, n_rescale, rec_rescale;
  double nc, nv, ec_eV, ev_eV; /* band densities and edges (physical) */

  int    rec_type; /* 0: linear a + (b n + c p), 1: SRH fixed temperature */
  double srh_ni, srh_tau_n, srh_tau_p;
  const double *rec_a_host, *rec_b_host, *rec_c_host; /* [ncells*nqc] or NULL */

  const double *doping_host; /* [ncells*nqc] rescaled doping at cell qps */
  double        tau[3];      /* fixed tau per component (rescaled) */
  const double *tau_host;    /* [ncells*2*dim*3] per cell/face tau, or NULL */
  const int32_t *face_bc_host;   /* [nfaces*3] enum ddhdg_bc */
  const double  *face_bc_val_host; /* [nfaces*3*nqf] rescaled BC data */
} ddhdg_problem_desc;

typedef struct ddhdg_ctx ddhdg_ctx;

typedef struct ddhdg_sizes
{
  int64_t ncells, nfaces;
  int     Nc_all; /* cell dofs per cell (all components) */
  int     Nt;     /* restricted trace dofs per cell */
  int     ncomp;  /* enabled components */
  int     nqc, nqf, nb, nf;
  int64_t n_trace_dofs; /* restricted global trace dofs */
  int64_t nnz;          /* nonzeros of the global trace matrix */
} ddhdg_sizes;

/* NPSolver construction + setup_overall_system (src/np_solver.cpp:553-655):
 * geometry tables, coefficient tables, trace sparsity.  Replaces
 * NPSolver::NPSolver + setup_overall_system + setup_restricted_trace_system. */
int ddhdg_ctx_create(const ddhdg_problem_desc *desc, ddhdg_ctx **ctx);
int ddhdg_ctx_destroy(ddhdg_ctx *ctx);
int ddhdg_get_sizes(const ddhdg_ctx *ctx, int thermo_eq, ddhdg_sizes *out);

/* replace_boundary_condition (src/np_solver.cpp:2160-2233): new BC types and
 * data for every face; the sparsity is unchanged. */
int ddhdg_set_boundary(ddhdg_ctx *ctx, const int32_t *face_bc_host,
                       const double *face_bc_val_host);
/* set_enabled_components (src/np_solver.cpp:1064-1093). */
int ddhdg_set_enabled(ddhdg_ctx *ctx, int V, int n, int p);

/* assemble_system(false, thermo_eq) per-cell part: for every cell, assemble
 * the local HDG system and condense it onto the cell's trace dofs
 * (include/assembling_methods.template.h:2290-2686).  Outputs per cell:
 *   tt   [ncells][Nt][Nt]  condensed trace matrix, Dirichlet rows/cols zero
 *   rhs  [ncells][Nt]      condensed right-hand side
 *   dflag[ncells][Nt]      1 where the trace dof is Dirichlet-constrained
 *   dval [ncells][Nt]      projected Dirichlet increment (T:1592-1691)
 * The cell's reconstruction data stays in the context for ddhdg_reconstruct.
 * cell_state [ncells][Nc_all], trace_state [nfaces][3][nf] on the device. */
int ddhdg_assemble_condense(ddhdg_ctx *ctx, const double *cell_state,
                            const double *trace_state, int thermo_eq,
                            double *tt, double *rhs, int32_t *dflag,
                            double *dval, ddhdg_stream_t stream);

/* Fixed size of the static scratch of ddhdg_assemble_condense_noalloc. */
#define DDHDG_NOALLOC_SCRATCH_BYTES (16u << 20)

/* No counterpart in the reference.  The same per-cell outputs as
 * ddhdg_assemble_condense, from a call that allocates no device memory: the
 * kernel's scratch (the per-cell Y cache and, for cells whose right-hand-side
 * block does not fit in shared memory, that block) lives in a static device
 * array of DDHDG_NOALLOC_SCRATCH_BYTES (16 MiB) inside the library.
 * It is for callers that cannot allocate device memory at this point: a
 * process whose device memory is already held by its own pool allocator (a
 * framework's caching allocator), where a cudaMalloc inside the library would
 * fail or fragment that pool, and latency-bound loops that cannot take the
 * device-wide synchronisation of cudaFree.
 * Limits.  A problem that needs more scratch than 16 MiB (about 2000 cells of
 * the 2D degree-2 three-component system) is rejected with DDHDG_BAD_ARG
 * before anything is launched.  The first call on each device looks up the
 * array's address (cudaGetSymbolAddress, with that device current); that
 * first call must happen before any stream capture begins.  All calls on one
 * device share the one array and the context's status word: overlapping calls
 * (several threads, or several streams in flight) race.  The Y cache written
 * here is not the one ddhdg_reconstruct reads; reconstruction still follows
 * ddhdg_assemble_condense. */
int ddhdg_assemble_condense_noalloc(ddhdg_ctx *ctx, const double *cell_state,
                                    const double *trace_state, int thermo_eq,
                                    double *tt, double *rhs, int32_t *dflag,
                                    double *dval, ddhdg_stream_t stream);

/* get_local_cell_system(level, index, thermo_eq) (src/np_solver.cpp:
 * 2337-2445), the per-cell parity probe: the local system of each listed cell
 * as the reference's per-cell worker leaves it before the Schur complement
 * (include/assembling_methods.template.h:2290-2647 with the Dirichlet columns
 * of ct folded into cc_rhs, src/local_condenser.cpp:142-160), assembled on the
 * device term by term.  Nc = ncomp * (dim + 1) * (k + 1)^dim enabled cell
 * dofs in the FESystem order restricted to the enabled components, Nt as in
 * ddhdg_get_sizes.  Cells: the device list cells[ncells], or, with cells ==
 * NULL, the range [first_cell, first_cell + ncells).  Outputs (device, any
 * may be NULL), per listed cell in list order:
 *   cc [Nc][Nc], ct [Nc][Nt], tc [Nt][Nc], tt [Nt][Nt], c [Nc], t [Nt]. */
int ddhdg_local_cell_system(ddhdg_ctx *ctx, const double *cell_state,
                            const double *trace_state, int thermo_eq,
                            int64_t ncells, const int64_t *cells,
                            int64_t first_cell, double *cc, double *ct,
                            double *tc, double *tt, double *c, double *t,
                            ddhdg_stream_t stream);

/* The reference's per-cell algorithm as written, on the device (FP64): the
 * full local system of every cell assembled term by term
 * (include/assembling_methods.template.h:134-2160), Dirichlet columns folded
 * (src/local_condenser.cpp:142-160), then the Schur complement through an LU
 * factorisation of the row-equilibrated cc with partial pivoting (in place of
 * cc.gauss_jordan(), T:2651-2686).  Same outputs as ddhdg_assemble_condense;
 * it keeps no reconstruction data: ddhdg_reconstruct_plain assembles the
 * cell systems again with the trace update and solves them (T:2688-2697),
 * as the reference's second assemble_system pass does.  This is the plain
 * FP64 GPU path that the block-eliminated kernels are measured against. */
int ddhdg_assemble_condense_plain(ddhdg_ctx *ctx, const double *cell_state,
                                  const double *trace_state, int thermo_eq,
                                  double *tt, double *rhs, int32_t *dflag,
                                  double *dval, ddhdg_stream_t stream);
int ddhdg_reconstruct_plain(ddhdg_ctx *ctx, const double *cell_state,
                            const double *trace_state,
                            const double *update_trace, double *update_cell,
                            int thermo_eq, ddhdg_stream_t stream);

/* copy_local_to_global (src/np_solver.cpp:1293-1322): scatter the per-cell
 * condensed systems into the global CSR trace matrix (values[nnz], rows and
 * columns from ddhdg_get_csr) and rhs[n_trace_dofs]; Dirichlet rows become
 * identity rows whose rhs is the constrained value. */
int ddhdg_scatter(ddhdg_ctx *ctx, const double *tt, const double *rhs,
                  const int32_t *dflag, const double *dval, double *csr_values,
                  double *global_rhs, int thermo_eq, ddhdg_stream_t stream);
/* Global trace sparsity (device arrays owned by the context). */
int ddhdg_get_csr(ddhdg_ctx *ctx, int thermo_eq, const int32_t **row_ptr,
                  const int32_t **col_idx);

/* solve_linear_problem (src/np_solver.cpp:1326-1354) on the device:
 * x = A^-1 b for the global trace system (cuSOLVER sparse QR). */
int ddhdg_solve_trace(ddhdg_ctx *ctx, const double *csr_values,
                      const double *global_rhs, double *x, int thermo_eq,
                      ddhdg_stream_t stream);

/* copy_local_to_global + solve_linear_problem (src/np_solver.cpp:1293-1354)
 * in one call: x = A^-1 b for the global trace system assembled from the
 * per-cell condensed blocks of ddhdg_assemble_condense (Dirichlet dofs take
 * their projected values).  Nested-dissection multifrontal LU on the device;
 * the first call on a context (and mode) builds the elimination tree and
 * allocates the fronts.  x has n_trace_dofs entries in the restricted trace
 * order. */
int ddhdg_solve_condensed(ddhdg_ctx *ctx, const double *tt, const double *rhs,
                          const int32_t *dflag, const double *dval, double *x,
                          int thermo_eq, ddhdg_stream_t stream);

/* No counterpart in the reference (its solve is UMFPACK or GMRES on the
 * host).  Whether ddhdg_solve_condensed (and so ddhdg_newton) captures the
 * numeric sequence of the trace solve in a CUDA graph on its second call with
 * the same buffers and replays it afterwards: enable = 1, the default.  With
 * enable = 0 every solve launches its kernels directly: no capture or
 * instantiation cost, for callers whose buffers change from call to call or
 * that make only a couple of solves per context.  Both give the same bits. */
int ddhdg_set_solver_graphs(ddhdg_ctx *ctx, int enable);

/* No counterpart in the reference.  Frees the trace solver of one mode
 * (thermo_eq 0: the full system, 1: the equilibrium system): its fronts,
 * library handles, side streams and graphs.  The next solve of that mode
 * builds it again (the host plan comes from the process-wide cache).  A
 * serving loop calls it when a request leaves the equilibrium phase.  No
 * solve of that mode may be in flight (the caller's to ensure); freeing
 * device memory waits for the device. */
int ddhdg_release_solver(ddhdg_ctx *ctx, int thermo_eq);

/* No counterpart in the reference (its solve is UMFPACK or GMRES on the
 * host).  Device bytes that the trace solver of a structured mesh allocates
 * (fronts, pivots, maps), from its host-side plan alone: `dim`, cells per
 * direction n[0..dim-1], `degree` and the enabled components `ncomp` (1-3;
 * 1 for the thermodynamic-equilibrium system).  No device is touched; the
 * plan is kept in the process-wide cache, so a solver built later on the same
 * mesh reuses it.  For memory admission of a serving layer. */
int ddhdg_trace_solver_bytes(int dim, const int *n, int degree, int ncomp, int64_t *bytes);

/* assemble_system(true, thermo_eq): cell update from the full trace update
 * update_trace [nfaces][3][nf] (include/assembling_methods.template.h:
 * 2122-2160 and 2688-2697).  Uses the reconstruction data kept by the last
 * ddhdg_assemble_condense on the same state. */
int ddhdg_reconstruct(ddhdg_ctx *ctx, const double *cell_state,
                      const double *trace_state, const double *update_trace,
                      double *update_cell, int thermo_eq,
                      ddhdg_stream_t stream);

/* The same two calls for callers whose state lives in host memory, as the
 * reference's NPSolver keeps current_solution_cell / current_solution_trace
 * and update_cell in host vectors (include/np_solver.h:881-887): the host
 * arrays are read and written by the calls themselves, and the copies overlap
 * the kernels.  ddhdg_assemble_condense_host copies the trace state, then the
 * cell state in 4 chunks of cells on an internal copy stream; each chunk is
 * condensed on `stream` as soon as it has arrived.  The context keeps the
 * device copies of the state.  ddhdg_reconstruct_host reconstructs that state
 * for update_trace in the same chunks and copies each chunk of update_cell
 * back on a second copy stream while the next chunk runs; the results are in
 * host memory when `stream` has completed.  Outputs of the condensation (tt,
 * rhs, dflag, dval) are device arrays as in ddhdg_assemble_condense.  The copies
 * overlap only for page-locked host memory (cudaHostAlloc / cudaHostRegister);
 * pageable memory gives the same results with serialised copies.  A context's
 * host-buffer calls must be issued on one stream at a time. */
int ddhdg_assemble_condense_host(ddhdg_ctx *ctx, const double *cell_state_host,
                                 const double *trace_state_host, int thermo_eq, double *tt,
                                 double *rhs, int32_t *dflag, double *dval,
                                 ddhdg_stream_t stream);
int ddhdg_reconstruct_host(ddhdg_ctx *ctx, const double *update_trace_host, int thermo_eq,
                           double *update_cell_host, ddhdg_stream_t stream);

/* private_run (src/np_solver.cpp:1452-1561) on device-resident state:
 * Newton iterations with damping alpha, absolute / relative stop on the
 * infinity norm of the update.  cell_state / trace_state are updated in
 * place.  Returns DDHDG_OK when converged, DDHDG_NOT_CONVERGED otherwise. */
int ddhdg_newton(ddhdg_ctx *ctx, double *cell_state, double *trace_state,
                 int thermo_eq, double abs_tol, double rel_tol, int max_it,
                 double alpha, int *iterations, double *last_update_norm,
                 ddhdg_stream_t stream);

/* Per-stage device times (ms) of the last ddhdg_newton call. */
int ddhdg_last_timings(const ddhdg_ctx *ctx, double *condense_ms,
                       double *solve_ms, double *reconstruct_ms, int *steps);

/* L2 projection of a scalar field given at cell and cell-face quadrature
 * points into component comp of cell_state (scalar and weak-gradient
 * displacement), as project_component (src/project_component.cpp:268-420) and
 * compute_local_charge_neutrality_on_cells (src/thermodynamic_equilibrium.cpp:
 * 47-213).  vals_cell [ncells][nqc], vals_face [ncells][2*dim][nqf]. */
int ddhdg_project_cell(ddhdg_ctx *ctx, const double *vals_cell,
                       const double *vals_face, int comp, double *cell_state,
                       ddhdg_stream_t stream);
/* L2 projection of face-point values [nfaces][nqf] onto the trace of comp. */
int ddhdg_project_trace(ddhdg_ctx *ctx, const double *vals_face, int comp,
                        double *trace_state, ddhdg_stream_t stream);
/* project_component(phi_c, qf) (src/project_component.cpp:575-654) followed
 * by project_cell_function_on_trace(l2_average) (src/copy_on_trace.cpp):
 * density of comp (1: n, 2: p) from the quasi Fermi potential qf and the
 * current V, projected on cells and averaged onto the trace. */
int ddhdg_project_density(ddhdg_ctx *ctx, int comp, double qf,
                          double *cell_state, double *trace_state,
                          ddhdg_stream_t stream);

/* get_solution_on_a_point (src/np_solver.cpp:1637-1700) for npoints points
 * [npoints][3] (mesh units, device): what = 0, 1, 2 gives V (volts), n, p
 * (m^-3) of the cell field; 3, 4 the quasi Fermi potentials phi_n, phi_p
 * (volts, include/solver.h:343-376).  The cell of a point on an interior face
 * is the one above it along each axis; points outside the mesh use the
 * nearest boundary cell.  out [npoints] on the device. */
int ddhdg_sample_points(ddhdg_ctx *ctx, const double *cell_state,
                        int64_t npoints, const double *points, int what,
                        double *out, ddhdg_stream_t stream);

/* Reference coordinates in [0,1]^dim of the quadrature points and support
 * points the kernels use for a (dim, degree) pair, so that callers evaluate
 * coefficient and boundary tables at exactly those points:
 *   qref_c   [nqc][3]          QGauss(k+1) cell points (x fastest)
 *   qref_f   [2*dim][nqf][3]   face points of local face f (axis f/2,
 *                              side f%2; tangential axes (a+1)%d, (a+2)%d)
 *   support  [k+1]             Gauss-Lobatto support points on [0,1]
 * Any output pointer may be NULL. */
int ddhdg_reference_points(int dim, int degree, double *qref_c, double *qref_f,
                           double *support);

/* ---------------------------------------------------------------------
 * Batched launches over many contexts: devices (diodes) of different mesh
 * sizes and degrees, of one dimension, condensed in ONE persistent launch
 * per Newton step, and reconstructed in one more.  The reference runs its
 * per-cell worker over one device's cells at a time (WorkStream,
 * include/assembling_methods.template.h:67-88); a batch hands out tiles
 * (device, range of its cells) from a work list to the CTAs of one grid.
 * Every device's outputs are bitwise those of its own
 * ddhdg_assemble_condense / ddhdg_reconstruct.  FP64 and mixed-precision
 * contexts may share a batch (each keeps its own precision).  The
 * pointers of an item are fixed for the life of the batch (the launches
 * are replayed from CUDA graphs); the batch keeps its own reconstruction
 * data, so ddhdg_batch_reconstruct follows ddhdg_batch_condense. */
typedef struct ddhdg_batch ddhdg_batch;
typedef struct ddhdg_batch_item
{
  ddhdg_ctx    *ctx;
  const double *cell_state, *trace_state; /* device state of this context */
  double       *tt, *rhs;                 /* condensation outputs, as in  */
  int32_t      *dflag;                    /* ddhdg_assemble_condense      */
  double       *dval;
  double       *update_trace; /* reconstruction input (or NULL); written by ddhdg_batch_newton_step */
  double       *update_cell;  /* reconstruction output (or NULL) */
} ddhdg_batch_item;

int ddhdg_batch_create(const ddhdg_batch_item *items, int nitems, int thermo_eq,
                       ddhdg_batch **batch);
int ddhdg_batch_destroy(ddhdg_batch *batch);
int ddhdg_batch_condense(ddhdg_batch *batch, ddhdg_stream_t stream);
int ddhdg_batch_reconstruct(ddhdg_batch *batch, ddhdg_stream_t stream);
/* One Newton step of private_run (src/np_solver.cpp:1470-1555) for every item:
 * the batched condensation, every item's trace solve (ddhdg_solve_condensed,
 * on side streams forked from `stream`, so that they overlap), the trace
 * update expanded into update_trace, the batched reconstruction, and
 * state += alpha[i] (update_cell, update_trace) in place.  norms_host[4 i ..]
 * (host) receives max |update_cell|, max |update_trace|, max |cell_state|,
 * max |trace_state| of item i before its update (the stopping rule of
 * private_run is the caller's); status_host[i] (host, may be NULL) the item's
 * status (DDHDG_SINGULAR_PIVOT, DDHDG_SOLVER_ERROR or 0).  Returns when the
 * step has completed. */
int ddhdg_batch_newton_step(ddhdg_batch *batch, const double *alpha, double *norms_host,
                            int *status_host, ddhdg_stream_t stream);
/* The same step in two halves, for a caller that drives several batches
 * from one host thread: _begin enqueues the step on `stream` and returns at
 * once (alpha is read before it returns); _end, with wait = 0, returns with
 * *done = 0 while the step is still running, and otherwise fills
 * norms_host / status_host as ddhdg_batch_newton_step does and sets
 * *done = 1.  One step per batch may be in flight. */
int ddhdg_batch_newton_step_begin(ddhdg_batch *batch, const double *alpha, ddhdg_stream_t stream);
int ddhdg_batch_newton_step_end(ddhdg_batch *batch, int wait, double *norms_host, int *status_host,
                                int *done);
/* Tile shape: cells per tile for degrees 1, 2, 3 (cells_per_tile[3]) and
 * CTAs per SM.  ddhdg_batch_autotune picks them by timing the batch's own
 * condensation launch (coordinate search, best of `reps` launches per
 * candidate, on `stream`; the outputs are written by every launch) and
 * returns the best time in ms. */
int ddhdg_batch_set_shape(ddhdg_batch *batch, const int *cells_per_tile, int ctas_per_sm);
int ddhdg_batch_get_shape(const ddhdg_batch *batch, int *cells_per_tile, int *ctas_per_sm,
                          int *grid, int *ntiles);
int ddhdg_batch_autotune(ddhdg_batch *batch, int reps, float *best_ms, ddhdg_stream_t stream);

/* Last error message of the calling thread (static storage). */
const char *ddhdg_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* DDHDG_B200_H */
