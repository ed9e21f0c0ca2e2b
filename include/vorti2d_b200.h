/*
 * vorti2d_b200 -- C ABI of the B200-native vorti2d hot path
 * (libvorti2d_b200.so, sm_100a).
 *
 * Every entry point returns an int status (V2D_OK = 0, negative on error) and
 * leaves a message for v2d_last_error().  No torch or C++ types cross this
 * boundary: plain pointers, sizes and POD structs only.
 *
 * Three groups:
 *  1. The kernel seam: drop-ins for the f2py module `vorti2d.core`
 *     (reference src/fortran/vorti2d_core.f90).  Host pointers in and out;
 *     the work runs on the current CUDA device.  `*_dev` variants take device
 *     pointers and a cudaStream_t (passed as void*).
 *  2. The linear-solver seam: drop-in for vorti2d.petsc_solver.MumpsSolver
 *     (reference vorti2d/petsc_solver.py:37-132): COO in, canonical CSR on the
 *     device, GMRES(m) solve, full solution out.
 *  3. The device-resident Newton / BDF2 driver behind vorti2d.Config / run()
 *     (reference vorti2d/solver.py:48-224): metrics, state, CSR, Krylov
 *     workspace and forces all live in HBM behind an opaque handle.
 *
 * Threading: a handle is owned by one host thread at a time; different
 * handles may be used concurrently from different threads.
 */
#ifndef VORTI2D_B200_H
#define VORTI2D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define V2D_OK 0
#define V2D_EARG (-1)          /* bad argument (shape, range, null pointer) */
#define V2D_ECAPACITY (-2)     /* caller buffer too small (e.g. maxnnz)      */
#define V2D_ECUDA (-3)         /* CUDA runtime error                         */
#define V2D_ENONFINITE (-4)    /* NaN/Inf detected in a result               */
#define V2D_ENOTCONVERGED (-5) /* Krylov solve hit max iterations            */
#define V2D_ETIMEOUT (-6)      /* a bounded device wait ran out              */
#define V2D_EBREAKDOWN (-7)    /* singular 2x2 block / Krylov breakdown      */
#define V2D_ENOMEM (-8)        /* device allocation failed                   */

const char *v2d_last_error(void);
int v2d_version(void);
/* Number of kernels launched by this library so far (CUDA-graph replays
 * count their kernel nodes).  Measurement aid; no reference counterpart. */
long long v2d_launch_count(void);

/* ------------------------------------------------- 1. kernel seam (_core) */

/* Replaces vorti2d_core.node_neighbors (vorti2d_core.f90:33-61).
 * 1-based (i, j) -> out[9] = k, e, w, n, s, ne, nw, se, sw (1-based). */
int v2d_node_neighbors(int i, int j, int imax, int *out9);

/* Replaces vorti2d_core.compute_metrics (vorti2d_core.f90:66-189; called at
 * vorti2d/solver.py:72-74).  xg, yg: Fortran-ordered (imax, jmax) doubles, i.e.
 * element (i, j) at [(i-1) + imax*(j-1)].  Each output has imax*jmax doubles in
 * pointer order k = imax*(j-1)+i.  Outputs in f2py tuple order: jac, alfa,
 * beta, gama, pmet, qmet, detadx, detady, xphys, yphys. */
int v2d_compute_metrics(int imax, int jmax, double dksi, double deta,
                        const double *xg, const double *yg,
                        double *jac, double *alfa, double *beta, double *gama,
                        double *pmet, double *qmet, double *detadx, double *detady,
                        double *xphys, double *yphys);

/* Replaces vorti2d_core.compute_metrics_local (vorti2d_core.f90:392-495;
 * called at vorti2d/dist_solver.py:92-93).  Ghosted local block gxm x jmax
 * (Fortran order), owned 1-based columns [il0, il1]; outputs gxm*jmax, zero
 * outside the owned columns except xphys/yphys. */
int v2d_compute_metrics_local(int gxm, int jmax, int il0, int il1, double dksi,
                              double deta, const double *xgl, const double *ygl,
                              double *jac, double *alfa, double *beta, double *gama,
                              double *pmet, double *qmet, double *detadx,
                              double *detady, double *xphys, double *yphys);

/* Replaces vorti2d_core.assemble_coo (vorti2d_core.f90:219-383; called at
 * vorti2d/solver.py:121-127).  Rows [r0, r1) of the field-blocked 2N system
 * (psi rows [0,N), ome rows [N,2N)).  COO triplets are written in the
 * reference's push order (0-based); *nnz receives the count; bvec has r1-r0
 * entries.  Unlike the reference (whose push has no bound check), a maxnnz
 * that is too small returns V2D_ECAPACITY and writes no triplet. */
int v2d_assemble_coo(int imax, int jmax, double re, double invdtau, double inv2dt,
                     double urot, double dksi, double deta, const double *jac,
                     const double *alfa, const double *beta, const double *gama,
                     const double *pmet, const double *qmet, const double *detadx,
                     const double *detady, const double *xphys, const double *yphys,
                     const double *psi, const double *ome, const double *omeold,
                     const double *omeoldold, int r0, int r1, int maxnnz, int ff_bc,
                     double ca, double sa, int *coo_i, int *coo_j, double *coo_v,
                     int *nnz, double *bvec);

/* Replaces vorti2d_core.assemble_coo_local (vorti2d_core.f90:510-661; called
 * at vorti2d/dist_solver.py:310-317).  Local ghosted arrays of gxm*jmax
 * doubles, lg[2*gxm*jmax] the 0-based global dof of (local node, component).
 * Owned rows are [r0, r0+nloc); bvec has nloc entries. */
int v2d_assemble_coo_local(int gxm, int jmax, int il0, int il1, double re,
                           double invdtau, double inv2dt, double urot, double dksi,
                           double deta, const double *jac, const double *alfa,
                           const double *beta, const double *gama, const double *pmet,
                           const double *qmet, const double *detadx, const double *detady,
                           const double *xphys, const double *yphys, const double *psi,
                           const double *ome, const double *omeold,
                           const double *omeoldold, int r0, int nloc, const int *lg,
                           int maxnnz, int ff_bc, double ca, double sa, int *coo_i,
                           int *coo_j, double *coo_v, int *nnz, double *bvec);

/* Allocation-free variant of v2d_assemble_coo.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory where
 * they assemble -- a framework that owns the GPU's memory through its own pool
 * and budget, or a time-critical loop that must avoid cudaMalloc/cudaFree,
 * which can synchronize the device and can fail under memory pressure.
 * Same rows, COO push order and right-hand side as v2d_assemble_coo, but every
 * array is a DEVICE pointer: d_fields14 is a host array of the 14 device input
 * fields in v2d_assemble_coo's order (jac ... omeoldold, imax*jmax doubles
 * each); d_coo_i/j/v have room for maxnnz entries, d_bvec for r1-r0; *nnz is
 * a host int.  The call allocates nothing: its only scratch (row offsets and
 * scan sums) is a fixed 4 MiB array in the library's device memory, which
 * every GPU that loads the library holds until the process exits.  It limits
 * a call to r1 - r0 <= 1048576 rows (larger ranges return V2D_EARG: assemble
 * them in pieces).  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress) with the device current; make that first call before
 * any stream capture.  All calls share the array, so calls whose work
 * overlaps on the GPU (concurrent streams or host threads on one device) race
 * and must be serialized by the caller.  The call
 * synchronizes `stream` (a cudaStream_t, may be 0) to read the entry count. */
int v2d_assemble_coo_noalloc(int imax, int jmax, double re, double invdtau, double inv2dt,
                             double urot, double dksi, double deta,
                             const double *const *d_fields14, int r0, int r1, int maxnnz,
                             int ff_bc, double ca, double sa, int *d_coo_i, int *d_coo_j,
                             double *d_coo_v, int *nnz, double *d_bvec, void *stream);

/* Device-pointer form of v2d_compute_metrics (same layouts; stream may be 0). */
int v2d_compute_metrics_dev(int imax, int jmax, double dksi, double deta,
                            const double *d_xg, const double *d_yg, double *const *d_out10,
                            void *stream);

/* Replaces vorti2d.forces.compute_force_coeffs (vorti2d/forces.py:82-194),
 * computed on the device from host arrays of imax*jmax doubles.
 * ref_length <= 0 selects the automatic body-diameter estimate.
 * out10 = cd, cl, cm, cdp, cdf, clp, clf, cmp, cmf, ref_length. */
int v2d_force_coeffs(int imax, int jmax, double re, double dksi, double deta,
                     const double *beta, const double *gama, const double *detadx,
                     const double *detady, const double *xphys, const double *yphys,
                     const double *ome, double ref_length, double x0, double y0,
                     double *out10);

/* Replaces vorti2d.velocity.compute_velocity (vorti2d/velocity.py:76-93):
 * Cartesian velocity from the streamfunction, computed on the device from host
 * arrays of imax*jmax doubles (pointer order).  vmag may be null. */
int v2d_compute_velocity(int imax, int jmax, double dksi, double deta, const double *jac,
                         const double *beta, const double *gama, const double *detadx,
                         const double *detady, const double *psi, double *u, double *v,
                         double *vmag);

/* ------------------------------------------------ Krylov solver parameters */
#define V2D_PC_NONE 0
#define V2D_PC_BJACOBI 1   /* 2x2 (psi, ome) node blocks                     */
#define V2D_PC_LU 2        /* multifrontal LU of the current Jacobian (nested
                              dissection of the O-grid); solver API only     */

#define V2D_PREC_FP64 0    /* FP64 Krylov                                     */
#define V2D_PREC_MIXED 1   /* FP32 SpMV/PC/Krylov vectors, FP64 Gram-Schmidt
                              sums, FP64 outer defect correction              */

typedef struct {
    int restart;          /* GMRES(m) restart length                  (30)   */
    int max_it;           /* max Krylov iterations per solve          (5000) */
    double rtol;          /* relative residual tolerance (1e-10); a solve whose
                             FP64 residual stops halving per restart cycle
                             within 100x of the target has reached the
                             attainable accuracy: it ends there and counts
                             as converged                                    */
    double atol;          /* absolute residual tolerance              (1e-50)*/
    int precond;          /* V2D_PC_*                                         */
    int precision;        /* V2D_PREC_*                                       */
    double inner_rtol;    /* mixed: FP32 GMRES tolerance per correction (1e-5)*/
    int dc_max_it;        /* mixed: max defect-correction passes       (20)  */
    int lu_leaf;          /* LU: max nodes of a leaf subdomain         (64)  */
    int lu_reuse_its;     /* LU: 0 factors every Newton Jacobian (default);
                             k > 0 keeps the factors across the Newton
                             iterations of one time step (the BDF2 history
                             shift refreshes them) while the last solve with
                             them took at most k Krylov iterations; a solve
                             with kept factors that needs more than k+5
                             iterations refactors and solves again.  Newton
                             steps are still solved to rtol.                */
    int lu_reuse_steps;   /* LU, with lu_reuse_its > 0: 1 keeps the factors
                             across the BDF2 history shift and
                             v2d_solver_set_state too, under the same
                             iteration rule; 0 refreshes them at the first
                             Newton iteration of every time step and after
                             every set_state (0)                            */
    int lu_solve;         /* LU: 0 the preconditioner solve is one dataflow
                             launch over the whole front tree (default);
                             1 one launch per tree level and sweep          */
    int lu_factor64;      /* LU in the mixed form: 0 factors in FP32 (0);
                             1 factors in FP64 and rounds them to FP32 for
                             the FP32 solve (better pivots, same solve bytes)*/
} v2d_krylov_params;

void v2d_krylov_defaults(v2d_krylov_params *p);

typedef struct {
    int iterations;       /* Krylov iterations (all restarts / corrections) */
    int restarts;
    int corrections;      /* mixed: outer defect-correction passes          */
    int converged;        /* 1 if the tolerance was met                     */
    double res0;          /* ||b||                                          */
    double res;           /* final true residual ||b - A x|| (FP64)         */
} v2d_lin_stats;

/* ----------------------------------------- 2. linear-solver seam (MumpsSolver) */
typedef struct v2d_linsys v2d_linsys;

/* Replaces MumpsSolver(n) (vorti2d/petsc_solver.py:38-70).  block_layout:
 * 0 point diagonal, 1 field-blocked 2x2 pairs (r, r+n/2), 2 interleaved
 * 2x2 pairs (2q, 2q+1).  With p->precond = V2D_PC_LU (block_layout 1 only)
 * every solve factors the assembled matrix (multifrontal LU, nested
 * dissection of the O-grid) and refines with GMRES to rtol, like the
 * reference's MUMPS direct solve (petsc_solver.py:55-61); lu_reuse_its > 0
 * keeps factors across solves under the rule of v2d_krylov_params. */
int v2d_linsys_create(int n, int block_layout, const v2d_krylov_params *p,
                      v2d_linsys **out);
/* The O-grid shape (n = 2 imax jmax) for the LU preconditioner; call before
 * the first assemble.  Without it the shape is recognised from the pattern at
 * the first assemble.  No reference counterpart (MUMPS orders the matrix
 * itself). */
int v2d_linsys_set_grid(v2d_linsys *s, int imax, int jmax);
/* Replaces MumpsSolver.assemble (vorti2d/petsc_solver.py:76-95): the first
 * call fixes the canonical CSR pattern (rows sorted, columns sorted,
 * duplicates summed); later calls must repeat the same (i, j) sequence and
 * only refresh the values. */
int v2d_linsys_assemble(v2d_linsys *s, const int *coo_i, const int *coo_j,
                        const double *coo_v, long long nnz, const double *b);
/* Replaces MumpsSolver.solve (vorti2d/petsc_solver.py:97-115). */
int v2d_linsys_solve(v2d_linsys *s, double *x, v2d_lin_stats *st);
/* Canonical CSR export (for parity checks): sizes n+1, nnz, nnz. */
int v2d_linsys_nnz(const v2d_linsys *s, long long *nnz);
int v2d_linsys_csr(const v2d_linsys *s, int *indptr, int *indices, double *data);
int v2d_linsys_destroy(v2d_linsys *s);

/* -------------------------------------------- 3. device-resident driver */
typedef struct v2d_solver v2d_solver;

typedef struct {
    double re;            /* Reynolds number (vorti2d/config.py:15)          */
    double invdtau;       /* 1/dtau, 0 for pure Newton (config.py:139-140)   */
    double inv2dt;        /* 1/(2 dt), 0 when steady (config.py:142-144)     */
    double ca, sa;        /* cos/sin of the angle of attack (config.py:146-150) */
    int ff_bc;            /* 0 dirichlet, 1 outflow, 2 outflow_psi           */
    v2d_krylov_params krylov;
} v2d_solver_params;

typedef struct {
    int newton_iters;
    int krylov_iters;     /* summed over the Newton iterations             */
    int corrections;
    double res;           /* reference measure ||dq||_2 / (2N)              */
    double lin_res_max;   /* worst relative linear residual of the solves  */
} v2d_newton_info;

/* Uploads the mesh (Fortran-ordered (imax, jmax) like v2d_compute_metrics),
 * evaluates the metrics on the device, builds the canonical CSR pattern and
 * initialises the state as vorti2d/solver.py:103-114 does. */
int v2d_solver_create(int imax, int jmax, const double *xg, const double *yg,
                      const v2d_solver_params *p, v2d_solver **out);
int v2d_solver_destroy(v2d_solver *s);
int v2d_solver_set_params(v2d_solver *s, const v2d_solver_params *p);
/* State transfer (host pointers, N = imax*jmax doubles each, pointer order). */
int v2d_solver_set_state(v2d_solver *s, const double *psi, const double *ome,
                         const double *omeold, const double *omeoldold);
int v2d_solver_get_state(v2d_solver *s, double *psi, double *ome, double *omeold,
                         double *omeoldold);
/* The 10 metric arrays in f2py order (host pointers, N doubles each). */
int v2d_solver_get_metrics(v2d_solver *s, double *const *out10);
/* One Newton iteration (vorti2d/solver.py:117-134): assemble on the device,
 * GMRES solve, q += dq; *res = ||dq||_2 / (2N). */
int v2d_solver_newton(v2d_solver *s, double urot, double *res, v2d_lin_stats *st);
/* Inner loop (vorti2d/solver.py:136-145): iterate while res > pseudo_tol and
 * it < max_iter. */
int v2d_solver_pseudo_solve(v2d_solver *s, double urot, double pseudo_tol, int max_iter,
                            v2d_newton_info *info);
/* BDF2 history shift omeoldold <- omeold <- ome (vorti2d/solver.py:186-188). */
int v2d_solver_shift_history(v2d_solver *s);
/* One physical step = pseudo_solve + (unsteady) history shift. */
int v2d_solver_step(v2d_solver *s, double urot, double pseudo_tol, int max_iter,
                    int unsteady, v2d_newton_info *info);
/* Force coefficients (vorti2d/forces.py:82-194) of the current state on the
 * device.  ref_length <= 0 selects the automatic body-diameter estimate.
 * out10 = cd, cl, cm, cdp, cdf, clp, clf, cmp, cmf, ref_length. */
int v2d_solver_forces(v2d_solver *s, double re, double ref_length, double x0, double y0,
                      double *out10);
/* Velocity of the current state (vorti2d/velocity.py:76-93) into host arrays
 * of N doubles; vmag may be null. */
int v2d_solver_velocity(v2d_solver *s, double *u, double *v, double *vmag);
/* Discrete adjoint (no reference counterpart; the reference has no adjoint):
 * J^T lambda = g for the Jacobian J = dR/dq of the current state (rotation
 * urot), R = -b the residual of the field-blocked 2N system.  FP64 multifrontal
 * factors of J are computed (kept while the state and J are unchanged), and
 * GMRES(30) in FP64 on J^T, preconditioned by the transposed multifrontal
 * solve, runs until ||g - J^T lambda|| <= rtol ||g|| or 30 * max_refine
 * iterations (a residual that stagnates below 1e-8 is accepted as the
 * attainable accuracy).  *refinements receives the GMRES iterations and
 * *rel_res the final relative residual.
 * g and lambda: host arrays of 2N doubles. */
int v2d_solver_adjoint(v2d_solver *s, double urot, const double *g, double *lambda, double rtol,
                       int max_refine, int *refinements, double *rel_res);
/* b = -R of the current state for the given scalar parameters (same far-field
 * BC and pattern as the handle), into a host array of 2N doubles: the
 * parameter derivatives of the residual for the adjoint. */
int v2d_solver_residual(v2d_solver *s, double re, double invdtau, double inv2dt, double urot,
                        double ca, double sa, double *b);
/* The same right-hand side b = -R at the handle's state, but with the metrics
 * of another mesh of the same shape (xg, yg: host, N doubles each, in the
 * handle's pointer order): the mesh derivative of the residual for shape
 * gradients (vorti2d_core.f90:66-189 then :219-381 on the given coordinates).
 * The handle is not changed.  When met_rows > 0, met receives rows
 * j < met_rows of the 10 metric arrays (10 blocks of imax*met_rows doubles, in
 * the order of v2d_solver_get_metrics), enough for the wall force integrals
 * with met_rows = 3. */
int v2d_solver_residual_mesh(v2d_solver *s, const double *xg, const double *yg, double re,
                             double invdtau, double inv2dt, double urot, double ca, double sa,
                             double *b, int met_rows, double *met);
/* Mesh sensitivities for shape gradients (no reference counterpart), on the
 * device: for each of the P = imax-1 wall nodes i and s = +1, -1, the
 * handle's mesh with grid line i (and the seam line with i = 0) moved by
 * s h (nx[i], ny[i]) phi[., i] (phi: N doubles, pointer order), its metrics,
 * the right-hand side b_s = -R at the handle's state and the wall force
 * coefficients (the 10 values of v2d_force_coeffs, ref_length <= 0: from the
 * wall).  dots[i] = lambda . (b_+ - b_-); forces[(2 i + (s < 0)) * 10 + c].
 * Host arrays: nx, ny (P), phi (N), lambda (2N), dots (P), forces (20 P). */
int v2d_solver_shape_gradient(v2d_solver *s, const double *nx, const double *ny,
                              const double *phi, const double *lambda, double h, double re,
                              double invdtau, double inv2dt, double urot, double ca, double sa,
                              double ref_length, double x0, double y0, double *dots,
                              double *forces);
/* Exact mesh sensitivities for shape gradients (no reference counterpart):
 * the same directions as v2d_solver_shape_gradient (grid line i, and the seam
 * line with i = 0, moved by (nx[i], ny[i]) phi[.]), differentiated by
 * forward-mode (tangent) derivatives through the metric computation
 * (vorti2d_core.f90:66-189), the residual rows (:219-381) and the wall force
 * integrals (vorti2d/forces.py:82-194) on the device -- no step size, no
 * displaced meshes.  dots[i] = lambda . db/dd_i (b = -R at the handle's state
 * with the given scalar parameters), dforces[10 i + c] = d(force value c)/dd_i
 * in the order of v2d_force_coeffs (ref_length <= 0: from the wall).
 * Host arrays: nx, ny (P = imax-1), phi (N), lambda (2N), dots (P),
 * dforces (10 P). */
int v2d_solver_shape_tangent(v2d_solver *s, const double *nx, const double *ny,
                             const double *phi, const double *lambda, double re, double invdtau,
                             double inv2dt, double urot, double ca, double sa, double ref_length,
                             double x0, double y0, double *dots, double *dforces);
/* Current system (after the last assembly): canonical CSR of the 2N system
 * and its right-hand side.  Sizes: 2N+1, nnz, nnz, 2N. */
int v2d_solver_nnz(const v2d_solver *s, long long *nnz);
int v2d_solver_assemble(v2d_solver *s, double urot);
int v2d_solver_export_system(v2d_solver *s, int *indptr, int *indices, double *data,
                             double *b);
/* Device pointers of the state (psi, ome, omeold, omeoldold) for zero-copy
 * interop (e.g. torch tensors via __cuda_array_interface__). */
int v2d_solver_state_ptrs(v2d_solver *s, double **psi, double **ome, double **omeold,
                          double **omeoldold);
/* Measurement aid (no reference counterpart): average duration in ms of
 * `reps` launches of the Krylov SpMV kernel on the current system (FP32
 * values if fp32 != 0), each preceded by a write of flush_bytes to evict L2;
 * CUDA events on the handle's stream. */
int v2d_solver_time_spmv(v2d_solver *s, int fp32, int reps, long long flush_bytes,
                         double *ms_avg);
/* Planning aid (no reference counterpart): host-only symbolic analysis of the
 * multifrontal LU preconditioner (V2D_PC_LU) for the canonical CSR pattern of
 * an imax x jmax O-grid system (indptr: 2*imax*jmax+1, indices: nnz).  No
 * device work.  out8 = fronts, levels, largest separator, largest front,
 * factor entries, factorization flop bound, front variables, contribution
 * entries. */
int v2d_lu_plan_info(int imax, int jmax, const int *indptr, const int *indices, int leaf,
                     long long *out8);
/* Planning aid for the preconditioner solve's work items (host only; no
 * reference counterpart): info4 = {work items, dependency counters, fronts,
 * levels}; when cap_items >= items, items gets 12 ints per item (kind 0
 * forward rows / 1 backward rows / 2 forward gather / 3 backward gather,
 * front, first row, end row, wait counter and target, second wait counter and
 * target, two done counters, tree level, 1 for the items of a front with
 * gather items else 0; -1 for none); when cap_fronts >= fronts, fronts3 gets each front's pivots S, size f and
 * parent (-1 at the root).  Items run in this order in the one-launch
 * dataflow solve; the plan checks that every wait is met by earlier items. */
int v2d_lu_solve_plan(int imax, int jmax, const int *indptr, const int *indices, int leaf,
                      int *info4, int *items, int cap_items, int *fronts3, int cap_fronts);

/* Planning aid (no reference counterpart): v2d_lu_solve_plan with an explicit
 * work-item split, rows[L] per tree level L (nrows = levels): 0 whole fronts,
 * R > 0 items of R rows, R < 0 items of -R rows after one gather item per
 * front split into several (kinds 2 forward and 3 backward in the table).
 * rows null: the default split. */
int v2d_lu_solve_plan_split(int imax, int jmax, const int *indptr, const int *indices, int leaf,
                            const int *rows, int nrows, int *info4, int *items, int cap_items,
                            int *fronts3, int cap_fronts);

/* Measurement aid (no reference counterpart): device time in ms, summed over
 * the Newton iterations since the last reset, of the four phases of a Newton
 * iteration (CUDA events on the handle's stream): out6 = assembly,
 * factorization (LU preconditioner), Krylov solve, update, iteration count,
 * LU factorizations performed. */
int v2d_solver_phase_times(v2d_solver *s, double *out6, int reset);

/* Measurement aid (no reference counterpart): average duration in ms of
 * `reps` applications of the current LU factors (the preconditioner solve of
 * one GMRES iteration), each preceded by a write of flush_bytes to evict L2;
 * *factor_bytes receives the bytes of factor entries one application reads
 * (per front the pivot-block inverses and the blocks G = L21 L11^-1 and
 * H = U11^-1 U12, which hold as many entries as L21 and U12). */
int v2d_solver_time_lu_apply(v2d_solver *s, int reps, long long flush_bytes, double *ms_avg,
                             long long *factor_bytes);

/* Measurement aid (no reference counterpart): sizes of the handle's LU
 * preconditioner -- out6 = fronts, tree levels, factor entries (sum f^2),
 * flops of one factorization (per front: the partial LU
 * 2 sum_{k<S} (f-k-1)^2, the pivot-block inverses 2 S^3 / 3, and
 * G = L21 L11^-1, H = U11^-1 U12 2 (f-S) S^2), factor entries one solve reads
 * (sum S (2f - S)), work items of the dataflow solve. */
int v2d_solver_lu_stats(v2d_solver *s, double *out6);

/* Measurement aid (no reference counterpart): one dataflow LU solve of the
 * current factors with a trace of every work item -- global-timer ns at its
 * ticket, at the end of its dependency wait and after its done counters
 * (ticks[3 i + k]) -- and the item table (items: 12 ints per item as in
 * v2d_lu_solve_plan, may be null); cap >= items, *n = items. */
int v2d_solver_trace_lu_apply(v2d_solver *s, unsigned long long *ticks, int *items, int cap,
                              int *n);

/* Tuning aid (no reference counterpart): the form of the dataflow LU solve
 * kernel -- 0: two resident CTAs per SM with 32 row registers per lane (16 in
 * FP64); 1: three CTAs per SM with 16 (8 in FP64).  form < 0 only reads the
 * current one into *current (may be null). */
int v2d_solver_lu_flow_form(v2d_solver *s, int form, int *current);

/* Tuning aid (no reference counterpart): the split form of the dataflow LU
 * solve -- level > 0 runs the tree levels [0, level) as launches of their own
 * (their forward items before, their backward items after the upper levels'
 * launch), with 128-thread CTAs and shared memory for their own largest
 * front, so that more of their many small work items are in flight per SM;
 * 0: one launch for the whole tree.  level < 0 only reads the current
 * setting into *current (may be null).  Every setting forms the same
 * products. */
int v2d_solver_lu_split(v2d_solver *s, int level, int *current);

/* Tuning aid (no reference counterpart): the work-item granularity of the
 * LU preconditioner solve, rows[L] rows of a front per work item on tree
 * level L (0: whole fronts); rows may be null to only read the current
 * setting into out_rows (cap >= levels) and *nlevels_out.  Every setting
 * forms the same products; only how the rows are split over CTAs (and the
 * order of a row's partial sums) changes. */
int v2d_solver_lu_item_rows(v2d_solver *s, const int *rows, int nlevels, int *out_rows, int cap,
                            int *nlevels_out);

/* Measurement aid (no reference counterpart): the device time of each
 * launch of one LU preconditioner solve, averaged over `reps` solves (each
 * after a write of flush_bytes; 0 keeps the factors warm in L2).  ms[k] and
 * codes[k] (kind * 1000 + level; kinds 0 forward level, 1 backward level,
 * 2 the one-launch dataflow solve) for k < *n <= cap. */
int v2d_solver_time_lu_launches(v2d_solver *s, int reps, long long flush_bytes, double *ms,
                                int *codes, int cap, int *n);
/* Measurement aid (no reference counterpart): the device time of each kernel
 * of one LU factorization of the last assembled Jacobian, launched directly,
 * averaged over `reps` (codes kind * 1000 + level; kinds 0 row scaling,
 * 1 scatter, 2 extend-add, 3 first panel, 4 L21 + row swaps + U12, 6 Schur
 * update + next panel, 7 pivot-block inversion, 8 inverse copy, 9 products
 * G = L21 L11^-1 and H = U11^-1 U12, 10 their copy). */
int v2d_solver_time_lu_factor(v2d_solver *s, int reps, double *ms, int *codes, int cap, int *n);

/* Measurement aid (no reference counterpart): average ms of `reps` launches
 * of one kernel on the handle's data, each after a write of flush_bytes:
 * which = 0 metrics, 1 Newton assembly (FP64 values), 2 Newton assembly with
 * the FP32 copy, 3 velocity reconstruction. */
int v2d_solver_time_kernel(v2d_solver *s, int which, int reps, long long flush_bytes,
                           double *ms_avg);

/* The stream the handle's kernels run on (cudaStream_t as void*). */
int v2d_solver_stream(v2d_solver *s, void **stream);

/* ------------------------------------------------ 4. batched steady solves */
/* Many steady Newton solves of uneven O-grids at once (no reference
 * counterpart: the reference runs one solve per process,
 * vorti2d/solver.py:136-145).  The instances' Newton systems are the diagonal
 * blocks of one block-diagonal system: each Newton iteration is one
 * assembly launch over all instances, one multifrontal factorization over
 * the forest of their separator trees, GMRES on the combined system and one
 * update launch.  params[i] holds instance i's Reynolds number, angle,
 * far-field BC and pseudo-time term; the Krylov parameters are params[0]'s
 * (precond must be V2D_PC_LU). */
typedef struct v2d_batch v2d_batch;
int v2d_batch_create(int ninst, const int *imax, const int *jmax, const double *const *xg,
                     const double *const *yg, const v2d_solver_params *params,
                     v2d_batch **out);
int v2d_batch_destroy(v2d_batch *b);
/* active[i] = 0 freezes instance i (its rows become identity rows with a zero
 * right-hand side: its state stays as it is); 1 iterates it (all start
 * active). */
int v2d_batch_set_active(v2d_batch *b, const int *active);
/* One Newton iteration of every active instance; res[i] = ||dq_i||_2 / (2 N_i)
 * (0 for a frozen one), flags[i] (may be null) the instance's assembly flags
 * (bit 1 non-finite right-hand side: no update is made then, V2D_ENONFINITE).
 * V2D_ENOTCONVERGED after the update when GMRES missed its tolerance. */
int v2d_batch_newton(v2d_batch *b, double *res, int *flags, v2d_lin_stats *st);
/* The solver handle of instance i (state, forces, metrics); owned by the
 * batch. */
int v2d_batch_instance(v2d_batch *b, int i, v2d_solver **out);
/* LU factorizations of the combined system so far. */
int v2d_batch_factorizations(const v2d_batch *b, long long *n);

#ifdef __cplusplus
}
#endif
#endif /* VORTI2D_B200_H */
