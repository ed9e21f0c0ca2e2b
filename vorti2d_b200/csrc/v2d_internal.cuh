// Internal interfaces between the translation units of libvorti2d_b200.
#pragma once

#include <vector>

#include "v2d_stencil.cuh"
#include "v2d_util.cuh"

namespace v2d {

// One replicated O-grid in HBM.  Every array is SoA in pointer order
// K = imax*j + i (i fastest); the Newton system is the field-blocked 2N
// system of the reference (psi rows [0,N), ome rows [N,2N)) in canonical CSR.
struct GridDev {
    int imax = 0, jmax = 0, N = 0, n = 0;
    double dksi = 0, deta = 0;
    double *x = nullptr, *y = nullptr;   // mesh, pointer order
    double *met[10] = {};                // jac alfa beta gama pmet qmet detadx detady xphys yphys
    double *psi = nullptr, *ome = nullptr, *omeold = nullptr, *omeoldold = nullptr;
    int *rowptr = nullptr, *colind = nullptr;
    long long nnz = 0;
    double *val = nullptr;               // FP64 values, canonical CSR order
    float *val32 = nullptr;              // FP32 copy (mixed precision)
    double *b = nullptr;                 // right-hand side
    double *dinv = nullptr;              // 2x2 block inverses, 4 x N (i00 i01 i10 i11)
    float *dinv32 = nullptr;
};

struct AsmParams {
    double re, invdtau, inv2dt, urot, ca, sa;
    int ff_bc;
};

// v2d_assemble.cu
int build_pattern(GridDev &g, const AsmParams &p, cudaStream_t s);  // rowptr/colind/nnz
int launch_metrics(GridDev &g, cudaStream_t s);
int launch_assemble(GridDev &g, const AsmParams &p, bool want32, int *d_flag, cudaStream_t s);
// b = -R at the handle's state for the given scalar parameters (no CSR writes).
int launch_residual(const GridDev &g, const AsmParams &p, double *d_b, cudaStream_t s);

// One instance of a batched assembly (v2d_batch.cu): its grid, scalars and
// fields, its own CSR pattern, and where its rows and entries sit in the
// combined block-diagonal system.
struct BatchInst {
    GlobalTopo T;
    Coeffs c;
    Fields f;
    const int *rowptr, *colind;
    long long nnz_off;
    int row_off;
};
// nodes per assembly block (one thread per node)
constexpr int kAsmNodesHost = 128;
// All instances' Newton systems in one launch of nblocks = sum ceil(N_i /
// kAsmNodesHost) blocks; d_blk0 (ninst + 1) holds each instance's first block.
int launch_assemble_batch(const BatchInst *d_inst, int ninst, const int *d_blk0, int nblocks,
                          const int *d_active, bool want32, double *val, float *val32, double *b,
                          int *d_flags, cudaStream_t s);

// v2d_velocity.cu (vorti2d/velocity.py:76-93); vmag may be null
int launch_velocity(int imax, int jmax, double dksi, double deta, const double *jac,
                    const double *beta, const double *gama, const double *detadx,
                    const double *detady, const double *psi, double *u, double *v, double *vmag,
                    cudaStream_t s);

// v2d_shape.cu: tangent derivatives along the P wall-normal displacement
// directions (grid line i moved by (nx[i], ny[i]) * phi): dots[i] =
// lambda . db/dd_i and dforces[10 i + c] = d(force value c)/dd_i.  phi, nx, ny,
// lam, dots, dforces are device arrays.
int launch_shape_tangent(const GridDev &g, const AsmParams &p, const double *phi,
                         const double *nx, const double *ny, const double *lam, double ref_length,
                         double x0, double y0, double *dots, double *dforces, cudaStream_t s);

// v2d_forces.cu
int launch_forces(const GridDev &g, double re, double ref_length, double x0, double y0,
                  double *d_out10, cudaStream_t s);

// ---------------------------------------------- multifrontal direct LU
// Symbolic plan of the nested-dissection multifrontal factorization of the
// field-blocked 2N system of one O-grid (v2d_mf.cu).  Fronts are numbered
// level by level; front q holds f[q] local variables (its S[q] fully summed
// ones first), stored densely (row-major f x f) at foff[q].
struct MfPlan {
    int N = 0, n = 0, nfront = 0, nlevel = 0, maxS = 0, maxf = 0;
    long long ftotal = 0, nasm = 0;
    int vtotal = 0, utotal = 0;
    double flops = 0.0;   // 2 * sum S f^2 (upper bound of the factorization flops)
    double factor_flops = 0.0;     // the factorization's flops, front_flops summed
    long long apply_entries = 0;   // factor entries one solve reads: sum S (2f - S)
    std::vector<int> S, f, voff, uoff, child0, child1, parent;
    std::vector<long long> foff;
    std::vector<long long> toff;   // offset of the front's S x S block in the level's scratch
    long long tmax = 0;            // largest sum of S^2 over the fronts of one level
    std::vector<long long> goff;   // offset of the front's G and H in the level's scratch
    long long gmax = 0;            // largest sum of 2 m S over the fronts of one level
    std::vector<int> lvl_off, lvl_maxS, lvl_maxf, lvl_maxm, lvl_maxm_child;
    std::vector<long long> lvl_fbeg, lvl_fend, lvl_abeg, lvl_aend;
    int *d_S = nullptr, *d_f = nullptr, *d_voff = nullptr, *d_uoff = nullptr;
    int *d_child0 = nullptr, *d_child1 = nullptr, *d_parent = nullptr;
    long long *d_foff = nullptr, *d_toff = nullptr, *d_goff = nullptr;
    int *d_vars = nullptr, *d_cbmap = nullptr, *d_asm_csr = nullptr, *d_asm_row = nullptr;
    long long *d_asm_pos = nullptr;
    // work items of the solve (12 ints each: kind, front, rows [beg, end),
    // two (counter, target) waits, two done counters), forward items level by
    // level bottom-up, then backward items top-down; the items of level L's
    // forward sweep are [lvl_fwd[L], lvl_fwd[L + 1]), of its backward sweep
    // [lvl_bwd[L], lvl_bwd[L + 1]) (lvl_bwd descends with L).  The order is
    // checked when the plan is built (see items_build).
    int nitems = 0, nctr = 0;
    std::vector<int> h_items, lvl_fwd, lvl_bwd;
    std::vector<int> item_rows;    // rows per item of each level (0: whole fronts; R < 0:
                                   // -R rows per item after one gather item per front)
    std::vector<int> lvl_fwd_g, lvl_bwd_g;   // gather items at the start of each level's
                                             // forward / backward range
    int *d_items = nullptr;
    long long items_ver = 0;       // bumped whenever d_items is replaced
    // host copies, kept only between the build and the upload
    std::vector<int> h_vars, h_cbmap, h_asm_csr, h_asm_row;
    std::vector<long long> h_asm_pos;
};

// Flops of one front's factorization into the solve's form (S pivots of f
// variables, m = f - S): the partial LU, 2 sum_{k<S} (f - k - 1)^2; the two
// inverses of the pivot block, 2 S^3 / 3; G = L21 L11^-1 and H = U11^-1 U12,
// 2 m S^2 (multiply and add each counted).
inline double front_flops(int S, int f)
{
    auto sq = [](double n) { return n * (n + 1.0) * (2.0 * n + 1.0) / 6.0; };   // sum_{j<=n} j^2
    const double m = f - S;
    return 2.0 * (sq(f - 1.0) - sq(m - 1.0)) + 2.0 * S * (double)S * S / 3.0 + 2.0 * m * S * S;
}

// Error state of the dataflow solve: err is set when a dependency wait ran
// out (read and reset by mf_check_barrier).
struct MfBarrier {
    unsigned int count, gen;
    int err, pad;
};

// Numeric factors of one plan in one precision.
struct MfFactor {
    int fp32 = 0;               // precision of the solve (Krylov vectors, applied factors)
    int fact64 = 0;             // with fp32: the factorization runs in FP64 and the factors
                                // are rounded to FP32 for the solve (F32)
    void *F = nullptr, *upd = nullptr, *z = nullptr;
    void *F32 = nullptr;        // fact64: FP32 copy of F that the solve reads
    void *tmp = nullptr;        // triangular inverses of one level before they replace L11 / U11
    void *gh = nullptr;         // G = L21 L11^-1 and H = U11^-1 U12 of one level before they
                                // replace L21 / U12
    void *inv_g = nullptr;      // inversion work space in global memory for separators too
                                // wide for shared memory (per CTA: S x (CW + 33))
    void *wb = nullptr;         // transposed solve: per-front adjoint right-hand sides (vtotal)
    void *tw = nullptr;         // solve: gathered fronts' t, w and struct x (vtotal)
    double *rs = nullptr;       // row scaling 1 / max |a_r.|
    int *ipiv = nullptr, *perm = nullptr, *flag = nullptr;
    MfBarrier *bar = nullptr;
    int *sctr = nullptr;        // dataflow solve: 3 counters per front + the work ticket
    int flow_grid = 0;          // most CTAs of the dataflow solve resident at once
    int flow_grid1 = 0;         // the same for its high-occupancy form (0: none)
    int flow_form = 0;          // 0: 2 CTAs per SM, 32 row registers; 1: 3 CTAs, 16
    int split = 0;              // > 0: tree levels [0, split) in launches of their own
                                // (forward before, backward after the upper levels)
    int low_grid = 0;           // CTAs of those launches
    size_t low_smem = 0;        // and their shared memory
    int low_wcap = 0;           // their largest front
    int flow = 1;               // 1: the solve is one dataflow launch; 0: one launch per level
                                // and sweep
    cudaGraphExec_t graph = nullptr;
    const double *graph_val = nullptr;
    const int *graph_rowptr = nullptr;
    long long launches_per_factor = 0;
};

// Kernel-side view of a plan + factor (passed by value).
struct MfDev {
    const int *S, *f, *voff, *uoff, *child0, *child1, *parent;
    const long long *foff;
    const int *vars, *cbmap, *perm;
    int maxS, maxf;
    void *tw;   // gathered fronts: t and w (forward), -x on the struct variables (backward)
};

// Host-only symbolic phase (validates every index it produces).
int mf_plan_build(int imax, int jmax, int n, const int *h_rowptr, const int *h_colind, int leaf,
                  MfPlan **out);
// mf_plan_build + upload of the index arrays.
int mf_plan_create(int imax, int jmax, int n, const int *h_rowptr, const int *h_colind, int leaf,
                   MfPlan **out);
void mf_plan_destroy(MfPlan *p);
// One plan over several host plans (mf_plan_build) of the diagonal blocks of a
// block-diagonal system: row_off / nnz_off place each block's rows and CSR
// entries in the combined system of n rows (v2d_mf.cu).
int mf_plan_forest(const std::vector<MfPlan *> &parts, const std::vector<int> &row_off,
                   const std::vector<long long> &nnz_off, int n, MfPlan **out);
// Work-item granularity of the solve per level (rows per item, 0: whole
// fronts); replaces the device item table.
int mf_plan_set_item_rows(MfPlan *P, const int *rows, int nlevels);
// Split form of the dataflow solve: levels [0, split) in launches of their
// own (0: one launch); sizes their shared memory and grid.
int mf_set_split(const MfPlan *P, MfFactor *M, int split);
// fp32: FP32 solve; fact64 (with fp32): FP64 factorization rounded to FP32.
int mf_factor_create(const MfPlan *P, int fp32, int fact64, MfFactor **out);
void mf_factor_destroy(MfFactor *M);
MfDev mf_dev(const MfPlan *P, const MfFactor *M);
// Factor the CSR values (FP64, row-scaled and rounded to the factor's precision).
int mf_factor(const MfPlan *P, MfFactor *M, const int *rowptr, const double *val, cudaStream_t s);
// x = A^-1 b with the factors (vectors in the factor's precision): one
// dataflow launch (M->flow) or one launch per level and sweep.  The kernels
// exit at once while *stop_a or *stop_b is non-zero (either may be null).
// *n_launches (if given) receives the number of kernels launched.
int mf_apply(const MfPlan *P, const MfFactor *M, const void *b, void *x, const int *stop_a,
             const int *stop_b, cudaStream_t s, long long *n_launches);
// lambda = A^-T g with the factors (the transposed solve: a bottom-up sweep
// with U11^-T / H^T, then a top-down sweep with L11^-T / G^T).
int mf_apply_transpose(const MfPlan *P, MfFactor *M, const void *g, void *lambda, cudaStream_t s,
                       long long *launches = nullptr);
int mf_flag(const MfFactor *M, int *flag, cudaStream_t s);
// V2D_ETIMEOUT (and a reset error state) if a dependency wait of the
// dataflow solve timed out since the last check.
int mf_check_barrier(MfFactor *M, cudaStream_t s);
// Average device time (ms) of `reps` LU applies to a zero vector, each after a
// write of flush_bytes (evicts L2); CUDA events on stream s.
int mf_time_apply(const MfPlan *P, const MfFactor *M, int reps, size_t flush_bytes, cudaStream_t s,
                  double *ms_avg);
// One dataflow solve with per-item global-timer ticks (3 per item: ticket,
// end of wait, done); *n = items.
int mf_trace_apply(const MfPlan *P, const MfFactor *M, cudaStream_t s, unsigned long long *ticks,
                   int cap, int *n);
// Per-launch device time of one solve (average of reps), with the launch
// codes (kind * 1000 + level; kinds: 0 forward level, 1 backward level,
// 2 the dataflow launch); *n receives the number of launches.
int mf_time_apply_launches(const MfPlan *P, const MfFactor *M, int reps, size_t flush_bytes,
                           cudaStream_t s, double *ms, int *codes, int cap, int *n);
// Per-kernel device time of one factorization launched directly (not from
// its graph), average of reps; codes kind * 1000 + level (kinds 0 rowscale,
// 1 scatter, 2 extend_add, 3 panel, 4 L21 + row swaps + U12, 6 gemm,
// 7 trinv, 8 trcopy, 9 G/H products, 10 G/H copy).  The factors are recomputed from the same values.
int mf_time_factor_launches(const MfPlan *P, MfFactor *M, const int *rowptr, const double *val,
                            int reps, cudaStream_t s, double *ms, int *codes, int cap, int *n);

// ------------------------------------------------------------- Krylov
// A CSR operator with optional FP32 copy and 2x2 block inverse.
// layout: 0 point (dinv holds 1/a_rr in slot 0), 1 field-blocked pairs (q, q+n/2),
//         2 interleaved pairs (2q, 2q+1).
struct CsrOp {
    int n = 0;
    long long nnz = 0;
    const int *rowptr = nullptr, *colind = nullptr;
    const double *val = nullptr;
    const float *val32 = nullptr;
    const double *dinv = nullptr;
    const float *dinv32 = nullptr;
    int layout = 1;
    int nblk = 0;  // number of 2x2 blocks (or n for point layout)
    const MfPlan *lu_plan = nullptr;   // V2D_PC_LU: factors of this operator
    const MfFactor *lu = nullptr;
    bool lu_transpose = false;         // the operator is J^T and lu factors J: the
                                       // preconditioner is the transposed solve
};

struct KrylovWork;  // defined in v2d_krylov.cu

int krylov_create(KrylovWork **out, int n, int restart, cudaStream_t s);
void krylov_destroy(KrylovWork *w);
// Solves A x = b (x is overwritten, starting from zero).  d_b, d_x device.
int krylov_solve(KrylovWork *w, const CsrOp &A, const double *d_b, double *d_x,
                 const v2d_krylov_params &prm, v2d_lin_stats *st, cudaStream_t s);

int time_spmv(const CsrOp &A, bool fp32, int reps, size_t flush_bytes, cudaStream_t s,
              double *ms_avg);

// 2x2 block inverse of a CSR operator (generic layouts).
int launch_block_inverse(CsrOp &A, double *dinv, float *dinv32, int *d_flag, cudaStream_t s);

}  // namespace v2d

// The device-resident solver handle behind the C ABI (v2d_solver.cu).
struct v2d_solver {
    v2d::GridDev g;
    v2d_solver_params prm{};
    v2d::AsmParams ap{};
    cudaStream_t s = nullptr;
    v2d::KrylovWork *kw = nullptr;
    double *delta = nullptr;      // Newton update (2N)
    double *partial = nullptr;    // reduction partials
    double *scal = nullptr;       // device scalars: [0] res, [1..10] forces
    int *flag = nullptr;
    unsigned int *counter = nullptr;
    double *host = nullptr;       // pinned mirror of scal
    int pattern_ff_bc = -1;
    double pattern_ca = 0, pattern_sa = 0;
    bool assembled = false;
    v2d::MfPlan *plan = nullptr;        // multifrontal plan of the current pattern
    int plan_leaf = 0;
    v2d::MfFactor *lu[2] = {nullptr, nullptr};  // [0] FP64 factors, [1] FP32 factors
    bool lu_valid = false;           // factors of an earlier Jacobian kept for reuse
    bool lu_ready = false;           // the factor storage holds some factorization
    int lu_last_its = 0;             // Krylov iterations of the last solve with them
    long long lu_factorizations = 0;
    int *tptr = nullptr, *tind = nullptr, *tperm = nullptr;   // transposed CSR pattern (adjoint)
    double *valT = nullptr;           // J^T values on that pattern (adjoint GMRES)
    double *adj_vec = nullptr;        // adjoint g, lambda and J^T lambda (3 x 2N; kept, since
                                      // the GMRES graphs write lambda by address)
    v2d::KrylovWork *kw_adj = nullptr;   // GMRES work space of the adjoint solves
    // versions for the adjoint's factor cache: the state (psi, ome) and the
    // parameters, the assembled values, and the FP64 factors lu[0]
    long long state_ver = 0, val_ver = 0, lu0_ver = 0;
    long long adj_key[3] = {-1, -1, -1};   // the versions when lu[0] last held J (adjoint)
    cudaEvent_t ev[5] = {};          // phase boundaries of the last Newton iteration
    double phase_ms[4] = {0, 0, 0, 0};
    long long phase_n = 0;
};

