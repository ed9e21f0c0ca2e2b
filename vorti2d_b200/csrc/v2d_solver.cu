// Device-resident Newton / BDF2 driver (reference vorti2d/solver.py:48-224).
//
// The whole replicated state -- mesh, metrics, psi/ome and their BDF2 history,
// the canonical CSR Jacobian, right-hand side, block inverses and the Krylov
// workspace -- lives in HBM behind one handle.  One Newton iteration is:
// fused assembly kernel (values written into fixed CSR slots + b + 2x2 block
// inverses), with the LU preconditioner the multifrontal factorization of the
// new Jacobian (one CUDA graph), GMRES(m) on the device, and a fused update
// kernel (q += dq and ||dq||_2 in one pass).  The host reads one scalar per Newton
// iteration to decide whether to continue, as the reference's loop does.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "v2d_internal.cuh"

using namespace v2d;


namespace {

constexpr int kUpdThreads = 256;
constexpr int kUpdBlocks = 2 * kSMs;

// q += dq (psi: dq[0,N), ome: dq[N,2N)); *res = ||dq||_2 / (2N)
// (vorti2d/solver.py:132-134).  Deterministic two-stage sum.
__global__ void __launch_bounds__(kUpdThreads) k_newton_update(int N, const double *__restrict__ dq,
                                                               double *psi, double *ome,
                                                               double *partial, unsigned int *counter,
                                                               double *res)
{
    __shared__ double red[32];
    __shared__ bool last;
    double acc = 0.0;
    V2D_GRID_STRIDE(t, N)
    {
        double a = dq[t], b = dq[N + t];
        psi[t] += a;
        ome[t] += b;
        acc += a * a + b * b;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last && threadIdx.x < 32) {
        __threadfence();
        double s = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) s += partial[b];
        s = warp_sum(s);
        if (threadIdx.x == 0) {
            *res = sqrt(s) / (2.0 * (double)N);
            *counter = 0;
        }
    }
}

// Far-field initial streamfunction (vorti2d/solver.py:103-112).
__global__ void k_init_state(int imax, int jmax, double ca, double sa, const double *xp,
                             const double *yp, double *psi, double *ome, double *omeold,
                             double *omeoldold)
{
    const int N = imax * jmax;
    V2D_GRID_STRIDE(t, N)
    {
        int K = (int)t;
        psi[K] = K >= imax * (jmax - 1) ? ca * yp[K] - sa * xp[K] : 0.0;
        ome[K] = 0.0;
        omeold[K] = 0.0;
        omeoldold[K] = 0.0;
    }
}

int check_params(const v2d_solver_params *p)
{
    V2D_ARG_CHECK(p, "null params");
    V2D_ARG_CHECK(p->re > 0.0 && std::isfinite(p->re), "re must be positive (got %g)", p->re);
    V2D_ARG_CHECK(p->ff_bc >= 0 && p->ff_bc <= 2, "ff_bc must be 0, 1 or 2 (got %d)", p->ff_bc);
    V2D_ARG_CHECK(p->krylov.restart >= 1 && p->krylov.restart <= 256,
                  "krylov restart must be in [1, 256] (got %d)", p->krylov.restart);
    V2D_ARG_CHECK(p->krylov.max_it >= 1, "krylov max_it must be >= 1");
    V2D_ARG_CHECK(p->krylov.precond == V2D_PC_NONE || p->krylov.precond == V2D_PC_BJACOBI ||
                      p->krylov.precond == V2D_PC_LU,
                  "unknown preconditioner %d", p->krylov.precond);
    V2D_ARG_CHECK(p->krylov.precision == V2D_PREC_FP64 || p->krylov.precision == V2D_PREC_MIXED,
                  "unknown precision %d", p->krylov.precision);
    return V2D_OK;
}

void drop_transpose(v2d_solver *S)
{
    for (int *p : {S->tptr, S->tind, S->tperm})
        if (p) cudaFree(p);
    S->tptr = S->tind = S->tperm = nullptr;
    if (S->valT) cudaFree(S->valT);
    S->valT = nullptr;
    if (S->adj_vec) cudaFree(S->adj_vec);
    S->adj_vec = nullptr;
    krylov_destroy(S->kw_adj);
    S->kw_adj = nullptr;
}

void drop_lu(v2d_solver *S)
{
    drop_transpose(S);   // follows the pattern like the plan
    S->lu_valid = false;
    S->lu_ready = false;
    for (int q = 0; q < 2; ++q) {
        mf_factor_destroy(S->lu[q]);
        S->lu[q] = nullptr;
    }
    mf_plan_destroy(S->plan);
    S->plan = nullptr;
}

int ensure_pattern(v2d_solver *S)
{
    const v2d_solver_params &p = S->prm;
    if (S->pattern_ff_bc == p.ff_bc && S->pattern_ca == p.ca && S->pattern_sa == p.sa) return V2D_OK;
    AsmParams ap{p.re, p.invdtau, p.inv2dt, 0.0, p.ca, p.sa, p.ff_bc};
    V2D_TRY(build_pattern(S->g, ap, S->s));
    S->pattern_ff_bc = p.ff_bc;
    S->pattern_ca = p.ca;
    S->pattern_sa = p.sa;
    S->assembled = false;
    drop_lu(S);   // the multifrontal plan follows the pattern
    return V2D_OK;
}

// Multifrontal plan (once per pattern) and factor storage of the current precision.
int ensure_lu(v2d_solver *S)
{
    const v2d_krylov_params &k = S->prm.krylov;
    if (k.precond != V2D_PC_LU) return V2D_OK;
    const int leaf = k.lu_leaf > 0 ? k.lu_leaf : 64;
    if (S->plan && S->plan_leaf != leaf) drop_lu(S);
    if (!S->plan) {
        const GridDev &g = S->g;
        std::vector<int> rp(g.n + 1), ci(g.nnz);
        V2D_CUDA_TRY(cudaMemcpyAsync(rp.data(), g.rowptr, (g.n + 1) * sizeof(int), cudaMemcpyDeviceToHost, S->s));
        V2D_CUDA_TRY(cudaMemcpyAsync(ci.data(), g.colind, g.nnz * sizeof(int), cudaMemcpyDeviceToHost, S->s));
        V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
        V2D_TRY(mf_plan_create(g.imax, g.jmax, g.n, rp.data(), ci.data(), leaf, &S->plan));
        S->plan_leaf = leaf;
    }
    const int q = k.precision == V2D_PREC_MIXED ? 1 : 0;
    const int f64 = q && k.lu_factor64 ? 1 : 0;
    if (S->lu[q] && S->lu[q]->fact64 != f64) {   // the factorization precision changed
        mf_factor_destroy(S->lu[q]);
        S->lu[q] = nullptr;
        S->lu_valid = false;
    }
    if (!S->lu[q]) V2D_TRY(mf_factor_create(S->plan, q, f64, &S->lu[q]));
    S->lu[q]->flow = k.lu_solve == 0 ? 1 : 0;
    return V2D_OK;
}

int sync_flag(v2d_solver *S, const char *what)
{
    int f = 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(&f, S->flag, sizeof(int), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    if (f & 4) {
        set_error("%s: a Jacobian row does not match the CSR pattern", what);
        return V2D_ECUDA;
    }
    if (f & 2) {
        set_error("%s: non-finite right-hand side (check the state / mesh)", what);
        return V2D_ENONFINITE;
    }
    if (f & 1) {
        set_error("%s: singular 2x2 (psi, ome) diagonal block", what);
        return V2D_EBREAKDOWN;
    }
    return V2D_OK;
}

}  // namespace

extern "C" void v2d_krylov_defaults(v2d_krylov_params *p)
{
    if (!p) return;
    p->restart = 30;
    p->max_it = 5000;
    p->rtol = 1e-10;
    p->atol = 1e-50;
    p->precond = V2D_PC_BJACOBI;
    p->precision = V2D_PREC_FP64;
    p->inner_rtol = 1e-5;
    p->dc_max_it = 20;
    p->lu_leaf = 64;
    p->lu_reuse_its = 0;
    p->lu_reuse_steps = 0;
    p->lu_solve = 0;
    p->lu_factor64 = 0;
}

extern "C" int v2d_solver_destroy(v2d_solver *S)
{
    if (!S) return V2D_OK;
    if (S->s) cudaStreamSynchronize(S->s);
    GridDev &g = S->g;
    drop_lu(S);
    for (cudaEvent_t e : S->ev)
        if (e) cudaEventDestroy(e);
    void *ptrs[] = {g.x, g.rowptr, g.colind, g.val, g.val32, g.b, g.dinv, g.dinv32,
                    S->delta, S->partial, S->scal, S->flag, S->counter};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (S->host) cudaFreeHost(S->host);
    krylov_destroy(S->kw);
    if (S->s) cudaStreamDestroy(S->s);
    delete S;
    return V2D_OK;
}

extern "C" int v2d_solver_create(int imax, int jmax, const double *xg, const double *yg,
                                 const v2d_solver_params *p, v2d_solver **out)
{
    V2D_ARG_CHECK(out && xg && yg, "solver_create: null pointer");
    *out = nullptr;
    V2D_ARG_CHECK(imax >= 4 && jmax >= 4, "mesh must be at least 4x4 (got %d x %d)", imax, jmax);
    V2D_ARG_CHECK((long long)imax * jmax * 2 < (1LL << 31) / 16, "mesh too large for int32 CSR");
    V2D_TRY(check_params(p));
    v2d_solver *S = new v2d_solver();
    S->prm = *p;
    GridDev &g = S->g;
    g.imax = imax; g.jmax = jmax; g.N = imax * jmax; g.n = 2 * g.N;
    g.dksi = 1.0 / (imax - 1);
    g.deta = 1.0 / (jmax - 1);
    const size_t N = g.N;
    cudaError_t e = cudaStreamCreateWithFlags(&S->s, cudaStreamNonBlocking);
    // one slab: x, y, 10 metrics, 4 state arrays
    if (e == cudaSuccess) e = cudaMalloc(&g.x, 16 * N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&g.rowptr, (2 * N + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&g.b, 2 * N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&g.dinv, 4 * N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&g.dinv32, 4 * N * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&S->delta, 2 * N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&S->partial, 4096 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&S->scal, 16 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&S->flag, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&S->counter, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&S->host, 16 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(S->counter, 0, sizeof(unsigned int), S->s);
    for (int q = 0; q < 5 && e == cudaSuccess; ++q) e = cudaEventCreate(&S->ev[q]);
    if (e != cudaSuccess) {
        set_error("solver_create: allocation failed: %s", cudaGetErrorString(e));
        v2d_solver_destroy(S);
        return V2D_ENOMEM;
    }
    g.y = g.x + N;
    for (int q = 0; q < 10; ++q) g.met[q] = g.x + (2 + q) * N;
    g.psi = g.x + 12 * N; g.ome = g.x + 13 * N; g.omeold = g.x + 14 * N; g.omeoldold = g.x + 15 * N;
    int st = V2D_OK;
    // Fortran-ordered (imax, jmax) is already pointer order
    if (cudaMemcpyAsync(g.x, xg, N * sizeof(double), cudaMemcpyHostToDevice, S->s) != cudaSuccess ||
        cudaMemcpyAsync(g.y, yg, N * sizeof(double), cudaMemcpyHostToDevice, S->s) != cudaSuccess) {
        set_error("solver_create: mesh upload failed");
        st = V2D_ECUDA;
    }
    if (st == V2D_OK) st = launch_metrics(g, S->s);
    if (st == V2D_OK) {
        k_init_state<<<grid_for(g.N, 256), 256, 0, S->s>>>(imax, jmax, p->ca, p->sa, g.met[8],
                                                            g.met[9], g.psi, g.ome, g.omeold,
                                                            g.omeoldold);
        if (cudaGetLastError() != cudaSuccess) st = V2D_ECUDA;
    }
    if (st == V2D_OK) st = ensure_pattern(S);
    if (st == V2D_OK) st = ensure_lu(S);
    if (st == V2D_OK) st = krylov_create(&S->kw, g.n, p->krylov.restart, S->s);
    if (st == V2D_OK && cudaStreamSynchronize(S->s) != cudaSuccess) {
        set_error("solver_create: %s", cudaGetErrorString(cudaGetLastError()));
        st = V2D_ECUDA;
    }
    if (st != V2D_OK) {
        v2d_solver_destroy(S);
        return st;
    }
    *out = S;
    return V2D_OK;
}

extern "C" int v2d_solver_set_params(v2d_solver *S, const v2d_solver_params *p)
{
    V2D_ARG_CHECK(S, "null solver");
    V2D_TRY(check_params(p));
    const int old_m = S->prm.krylov.restart;
    S->prm = *p;
    S->lu_valid = false;
    ++S->state_ver;   // the Jacobian depends on the parameters
    V2D_TRY(ensure_pattern(S));
    V2D_TRY(ensure_lu(S));
    if (p->krylov.restart != old_m) {
        V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
        krylov_destroy(S->kw);
        S->kw = nullptr;
        V2D_TRY(krylov_create(&S->kw, S->g.n, p->krylov.restart, S->s));
    }
    return V2D_OK;
}

extern "C" int v2d_solver_set_state(v2d_solver *S, const double *psi, const double *ome,
                                    const double *omeold, const double *omeoldold)
{
    V2D_ARG_CHECK(S, "null solver");
    const size_t bytes = (size_t)S->g.N * sizeof(double);
    const double *src[4] = {psi, ome, omeold, omeoldold};
    double *dst[4] = {S->g.psi, S->g.ome, S->g.omeold, S->g.omeoldold};
    for (int q = 0; q < 4; ++q)
        if (src[q]) V2D_CUDA_TRY(cudaMemcpyAsync(dst[q], src[q], bytes, cudaMemcpyHostToDevice, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    S->assembled = false;
    ++S->state_ver;
    // a new state: old factors precondition it only when the caller keeps
    // factors across steps (a solve that needs more than lu_reuse_its + 5
    // iterations with them refactors and solves again)
    if (!S->prm.krylov.lu_reuse_steps) S->lu_valid = false;
    return V2D_OK;
}

extern "C" int v2d_solver_get_state(v2d_solver *S, double *psi, double *ome, double *omeold,
                                    double *omeoldold)
{
    V2D_ARG_CHECK(S, "null solver");
    const size_t bytes = (size_t)S->g.N * sizeof(double);
    double *dst[4] = {psi, ome, omeold, omeoldold};
    const double *src[4] = {S->g.psi, S->g.ome, S->g.omeold, S->g.omeoldold};
    for (int q = 0; q < 4; ++q)
        if (dst[q]) V2D_CUDA_TRY(cudaMemcpyAsync(dst[q], src[q], bytes, cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

extern "C" int v2d_solver_get_metrics(v2d_solver *S, double *const *out10)
{
    V2D_ARG_CHECK(S && out10, "null pointer");
    const size_t bytes = (size_t)S->g.N * sizeof(double);
    for (int q = 0; q < 10; ++q) {
        V2D_ARG_CHECK(out10[q], "get_metrics: null output %d", q);
        V2D_CUDA_TRY(cudaMemcpyAsync(out10[q], S->g.met[q], bytes, cudaMemcpyDeviceToHost, S->s));
    }
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

// Newton system of the current state; pseudo = false leaves out the
// pseudo-time term invdtau (the adjoint needs dR/dq of the physical residual).
static int assemble_now(v2d_solver *S, double urot, bool pseudo = true)
{
    V2D_TRY(ensure_pattern(S));
    const v2d_solver_params &p = S->prm;
    AsmParams ap{p.re, pseudo ? p.invdtau : 0.0, p.inv2dt, urot, p.ca, p.sa, p.ff_bc};
    ++S->val_ver;
    V2D_CUDA_TRY(cudaMemsetAsync(S->flag, 0, sizeof(int), S->s));
    V2D_TRY(launch_assemble(S->g, ap, p.krylov.precision == V2D_PREC_MIXED, S->flag, S->s));
    S->assembled = true;
    return V2D_OK;
}

extern "C" int v2d_solver_assemble(v2d_solver *S, double urot)
{
    V2D_ARG_CHECK(S, "null solver");
    V2D_TRY(assemble_now(S, urot));
    return sync_flag(S, "assemble");
}

extern "C" int v2d_solver_newton(v2d_solver *S, double urot, double *res, v2d_lin_stats *st)
{
    V2D_ARG_CHECK(S, "null solver");
    GridDev &g = S->g;
    V2D_CUDA_TRY(cudaEventRecord(S->ev[0], S->s));
    V2D_TRY(assemble_now(S, urot));
    V2D_CUDA_TRY(cudaEventRecord(S->ev[1], S->s));
    V2D_TRY(sync_flag(S, "newton assembly"));
    CsrOp A;
    A.n = g.n; A.nnz = g.nnz; A.rowptr = g.rowptr; A.colind = g.colind; A.val = g.val;
    A.val32 = g.val32; A.dinv = g.dinv; A.dinv32 = g.dinv32; A.layout = 1; A.nblk = g.N;
    const v2d_krylov_params &kp = S->prm.krylov;
    const bool lu = kp.precond == V2D_PC_LU;
    const int mixed = kp.precision == V2D_PREC_MIXED ? 1 : 0;
    bool refactored = false;
    if (lu) {
        V2D_TRY(ensure_lu(S));
        const bool reuse = kp.lu_reuse_its > 0 && S->lu_valid && S->lu_last_its <= kp.lu_reuse_its;
        if (!reuse) {
            V2D_TRY(mf_factor(S->plan, S->lu[mixed], g.rowptr, g.val, S->s));
            if (!mixed) ++S->lu0_ver;
            ++S->lu_factorizations;
            S->lu_ready = true;
            refactored = true;
        }
        A.lu_plan = S->plan;
        A.lu = S->lu[mixed];
    }
    V2D_CUDA_TRY(cudaEventRecord(S->ev[2], S->s));
    v2d_lin_stats ls{};
    if (lu && !refactored) {
        // stale factors: bounded attempt, then refactor and solve again
        v2d_krylov_params k2 = kp;
        k2.max_it = std::min(kp.max_it, kp.lu_reuse_its + 5);
        V2D_TRY(krylov_solve(S->kw, A, g.b, S->delta, k2, &ls, S->s));
        V2D_TRY(mf_check_barrier(S->lu[mixed], S->s));   // a timed-out solve is no retry case
        if (!ls.converged) {
            const int its0 = ls.iterations;
            V2D_TRY(mf_factor(S->plan, S->lu[mixed], g.rowptr, g.val, S->s));
            if (!mixed) ++S->lu0_ver;
            ++S->lu_factorizations;
            S->lu_ready = true;
            refactored = true;
            V2D_TRY(krylov_solve(S->kw, A, g.b, S->delta, kp, &ls, S->s));
            ls.iterations += its0;
        }
    } else {
        V2D_TRY(krylov_solve(S->kw, A, g.b, S->delta, kp, &ls, S->s));
    }
    if (lu) {
        V2D_TRY(mf_check_barrier(S->lu[mixed], S->s));
        S->lu_valid = true;
        S->lu_last_its = refactored ? 0 : ls.iterations;
    }
    V2D_CUDA_TRY(cudaEventRecord(S->ev[3], S->s));
    if (st) *st = ls;
    const int grid = std::max(1, std::min(kUpdBlocks, (g.N + kUpdThreads * 8 - 1) / (kUpdThreads * 8)));
    k_newton_update<<<grid, kUpdThreads, 0, S->s>>>(g.N, S->delta, g.psi, g.ome, S->partial,
                                                     S->counter, S->scal);
    ++S->state_ver;
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    V2D_CUDA_TRY(cudaEventRecord(S->ev[4], S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(S->host, S->scal, sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    for (int q = 0; q < 4; ++q) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, S->ev[q], S->ev[q + 1]) == cudaSuccess) S->phase_ms[q] += ms;
    }
    ++S->phase_n;
    S->assembled = false;
    const double r = S->host[0];
    if (res) *res = r;
    if (!std::isfinite(r)) {
        set_error("newton: non-finite update norm");
        return V2D_ENONFINITE;
    }
    if (!ls.converged) {
        set_error("newton: Krylov solve did not converge (%d iterations, |r|/|b| = %.3e)",
                  ls.iterations, ls.res0 > 0 ? ls.res / ls.res0 : 0.0);
        return V2D_ENOTCONVERGED;
    }
    return V2D_OK;
}

extern "C" int v2d_solver_pseudo_solve(v2d_solver *S, double urot, double pseudo_tol,
                                       int max_iter, v2d_newton_info *info)
{
    V2D_ARG_CHECK(S, "null solver");
    double res = 1.0e5;
    int it = 0;
    v2d_newton_info inf{};
    int status = V2D_OK;
    while (res > pseudo_tol && it < max_iter) {
        v2d_lin_stats ls{};
        status = v2d_solver_newton(S, urot, &res, &ls);
        inf.krylov_iters += ls.iterations;
        inf.corrections += ls.corrections;
        double rel = ls.res0 > 0 ? ls.res / ls.res0 : 0.0;
        if (rel > inf.lin_res_max) inf.lin_res_max = rel;
        ++it;
        if (status != V2D_OK) break;
    }
    inf.newton_iters = it;
    inf.res = res;
    if (info) *info = inf;
    return status;
}

extern "C" int v2d_solver_shift_history(v2d_solver *S)
{
    V2D_ARG_CHECK(S, "null solver");
    const size_t bytes = (size_t)S->g.N * sizeof(double);
    V2D_CUDA_TRY(cudaMemcpyAsync(S->g.omeoldold, S->g.omeold, bytes, cudaMemcpyDeviceToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(S->g.omeold, S->g.ome, bytes, cudaMemcpyDeviceToDevice, S->s));
    // factors are reused within a time step and refreshed at the next, unless
    // the caller keeps them across steps under the same iteration rule
    if (!S->prm.krylov.lu_reuse_steps) S->lu_valid = false;
    return V2D_OK;
}

extern "C" int v2d_solver_step(v2d_solver *S, double urot, double pseudo_tol, int max_iter,
                               int unsteady, v2d_newton_info *info)
{
    int st = v2d_solver_pseudo_solve(S, urot, pseudo_tol, max_iter, info);
    if (st != V2D_OK) return st;
    if (unsteady) V2D_TRY(v2d_solver_shift_history(S));
    return V2D_OK;
}

extern "C" int v2d_solver_forces(v2d_solver *S, double re, double ref_length, double x0,
                                 double y0, double *out10)
{
    V2D_ARG_CHECK(S && out10, "null pointer");
    V2D_TRY(launch_forces(S->g, re, ref_length, x0, y0, S->scal + 1, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(S->host + 1, S->scal + 1, 10 * sizeof(double),
                                 cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    std::memcpy(out10, S->host + 1, 10 * sizeof(double));
    return V2D_OK;
}

extern "C" int v2d_solver_velocity(v2d_solver *S, double *u, double *v, double *vmag)
{
    V2D_ARG_CHECK(S && u && v, "solver_velocity: null pointer");
    const GridDev &g = S->g;
    const size_t N = g.N;
    DevBuf<double> buf;
    V2D_TRY(buf.alloc(3 * N, S->s));
    V2D_TRY(launch_velocity(g.imax, g.jmax, g.dksi, g.deta, g.met[0], g.met[2], g.met[3], g.met[6],
                            g.met[7], g.psi, buf.p, buf.p + N, vmag ? buf.p + 2 * N : nullptr,
                            S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(u, buf.p, N * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(v, buf.p + N, N * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    if (vmag)
        V2D_CUDA_TRY(cudaMemcpyAsync(vmag, buf.p + 2 * N, N * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

// ------------------------------------------------------------------ adjoint
namespace {

// GMRES restart length of the adjoint solves
constexpr int kAdjRestart = 30;

// valT[e] = val[tperm[e]]: J's values in the order of the transposed pattern.
__global__ void k_gather_vals(long long nnz, const int *__restrict__ tperm,
                              const double *__restrict__ val, double *valT)
{
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (long long)gridDim.x * blockDim.x)
        valT[e] = val[tperm[e]];
}

// y = J^T x over the transposed pattern (values gathered through tperm).
__global__ void k_spmv_t(int n, const int *__restrict__ tptr, const int *__restrict__ tind,
                         const int *__restrict__ tperm, const double *__restrict__ val,
                         const double *__restrict__ x, double *y)
{
    V2D_GRID_STRIDE(r, n)
    {
        double s = 0.0;
        for (int e = tptr[r]; e < tptr[r + 1]; ++e) s += val[tperm[e]] * x[tind[e]];
        y[r] = s;
    }
}

int ensure_transpose(v2d_solver *S)
{
    if (S->tptr) return V2D_OK;
    const GridDev &g = S->g;
    std::vector<int> rp(g.n + 1), ci(g.nnz);
    V2D_CUDA_TRY(cudaMemcpyAsync(rp.data(), g.rowptr, (g.n + 1) * sizeof(int), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(ci.data(), g.colind, g.nnz * sizeof(int), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    std::vector<int> tp(g.n + 1, 0), ti(g.nnz), tq(g.nnz);
    for (long long e = 0; e < g.nnz; ++e) tp[ci[e] + 1]++;
    for (int r = 0; r < g.n; ++r) tp[r + 1] += tp[r];
    std::vector<int> fill(tp.begin(), tp.end() - 1);
    for (int r = 0; r < g.n; ++r)
        for (int e = rp[r]; e < rp[r + 1]; ++e) {
            const int o = fill[ci[e]]++;
            ti[o] = r;
            tq[o] = e;
        }
    V2D_CUDA_TRY(cudaMalloc(&S->tptr, (g.n + 1) * sizeof(int)));
    V2D_CUDA_TRY(cudaMalloc(&S->tind, g.nnz * sizeof(int)));
    V2D_CUDA_TRY(cudaMalloc(&S->tperm, g.nnz * sizeof(int)));
    V2D_CUDA_TRY(cudaMemcpy(S->tptr, tp.data(), (g.n + 1) * sizeof(int), cudaMemcpyHostToDevice));
    V2D_CUDA_TRY(cudaMemcpy(S->tind, ti.data(), g.nnz * sizeof(int), cudaMemcpyHostToDevice));
    V2D_CUDA_TRY(cudaMemcpy(S->tperm, tq.data(), g.nnz * sizeof(int), cudaMemcpyHostToDevice));
    return V2D_OK;
}

double host_norm(const std::vector<double> &v)
{
    double s = 0.0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
}

}  // namespace

extern "C" int v2d_solver_residual(v2d_solver *S, double re, double invdtau, double inv2dt,
                                   double urot, double ca, double sa, double *b)
{
    V2D_ARG_CHECK(S && b, "solver_residual: null pointer");
    V2D_ARG_CHECK(re > 0.0, "solver_residual: re must be positive");
    const GridDev &g = S->g;
    DevBuf<double> d;
    V2D_TRY(d.alloc(g.n, S->s));
    AsmParams ap{re, invdtau, inv2dt, urot, ca, sa, S->prm.ff_bc};
    V2D_TRY(launch_residual(g, ap, d.p, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(b, d.p, g.n * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

extern "C" int v2d_solver_residual_mesh(v2d_solver *S, const double *xg, const double *yg,
                                        double re, double invdtau, double inv2dt, double urot,
                                        double ca, double sa, double *b, int met_rows,
                                        double *met)
{
    V2D_ARG_CHECK(S && xg && yg && b, "solver_residual_mesh: null pointer");
    V2D_ARG_CHECK(re > 0.0, "solver_residual_mesh: re must be positive");
    V2D_ARG_CHECK(met_rows >= 0 && met_rows <= S->g.jmax && (met_rows == 0 || met),
                  "solver_residual_mesh: met_rows=%d outside [0, %d] or null output", met_rows,
                  S->g.jmax);
    // a copy of the grid description whose mesh and metric arrays point to
    // scratch: the state is the handle's, the handle itself is not changed
    GridDev g = S->g;
    const size_t N = (size_t)g.N;
    DevBuf<double> buf;
    V2D_TRY(buf.alloc(12 * N + (size_t)g.n, S->s));
    g.x = buf.p;
    g.y = buf.p + N;
    for (int q = 0; q < 10; ++q) g.met[q] = buf.p + (2 + q) * N;
    double *d = buf.p + 12 * N;
    V2D_CUDA_TRY(cudaMemcpyAsync(g.x, xg, N * sizeof(double), cudaMemcpyHostToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(g.y, yg, N * sizeof(double), cudaMemcpyHostToDevice, S->s));
    V2D_TRY(launch_metrics(g, S->s));
    count_launches(1);
    AsmParams ap{re, invdtau, inv2dt, urot, ca, sa, S->prm.ff_bc};
    V2D_TRY(launch_residual(g, ap, d, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(b, d, g.n * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    const size_t rows = (size_t)g.imax * met_rows;
    for (int q = 0; q < 10 && rows > 0; ++q)
        V2D_CUDA_TRY(cudaMemcpyAsync(met + q * rows, g.met[q], rows * sizeof(double),
                                     cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

namespace v2d {

// Column i of the mesh (and the seam column imax-1 with i = 0) set to the base
// coordinates plus (ax, ay) * phi, or back to the base with restore; the
// product and the sum are rounded separately, as on the host.
static __global__ void k_shape_column(int imax, int jmax, int i, double ax, double ay, int restore,
                               const double *__restrict__ phi, const double *__restrict__ x0,
                               const double *__restrict__ y0, double *x, double *y)
{
    const int cols = i == 0 ? 2 : 1;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cols * jmax;
         t += gridDim.x * blockDim.x) {
        const int j = t % jmax;
        const int c = t < jmax ? i : imax - 1;
        const int k = c + imax * j;
        x[k] = restore ? x0[k] : __dadd_rn(x0[k], __dmul_rn(ax, phi[k]));
        y[k] = restore ? y0[k] : __dadd_rn(y0[k], __dmul_rn(ay, phi[k]));
    }
}

// out[i] = lambda . (bp - bm), one block, fixed summation order.
static __global__ void __launch_bounds__(1024) k_lambda_diff(int n, const double *__restrict__ lam,
                                                      const double *__restrict__ bp,
                                                      const double *__restrict__ bm, double *out,
                                                      int i)
{
    __shared__ double red[32];
    double a = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) a += lam[k] * (bp[k] - bm[k]);
    a = block_sum(a, red);
    if (threadIdx.x == 0) out[i] = a;
}

}  // namespace v2d

extern "C" int v2d_solver_shape_gradient(v2d_solver *S, const double *nx, const double *ny,
                                         const double *phi, const double *lambda, double h,
                                         double re, double invdtau, double inv2dt, double urot,
                                         double ca, double sa, double ref_length, double x0,
                                         double y0, double *dots, double *forces)
{
    V2D_ARG_CHECK(S && nx && ny && phi && lambda && dots && forces,
                  "solver_shape_gradient: null pointer");
    V2D_ARG_CHECK(re > 0.0 && h > 0.0, "solver_shape_gradient: re and h must be positive");
    const GridDev &g0 = S->g;
    const int P = g0.imax - 1;
    const size_t N = (size_t)g0.N, n = (size_t)g0.n;
    DevBuf<double> buf;
    V2D_TRY(buf.alloc(12 * N + 2 * n + n + N + 2 * P + (size_t)P * 20 + P, S->s));
    GridDev g = g0;   // the state is the handle's; mesh and metrics point to scratch
    g.x = buf.p;
    g.y = buf.p + N;
    for (int q = 0; q < 10; ++q) g.met[q] = buf.p + (2 + q) * N;
    double *bp = buf.p + 12 * N, *bm = bp + n, *dlam = bm + n, *dphi = dlam + n;
    double *dnx = dphi + N, *dny = dnx + P, *dforce = dny + P, *ddot = dforce + (size_t)P * 20;
    V2D_CUDA_TRY(cudaMemcpyAsync(g.x, g0.x, N * sizeof(double), cudaMemcpyDeviceToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(g.y, g0.y, N * sizeof(double), cudaMemcpyDeviceToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(dlam, lambda, n * sizeof(double), cudaMemcpyHostToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(dphi, phi, N * sizeof(double), cudaMemcpyHostToDevice, S->s));
    AsmParams ap{re, invdtau, inv2dt, urot, ca, sa, S->prm.ff_bc};
    const int gcol = std::max(1, (2 * g.jmax + 255) / 256);
    for (int i = 0; i < P; ++i) {
        for (int sg = 0; sg < 2; ++sg) {
            const double sgn = sg == 0 ? 1.0 : -1.0;
            k_shape_column<<<gcol, 256, 0, S->s>>>(g.imax, g.jmax, i, sgn * h * nx[i],
                                                   sgn * h * ny[i], 0, dphi, g0.x, g0.y, g.x,
                                                   g.y);
            V2D_CUDA_TRY(cudaGetLastError());
            V2D_TRY(launch_metrics(g, S->s));
            V2D_TRY(launch_residual(g, ap, sg == 0 ? bp : bm, S->s));
            V2D_TRY(launch_forces(g, re, ref_length, x0, y0, dforce + ((size_t)i * 2 + sg) * 10,
                                  S->s));
            count_launches(2);
        }
        k_lambda_diff<<<1, 1024, 0, S->s>>>((int)n, dlam, bp, bm, ddot, i);
        k_shape_column<<<gcol, 256, 0, S->s>>>(g.imax, g.jmax, i, 0.0, 0.0, 1, dphi, g0.x, g0.y,
                                               g.x, g.y);
        V2D_CUDA_TRY(cudaGetLastError());
        count_launches(2);
    }
    V2D_CUDA_TRY(cudaMemcpyAsync(dots, ddot, P * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(forces, dforce, (size_t)P * 20 * sizeof(double),
                                 cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

extern "C" int v2d_solver_shape_tangent(v2d_solver *S, const double *nx, const double *ny,
                                        const double *phi, const double *lambda, double re,
                                        double invdtau, double inv2dt, double urot, double ca,
                                        double sa, double ref_length, double x0, double y0,
                                        double *dots, double *dforces)
{
    V2D_ARG_CHECK(S && nx && ny && phi && lambda && dots && dforces,
                  "solver_shape_tangent: null pointer");
    V2D_ARG_CHECK(re > 0.0, "solver_shape_tangent: re must be positive");
    const GridDev &g = S->g;
    const int P = g.imax - 1;
    const size_t N = (size_t)g.N, n = (size_t)g.n;
    DevBuf<double> buf;
    V2D_TRY(buf.alloc(N + n + 2 * (size_t)P + (size_t)P * 11, S->s));
    double *dphi = buf.p, *dlam = dphi + N, *dnx = dlam + n, *dny = dnx + P, *ddot = dny + P;
    double *dfor = ddot + P;
    V2D_CUDA_TRY(cudaMemcpyAsync(dphi, phi, N * sizeof(double), cudaMemcpyHostToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(dlam, lambda, n * sizeof(double), cudaMemcpyHostToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(dnx, nx, P * sizeof(double), cudaMemcpyHostToDevice, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(dny, ny, P * sizeof(double), cudaMemcpyHostToDevice, S->s));
    AsmParams ap{re, invdtau, inv2dt, urot, ca, sa, S->prm.ff_bc};
    V2D_TRY(launch_shape_tangent(g, ap, dphi, dnx, dny, dlam, ref_length, x0, y0, ddot, dfor,
                                 S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(dots, ddot, P * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(dforces, dfor, (size_t)P * 10 * sizeof(double),
                                 cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

extern "C" int v2d_solver_trace_lu_apply(v2d_solver *S, unsigned long long *ticks, int *items,
                                         int cap, int *n)
{
    V2D_ARG_CHECK(S && ticks && n, "trace_lu_apply: null pointer");
    const int q = S->prm.krylov.precision == V2D_PREC_MIXED ? 1 : 0;
    V2D_ARG_CHECK(S->plan && S->lu[q] && S->lu_ready,
                  "trace_lu_apply: no factors yet (run a Newton iteration)");
    V2D_TRY(mf_trace_apply(S->plan, S->lu[q], S->s, ticks, cap, n));
    if (items)
        std::copy(S->plan->h_items.begin(), S->plan->h_items.end(), items);
    return V2D_OK;
}

extern "C" int v2d_solver_lu_flow_form(v2d_solver *S, int form, int *current)
{
    V2D_ARG_CHECK(S, "null solver");
    const int q = S->prm.krylov.precision == V2D_PREC_MIXED ? 1 : 0;
    V2D_ARG_CHECK(S->lu[q], "lu_flow_form: no LU factors (precond must be V2D_PC_LU)");
    MfFactor *M = S->lu[q];
    if (form >= 0) {
        V2D_ARG_CHECK(form <= 1, "lu_flow_form: form %d (0 or 1)", form);
        V2D_ARG_CHECK(form == 0 || M->flow_grid1 > 0,
                      "lu_flow_form: form 1 does not fit on this GPU");
        V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
        M->flow_form = form;
    }
    if (current) *current = M->flow_form;
    return V2D_OK;
}

extern "C" int v2d_solver_lu_split(v2d_solver *S, int level, int *current)
{
    V2D_ARG_CHECK(S, "null solver");
    const int q = S->prm.krylov.precision == V2D_PREC_MIXED ? 1 : 0;
    V2D_ARG_CHECK(S->lu[q] && S->plan, "lu_split: no LU factors (precond must be V2D_PC_LU)");
    if (level >= 0) {
        V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
        V2D_TRY(mf_set_split(S->plan, S->lu[q], level));
    }
    if (current) *current = S->lu[q]->split;
    return V2D_OK;
}

extern "C" int v2d_solver_lu_item_rows(v2d_solver *S, const int *rows, int nlevels, int *out_rows,
                                       int cap, int *nlevels_out)
{
    V2D_ARG_CHECK(S, "null solver");
    V2D_ARG_CHECK(S->plan, "lu_item_rows: no LU plan (precond must be V2D_PC_LU)");
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    if (rows) V2D_TRY(mf_plan_set_item_rows(S->plan, rows, nlevels));
    if (nlevels_out) *nlevels_out = S->plan->nlevel;
    if (out_rows && cap >= S->plan->nlevel)
        for (int L = 0; L < S->plan->nlevel; ++L) out_rows[L] = S->plan->item_rows[L];
    return V2D_OK;
}

extern "C" int v2d_solver_adjoint(v2d_solver *S, double urot, const double *g_host, double *lam_host,
                                  double rtol, int max_refine, int *refinements, double *rel_res)
{
    V2D_ARG_CHECK(S && g_host && lam_host, "solver_adjoint: null pointer");
    V2D_ARG_CHECK(S->plan || S->prm.krylov.precond == V2D_PC_LU,
                  "solver_adjoint: needs the LU preconditioner");
    V2D_ARG_CHECK(max_refine >= 1, "solver_adjoint: max_refine must be >= 1");
    GridDev &g = S->g;
    // FP64 factors of the Jacobian dR/dq at the current state -- the
    // physical residual's, without the pseudo-time term -- unless lu[0] and
    // the assembled values still hold them from the last adjoint solve
    // (J does not depend on urot: the rotation enters the wall rows' right-
    // hand side only)
    const bool cached = S->lu[0] && S->adj_key[0] == S->state_ver &&
                        S->adj_key[1] == S->val_ver && S->adj_key[2] == S->lu0_ver;
    if (!cached) {
        V2D_TRY(assemble_now(S, urot, false));
        V2D_TRY(sync_flag(S, "adjoint assembly"));
        if (!S->plan) {
            v2d_krylov_params keep = S->prm.krylov;
            S->prm.krylov.precond = V2D_PC_LU;
            const int st = ensure_lu(S);
            S->prm.krylov = keep;
            V2D_TRY(st);
        }
        if (!S->lu[0]) V2D_TRY(mf_factor_create(S->plan, 0, 0, &S->lu[0]));
        V2D_TRY(mf_factor(S->plan, S->lu[0], g.rowptr, g.val, S->s));
        ++S->lu0_ver;
        S->lu_valid = false;   // lu[0] no longer holds the Newton solve's factors
        S->adj_key[0] = S->state_ver;
        S->adj_key[1] = S->val_ver;
        S->adj_key[2] = S->lu0_ver;
    }
    V2D_TRY(ensure_transpose(S));
    const size_t n = g.n;
    // J^T on the transposed pattern, solved by GMRES(30) in FP64 with the
    // transposed LU solve as the preconditioner: with factors whose pivoting
    // stays inside 32-row blocks, the plain iterative refinement x += (LU)^-T r
    // stalls on wide fronts; GMRES converges in a few iterations instead
    if (!S->valT) V2D_CUDA_TRY(cudaMalloc(&S->valT, (size_t)g.nnz * sizeof(double)));
    if (!S->kw_adj) V2D_TRY(krylov_create(&S->kw_adj, g.n, kAdjRestart, S->s));
    k_gather_vals<<<grid_for(g.nnz, 256), 256, 0, S->s>>>(g.nnz, S->tperm, g.val, S->valT);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    if (!S->adj_vec) V2D_CUDA_TRY(cudaMalloc(&S->adj_vec, 3 * n * sizeof(double)));
    double *dg = S->adj_vec, *lam = dg + n, *jtl = lam + n;
    V2D_CUDA_TRY(cudaMemcpyAsync(dg, g_host, n * sizeof(double), cudaMemcpyHostToDevice, S->s));
    CsrOp AT;
    AT.n = g.n;
    AT.nnz = g.nnz;
    AT.rowptr = S->tptr;
    AT.colind = S->tind;
    AT.val = S->valT;
    AT.layout = 0;
    AT.nblk = g.n;
    AT.lu_plan = S->plan;
    AT.lu = S->lu[0];
    AT.lu_transpose = true;
    v2d_krylov_params kp;
    v2d_krylov_defaults(&kp);
    kp.restart = kAdjRestart;
    kp.max_it = kAdjRestart * max_refine;
    kp.rtol = rtol;
    kp.atol = 0.0;
    kp.precond = V2D_PC_LU;
    kp.precision = V2D_PREC_FP64;
    v2d_lin_stats ls{};
    V2D_TRY(krylov_solve(S->kw_adj, AT, dg, lam, kp, &ls, S->s));
    // the true residual g - J^T lambda, on the original pattern
    const int grid = grid_for(n, 256);
    k_spmv_t<<<grid, 256, 0, S->s>>>(g.n, S->tptr, S->tind, S->tperm, g.val, lam, jtl);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    std::vector<double> hr(n), hg(g_host, g_host + n);
    V2D_CUDA_TRY(cudaMemcpyAsync(hr.data(), jtl, n * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(lam_host, lam, n * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    for (size_t i = 0; i < n; ++i) hr[i] = hg[i] - hr[i];
    const double gn = host_norm(hg);
    const double rel = gn > 0.0 ? host_norm(hr) / gn : 0.0;
    if (!std::isfinite(rel)) {
        set_error("solver_adjoint: non-finite residual");
        return V2D_ENONFINITE;
    }
    if (refinements) *refinements = ls.iterations;
    if (rel_res) *rel_res = rel;
    if (rel > rtol && rel > 1e-8) {
        set_error("solver_adjoint: residual %.3e after %d GMRES iterations", rel, ls.iterations);
        return V2D_ENOTCONVERGED;
    }
    return V2D_OK;
}

extern "C" int v2d_solver_nnz(const v2d_solver *S, long long *nnz)
{
    V2D_ARG_CHECK(S && nnz, "null pointer");
    *nnz = S->g.nnz;
    return V2D_OK;
}

extern "C" int v2d_solver_export_system(v2d_solver *S, int *indptr, int *indices, double *data,
                                        double *b)
{
    V2D_ARG_CHECK(S, "null solver");
    const GridDev &g = S->g;
    if (indptr)
        V2D_CUDA_TRY(cudaMemcpyAsync(indptr, g.rowptr, (g.n + 1) * sizeof(int), cudaMemcpyDeviceToHost, S->s));
    if (indices)
        V2D_CUDA_TRY(cudaMemcpyAsync(indices, g.colind, g.nnz * sizeof(int), cudaMemcpyDeviceToHost, S->s));
    if (data)
        V2D_CUDA_TRY(cudaMemcpyAsync(data, g.val, g.nnz * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    if (b) V2D_CUDA_TRY(cudaMemcpyAsync(b, g.b, g.n * sizeof(double), cudaMemcpyDeviceToHost, S->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    return V2D_OK;
}

extern "C" int v2d_solver_state_ptrs(v2d_solver *S, double **psi, double **ome, double **omeold,
                                     double **omeoldold)
{
    V2D_ARG_CHECK(S, "null solver");
    if (psi) *psi = S->g.psi;
    if (ome) *ome = S->g.ome;
    if (omeold) *omeold = S->g.omeold;
    if (omeoldold) *omeoldold = S->g.omeoldold;
    return V2D_OK;
}

extern "C" int v2d_solver_time_spmv(v2d_solver *S, int fp32, int reps, long long flush_bytes,
                                    double *ms_avg)
{
    V2D_ARG_CHECK(S && ms_avg && reps > 0 && flush_bytes >= 0, "time_spmv: bad arguments");
    GridDev &g = S->g;
    CsrOp A;
    A.n = g.n; A.nnz = g.nnz; A.rowptr = g.rowptr; A.colind = g.colind; A.val = g.val;
    A.val32 = g.val32; A.layout = 1; A.nblk = g.N;
    return time_spmv(A, fp32 != 0, reps, (size_t)flush_bytes, S->s, ms_avg);
}

extern "C" int v2d_solver_phase_times(v2d_solver *S, double *out6, int reset)
{
    V2D_ARG_CHECK(S && out6, "null pointer");
    double *out5 = out6;
    for (int q = 0; q < 4; ++q) out5[q] = S->phase_ms[q];
    out5[4] = (double)S->phase_n;
    out5[5] = (double)S->lu_factorizations;
    if (reset) {
        for (double &v : S->phase_ms) v = 0.0;
        S->phase_n = 0;
        S->lu_factorizations = 0;
    }
    return V2D_OK;
}

extern "C" int v2d_solver_time_lu_apply(v2d_solver *S, int reps, long long flush_bytes,
                                        double *ms_avg, long long *factor_bytes)
{
    V2D_ARG_CHECK(S && ms_avg && factor_bytes && reps > 0 && flush_bytes >= 0,
                  "time_lu_apply: bad arguments");
    V2D_ARG_CHECK(S->prm.krylov.precond == V2D_PC_LU && S->plan,
                  "time_lu_apply: the handle does not use the LU preconditioner");
    const int q = S->prm.krylov.precision == V2D_PREC_MIXED ? 1 : 0;
    V2D_ARG_CHECK(S->lu[q] && S->lu_ready, "time_lu_apply: no factors yet (run a Newton iteration)");
    *factor_bytes = S->plan->apply_entries * (long long)(q ? sizeof(float) : sizeof(double));
    return mf_time_apply(S->plan, S->lu[q], reps, (size_t)flush_bytes, S->s, ms_avg);
}

extern "C" int v2d_solver_lu_stats(v2d_solver *S, double *out6)
{
    V2D_ARG_CHECK(S && out6, "lu_stats: bad arguments");
    V2D_ARG_CHECK(S->prm.krylov.precond == V2D_PC_LU && S->plan,
                  "lu_stats: the handle does not use the LU preconditioner");
    const MfPlan *P = S->plan;
    out6[0] = P->nfront;
    out6[1] = P->nlevel;
    out6[2] = (double)P->ftotal;
    out6[3] = P->factor_flops;
    out6[4] = (double)P->apply_entries;
    out6[5] = P->nitems;
    return V2D_OK;
}

extern "C" int v2d_solver_time_lu_launches(v2d_solver *S, int reps, long long flush_bytes,
                                           double *ms, int *codes, int cap, int *n)
{
    V2D_ARG_CHECK(S && ms && codes && n && reps > 0 && flush_bytes >= 0 && cap > 0,
                  "time_lu_launches: bad arguments");
    V2D_ARG_CHECK(S->prm.krylov.precond == V2D_PC_LU && S->plan,
                  "time_lu_launches: the handle does not use the LU preconditioner");
    const int q = S->prm.krylov.precision == V2D_PREC_MIXED ? 1 : 0;
    V2D_ARG_CHECK(S->lu[q] && S->lu_ready,
                  "time_lu_launches: no current factors (run a Newton iteration first)");
    return mf_time_apply_launches(S->plan, S->lu[q], reps, (size_t)flush_bytes, S->s, ms, codes,
                                  cap, n);
}

extern "C" int v2d_solver_time_lu_factor(v2d_solver *S, int reps, double *ms, int *codes, int cap,
                                         int *n)
{
    V2D_ARG_CHECK(S && ms && codes && n && reps > 0 && cap > 0,
                  "time_lu_factor: bad arguments");
    V2D_ARG_CHECK(S->prm.krylov.precond == V2D_PC_LU && S->plan,
                  "time_lu_factor: the handle does not use the LU preconditioner");
    const int q = S->prm.krylov.precision == V2D_PREC_MIXED ? 1 : 0;
    V2D_ARG_CHECK(S->lu[q] && S->lu_ready,
                  "time_lu_factor: no current factors (run a Newton iteration first)");
    if (q == 0) ++S->lu0_ver;   // refactors lu[0]
    return mf_time_factor_launches(S->plan, S->lu[q], S->g.rowptr, S->g.val, reps, S->s, ms,
                                   codes, cap, n);
}

// Kernel timing (no reference counterpart): average ms of `reps` launches of
// one kernel of the Newton iteration on the handle's current data, each after
// a write of flush_bytes (evicts L2).
extern "C" int v2d_solver_time_kernel(v2d_solver *S, int which, int reps, long long flush_bytes,
                                      double *ms_avg)
{
    V2D_ARG_CHECK(S && ms_avg && reps > 0 && flush_bytes >= 0, "time_kernel: bad arguments");
    V2D_ARG_CHECK(which >= 0 && which <= 3, "time_kernel: unknown kernel %d", which);
    GridDev &g = S->g;
    DevBuf<char> fl;
    V2D_TRY(fl.alloc((size_t)flush_bytes + 16, S->s));
    DevBuf<double> vel;
    if (which == 3) V2D_TRY(vel.alloc(3 * (size_t)g.N, S->s));
    V2D_TRY(ensure_pattern(S));
    const v2d_solver_params &p = S->prm;
    AsmParams ap{p.re, p.invdtau, p.inv2dt, 0.0, p.ca, p.sa, p.ff_bc};
    if (which == 1 || which == 2) ++S->val_ver;   // the timed assembly rewrites the values
    cudaEvent_t e0, e1;
    V2D_CUDA_TRY(cudaEventCreate(&e0));
    V2D_CUDA_TRY(cudaEventCreate(&e1));
    double total = 0.0;
    int st = V2D_OK;
    for (int r = 0; r < reps && st == V2D_OK; ++r) {
        if (flush_bytes) cudaMemsetAsync(fl.p, r & 0xff, (size_t)flush_bytes, S->s);
        cudaEventRecord(e0, S->s);
        if (which == 0) st = launch_metrics(g, S->s);
        else if (which == 1) st = launch_assemble(g, ap, false, S->flag, S->s);
        else if (which == 2) st = launch_assemble(g, ap, true, S->flag, S->s);
        else st = launch_velocity(g.imax, g.jmax, g.dksi, g.deta, g.met[0], g.met[2], g.met[3],
                                  g.met[6], g.met[7], g.psi, vel.p, vel.p + g.N, vel.p + 2 * g.N,
                                  S->s);
        cudaEventRecord(e1, S->s);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = V2D_ECUDA;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != V2D_OK) return st;
    *ms_avg = total / reps;
    S->assembled = false;
    return V2D_OK;
}

extern "C" int v2d_solver_stream(v2d_solver *S, void **stream)
{
    V2D_ARG_CHECK(S && stream, "null pointer");
    *stream = (void *)S->s;
    return V2D_OK;
}
