// Batched steady solves: many O-grid instances of uneven sizes (cylinders,
// airfoil sections; each with its own Reynolds number, angle of attack and
// far-field BC) advanced by Newton together, one launch per phase.
//
// The instances' Newton systems are the diagonal blocks of one block-diagonal
// system.  Per Newton iteration:
//   assembly     one launch over a ragged table of instances (assemble_batch):
//                each writes its values into its slice of the combined CSR;
//                a frozen instance (converged or given up) writes identity
//                rows with a zero right-hand side;
//   factor       the multifrontal LU of the block-diagonal matrix over the
//                forest of all instances' separator trees (mf_plan_forest):
//                the same level-by-level launches as one instance, each
//                processing every instance's fronts of that level;
//   Krylov       GMRES(m) on the combined system: one SpMV, one dataflow
//                solve of the forest and the same Arnoldi kernels per
//                iteration.  With a direct-solve-quality preconditioner on
//                every block the combined iteration converges as the worst
//                block does; each instance's rows are scaled by the inverse
//                norm of its right-hand side first, so the relative tolerance
//                holds per instance;
//   update       one launch: q_i += dq_i and ||dq_i|| / (2 N_i) per instance
//                (deterministic two-stage sums), the reference's Newton
//                measure (vorti2d/solver.py:117-145).
// The host reads one residual per instance per iteration and decides which
// instances go on.
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "v2d_internal.cuh"

using namespace v2d;

namespace {

constexpr int kBatchUpd = 256;   // nodes per update block

// dq -> q for active instances; per block the sum of the squared updates of
// its nodes (psi and ome).  Block kb belongs to instance i with
// ublk0[i] <= kb < ublk0[i + 1].
__global__ void __launch_bounds__(kBatchUpd) k_batch_update(
    int ninst, const int *__restrict__ ublk0, const int *__restrict__ nodes,
    const int *__restrict__ row_off, double *const *psi, double *const *ome,
    const int *__restrict__ active, const double *__restrict__ dq, double *partial)
{
    __shared__ double red[32];
    const int kb = blockIdx.x;
    int lo = 0, hi = ninst;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (ublk0[mid] <= kb) lo = mid;
        else hi = mid;
    }
    const int N = nodes[lo], K = (kb - ublk0[lo]) * kBatchUpd + threadIdx.x;
    double s = 0.0;
    if (active[lo] && K < N) {
        const double dp = dq[row_off[lo] + K], dw = dq[row_off[lo] + N + K];
        psi[lo][K] += dp;
        ome[lo][K] += dw;
        s = dp * dp + dw * dw;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) partial[kb] = s;
}

// Per instance the sum of its block partials, in block order (one warp per
// instance): mode 0 writes res[i] = sqrt(sum) / (2 N_i), the Newton measure;
// mode 1 the row scale 1 / sqrt(sum) of its block (1 for a zero or
// non-finite sum).
__global__ void k_batch_sums(int ninst, const int *__restrict__ ublk0,
                             const int *__restrict__ nodes, const double *__restrict__ partial,
                             int mode, double *out)
{
    const int i = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (i >= ninst) return;
    double s = 0.0;
    for (int k = ublk0[i] + lane; k < ublk0[i + 1]; k += 32) s += partial[k];
    s = warp_sum(s);
    if (lane != 0) return;
    if (mode == 0) {
        out[i] = sqrt(s) / (2.0 * nodes[i]);
    } else {
        const double nb = sqrt(s);
        out[i] = (nb > 0.0 && isfinite(nb)) ? 1.0 / nb : 1.0;
    }
}

// Row scaling of each instance's block by 1 / ||b_i||_2 (1 for a zero or
// frozen block), so that one relative tolerance on the combined system is
// the same relative tolerance on every block: per block the squared norm of
// its right-hand side (block kb as in the update), then the scaling of the
// rows' values and right-hand side.
__global__ void __launch_bounds__(kBatchUpd) k_batch_bnorm(int ninst, const int *__restrict__ ublk0,
                                                           const int *__restrict__ nodes,
                                                           const int *__restrict__ row_off,
                                                           const double *__restrict__ b,
                                                           double *partial)
{
    __shared__ double red[32];
    const int kb = blockIdx.x;
    int lo = 0, hi = ninst;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (ublk0[mid] <= kb) lo = mid;
        else hi = mid;
    }
    const int N = nodes[lo], K = (kb - ublk0[lo]) * kBatchUpd + threadIdx.x;
    double s = 0.0;
    if (K < N) {
        const double a = b[row_off[lo] + K], c = b[row_off[lo] + N + K];
        s = a * a + c * c;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) partial[kb] = s;
}

__global__ void k_batch_scale(int n, const int *__restrict__ rowptr,
                              const int *__restrict__ row_inst, const double *__restrict__ scale,
                              double *val, float *val32, double *b)
{
    V2D_GRID_STRIDE(t, n)
    {
        const int r = (int)t;
        const double sc = scale[row_inst[r]];
        for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) {
            val[p] *= sc;
            if (val32) val32[p] = (float)val[p];
        }
        b[r] *= sc;
    }
}

}  // namespace

struct v2d_batch {
    int ninst = 0, n = 0;
    long long nnz = 0;
    std::vector<v2d_solver *> inst;
    std::vector<int> row_off, active;
    std::vector<long long> nnz_off;
    v2d_krylov_params kp{};
    bool mixed = false;
    cudaStream_t s = nullptr;
    int *rowptr = nullptr, *colind = nullptr, *row_inst = nullptr;
    double *val = nullptr, *b = nullptr, *x = nullptr;
    float *val32 = nullptr;
    BatchInst *d_inst = nullptr;
    int *d_blk0 = nullptr, *d_ublk0 = nullptr, *d_nodes = nullptr, *d_rowoff = nullptr;
    int *d_active = nullptr, *d_flags = nullptr;
    double **d_psi = nullptr, **d_ome = nullptr;
    double *d_partial = nullptr, *d_res = nullptr, *d_scale = nullptr;
    int nblk = 0, nublk = 0;
    MfPlan *plan = nullptr;
    MfFactor *lu = nullptr;
    KrylovWork *kw = nullptr;
    bool lu_valid = false;
    int lu_last_its = 0;
    long long factorizations = 0;
};

extern "C" int v2d_batch_destroy(v2d_batch *B)
{
    if (!B) return V2D_OK;
    if (B->s) cudaStreamSynchronize(B->s);
    krylov_destroy(B->kw);
    mf_factor_destroy(B->lu);
    mf_plan_destroy(B->plan);
    void *ptrs[] = {B->rowptr, B->colind, B->row_inst, B->val, B->b, B->x, B->val32,
                    B->d_inst, B->d_blk0, B->d_ublk0, B->d_nodes, B->d_rowoff, B->d_active,
                    B->d_flags, B->d_psi, B->d_ome, B->d_partial, B->d_res, B->d_scale};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (v2d_solver *S : B->inst) v2d_solver_destroy(S);
    if (B->s) cudaStreamDestroy(B->s);
    delete B;
    return V2D_OK;
}

template <class T>
static int upload(T **d, const std::vector<T> &h, cudaStream_t s)
{
    V2D_CUDA_TRY(cudaMalloc((void **)d, std::max<size_t>(h.size(), 1) * sizeof(T)));
    if (!h.empty())
        V2D_CUDA_TRY(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return V2D_OK;
}

static int batch_build(v2d_batch *B, int ninst, const int *imax, const int *jmax,
                       const double *const *xg, const double *const *yg,
                       const v2d_solver_params *params)
{
    B->ninst = ninst;
    B->kp = params[0].krylov;
    B->mixed = B->kp.precision == V2D_PREC_MIXED;
    V2D_ARG_CHECK(B->kp.precond == V2D_PC_LU, "batch_create: the batch needs the LU preconditioner");
    V2D_CUDA_TRY(cudaStreamCreateWithFlags(&B->s, cudaStreamNonBlocking));
    // the instances: mesh, metrics, state and CSR pattern on the device (their
    // own Krylov and LU machinery is not used)
    std::vector<std::vector<int>> rp(ninst), ci(ninst);
    std::vector<MfPlan *> parts(ninst, nullptr);
    int st = V2D_OK;
    for (int i = 0; i < ninst && st == V2D_OK; ++i) {
        v2d_solver_params p = params[i];
        p.krylov = B->kp;
        p.krylov.precond = V2D_PC_BJACOBI;
        p.krylov.restart = 1;
        v2d_solver *S = nullptr;
        st = v2d_solver_create(imax[i], jmax[i], xg[i], yg[i], &p, &S);
        if (st != V2D_OK) break;
        B->inst.push_back(S);
        const GridDev &g = S->g;
        rp[i].resize(g.n + 1);
        ci[i].resize(g.nnz);
        if (cudaMemcpy(rp[i].data(), g.rowptr, (g.n + 1) * sizeof(int), cudaMemcpyDeviceToHost) !=
                cudaSuccess ||
            cudaMemcpy(ci[i].data(), g.colind, g.nnz * sizeof(int), cudaMemcpyDeviceToHost) !=
                cudaSuccess) {
            set_error("batch_create: pattern copy failed");
            st = V2D_ECUDA;
            break;
        }
        const int leaf = B->kp.lu_leaf > 0 ? B->kp.lu_leaf : 64;
        st = mf_plan_build(imax[i], jmax[i], g.n, rp[i].data(), ci[i].data(), leaf, &parts[i]);
    }
    if (st == V2D_OK) {
        B->row_off.resize(ninst);
        B->nnz_off.resize(ninst);
        int n = 0;
        long long nnz = 0;
        for (int i = 0; i < ninst; ++i) {
            B->row_off[i] = n;
            B->nnz_off[i] = nnz;
            n += B->inst[i]->g.n;
            nnz += B->inst[i]->g.nnz;
        }
        if (nnz > INT_MAX) {
            set_error("batch_create: %lld nonzeros exceed the 32-bit CSR index", nnz);
            st = V2D_EARG;
        }
        B->n = n;
        B->nnz = nnz;
    }
    if (st == V2D_OK) st = mf_plan_forest(parts, B->row_off, B->nnz_off, B->n, &B->plan);
    for (MfPlan *Q : parts) mf_plan_destroy(Q);
    V2D_TRY(st);
    // the combined CSR pattern and the instance tables
    std::vector<int> grp(B->n + 1), gci(B->nnz), rinst(B->n), blk0(ninst + 1), ublk0(ninst + 1);
    std::vector<int> nodes(ninst);
    std::vector<BatchInst> tab(ninst);
    std::vector<double *> psi(ninst), ome(ninst);
    int nb = 0, nub = 0;
    for (int i = 0; i < ninst; ++i) {
        const GridDev &g = B->inst[i]->g;
        const int ro = B->row_off[i];
        const long long no = B->nnz_off[i];
        for (int r = 0; r < g.n; ++r) {
            grp[ro + r] = (int)(rp[i][r] + no);
            rinst[ro + r] = i;
        }
        for (long long e = 0; e < g.nnz; ++e) gci[no + e] = ci[i][e] + ro;
        blk0[i] = nb;
        nb += (g.N + kAsmNodesHost - 1) / kAsmNodesHost;
        ublk0[i] = nub;
        nub += (g.N + kBatchUpd - 1) / kBatchUpd;
        nodes[i] = g.N;
        const v2d_solver_params &p = params[i];
        BatchInst &I = tab[i];
        I.T = GlobalTopo{g.imax, g.jmax, g.N};
        I.c = Coeffs{p.re, p.invdtau, p.inv2dt, 0.0, g.dksi, g.deta, p.ca, p.sa, p.ff_bc};
        I.f.jac = g.met[0]; I.f.alfa = g.met[1]; I.f.beta = g.met[2]; I.f.gama = g.met[3];
        I.f.pmet = g.met[4]; I.f.qmet = g.met[5]; I.f.detadx = g.met[6]; I.f.detady = g.met[7];
        I.f.xphys = g.met[8]; I.f.yphys = g.met[9];
        I.f.psi = g.psi; I.f.ome = g.ome; I.f.omeold = g.omeold; I.f.omeoldold = g.omeoldold;
        I.rowptr = g.rowptr;
        I.colind = g.colind;
        I.nnz_off = no;
        I.row_off = ro;
        psi[i] = g.psi;
        ome[i] = g.ome;
    }
    grp[B->n] = (int)B->nnz;
    blk0[ninst] = nb;
    ublk0[ninst] = nub;
    B->nblk = nb;
    B->nublk = nub;
    B->active.assign(ninst, 1);
    cudaStream_t s = B->s;
    V2D_TRY(upload(&B->rowptr, grp, s));
    V2D_TRY(upload(&B->colind, gci, s));
    V2D_TRY(upload(&B->row_inst, rinst, s));
    V2D_TRY(upload(&B->d_blk0, blk0, s));
    V2D_TRY(upload(&B->d_ublk0, ublk0, s));
    V2D_TRY(upload(&B->d_nodes, nodes, s));
    V2D_TRY(upload(&B->d_rowoff, B->row_off, s));
    V2D_TRY(upload(&B->d_active, B->active, s));
    V2D_TRY(upload(&B->d_inst, tab, s));
    V2D_TRY(upload(&B->d_psi, psi, s));
    V2D_TRY(upload(&B->d_ome, ome, s));
    V2D_CUDA_TRY(cudaMalloc(&B->val, B->nnz * sizeof(double)));
    if (B->mixed) V2D_CUDA_TRY(cudaMalloc(&B->val32, B->nnz * sizeof(float)));
    V2D_CUDA_TRY(cudaMalloc(&B->b, (size_t)B->n * sizeof(double)));
    V2D_CUDA_TRY(cudaMalloc(&B->x, (size_t)B->n * sizeof(double)));
    V2D_CUDA_TRY(cudaMalloc(&B->d_flags, ninst * sizeof(int)));
    V2D_CUDA_TRY(cudaMalloc(&B->d_partial, (size_t)nub * sizeof(double)));
    V2D_CUDA_TRY(cudaMalloc(&B->d_res, ninst * sizeof(double)));
    V2D_CUDA_TRY(cudaMalloc(&B->d_scale, ninst * sizeof(double)));
    V2D_TRY(mf_factor_create(B->plan, B->mixed ? 1 : 0, B->kp.lu_factor64, &B->lu));
    B->lu->flow = B->kp.lu_solve == 0 ? 1 : 0;
    V2D_TRY(krylov_create(&B->kw, B->n, B->kp.restart, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    return V2D_OK;
}

extern "C" int v2d_batch_create(int ninst, const int *imax, const int *jmax,
                                const double *const *xg, const double *const *yg,
                                const v2d_solver_params *params, v2d_batch **out)
{
    V2D_ARG_CHECK(out && imax && jmax && xg && yg && params, "batch_create: null pointer");
    *out = nullptr;
    V2D_ARG_CHECK(ninst >= 1, "batch_create: %d instances", ninst);
    for (int i = 0; i < ninst; ++i)
        V2D_ARG_CHECK(params[i].ff_bc >= 0 && params[i].ff_bc <= 2 && params[i].re > 0.0,
                      "batch_create: instance %d: ff_bc %d, re %g", i, params[i].ff_bc,
                      params[i].re);
    v2d_batch *B = new v2d_batch();
    const int st = batch_build(B, ninst, imax, jmax, xg, yg, params);
    if (st != V2D_OK) {
        v2d_batch_destroy(B);
        return st;
    }
    *out = B;
    return V2D_OK;
}

extern "C" int v2d_batch_set_active(v2d_batch *B, const int *active)
{
    V2D_ARG_CHECK(B && active, "batch_set_active: null pointer");
    for (int i = 0; i < B->ninst; ++i) B->active[i] = active[i] ? 1 : 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(B->d_active, B->active.data(), B->ninst * sizeof(int),
                                 cudaMemcpyHostToDevice, B->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(B->s));
    return V2D_OK;
}

extern "C" int v2d_batch_instance(v2d_batch *B, int i, v2d_solver **out)
{
    V2D_ARG_CHECK(B && out && i >= 0 && i < B->ninst, "batch_instance: bad argument");
    *out = B->inst[i];
    return V2D_OK;
}

extern "C" int v2d_batch_newton(v2d_batch *B, double *res, int *flags, v2d_lin_stats *st)
{
    V2D_ARG_CHECK(B && res, "batch_newton: null pointer");
    cudaStream_t s = B->s;
    const int ni = B->ninst;
    // the instances' states may have been changed through their handles
    for (v2d_solver *S : B->inst) V2D_CUDA_TRY(cudaStreamSynchronize(S->s));
    V2D_CUDA_TRY(cudaMemsetAsync(B->d_flags, 0, ni * sizeof(int), s));
    V2D_TRY(launch_assemble_batch(B->d_inst, ni, B->d_blk0, B->nblk, B->d_active, B->mixed,
                                  B->val, B->val32, B->b, B->d_flags, s));
    std::vector<int> hf(ni);
    V2D_CUDA_TRY(cudaMemcpyAsync(hf.data(), B->d_flags, ni * sizeof(int), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    bool bad = false;
    for (int i = 0; i < ni; ++i) {
        if (flags) flags[i] = hf[i];
        bad = bad || (hf[i] & 6);
    }
    if (bad) {
        set_error("batch_newton: non-finite right-hand side or pattern mismatch in an instance "
                  "(flags per instance)");
        return V2D_ENONFINITE;
    }
    // each block's rows scaled by 1 / ||b_i||: the relative tolerance then
    // holds block by block (tightened by sqrt of the active blocks, whose
    // unit right-hand sides add up in the combined norm)
    const int wgrid = (ni + 7) / 8;
    k_batch_bnorm<<<B->nublk, kBatchUpd, 0, s>>>(ni, B->d_ublk0, B->d_nodes, B->d_rowoff, B->b,
                                                  B->d_partial);
    k_batch_sums<<<wgrid, 256, 0, s>>>(ni, B->d_ublk0, B->d_nodes, B->d_partial, 1, B->d_scale);
    k_batch_scale<<<grid_for(B->n, 256), 256, 0, s>>>(B->n, B->rowptr, B->row_inst, B->d_scale,
                                                       B->val, B->val32, B->b);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(3);
    int nact = 0;
    for (int a : B->active) nact += a;
    CsrOp A;
    A.n = B->n; A.nnz = B->nnz; A.rowptr = B->rowptr; A.colind = B->colind; A.val = B->val;
    A.val32 = B->val32; A.layout = 1; A.nblk = B->n / 2;
    A.lu_plan = B->plan;
    A.lu = B->lu;
    v2d_krylov_params kp = B->kp;
    kp.rtol = B->kp.rtol / std::sqrt((double)std::max(1, nact));
    bool refactor = !(kp.lu_reuse_its > 0 && B->lu_valid && B->lu_last_its <= kp.lu_reuse_its);
    v2d_lin_stats ls{};
    if (refactor) {
        V2D_TRY(mf_factor(B->plan, B->lu, B->rowptr, B->val, s));
        ++B->factorizations;
        V2D_TRY(krylov_solve(B->kw, A, B->b, B->x, kp, &ls, s));
    } else {
        v2d_krylov_params k2 = kp;
        k2.max_it = std::min(kp.max_it, kp.lu_reuse_its + 5);
        V2D_TRY(krylov_solve(B->kw, A, B->b, B->x, k2, &ls, s));
        V2D_TRY(mf_check_barrier(B->lu, s));
        if (!ls.converged) {
            const int its0 = ls.iterations;
            V2D_TRY(mf_factor(B->plan, B->lu, B->rowptr, B->val, s));
            ++B->factorizations;
            refactor = true;
            V2D_TRY(krylov_solve(B->kw, A, B->b, B->x, kp, &ls, s));
            ls.iterations += its0;
        }
    }
    V2D_TRY(mf_check_barrier(B->lu, s));
    B->lu_valid = true;
    B->lu_last_its = refactor ? 0 : ls.iterations;
    if (st) *st = ls;
    k_batch_update<<<B->nublk, kBatchUpd, 0, s>>>(ni, B->d_ublk0, B->d_nodes, B->d_rowoff,
                                                   B->d_psi, B->d_ome, B->d_active, B->x,
                                                   B->d_partial);
    k_batch_sums<<<wgrid, 256, 0, s>>>(ni, B->d_ublk0, B->d_nodes, B->d_partial, 0, B->d_res);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(2);
    V2D_CUDA_TRY(cudaMemcpyAsync(res, B->d_res, ni * sizeof(double), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    for (v2d_solver *S : B->inst) {
        ++S->state_ver;
        S->assembled = false;
    }
    if (!ls.converged) {
        set_error("batch_newton: GMRES did not converge (%d iterations, |r|/|b| = %.3e)",
                  ls.iterations, ls.res0 > 0 ? ls.res / ls.res0 : 0.0);
        return V2D_ENOTCONVERGED;
    }
    return V2D_OK;
}

extern "C" int v2d_batch_factorizations(const v2d_batch *B, long long *n)
{
    V2D_ARG_CHECK(B && n, "null pointer");
    *n = B->factorizations;
    return V2D_OK;
}
