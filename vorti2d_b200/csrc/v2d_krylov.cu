// Restarted GMRES(m) with right preconditioning, entirely on the device.
//
// Replaces the PETSc KSP GMRES + PCJACOBI solve of the reference's GPU path
// (vorti2d/dist_solver.py:159-172) and the MUMPS solve of the replicated path
// (vorti2d/petsc_solver.py:97-115).  Design:
//
//  * Arnoldi with classical Gram-Schmidt applied twice (CGS2): each pass is
//    one multi-dot kernel (all j+1 projections in one sweep over w) and one
//    update kernel (w -= V h fused with the partial norm).  Sums are two-stage
//    and deterministic: per-block partials, then the last block to finish
//    reduces them in a fixed order (no floating-point atomics).
//  * Hessenberg / Givens / back-substitution live in device memory and are
//    updated by the last block of a reduction, so a whole restart cycle runs
//    without the host; a device control block makes the remaining kernels of
//    a cycle exit at once after convergence or breakdown.
//  * Each cycle is captured once as a few CUDA graphs (Arnoldi segments of
//    growing length + a finishing graph) and replayed; the host checks the
//    control block between segments.
//  * Preconditioners: 2x2 (psi, ome) block Jacobi applied inline, or the
//    multifrontal LU of the current Jacobian (v2d_mf.cu) applied by its own
//    per-level kernels; with LU the preconditioned vectors Z_j = M^-1 v_j are
//    kept (m extra vectors) so the cycle's correction x += Z y needs no
//    further solve.
//  * Precision T = double (plain FP64) or float (FP32 SpMV, preconditioner
//    and Krylov vectors, FP64 dot-product accumulation and Hessenberg).  The
//    true residual b - A x is recomputed in FP64 at every restart, so the
//    FP32 cycles act as inner solves of an FP64 defect correction.
#include <algorithm>
#include <cmath>
#include <vector>

#include "v2d_internal.cuh"

namespace v2d {

constexpr int kMaxRestart = 256;
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 2 * kSMs;
constexpr int kSpmvThreads = 256;
constexpr int kTPR = 4;  // threads per CSR row

struct Ctl {
    double beta;         // ||r|| at the start of the current cycle (FP64 true residual)
    double resid;        // running residual estimate |g_{j+1}|
    double tol_cycle;    // stop the Arnoldi loop once resid <= tol_cycle
    double tol_abs;      // convergence target for the true residual
    double inner_rtol;   // FP32 cycles: relative tolerance per cycle
    double res0;
    int conv;            // converged: every kernel exits
    int cyc_stop;        // the current cycle's Arnoldi loop ended
    int jdone;           // Arnoldi columns completed in this cycle
    int its;             // total Arnoldi iterations
    int max_it;
    int breakdown;
    int cycles;
    int nonfinite;
    int stagnated;       // a cycle failed to halve the residual near the target
    double prev_beta;
    unsigned int cnt[4]; // last-block counters
};

// Operator + vectors of one solve, read by the kernels through a pointer so
// the captured graphs stay valid for any operator of the same size.
struct Desc {
    int n, nblk, layout, m;
    const int *rowptr, *colind;
    const double *val;
    const float *val32;
    const double *dinv;
    const float *dinv32;
    const double *b;
    double *x;
    int precond;
};

struct KrylovWork {
    int n = 0, m = 0;
    cudaStream_t s = 0;
    // FP64 and FP32 Arnoldi bases (allocated on first use of each precision)
    double *V64 = nullptr, *w64 = nullptr, *z64 = nullptr, *Z64 = nullptr;
    float *V32 = nullptr, *w32 = nullptr, *z32 = nullptr, *Z32 = nullptr;
    double *r = nullptr;          // FP64 residual
    double *H = nullptr;          // (m+1) x m column-major
    double *g = nullptr, *cs = nullptr, *sn = nullptr, *y = nullptr, *hcur = nullptr;
    double *partial = nullptr;    // kTileBlocks x (m+2)
    Ctl *ctl = nullptr;
    Ctl *ctl_host = nullptr;      // pinned mirror
    Desc *desc = nullptr;
    std::vector<cudaGraphExec_t> seg[2];   // Arnoldi segments per precision
    std::vector<int> seg_bounds[2];
    std::vector<long long> seg_launches[2];  // kernels per segment replay
    cudaGraphExec_t fin[2] = {nullptr, nullptr};
    int graph_m[2] = {0, 0};
    int graph_pc[2] = {-1, -1};
    const void *graph_lu[2] = {nullptr, nullptr};
    int graph_lu_flow[2] = {-1, -1};   // the LU solve form the graph was captured with
    long long graph_lu_items[2] = {-1, -1};   // and the plan's work-item table
    const double *graph_x[2] = {nullptr, nullptr};   // the solution vector k_correct writes
};

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ bool last_block(unsigned int *counter)
{
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(counter, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

template <class T>
__device__ __forceinline__ const T *vals_of(const Desc *d);
template <>
__device__ __forceinline__ const double *vals_of<double>(const Desc *d) { return d->val; }
template <>
__device__ __forceinline__ const float *vals_of<float>(const Desc *d) { return d->val32; }
template <class T>
__device__ __forceinline__ const T *dinv_of(const Desc *d);
template <>
__device__ __forceinline__ const double *dinv_of<double>(const Desc *d) { return d->dinv; }
template <>
__device__ __forceinline__ const float *dinv_of<float>(const Desc *d) { return d->dinv32; }

// Row indices of 2x2 block q for the layouts of CsrOp.
__device__ __forceinline__ void block_rows(int layout, int nblk, int q, int &r0, int &r1)
{
    if (layout == 1) {
        r0 = q; r1 = q + nblk;
    } else {
        r0 = 2 * q; r1 = 2 * q + 1;
    }
}

// z = M^-1 v on one block (or one row for point Jacobi / none).
template <class T>
__device__ __forceinline__ void precond_block(const Desc *d, int q, const T *v, T *z)
{
    if (d->precond == V2D_PC_LU) return;   // applied by the multifrontal kernels
    if (d->precond == V2D_PC_NONE) {
        z[q] = v[q];
        return;
    }
    const T *di = dinv_of<T>(d);
    const int nb = d->nblk;
    if (d->layout == 0) {
        z[q] = di[q] * v[q];
        return;
    }
    int r0, r1;
    block_rows(d->layout, nb, q, r0, r1);
    T a = v[r0], c = v[r1];
    z[r0] = di[q] * a + di[nb + q] * c;
    z[r1] = di[2 * nb + q] * a + di[3 * nb + q] * c;
}

__device__ __forceinline__ int precond_units(const Desc *d)
{
    return (d->precond != V2D_PC_BJACOBI || d->layout == 0) ? d->n : d->nblk;
}

// ----------------------------------------------------------------- kernels
// Start of Arnoldi step j: v_j = src / scale, z = M^-1 v_j.
//  j == 0: src = FP64 residual r, scale = beta.   j > 0: src = w, scale = H[j, j-1].
template <class T>
__global__ void __launch_bounds__(256) k_scale_precond(const Desc *d, Ctl *ctl, int j, const double *r,
                                                       const T *w, T *V, const double *H, T *z)
{
    if (ctl->conv || ctl->cyc_stop) return;
    const int n = d->n, m = d->m;
    T *vj = V + (size_t)j * n;
    const double scale = j == 0 ? ctl->beta : H[j + (size_t)(j - 1) * (m + 1)];
    const double inv = 1.0 / scale;
    const int units = precond_units(d);
    V2D_GRID_STRIDE(q, units)
    {
        if (d->precond != V2D_PC_BJACOBI || d->layout == 0) {
            int r0 = (int)q;
            vj[r0] = j == 0 ? (T)(r[r0] * inv) : (T)(w[r0] * inv);
        } else {
            int r0, r1;
            block_rows(d->layout, d->nblk, (int)q, r0, r1);
            vj[r0] = j == 0 ? (T)(r[r0] * inv) : (T)((double)w[r0] * inv);
            vj[r1] = j == 0 ? (T)(r[r1] * inv) : (T)((double)w[r1] * inv);
        }
    }
    // precondition after the whole block of v is written by this thread
    V2D_GRID_STRIDE(q, units) { precond_block<T>(d, (int)q, vj, z); }
}

// Entries of a row one lane takes with all its loads issued together: the
// 9-point stencil's rows hold at most 13 entries, kTPR * kSpmvRowRegs = 16.
constexpr int kSpmvRowRegs = 4;

// y = A x, kTPR threads per row, FP32 or FP64 values/vectors.  A lane's
// first kSpmvRowRegs entries load their column indices and values first and
// then the gathered x, so a row's loads overlap instead of chaining index ->
// gather per entry; longer rows finish in a plain loop.  The sum runs over
// the lane's entries in column-position order either way.
template <class T>
__device__ __forceinline__ void spmv_rows(const int *__restrict__ rowptr, const int *__restrict__ colind,
                                          const T *__restrict__ val, const T *__restrict__ x,
                                          T *__restrict__ y, int n)
{
    const int lane = threadIdx.x & (kTPR - 1);
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long total = (long long)n * kTPR;
    const int wl = threadIdx.x & 31;
    // loop bound is uniform across the warp (t - wl is the warp's base), so
    // every lane reaches the shuffles
    for (long long t = tid; t - wl < total; t += stride) {
        const bool valid = t < total;
        int row = valid ? (int)(t / kTPR) : 0;
        T acc = 0;
        if (valid) {
            const int p0 = rowptr[row], p1 = rowptr[row + 1];
            int c[kSpmvRowRegs];
            T v[kSpmvRowRegs], xv[kSpmvRowRegs];
#pragma unroll
            for (int k = 0; k < kSpmvRowRegs; ++k) {
                const int p = p0 + lane + k * kTPR;
                c[k] = p < p1 ? colind[p] : -1;
                v[k] = p < p1 ? val[p] : T(0);
            }
#pragma unroll
            for (int k = 0; k < kSpmvRowRegs; ++k) xv[k] = c[k] >= 0 ? x[c[k]] : T(0);
#pragma unroll
            for (int k = 0; k < kSpmvRowRegs; ++k)
                if (c[k] >= 0) acc += v[k] * xv[k];
            for (int p = p0 + lane + kSpmvRowRegs * kTPR; p < p1; p += kTPR)
                acc += val[p] * x[colind[p]];
        }
#pragma unroll
        for (int o = kTPR / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, kTPR);
        if (valid && lane == 0) y[row] = acc;
    }
}

template <class T>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv(const Desc *d, Ctl *ctl, const T *z, T *w)
{
    if (ctl->conv || ctl->cyc_stop) return;
    spmv_rows<T>(d->rowptr, d->colind, vals_of<T>(d), z, w, d->n);
}

// Multi-dot: hcur[i] = V_i . w, i = 0..j; pass 0 writes H[:, j], pass 1 adds.
// Vectors are processed 8 at a time with register accumulators, so each
// thread keeps 8 independent loads in flight per element of w.
constexpr int kDotChunk = 8;

// Sum of the per-block partials of column `col` (stride ld) by one warp,
// in a fixed order: lane l takes blocks l, l+32, ...; then a warp tree.
__device__ __forceinline__ double warp_sum_partials(const double *partial, int nblk, int ld,
                                                    int col)
{
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += partial[(size_t)b * ld + col];
    return warp_sum(s);
}

// Grid: blockIdx.x = element tile (grid-stride), blockIdx.y = chunk of
// kDotChunk basis vectors; each thread keeps kDotChunk loads in flight.
// Partials land in partial[tile][i]; the last block to finish sums them.
template <class T>
__global__ void __launch_bounds__(kRedThreads) k_mdot(const Desc *d, Ctl *ctl, int j, int pass,
                                                      const T *V, const T *w, double *partial,
                                                      double *H, double *hcur)
{
    if (ctl->conv || ctl->cyc_stop) return;
    __shared__ double red[kDotChunk][kRedThreads / 32];
    const int n = d->n, m = d->m, nj = j + 1;
    const int i0 = blockIdx.y * kDotChunk;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ntiles = gridDim.x;
    double acc[kDotChunk];
#pragma unroll
    for (int q = 0; q < kDotChunk; ++q) acc[q] = 0.0;
    if (i0 < nj) {
        for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
             t += (long long)ntiles * blockDim.x) {
            const double wt = (double)w[t];
#pragma unroll
            for (int q = 0; q < kDotChunk; ++q)
                if (i0 + q < nj) acc[q] += (double)V[(size_t)(i0 + q) * n + t] * wt;
        }
    }
#pragma unroll
    for (int q = 0; q < kDotChunk; ++q) {
        double v = warp_sum(acc[q]);
        if (lane == 0) red[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < kDotChunk && i0 + (int)threadIdx.x < nj) {
        double s = 0.0;
        for (int q = 0; q < kRedThreads / 32; ++q) s += red[threadIdx.x][q];
        partial[(size_t)blockIdx.x * (m + 2) + i0 + threadIdx.x] = s;
    }
    // last block over the whole (x, y) grid reduces every column
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        is_last = atomicAdd(&ctl->cnt[0], 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (is_last) {
        __threadfence();
        double *hc = H + (size_t)j * (m + 1);
        for (int i = wid; i < nj; i += kRedThreads / 32) {
            double sum = warp_sum_partials(partial, ntiles, m + 2, i);
            if (lane == 0) {
                hcur[i] = sum;
                hc[i] = pass == 0 ? sum : hc[i] + sum;
            }
        }
        if (threadIdx.x == 0) ctl->cnt[0] = 0;
    }
}

// w -= V hcur; partial ||w||^2.  On the final pass the last block completes
// the Arnoldi column: H[j+1, j] = ||w||, Givens rotation, residual estimate.
template <class T>
__global__ void __launch_bounds__(kRedThreads) k_update(const Desc *d, Ctl *ctl, int j, int final_pass,
                                                        const T *V, T *w, double *partial,
                                                        double *H, const double *hcur, double *g,
                                                        double *cs, double *sn)
{
    if (ctl->conv || ctl->cyc_stop) return;
    __shared__ double hs[kMaxRestart + 1];
    __shared__ double red[32];
    const int n = d->n, m = d->m, nj = j + 1;
    for (int i = threadIdx.x; i < nj; i += blockDim.x) hs[i] = hcur[i];
    __syncthreads();
    double acc = 0.0;
    V2D_GRID_STRIDE(t, n)
    {
        double s = (double)w[t];
#pragma unroll 8
        for (int i = 0; i < nj; ++i) s -= hs[i] * (double)V[(size_t)i * n + t];
        T st = (T)s;
        w[t] = st;
        acc += (double)st * (double)st;
    }
    acc = block_sum(acc, red);
    if (!final_pass) return;
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * (m + 2) + m + 1] = acc;
    if (last_block(&ctl->cnt[1])) {
        double s = 0.0;
        if (threadIdx.x < 32) s = warp_sum_partials(partial, gridDim.x, m + 2, m + 1);
        if (threadIdx.x == 0) {
            double hn = sqrt(s);
            double *hc = H + (size_t)j * (m + 1);
            hc[j + 1] = hn;
            // apply the previous rotations to column j
            for (int i = 0; i < j; ++i) {
                double a = hc[i], bb = hc[i + 1];
                hc[i] = cs[i] * a + sn[i] * bb;
                hc[i + 1] = -sn[i] * a + cs[i] * bb;
            }
            double a = hc[j], bb = hc[j + 1];
            double rr = hypot(a, bb);
            double c = rr > 0.0 ? a / rr : 1.0, sgn = rr > 0.0 ? bb / rr : 0.0;
            cs[j] = c; sn[j] = sgn;
            hc[j] = rr;
            double gj = g[j];
            g[j] = c * gj;
            g[j + 1] = -sgn * gj;
            ctl->resid = fabs(g[j + 1]);
            ctl->jdone = j + 1;
            ctl->its += 1;
            // keep the un-rotated subdiagonal for the next v_{j+1} = w / h
            H[(size_t)j * (m + 1) + (j + 1)] = hn;
            if (!isfinite(ctl->resid) || !isfinite(hn)) {
                ctl->nonfinite = 1;
                ctl->cyc_stop = 1;
            } else if (ctl->resid <= ctl->tol_cycle || ctl->its >= ctl->max_it || j + 1 >= m) {
                ctl->cyc_stop = 1;
            } else if (hn <= 1e-300 || hn <= 1e-14 * rr) {
                ctl->breakdown = 1;  // (lucky) breakdown: the Krylov space is invariant
                ctl->cyc_stop = 1;
            }
            ctl->cnt[1] = 0;
        }
    }
}

// End of a cycle: back-substitution R y = g over the completed columns.
__global__ void k_backsolve(const Desc *d, Ctl *ctl, const double *H, const double *g, double *y)
{
    if (ctl->conv) return;
    if (threadIdx.x != 0) return;
    const int m = d->m, jj = ctl->jdone;
    for (int i = jj - 1; i >= 0; --i) {
        double s = g[i];
        for (int k = i + 1; k < jj; ++k) s -= H[i + (size_t)k * (m + 1)] * y[k];
        double hii = H[i + (size_t)i * (m + 1)];
        y[i] = hii != 0.0 ? s / hii : 0.0;
    }
}

// x += M^-1 (V y), x in FP64.
template <class T>
__global__ void __launch_bounds__(256) k_correct(const Desc *d, Ctl *ctl, const T *V, const double *y,
                                                 T *t_scratch, double *x, const T *Z)
{
    if (ctl->conv) return;
    const int n = d->n, jj = ctl->jdone;
    if (d->precond == V2D_PC_LU) {   // x += Z y
        V2D_GRID_STRIDE(r, n)
        {
            double s = 0.0;
            for (int i = 0; i < jj; ++i) s += y[i] * (double)Z[(size_t)i * n + r];
            x[r] += s;
        }
        return;
    }
    const int units = precond_units(d);
    V2D_GRID_STRIDE(q, units)
    {
        if (d->precond == V2D_PC_NONE || d->layout == 0) {
            int r0 = (int)q;
            double s = 0.0;
            for (int i = 0; i < jj; ++i) s += y[i] * (double)V[(size_t)i * n + r0];
            t_scratch[r0] = (T)s;
        } else {
            int r0, r1;
            block_rows(d->layout, d->nblk, (int)q, r0, r1);
            double s0 = 0.0, s1 = 0.0;
            for (int i = 0; i < jj; ++i) {
                s0 += y[i] * (double)V[(size_t)i * n + r0];
                s1 += y[i] * (double)V[(size_t)i * n + r1];
            }
            t_scratch[r0] = (T)s0;
            t_scratch[r1] = (T)s1;
        }
    }
    // M^-1 on the same units this thread wrote: no grid dependency
    V2D_GRID_STRIDE(q, units)
    {
        if (d->precond == V2D_PC_NONE) {
            x[q] += (double)t_scratch[q];
        } else if (d->layout == 0) {
            x[q] += (double)(dinv_of<T>(d)[q] * t_scratch[q]);
        } else {
            int r0, r1;
            block_rows(d->layout, d->nblk, (int)q, r0, r1);
            const T *di = dinv_of<T>(d);
            const int nb = d->nblk;
            double a = (double)t_scratch[r0], c = (double)t_scratch[r1];
            x[r0] += (double)di[q] * a + (double)di[nb + q] * c;
            x[r1] += (double)di[2 * nb + q] * a + (double)di[3 * nb + q] * c;
        }
    }
}

// FP64 true residual r = b - A x and its norm; the last block decides
// convergence and resets the cycle state.
__global__ void __launch_bounds__(kSpmvThreads) k_residual(const Desc *d, Ctl *ctl, double *r,
                                                           double *partial, double *g, int first)
{
    if (ctl->conv) return;
    __shared__ double red[32];
    const int n = d->n, m = d->m;
    const int lane = threadIdx.x & (kTPR - 1);
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    double acc = 0.0;
    const long long total = (long long)n * kTPR;
    const int wl = threadIdx.x & 31;
    for (long long t = tid; t - wl < total; t += stride) {
        const bool valid = t < total;
        int row = valid ? (int)(t / kTPR) : 0;
        double s = 0.0;
        if (valid && !first) {
            int p0 = d->rowptr[row], p1 = d->rowptr[row + 1];
            for (int p = p0 + lane; p < p1; p += kTPR) s += d->val[p] * d->x[d->colind[p]];
        }
#pragma unroll
        for (int o = kTPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, kTPR);
        if (valid && lane == 0) {
            double rv = d->b[row] - s;
            r[row] = rv;
            acc += rv * rv;
        }
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * (m + 2) + m + 1] = acc;
    if (last_block(&ctl->cnt[2])) {
        double s = 0.0;
        if (threadIdx.x < 32) s = warp_sum_partials(partial, gridDim.x, m + 2, m + 1);
        if (threadIdx.x == 0) {
            double beta = sqrt(s);
            ctl->beta = beta;
            if (first) {
                ctl->res0 = beta;
                ctl->tol_abs = ctl->tol_abs * beta;  // rtol * ||b||
            }
            ctl->resid = beta;
            ctl->cycles += first ? 0 : 1;
            if (!isfinite(beta)) {
                ctl->nonfinite = 1;
                ctl->conv = 1;
            } else if (beta <= ctl->tol_abs || beta == 0.0) {
                ctl->conv = 1;
            } else if (!first && beta > 0.5 * ctl->prev_beta && beta <= 100.0 * ctl->tol_abs) {
                // the FP64 residual has reached the attainable accuracy
                ctl->stagnated = 1;
                ctl->conv = 1;
            } else if (ctl->its >= ctl->max_it || ctl->breakdown) {
                ctl->conv = 1;  // stop: not converged (host reads beta)
            }
            ctl->prev_beta = beta;
            // next cycle
            g[0] = beta;
            for (int i = 1; i <= m; ++i) g[i] = 0.0;
            ctl->jdone = 0;
            ctl->cyc_stop = 0;
            double tc = ctl->tol_abs;
            if (ctl->inner_rtol > 0.0) tc = fmax(tc, ctl->inner_rtol * beta);
            ctl->tol_cycle = tc;
            ctl->cnt[2] = 0;
        }
    }
}

// ------------------------------------------------------------------ host
// Reduction grids: about 8 elements per thread (independent loads in flight),
// at most 2 blocks per SM.
static int red_grid(long long n)
{
    long long g = (n + kRedThreads * 8 - 1) / (kRedThreads * 8);
    return (int)std::max(1LL, std::min<long long>(kRedBlocks, g));
}

// Gram-Schmidt grids: one element per thread up to kTileBlocks blocks
// (latency hiding needs many loads in flight), grid-stride beyond.
constexpr int kTileBlocks = 8 * kSMs;

// FP64 residual grid: one CSR row per kTPR threads up to kTileBlocks blocks
// (each row's index -> vector gather chain is latency bound; a small grid
// would walk tens of rows per thread one after another).
static int res_grid(long long n)
{
    const long long g = (n * kTPR + kSpmvThreads - 1) / kSpmvThreads;
    return (int)std::max(1LL, std::min<long long>(kTileBlocks, g));
}
static int tile_grid(long long n)
{
    long long g = (n + kRedThreads - 1) / kRedThreads;
    return (int)std::max(1LL, std::min<long long>(kTileBlocks, g));
}

// A restart cycle runs as a few captured segments of Arnoldi steps
// ([0,2), [2,6), [6,10), [10,14), then 8 at a time), then a finishing graph
// (back-substitution, correction, FP64 residual).  The host reads the control
// block after each segment and skips the remaining segments once the cycle
// has stopped, so a cycle that converges in a few steps (the usual case with
// the LU preconditioner: 6-12 with factors kept across Newton iterations)
// launches few steps past its last one; each step after the stop is a chain
// of launches that return at once.
static std::vector<int> segment_bounds(int m)
{
    std::vector<int> b{0};
    const int len[] = {2, 4, 4, 4};
    for (int q = 0; b.back() < m; ++q)
        b.push_back(std::min(m, b.back() + (q < 4 ? len[q] : 8)));
    return b;
}

static int end_capture(cudaStream_t s, cudaGraphExec_t *out)
{
    cudaGraph_t gph = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &gph);
    if (e != cudaSuccess) {
        if (gph) cudaGraphDestroy(gph);
        set_error("GMRES graph capture failed: %s", cudaGetErrorString(e));
        return V2D_ECUDA;
    }
    e = cudaGraphInstantiate(out, gph, 0);
    cudaGraphDestroy(gph);
    if (e != cudaSuccess) {
        *out = nullptr;
        set_error("GMRES graph instantiate failed: %s", cudaGetErrorString(e));
        return V2D_ECUDA;
    }
    return V2D_OK;
}

// A launch that fails during a capture invalidates it, and every later call
// reports only "a previous error during capture": each launch is checked as
// it is captured, so the error names the first one that failed.
static bool capture_launch_failed(cudaStream_t s, const char *what, int j)
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return false;
    cudaGraph_t junk = nullptr;
    cudaStreamEndCapture(s, &junk);
    if (junk) cudaGraphDestroy(junk);
    cudaGetLastError();
    set_error("GMRES graph capture: launch of %s (basis column %d) failed: %s", what, j,
              cudaGetErrorString(e));
    return true;
}

static void drop_graphs(KrylovWork *w, int which)
{
    for (cudaGraphExec_t g : w->seg[which])
        if (g) cudaGraphExecDestroy(g);
    w->seg[which].clear();
    if (w->fin[which]) cudaGraphExecDestroy(w->fin[which]);
    w->fin[which] = nullptr;
}

// The LU solve a captured cycle launches: -1 none, -2 the transposed solve,
// else 1000 * split level + 10 * (dataflow) + kernel form.
static int lu_form(const CsrOp &A)
{
    if (!A.lu) return -1;
    return A.lu_transpose ? -2 : 1000 * A.lu->split + 10 * A.lu->flow + A.lu->flow_form;
}

template <class T>
static int capture_cycle(KrylovWork *w, int which, T *V, T *wv, T *z, T *Z, double *x,
                         const CsrOp &A, int precond, cudaStream_t s)
{
    const int n = w->n;
    const int gp = grid_for(n, 256);
    const int gs = grid_for((long long)n * kTPR, kSpmvThreads);
    const int gr = red_grid(n);
    const int gt = tile_grid(n);
    const bool lu = precond == V2D_PC_LU;
    drop_graphs(w, which);
    w->seg_launches[which].clear();
    const std::vector<int> bnd = segment_bounds(w->m);
    for (size_t q = 0; q + 1 < bnd.size(); ++q) {
        long long nl = 0;
        V2D_CUDA_TRY(cudaGetLastError());
        V2D_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int j = bnd[q]; j < bnd[q + 1]; ++j) {
            nl += 6;
            k_scale_precond<T><<<gp, 256, 0, s>>>(w->desc, w->ctl, j, w->r, wv, V, w->H, z);
            if (capture_launch_failed(s, "k_scale_precond", j)) return V2D_ECUDA;
            T *zj = z;
            if (lu) {
                zj = Z + (size_t)j * n;
                long long na = 0;
                int st = A.lu_transpose
                             ? mf_apply_transpose(A.lu_plan, const_cast<MfFactor *>(A.lu),
                                                  V + (size_t)j * n, zj, s, &na)
                             : mf_apply(A.lu_plan, A.lu, V + (size_t)j * n, zj, &w->ctl->conv,
                                        &w->ctl->cyc_stop, s, &na);
                nl += na;
                if (st != V2D_OK) {
                    cudaGraph_t junk = nullptr;
                    cudaStreamEndCapture(s, &junk);
                    if (junk) cudaGraphDestroy(junk);
                    return st;
                }
            }
            k_spmv<T><<<gs, kSpmvThreads, 0, s>>>(w->desc, w->ctl, zj, wv);
            if (capture_launch_failed(s, "k_spmv", j)) return V2D_ECUDA;
            const dim3 gdot(gt, (j + 1 + kDotChunk - 1) / kDotChunk);
            for (int pass = 0; pass < 2; ++pass) {
                k_mdot<T><<<gdot, kRedThreads, 0, s>>>(w->desc, w->ctl, j, pass, V, wv, w->partial,
                                                       w->H, w->hcur);
                if (capture_launch_failed(s, "k_mdot", j)) return V2D_ECUDA;
                k_update<T><<<gt, kRedThreads, 0, s>>>(w->desc, w->ctl, j, pass, V, wv, w->partial,
                                                       w->H, w->hcur, w->g, w->cs, w->sn);
                if (capture_launch_failed(s, "k_update", j)) return V2D_ECUDA;
            }
        }
        cudaGraphExec_t ge = nullptr;
        V2D_TRY(end_capture(s, &ge));
        w->seg[which].push_back(ge);
        w->seg_launches[which].push_back(nl);
    }
    V2D_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    k_backsolve<<<1, 32, 0, s>>>(w->desc, w->ctl, w->H, w->g, w->y);
    k_correct<T><<<gp, 256, 0, s>>>(w->desc, w->ctl, V, w->y, z, x, Z);
    k_residual<<<res_grid(n), kSpmvThreads, 0, s>>>(w->desc, w->ctl, w->r, w->partial, w->g, 0);
    V2D_TRY(end_capture(s, &w->fin[which]));
    w->seg_bounds[which] = bnd;
    w->graph_m[which] = w->m;
    w->graph_pc[which] = precond;
    w->graph_lu[which] = lu ? (const void *)A.lu : nullptr;
    w->graph_lu_flow[which] = lu_form(A);
    w->graph_lu_items[which] = lu ? A.lu_plan->items_ver : -1;
    w->graph_x[which] = x;
    return V2D_OK;
}

// One restart cycle; *h receives the control block at its end.
template <class T>
static int run_cycle(KrylovWork *w, int which, T *V, T *wv, T *z, T *Z, double *x, const CsrOp &A,
                     int precond, cudaStream_t s, Ctl *h)
{
    const bool lu = precond == V2D_PC_LU;
    if (w->seg[which].empty() || !w->fin[which] || w->graph_m[which] != w->m ||
        w->graph_pc[which] != precond ||
        w->graph_lu[which] != (lu ? (const void *)A.lu : nullptr) ||
        w->graph_lu_flow[which] != lu_form(A) ||
        w->graph_lu_items[which] != (lu ? A.lu_plan->items_ver : -1) ||
        w->graph_x[which] != x)
        V2D_TRY(capture_cycle<T>(w, which, V, wv, z, Z, x, A, precond, s));
    for (size_t q = 0; q < w->seg[which].size(); ++q) {
        V2D_CUDA_TRY(cudaGraphLaunch(w->seg[which][q], s));
        count_launches(w->seg_launches[which][q]);
        V2D_CUDA_TRY(cudaMemcpyAsync(w->ctl_host, w->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
        V2D_CUDA_TRY(cudaStreamSynchronize(s));
        if (w->ctl_host->cyc_stop || w->ctl_host->conv) break;
    }
    V2D_CUDA_TRY(cudaGraphLaunch(w->fin[which], s));
    count_launches(3);
    V2D_CUDA_TRY(cudaMemcpyAsync(w->ctl_host, w->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    *h = *w->ctl_host;
    return V2D_OK;
}

int krylov_create(KrylovWork **out, int n, int restart, cudaStream_t s)
{
    V2D_ARG_CHECK(n > 0 && restart >= 1 && restart <= kMaxRestart,
                  "krylov: n=%d restart=%d (restart must be in [1, %d])", n, restart, kMaxRestart);
    KrylovWork *w = new KrylovWork();
    w->n = n;
    w->m = restart;
    w->s = s;
    const int m = restart;
    cudaError_t e = cudaSuccess;
    auto grab = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    grab((void **)&w->r, (size_t)n * sizeof(double));
    grab((void **)&w->H, (size_t)(m + 1) * m * sizeof(double));
    grab((void **)&w->g, (size_t)(m + 1) * sizeof(double));
    grab((void **)&w->cs, (size_t)m * sizeof(double));
    grab((void **)&w->sn, (size_t)m * sizeof(double));
    grab((void **)&w->y, (size_t)m * sizeof(double));
    grab((void **)&w->hcur, (size_t)(m + 1) * sizeof(double));
    grab((void **)&w->partial, (size_t)kTileBlocks * (m + 2) * sizeof(double));
    grab((void **)&w->ctl, sizeof(Ctl));
    grab((void **)&w->desc, sizeof(Desc));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&w->ctl_host, sizeof(Ctl));
    if (e == cudaSuccess) e = cudaMemsetAsync(w->ctl, 0, sizeof(Ctl), s);
    if (e != cudaSuccess) {
        set_error("krylov workspace allocation failed: %s", cudaGetErrorString(e));
        krylov_destroy(w);
        return V2D_ENOMEM;
    }
    *out = w;
    return V2D_OK;
}

void krylov_destroy(KrylovWork *w)
{
    if (!w) return;
    for (int q = 0; q < 2; ++q) drop_graphs(w, q);
    void *ptrs[] = {w->V64, w->w64, w->z64, w->Z64, w->V32, w->w32, w->z32, w->Z32, w->r, w->H, w->g,
                    w->cs, w->sn, w->y, w->hcur, w->partial, w->ctl, w->desc};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (w->ctl_host) cudaFreeHost(w->ctl_host);
    delete w;
}

static int ensure_basis(KrylovWork *w, bool fp32, bool lu)
{
    const size_t n = w->n, m = w->m;
    if (lu && fp32 && !w->Z32) V2D_CUDA_TRY(cudaMalloc(&w->Z32, m * n * sizeof(float)));
    if (lu && !fp32 && !w->Z64) V2D_CUDA_TRY(cudaMalloc(&w->Z64, m * n * sizeof(double)));
    if (fp32 && !w->V32) {
        V2D_CUDA_TRY(cudaMalloc(&w->V32, (m + 1) * n * sizeof(float)));
        V2D_CUDA_TRY(cudaMalloc(&w->w32, n * sizeof(float)));
        V2D_CUDA_TRY(cudaMalloc(&w->z32, n * sizeof(float)));
    }
    if (!fp32 && !w->V64) {
        V2D_CUDA_TRY(cudaMalloc(&w->V64, (m + 1) * n * sizeof(double)));
        V2D_CUDA_TRY(cudaMalloc(&w->w64, n * sizeof(double)));
        V2D_CUDA_TRY(cudaMalloc(&w->z64, n * sizeof(double)));
    }
    return V2D_OK;
}

int krylov_solve(KrylovWork *w, const CsrOp &A, const double *d_b, double *d_x,
                 const v2d_krylov_params &prm, v2d_lin_stats *st, cudaStream_t s)
{
    V2D_ARG_CHECK(A.n == w->n, "krylov_solve: operator size %d != workspace size %d", A.n, w->n);
    V2D_ARG_CHECK(prm.restart == w->m, "krylov_solve: restart changed (%d != %d)", prm.restart, w->m);
    const bool fp32 = prm.precision == V2D_PREC_MIXED;
    const bool lu = prm.precond == V2D_PC_LU;
    V2D_ARG_CHECK(!fp32 || (A.val32 && (A.dinv32 || prm.precond != V2D_PC_BJACOBI)),
                  "krylov_solve: mixed precision needs FP32 values");
    V2D_ARG_CHECK(!lu || (A.lu && A.lu_plan && A.lu->fp32 == (fp32 ? 1 : 0)),
                  "krylov_solve: LU preconditioner needs factors in the Krylov precision");
    V2D_TRY(ensure_basis(w, fp32, lu));
    Desc hd;
    hd.n = A.n; hd.nblk = A.nblk; hd.layout = A.layout; hd.m = w->m;
    hd.rowptr = A.rowptr; hd.colind = A.colind; hd.val = A.val; hd.val32 = A.val32;
    hd.dinv = A.dinv; hd.dinv32 = A.dinv32; hd.b = d_b; hd.x = d_x;
    hd.precond = (prm.precond == V2D_PC_BJACOBI || prm.precond == V2D_PC_LU) ? prm.precond
                                                                              : V2D_PC_NONE;
    V2D_CUDA_TRY(cudaMemcpyAsync(w->desc, &hd, sizeof(Desc), cudaMemcpyHostToDevice, s));
    Ctl c{};
    c.tol_abs = prm.rtol;  // scaled by ||b|| in the first residual pass (atol applied below)
    c.max_it = prm.max_it;
    c.inner_rtol = fp32 ? prm.inner_rtol : 0.0;
    V2D_CUDA_TRY(cudaMemcpyAsync(w->ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    V2D_CUDA_TRY(cudaMemsetAsync(d_x, 0, (size_t)A.n * sizeof(double), s));
    const int gr = red_grid(A.n);
    k_residual<<<res_grid(A.n), kSpmvThreads, 0, s>>>(w->desc, w->ctl, w->r, w->partial, w->g, 1);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    // atol: tol_abs = max(rtol * ||b||, atol) -- applied on the host after the first pass
    V2D_CUDA_TRY(cudaMemcpyAsync(w->ctl_host, w->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    Ctl h = *w->ctl_host;
    if (!h.conv && prm.atol > h.tol_abs) {
        double ta = prm.atol;
        V2D_CUDA_TRY(cudaMemcpyAsync(&w->ctl->tol_abs, &ta, sizeof(double), cudaMemcpyHostToDevice, s));
        if (h.beta <= ta) h.conv = 1;
    }
    int guard = 0;
    while (!h.conv) {
        int status = fp32 ? run_cycle<float>(w, 1, w->V32, w->w32, w->z32, w->Z32, d_x, A,
                                             hd.precond, s, &h)
                          : run_cycle<double>(w, 0, w->V64, w->w64, w->z64, w->Z64, d_x, A,
                                              hd.precond, s, &h);
        if (status != V2D_OK) return status;
        if (++guard > 1000000) break;
    }
    const bool converged = (h.beta <= fmax(h.tol_abs, prm.atol) || h.stagnated) && !h.nonfinite;
    if (st) {
        st->iterations = h.its;
        st->restarts = h.cycles;
        st->corrections = fp32 ? h.cycles : 0;
        st->converged = converged ? 1 : 0;
        st->res0 = h.res0;
        st->res = h.beta;
    }
    if (h.nonfinite) {
        set_error("GMRES: non-finite residual (iteration %d)", h.its);
        return V2D_ENONFINITE;
    }
    return V2D_OK;
}

// ------------------------------------------------------ SpMV timing hook
__global__ void k_spmv_plain64(CsrOp A, const double *x, double *y)
{
    spmv_rows<double>(A.rowptr, A.colind, A.val, x, y, A.n);
}
__global__ void k_spmv_plain32(CsrOp A, const float *x, float *y)
{
    spmv_rows<float>(A.rowptr, A.colind, A.val32, x, y, A.n);
}
__global__ void k_fill_bytes(unsigned int *p, size_t n, unsigned int v)
{
    V2D_GRID_STRIDE(t, n) { p[t] = v + (unsigned int)t; }
}

// Average duration (ms) of `reps` launches of the Krylov SpMV kernel on this
// operator, each launched after a write of `flush_bytes` (evicts L2), timed
// with events on stream s.
int time_spmv(const CsrOp &A, bool fp32, int reps, size_t flush_bytes, cudaStream_t s,
              double *ms_avg)
{
    DevBuf<char> buf;
    const size_t vec = (size_t)A.n * (fp32 ? sizeof(float) : sizeof(double));
    V2D_TRY(buf.alloc(2 * vec + flush_bytes + 256, s));
    V2D_CUDA_TRY(cudaMemsetAsync(buf.p, 0, 2 * vec, s));
    unsigned int *fl = (unsigned int *)(buf.p + 2 * vec + 128 - ((uintptr_t)(buf.p + 2 * vec) % 128));
    const size_t nfl = flush_bytes / sizeof(unsigned int);
    cudaEvent_t e0, e1;
    V2D_CUDA_TRY(cudaEventCreate(&e0));
    V2D_CUDA_TRY(cudaEventCreate(&e1));
    const int gs = grid_for((long long)A.n * kTPR, kSpmvThreads);
    double total = 0.0;
    for (int r = 0; r < reps; ++r) {
        if (nfl) k_fill_bytes<<<grid_for(nfl, 256), 256, 0, s>>>(fl, nfl, (unsigned)r);
        cudaEventRecord(e0, s);
        if (fp32)
            k_spmv_plain32<<<gs, kSpmvThreads, 0, s>>>(A, (const float *)buf.p, (float *)(buf.p + vec));
        else
            k_spmv_plain64<<<gs, kSpmvThreads, 0, s>>>(A, (const double *)buf.p, (double *)(buf.p + vec));
        cudaEventRecord(e1, s);
        V2D_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
    }
    count_launches(2LL * reps);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_avg = total / reps;
    return V2D_OK;
}

// ------------------------------------------------- generic block inverse
__global__ void k_block_inverse(CsrOp A, double *dinv, float *dinv32, int *flag)
{
    V2D_GRID_STRIDE(q, A.nblk)
    {
        auto get = [&](int r, int c) {
            double v = 0.0;
            for (int p = A.rowptr[r]; p < A.rowptr[r + 1]; ++p)
                if (A.colind[p] == c) v += A.val[p];
            return v;
        };
        if (A.layout == 0) {
            double a = get((int)q, (int)q);
            double i0 = (a != 0.0) ? 1.0 / a : 0.0;
            if (a == 0.0) atomicOr(flag, 1);
            dinv[q] = i0;
            if (dinv32) dinv32[q] = (float)i0;
            continue;
        }
        int r0, r1;
        if (A.layout == 1) {
            r0 = (int)q; r1 = (int)q + A.nblk;
        } else {
            r0 = 2 * (int)q; r1 = 2 * (int)q + 1;
        }
        double a00 = get(r0, r0), a01 = get(r0, r1), a10 = get(r1, r0), a11 = get(r1, r1);
        double det = a00 * a11 - a01 * a10;
        double i00 = 0, i01 = 0, i10 = 0, i11 = 0;
        if (det != 0.0 && isfinite(det)) {
            double r = 1.0 / det;
            i00 = a11 * r; i01 = -a01 * r; i10 = -a10 * r; i11 = a00 * r;
        } else {
            atomicOr(flag, 1);
        }
        const int nb = A.nblk;
        dinv[q] = i00; dinv[nb + q] = i01; dinv[2 * nb + q] = i10; dinv[3 * nb + q] = i11;
        if (dinv32) {
            dinv32[q] = (float)i00; dinv32[nb + q] = (float)i01;
            dinv32[2 * nb + q] = (float)i10; dinv32[3 * nb + q] = (float)i11;
        }
    }
}

int launch_block_inverse(CsrOp &A, double *dinv, float *dinv32, int *d_flag, cudaStream_t s)
{
    k_block_inverse<<<grid_for(A.nblk, 256), 256, 0, s>>>(A, dinv, dinv32, d_flag);
    V2D_CUDA_TRY(cudaGetLastError());
    return V2D_OK;
}

}  // namespace v2d
