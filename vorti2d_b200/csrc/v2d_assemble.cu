// Newton-system assembly into a fixed canonical CSR (built with -fmad=false).
//
// The reference assembles COO triplets every iteration and converts them to
// CSR on the host (vorti2d/petsc_solver.py:76-95); here the pattern is built
// once per mesh on the device and each Newton iteration writes values straight
// into their canonical slots: one thread per node computes the psi row and
// the ome row (vorti2d_core.f90:247-381), places each entry at
// rowptr[row] + (rank of its column in the row), writes b, the optional FP32
// copy and the 2x2 (psi_k, ome_k) block inverse used by block Jacobi.
#include "v2d_internal.cuh"
#include "v2d_stencil.cuh"

namespace v2d {

static Fields fields_of(const GridDev &g)
{
    Fields f;
    f.jac = g.met[0]; f.alfa = g.met[1]; f.beta = g.met[2]; f.gama = g.met[3];
    f.pmet = g.met[4]; f.qmet = g.met[5]; f.detadx = g.met[6]; f.detady = g.met[7];
    f.xphys = g.met[8]; f.yphys = g.met[9];
    f.psi = g.psi; f.ome = g.ome; f.omeold = g.omeold; f.omeoldold = g.omeoldold;
    return f;
}

__global__ void metrics_grid_kernel(int imax, int jmax, double dksi, double deta,
                                    const double *__restrict__ x, const double *__restrict__ y,
                                    double *jac, double *alfa, double *beta, double *gama,
                                    double *pmet, double *qmet, double *detadx, double *detady,
                                    double *xp, double *yp)
{
    const int N = imax * jmax;
    V2D_GRID_STRIDE(t, N)
    {
        int K = (int)t;
        int j = K / imax, i = K - j * imax;
        Nbr nb = wrap_neighbors(i, j, imax);
        MetricOut m = metrics_at(x, y, K, nb.e, nb.w, j, jmax, imax, dksi, deta);
        jac[K] = m.jac; alfa[K] = m.alfa; beta[K] = m.beta; gama[K] = m.gama;
        pmet[K] = m.pmet; qmet[K] = m.qmet; detadx[K] = m.detadx; detady[K] = m.detady;
        xp[K] = x[K]; yp[K] = y[K];
    }
}

int launch_metrics(GridDev &g, cudaStream_t s)
{
    metrics_grid_kernel<<<grid_for(g.N, 256), 256, 0, s>>>(
        g.imax, g.jmax, g.dksi, g.deta, g.x, g.y, g.met[0], g.met[1], g.met[2], g.met[3],
        g.met[4], g.met[5], g.met[6], g.met[7], g.met[8], g.met[9]);
    V2D_CUDA_TRY(cudaGetLastError());
    return V2D_OK;
}

__global__ void pattern_count(GlobalTopo T, Coeffs c, Fields f, int *cnt)
{
    V2D_GRID_STRIDE(t, 2 * T.N)
    {
        int r = (int)t;
        cnt[r] = r < T.N ? psi_row_count(T, c, f, r) : ome_row_count(T, c, f, r - T.N);
    }
}

__global__ void pattern_fill(GlobalTopo T, Coeffs c, Fields f, const int *__restrict__ rowptr,
                             int *colind)
{
    V2D_GRID_STRIDE(t, 2 * T.N)
    {
        int r = (int)t;
        int col[kOmeMax];
        int n = r < T.N ? psi_row<false>(T, c, f, r, col, nullptr, nullptr)
                        : ome_row<false>(T, c, f, r - T.N, col, nullptr, nullptr);
        int base = rowptr[r];
        for (int e = 0; e < n; ++e) colind[base + col_rank<kOmeMax>(col, n, e)] = col[e];
    }
}

int build_pattern(GridDev &g, const AsmParams &p, cudaStream_t s)
{
    GlobalTopo T{g.imax, g.jmax, g.N};
    Coeffs c{p.re, p.invdtau, p.inv2dt, p.urot, g.dksi, g.deta, p.ca, p.sa, p.ff_bc};
    Fields f = fields_of(g);
    DevBuf<int> scratch;
    V2D_TRY(scratch.alloc(scan_scratch_ints(g.n) + 1, s));
    pattern_count<<<grid_for(g.n, 256), 256, 0, s>>>(T, c, f, g.rowptr);
    V2D_CUDA_TRY(cudaGetLastError());
    V2D_TRY(exclusive_scan_i32(g.rowptr, g.rowptr, g.n, g.rowptr + g.n, scratch.p, s));
    int nnz = 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(&nnz, g.rowptr + g.n, sizeof(int), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    g.nnz = nnz;
    if (g.colind) cudaFree(g.colind);
    if (g.val) cudaFree(g.val);
    if (g.val32) cudaFree(g.val32);
    g.colind = nullptr; g.val = nullptr; g.val32 = nullptr;
    V2D_CUDA_TRY(cudaMalloc(&g.colind, (size_t)nnz * sizeof(int)));
    V2D_CUDA_TRY(cudaMalloc(&g.val, (size_t)nnz * sizeof(double)));
    V2D_CUDA_TRY(cudaMalloc(&g.val32, (size_t)nnz * sizeof(float)));
    pattern_fill<<<grid_for(g.n, 256), 256, 0, s>>>(T, c, f, g.rowptr, g.colind);
    V2D_CUDA_TRY(cudaGetLastError());
    return V2D_OK;
}

// One thread per node: psi row K and ome row N+K.  A block's 128 nodes own a
// contiguous range of the value array for their psi rows and another for
// their ome rows; each thread places its entries at their canonical slots in
// a shared-memory copy of the range, and the block then writes the range with
// coalesced stores (one row per thread would scatter every warp store over
// 32 rows).
constexpr int kAsmNodes = kAsmNodesHost;

// One block of kAsmNodes nodes starting at node K0 (blockDim.x == kAsmNodes).
template <bool W32>
__device__ __forceinline__ void assemble_block(const GlobalTopo &T, const Coeffs &c,
                                               const Fields &f, const int *__restrict__ rowptr,
                                               double *__restrict__ val,
                                               float *__restrict__ val32,
                                               double *__restrict__ b, double *__restrict__ dinv,
                                               float *__restrict__ dinv32, int *flag, int K0,
                                               double *stage)
{
    const int N = T.N;
    {
        const int K = K0 + threadIdx.x;
        const bool live = K < N;
        const int K1 = min(K0 + kAsmNodes, N);
        int col[kOmeMax];
        double v[kOmeMax];
        double bk = 0.0;
        double a00 = 0, a01 = 0, a10 = 0, a11 = 0;
        // psi rows
        const int pbeg = rowptr[K0], pend = rowptr[K1];
        if (live) {
            int n = psi_row<true>(T, c, f, K, col, v, &bk);
            const int base = rowptr[K] - pbeg;
            if (n != rowptr[K + 1] - rowptr[K]) {   // pattern out of date: write nothing
                atomicOr(flag, 4);
                n = 0;
            }
#pragma unroll
            for (int e = 0; e < kPsiMax; ++e) {
                if (e < n) {
                    stage[base + col_rank<kPsiMax>(col, n, e)] = v[e];
                    if (col[e] == K) a00 += v[e];
                    if (col[e] == N + K) a01 += v[e];
                }
            }
            b[K] = bk;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < pend - pbeg; e += kAsmNodes) {
            const double x = stage[e];
            val[pbeg + e] = x;
            if (W32) val32[pbeg + e] = (float)x;
        }
        __syncthreads();
        // ome rows
        const int obeg = rowptr[N + K0], oend = rowptr[N + K1];
        if (live) {
            int n = ome_row<true>(T, c, f, K, col, v, &bk);
            const int base = rowptr[N + K] - obeg;
            if (n != rowptr[N + K + 1] - rowptr[N + K]) {
                atomicOr(flag, 4);
                n = 0;
            }
#pragma unroll
            for (int e = 0; e < kOmeMax; ++e) {
                if (e < n) {
                    stage[base + col_rank<kOmeMax>(col, n, e)] = v[e];
                    if (col[e] == K) a10 += v[e];
                    if (col[e] == N + K) a11 += v[e];
                }
            }
            b[N + K] = bk;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < oend - obeg; e += kAsmNodes) {
            const double x = stage[e];
            val[obeg + e] = x;
            if (W32) val32[obeg + e] = (float)x;
        }
        __syncthreads();
        if (live && dinv) {
            // 2x2 block inverse for block Jacobi
            double det = a00 * a11 - a01 * a10;
            double i00, i01, i10, i11;
            if (det != 0.0 && isfinite(det)) {
                double r = 1.0 / det;
                i00 = a11 * r; i01 = -a01 * r; i10 = -a10 * r; i11 = a00 * r;
            } else {
                i00 = i01 = i10 = i11 = 0.0;
                atomicOr(flag, 1);
            }
            dinv[K] = i00; dinv[N + K] = i01; dinv[2 * N + K] = i10; dinv[3 * N + K] = i11;
            if (W32) {
                dinv32[K] = (float)i00; dinv32[N + K] = (float)i01;
                dinv32[2 * N + K] = (float)i10; dinv32[3 * N + K] = (float)i11;
            }
        }
        if (live && !isfinite(bk)) atomicOr(flag, 2);
    }
}

template <bool W32>
__global__ void __launch_bounds__(kAsmNodes) assemble_newton(GlobalTopo T, Coeffs c, Fields f,
                                                             const int *__restrict__ rowptr,
                                                             double *__restrict__ val,
                                                             float *__restrict__ val32,
                                                             double *__restrict__ b,
                                                             double *__restrict__ dinv,
                                                             float *__restrict__ dinv32, int *flag)
{
    __shared__ double stage[kAsmNodes * kOmeMax];
    for (int K0 = blockIdx.x * kAsmNodes; K0 < T.N; K0 += gridDim.x * kAsmNodes)
        assemble_block<W32>(T, c, f, rowptr, val, val32, b, dinv, dinv32, flag, K0, stage);
}

// Many instances' Newton systems in one launch (the batched sweep): block
// kb belongs to the instance i with blk0[i] <= kb < blk0[i + 1] and covers its
// nodes from (kb - blk0[i]) * kAsmNodes.  An active instance assembles into
// its slices of the combined value and right-hand side arrays; a frozen one
// (converged or given up) writes identity rows with a zero right-hand side,
// so its update is zero and the combined pattern stays fixed.  flags[i] gets
// the instance's assembly flags (bit 1: non-finite right-hand side).
template <bool W32>
__global__ void __launch_bounds__(kAsmNodes) assemble_batch(const BatchInst *__restrict__ inst,
                                                            int ninst, const int *__restrict__ blk0,
                                                            const int *__restrict__ active,
                                                            double *val, float *val32, double *b,
                                                            int *flags)
{
    __shared__ double stage[kAsmNodes * kOmeMax];
    const int kb = blockIdx.x;
    int lo = 0, hi = ninst;   // largest i with blk0[i] <= kb
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (blk0[mid] <= kb) lo = mid;
        else hi = mid;
    }
    const BatchInst I = inst[lo];
    const int K0 = (kb - blk0[lo]) * kAsmNodes;
    double *v = val + I.nnz_off;
    float *v32 = W32 ? val32 + I.nnz_off : nullptr;
    double *bb = b + I.row_off;
    if (active[lo]) {
        assemble_block<W32>(I.T, I.c, I.f, I.rowptr, v, v32, bb, nullptr, nullptr, flags + lo,
                            K0, stage);
        return;
    }
    const int N = I.T.N, K = K0 + threadIdx.x;
    if (K >= N) return;
    for (int r : {K, N + K}) {
        for (int p = I.rowptr[r]; p < I.rowptr[r + 1]; ++p) {
            const double x = I.colind[p] == r ? 1.0 : 0.0;
            v[p] = x;
            if (W32) v32[p] = (float)x;
        }
        bb[r] = 0.0;
    }
}

int launch_assemble_batch(const BatchInst *d_inst, int ninst, const int *d_blk0, int nblocks,
                          const int *d_active, bool want32, double *val, float *val32, double *b,
                          int *d_flags, cudaStream_t s)
{
    if (want32)
        assemble_batch<true><<<nblocks, kAsmNodes, 0, s>>>(d_inst, ninst, d_blk0, d_active, val,
                                                           val32, b, d_flags);
    else
        assemble_batch<false><<<nblocks, kAsmNodes, 0, s>>>(d_inst, ninst, d_blk0, d_active, val,
                                                            val32, b, d_flags);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    return V2D_OK;
}

// Right-hand side b = -R of the Newton system only (no Jacobian values), for
// scalar parameters that may differ from the handle's: the parameter
// derivatives of the residual used by the adjoint.
__global__ void __launch_bounds__(128) residual_only(GlobalTopo T, Coeffs c, Fields f,
                                                     double *__restrict__ b)
{
    V2D_GRID_STRIDE(t, T.N)
    {
        const int K = (int)t;
        int col[kOmeMax];
        double v[kOmeMax];
        double bk;
        psi_row<true>(T, c, f, K, col, v, &bk);
        b[K] = bk;
        ome_row<true>(T, c, f, K, col, v, &bk);
        b[T.N + K] = bk;
    }
}

int launch_residual(const GridDev &g, const AsmParams &p, double *d_b, cudaStream_t s)
{
    GlobalTopo T{g.imax, g.jmax, g.N};
    Coeffs c{p.re, p.invdtau, p.inv2dt, p.urot, g.dksi, g.deta, p.ca, p.sa, p.ff_bc};
    Fields f = fields_of(g);
    residual_only<<<grid_for(g.N, 128), 128, 0, s>>>(T, c, f, d_b);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    return V2D_OK;
}

int launch_assemble(GridDev &g, const AsmParams &p, bool want32, int *d_flag, cudaStream_t s)
{
    GlobalTopo T{g.imax, g.jmax, g.N};
    Coeffs c{p.re, p.invdtau, p.inv2dt, p.urot, g.dksi, g.deta, p.ca, p.sa, p.ff_bc};
    Fields f = fields_of(g);
    int grid = grid_for(g.N, kAsmNodes);
    if (want32)
        assemble_newton<true><<<grid, kAsmNodes, 0, s>>>(T, c, f, g.rowptr, g.val, g.val32, g.b,
                                                         g.dinv, g.dinv32, d_flag);
    else
        assemble_newton<false><<<grid, kAsmNodes, 0, s>>>(T, c, f, g.rowptr, g.val, g.val32, g.b,
                                                          g.dinv, g.dinv32, d_flag);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    return V2D_OK;
}

}  // namespace v2d
