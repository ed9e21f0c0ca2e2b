// Kernel seam: the five routines of the reference's f2py module
// (src/fortran/vorti2d_core.f90:24-25) as sm_100a kernels plus host entry
// points with the f2py argument order.  Built with -fmad=false: the values are
// bit-identical to the CPU restatement of the Fortran.
#include <mutex>

#include "v2d_stencil.cuh"
#include "v2d_util.cuh"

namespace v2d {

// --------------------------------------------------------------- metrics
// One thread per node, i fastest: each warp reads 32 consecutive x/y values
// per stencil tap; the +-1 column taps of the cross derivative hit the same
// cache lines.  Output: 10 SoA arrays in pointer order.
__global__ void __launch_bounds__(256) metrics_global_kernel(int imax, int jmax, double dksi,
                                                             double deta, const double *__restrict__ x,
                                                             const double *__restrict__ y,
                                                             double *const *out)
{
    const int N = imax * jmax;
    V2D_GRID_STRIDE(t, N)
    {
        int K = (int)t;
        int j = K / imax, i = K - j * imax;
        Nbr nb = wrap_neighbors(i, j, imax);
        MetricOut m = metrics_at(x, y, K, nb.e, nb.w, j, jmax, imax, dksi, deta);
        out[0][K] = m.jac; out[1][K] = m.alfa; out[2][K] = m.beta; out[3][K] = m.gama;
        out[4][K] = m.pmet; out[5][K] = m.qmet; out[6][K] = m.detadx; out[7][K] = m.detady;
        out[8][K] = x[K]; out[9][K] = y[K];
    }
}

// Ghosted local block (vorti2d_core.f90:392-495): owned 0-based columns
// [c0, c1]; everything outside is zero except the coordinates.
__global__ void __launch_bounds__(256) metrics_local_kernel(int gxm, int jmax, int c0, int c1,
                                                            double dksi, double deta,
                                                            const double *__restrict__ x,
                                                            const double *__restrict__ y,
                                                            double *const *out)
{
    const int N = gxm * jmax;
    V2D_GRID_STRIDE(t, N)
    {
        int K = (int)t;
        int j = K / gxm, il = K - j * gxm;
        if (il >= c0 && il <= c1) {
            MetricOut m = metrics_at(x, y, K, K + 1, K - 1, j, jmax, gxm, dksi, deta);
            out[0][K] = m.jac; out[1][K] = m.alfa; out[2][K] = m.beta; out[3][K] = m.gama;
            out[4][K] = m.pmet; out[5][K] = m.qmet; out[6][K] = m.detadx; out[7][K] = m.detady;
        } else {
            for (int q = 0; q < 8; ++q) out[q][K] = 0.0;
        }
        out[8][K] = x[K]; out[9][K] = y[K];
    }
}

// ----------------------------------------------------- COO (push order)
// Global system: one thread per row r in [r0, r1).  Pass 1 counts, a scan
// gives each row its COO offset (the reference emits rows in ascending order,
// entries in push order within a row), pass 2 writes triplets and b.
__global__ void coo_count_global(GlobalTopo T, Coeffs c, Fields f, int r0, int r1, int *cnt)
{
    V2D_GRID_STRIDE(t, r1 - r0)
    {
        int r = r0 + (int)t;
        cnt[t] = r < T.N ? psi_row_count(T, c, f, r) : ome_row_count(T, c, f, r - T.N);
    }
}

__global__ void coo_fill_global(GlobalTopo T, Coeffs c, Fields f, int r0, int r1,
                                const int *__restrict__ off, int *ci, int *cj, double *cv,
                                double *bvec)
{
    V2D_GRID_STRIDE(t, r1 - r0)
    {
        int r = r0 + (int)t;
        int col[kOmeMax];
        double val[kOmeMax];
        double b;
        int n = r < T.N ? psi_row<true>(T, c, f, r, col, val, &b)
                        : ome_row<true>(T, c, f, r - T.N, col, val, &b);
        int o = off[t];
        for (int e = 0; e < n; ++e) {
            ci[o + e] = r;
            cj[o + e] = col[e];
            cv[o + e] = val[e];
        }
        bvec[t] = b;
    }
}

// Local system: the reference loops jj, then owned il, emitting the psi row
// then the ome row of each node (vorti2d_core.f90:535-652).  One thread per
// owned node; offsets come from a scan of (psi count + ome count).
__global__ void coo_count_local(LocalTopo T, Coeffs c, Fields f, int c0, int nown, int *cnt)
{
    V2D_GRID_STRIDE(t, (long long)nown * T.jmax)
    {
        int j = (int)(t / nown), il = c0 + (int)(t - (long long)j * nown);
        int K = j * T.gxm + il;
        cnt[t] = psi_row_count(T, c, f, K) + ome_row_count(T, c, f, K);
    }
}

__global__ void coo_fill_local(LocalTopo T, Coeffs c, Fields f, int c0, int nown, int r0,
                               int nloc, const int *__restrict__ off, int *ci, int *cj,
                               double *cv, double *bvec, int *bad_row)
{
    V2D_GRID_STRIDE(t, (long long)nown * T.jmax)
    {
        int j = (int)(t / nown), il = c0 + (int)(t - (long long)j * nown);
        int K = j * T.gxm + il;
        int col[kOmeMax];
        double val[kOmeMax];
        double b;
        int o = off[t];
        for (int comp = 0; comp < 2; ++comp) {
            int row = T.dof(K, comp);
            int n = comp == 0 ? psi_row<true>(T, c, f, K, col, val, &b)
                              : ome_row<true>(T, c, f, K, col, val, &b);
            for (int e = 0; e < n; ++e) {
                ci[o + e] = row;
                cj[o + e] = col[e];
                cv[o + e] = val[e];
            }
            o += n;
            if (row - r0 >= 0 && row - r0 < nloc)
                bvec[row - r0] = b;
            else
                atomicExch(bad_row, 1);
        }
    }
}

// ------------------------------------------------------------ host helpers
struct HostCopy {
    static int up(double *d, const double *h, size_t n, cudaStream_t s)
    {
        V2D_CUDA_TRY(cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, s));
        return V2D_OK;
    }
};

static int check_finite_mesh(int imax, int jmax)
{
    V2D_ARG_CHECK(imax >= 4 && jmax >= 4, "mesh must be at least 4x4 (got %d x %d)", imax, jmax);
    V2D_ARG_CHECK((long long)imax * jmax < (1LL << 30), "mesh too large");
    return V2D_OK;
}

}  // namespace v2d

using namespace v2d;

extern "C" int v2d_node_neighbors(int i, int j, int imax, int *out9)
{
    V2D_ARG_CHECK(out9 && imax >= 3 && i >= 1 && i <= imax && j >= 1,
                  "node_neighbors: bad arguments (i=%d j=%d imax=%d)", i, j, imax);
    Nbr b = wrap_neighbors(i - 1, j - 1, imax);
    int v[9] = {b.k, b.e, b.w, b.n, b.s, b.ne, b.nw, b.se, b.sw};
    for (int q = 0; q < 9; ++q) out9[q] = v[q] + 1;
    return V2D_OK;
}

extern "C" int v2d_compute_metrics_dev(int imax, int jmax, double dksi, double deta,
                                       const double *d_xg, const double *d_yg,
                                       double *const *d_out10, void *stream)
{
    V2D_TRY(check_finite_mesh(imax, jmax));
    V2D_ARG_CHECK(d_xg && d_yg && d_out10, "compute_metrics_dev: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf<double *> outp;
    V2D_TRY(outp.alloc(10, s));
    V2D_CUDA_TRY(cudaMemcpyAsync(outp.p, d_out10, 10 * sizeof(double *), cudaMemcpyHostToDevice, s));
    int N = imax * jmax;
    metrics_global_kernel<<<grid_for(N, 256), 256, 0, s>>>(imax, jmax, dksi, deta, d_xg, d_yg,
                                                            outp.p);
    V2D_CUDA_TRY(cudaGetLastError());
    return V2D_OK;
}

static int metrics_host(bool local, int gxm, int jmax, int c0, int c1, double dksi, double deta,
                        const double *xg, const double *yg, double *const *hout)
{
    cudaStream_t s = 0;
    const size_t N = (size_t)gxm * jmax;
    DevBuf<double> buf;
    V2D_TRY(buf.alloc(12 * N, s));
    double *dx = buf.p, *dy = buf.p + N;
    double *dout[10];
    for (int q = 0; q < 10; ++q) dout[q] = buf.p + (2 + q) * N;
    V2D_TRY(HostCopy::up(dx, xg, N, s));
    V2D_TRY(HostCopy::up(dy, yg, N, s));
    DevBuf<double *> outp;
    V2D_TRY(outp.alloc(10, s));
    V2D_CUDA_TRY(cudaMemcpyAsync(outp.p, dout, sizeof(dout), cudaMemcpyHostToDevice, s));
    if (local)
        metrics_local_kernel<<<grid_for(N, 256), 256, 0, s>>>(gxm, jmax, c0, c1, dksi, deta, dx, dy,
                                                               outp.p);
    else
        metrics_global_kernel<<<grid_for(N, 256), 256, 0, s>>>(gxm, jmax, dksi, deta, dx, dy,
                                                                outp.p);
    V2D_CUDA_TRY(cudaGetLastError());
    for (int q = 0; q < 10; ++q)
        V2D_CUDA_TRY(cudaMemcpyAsync(hout[q], dout[q], N * sizeof(double), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    return V2D_OK;
}

extern "C" int v2d_compute_metrics(int imax, int jmax, double dksi, double deta,
                                   const double *xg, const double *yg, double *jac, double *alfa,
                                   double *beta, double *gama, double *pmet, double *qmet,
                                   double *detadx, double *detady, double *xphys, double *yphys)
{
    V2D_TRY(check_finite_mesh(imax, jmax));
    double *outs[10] = {jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys, yphys};
    V2D_ARG_CHECK(xg && yg, "compute_metrics: null mesh pointer");
    for (int q = 0; q < 10; ++q) V2D_ARG_CHECK(outs[q], "compute_metrics: null output %d", q);
    return metrics_host(false, imax, jmax, 0, 0, dksi, deta, xg, yg, outs);
}

extern "C" int v2d_compute_metrics_local(int gxm, int jmax, int il0, int il1, double dksi,
                                         double deta, const double *xgl, const double *ygl,
                                         double *jac, double *alfa, double *beta, double *gama,
                                         double *pmet, double *qmet, double *detadx,
                                         double *detady, double *xphys, double *yphys)
{
    V2D_ARG_CHECK(jmax >= 4 && gxm >= 3, "compute_metrics_local: block %d x %d too small", gxm, jmax);
    V2D_ARG_CHECK(il0 >= 2 && il1 <= gxm - 1 && il0 <= il1,
                  "compute_metrics_local: owned columns [%d,%d] need a ghost on both sides of 1..%d",
                  il0, il1, gxm);
    double *outs[10] = {jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys, yphys};
    V2D_ARG_CHECK(xgl && ygl, "compute_metrics_local: null mesh pointer");
    for (int q = 0; q < 10; ++q) V2D_ARG_CHECK(outs[q], "compute_metrics_local: null output %d", q);
    return metrics_host(true, gxm, jmax, il0 - 1, il1 - 1, dksi, deta, xgl, ygl, outs);
}

// Uploads the 14 field arrays of one assembly call into one device slab.
static int upload_fields(const double *const *h, size_t N, DevBuf<double> &buf, Fields &f,
                         cudaStream_t s)
{
    V2D_TRY(buf.alloc(14 * N, s));
    const double **dst[14] = {&f.jac, &f.alfa, &f.beta, &f.gama, &f.pmet, &f.qmet, &f.detadx,
                              &f.detady, &f.xphys, &f.yphys, &f.psi, &f.ome, &f.omeold,
                              &f.omeoldold};
    for (int q = 0; q < 14; ++q) {
        V2D_ARG_CHECK(h[q], "assemble: null field pointer %d", q);
        V2D_TRY(HostCopy::up(buf.p + q * N, h[q], N, s));
        *dst[q] = buf.p + q * N;
    }
    return V2D_OK;
}

extern "C" int v2d_assemble_coo(int imax, int jmax, double re, double invdtau, double inv2dt,
                                double urot, double dksi, double deta, const double *jac,
                                const double *alfa, const double *beta, const double *gama,
                                const double *pmet, const double *qmet, const double *detadx,
                                const double *detady, const double *xphys, const double *yphys,
                                const double *psi, const double *ome, const double *omeold,
                                const double *omeoldold, int r0, int r1, int maxnnz, int ff_bc,
                                double ca, double sa, int *coo_i, int *coo_j, double *coo_v,
                                int *nnz, double *bvec)
{
    V2D_TRY(check_finite_mesh(imax, jmax));
    const int N = imax * jmax;
    V2D_ARG_CHECK(r0 >= 0 && r1 <= 2 * N && r0 <= r1, "assemble_coo: rows [%d,%d) outside [0,%d)",
                  r0, r1, 2 * N);
    V2D_ARG_CHECK(nnz && (r1 == r0 || bvec), "assemble_coo: null output pointer");
    cudaStream_t s = 0;
    const double *h[14] = {jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys, yphys,
                           psi, ome, omeold, omeoldold};
    DevBuf<double> fbuf;
    Fields f;
    V2D_TRY(upload_fields(h, N, fbuf, f, s));
    GlobalTopo T{imax, jmax, N};
    Coeffs c{re, invdtau, inv2dt, urot, dksi, deta, ca, sa, ff_bc};
    const int nrows = r1 - r0;
    DevBuf<int> ibuf;
    V2D_TRY(ibuf.alloc((size_t)nrows + 1 + scan_scratch_ints(nrows), s));
    int *cnt = ibuf.p, *total = ibuf.p + nrows, *scratch = total + 1;
    if (nrows > 0) {
        coo_count_global<<<grid_for(nrows, 256), 256, 0, s>>>(T, c, f, r0, r1, cnt);
        V2D_CUDA_TRY(cudaGetLastError());
    }
    V2D_TRY(exclusive_scan_i32(cnt, cnt, nrows, total, scratch, s));
    int m = 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(&m, total, sizeof(int), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    *nnz = 0;
    if (m > maxnnz) {
        set_error("assemble_coo: %d entries exceed maxnnz=%d", m, maxnnz);
        return V2D_ECAPACITY;
    }
    V2D_ARG_CHECK(m == 0 || (coo_i && coo_j && coo_v), "assemble_coo: null COO pointer");
    DevBuf<int> cbuf;
    DevBuf<double> vbuf;
    V2D_TRY(cbuf.alloc(2 * (size_t)m + 1, s));
    V2D_TRY(vbuf.alloc((size_t)m + nrows + 1, s));
    if (nrows > 0) {
        coo_fill_global<<<grid_for(nrows, 256), 256, 0, s>>>(T, c, f, r0, r1, cnt, cbuf.p,
                                                              cbuf.p + m, vbuf.p, vbuf.p + m);
        V2D_CUDA_TRY(cudaGetLastError());
    }
    if (m > 0) {
        V2D_CUDA_TRY(cudaMemcpyAsync(coo_i, cbuf.p, m * sizeof(int), cudaMemcpyDeviceToHost, s));
        V2D_CUDA_TRY(cudaMemcpyAsync(coo_j, cbuf.p + m, m * sizeof(int), cudaMemcpyDeviceToHost, s));
        V2D_CUDA_TRY(cudaMemcpyAsync(coo_v, vbuf.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (nrows > 0)
        V2D_CUDA_TRY(cudaMemcpyAsync(bvec, vbuf.p + m, nrows * sizeof(double), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    *nnz = m;
    return V2D_OK;
}

extern "C" int v2d_assemble_coo_local(int gxm, int jmax, int il0, int il1, double re,
                                      double invdtau, double inv2dt, double urot, double dksi,
                                      double deta, const double *jac, const double *alfa,
                                      const double *beta, const double *gama, const double *pmet,
                                      const double *qmet, const double *detadx,
                                      const double *detady, const double *xphys,
                                      const double *yphys, const double *psi, const double *ome,
                                      const double *omeold, const double *omeoldold, int r0,
                                      int nloc, const int *lg, int maxnnz, int ff_bc, double ca,
                                      double sa, int *coo_i, int *coo_j, double *coo_v, int *nnz,
                                      double *bvec)
{
    V2D_ARG_CHECK(jmax >= 4 && gxm >= 3, "assemble_coo_local: block %d x %d too small", gxm, jmax);
    V2D_ARG_CHECK(il0 >= 2 && il1 <= gxm - 1 && il0 <= il1,
                  "assemble_coo_local: owned columns [%d,%d] need a ghost on both sides of 1..%d",
                  il0, il1, gxm);
    V2D_ARG_CHECK(lg && nnz && (nloc == 0 || bvec) && nloc >= 0, "assemble_coo_local: bad pointer");
    cudaStream_t s = 0;
    const size_t N = (size_t)gxm * jmax;
    const double *h[14] = {jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys, yphys,
                           psi, ome, omeold, omeoldold};
    DevBuf<double> fbuf;
    Fields f;
    V2D_TRY(upload_fields(h, N, fbuf, f, s));
    DevBuf<int> lgbuf;
    V2D_TRY(lgbuf.alloc(2 * N, s));
    V2D_CUDA_TRY(cudaMemcpyAsync(lgbuf.p, lg, 2 * N * sizeof(int), cudaMemcpyHostToDevice, s));
    LocalTopo T{gxm, jmax, lgbuf.p};
    Coeffs c{re, invdtau, inv2dt, urot, dksi, deta, ca, sa, ff_bc};
    const int nown = il1 - il0 + 1;
    const long long nnode = (long long)nown * jmax;
    DevBuf<int> ibuf;
    V2D_TRY(ibuf.alloc((size_t)nnode + 2 + scan_scratch_ints(nnode), s));
    int *cnt = ibuf.p, *total = ibuf.p + nnode, *bad = total + 1, *scratch = bad + 1;
    V2D_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
    coo_count_local<<<grid_for(nnode, 256), 256, 0, s>>>(T, c, f, il0 - 1, nown, cnt);
    V2D_CUDA_TRY(cudaGetLastError());
    V2D_TRY(exclusive_scan_i32(cnt, cnt, nnode, total, scratch, s));
    int m = 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(&m, total, sizeof(int), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    *nnz = 0;
    if (m > maxnnz) {
        set_error("assemble_coo_local: %d entries exceed maxnnz=%d", m, maxnnz);
        return V2D_ECAPACITY;
    }
    DevBuf<int> cbuf;
    DevBuf<double> vbuf;
    V2D_TRY(cbuf.alloc(2 * (size_t)m + 1, s));
    V2D_TRY(vbuf.alloc((size_t)m + nloc + 1, s));
    V2D_CUDA_TRY(cudaMemsetAsync(vbuf.p + m, 0, (size_t)nloc * sizeof(double), s));
    coo_fill_local<<<grid_for(nnode, 256), 256, 0, s>>>(T, c, f, il0 - 1, nown, r0, nloc, cnt,
                                                         cbuf.p, cbuf.p + m, vbuf.p, vbuf.p + m, bad);
    V2D_CUDA_TRY(cudaGetLastError());
    int badrow = 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(&badrow, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (m > 0) {
        V2D_CUDA_TRY(cudaMemcpyAsync(coo_i, cbuf.p, m * sizeof(int), cudaMemcpyDeviceToHost, s));
        V2D_CUDA_TRY(cudaMemcpyAsync(coo_j, cbuf.p + m, m * sizeof(int), cudaMemcpyDeviceToHost, s));
        V2D_CUDA_TRY(cudaMemcpyAsync(coo_v, vbuf.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (nloc > 0)
        V2D_CUDA_TRY(cudaMemcpyAsync(bvec, vbuf.p + m, nloc * sizeof(double), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    if (badrow) {
        set_error("assemble_coo_local: an owned row falls outside [r0, r0+nloc) = [%d, %d)", r0,
                  r0 + nloc);
        return V2D_EARG;
    }
    *nnz = m;
    return V2D_OK;
}

// ------------------------------------------- allocation-free COO assembly
// Some callers cannot allocate device memory at the point where they
// assemble: a framework that owns all of the GPU's memory through its own pool
// and budget, or a time-critical loop that must not hit cudaMalloc/cudaFree
// (both can synchronize the device and cudaMalloc can fail under memory
// pressure).  v2d_assemble_coo_noalloc serves them: the caller passes device
// buffers for every input and output, and the only scratch the kernels need
// (per-row entry counts turned into row offsets, plus the scan's tile sums)
// lives in the file-scope array below, which every GPU that loads this
// library holds until the process exits.
namespace v2d {

constexpr int kNoAllocMaxRows = 1 << 20;
static __device__ __align__(256) int g_coo_scratch[kNoAllocMaxRows + 2048];

}  // namespace v2d

extern "C" int v2d_assemble_coo_noalloc(int imax, int jmax, double re, double invdtau,
                                        double inv2dt, double urot, double dksi, double deta,
                                        const double *const *d_fields14, int r0, int r1,
                                        int maxnnz, int ff_bc, double ca, double sa, int *d_coo_i,
                                        int *d_coo_j, double *d_coo_v, int *nnz, double *d_bvec,
                                        void *stream)
{
    using namespace v2d;
    static std::mutex mu;
    static int *scratch_of_device[256] = {};
    V2D_TRY(check_finite_mesh(imax, jmax));
    const int N = imax * jmax;
    V2D_ARG_CHECK(d_fields14 && nnz, "assemble_coo_noalloc: null pointer");
    for (int q = 0; q < 14; ++q)
        V2D_ARG_CHECK(d_fields14[q], "assemble_coo_noalloc: field %d is null", q);
    V2D_ARG_CHECK(r0 >= 0 && r1 <= 2 * N && r0 <= r1,
                  "assemble_coo_noalloc: rows [%d,%d) outside [0,%d)", r0, r1, 2 * N);
    const int nrows = r1 - r0;
    V2D_ARG_CHECK(nrows <= kNoAllocMaxRows,
                  "assemble_coo_noalloc: %d rows exceed the fixed scratch of %d rows; use "
                  "v2d_assemble_coo or assemble in row ranges of at most %d rows",
                  nrows, kNoAllocMaxRows, kNoAllocMaxRows);
    V2D_ARG_CHECK(nrows == 0 || d_bvec, "assemble_coo_noalloc: null bvec");
    // device address of the scratch array, looked up once per device with
    // that device current
    int dev = 0;
    V2D_CUDA_TRY(cudaGetDevice(&dev));
    V2D_ARG_CHECK(dev >= 0 && dev < 256, "assemble_coo_noalloc: device %d out of range", dev);
    int *scratch_base = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!scratch_of_device[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_coo_scratch);
            if (e != cudaSuccess || !p) {
                set_error("assemble_coo_noalloc: cudaGetSymbolAddress failed on device %d: %s",
                          dev, cudaGetErrorString(e));
                return V2D_ECUDA;
            }
            scratch_of_device[dev] = (int *)p;
        }
        scratch_base = scratch_of_device[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    Fields f;
    f.jac = d_fields14[0]; f.alfa = d_fields14[1]; f.beta = d_fields14[2]; f.gama = d_fields14[3];
    f.pmet = d_fields14[4]; f.qmet = d_fields14[5]; f.detadx = d_fields14[6];
    f.detady = d_fields14[7]; f.xphys = d_fields14[8]; f.yphys = d_fields14[9];
    f.psi = d_fields14[10]; f.ome = d_fields14[11]; f.omeold = d_fields14[12];
    f.omeoldold = d_fields14[13];
    GlobalTopo T{imax, jmax, N};
    Coeffs c{re, invdtau, inv2dt, urot, dksi, deta, ca, sa, ff_bc};
    // counts -> offsets in place; the total after them; then the scan's tile
    // sums.  Every entry the kernels read is written earlier in this call, so
    // nothing left by a previous call is used.
    int *cnt = scratch_base, *total = scratch_base + nrows, *tiles = total + 1;
    if (nrows > 0) {
        coo_count_global<<<grid_for(nrows, 256), 256, 0, s>>>(T, c, f, r0, r1, cnt);
        V2D_CUDA_TRY(cudaGetLastError());
    }
    V2D_TRY(exclusive_scan_i32(cnt, cnt, nrows, total, tiles, s));
    int m = 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(&m, total, sizeof(int), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    *nnz = 0;
    if (m > maxnnz) {
        set_error("assemble_coo_noalloc: %d entries exceed maxnnz=%d", m, maxnnz);
        return V2D_ECAPACITY;
    }
    V2D_ARG_CHECK(m == 0 || (d_coo_i && d_coo_j && d_coo_v), "assemble_coo_noalloc: null COO pointer");
    if (nrows > 0) {
        coo_fill_global<<<grid_for(nrows, 256), 256, 0, s>>>(T, c, f, r0, r1, cnt, d_coo_i,
                                                              d_coo_j, d_coo_v, d_bvec);
        V2D_CUDA_TRY(cudaGetLastError());
    }
    count_launches(nrows > 0 ? 2 : 0);   // the scan counts its own launches
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    *nnz = m;
    return V2D_OK;
}
