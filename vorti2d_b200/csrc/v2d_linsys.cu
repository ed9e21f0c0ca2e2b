// Linear-solver seam: drop-in for vorti2d.petsc_solver.MumpsSolver
// (reference vorti2d/petsc_solver.py:37-132).
//
// assemble(): the first call turns the COO triplets into the canonical CSR
// pattern on the device (rows ascending, columns ascending, duplicates summed
// -- what scipy's csr_matrix produces at vorti2d/petsc_solver.py:81-84) and
// keeps the COO->slot structure; later calls only gather the new values
// (the cached-permutation refresh of vorti2d/dist_solver.py:327-366).
// solve(): GMRES(m) on the device, full solution returned.  The default
// preconditioner is the multifrontal LU of the assembled matrix (V2D_PC_LU),
// refreshed at every solve, so each solve is a direct solve refined by GMRES
// to rtol -- the role of the reference's MUMPS LU (petsc_solver.py:55-61).
// Its nested-dissection ordering needs the O-grid shape (imax, jmax): given by
// v2d_linsys_set_grid, or recognised from the pattern at the first assemble
// (the only imax that divides n/2 whose interior rows have the 9-point
// psi/omega stencil); block Jacobi and no preconditioner need no grid.
//
// Pattern build: row histogram (integer atomics), scan, scatter of COO
// indices into row buckets, then one thread per row sorts its bucket by
// (column, COO index) -- the result does not depend on the atomic order, so
// the pattern and the duplicate summation order are deterministic.
#include <algorithm>
#include <cstring>
#include <vector>

#include "v2d_internal.cuh"

using namespace v2d;

struct v2d_linsys {
    int n = 0, layout = 1;
    v2d_krylov_params prm{};
    cudaStream_t s = nullptr;
    long long nnz_coo = 0, nnz = 0;
    int *coo_i = nullptr, *coo_j = nullptr;   // stored pattern (validation)
    double *coo_v = nullptr;
    int *bucket_ptr = nullptr;   // n+1, COO offsets per row
    int *bucket = nullptr;       // COO indices sorted by (col, index) within each row
    int *indptr = nullptr, *indices = nullptr;
    double *data = nullptr;
    float *data32 = nullptr;
    double *b = nullptr, *x = nullptr;
    double *dinv = nullptr;
    float *dinv32 = nullptr;
    int *flag = nullptr;
    KrylovWork *kw = nullptr;
    bool has_pattern = false, has_values = false;
    // LU preconditioner (field-blocked O-grid systems)
    int imax = 0, jmax = 0;
    MfPlan *plan = nullptr;
    MfFactor *lu = nullptr;
    bool lu_fresh = false;      // factors of the current values
    int lu_last_its = 0;
};

namespace {

__global__ void k_row_hist(const int *ci, const int *cj, long long nnz, int n, int *cnt, int *flag)
{
    V2D_GRID_STRIDE(e, nnz)
    {
        int r = ci[e], c = cj[e];
        if (r < 0 || r >= n || c < 0 || c >= n) {
            atomicOr(flag, 1);
            continue;
        }
        atomicAdd(&cnt[r], 1);
    }
}

__global__ void k_row_scatter(const int *ci, long long nnz, int n, const int *bptr, int *fill,
                              int *bucket)
{
    V2D_GRID_STRIDE(e, nnz)
    {
        int r = ci[e];
        if (r < 0 || r >= n) continue;
        int pos = bptr[r] + atomicAdd(&fill[r], 1);
        bucket[pos] = (int)e;
    }
}

// Insertion sort of each row bucket by (column, COO index); counts the
// distinct columns of the row.
__global__ void k_row_sort(int n, const int *cj, const int *bptr, int *bucket, int *ucnt)
{
    V2D_GRID_STRIDE(r, n)
    {
        int p0 = bptr[r], p1 = bptr[r + 1];
        for (int p = p0 + 1; p < p1; ++p) {
            int e = bucket[p];
            int ce = cj[e];
            int q = p - 1;
            while (q >= p0) {
                int f = bucket[q];
                int cf = cj[f];
                if (cf < ce || (cf == ce && f < e)) break;
                bucket[q + 1] = f;
                --q;
            }
            bucket[q + 1] = e;
        }
        int u = 0, last = -1;
        for (int p = p0; p < p1; ++p) {
            int c = cj[bucket[p]];
            if (c != last) ++u;
            last = c;
        }
        ucnt[r] = u;
    }
}

__global__ void k_row_indices(int n, const int *cj, const int *bptr, const int *bucket,
                              const int *indptr, int *indices)
{
    V2D_GRID_STRIDE(r, n)
    {
        int o = indptr[r] - 1, last = -1;
        for (int p = bptr[r]; p < bptr[r + 1]; ++p) {
            int c = cj[bucket[p]];
            if (c != last) indices[++o] = c;
            last = c;
        }
    }
}

// Value refresh: duplicates summed in (column, COO index) order.
__global__ void k_row_values(int n, const int *cj, const double *cv, const int *bptr,
                             const int *bucket, const int *indptr, double *data, float *data32)
{
    V2D_GRID_STRIDE(r, n)
    {
        int o = indptr[r] - 1, last = -1;
        double acc = 0.0;
        for (int p = bptr[r]; p < bptr[r + 1]; ++p) {
            int e = bucket[p];
            int c = cj[e];
            if (c != last) {
                if (o >= indptr[r]) {
                    data[o] = acc;
                    data32[o] = (float)acc;
                }
                ++o;
                acc = 0.0;
            }
            acc += cv[e];
            last = c;
        }
        if (o >= indptr[r]) {
            data[o] = acc;
            data32[o] = (float)acc;
        }
    }
}

__global__ void k_same_pattern(const int *a, const int *b, long long n, int *flag)
{
    V2D_GRID_STRIDE(e, n)
    {
        if (a[e] != b[e]) atomicOr(flag, 4);
    }
}

template <class T>
int upload(T *d, const T *h, size_t n, cudaStream_t s)
{
    if (n) V2D_CUDA_TRY(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return V2D_OK;
}

}  // namespace

extern "C" int v2d_linsys_destroy(v2d_linsys *L)
{
    if (!L) return V2D_OK;
    if (L->s) cudaStreamSynchronize(L->s);
    void *ptrs[] = {L->coo_i, L->coo_j, L->coo_v, L->bucket_ptr, L->bucket, L->indptr, L->indices,
                    L->data, L->data32, L->b, L->x, L->dinv, L->dinv32, L->flag};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    krylov_destroy(L->kw);
    mf_factor_destroy(L->lu);
    mf_plan_destroy(L->plan);
    if (L->s) cudaStreamDestroy(L->s);
    delete L;
    return V2D_OK;
}

// The O-grid shape of a field-blocked 2N system (psi rows [0, N), omega rows
// [N, 2N), node K = imax*j + i) from its pattern: a candidate imax (a divisor
// of N) is accepted when three interior nodes away from the seam, the wall
// and the far field have exactly the interior columns of
// vorti2d_core.f90:276-293 (psi: the 9 psi neighbours and omega_K) and
// :341-378 (omega: the 9 omega neighbours and psi n, s, e, w).
static bool interior_rows_match(int imax, int N, const int *rp, const int *ci, int i, int j)
{
    const int K = imax * j + i;
    int want_psi[10], want_ome[13], a = 0;
    for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) want_psi[a++] = K + dj * imax + di;
    want_psi[a++] = N + K;
    a = 0;
    for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) want_ome[a++] = N + K + dj * imax + di;
    want_ome[a++] = K - imax;
    want_ome[a++] = K - 1;
    want_ome[a++] = K + 1;
    want_ome[a++] = K + imax;
    std::sort(want_psi, want_psi + 10);
    std::sort(want_ome, want_ome + 13);
    auto same = [&](int r, const int *w, int nw) {
        std::vector<int> c(ci + rp[r], ci + rp[r + 1]);
        std::sort(c.begin(), c.end());
        c.erase(std::unique(c.begin(), c.end()), c.end());
        return (int)c.size() == nw && std::equal(c.begin(), c.end(), w);
    };
    return same(K, want_psi, 10) && same(N + K, want_ome, 13);
}

static int infer_grid(int n, const std::vector<int> &rp, const std::vector<int> &ci, int *imax,
                      int *jmax)
{
    const int N = n / 2;
    int found = 0, fi = 0;
    for (int im = 5; im <= N / 6; ++im) {
        if (N % im) continue;
        const int jm = N / im;
        if (jm < 6) continue;
        const int probes[3][2] = {{im / 2, jm / 2}, {1, 2}, {im - 2, jm - 3}};
        bool ok = true;
        for (auto &pr : probes)
            ok = ok && interior_rows_match(im, N, rp.data(), ci.data(), pr[0], pr[1]);
        if (ok) {
            ++found;
            fi = im;
        }
    }
    if (found != 1) {
        set_error("linsys: the LU preconditioner needs the O-grid shape; %s (call "
                  "v2d_linsys_set_grid, or use block Jacobi)",
                  found ? "several grid shapes fit the pattern" : "the pattern is not a "
                  "field-blocked psi-omega O-grid system with at least 6 rows");
        return V2D_EARG;
    }
    *imax = fi;
    *jmax = N / fi;
    return V2D_OK;
}

extern "C" int v2d_linsys_set_grid(v2d_linsys *L, int imax, int jmax)
{
    V2D_ARG_CHECK(L, "linsys_set_grid: null handle");
    V2D_ARG_CHECK(!L->has_pattern, "linsys_set_grid: the pattern is already fixed");
    V2D_ARG_CHECK(imax >= 5 && jmax >= 4 && (long long)imax * jmax * 2 == L->n,
                  "linsys_set_grid: 2 * %d * %d != n = %d", imax, jmax, L->n);
    L->imax = imax;
    L->jmax = jmax;
    return V2D_OK;
}

// Symbolic LU plan and factor storage for the fixed pattern.
static int setup_lu(v2d_linsys *L)
{
    V2D_ARG_CHECK(L->layout == 1, "linsys: the LU preconditioner needs the field-blocked "
                  "layout (block_layout 1)");
    std::vector<int> rp(L->n + 1), ci(L->nnz);
    V2D_CUDA_TRY(cudaMemcpyAsync(rp.data(), L->indptr, (L->n + 1) * sizeof(int),
                                 cudaMemcpyDeviceToHost, L->s));
    V2D_CUDA_TRY(cudaMemcpyAsync(ci.data(), L->indices, L->nnz * sizeof(int),
                                 cudaMemcpyDeviceToHost, L->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(L->s));
    if (!L->imax) V2D_TRY(infer_grid(L->n, rp, ci, &L->imax, &L->jmax));
    const int leaf = L->prm.lu_leaf > 0 ? L->prm.lu_leaf : 64;
    V2D_TRY(mf_plan_create(L->imax, L->jmax, L->n, rp.data(), ci.data(), leaf, &L->plan));
    V2D_TRY(mf_factor_create(L->plan, L->prm.precision == V2D_PREC_MIXED ? 1 : 0,
                             L->prm.lu_factor64, &L->lu));
    L->lu->flow = L->prm.lu_solve == 0 ? 1 : 0;
    return V2D_OK;
}

extern "C" int v2d_linsys_create(int n, int block_layout, const v2d_krylov_params *p,
                                 v2d_linsys **out)
{
    V2D_ARG_CHECK(out && p, "linsys_create: null pointer");
    *out = nullptr;
    V2D_ARG_CHECK(n > 0, "linsys_create: n must be positive (got %d)", n);
    V2D_ARG_CHECK(block_layout >= 0 && block_layout <= 2, "linsys_create: layout %d", block_layout);
    V2D_ARG_CHECK(block_layout == 0 || n % 2 == 0, "linsys_create: 2x2 layouts need an even n");
    V2D_ARG_CHECK(p->precond != V2D_PC_LU || block_layout == 1,
                  "linsys_create: the LU preconditioner needs the field-blocked layout "
                  "(block_layout 1)");
    v2d_linsys *L = new v2d_linsys();
    L->n = n;
    L->layout = block_layout;
    L->prm = *p;
    cudaError_t e = cudaStreamCreateWithFlags(&L->s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&L->bucket_ptr, (size_t)(n + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&L->indptr, (size_t)(n + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&L->b, (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&L->x, (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&L->dinv, (size_t)4 * n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&L->dinv32, (size_t)4 * n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&L->flag, sizeof(int));
    if (e != cudaSuccess) {
        set_error("linsys_create: allocation failed: %s", cudaGetErrorString(e));
        v2d_linsys_destroy(L);
        return V2D_ENOMEM;
    }
    int st = krylov_create(&L->kw, n, p->restart, L->s);
    if (st != V2D_OK) {
        v2d_linsys_destroy(L);
        return st;
    }
    *out = L;
    return V2D_OK;
}

static int read_flag(v2d_linsys *L, int *f)
{
    V2D_CUDA_TRY(cudaMemcpyAsync(f, L->flag, sizeof(int), cudaMemcpyDeviceToHost, L->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(L->s));
    return V2D_OK;
}

extern "C" int v2d_linsys_assemble(v2d_linsys *L, const int *coo_i, const int *coo_j,
                                   const double *coo_v, long long nnz, const double *b)
{
    V2D_ARG_CHECK(L && b && nnz >= 0 && (nnz == 0 || (coo_i && coo_j && coo_v)),
                  "linsys_assemble: bad arguments");
    const int n = L->n;
    cudaStream_t s = L->s;
    V2D_CUDA_TRY(cudaMemsetAsync(L->flag, 0, sizeof(int), s));
    if (!L->has_pattern) {
        L->nnz_coo = nnz;
        V2D_CUDA_TRY(cudaMalloc(&L->coo_i, (size_t)(nnz + 1) * sizeof(int)));
        V2D_CUDA_TRY(cudaMalloc(&L->coo_j, (size_t)(nnz + 1) * sizeof(int)));
        V2D_CUDA_TRY(cudaMalloc(&L->coo_v, (size_t)(nnz + 1) * sizeof(double)));
        V2D_CUDA_TRY(cudaMalloc(&L->bucket, (size_t)(nnz + 1) * sizeof(int)));
        V2D_TRY(upload(L->coo_i, coo_i, nnz, s));
        V2D_TRY(upload(L->coo_j, coo_j, nnz, s));
        DevBuf<int> tmp;
        V2D_TRY(tmp.alloc((size_t)2 * (n + 1) + scan_scratch_ints(n + 1), s));
        int *cnt = tmp.p, *fill = tmp.p + (n + 1), *scratch = tmp.p + 2 * (n + 1);
        V2D_CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)2 * (n + 1) * sizeof(int), s));
        k_row_hist<<<grid_for(nnz, 256), 256, 0, s>>>(L->coo_i, L->coo_j, nnz, n, cnt, L->flag);
        V2D_TRY(exclusive_scan_i32(cnt, L->bucket_ptr, n, L->bucket_ptr + n, scratch, s));
        k_row_scatter<<<grid_for(nnz, 256), 256, 0, s>>>(L->coo_i, nnz, n, L->bucket_ptr, fill,
                                                         L->bucket);
        k_row_sort<<<grid_for(n, 128), 128, 0, s>>>(n, L->coo_j, L->bucket_ptr, L->bucket, cnt);
        V2D_TRY(exclusive_scan_i32(cnt, L->indptr, n, L->indptr + n, scratch, s));
        V2D_CUDA_TRY(cudaGetLastError());
        int f = 0, m = 0;
        V2D_CUDA_TRY(cudaMemcpyAsync(&m, L->indptr + n, sizeof(int), cudaMemcpyDeviceToHost, s));
        V2D_TRY(read_flag(L, &f));
        if (f & 1) {
            set_error("linsys_assemble: COO index outside [0, %d)", n);
            return V2D_EARG;
        }
        L->nnz = m;
        V2D_CUDA_TRY(cudaMalloc(&L->indices, (size_t)(m + 1) * sizeof(int)));
        V2D_CUDA_TRY(cudaMalloc(&L->data, (size_t)(m + 1) * sizeof(double)));
        V2D_CUDA_TRY(cudaMalloc(&L->data32, (size_t)(m + 1) * sizeof(float)));
        k_row_indices<<<grid_for(n, 128), 128, 0, s>>>(n, L->coo_j, L->bucket_ptr, L->bucket,
                                                        L->indptr, L->indices);
        V2D_CUDA_TRY(cudaGetLastError());
        if (L->prm.precond == V2D_PC_LU) V2D_TRY(setup_lu(L));
        L->has_pattern = true;
    } else {
        V2D_ARG_CHECK(nnz == L->nnz_coo,
                      "linsys_assemble: %lld triplets, the pattern was fixed with %lld", nnz,
                      L->nnz_coo);
        DevBuf<int> chk;
        V2D_TRY(chk.alloc((size_t)2 * nnz + 1, s));
        V2D_TRY(upload(chk.p, coo_i, nnz, s));
        V2D_TRY(upload(chk.p + nnz, coo_j, nnz, s));
        k_same_pattern<<<grid_for(nnz, 256), 256, 0, s>>>(chk.p, L->coo_i, nnz, L->flag);
        k_same_pattern<<<grid_for(nnz, 256), 256, 0, s>>>(chk.p + nnz, L->coo_j, nnz, L->flag);
        V2D_CUDA_TRY(cudaGetLastError());
    }
    V2D_TRY(upload(L->coo_v, coo_v, nnz, s));
    V2D_TRY(upload(L->b, b, n, s));
    k_row_values<<<grid_for(n, 128), 128, 0, s>>>(n, L->coo_j, L->coo_v, L->bucket_ptr, L->bucket,
                                                   L->indptr, L->data, L->data32);
    V2D_CUDA_TRY(cudaGetLastError());
    CsrOp A;
    A.n = n; A.nnz = L->nnz; A.rowptr = L->indptr; A.colind = L->indices; A.val = L->data;
    A.val32 = L->data32; A.layout = L->layout; A.nblk = L->layout == 0 ? n : n / 2;
    if (L->prm.precond == V2D_PC_BJACOBI) V2D_TRY(launch_block_inverse(A, L->dinv, L->dinv32, L->flag, s));
    int f = 0;
    V2D_TRY(read_flag(L, &f));
    if (f & 4) {
        set_error("linsys_assemble: the (i, j) sequence differs from the fixed pattern");
        return V2D_EARG;
    }
    if (f & 1) {
        set_error("linsys_assemble: singular diagonal block for Jacobi");
        return V2D_EBREAKDOWN;
    }
    L->has_values = true;
    L->lu_fresh = false;
    return V2D_OK;
}

extern "C" int v2d_linsys_solve(v2d_linsys *L, double *x, v2d_lin_stats *st)
{
    V2D_ARG_CHECK(L && x, "linsys_solve: null pointer");
    V2D_ARG_CHECK(L->has_values, "linsys_solve: assemble() first");
    CsrOp A;
    A.n = L->n; A.nnz = L->nnz; A.rowptr = L->indptr; A.colind = L->indices; A.val = L->data;
    A.val32 = L->data32; A.dinv = L->dinv; A.dinv32 = L->dinv32; A.layout = L->layout;
    A.nblk = L->layout == 0 ? L->n : L->n / 2;
    v2d_lin_stats ls{};
    if (L->prm.precond == V2D_PC_LU) {
        // factors of the current values, or (lu_reuse_its > 0) the last
        // factors while the solves with them stay within that many
        // iterations: a bounded attempt, then refactor and solve again
        const v2d_krylov_params &kp = L->prm;
        A.lu_plan = L->plan;
        A.lu = L->lu;
        bool fresh = L->lu_fresh;
        const bool reuse = !fresh && kp.lu_reuse_its > 0 && L->lu_last_its >= 0 &&
                           L->lu_last_its <= kp.lu_reuse_its;
        if (!fresh && !reuse) {
            V2D_TRY(mf_factor(L->plan, L->lu, L->indptr, L->data, L->s));
            fresh = true;
        }
        int its0 = 0;
        if (!fresh) {
            v2d_krylov_params k2 = kp;
            k2.max_it = std::min(kp.max_it, kp.lu_reuse_its + 5);
            V2D_TRY(krylov_solve(L->kw, A, L->b, L->x, k2, &ls, L->s));
            V2D_TRY(mf_check_barrier(L->lu, L->s));
            if (!ls.converged) {
                its0 = ls.iterations;
                V2D_TRY(mf_factor(L->plan, L->lu, L->indptr, L->data, L->s));
                fresh = true;
            }
        }
        if (fresh) {
            V2D_TRY(krylov_solve(L->kw, A, L->b, L->x, kp, &ls, L->s));
            V2D_TRY(mf_check_barrier(L->lu, L->s));
            ls.iterations += its0;
        }
        const bool refactored = fresh && !L->lu_fresh;
        if (fresh) L->lu_fresh = true;
        L->lu_last_its = refactored ? 0 : ls.iterations;
    } else {
        V2D_TRY(krylov_solve(L->kw, A, L->b, L->x, L->prm, &ls, L->s));
    }
    V2D_CUDA_TRY(cudaMemcpyAsync(x, L->x, (size_t)L->n * sizeof(double), cudaMemcpyDeviceToHost, L->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(L->s));
    if (st) *st = ls;
    if (!ls.converged) {
        set_error("linsys_solve: GMRES did not converge (%d iterations, |r|/|b| = %.3e)",
                  ls.iterations, ls.res0 > 0 ? ls.res / ls.res0 : 0.0);
        return V2D_ENOTCONVERGED;
    }
    return V2D_OK;
}

extern "C" int v2d_linsys_nnz(const v2d_linsys *L, long long *nnz)
{
    V2D_ARG_CHECK(L && nnz, "null pointer");
    *nnz = L->nnz;
    return V2D_OK;
}

extern "C" int v2d_linsys_csr(const v2d_linsys *L, int *indptr, int *indices, double *data)
{
    V2D_ARG_CHECK(L && L->has_pattern, "linsys_csr: no pattern yet");
    if (indptr)
        V2D_CUDA_TRY(cudaMemcpyAsync(indptr, L->indptr, (L->n + 1) * sizeof(int), cudaMemcpyDeviceToHost, L->s));
    if (indices)
        V2D_CUDA_TRY(cudaMemcpyAsync(indices, L->indices, L->nnz * sizeof(int), cudaMemcpyDeviceToHost, L->s));
    if (data)
        V2D_CUDA_TRY(cudaMemcpyAsync(data, L->data, L->nnz * sizeof(double), cudaMemcpyDeviceToHost, L->s));
    V2D_CUDA_TRY(cudaStreamSynchronize(L->s));
    return V2D_OK;
}
