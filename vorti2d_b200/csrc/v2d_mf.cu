// Sparse direct factorization of the Newton system on the device: a
// multifrontal LU over a nested-dissection separator tree of the O-grid.
//
// It takes the place of the direct LU (MUMPS) of the reference's replicated
// solve (vorti2d/petsc_solver.py:55-61, 97-115): pure Newton (dtau = inf)
// systems of this discretisation defeat point / line block Jacobi and
// multigrid preconditioners, so every Newton iteration factors the current
// Jacobian and uses the factors as the right preconditioner of GMRES(m) (FP32
// factors inside FP64 defect correction in the mixed-precision form; FP64
// factors in the plain form).
//
// Symbolic phase (host, once per mesh and sparsity pattern):
//  * the separator tree is geometric: the root separator is the
//    circumferential row jmax/2, which splits the O-grid into an inner and an
//    outer annulus; each annulus is opened by its two seam columns into one
//    rectangle, and rectangles are split recursively by their middle column
//    or row (never rows 1 or jmax-2, whose boundary rows reach two rows away:
//    the Thom wall row, vorti2d_core.f90:322-339, and the outflow rows,
//    :254-269, :307-321) until they hold at most `leaf` nodes.  Every
//    separator thus spans at most one row or two half-columns, which keeps
//    the dense top fronts small;
//  * fronts are numbered level by level (level = height above the leaves), so
//    the fronts of one level, their dense storage and their assembly entries
//    are contiguous and each level is processed by a fixed set of batched
//    launches;
//  * struct(front) = (struct(children) U adj(separator)) minus the subtree,
//    over the symmetrised node graph of the CSR pattern; each CSR entry goes
//    to the front of whichever of its two nodes is eliminated first.
//
// Numeric phase (device, per Newton iteration), per level bottom-up:
//  row-scaled CSR values scattered into the zeroed fronts, children's
//  contribution blocks added (one child slot per launch: deterministic, no
//  atomics), then a blocked right-looking partial LU of each front, four
//  batched launches per 32-column panel: the diagonal block (one CTA per
//  front, pivoting among the block's rows), L21 for the rows below (row
//  chunks), row swaps + TRSM for the U12 block row (column chunks), GEMM
//  update of the trailing block (which leaves the Schur complement for the
//  parent).
//
// After each level's factorization the S x S pivot block of every front is
// replaced by the explicit inverses of its triangular factors (L11^-1 below
// the diagonal, U11^-1 on and above it).
//
// Solve (device): forward per level bottom-up (gather, permute, z = L11^-1 w,
// contribution vector for the parent), backward top-down (U12 x_struct,
// x = U11^-1 y, scatter).  Every step is a row-parallel product split over
// CTAs of 8 rows, so the large top fronts spread over many SMs.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "v2d_internal.cuh"

namespace v2d {

// rows per work item of the solve on levels with few fronts
constexpr int kSolveRowsHost = 8;
// threads of a solve work item (8 warps)
constexpr int kSolveThreadsHost = 256;
// the default work-item split aims at about this many items per level
constexpr int kItemsPerLevel = 600;

// Counters of the dataflow solve, three per front q: forward items of q
// that wrote z rows (fz), the children's forward items that wrote
// contribution rows (fin), backward items of q (bx); the work ticket after
// them.
__host__ __device__ inline int ctr_fz(int q, int nf) { return q; }
__host__ __device__ inline int ctr_fin(int q, int nf) { return nf + q; }
__host__ __device__ inline int ctr_bx(int q, int nf) { return 2 * nf + q; }
__host__ __device__ inline int ctr_fg(int q, int nf) { return 3 * nf + q; }
__host__ __device__ inline int ctr_bg(int q, int nf) { return 4 * nf + q; }
constexpr int kCtrPerFront = 5;

// ================================================================ symbolic
namespace {

struct TreeNode {
    std::vector<int> sep;   // node ids (pointer order K = imax*j + i)
    int kid[2] = {-1, -1};
    int parent = -1;
};

struct TreeBuilder {
    int imax, jmax, leaf;
    std::vector<TreeNode> t;  // postorder

    int add(std::vector<int> &&sep, int a, int b)
    {
        TreeNode nd;
        nd.sep = std::move(sep);
        int q = 0;
        if (a >= 0) nd.kid[q++] = a;
        if (b >= 0) nd.kid[q++] = b;
        t.push_back(std::move(nd));
        const int id = (int)t.size() - 1;
        for (int c : t[id].kid)
            if (c >= 0) t[c].parent = id;
        return id;
    }
    std::vector<int> block(int i0, int i1, int j0, int j1) const
    {
        std::vector<int> v;
        for (int j = j0; j < j1; ++j)
            for (int i = i0; i < i1; ++i) v.push_back(j * imax + i);
        return v;
    }
    int col_cut(int i0, int i1, int j0, int j1)
    {
        const int c = (i0 + i1) / 2;
        int a = rect(i0, c, j0, j1);
        int b = rect(c + 1, i1, j0, j1);
        return add(block(c, c + 1, j0, j1), a, b);
    }
    // Rectangle [i0,i1) x [j0,j1) of the non-periodic part of the ring.
    int rect(int i0, int i1, int j0, int j1)
    {
        const int w = i1 - i0, h = j1 - j0;
        if (w <= 0 || h <= 0) return -1;
        if (w * h <= leaf) return add(block(i0, i1, j0, j1), -1, -1);
        if (w >= h && w >= 3) return col_cut(i0, i1, j0, j1);
        int best = -1;
        const int mid = (j0 + j1) / 2;
        for (int r = j0 + 1; r < j1 - 1; ++r) {
            if (r == 1 || r == jmax - 2) continue;
            if (best < 0 || std::abs(r - mid) < std::abs(best - mid)) best = r;
        }
        if (best < 0) {
            if (w >= 3) return col_cut(i0, i1, j0, j1);
            return add(block(i0, i1, j0, j1), -1, -1);
        }
        int a = rect(i0, i1, j0, best);
        int b = rect(i0, i1, best + 1, j1);
        return add(block(i0, i1, best, best + 1), a, b);
    }
    // Annulus rows [j0, j1): cutting the two seam columns leaves one
    // (non-periodic) rectangle [1, imax-1) x [j0, j1).
    int annulus(int j0, int j1)
    {
        if (j1 <= j0) return -1;
        int kid = rect(1, imax - 1, j0, j1);
        std::vector<int> sep;
        for (int c : {0, imax - 1})
            for (int j = j0; j < j1; ++j) sep.push_back(j * imax + c);
        return add(std::move(sep), kid, -1);
    }
    void build()
    {
        // Ring first: the root is the circumferential row jc, which splits the
        // O-grid into an inner and an outer annulus (each keeps the wall or the
        // far-field rows and their two-row reach); every separator then spans
        // at most one row or two half-columns.  Grids with too few rows for
        // that use the seam columns plus the middle column as the root.
        int jc = jmax / 2;
        if (jc == 1 || jc == jmax - 2) ++jc;
        if (jmax >= 8 && jc >= 2 && jc <= jmax - 4) {
            int a = annulus(0, jc);
            int b = annulus(jc + 1, jmax);
            std::vector<int> root;
            for (int i = 0; i < imax; ++i) root.push_back(jc * imax + i);
            add(std::move(root), a, b);
            return;
        }
        const int mid = imax / 2;
        int a = rect(1, mid, 0, jmax);
        int b = rect(mid + 1, imax - 1, 0, jmax);
        std::vector<int> root;
        for (int c : {0, mid, imax - 1})
            for (int j = 0; j < jmax; ++j) root.push_back(j * imax + c);
        add(std::move(root), a, b);
    }
};

// Node adjacency in CSR form: node v's neighbours are nb[off[v], off[v] + len[v]).
struct NodeGraph {
    std::vector<int> off, len, nb;
    struct Range {
        const int *b, *e;
        const int *begin() const { return b; }
        const int *end() const { return e; }
    };
    Range of(int v) const { return {nb.data() + off[v], nb.data() + off[v] + len[v]}; }
};

template <class T>
int upload_vec(T **d, const std::vector<T> &h)
{
    *d = nullptr;
    const size_t bytes = std::max<size_t>(1, h.size()) * sizeof(T);
    V2D_CUDA_TRY(cudaMalloc((void **)d, bytes));
    if (!h.empty()) V2D_CUDA_TRY(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return V2D_OK;
}

}  // namespace

void mf_plan_destroy(MfPlan *p)
{
    if (!p) return;
    void *ptrs[] = {p->d_S, p->d_f, p->d_voff, p->d_uoff, p->d_child0, p->d_child1, p->d_parent,
                    p->d_foff, p->d_toff, p->d_goff, p->d_vars, p->d_cbmap, p->d_asm_csr,
                    p->d_asm_row, p->d_asm_pos, p->d_items};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    delete p;
}

// Work items of the solve.  Forward: per level bottom-up, per front, rows
// [0, f) -- whole fronts, or chunks of the level's rows-per-item count
// (item_rows, set by default from the level's size).  Backward: per level top-down, rows
// [0, S) in the same granularity.  Waits and done counters:
//   forward item of q   waits fin[q] = all children's items with contribution
//                       rows; done: fz[q] if it has z rows, fin[parent] if
//                       it has contribution rows
//   backward item of q  waits fz[q] = all of q's forward items with z rows,
//                       and bx[parent] = all of the parent's backward items
//                       (which waited for theirs: all ancestors' x);
//                       done: bx[q]
// On levels whose rows-per-item entry is negative, a front split into
// several items gets a gather item first in each sweep:
//   forward gather of q   waits fin[q]; writes t and the contribution rows'
//                         w to tw; done: fg[q]; q's forward items wait fg[q]
//   backward gather of q  waits bx[parent] (which implies that q's own
//                         contribution rows, the last readers of tw's w part,
//                         are done); writes -x of q's struct variables to
//                         tw; done: bg[q]; q's backward items wait fz[q] and
//                         bg[q]
// The check: every wait's counter reaches exactly its target in all, and
// only through items earlier in the order; so the items an item reads have
// all finished before it starts, and a CTA that takes items in order only
// waits for items that running CTAs hold.
static int items_build(MfPlan *P)
{
    const int nf = P->nfront, nl = P->nlevel;
    std::vector<int> &it = P->h_items;
    it.clear();
    P->lvl_fwd.assign(nl + 1, 0);
    P->lvl_bwd.assign(nl + 1, 0);
    // rows per item of each level (0: whole fronts).  The default aims at
    // about kItemsPerLevel items per level: the level's rows over that
    // count, rounded down to a power of two in [kSolveRowsHost, 256]; whole
    // fronts where no front of the level is longer than that
    if ((int)P->item_rows.size() != nl) {
        P->item_rows.assign(nl, kSolveRowsHost);
        for (int L = 0; L < nl; ++L) {
            long long rows = 0;
            for (int q = P->lvl_off[L]; q < P->lvl_off[L + 1]; ++q) rows += P->f[q];
            int R = kSolveRowsHost;
            while (R < 256 && 2LL * R * kItemsPerLevel <= rows) R *= 2;
            P->item_rows[L] = P->lvl_maxf[L] <= R ? 0 : R;
        }
    }
    // rows per item; a negative entry -R splits fronts of more than R rows
    // into R-row items after one gather item per front (kind 2 forward: w and
    // t = P w_FS into tw; kind 3 backward: -x of the struct variables into
    // tw), so the front's items read one contiguous vector instead of each
    // repeating the gather
    auto per = [&](int L) {
        const int r = P->item_rows[L];
        return r > 0 ? r : (r < 0 ? -r : INT_MAX);
    };
    auto gath_f = [&](int L, int q) { return P->item_rows[L] < 0 && P->f[q] > per(L); };
    auto gath_b = [&](int L, int q) {
        return P->item_rows[L] < 0 && P->S[q] > per(L) && P->f[q] > P->S[q];
    };
    int cur_level = 0;
    auto push = [&](int kind, int q, int rb, int re, int flag) {
        const int v[12] = {kind, q, rb, re, -1, 0, -1, 0, -1, -1, cur_level, flag};
        it.insert(it.end(), v, v + 12);
    };
    P->lvl_fwd_g.assign(nl, 0);
    P->lvl_bwd_g.assign(nl, 0);
    for (int L = 0; L < nl; ++L) {
        P->lvl_fwd[L] = (int)it.size() / 12;
        cur_level = L;
        const int R = per(L);
        for (int q = P->lvl_off[L]; q < P->lvl_off[L + 1]; ++q)
            if (gath_f(L, q)) {
                push(2, q, 0, P->f[q], 1);
                ++P->lvl_fwd_g[L];
            }
        for (int q = P->lvl_off[L]; q < P->lvl_off[L + 1]; ++q)
            for (int rb = 0; rb < P->f[q]; rb += std::min(R, P->f[q]))
                push(0, q, rb, (int)std::min<long long>((long long)rb + R, P->f[q]),
                     gath_f(L, q) ? 1 : 0);
    }
    P->lvl_fwd[nl] = (int)it.size() / 12;
    for (int L = nl - 1; L >= 0; --L) {
        P->lvl_bwd[L + 1] = (int)it.size() / 12;
        cur_level = L;
        const int R = per(L);
        for (int q = P->lvl_off[L]; q < P->lvl_off[L + 1]; ++q)
            if (gath_b(L, q)) {
                push(3, q, 0, P->S[q], 1);
                ++P->lvl_bwd_g[L];
            }
        for (int q = P->lvl_off[L]; q < P->lvl_off[L + 1]; ++q)
            for (int rb = 0; rb < P->S[q]; rb += std::min(R, P->S[q]))
                push(1, q, rb, (int)std::min<long long>((long long)rb + R, P->S[q]),
                     gath_b(L, q) ? 1 : 0);
    }
    P->lvl_bwd[0] = (int)it.size() / 12;
    const int ni = (int)it.size() / 12;
    // totals per front (row items only; a gather item counts once into its
    // own counter)
    std::vector<int> nfz(nf, 0), nfin(nf, 0), nbx(nf, 0);
    for (int k = 0; k < ni; ++k) {
        const int *v = &it[12 * k];
        const int q = v[1];
        if (v[0] == 0) {
            if (v[2] < P->S[q]) ++nfz[q];
            if (v[3] > P->S[q] && P->parent[q] >= 0) ++nfin[P->parent[q]];
        } else if (v[0] == 1) {
            ++nbx[q];
        }
    }
    for (int k = 0; k < ni; ++k) {
        int *v = &it[12 * k];
        const int q = v[1], pa = P->parent[q];
        switch (v[0]) {
        case 0:   // forward rows: the front's gather item, or the children's rows
            if (v[11]) { v[4] = ctr_fg(q, nf); v[5] = 1; }
            else if (nfin[q] > 0) { v[4] = ctr_fin(q, nf); v[5] = nfin[q]; }
            if (v[2] < P->S[q]) v[8] = ctr_fz(q, nf);
            if (v[3] > P->S[q] && pa >= 0) v[9] = ctr_fin(pa, nf);
            break;
        case 2:   // forward gather: the children's rows
            if (nfin[q] > 0) { v[4] = ctr_fin(q, nf); v[5] = nfin[q]; }
            v[8] = ctr_fg(q, nf);
            break;
        case 1:   // backward rows: the front's z, and the gather item or the parent's x
            v[4] = ctr_fz(q, nf);
            v[5] = nfz[q];
            if (v[11]) { v[6] = ctr_bg(q, nf); v[7] = 1; }
            else if (pa >= 0) { v[6] = ctr_bx(pa, nf); v[7] = nbx[pa]; }
            v[8] = ctr_bx(q, nf);
            break;
        case 3:   // backward gather: the parent's x (hence every ancestor's)
            if (pa >= 0) { v[4] = ctr_bx(pa, nf); v[5] = nbx[pa]; }
            v[8] = ctr_bg(q, nf);
            break;
        }
    }
    // the check
    const int nc = kCtrPerFront * nf;
    std::vector<int> total(nc, 0), seen(nc, 0);
    bool ok = true;
    for (int q = 0; q < nf; ++q)
        ok = ok && P->S[q] > 0 && (P->f[q] == P->S[q] || P->parent[q] >= 0);
    for (int k = 0; k < ni && ok; ++k) {
        const int *v = &it[12 * k];
        const int q = v[1], kind = v[0];
        ok = ok && kind >= 0 && kind <= 3 && q >= 0 && q < nf && v[2] >= 0 && v[3] > v[2] &&
             v[3] <= ((kind == 0 || kind == 2) ? P->f[q] : P->S[q]) && (v[11] == 0 || v[11] == 1);
        if (ok && kind >= 2)   // a gather item covers its whole front, once
            ok = v[11] == 1 && v[2] == 0 && v[3] == (kind == 2 ? P->f[q] : P->S[q]) &&
                 (kind == 2 || P->parent[q] >= 0);
        for (int d : {v[8], v[9]}) {
            ok = ok && d >= -1 && d < nc;
            if (ok && d >= 0) ++total[d];
        }
    }
    for (int k = 0; k < ni && ok; ++k) {
        const int *v = &it[12 * k];
        const int q = v[1], pa = P->parent[q];
        for (int w : {0, 1}) {
            const int c = v[4 + 2 * w], t = v[5 + 2 * w];
            if (c < 0) continue;
            ok = ok && c < nc && t > 0 && total[c] == t && seen[c] == t;
        }
        // what each kind must have waited for, from the algorithm
        if (v[0] == 0)
            ok = ok && (v[11] ? v[4] == ctr_fg(q, nf) && v[5] == 1
                              : (nfin[q] == 0 || (v[4] == ctr_fin(q, nf) && v[5] == nfin[q])));
        else if (v[0] == 2)
            ok = ok && (nfin[q] == 0 || (v[4] == ctr_fin(q, nf) && v[5] == nfin[q]));
        else if (v[0] == 1)
            ok = ok && v[4] == ctr_fz(q, nf) && v[5] == nfz[q] &&
                 (v[11] ? v[6] == ctr_bg(q, nf) && v[7] == 1
                        : (pa < 0 || (v[6] == ctr_bx(pa, nf) && v[7] == nbx[pa])));
        else
            ok = ok && v[4] == ctr_bx(pa, nf) && v[5] == nbx[pa];
        for (int d : {v[8], v[9]})
            if (d >= 0) ++seen[d];
    }
    if (!ok) {
        set_error("mf_plan: solve work items failed their order check");
        it.clear();
        return V2D_EARG;
    }
    P->nitems = ni;
    P->nctr = nc;
    return V2D_OK;
}

int mf_plan_build(int imax, int jmax, int n, const int *h_rowptr, const int *h_colind,
                  int leaf, MfPlan **out)
{
    *out = nullptr;
    const int N = imax * jmax;
    V2D_ARG_CHECK(n == 2 * N, "mf_plan: system size %d != 2 * %d nodes", n, N);
    V2D_ARG_CHECK(imax >= 5 && jmax >= 4, "mf_plan: grid %d x %d too small", imax, jmax);
    // the CSR pattern: row pointers from 0, non-decreasing; columns in [0, n)
    V2D_ARG_CHECK(h_rowptr[0] == 0, "mf_plan: indptr[0] = %d, not 0", h_rowptr[0]);
    for (int r = 0; r < n; ++r)
        V2D_ARG_CHECK(h_rowptr[r + 1] >= h_rowptr[r], "mf_plan: indptr decreases at row %d", r);
    for (int p = 0; p < h_rowptr[n]; ++p)
        V2D_ARG_CHECK(h_colind[p] >= 0 && h_colind[p] < n,
                      "mf_plan: column index %d at entry %d outside [0, %d)", h_colind[p], p, n);
    TreeBuilder tb{imax, jmax, std::max(4, leaf), {}};
    tb.build();
    const int nf = (int)tb.t.size();
    // --- symmetrised node graph (CSR): the distinct other nodes of each
    // node's two rows, then every such edge in both directions
    NodeGraph adj;
    {
        std::vector<int> foff(N + 1, 0), fwd, mark(N, -1);
        fwd.reserve((size_t)h_rowptr[n] / 2 + 16);
        for (int a = 0; a < N; ++a) {
            for (int r : {a, N + a})
                for (int p = h_rowptr[r]; p < h_rowptr[r + 1]; ++p) {
                    const int c = h_colind[p], b = c < N ? c : c - N;
                    if (b != a && mark[b] != a) {
                        mark[b] = a;
                        fwd.push_back(b);
                    }
                }
            foff[a + 1] = (int)fwd.size();
        }
        adj.off.assign(N + 1, 0);
        for (int a = 0; a < N; ++a)
            for (int p = foff[a]; p < foff[a + 1]; ++p) {
                ++adj.off[a + 1];
                ++adj.off[fwd[p] + 1];
            }
        for (int a = 0; a < N; ++a) adj.off[a + 1] += adj.off[a];
        adj.nb.resize(adj.off[N]);
        std::vector<int> fill(adj.off.begin(), adj.off.end() - 1);
        for (int a = 0; a < N; ++a)
            for (int p = foff[a]; p < foff[a + 1]; ++p) {
                adj.nb[fill[a]++] = fwd[p];
                adj.nb[fill[fwd[p]]++] = a;
            }
        adj.len.resize(N);
        for (int a = 0; a < N; ++a) {
            int *b = adj.nb.data() + adj.off[a], *e = adj.nb.data() + adj.off[a + 1];
            std::sort(b, e);
            adj.len[a] = (int)(std::unique(b, e) - b);
        }
    }
    // --- elimination order (postorder of the tree)
    std::vector<int> elim(N, -1), owner(N, -1), last_elim(nf);
    int order = 0;
    for (int q = 0; q < nf; ++q) {
        for (int v : tb.t[q].sep) {
            if (elim[v] >= 0) {
                set_error("mf_plan: node %d in two separators", v);
                return V2D_EARG;
            }
            elim[v] = order++;
            owner[v] = q;
        }
        last_elim[q] = order - 1;
    }
    if (order != N) {
        set_error("mf_plan: tree covers %d of %d nodes", order, N);
        return V2D_EARG;
    }
    // --- struct sets
    std::vector<std::vector<int>> st(nf);
    std::vector<int> stamp(N, -1);
    for (int q = 0; q < nf; ++q) {
        std::vector<int> s;
        auto take = [&](int u) {
            if (elim[u] > last_elim[q] && stamp[u] != q) {
                stamp[u] = q;
                s.push_back(u);
            }
        };
        for (int c : tb.t[q].kid)
            if (c >= 0)
                for (int u : st[c]) take(u);
        for (int v : tb.t[q].sep)
            for (int u : adj.of(v)) take(u);
        std::sort(s.begin(), s.end(), [&](int a, int b) { return elim[a] < elim[b]; });
        st[q] = std::move(s);
    }
    // a separator may couple only into its own subtree or to ancestors
    std::vector<int> first_elim(nf);
    for (int q = 0; q < nf; ++q) {
        int fe = last_elim[q] - (int)tb.t[q].sep.size() + 1;
        for (int c : tb.t[q].kid)
            if (c >= 0) fe = std::min(fe, first_elim[c]);
        first_elim[q] = fe;
    }
    for (int q = 0; q < nf; ++q)
        for (int v : tb.t[q].sep)
            for (int u : adj.of(v))
                if (elim[u] < first_elim[q]) {
                    set_error("mf_plan: node %d couples to node %d of a sibling subtree", v, u);
                    return V2D_EARG;
                }
    // every struct node must belong to an ancestor (no coupling across subtrees)
    for (int q = 0; q < nf; ++q)
        for (int u : st[q]) {
            int a = tb.t[q].parent;
            while (a >= 0 && a != owner[u]) a = tb.t[a].parent;
            if (a < 0) {
                set_error("mf_plan: node %d couples across sibling subtrees", u);
                return V2D_EARG;
            }
        }
    // --- levels and level-major numbering
    std::vector<int> height(nf, 0);
    int nlevel = 0;
    for (int q = 0; q < nf; ++q) {
        int h = 0;
        for (int c : tb.t[q].kid)
            if (c >= 0) h = std::max(h, height[c] + 1);
        height[q] = h;
        nlevel = std::max(nlevel, h + 1);
    }
    std::vector<int> newid(nf), oldid;
    for (int L = 0; L < nlevel; ++L)
        for (int q = 0; q < nf; ++q)
            if (height[q] == L) {
                newid[q] = (int)oldid.size();
                oldid.push_back(q);
            }
    MfPlan *P = new MfPlan();
    P->N = N; P->n = n; P->nfront = nf; P->nlevel = nlevel;
    P->S.resize(nf); P->f.resize(nf); P->voff.resize(nf); P->uoff.resize(nf);
    P->child0.assign(nf, -1); P->child1.assign(nf, -1); P->parent.assign(nf, -1);
    P->foff.resize(nf);
    P->lvl_off.assign(nlevel + 1, 0);
    P->lvl_fbeg.assign(nlevel, 0); P->lvl_fend.assign(nlevel, 0);
    P->lvl_abeg.assign(nlevel, 0); P->lvl_aend.assign(nlevel, 0);
    P->lvl_maxS.assign(nlevel, 0); P->lvl_maxf.assign(nlevel, 0); P->lvl_maxm.assign(nlevel, 0);
    P->lvl_maxm_child.assign(nlevel, 0);
    std::vector<int> vars, cbmap;
    long long ftot = 0;
    int vtot = 0, utot = 0;
    for (int id = 0; id < nf; ++id) {
        const int q = oldid[id];
        const int s = (int)tb.t[q].sep.size(), m = (int)st[q].size();
        const int S = 2 * s, f = 2 * (s + m);
        P->S[id] = S; P->f[id] = f;
        P->voff[id] = vtot; vtot += f;
        P->uoff[id] = utot; utot += f - S;
        P->foff[id] = ftot; ftot += (long long)f * f;
        const int L = height[q];
        P->lvl_off[L + 1]++;
        P->lvl_maxS[L] = std::max(P->lvl_maxS[L], S);
        P->lvl_maxf[L] = std::max(P->lvl_maxf[L], f);
        P->lvl_maxm[L] = std::max(P->lvl_maxm[L], f - S);
        if (tb.t[q].parent >= 0) P->parent[id] = newid[tb.t[q].parent];
        if (tb.t[q].kid[0] >= 0) P->child0[id] = newid[tb.t[q].kid[0]];
        if (tb.t[q].kid[1] >= 0) P->child1[id] = newid[tb.t[q].kid[1]];
        // front-local variables: node p -> vars 2p (psi, row/col p) and 2p+1 (ome, N+p)
        for (int u : tb.t[q].sep) { vars.push_back(u); vars.push_back(N + u); }
        for (int u : st[q]) { vars.push_back(u); vars.push_back(N + u); }
        P->maxS = std::max(P->maxS, S);
        P->maxf = std::max(P->maxf, f);
    }
    for (int L = 0; L < nlevel; ++L) P->lvl_off[L + 1] += P->lvl_off[L];
    P->toff.assign(nf, 0);
    for (int L = 0; L < nlevel; ++L) {
        long long t = 0;
        for (int id = P->lvl_off[L]; id < P->lvl_off[L + 1]; ++id) {
            P->toff[id] = t;
            t += (long long)P->S[id] * P->S[id];
        }
        P->tmax = std::max(P->tmax, t);
    }
    P->goff.assign(nf, 0);
    for (int L = 0; L < nlevel; ++L) {
        long long t = 0;
        for (int id = P->lvl_off[L]; id < P->lvl_off[L + 1]; ++id) {
            P->goff[id] = t;
            t += 2LL * P->S[id] * (P->f[id] - P->S[id]);
        }
        P->gmax = std::max(P->gmax, t);
    }
    for (int L = 0; L < nlevel; ++L) {
        const int a = P->lvl_off[L], b = P->lvl_off[L + 1];
        P->lvl_fbeg[L] = P->foff[a];
        P->lvl_fend[L] = P->foff[b - 1] + (long long)P->f[b - 1] * P->f[b - 1];
        for (int id = a; id < b; ++id)
            for (int c : {P->child0[id], P->child1[id]})
                if (c >= 0) P->lvl_maxm_child[L] = std::max(P->lvl_maxm_child[L], P->f[c] - P->S[c]);
    }
    // contribution-block maps: struct var of child -> local index in parent
    cbmap.assign(utot, -1);
    std::vector<int> loc(n, -1);
    for (int id = 0; id < nf; ++id) {
        const int pa = P->parent[id];
        if (pa < 0) continue;
        for (int t = 0; t < P->f[pa]; ++t) loc[vars[P->voff[pa] + t]] = t;
        for (int t = P->S[id]; t < P->f[id]; ++t) {
            const int li = loc[vars[P->voff[id] + t]];
            if (li < 0) {
                set_error("mf_plan: struct variable of front %d missing in its parent", id);
                mf_plan_destroy(P);
                return V2D_EARG;
            }
            cbmap[P->uoff[id] + t - P->S[id]] = li;
        }
        for (int t = 0; t < P->f[pa]; ++t) loc[vars[P->voff[pa] + t]] = -1;
    }
    // assembly entries grouped by front (level-major)
    std::vector<int> cnt(nf + 1, 0), entry_front(h_rowptr[n]);
    for (int r = 0; r < n; ++r)
        for (int p = h_rowptr[r]; p < h_rowptr[r + 1]; ++p) {
            const int c = h_colind[p];
            const int a = r < N ? r : r - N, b = c < N ? c : c - N;
            const int fr = newid[elim[a] < elim[b] ? owner[a] : owner[b]];
            entry_front[p] = fr;
            cnt[fr + 1]++;
        }
    for (int q = 0; q < nf; ++q) cnt[q + 1] += cnt[q];
    const long long nnz = h_rowptr[n];
    std::vector<int> asm_csr(nnz), asm_row(nnz);
    std::vector<long long> asm_pos(nnz);
    {
        // entries of each front in row order (a counting sort by front),
        // then each front's local positions from its variables' lookup
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int r = 0; r < n; ++r)
            for (int p = h_rowptr[r]; p < h_rowptr[r + 1]; ++p) {
                const int o = fill[entry_front[p]]++;
                asm_csr[o] = p;
                asm_row[o] = r;
            }
        for (int id = 0; id < nf; ++id) {
            const int f = P->f[id];
            for (int t = 0; t < f; ++t) loc[vars[P->voff[id] + t]] = t;
            for (int o = cnt[id]; o < cnt[id + 1]; ++o) {
                const int r = asm_row[o], c = h_colind[asm_csr[o]];
                const int lr = loc[r], lc = loc[c];
                if (lr < 0 || lc < 0) {
                    set_error("mf_plan: entry (%d, %d) outside its front", r, c);
                    mf_plan_destroy(P);
                    return V2D_EARG;
                }
                asm_pos[o] = P->foff[id] + (long long)lr * f + lc;
            }
            for (int t = 0; t < f; ++t) loc[vars[P->voff[id] + t]] = -1;
        }
    }
    for (int L = 0; L < nlevel; ++L) {
        P->lvl_abeg[L] = cnt[P->lvl_off[L]];
        P->lvl_aend[L] = cnt[P->lvl_off[L + 1]];
    }
    P->ftotal = ftot; P->vtotal = vtot; P->utotal = utot; P->nasm = nnz;
    double fl = 0.0;
    for (int id = 0; id < nf; ++id) {
        fl += 2.0 * P->S[id] * (double)P->f[id] * P->f[id];
        P->factor_flops += front_flops(P->S[id], P->f[id]);
        P->apply_entries += (long long)P->S[id] * (2LL * P->f[id] - P->S[id]);
    }
    P->flops = fl;
    // every index the kernels dereference stays inside its buffer
    bool ok = (long long)vars.size() == vtot && (long long)cbmap.size() == utot;
    for (int v : vars) ok = ok && v >= 0 && v < n;
    for (int id = 0; id < nf && ok; ++id) {
        ok = ok && P->S[id] > 0 && P->S[id] <= P->f[id] && P->S[id] % 2 == 0;
        const int pa = P->parent[id];
        if (pa >= 0)
            for (int t = 0; t < P->f[id] - P->S[id]; ++t) {
                const int li = cbmap[P->uoff[id] + t];
                ok = ok && li >= 0 && li < P->f[pa];
            }
        else
            ok = ok && P->f[id] == P->S[id];   // the root has no contribution block
        for (int c : {P->child0[id], P->child1[id]}) ok = ok && (c < 0 || (c < id && P->parent[c] == id));
    }
    for (long long e = 0; e < nnz && ok; ++e)
        ok = asm_pos[e] >= 0 && asm_pos[e] < ftot && asm_csr[e] >= 0 && asm_csr[e] < nnz &&
             asm_row[e] >= 0 && asm_row[e] < n;
    if (!ok) {
        set_error("mf_plan: internal index check failed (%d x %d grid)", imax, jmax);
        mf_plan_destroy(P);
        return V2D_EARG;
    }
    P->h_vars = std::move(vars);
    P->h_cbmap = std::move(cbmap);
    P->h_asm_csr = std::move(asm_csr);
    P->h_asm_row = std::move(asm_row);
    P->h_asm_pos = std::move(asm_pos);
    if (items_build(P) != V2D_OK) {
        mf_plan_destroy(P);
        return V2D_EARG;
    }
    *out = P;
    return V2D_OK;
}

// Device copies of a host plan's arrays; the host copies of the large index
// arrays are released.  On failure the plan is destroyed.
static int mf_plan_upload(MfPlan *P)
{
    int st_up = V2D_OK;
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_S, P->S);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_f, P->f);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_voff, P->voff);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_uoff, P->uoff);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_child0, P->child0);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_child1, P->child1);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_parent, P->parent);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_foff, P->foff);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_toff, P->toff);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_goff, P->goff);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_vars, P->h_vars);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_cbmap, P->h_cbmap);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_asm_csr, P->h_asm_csr);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_asm_row, P->h_asm_row);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_asm_pos, P->h_asm_pos);
    if (st_up == V2D_OK) st_up = upload_vec(&P->d_items, P->h_items);
    if (st_up != V2D_OK) {
        mf_plan_destroy(P);
        return st_up;
    }
    // host copies are not needed once uploaded
    std::vector<int>().swap(P->h_vars);
    std::vector<int>().swap(P->h_cbmap);
    std::vector<int>().swap(P->h_asm_csr);
    std::vector<int>().swap(P->h_asm_row);
    std::vector<long long>().swap(P->h_asm_pos);
    return V2D_OK;
}

int mf_plan_create(int imax, int jmax, int n, const int *h_rowptr, const int *h_colind,
                   int leaf, MfPlan **out)
{
    *out = nullptr;
    MfPlan *P = nullptr;
    V2D_TRY(mf_plan_build(imax, jmax, n, h_rowptr, h_colind, leaf, &P));
    V2D_TRY(mf_plan_upload(P));
    *out = P;
    return V2D_OK;
}

// New work-item granularity for the solve: rows[L] rows per item on level L
// (0: whole fronts; R > 0: R rows; R < 0: -R rows after one gather item per
// front).  Rebuilds and
// re-uploads the item table (its order is checked again); the device pointer
// changes, so solves captured in graphs before must be captured again
// (items_ver counts the tables).
int mf_plan_set_item_rows(MfPlan *P, const int *rows, int nlevels)
{
    V2D_ARG_CHECK(rows && nlevels == P->nlevel, "lu item rows: %d levels given, the plan has %d",
                  nlevels, P->nlevel);
    for (int L = 0; L < nlevels; ++L)
        V2D_ARG_CHECK(rows[L] >= -4096 && rows[L] <= 4096, "lu item rows: level %d: %d", L,
                      rows[L]);
    std::vector<int> keep = P->item_rows;
    P->item_rows.assign(rows, rows + nlevels);
    if (items_build(P) != V2D_OK) {
        P->item_rows = keep;
        items_build(P);
        return V2D_EARG;
    }
    int *d = nullptr;
    V2D_TRY(upload_vec(&d, P->h_items));
    if (P->d_items) cudaFree(P->d_items);
    P->d_items = d;
    ++P->items_ver;
    return V2D_OK;
}

// One plan for a block-diagonal system of several O-grid systems: the union
// of their front trees (a forest), fronts renumbered level by level across
// the parts, each part's variables, CSR entries and factor positions shifted
// by its offsets.  The factorization and the solve then treat every part in
// the same launches.  parts are host plans (mf_plan_build); row_off[k] and
// nnz_off[k] place part k's rows and CSR entries in the combined system of
// n rows.
int mf_plan_forest(const std::vector<MfPlan *> &parts, const std::vector<int> &row_off,
                   const std::vector<long long> &nnz_off, int n, MfPlan **out)
{
    *out = nullptr;
    const int np = (int)parts.size();
    V2D_ARG_CHECK(np > 0 && (int)row_off.size() == np && (int)nnz_off.size() == np,
                  "mf_plan_forest: %d parts, %zu row offsets, %zu entry offsets", np,
                  row_off.size(), nnz_off.size());
    int nl = 0;
    for (const MfPlan *Q : parts) {
        V2D_ARG_CHECK(Q && !Q->h_vars.empty(), "mf_plan_forest: a part without host arrays");
        nl = std::max(nl, Q->nlevel);
    }
    MfPlan *P = new MfPlan();
    P->n = n;
    P->nlevel = nl;
    // new front ids: level-major, parts in order within a level
    std::vector<std::vector<int>> nid(np);
    int nf = 0;
    P->lvl_off.assign(nl + 1, 0);
    for (int L = 0; L < nl; ++L) {
        P->lvl_off[L] = nf;
        for (int k = 0; k < np; ++k) {
            const MfPlan *Q = parts[k];
            if (nid[k].empty()) nid[k].assign(Q->nfront, -1);
            if (L >= Q->nlevel) continue;
            for (int q = Q->lvl_off[L]; q < Q->lvl_off[L + 1]; ++q) nid[k][q] = nf++;
        }
    }
    P->lvl_off[nl] = nf;
    P->nfront = nf;
    P->S.assign(nf, 0); P->f.assign(nf, 0); P->voff.assign(nf, 0); P->uoff.assign(nf, 0);
    P->child0.assign(nf, -1); P->child1.assign(nf, -1); P->parent.assign(nf, -1);
    P->foff.assign(nf, 0);
    std::vector<int> part_of(nf), old_of(nf);
    for (int k = 0; k < np; ++k)
        for (int q = 0; q < parts[k]->nfront; ++q) {
            part_of[nid[k][q]] = k;
            old_of[nid[k][q]] = q;
        }
    long long ftot = 0;
    int vtot = 0, utot = 0;
    for (int id = 0; id < nf; ++id) {
        const MfPlan *Q = parts[part_of[id]];
        const int q = old_of[id], k = part_of[id];
        P->S[id] = Q->S[q];
        P->f[id] = Q->f[q];
        P->voff[id] = vtot; vtot += Q->f[q];
        P->uoff[id] = utot; utot += Q->f[q] - Q->S[q];
        P->foff[id] = ftot; ftot += (long long)Q->f[q] * Q->f[q];
        if (Q->child0[q] >= 0) P->child0[id] = nid[k][Q->child0[q]];
        if (Q->child1[q] >= 0) P->child1[id] = nid[k][Q->child1[q]];
        if (Q->parent[q] >= 0) P->parent[id] = nid[k][Q->parent[q]];
        P->maxS = std::max(P->maxS, Q->S[q]);
        P->maxf = std::max(P->maxf, Q->f[q]);
        P->flops += 2.0 * Q->S[q] * (double)Q->f[q] * Q->f[q];
        P->factor_flops += front_flops(Q->S[q], Q->f[q]);
        P->apply_entries += (long long)Q->S[q] * (2LL * Q->f[q] - Q->S[q]);
    }
    P->ftotal = ftot; P->vtotal = vtot; P->utotal = utot;
    P->lvl_maxS.assign(nl, 0); P->lvl_maxf.assign(nl, 0); P->lvl_maxm.assign(nl, 0);
    P->lvl_maxm_child.assign(nl, 0);
    P->lvl_fbeg.assign(nl, 0); P->lvl_fend.assign(nl, 0);
    P->lvl_abeg.assign(nl, 0); P->lvl_aend.assign(nl, 0);
    P->toff.assign(nf, 0);
    P->goff.assign(nf, 0);
    for (int L = 0; L < nl; ++L) {
        const int a = P->lvl_off[L], b = P->lvl_off[L + 1];
        long long t = 0, g = 0;
        for (int id = a; id < b; ++id) {
            P->lvl_maxS[L] = std::max(P->lvl_maxS[L], P->S[id]);
            P->lvl_maxf[L] = std::max(P->lvl_maxf[L], P->f[id]);
            P->lvl_maxm[L] = std::max(P->lvl_maxm[L], P->f[id] - P->S[id]);
            for (int c : {P->child0[id], P->child1[id]})
                if (c >= 0) P->lvl_maxm_child[L] = std::max(P->lvl_maxm_child[L], P->f[c] - P->S[c]);
            P->toff[id] = t;
            t += (long long)P->S[id] * P->S[id];
            P->goff[id] = g;
            g += 2LL * P->S[id] * (P->f[id] - P->S[id]);
        }
        P->tmax = std::max(P->tmax, t);
        P->gmax = std::max(P->gmax, g);
        if (b > a) {
            P->lvl_fbeg[L] = P->foff[a];
            P->lvl_fend[L] = P->foff[b - 1] + (long long)P->f[b - 1] * P->f[b - 1];
        }
    }
    // front variables (shifted rows) and contribution maps (front-local)
    P->h_vars.resize(vtot);
    P->h_cbmap.resize(utot);
    for (int id = 0; id < nf; ++id) {
        const MfPlan *Q = parts[part_of[id]];
        const int q = old_of[id], ro = row_off[part_of[id]];
        for (int t = 0; t < Q->f[q]; ++t) P->h_vars[P->voff[id] + t] = Q->h_vars[Q->voff[q] + t] + ro;
        for (int t = 0; t < Q->f[q] - Q->S[q]; ++t)
            P->h_cbmap[P->uoff[id] + t] = Q->h_cbmap[Q->uoff[q] + t];
    }
    // assembly entries, level by level: each part's entries of the level with
    // shifted CSR entry, row and factor position (the front of an entry is
    // the one whose storage holds its position)
    long long nasm = 0;
    for (const MfPlan *Q : parts) nasm += Q->nasm;
    P->nasm = nasm;
    P->h_asm_csr.resize(nasm);
    P->h_asm_row.resize(nasm);
    P->h_asm_pos.resize(nasm);
    long long o = 0;
    for (int L = 0; L < nl; ++L) {
        P->lvl_abeg[L] = o;
        for (int k = 0; k < np; ++k) {
            const MfPlan *Q = parts[k];
            if (L >= Q->nlevel) continue;
            int q = Q->lvl_off[L];
            for (long long e = Q->lvl_abeg[L]; e < Q->lvl_aend[L]; ++e, ++o) {
                const long long pos = Q->h_asm_pos[e];
                while (q + 1 < Q->lvl_off[L + 1] && pos >= Q->foff[q + 1]) ++q;
                if (pos < Q->foff[q] || pos >= Q->foff[q] + (long long)Q->f[q] * Q->f[q]) {
                    set_error("mf_plan_forest: assembly entry outside its level's fronts");
                    mf_plan_destroy(P);
                    return V2D_EARG;
                }
                P->h_asm_csr[o] = (int)(Q->h_asm_csr[e] + nnz_off[k]);
                P->h_asm_row[o] = Q->h_asm_row[e] + row_off[k];
                P->h_asm_pos[o] = P->foff[nid[k][q]] + (pos - Q->foff[q]);
            }
        }
        P->lvl_aend[L] = o;
    }
    bool ok = o == nasm;
    for (int v : P->h_vars) ok = ok && v >= 0 && v < n;
    for (long long e = 0; e < nasm && ok; ++e)
        ok = P->h_asm_pos[e] >= 0 && P->h_asm_pos[e] < ftot && P->h_asm_row[e] >= 0 &&
             P->h_asm_row[e] < n && P->h_asm_csr[e] >= 0;
    if (!ok) {
        set_error("mf_plan_forest: index check failed");
        mf_plan_destroy(P);
        return V2D_EARG;
    }
    if (items_build(P) != V2D_OK) {
        mf_plan_destroy(P);
        return V2D_EARG;
    }
    V2D_TRY(mf_plan_upload(P));
    *out = P;
    return V2D_OK;
}

}  // namespace v2d

// Planning aid (no reference counterpart): runs only the host symbolic phase.
extern "C" int v2d_lu_plan_info(int imax, int jmax, const int *indptr, const int *indices,
                                int leaf, long long *out8)
{
    using namespace v2d;
    V2D_ARG_CHECK(indptr && indices && out8, "lu_plan_info: null pointer");
    MfPlan *P = nullptr;
    V2D_TRY(mf_plan_build(imax, jmax, 2 * imax * jmax, indptr, indices, leaf, &P));
    out8[0] = P->nfront;
    out8[1] = P->nlevel;
    out8[2] = P->maxS;
    out8[3] = P->maxf;
    out8[4] = P->ftotal;
    out8[5] = (long long)P->flops;
    out8[6] = P->vtotal;
    out8[7] = P->utotal;
    mf_plan_destroy(P);
    return V2D_OK;
}

// Planning aid for the solve's work items (host only): info4 = {work items,
// counters, fronts, levels}; when cap_items >= items, items gets 12 ints per
// item (kind 0 forward / 1 backward, front, first row, end row, wait counter
// and target, second wait counter and target, two done counters, 0, 0; -1
// for none); when cap_fronts >= fronts, fronts3 gets S, f and the parent of
// each front.
extern "C" int v2d_lu_solve_plan(int imax, int jmax, const int *indptr, const int *indices,
                                 int leaf, int *info4, int *items, int cap_items, int *fronts3,
                                 int cap_fronts)
{
    return v2d_lu_solve_plan_split(imax, jmax, indptr, indices, leaf, nullptr, 0, info4, items,
                                   cap_items, fronts3, cap_fronts);
}

extern "C" int v2d_lu_solve_plan_split(int imax, int jmax, const int *indptr, const int *indices,
                                       int leaf, const int *rows, int nrows, int *info4,
                                       int *items, int cap_items, int *fronts3, int cap_fronts)
{
    using namespace v2d;
    V2D_ARG_CHECK(indptr && indices && info4, "lu_solve_plan: null pointer");
    MfPlan *P = nullptr;
    V2D_TRY(mf_plan_build(imax, jmax, 2 * imax * jmax, indptr, indices, leaf, &P));
    if (rows) {
        if (nrows != P->nlevel) {
            set_error("lu_solve_plan: %d rows-per-item entries, the plan has %d levels", nrows,
                      P->nlevel);
            mf_plan_destroy(P);
            return V2D_EARG;
        }
        P->item_rows.assign(rows, rows + nrows);
        const int st = items_build(P);
        if (st != V2D_OK) {
            mf_plan_destroy(P);
            return st;
        }
    }
    info4[0] = P->nitems;
    info4[1] = P->nctr;
    info4[2] = P->nfront;
    info4[3] = P->nlevel;
    if (items && cap_items >= P->nitems) std::copy(P->h_items.begin(), P->h_items.end(), items);
    if (fronts3 && cap_fronts >= P->nfront)
        for (int q = 0; q < P->nfront; ++q) {
            fronts3[3 * q] = P->S[q];
            fronts3[3 * q + 1] = P->f[q];
            fronts3[3 * q + 2] = P->parent[q];
        }
    mf_plan_destroy(P);
    return V2D_OK;
}

namespace v2d {

// ================================================================ numeric
namespace {

constexpr int kMfThreads = 256;
constexpr int kGemmTile = 64;
constexpr int kTileStages = 2;   // operand slices in flight in the tile engine
// levels whose largest front has at least kDelayFront variables update the
// trailing block once per kDelayPanels panels (k_gemm)
constexpr int kDelayFront = 1024;
constexpr int kDelayPanels = 8;

template <class T> struct PanelWidth;
template <> struct PanelWidth<float> { static constexpr int v = 32; };
template <> struct PanelWidth<double> { static constexpr int v = 32; };

// rs[r] = 1 / max_c |a_rc| (1 for an empty row).
__global__ void k_rowscale(int n, const int *__restrict__ rowptr, const double *__restrict__ val,
                           double *rs)
{
    V2D_GRID_STRIDE(r, n)
    {
        double m = 0.0;
        for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) m = fmax(m, fabs(val[p]));
        rs[r] = m > 0.0 ? 1.0 / m : 1.0;
    }
}

template <class T>
__global__ void k_scatter(long long a0, long long a1, const int *__restrict__ csr,
                          const int *__restrict__ row, const long long *__restrict__ pos,
                          const double *__restrict__ val, const double *__restrict__ rs, T *F)
{
    for (long long e = a0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; e < a1;
         e += (long long)gridDim.x * blockDim.x)
        F[pos[e]] += (T)(val[csr[e]] * rs[row[e]]);
}

// Add child `slot`'s contribution block into each front of the level.
template <class T>
__global__ void k_extend_add(int q0, int slot, const int *__restrict__ S, const int *__restrict__ f,
                             const long long *__restrict__ foff, const int *__restrict__ uoff,
                             const int *__restrict__ child0, const int *__restrict__ child1,
                             const int *__restrict__ cbmap, T *F)
{
    const int P = q0 + blockIdx.y;
    const int c = slot == 0 ? child0[P] : child1[P];
    if (c < 0) return;
    const int Sc = S[c], fc = f[c], m = fc - Sc, fp = f[P];
    const T *src = F + foff[c];
    T *dst = F + foff[P];
    const int *map = cbmap + uoff[c];
    const long long tot = (long long)m * m;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(e / m), b = (int)(e - (long long)a * m);
        dst[(long long)map[a] * fp + map[b]] += src[(long long)(Sc + a) * fc + Sc + b];
    }
}

// Panel factorization of columns [k, k+w) of every front of the level with
// S > k.  One warp factors the w x w diagonal block in shared memory with
// partial pivoting restricted to the block's rows and records both the swap
// sequence (ipiv) and the block's part of the row permutation; the row scaling applied at
// assembly keeps the pivots meaningful and the FP64 Krylov iteration around
// the factors absorbs the weaker pivoting.  The rows below the block (fully
// summed and contribution rows alike) get their L entries from l21_rows.
// k_panel factors a level's first panel; every later panel is factored by
// the trailing update of the panel before it (k_gemm).
template <class T>
__device__ __forceinline__ void panel_factor(T *A, int f, int S, int k, int vo, int *ipiv,
                                             int *perm, int *flag,
                                             T (*U)[PanelWidth<T>::v + 1], int *pv)
{
    constexpr int NB = PanelWidth<T>::v;
    const int w = min(NB, S - k);
    const int tid = threadIdx.x, lane = tid & 31;
    for (int e = tid; e < NB * NB; e += blockDim.x) {
        const int r = e / NB, c = e - r * NB;
        U[r][c] = (r < w && c < w) ? A[(long long)(k + r) * f + k + c] : T(0);
    }
    __syncthreads();
    if (tid < 32) {
        // one warp; lane = row for the pivot search and the elimination,
        // lane = column for the row swap
        int bad = 0;
        if (lane < NB) pv[lane] = lane;
        __syncwarp();
        for (int c = 0; c < w; ++c) {
            T v = (lane >= c && lane < w) ? (T)fabs(U[lane][c]) : T(-1);
            int idx = lane;
            for (int o = 16; o > 0; o >>= 1) {
                const T ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
                if (ov > v || (ov == v && oi < idx)) {
                    v = ov;
                    idx = oi;
                }
            }
            int p = idx;
            if (!(v > T(0)) || p < c || p >= w) {
                p = c;
                bad = 1;
            }
            if (lane == 0) {
                ipiv[vo + k + c] = k + p;
                const int t = pv[c];
                pv[c] = pv[p];
                pv[p] = t;
            }
            if (p != c && lane < NB) {
                const T t = U[c][lane];
                U[c][lane] = U[p][lane];
                U[p][lane] = t;
            }
            __syncwarp();
            const T d = U[c][c];
            const T inv = d != T(0) ? T(1) / d : T(0);
            if (lane > c && lane < w) {
                const T l = U[lane][c] * inv;
                U[lane][c] = l;
                // eight entries per batch: their loads issue together (a store
                // to this lane's row may not be reordered with the next
                // entry's loads, so one entry at a time is a chain of
                // shared-memory round trips)
                int j = c + 1;
                for (; j + 7 < w; j += 8) {
                    T a[8], bv[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        a[u] = U[lane][j + u];
                        bv[u] = U[c][j + u];
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u) U[lane][j + u] = a[u] - l * bv[u];
                }
                for (; j < w; ++j) U[lane][j] -= l * U[c][j];
            }
            __syncwarp();
        }
        if (bad && lane == 0) atomicOr(flag, 1);
        // row i of the factored front came from local row perm[i]; the swaps
        // stay inside the panel's rows, so the panel fixes its own entries
        if (lane < w) perm[vo + k + lane] = k + pv[lane];
    }
    __syncthreads();
    for (int e = tid; e < w * w; e += blockDim.x) {
        const int r = e / w, c = e - r * w;
        A[(long long)(k + r) * f + k + c] = U[r][c];
    }
}

template <class T>
__global__ void __launch_bounds__(kMfThreads) k_panel(int q0, int k, const int *__restrict__ S_,
                                                      const int *__restrict__ f_,
                                                      const long long *__restrict__ foff,
                                                      const int *__restrict__ voff, T *F,
                                                      int *ipiv, int *perm, int *flag)
{
    constexpr int NB = PanelWidth<T>::v;
    __shared__ T U[NB][NB + 1];
    __shared__ int pv[NB];
    const int q = q0 + blockIdx.x;
    const int S = S_[q], f = f_[q];
    if (S <= k) return;
    panel_factor<T>(F + foff[q], f, S, k, voff[q], ipiv, perm, flag, U, pv);
}

// L entries of the panel for the rows below its diagonal block: x U = a with
// U the upper triangle of the factored block (no pivoting outside the block).
// Grid: (chunks of kL21Rows rows, fronts); one thread per row.
constexpr int kL21Rows = 64;

// L21 entries of row r: x U = a, U the upper triangle of the factored w x w
// diagonal block (in shared memory).
template <class T>
__device__ __forceinline__ void l21_row(T *A, int f, int k, int w, int r,
                                        const T (*U)[PanelWidth<T>::v + 1])
{
    constexpr int NB = PanelWidth<T>::v;
    T x[NB];
    T *row = A + (long long)r * f + k;
#pragma unroll
    for (int c = 0; c < NB; ++c) x[c] = c < w ? row[c] : T(0);
    // by rows of U: each finished entry updates the entries after it, so the
    // dependent chain is NB steps long, not NB^2 / 2 products
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        const T d = U[c][c];
        const T xc = (c < w && d != T(0)) ? x[c] / d : T(0);
        x[c] = xc;
#pragma unroll
        for (int j = c + 1; j < NB; ++j) x[j] -= xc * U[c][j];
    }
#pragma unroll
    for (int c = 0; c < NB; ++c)
        if (c < w) row[c] = x[c];
}

template <class T>
__device__ __forceinline__ void l21_rows(T *A, int f, int S, int k, int chunk,
                                         T (*U)[PanelWidth<T>::v + 1])
{
    constexpr int NB = PanelWidth<T>::v;
    const int w = min(NB, S - k);
    const int rbeg = k + w + chunk * kL21Rows;
    if (rbeg >= f) return;
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
        const int r = e / NB, c = e - r * NB;
        U[r][c] = (r < w && c < w) ? A[(long long)(k + r) * f + k + c] : T(0);
    }
    __syncthreads();
    const int r = rbeg + threadIdx.x;
    if (r >= f) return;
    l21_row<T>(A, f, k, w, r, U);
}

// The panel's row swaps (confined to its w rows) applied to every column
// outside the panel, then U12 = L11^-1 A12 for the panel's block row.  One
// thread per column: the w entries are gathered through the block
// permutation into registers, solved and written back.
// Column col outside the panel: the panel's row swaps (new row t = old row
// src[t]) applied to its w entries, then U12 = L11^-1 A12 for col >= k + w.
template <class T>
__device__ __forceinline__ void swap_trsm_col(T *A, int f, int k, int w, int col,
                                              const T (*Ld)[PanelWidth<T>::v + 1],
                                              const int *src)
{
    constexpr int NB = PanelWidth<T>::v;
    T x[NB];
#pragma unroll
    for (int t = 0; t < NB; ++t) x[t] = t < w ? A[(long long)(k + src[t]) * f + col] : T(0);
    if (col >= k + w) {
#pragma unroll
        for (int u = 0; u < NB - 1; ++u) {   // by columns of L: an NB-step chain
            const T xu = x[u];
#pragma unroll
            for (int t = u + 1; t < NB; ++t) x[t] -= Ld[t][u] * xu;
        }
    }
#pragma unroll
    for (int t = 0; t < NB; ++t)
        if (t < w) A[(long long)(k + t) * f + col] = x[t];
}

template <class T>
__device__ __forceinline__ void swap_trsm_cols(T *A, int f, int S, int k, int vo, int chunk,
                                               const int *__restrict__ ipiv,
                                               T (*Ld)[PanelWidth<T>::v + 1], int *src)
{
    constexpr int NB = PanelWidth<T>::v;
    const int w = min(NB, S - k);
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
        const int r = e / NB, c = e - r * NB;
        Ld[r][c] = (r < w && c < w) ? A[(long long)(k + r) * f + k + c] : T(0);
    }
    // the panel's pivot rows, loaded by the first NB threads at once (thread 0
    // loading them one after another would wait out NB dependent load
    // latencies), then new row t of the block = old row src[t]
    if (threadIdx.x < NB) src[NB + threadIdx.x] = threadIdx.x < w ? ipiv[vo + k + threadIdx.x] - k : 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int t = 0; t < NB; ++t) src[t] = t;
        for (int t = 0; t < w; ++t) {
            const int p = src[NB + t];
            const int u = src[t];
            src[t] = src[p];
            src[p] = u;
        }
    }
    __syncthreads();
    const int col = chunk * blockDim.x + threadIdx.x;
    if (col >= f || (col >= k && col < k + w)) return;
    swap_trsm_col<T>(A, f, k, w, col, Ld, src);
}

// Both panel steps that only read the factored diagonal block, in one launch:
// blocks [0, nl) compute L21 for kL21Rows rows each, blocks [nl, gridDim.x)
// apply the row swaps and U12 for kL21Rows columns each.  The two write
// disjoint parts of the front (rows below the block in its columns; the
// block's rows outside its columns) and read neither's output.
template <class T>
__global__ void __launch_bounds__(kL21Rows) k_l21_trsm(int q0, int k, int nl,
                                                       const int *__restrict__ S_,
                                                       const int *__restrict__ f_,
                                                       const long long *__restrict__ foff,
                                                       const int *__restrict__ voff, T *F,
                                                       const int *__restrict__ ipiv)
{
    constexpr int NB = PanelWidth<T>::v;
    __shared__ T D[NB][NB + 1];
    __shared__ int src[2 * NB];
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q];
    if (S <= k) return;
    T *A = F + foff[q];
    if ((int)blockIdx.x < nl)
        l21_rows<T>(A, f, S, k, blockIdx.x, D);
    else
        swap_trsm_cols<T>(A, f, S, k, voff[q], blockIdx.x - nl, ipiv, D, src);
}

// Accumulator of one 64 x 64 output tile of a CTA of 256 threads, fed NB-wide
// slices of its two operands through shared memory (Smem: a(rr, t) at
// refA, b(t, cc) at refB; staged by tile_mac, t fastest for A and cc fastest
// for B, then mac).
//   float:  CUDA cores, each thread 4 x 4 outputs (rows ty + 16 a, columns
//           tx + 16 b).
//   double: FP64 tensor cores, mma.sync m8n8k4 (the one FP64 tensor-core
//           instruction on sm_100a: tcgen05 has no FP64 kind).  Warp w owns
//           rows 32 (w / 4) .. + 32 and columns 16 (w % 4) .. + 16, i.e. 4 x 2
//           8x8 blocks; per k step of 4 a lane holds A[8 mi + g][t], the B
//           element [t][8 ni + g] and the outputs [8 mi + g][8 ni + 2 t + j]
//           (g = lane / 4, t = lane % 4).  Row strides of 36 and 72 doubles
//           spread a warp's 32 fragment reads evenly over the shared-memory
//           banks (two wavefronts, the minimum for 256 bytes).
template <class T> struct TileAcc;

template <> struct TileAcc<float> {
    static constexpr int NB = PanelWidth<float>::v, TL = kGemmTile;
    struct Smem {
        float A[NB][TL + 1];
        float B[NB][TL];
    };
    float acc[4][4];
    __device__ __forceinline__ static float &refA(Smem &s, int rr, int t) { return s.A[t][rr]; }
    __device__ __forceinline__ static float &refB(Smem &s, int t, int cc) { return s.B[t][cc]; }
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
    }
    __device__ __forceinline__ void mac(const Smem &s)
    {
        const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
#pragma unroll 4
        for (int t = 0; t < NB; ++t) {
            float av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = s.A[t][ty + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = s.B[t][tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
        }
    }
    // fn(rr, cc, value) for every output of the thread
    template <class Fn> __device__ __forceinline__ void each(Fn fn) const
    {
        const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) fn(ty + 16 * a, tx + 16 * b, acc[a][b]);
    }
};

__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <> struct TileAcc<double> {
    static constexpr int NB = PanelWidth<double>::v, TL = kGemmTile;
    struct Smem {
        double A[TL][NB + 4];
        double B[NB][TL + 8];
    };
    double acc[4][2][2];
    __device__ __forceinline__ static double &refA(Smem &s, int rr, int t) { return s.A[rr][t]; }
    __device__ __forceinline__ static double &refB(Smem &s, int t, int cc) { return s.B[t][cc]; }
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    }
    __device__ __forceinline__ void mac(const Smem &s)
    {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
        const int wr = (w >> 2) * 32, wc = (w & 3) * 16;
#pragma unroll
        for (int k = 0; k < NB; k += 4) {
            double a[4], b[2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) a[mi] = s.A[wr + 8 * mi + g][k + t];
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) b[ni] = s.B[k + t][wc + 8 * ni + g];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
                    dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
    }
    template <class Fn> __device__ __forceinline__ void each(Fn fn) const
    {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
        const int wr = (w >> 2) * 32, wc = (w & 3) * 16;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni)
#pragma unroll
                for (int j = 0; j < 2; ++j)
                    fn(wr + 8 * mi + g, wc + 8 * ni + 2 * t + j, acc[mi][ni][j]);
    }
};

// Asynchronous global -> shared copy of one element (cp.async, L1-allocating
// form: 4- and 8-byte copies need no 16-byte alignment, so any row stride
// works); ok == false writes zero and reads nothing.
template <class T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src, bool ok)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src),
                 "n"((int)sizeof(T)), "r"(ok ? (int)sizeof(T) : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// acc += sum over k in [ka, kb) of a(rr, k) b(k, cc), in NB-wide slices
// through kTileStages shared buffers (sm[0 .. kTileStages)): the copies of
// the next kTileStages - 1 slices are in flight while the tensor cores (or
// CUDA cores) work on slice s.  Two buffers leave room for three CTAs per SM
// in FP64, which hide the copies' latency better than a third buffer.  srcA(rr, k)
// and srcB(k, cc) give the element's address or nullptr (zero); oneA(rr, k)
// and oneB(k, cc) mark entries that are 1 instead (a unit diagonal), written
// after the slice's copies have landed.  base: any valid address (the source
// of zero-filled copies, never read).
struct NoOnes {
    __device__ __forceinline__ bool operator()(int, int) const { return false; }
};

template <class T, class SA, class SB, class OB, class OA = NoOnes>
__device__ __forceinline__ void tile_mac(TileAcc<T> &acc, typename TileAcc<T>::Smem *sm, int ka,
                                         int kb, const T *base, SA srcA, SB srcB, OB oneB,
                                         OA oneA = OA())
{
    constexpr int NB = PanelWidth<T>::v;
    constexpr int TL = kGemmTile;
    const int tid = threadIdx.x;
    const int ns = (kb - ka + NB - 1) / NB;
    auto stage = [&](int sl) {
        const int k = ka + sl * NB;
        typename TileAcc<T>::Smem &b = sm[sl % kTileStages];
        for (int e = tid; e < TL * NB; e += blockDim.x) {
            const int rr = e / NB, t = e - rr * NB;
            const T *p = k + t < kb ? srcA(rr, k + t) : nullptr;
            cp_async_elem(&TileAcc<T>::refA(b, rr, t), p ? p : base, p != nullptr);
        }
        for (int e = tid; e < NB * TL; e += blockDim.x) {
            const int t = e / TL, cc = e - t * TL;
            const T *p = k + t < kb ? srcB(k + t, cc) : nullptr;
            cp_async_elem(&TileAcc<T>::refB(b, t, cc), p ? p : base, p != nullptr);
        }
        cp_async_commit();
    };
    auto ones = [&](int sl) {
        const int k = ka + sl * NB;
        typename TileAcc<T>::Smem &b = sm[sl % kTileStages];
        for (int e = tid; e < NB * TL; e += blockDim.x) {
            const int t = e / TL, cc = e - t * TL;
            if (k + t < kb && oneB(k + t, cc)) TileAcc<T>::refB(b, t, cc) = T(1);
        }
        for (int e = tid; e < TL * NB; e += blockDim.x) {
            const int rr = e / NB, t = e - rr * NB;
            if (k + t < kb && oneA(rr, k + t)) TileAcc<T>::refA(b, rr, t) = T(1);
        }
    };
    static_assert(kTileStages == 2 || kTileStages == 3, "two or three stages");
    for (int p = 0; p < kTileStages - 1 && p < ns; ++p) stage(p);
    for (int sl = 0; sl < ns; ++sl) {
        // slice sl has landed once at most the later slices already issued pend
        if (kTileStages == 3 && sl + 1 < ns) cp_async_wait<kTileStages - 2>();
        else cp_async_wait<0>();
        ones(sl);
        __syncthreads();
        // the buffer of slice sl + kTileStages - 1 held slice sl - 1, which
        // every thread finished before the barrier above
        if (sl + kTileStages - 1 < ns) stage(sl + kTileStages - 1);
        acc.mac(sm[sl % kTileStages]);
    }
    __syncthreads();   // the buffers may be reused after the last slice
}

// One 64 x 64 tile of a trailing update: A[r][c] -= sum_{t in [ka, kb)}
// A[r][t] A[t][c] for rows [r0, min(r0 + 64, r1)) and columns
// [c0, min(c0 + 64, c1)).
template <class T>
__device__ __forceinline__ void gemm_tile_range(T *A, int f, int r0, int r1, int c0, int c1,
                                                int ka, int kb, typename TileAcc<T>::Smem *sm)
{
    TileAcc<T> acc;
    acc.zero();
    tile_mac<T>(
        acc, sm, ka, kb, A,
        [&](int rr, int k) -> const T * {
            const int r = r0 + rr;
            return r < r1 ? A + (long long)r * f + k : nullptr;
        },
        [&](int k, int cc) -> const T * {
            const int c = c0 + cc;
            return c < c1 ? A + (long long)k * f + c : nullptr;
        },
        [](int, int) { return false; });
    acc.each([&](int rr, int cc, T v) {
        const int r = r0 + rr, c = c0 + cc;
        if (r < r1 && c < c1) A[(long long)r * f + c] -= v;
    });
}

// dynamic shared memory of the tile engine's kernels: the operand buffers
template <class T> constexpr size_t tile_smem_bytes()
{
    return kTileStages * sizeof(typename TileAcc<T>::Smem);
}

// Trailing updates after panel [k, k + w), with delayed updates in
// super-panels of W columns (a multiple of NB; W = NB is the plain
// right-looking scheme).  Within the super-panel [k0, E), E = min(k0 + W, S),
// the panel's rank-w update goes only to the super-panel's remaining columns
// [kn, E) (all rows below, kn = k + w), and the next panel's rows [kn,
// kn + w') of the columns beyond it get the delayed contributions of the
// super-panel's panels so far (rank kn - k0), so that the next panel's swaps
// and U12 see updated rows; after the super-panel's last panel, one rank-W
// update covers rows and columns [E, f).  A big trailing block is then read
// and written once per W columns instead of once per panel.  Tiles are
// numbered per front for whichever case applies to it; the tile holding the
// next panel's diagonal block (the first one) factors that panel after its
// update (panel_factor), which saves the next step's panel launch.
template <class T>
__global__ void __launch_bounds__(256) k_gemm(int q0, int k, int W, const int *__restrict__ S_,
                                              const int *__restrict__ f_,
                                              const long long *__restrict__ foff,
                                              const int *__restrict__ voff, T *F, int *ipiv,
                                              int *perm, int *flag)
{
    constexpr int NB = PanelWidth<T>::v;
    constexpr int TL = kGemmTile;
    extern __shared__ __align__(16) unsigned char tile_raw[];
    typename TileAcc<T>::Smem *sm = reinterpret_cast<typename TileAcc<T>::Smem *>(tile_raw);
    // the next panel's block and pivots reuse the operand buffers once the
    // tile is done
    T(*U)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(tile_raw);
    int *pv = reinterpret_cast<int *>(tile_raw + sizeof(T) * NB * (NB + 1));
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q];
    if (S <= k) return;
    const int w = min(NB, S - k), kn = k + w;
    const int k0 = (k / W) * W, E = min(k0 + W, S);
    T *A = F + foff[q];
    int t = blockIdx.x;
    bool first = false;
    if (kn < E) {
        const int nr = (f - kn + TL - 1) / TL, nc = (E - kn + TL - 1) / TL;
        if (t < nr * nc) {
            gemm_tile_range<T>(A, f, kn + (t / nc) * TL, f, kn + (t % nc) * TL, E, k, kn, sm);
            first = t == 0;
        } else {
            t -= nr * nc;
            const int wn = min(NB, S - kn), nf = (f - E + TL - 1) / TL;
            if (t >= nf) return;
            gemm_tile_range<T>(A, f, kn, kn + wn, E + t * TL, f, k0, kn, sm);
        }
    } else {
        const int rem = f - E;
        if (rem <= 0) return;
        const int nt = (rem + TL - 1) / TL;
        if (t >= nt * nt) return;
        gemm_tile_range<T>(A, f, E + (t / nt) * TL, f, E + (t % nt) * TL, f, k0, E, sm);
        first = t == 0;
    }
    if (first && kn < S) {
        __syncthreads();   // the tile's updated entries are visible to the block
        panel_factor<T>(A, f, S, kn, voff[q], ipiv, perm, flag, U, pv);
    }
}

// Explicit inverses of the factored S x S block of every front of a level:
// strictly lower part <- L11^-1 (unit diagonal implied), upper part incl. the
// diagonal <- U11^-1, written to the level's scratch and copied back by
// k_trcopy.  One CTA per (front, column block of CW columns); the column
// block of each inverse is solved against the identity right-looking: the CTA
// keeps the S x CW block in shared memory, solves one 32-row diagonal block
// (one thread per column), then updates every remaining row with a rank-32
// product (all threads).  With the inverses the solve applies each front by
// row-parallel products instead of a chain of dependent triangular blocks.
constexpr int kTrinvThreads = 512;
// levels with more column blocks than SMs launch k_trinv with this many
// threads: at about 100 (FP32) / 128 (FP64) registers a 512-thread CTA fills
// an SM's register file alone, 128-thread CTAs fit four or five per SM, and
// on those levels resident CTAs matter more than the row updates' thread
// count
constexpr int kTrinvThreadsMany = 128;
constexpr int kTrinvManyCtas = 148;
template <class T> struct InvWidth;
template <> struct InvWidth<float> { static constexpr int v = 32; };
template <> struct InvWidth<double> { static constexpr int v = 16; };

// Columns [c0, c0 + CW) of L11^-1 (unit lower) and U11^-1 of one front's
// factored pivot block, into X (S x S, row-major); Xs (S x CW) and Lp (S x 33)
// in shared memory, Dg a 32 x 33 shared tile.
template <class T>
__device__ __forceinline__ void trinv_colblock(const T *A, int S, int f, T *X, int c0, T *Xs,
                                               T *Lp, T (*Dg)[33])
{
    constexpr int CW = InvWidth<T>::v;
    const int cw = min(CW, S - c0);
    const int tid = threadIdx.x;
    // ---------------- L11^-1 (unit lower): rows [c0, S)
    for (int e = tid; e < S * CW; e += blockDim.x) {
        const int r = e / CW, cc = e - r * CW;
        Xs[e] = (r == c0 + cc) ? T(1) : T(0);
    }
    __syncthreads();
    for (int r0 = (c0 / 32) * 32; r0 < S; r0 += 32) {
        const int bh = min(32, S - r0);
        // the diagonal block and the L panel below it do not depend on each
        // other: load both in one phase
        const int rows = S - r0 - bh;
        for (int e = tid; e < 1024; e += blockDim.x) {
            const int rr = e >> 5, cc = e & 31;
            Dg[rr][cc] = (rr < bh && cc < bh) ? A[(long long)(r0 + rr) * f + r0 + cc] : T(0);
        }
        for (int e = tid; e < rows * 32; e += blockDim.x) {    // stage L[r0+bh.., r0..r0+32)
            const int rr = e >> 5, t = e & 31;
            Lp[rr * 33 + t] = t < bh ? A[(long long)(r0 + bh + rr) * f + r0 + t] : T(0);
        }
        __syncthreads();
        if (tid < CW) {   // diagonal block, one thread per column, column in registers
            T xr[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) xr[r] = r < bh ? Xs[(r0 + r) * CW + tid] : T(0);
#pragma unroll
            for (int t = 0; t < 31; ++t) {   // by columns: a 31-step chain
                const T xt = xr[t];
#pragma unroll
                for (int r = t + 1; r < 32; ++r) xr[r] -= Dg[r][t] * xt;
            }
#pragma unroll
            for (int r = 1; r < 32; ++r)
                if (r < bh) Xs[(r0 + r) * CW + tid] = xr[r];
        }
        __syncthreads();
        for (int e = tid; e < rows * CW; e += blockDim.x) {   // rank-bh update below
            const int rr = e / CW, cc = e % CW;
            const T *lr = Lp + rr * 33;
            T v0 = T(0), v1 = T(0);
            int t = 0;
            for (; t + 1 < bh; t += 2) {   // rows r0 .. r0+bh-1 of Xs only
                v0 += lr[t] * Xs[(r0 + t) * CW + cc];
                v1 += lr[t + 1] * Xs[(r0 + t + 1) * CW + cc];
            }
            if (t < bh) v0 += lr[t] * Xs[(r0 + t) * CW + cc];
            Xs[(r0 + bh + rr) * CW + cc] -= v0 + v1;
        }
        __syncthreads();
    }
    for (int e = tid; e < S * CW; e += blockDim.x) {
        const int r = e / CW, cc = e - r * CW;
        if (cc < cw && r > c0 + cc) X[(long long)r * S + c0 + cc] = Xs[e];
    }
    __syncthreads();
    // ---------------- U11^-1 (upper): rows [0, c0 + cw)
    const int rtop = c0 + cw;
    for (int e = tid; e < rtop * CW; e += blockDim.x) {
        const int r = e / CW, cc = e - r * CW;
        Xs[e] = (r == c0 + cc) ? T(1) : T(0);
    }
    __syncthreads();
    for (int r0 = ((rtop - 1) / 32) * 32; r0 >= 0; r0 -= 32) {
        const int r1 = min(r0 + 32, rtop);
        const int bh = r1 - r0;
        for (int e = tid; e < 1024; e += blockDim.x) {
            const int rr = e >> 5, cc = e & 31;
            Dg[rr][cc] = (rr < bh && cc < bh) ? A[(long long)(r0 + rr) * f + r0 + cc] : T(0);
        }
        for (int e = tid; e < r0 * 32; e += blockDim.x) {      // stage U[0..r0, r0..r0+32)
            const int rr = e >> 5, t = e & 31;
            Lp[rr * 33 + t] = t < bh ? A[(long long)rr * f + r0 + t] : T(0);
        }
        __syncthreads();
        if (tid < CW) {   // column in registers
            T xr[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) xr[r] = r < bh ? Xs[(r0 + r) * CW + tid] : T(0);
#pragma unroll
            for (int t = 31; t >= 0; --t) {   // by columns, from the bottom row up
                if (t < bh) {
                    const T d = Dg[t][t];
                    const T xt = d != T(0) ? xr[t] / d : T(0);
                    xr[t] = xt;
#pragma unroll
                    for (int r = 0; r < t; ++r) xr[r] -= Dg[r][t] * xt;
                }
            }
#pragma unroll
            for (int r = 0; r < 32; ++r)
                if (r < bh) Xs[(r0 + r) * CW + tid] = xr[r];
        }
        __syncthreads();
        for (int e = tid; e < r0 * CW; e += blockDim.x) {   // rank update above
            const int r = e / CW, cc = e % CW;
            const T *ur = Lp + r * 33;
            T v0 = T(0), v1 = T(0);
            int t = 0;
            for (; t + 1 < bh; t += 2) {   // rows r0 .. r0+bh-1 of Xs only
                v0 += ur[t] * Xs[(r0 + t) * CW + cc];
                v1 += ur[t + 1] * Xs[(r0 + t + 1) * CW + cc];
            }
            if (t < bh) v0 += ur[t] * Xs[(r0 + t) * CW + cc];
            Xs[r * CW + cc] -= v0 + v1;
        }
        __syncthreads();
    }
    for (int e = tid; e < rtop * CW; e += blockDim.x) {
        const int r = e / CW, cc = e - r * CW;
        if (cc < cw && r <= c0 + cc) X[(long long)r * S + c0 + cc] = Xs[e];
    }
}

template <class T>
__global__ void __launch_bounds__(kTrinvThreads) k_trinv(int q0, const int *__restrict__ S_,
                                                         const long long *__restrict__ foff,
                                                         const int *__restrict__ f_,
                                                         const long long *__restrict__ toff,
                                                         const T *__restrict__ F, T *tmp)
{
    constexpr int CW = InvWidth<T>::v;
    extern __shared__ unsigned char smem_raw[];
    T *Xs = reinterpret_cast<T *>(smem_raw);    // S x CW
    T *Lp = Xs + (size_t)S_[q0 + blockIdx.y] * CW;   // S x 33: the 32 columns of the current step
    __shared__ T Dg[32][33];                     // current 32 x 32 diagonal block
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q];
    const int c0 = blockIdx.x * CW;
    if (c0 >= S) return;
    trinv_colblock<T>(F + foff[q], S, f, tmp + toff[q], c0, Xs, Lp, Dg);
}

// The same inversion for separators whose column block does not fit in
// shared memory: the S x CW block and the S x 33 panel live in a global work
// space, one slice of S x (CW + 33) per CTA (sstride elements apart).
constexpr size_t kInvSmemMax = 200 * 1024;
// grids with one y index per front take at most this many fronts per launch
// (the grid's y dimension is limited to 65535)
constexpr int kMaxFrontsY = 65535;
constexpr int kTrinvThreadsG = 256;

template <class T>
__global__ void __launch_bounds__(kTrinvThreadsG) k_trinv_g(int q0, const int *__restrict__ S_,
                                                           const long long *__restrict__ foff,
                                                           const int *__restrict__ f_,
                                                           const long long *__restrict__ toff,
                                                           const T *__restrict__ F, T *tmp,
                                                           T *work, long long sstride)
{
    constexpr int CW = InvWidth<T>::v;
    __shared__ T Dg[32][33];
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q];
    const int c0 = blockIdx.x * CW;
    if (c0 >= S) return;
    T *Xs = work + ((long long)blockIdx.y * gridDim.x + blockIdx.x) * sstride;
    T *Lp = Xs + (size_t)S * CW;
    trinv_colblock<T>(F + foff[q], S, f, tmp + toff[q], c0, Xs, Lp, Dg);
}

// Explicit inverses of separators too wide for the shared-memory column
// blocks (FP64), by 64 x 64 blocks on the tile engine.  With X = L11^-1 and
// Y = U11^-1 in blocks of 64 (nb blocks), X L11 = I and U11 Y = I give, for
// s = nb-2 down to 0,
//   X_is = -sum_{k=s+1..i} X_ik (L_ks X_ss)     (i > s, block column s)
//   Y_sj = -sum_{k=s+1..j} (Y_ss U_sk) Y_kj     (j > s, block row s)
// from blocks of later steps and the diagonal blocks' inverses X_kk (unit
// diagonal, stored strictly below it) and Y_kk.  k_trinv_diag inverts every
// diagonal block; each step is two launches of k_trinv_step: phase 0 forms
// W_k = L_ks X_ss and V_sk = Y_ss U_sk in place of L_ks and U_sk (read by
// this step only; the whole pivot block is replaced by k_trcopy afterwards),
// phase 1 the products.  Results go to the level's scratch like k_trinv's.
constexpr int kInvBlk = 64;   // the tile engine's tile
// separators from this width on are inverted by blocks (fewer dependent
// steps per CTA than the column-block solves; measured on 362-wide ones)
constexpr int kBlockedInvMinS = 256;
constexpr int kTrinvDiagThreads = 128;

template <class T> constexpr size_t trinv_diag_smem() { return 3 * kInvBlk * (kInvBlk + 1) * sizeof(T); }

template <class T>
__global__ void __launch_bounds__(kTrinvDiagThreads) k_trinv_diag(int q0, const int *__restrict__ S_,
                                                                  const int *__restrict__ f_,
                                                                  const long long *__restrict__ foff,
                                                                  const long long *__restrict__ toff,
                                                                  const T *__restrict__ F, T *tmp)
{
    constexpr int B = kInvBlk;
    extern __shared__ __align__(16) unsigned char diag_raw[];
    T (*Ab)[B + 1] = reinterpret_cast<T (*)[B + 1]>(diag_raw);
    T (*Xs)[B + 1] = Ab + B;
    T (*Ys)[B + 1] = Xs + B;
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q], s0 = blockIdx.x * B;
    if (s0 >= S) return;
    const int bs = min(B, S - s0), tid = threadIdx.x;
    const T *A = F + foff[q] + (long long)s0 * f + s0;
    for (int e = tid; e < B * B; e += blockDim.x) {
        const int r = e / B, c = e - r * B;
        Ab[r][c] = (r < bs && c < bs) ? A[(long long)r * f + c] : T(0);
    }
    __syncthreads();
    // One column of an inverse per thread, held in registers and solved by
    // columns of the block (each finished entry updates all rows after it):
    // the dependent chain is B steps long instead of B^2 / 2 dependent
    // products through shared memory.  The padding beyond bs is zero and
    // leaves the solution's zeros in place.
    const int c = tid & (B - 1);
    if (c < bs) {
        T x[B];
#pragma unroll
        for (int r = 0; r < B; ++r) x[r] = r == c ? T(1) : T(0);
        if (tid < B) {   // column c of L^-1 (unit lower): L x = e_c
#pragma unroll
            for (int t = 0; t < B - 1; ++t) {
                const T xt = x[t];
#pragma unroll
                for (int r = t + 1; r < B; ++r) x[r] -= Ab[r][t] * xt;
            }
#pragma unroll
            for (int r = 0; r < B; ++r) Xs[r][c] = x[r];
        } else {         // column c of U^-1: U x = e_c from the bottom row up
#pragma unroll
            for (int t = B - 1; t >= 0; --t) {
                const T d = Ab[t][t];
                const T xt = d != T(0) ? x[t] / d : T(0);
                x[t] = xt;
#pragma unroll
                for (int r = 0; r < t; ++r) x[r] -= Ab[r][t] * xt;
            }
#pragma unroll
            for (int r = 0; r < B; ++r) Ys[r][c] = x[r];
        }
    }
    __syncthreads();
    T *X = tmp + toff[q] + (long long)s0 * S + s0;
    for (int e = tid; e < bs * bs; e += blockDim.x) {
        const int r = e / bs, cc = e - r * bs;
        X[(long long)r * S + cc] = r > cc ? Xs[r][cc] : Ys[r][cc];
    }
}

// One step s of the blocked inversion (see k_trinv_diag); grid: (2 half,
// fronts), tiles [0, half) the blocks k = s + 1 + t of L's block column s,
// [half, 2 half) those of U's block row s.
template <class T>
__global__ void __launch_bounds__(256) k_trinv_step(int q0, int s, int phase, int half,
                                                    const int *__restrict__ S_,
                                                    const int *__restrict__ f_,
                                                    const long long *__restrict__ foff,
                                                    const long long *__restrict__ toff, T *F,
                                                    T *tmp)
{
    constexpr int B = kInvBlk;
    extern __shared__ __align__(16) unsigned char tile_raw[];
    typename TileAcc<T>::Smem *sm = reinterpret_cast<typename TileAcc<T>::Smem *>(tile_raw);
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q], nb = (S + B - 1) / B;
    int t = blockIdx.x;
    const bool up = t >= half;
    if (up) t -= half;
    const int k = s + 1 + t;
    if (k >= nb) return;
    T *A = F + foff[q];
    T *X = tmp + toff[q];
    const int s0 = s * B, k0 = k * B, se = s0 + B, ke = min(k0 + B, S);
    TileAcc<T> acc;
    acc.zero();
    if (phase == 0 && !up) {          // W_k = L_ks X_ss (in place of L_ks)
        tile_mac<T>(
            acc, sm, s0, se, A,
            [&](int rr, int j) -> const T * {
                const int r = k0 + rr;
                return r < ke ? A + (long long)r * f + j : nullptr;
            },
            [&](int j, int cc) -> const T * {
                return j > s0 + cc ? X + (long long)j * S + s0 + cc : nullptr;
            },
            [&](int j, int cc) { return j == s0 + cc; });
        acc.each([&](int rr, int cc, T v) {
            if (k0 + rr < ke) A[(long long)(k0 + rr) * f + s0 + cc] = v;
        });
    } else if (phase == 0) {          // V_sk = Y_ss U_sk (in place of U_sk)
        tile_mac<T>(
            acc, sm, s0, se, A,
            [&](int rr, int j) -> const T * {
                return j >= s0 + rr ? X + (long long)(s0 + rr) * S + j : nullptr;
            },
            [&](int j, int cc) -> const T * {
                const int c = k0 + cc;
                return c < ke ? A + (long long)j * f + c : nullptr;
            },
            NoOnes());
        acc.each([&](int rr, int cc, T v) {
            if (k0 + cc < ke) A[(long long)(s0 + rr) * f + k0 + cc] = v;
        });
    } else if (!up) {                 // X_ks = -sum_{m=s+1..k} X_km W_m
        tile_mac<T>(
            acc, sm, se, ke, A,
            [&](int rr, int j) -> const T * {
                const int r = k0 + rr;
                if (r >= ke || (j >= k0 && j >= r)) return nullptr;   // X_kk: strictly lower
                return X + (long long)r * S + j;
            },
            [&](int j, int cc) -> const T * { return A + (long long)j * f + s0 + cc; },
            NoOnes(), [&](int rr, int j) { return k0 + rr == j; });
        acc.each([&](int rr, int cc, T v) {
            if (k0 + rr < ke) X[(long long)(k0 + rr) * S + s0 + cc] = -v;
        });
    } else {                          // Y_sk = -sum_{m=s+1..k} V_sm Y_mk
        tile_mac<T>(
            acc, sm, se, ke, A,
            [&](int rr, int j) -> const T * { return A + (long long)(s0 + rr) * f + j; },
            [&](int j, int cc) -> const T * {
                const int c = k0 + cc;
                if (c >= ke || (j >= k0 && j > c)) return nullptr;    // Y_kk: upper
                return X + (long long)j * S + c;
            },
            NoOnes());
        acc.each([&](int rr, int cc, T v) {
            if (k0 + cc < ke) X[(long long)(s0 + rr) * S + k0 + cc] = -v;
        });
    }
}

// Inverted S x S blocks of the level's fronts: scratch -> factor storage.
template <class T>
__global__ void k_trcopy(int q0, const int *__restrict__ S_, const int *__restrict__ f_,
                         const long long *__restrict__ foff, const long long *__restrict__ toff,
                         const T *__restrict__ tmp, T *F)
{
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q];
    const T *src = tmp + toff[q];
    T *dst = F + foff[q];
    const long long tot = (long long)S * S;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e / S), c = (int)(e - (long long)r * S);
        dst[(long long)r * f + c] = src[e];
    }
}

// FP64 factors rounded to FP32 (the solve of the mixed form with FP64
// factorization).
__global__ void k_round_f32(const double *__restrict__ a, float *__restrict__ b, long long n)
{
    V2D_GRID_STRIDE(i, n) { b[i] = (float)a[i]; }
}

// G = L21 L11^-1 (rows [S, f) x columns [0, S)) and H = U11^-1 U12 (rows
// [0, S) x columns [S, f)) of every front of a level, from the inverted pivot
// block, into the level's scratch (G row-major m x S, then H S x m; copied over
// L21 and U12 by k_ghcopy: each tile of G reads L21 entries that other tiles
// overwrite).  One CTA per 64 x 64 output tile (TileAcc: CUDA cores in FP32,
// FP64 tensor cores in FP64); the triangular factor bounds the inner range (G: k >= c0,
// with L11^-1's unit diagonal; H: k >= r0).  Grid: (tiles of G then of H for
// the level's largest front, fronts).
template <class T>
__global__ void __launch_bounds__(256) k_gh(int q0, const int *__restrict__ S_,
                                            const int *__restrict__ f_,
                                            const long long *__restrict__ foff,
                                            const long long *__restrict__ goff, const T *F, T *gh)
{
    constexpr int TL = kGemmTile;
    extern __shared__ __align__(16) unsigned char tile_raw[];
    typename TileAcc<T>::Smem *sm = reinterpret_cast<typename TileAcc<T>::Smem *>(tile_raw);
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q], m = f - S;
    if (m <= 0) return;
    const int ts = (S + TL - 1) / TL, tm = (m + TL - 1) / TL;
    int t = blockIdx.x;
    const bool isG = t < tm * ts;
    if (!isG) t -= tm * ts;
    if (t >= tm * ts) return;
    const T *A = F + foff[q];
    T *out = gh + goff[q];
    int r0, c0, kb;
    if (isG) {
        r0 = S + (t / ts) * TL;
        c0 = (t % ts) * TL;
        kb = c0;
    } else {
        r0 = (t / tm) * TL;
        c0 = S + (t % tm) * TL;
        kb = r0;
    }
    TileAcc<T> acc;
    acc.zero();
    // G: L21 rows times L11^-1 (strictly lower part stored, unit diagonal);
    // H: U11^-1 (upper part with the diagonal) times U12
    tile_mac<T>(
        acc, sm, kb, S, A,
        [&](int rr, int kk) -> const T * {
            const int r = r0 + rr;
            return (isG ? r < f : (r < S && kk >= r)) ? A + (long long)r * f + kk : nullptr;
        },
        [&](int kk, int cc) -> const T * {
            const int c = c0 + cc;
            return (isG ? (c < S && kk > c) : c < f) ? A + (long long)kk * f + c : nullptr;
        },
        [&](int kk, int cc) { return isG && kk == c0 + cc; });
    acc.each([&](int rr, int cc, T v) {
        const int r = r0 + rr, col = c0 + cc;
        if (isG) {
            if (r < f && col < S) out[(long long)(r - S) * S + col] = v;
        } else if (r < S && col < f) {
            out[(long long)m * S + (long long)r * m + (col - S)] = v;
        }
    });
}

// G and H of the level's fronts: scratch -> factor storage.
template <class T>
__global__ void k_ghcopy(int q0, const int *__restrict__ S_, const int *__restrict__ f_,
                         const long long *__restrict__ foff, const long long *__restrict__ goff,
                         const T *__restrict__ gh, T *F)
{
    const int q = q0 + blockIdx.y;
    const int S = S_[q], f = f_[q], m = f - S;
    const T *src = gh + goff[q];
    T *dst = F + foff[q];
    const long long ng = (long long)m * S, tot = 2 * ng;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        long long r, c;
        if (e < ng) {
            r = S + e / S;
            c = e % S;
        } else {
            r = (e - ng) / m;
            c = S + (e - ng) % m;
        }
        dst[r * f + c] = src[e];
    }
}

// ------------------------------------------------------------------ solve
// After the factorization each front's storage holds, row-major f x f:
//   [0,S) x [0,S)   L11^-1 strictly below the diagonal (unit diagonal implied)
//                   and U11^-1 on and above it,
//   [S,f) x [0,S)   G = L21 L11^-1,
//   [0,S) x [S,f)   H = U11^-1 U12,
// so every row of the solve is one contiguous dot product with a vector
// gathered once per work item:
//   forward,  r <  S:  z_r = t_r + F[r, 0:r] . t[0:r]      t = P w_FS (permuted)
//             r >= S:  u_r = w_r - F[r, 0:S] . t[0:S]      contribution to the parent
//   backward, r <  S:  x_r = F[r, r:f] . v[r:f]            v = (z, -x_struct)
// A front's forward rows need only its children's contributions and its
// backward rows only its own z and its ancestors' x: one dependent step per
// level and sweep.  G and H hold as many entries as L21 and U12, so a solve
// still reads sum S (2f - S) factor entries.

__device__ __forceinline__ bool stopped(const int *a, const int *b)
{
    return (a && *a) || (b && *b);
}

constexpr int kSolveThreads = kSolveThreadsHost;   // 8 warps per work item
constexpr int kFlowSlots = 3;   // ticket counters after the dependency counters
constexpr int kGatherRegs = 4;   // staged gather entries per thread (fronts up to 4 x 256)
constexpr int kThreadRowMaxF = 256;   // fronts whose forward rows a thread sums alone

// Row registers: a warp that computes a single row of an item loads it into
// registers before the item's dependency wait; rows up to kRowRegs<T> x 32
// entries (from a 32-aligned start).
template <class T> struct RowRegs;
template <> struct RowRegs<float> { static constexpr int v = 32; };
template <> struct RowRegs<double> { static constexpr int v = 16; };
// the three-CTAs-per-SM form of the dataflow solve: fewer row registers
template <class T> struct RowRegs3;
template <> struct RowRegs3<float> { static constexpr int v = 16; };
template <> struct RowRegs3<double> { static constexpr int v = 8; };

template <class T, int R>
__device__ __forceinline__ void row_load(T (&reg)[R], const T *row, int base, int lo, int hi)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int c = base + lane + 32 * k;
        reg[k] = (c >= lo && c < hi) ? row[c] : T(0);
    }
}

template <class T, int R>
__device__ __forceinline__ T row_dot_reg(const T (&reg)[R], const T *v, int base, int lo, int hi)
{
    const int lane = threadIdx.x & 31;
    T a0 = T(0), a1 = T(0);
#pragma unroll
    for (int k = 0; k < R; k += 2) {
        const int c = base + lane + 32 * k;
        if (c >= lo && c < hi) a0 += reg[k] * v[c];
        if (c + 32 >= lo && c + 32 < hi) a1 += reg[k + 1] * v[c + 32];
    }
    return warp_sum(a0 + a1);
}

// N rows' dot products by one warp at once: row u's entries [b_u, e_u) with
// v (an empty range for an absent row), all loads in flight together.  Each
// row has its own accumulator, so its sum does not depend on N.
template <class T, int N, int K = (N >= 8 ? 2 : 4)>
__device__ __forceinline__ void dotN(const T *const (&p)[N], const int (&b)[N], const int (&e)[N],
                                     const T *v, T (&s)[N])
{
    const int lane = threadIdx.x & 31;
    int lo = b[0], hi = e[0];
#pragma unroll
    for (int u = 1; u < N; ++u) {
        lo = min(lo, b[u]);
        hi = max(hi, e[u]);
    }
    // K column chunks of each of the N rows are loaded before any is used:
    // N * K loads of the factor rows in flight per lane
    T a[N];
#pragma unroll
    for (int u = 0; u < N; ++u) a[u] = T(0);
    int c = (lo & ~31) + lane;
    for (; c + 32 * (K - 1) < hi; c += 32 * K) {
        T xv[K], rv[N][K];
#pragma unroll
        for (int k = 0; k < K; ++k) xv[k] = v[c + 32 * k];
#pragma unroll
        for (int u = 0; u < N; ++u)
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int cc = c + 32 * k;
                rv[u][k] = (cc >= b[u] && cc < e[u]) ? p[u][cc] : T(0);
            }
#pragma unroll
        for (int u = 0; u < N; ++u)
#pragma unroll
            for (int k = 0; k < K; ++k) a[u] += rv[u][k] * xv[k];
    }
    for (; c < hi; c += 32) {
        const T x = v[c];
#pragma unroll
        for (int u = 0; u < N; ++u)
            if (c >= b[u] && c < e[u]) a[u] += p[u][c] * x;
    }
#pragma unroll
    for (int u = 0; u < N; ++u) s[u] = warp_sum(a[u]);
}

template <class T>
__device__ __forceinline__ void dot4(const T *const (&p)[4], const int (&b)[4], const int (&e)[4],
                                     const T *v, T (&s)[4])
{
    dotN<T, 4>(p, b, e, v, s);
}

// Column range of row r of front (S, f) in the forward (fwd) or backward sweep.
__device__ __forceinline__ void row_range(bool fwd, int r, int S, int f, int &lo, int &hi)
{
    if (fwd) {
        lo = 0;
        hi = r < S ? r : S;
    } else {
        lo = r;
        hi = f;
    }
}

// A work item: rows [rbeg, rend) of front q in one sweep.  The parts that
// depend on no other item (indices, scaled right-hand side, the single row a
// warp owns) are loaded by pre(); run() then gathers the vector the rows
// multiply (after the item's dependencies are met) and computes the rows.
template <class T, int R = RowRegs<T>::v>
struct SolveItemCtx {
    bool fwd;
    int kind;    // 0 forward rows, 1 backward rows, 2 forward gather, 3 backward gather
    bool gath;   // rows of a front whose gather item ran (its vectors are in tw)
    int q, S, f, vo, rbeg, rend;
    const T *A;
    // staged gather (forward: vars/perm/child maps; backward: struct vars)
    bool staged;
    int ch[2], m[2], uof[2];
    int pi[kGatherRegs], mp[2][kGatherRegs], xi[kGatherRegs];
    T rsb[kGatherRegs];
    // this warp's single row, if the item has at most one row per warp
    bool onerow;
    int base;
    T reg[R];

    __device__ __forceinline__ void pre(const MfDev &D, const T *F, const T *b,
                                        const double *__restrict__ rs, int kind_, int gath_,
                                        int q_, int rbeg_, int rend_)
    {
        kind = kind_;
        fwd = kind == 0 || kind == 2;
        gath = gath_ != 0 && kind < 2;
        q = q_;
        rbeg = rbeg_;
        rend = rend_;
        S = D.S[q];
        f = D.f[q];
        vo = D.voff[q];
        A = F + D.foff[q];
        const int tid = threadIdx.x, nt = blockDim.x, wid = tid >> 5, nw = nt >> 5;
        const int *vars = D.vars + vo;
        onerow = kind < 2 && rend - rbeg <= nw;
        const int r = rbeg + wid;
        if (onerow && r < rend) {
            int lo, hi;
            row_range(fwd, r, S, f, lo, hi);
            base = lo & ~31;
            if (hi - base <= 32 * R) row_load<T, R>(reg, A + (long long)r * f, base, lo, hi);
            else onerow = false;
        } else {
            onerow = false;
        }
        if (gath) {
            staged = false;   // the rows read the gather item's vectors
        } else if (fwd) {
            ch[0] = D.child0[q];
            ch[1] = D.child1[q];
            for (int sl = 0; sl < 2; ++sl) {
                m[sl] = ch[sl] >= 0 ? D.f[ch[sl]] - D.S[ch[sl]] : 0;
                uof[sl] = ch[sl] >= 0 ? D.uoff[ch[sl]] : 0;
            }
            staged = f <= kGatherRegs * nt && m[0] <= kGatherRegs * nt &&
                     m[1] <= kGatherRegs * nt;
            if (staged) {
                int vi[kGatherRegs];
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k) {
                    const int p = tid + k * nt;
                    vi[k] = p < S ? vars[p] : -1;
                    pi[k] = p < S ? D.perm[vo + p] : 0;
#pragma unroll
                    for (int sl = 0; sl < 2; ++sl) mp[sl][k] = p < m[sl] ? D.cbmap[uof[sl] + p] : 0;
                }
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k)
                    rsb[k] = vi[k] >= 0 ? (T)(rs[vi[k]] * (double)b[vi[k]]) : T(0);
            }
        } else {
            staged = f - S <= kGatherRegs * nt;
            if (staged) {
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k) {
                    const int e = tid + k * nt;
                    xi[k] = e < f - S ? vars[S + e] : 0;
                }
            }
        }
    }

    // Forward gather: w (f entries: scaled b on the fully summed rows plus
    // the children's contributions), t = P w_FS, in shared memory.
    __device__ __forceinline__ void gather_w(const MfDev &D, const T *b,
                                             const double *__restrict__ rs, const T *upd, T *w,
                                             T *t)
    {
        const int tid = threadIdx.x, nt = blockDim.x;
        if (staged) {
            T uv[2][kGatherRegs];
#pragma unroll
            for (int sl = 0; sl < 2; ++sl)
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k) {
                    const int e = tid + k * nt;
                    uv[sl][k] = e < m[sl] ? __ldcg(upd + uof[sl] + e) : T(0);
                }
#pragma unroll
            for (int k = 0; k < kGatherRegs; ++k) {
                const int p = tid + k * nt;
                if (p < f) w[p] = rsb[k];
            }
            __syncthreads();
#pragma unroll
            for (int sl = 0; sl < 2; ++sl) {
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k)
                    if (tid + k * nt < m[sl]) w[mp[sl][k]] += uv[sl][k];
                __syncthreads();
            }
#pragma unroll
            for (int k = 0; k < kGatherRegs; ++k)
                if (tid + k * nt < S) t[tid + k * nt] = w[pi[k]];
        } else {
            // wide fronts: the same in batches of kGatherRegs entries per
            // thread, each batch's index loads issued before its gathers
            const int *vars = D.vars + vo;
            for (int p0 = tid; p0 < f; p0 += kGatherRegs * nt) {
                int vi[kGatherRegs];
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k) {
                    const int p = p0 + k * nt;
                    vi[k] = p < S ? vars[p] : -1;
                }
                T val[kGatherRegs];
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k)
                    val[k] = vi[k] >= 0 ? (T)(rs[vi[k]] * (double)b[vi[k]]) : T(0);
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k)
                    if (p0 + k * nt < f) w[p0 + k * nt] = val[k];
            }
            __syncthreads();
            for (int sl = 0; sl < 2; ++sl) {
                const int *map = D.cbmap + uof[sl];
                const T *u = upd + uof[sl];
                for (int e0 = tid; e0 < m[sl]; e0 += kGatherRegs * nt) {
                    int mi[kGatherRegs];
                    T uv[kGatherRegs];
#pragma unroll
                    for (int k = 0; k < kGatherRegs; ++k) {
                        const int e = e0 + k * nt;
                        mi[k] = e < m[sl] ? map[e] : -1;
                        uv[k] = e < m[sl] ? __ldcg(u + e) : T(0);
                    }
#pragma unroll
                    for (int k = 0; k < kGatherRegs; ++k)
                        if (mi[k] >= 0) w[mi[k]] += uv[k];
                }
                __syncthreads();
            }
            for (int i0 = tid; i0 < S; i0 += kGatherRegs * nt) {
                int pk[kGatherRegs];
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k)
                    pk[k] = i0 + k * nt < S ? D.perm[vo + i0 + k * nt] : -1;
#pragma unroll
                for (int k = 0; k < kGatherRegs; ++k)
                    if (pk[k] >= 0) t[i0 + k * nt] = w[pk[k]];
            }
        }
        __syncthreads();
    }

    // -x on the struct variables [S, f) into dst[0, f - S), in batches of
    // kGatherRegs entries per thread (index loads first)
    __device__ __forceinline__ void gather_struct_x(const MfDev &D, const T *x, T *dst) const
    {
        const int tid = threadIdx.x, nt = blockDim.x, mm = f - S;
        if (staged) {
#pragma unroll
            for (int k = 0; k < kGatherRegs; ++k) {
                const int e = tid + k * nt;
                if (e < mm) dst[e] = -__ldcg(x + xi[k]);
            }
            return;
        }
        const int *vars = D.vars + vo + S;
        for (int e0 = tid; e0 < mm; e0 += kGatherRegs * nt) {
            int vi[kGatherRegs];
#pragma unroll
            for (int k = 0; k < kGatherRegs; ++k) vi[k] = e0 + k * nt < mm ? vars[e0 + k * nt] : -1;
            T xv[kGatherRegs];
#pragma unroll
            for (int k = 0; k < kGatherRegs; ++k) xv[k] = vi[k] >= 0 ? __ldcg(x + vi[k]) : T(0);
#pragma unroll
            for (int k = 0; k < kGatherRegs; ++k)
                if (vi[k] >= 0) dst[e0 + k * nt] = -xv[k];
        }
    }

    // Forward rows: t from the gather item (gathered fronts) or gathered
    // here; then z_r = t_r + F[r, 0:r] t on pivot rows and u_r = w_r -
    // F[r, 0:S] t on contribution rows.
    __device__ __forceinline__ void run_fwd(const MfDev &D, const T *b,
                                            const double *__restrict__ rs, T *zbuf, T *upd, T *w,
                                            T *t)
    {
        T *uo = upd + D.uoff[q] - S;   // row r >= S -> uo[r]
        if (gath) {
            const T *tw = (const T *)D.tw + vo;
            for (int i = threadIdx.x; i < S; i += blockDim.x) t[i] = __ldcg(tw + i);
            __syncthreads();
            rows(t, [&](int r, T v) {
                if (r < S) zbuf[vo + r] = t[r] + v;
                else uo[r] = __ldcg(tw + r) - v;
            });
            return;
        }
        gather_w(D, b, rs, upd, w, t);
        rows(t, [&](int r, T v) {
            if (r < S) zbuf[vo + r] = t[r] + v;
            else uo[r] = w[r] - v;
        });
    }

    // Forward gather item: t on the pivot positions and w on the
    // contribution rows into tw, once for all of the front's row items.
    __device__ __forceinline__ void run_gather_fwd(const MfDev &D, const T *b,
                                                   const double *__restrict__ rs, const T *upd,
                                                   T *w, T *t)
    {
        gather_w(D, b, rs, upd, w, t);
        T *tw = (T *)D.tw + vo;
        for (int i = threadIdx.x; i < f; i += blockDim.x) tw[i] = i < S ? t[i] : w[i];
    }

    // Backward gather item: -x on the front's struct variables into tw.
    __device__ __forceinline__ void run_gather_bwd(const MfDev &D, const T *x)
    {
        gather_struct_x(D, x, (T *)D.tw + vo + S);
    }

    // Backward: v = (z, -x on the front's struct variables); then the rows.
    __device__ __forceinline__ void run_bwd(const MfDev &D, const T *zbuf, T *x, T *v)
    {
        const int tid = threadIdx.x, nt = blockDim.x, mm = f - S;
        const int *vars = D.vars + vo;
        for (int i = tid; i < S; i += nt) v[i] = __ldcg(zbuf + vo + i);
        if (gath) {
            const T *tw = (const T *)D.tw + vo + S;
            for (int e = tid; e < mm; e += nt) v[S + e] = __ldcg(tw + e);
        } else {
            gather_struct_x(D, x, v + S);
        }
        __syncthreads();
        rows(v, [&](int r, T val) { x[vars[r]] = val; });
    }

    // The item's rows: one per thread when a forward item has at least half
    // as many rows as threads, in fronts of at most kThreadRowMaxF variables
    // (each thread sums its row left to right, four partial sums;
    // the row's entries come through L1 line by line and the vector entries
    // from shared memory); one per warp from registers (at most one row per
    // warp); otherwise G rows per warp at a time (dotN).
    template <class Out>
    __device__ __forceinline__ void rows(const T *vec, Out out)
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
        // one row per thread: short FP32 rows only (a warp's loads touch 32
        // rows at once, which pays only while the rows stay in L1)
        if (fwd && f <= kThreadRowMaxF && 2 * (rend - rbeg) >= (int)blockDim.x) {
            for (int r = rbeg + (int)threadIdx.x; r < rend; r += blockDim.x) {
                int lo, hi;
                row_range(fwd, r, S, f, lo, hi);
                const T *row = A + (long long)r * f;
                T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
                int c = lo;
#pragma unroll 4
                for (; c + 3 < hi; c += 4) {
                    a0 += row[c] * vec[c];
                    a1 += row[c + 1] * vec[c + 1];
                    a2 += row[c + 2] * vec[c + 2];
                    a3 += row[c + 3] * vec[c + 3];
                }
                for (; c < hi; ++c) a0 += row[c] * vec[c];
                out(r, (a0 + a1) + (a2 + a3));
            }
            return;
        }
        if (rend - rbeg <= nw) {
            const int r = rbeg + wid;
            if (r < rend) {
                int lo, hi;
                row_range(fwd, r, S, f, lo, hi);
                T s = T(0);
                if (onerow) {
                    s = row_dot_reg<T, R>(reg, vec, base, lo, hi);
                } else {
                    const T *p[4] = {A + (long long)r * f, A, A, A};
                    const int bb[4] = {lo, 0, 0, 0}, ee[4] = {hi, 0, 0, 0};
                    T s4[4];
                    dot4<T>(p, bb, ee, vec, s4);
                    s = s4[0];
                }
                if (lane == 0) out(r, s);
            }
            return;
        }
        constexpr int G = R >= 32 ? 8 : 4;   // rows per warp in flight (register budget)
        // column chunks per row in flight: 2 in the small-register forms
        constexpr int KC = (R < RowRegs<T>::v || G >= 8) ? 2 : 4;
        for (int r = rbeg + wid; r < rend; r += G * nw) {
            const T *p[G];
            int bb[G], ee[G], rr[G];
#pragma unroll
            for (int u = 0; u < G; ++u) {
                rr[u] = r + u * nw;
                if (rr[u] < rend) {
                    row_range(fwd, rr[u], S, f, bb[u], ee[u]);
                    p[u] = A + (long long)rr[u] * f;
                } else {
                    bb[u] = ee[u] = 0;
                    p[u] = A;
                }
            }
            T sg[G];
            dotN<T, G, KC>(p, bb, ee, vec, sg);
            if (lane == 0) {
#pragma unroll
                for (int u = 0; u < G; ++u)
                    if (rr[u] < rend) out(rr[u], sg[u]);
            }
        }
    }
};

// Work item table entry: 12 ints.
//   x: kind (0 forward, 1 backward), front, first row, end row
//   y: wait counter 0, its target, wait counter 1, its target (-1 / 0: none)
//   z: done counters 0 and 1 (-1: none), unused, unused
struct SolveItemDev {
    int4 x, y, z;
};

template <class T, int R>
__device__ __forceinline__ void run_item(SolveItemCtx<T, R> &c, const MfDev &D, const T *b,
                                         const double *__restrict__ rs, T *zbuf, T *upd, T *x,
                                         T *smem, int wcap)
{
    // shared memory: w (wcap entries, the largest front of the launch), then t
    switch (c.kind) {
    case 0: c.run_fwd(D, b, rs, zbuf, upd, smem, smem + wcap); break;
    case 1: c.run_bwd(D, zbuf, x, smem); break;
    case 2: c.run_gather_fwd(D, b, rs, upd, smem, smem + wcap); break;
    default: c.run_gather_bwd(D, x); break;
    }
}

// One launch per level and sweep: block i runs item i0 + i (its
// dependencies are the previous launches).
template <class T>
__global__ void __launch_bounds__(kSolveThreads, 2) k_solve_level(
    const MfDev D, const T *F, const T *b, const double *__restrict__ rs, T *zbuf, T *upd, T *x,
    const SolveItemDev *__restrict__ items, int i0, const int *stop_a, const int *stop_b)
{
    if (stopped(stop_a, stop_b)) return;
    extern __shared__ unsigned char smem_raw[];
    T *smem = reinterpret_cast<T *>(smem_raw);
    const SolveItemDev it = items[i0 + blockIdx.x];
    SolveItemCtx<T> c;
    c.pre(D, F, b, rs, it.x.x, it.z.w, it.x.y, it.x.z, it.x.w);
    run_item(c, D, b, rs, zbuf, upd, x, smem, D.maxf);
}

// The split form's lower-level launches: CTA size and resident CTAs per SM.
constexpr int kLowThreads = 128;
constexpr int kLowMinBlocks = 4;

// Polls of one dependency counter before a CTA of the dataflow solve gives
// up (each poll sleeps ~40 ns: well under a second in all).
constexpr long long kFlowSpins = 1LL << 22;

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Global nanosecond timer (per-item traces of the dataflow solve).
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait until *ctr >= target; false if it ran out or another CTA
// reported an error meanwhile.
__device__ __forceinline__ void red_release_gpu(int *p, int v)
{
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool wait_count(const int *ctr, int target, volatile int *err)
{
    long long spins = 0;
    while (ld_acquire_gpu(ctr) < target) {
        if (*err || ++spins > kFlowSpins) return false;
        __nanosleep(40);
    }
    return true;
}

// The whole solve as one launch of work items in the plan's order (forward
// bottom-up, then backward top-down).  A CTA takes items by ticket
// (ctr[nctr]), loads what needs no other item, waits (thread 0, acquire
// loads) until the item's counters reach their targets, runs the item and,
// after a barrier, adds one to the item's done counters with release
// semantics.  The plan checks that
// every counter an item waits on is advanced only by items before it, so a
// CTA only ever waits for items held by running CTAs: no co-resident grid is
// needed.  A wait that runs out (or an error seen while waiting) sets
// bar->err (bit 2) and *stop_a (so GMRES stops instead of using an
// unfinished preconditioner) and ends the CTA.  ctr is zeroed before each
// launch.
// Two forms (the autotuner picks one): MINB resident CTAs per SM at least,
// R row registers per lane (rows up to 32 R entries prefetched before the
// wait).  Form 0: 2 CTAs and RowRegs<T> registers; form 1: 3 CTAs per SM
// with RowRegs3<T>, more warps in flight for the levels whose items are
// whole fronts.  A launch runs the items [item0, item1) with ticket counter
// ctr[nctr + slot]: the whole table, or (split form) the lower levels'
// forward items, the upper levels, the lower levels' backward items as three
// launches in stream order -- an item then only waits for items of its own
// launch or of an earlier, finished one.  The lower launches use NT = 128
// threads and shared memory for their own largest front (wcap), so more of
// their many small items are in flight per SM.
template <class T, int R, int MINB, int NT = kSolveThreads>
__global__ void __launch_bounds__(NT, MINB) k_solve_flow(
    const MfDev D, const T *F, const T *b, const double *__restrict__ rs, T *zbuf, T *upd, T *x,
    const SolveItemDev *__restrict__ items, int item0, int item1, int wcap, int *ctr, int nctr,
    int slot, MfBarrier *bar, const int *stop_a, const int *stop_b, unsigned long long *trace)
{
    if (stopped(stop_a, stop_b)) return;   // the flags are the same for every CTA
    extern __shared__ unsigned char smem_raw[];
    T *smem = reinterpret_cast<T *>(smem_raw);
    __shared__ int item_s, ok_s;
    volatile int *err = &bar->err;
    int *ticket = ctr + nctr + slot;
    int next = threadIdx.x == 0 ? item0 + atomicAdd(ticket, 1) : 0;
    for (;;) {
        if (threadIdx.x == 0) item_s = next;
        __syncthreads();
        const int i = item_s;
        if (i >= item1) return;
        const SolveItemDev it = items[i];
        if (trace && threadIdx.x == 0) trace[3 * i] = globaltimer_ns();
        SolveItemCtx<T, R> c;
        c.pre(D, F, b, rs, it.x.x, it.z.w, it.x.y, it.x.z, it.x.w);
        if (threadIdx.x == 0) {
            next = item0 + atomicAdd(ticket, 1);   // in flight during the wait
            bool ok = true;
            if (it.y.x >= 0 && it.y.y > 0) ok = wait_count(ctr + it.y.x, it.y.y, err);
            if (ok && it.y.z >= 0 && it.y.w > 0) ok = wait_count(ctr + it.y.z, it.y.w, err);
            if (!ok) {
                atomicOr(&bar->err, 2);
                if (stop_a) atomicExch(const_cast<int *>(stop_a), 1);
            }
            ok_s = ok;
        }
        __syncthreads();
        if (!ok_s) return;
        if (trace && threadIdx.x == 0) trace[3 * i + 1] = globaltimer_ns();
        run_item(c, D, b, rs, zbuf, upd, x, smem, wcap);
        // the barrier orders every thread's writes before thread 0's release
        // additions (cumulative at GPU scope), which the waiters' acquire
        // loads pair with
        __syncthreads();
        if (threadIdx.x == 0) {
            if (it.z.x >= 0) red_release_gpu(ctr + it.z.x, 1);
            if (it.z.y >= 0) red_release_gpu(ctr + it.z.y, 1);
            if (trace) trace[3 * i + 2] = globaltimer_ns();
        }
    }
}

// ---------------------------------------------------------- transposed solve
// The transposed solve is the adjoint of the solve's steps taken in reverse
// order.  Bottom-up (adjoint of the backward sweep): the front gathers g on
// its fully summed variables plus its children's contributions (the same
// contribution-block maps as the forward sweep), forms ybar = U11^-T acc_FS
// (kept in zbuf) and passes acc_CB - H^T acc_FS up.  Top-down (adjoint of the
// forward sweep): the front takes its parent's adjoint right-hand side
// upd_bar on its contribution rows, t = L11^-T ybar - G^T upd_bar (unit
// diagonal), scatters t through the row permutation and writes
// lambda = rs .* w_bar on its fully summed variables.  One CTA per front; the
// transposed products read the factor rows column-wise (one thread per
// column, coalesced across the warp).
template <class T>
__global__ void __launch_bounds__(kSolveThreads) k_tup_front(int q0, const MfDev D, const T *F,
                                                              const T *g, T *zbuf, T *upd)
{
    extern __shared__ unsigned char smem_raw[];
    T *acc = reinterpret_cast<T *>(smem_raw);   // f
    T *yb = acc + D.maxf;                         // S
    const int q = q0 + blockIdx.x;
    const int S = D.S[q], f = D.f[q], vo = D.voff[q], m = f - S;
    const T *A = F + D.foff[q];
    const int *vars = D.vars + vo;
    const int tid = threadIdx.x;
    for (int p = tid; p < f; p += blockDim.x) acc[p] = p < S ? g[vars[p]] : T(0);
    __syncthreads();
    for (int slot = 0; slot < 2; ++slot) {
        const int c = slot == 0 ? D.child0[q] : D.child1[q];
        if (c >= 0) {
            const int mc = D.f[c] - D.S[c];
            const int *map = D.cbmap + D.uoff[c];
            const T *u = upd + D.uoff[c];
            for (int e = tid; e < mc; e += blockDim.x) acc[map[e]] += u[e];
        }
        __syncthreads();
    }
    for (int j = tid; j < S; j += blockDim.x) {     // ybar = Uinv^T acc_FS
        T v = T(0);
        for (int i = 0; i <= j; ++i) v += A[(long long)i * f + j] * acc[i];
        yb[j] = v;
    }
    __syncthreads();
    for (int j = tid; j < S; j += blockDim.x) zbuf[vo + j] = yb[j];
    T *uo = upd + D.uoff[q];
    for (int k = tid; k < m; k += blockDim.x) {     // acc_CB - H^T acc_FS
        T v = T(0);
        for (int i = 0; i < S; ++i) v += A[(long long)i * f + S + k] * acc[i];
        uo[k] = acc[S + k] - v;
    }
}

template <class T>
__global__ void __launch_bounds__(kSolveThreads) k_tdown_front(int q0, const MfDev D, const T *F,
                                                               const double *__restrict__ rs,
                                                               const T *zbuf, T *wb, T *lam)
{
    extern __shared__ unsigned char smem_raw[];
    T *wbar = reinterpret_cast<T *>(smem_raw);  // f
    T *v = wbar + D.maxf;                         // f: (ybar, -upd_bar)
    const int q = q0 + blockIdx.x;
    const int S = D.S[q], f = D.f[q], vo = D.voff[q], m = f - S;
    const T *A = F + D.foff[q];
    const int *vars = D.vars + vo;
    const int tid = threadIdx.x;
    const int pa = D.parent[q];
    for (int k = tid; k < m; k += blockDim.x) {     // upd_bar from the parent
        const T u = pa >= 0 ? wb[D.voff[pa] + D.cbmap[D.uoff[q] + k]] : T(0);
        wbar[S + k] = u;
        v[S + k] = -u;
    }
    for (int j = tid; j < S; j += blockDim.x) v[j] = zbuf[vo + j];
    __syncthreads();
    const int *perm = D.perm + vo;
    // t = Linv^T ybar - G^T upd_bar: column i of rows (i, f); w_bar[perm[i]] = t
    for (int i = tid; i < S; i += blockDim.x) {
        T t = v[i];
        for (int j = i + 1; j < f; ++j) t += A[(long long)j * f + i] * v[j];
        wbar[perm[i]] = t;
    }
    __syncthreads();
    for (int p = tid; p < f; p += blockDim.x) wb[vo + p] = wbar[p];
    for (int p = tid; p < S; p += blockDim.x) lam[vars[p]] = (T)(rs[vars[p]] * (double)wbar[p]);
}

}  // namespace

// ------------------------------------------------------------ host drivers
// The dynamic shared memory limit of a kernel (cudaFuncSetAttribute) holds
// per function and device for the whole process, so every handle shares it:
// it is only ever raised, to the largest size any handle launches with.
// Setting it to one handle's smaller size would make the launches of a
// handle with larger fronts fail.  Until it is set, a launch may use the
// default 48 KB less the kernel's static shared memory.
static cudaError_t raise_dyn_smem(const void *fn, size_t bytes)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    const size_t room = fa.sharedSizeBytes < 48 * 1024 ? 48 * 1024 - fa.sharedSizeBytes : 0;
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = limit[{fn, dev}];
    if (bytes <= std::max(cur, room)) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

int mf_factor_create(const MfPlan *P, int fp32, int fact64, MfFactor **out)
{
    *out = nullptr;
    MfFactor *M = new MfFactor();
    M->fp32 = fp32;
    M->fact64 = fp32 && fact64 ? 1 : 0;
    const size_t es = fp32 ? sizeof(float) : sizeof(double);          // solve
    const size_t esf = fp32 && !M->fact64 ? sizeof(float) : sizeof(double);   // factorization
    cudaError_t e = cudaSuccess;
    auto grab = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    };
    grab(&M->F, (size_t)P->ftotal * esf);
    if (M->fact64) grab(&M->F32, (size_t)P->ftotal * sizeof(float));
    grab(&M->upd, (size_t)P->utotal * es);
    grab(&M->z, (size_t)P->vtotal * es);
    grab(&M->tmp, (size_t)P->tmax * esf);
    grab(&M->gh, (size_t)P->gmax * esf);
    grab((void **)&M->sctr, (size_t)(P->nctr + kFlowSlots) * sizeof(int));
    grab(&M->wb, (size_t)P->vtotal * es);
    grab(&M->tw, (size_t)P->vtotal * es);
    grab((void **)&M->rs, (size_t)P->n * sizeof(double));
    grab((void **)&M->ipiv, (size_t)P->vtotal * sizeof(int));
    grab((void **)&M->perm, (size_t)P->vtotal * sizeof(int));
    grab((void **)&M->flag, sizeof(int));
    grab((void **)&M->bar, sizeof(MfBarrier));
    if (e == cudaSuccess) e = cudaMemset(M->bar, 0, sizeof(MfBarrier));
    if (e != cudaSuccess) {
        set_error("mf_factor: allocation of %.1f MB failed: %s",
                  ((double)P->ftotal * (esf + (M->fact64 ? 4 : 0))) / 1e6, cudaGetErrorString(e));
        mf_factor_destroy(M);
        return V2D_ENOMEM;
    }
    // dynamic shared memory of the solve and inversion kernels (set once,
    // outside any stream capture)
    const size_t solve = (size_t)(P->maxf + P->maxS) * es;
    const int cw = esf == sizeof(float) ? InvWidth<float>::v : InvWidth<double>::v;
    // shared-memory inversion where its column block fits, the global work
    // space elsewhere (sized for the largest such level)
    size_t inv = 0, inv_g = 0;
    for (int L = 0; L < P->nlevel; ++L) {
        const size_t sl = (size_t)P->lvl_maxS[L] * (cw + 33);
        if (sl * esf <= kInvSmemMax) {
            inv = std::max(inv, sl * esf);
        } else if (esf == sizeof(float)) {   // FP64 inverts these by blocks in place
            const size_t nbc = (P->lvl_maxS[L] + cw - 1) / cw;
            inv_g = std::max(inv_g, nbc * (size_t)(P->lvl_off[L + 1] - P->lvl_off[L]) * sl);
        }
    }
    if (solve > 227 * 1024) {
        set_error("mf_factor: front of %d unknowns (separator %d) exceeds shared memory",
                  P->maxf, P->maxS);
        mf_factor_destroy(M);
        return V2D_EARG;
    }
    if (inv_g > 0) {
        cudaError_t ge = cudaMalloc(&M->inv_g, inv_g * esf);
        if (ge != cudaSuccess) {
            set_error("mf_factor: inversion work space of %.1f MB: %s", inv_g * esf / 1e6,
                      cudaGetErrorString(ge));
            mf_factor_destroy(M);
            return V2D_ENOMEM;
        }
    }
    auto attr = [&](const void *fn, size_t bytes) {
        if (e == cudaSuccess) e = raise_dyn_smem(fn, bytes);
    };
    const size_t tsolve = (size_t)2 * P->maxf * es;   // transposed solve: two f vectors
    if (tsolve > 227 * 1024) {
        set_error("mf_factor: front of %d unknowns exceeds shared memory (transposed solve)",
                  P->maxf);
        mf_factor_destroy(M);
        return V2D_EARG;
    }
    if (fp32) {
        attr((const void *)k_solve_level<float>, solve);
        attr((const void *)k_solve_flow<float, RowRegs<float>::v, 2>, solve);
        attr((const void *)k_solve_flow<float, RowRegs3<float>::v, 3>, solve);
        attr((const void *)k_tup_front<float>, tsolve);
        attr((const void *)k_tdown_front<float>, tsolve);
    } else {
        attr((const void *)k_solve_level<double>, solve);
        attr((const void *)k_solve_flow<double, RowRegs<double>::v, 2>, solve);
        attr((const void *)k_solve_flow<double, RowRegs3<double>::v, 3>, solve);
        attr((const void *)k_tup_front<double>, tsolve);
        attr((const void *)k_tdown_front<double>, tsolve);
    }
    if (esf == sizeof(float)) attr((const void *)k_trinv<float>, inv);
    else attr((const void *)k_trinv<double>, inv);
    if (e != cudaSuccess) {
        set_error("mf_factor: %s", cudaGetErrorString(e));
        mf_factor_destroy(M);
        return V2D_ECUDA;
    }
    // dataflow solve: as many CTAs as can be resident at once (two per SM at
    // most), never more than there are work items
    int dev = 0, nsm = 0, per_sm = 0;
    cudaError_t oe = cudaGetDevice(&dev);
    if (oe == cudaSuccess) oe = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (oe == cudaSuccess)
        oe = fp32 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                        &per_sm, k_solve_flow<float, RowRegs<float>::v, 2>, kSolveThreads, solve)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                        &per_sm, k_solve_flow<double, RowRegs<double>::v, 2>, kSolveThreads,
                        solve);
    int per_sm1 = 0;
    if (oe == cudaSuccess)
        oe = fp32 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                        &per_sm1, k_solve_flow<float, RowRegs3<float>::v, 3>, kSolveThreads,
                        solve)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                        &per_sm1, k_solve_flow<double, RowRegs3<double>::v, 3>, kSolveThreads,
                        solve);
    if (oe != cudaSuccess || per_sm <= 0) {
        set_error("mf_factor: occupancy of the dataflow solve: %s",
                  oe != cudaSuccess ? cudaGetErrorString(oe) : "no CTA fits on an SM");
        mf_factor_destroy(M);
        return V2D_ECUDA;
    }
    M->flow_grid = std::max(1, nsm * std::min(per_sm, 2));
    M->flow_grid1 = per_sm1 > 0 ? nsm * std::min(per_sm1, 3) : 0;
    cudaGetLastError();
    *out = M;
    return V2D_OK;
}

void mf_factor_destroy(MfFactor *M)
{
    if (!M) return;
    if (M->graph) cudaGraphExecDestroy(M->graph);
    void *ptrs[] = {M->F,    M->F32,  M->upd,  M->z,    M->tmp,   M->gh,    M->wb,  M->tw,
                    M->rs,   M->ipiv, M->perm, M->flag, M->bar,  M->inv_g, M->sctr};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    delete M;
}

MfDev mf_dev(const MfPlan *P, const MfFactor *M)
{
    MfDev D;
    D.S = P->d_S; D.f = P->d_f; D.voff = P->d_voff; D.uoff = P->d_uoff;
    D.child0 = P->d_child0; D.child1 = P->d_child1; D.parent = P->d_parent; D.foff = P->d_foff;
    D.vars = P->d_vars; D.cbmap = P->d_cbmap; D.perm = M->perm;
    D.maxS = P->maxS; D.maxf = P->maxf;
    D.tw = M->tw;
    return D;
}

template <class T>
static int factor_launches(const MfPlan *P, MfFactor *M, const int *rowptr, const double *val,
                           cudaStream_t s, cudaEvent_t *ev = nullptr, int *codes = nullptr,
                           int cap = 0, int *nev_out = nullptr)
{
    constexpr int NB = PanelWidth<T>::v;
    T *F = (T *)M->F;
    long long launches = 0;
    const size_t tile_smem = tile_smem_bytes<T>();
    V2D_CUDA_TRY(raise_dyn_smem((const void *)k_gemm<T>, tile_smem));
    V2D_CUDA_TRY(raise_dyn_smem((const void *)k_gh<T>, tile_smem));
    V2D_CUDA_TRY(raise_dyn_smem((const void *)k_trinv_step<T>, tile_smem));
    V2D_CUDA_TRY(raise_dyn_smem((const void *)k_trinv_diag<T>, trinv_diag_smem<T>()));
    // with ev: an event is recorded after each kernel (kind * 1000 + level;
    // kinds 0 rowscale, 1 scatter, 2 extend_add, 3 first panel, 4 L21 + row
    // swaps + U12, 6 trailing update + next panel, 7 trinv, 8 trcopy, 9 G/H
    // products, 10 G/H copy)
    int nev = 0;
    auto mark = [&](int code) -> int {
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) {
            set_error("LU factor: launch of kind %d at level %d failed: %s", code / 1000,
                      code % 1000, cudaGetErrorString(le));
            return V2D_ECUDA;
        }
        if (!ev) return V2D_OK;
        if (nev >= cap) {
            set_error("LU factor timing: more than %d launches", cap);
            return V2D_EARG;
        }
        codes[nev] = code;
        V2D_CUDA_TRY(cudaEventRecord(ev[nev], s));
        ++nev;
        return V2D_OK;
    };
    k_rowscale<<<grid_for(P->n, 256), 256, 0, s>>>(P->n, rowptr, val, M->rs);
    V2D_TRY(mark(0));
    ++launches;
    for (int L = 0; L < P->nlevel; ++L) {
        const int q0 = P->lvl_off[L], nq = P->lvl_off[L + 1] - q0;
        V2D_CUDA_TRY(cudaMemsetAsync(F + P->lvl_fbeg[L], 0,
                                     (size_t)(P->lvl_fend[L] - P->lvl_fbeg[L]) * sizeof(T), s));
        const long long na = P->lvl_aend[L] - P->lvl_abeg[L];
        if (na > 0) {
            k_scatter<T><<<grid_for(na, 256), 256, 0, s>>>(P->lvl_abeg[L], P->lvl_aend[L],
                                                         P->d_asm_csr, P->d_asm_row,
                                                         P->d_asm_pos, val, M->rs, F);
            V2D_TRY(mark(1000 + L));
            ++launches;
        }
        if (L > 0) {
            const long long mm = (long long)P->lvl_maxm_child[L] * P->lvl_maxm_child[L];
            const int gx = (int)std::max(1LL, std::min<long long>((mm + 255) / 256, 64));
            for (int slot = 0; slot < 2; ++slot) {
                for (int qb = 0; qb < nq; qb += kMaxFrontsY) {
                    k_extend_add<T><<<dim3(gx, std::min(nq - qb, kMaxFrontsY)), 256, 0, s>>>(
                        q0 + qb, slot, P->d_S, P->d_f, P->d_foff, P->d_uoff, P->d_child0,
                        P->d_child1, P->d_cbmap, F);
                    ++launches;
                }
                V2D_TRY(mark(2000 + L));
            }
        }
        const int maxf = P->lvl_maxf[L];
        // delayed trailing updates on levels with large fronts
        const int W = maxf >= kDelayFront ? kDelayPanels * NB : NB;
        for (int k = 0; k < P->lvl_maxS[L]; k += NB) {
            if (k == 0) {   // later panels are factored by the previous trailing update
                k_panel<T><<<nq, kMfThreads, 0, s>>>(q0, k, P->d_S, P->d_f, P->d_foff, P->d_voff,
                                                     F, M->ipiv, M->perm, M->flag);
                V2D_TRY(mark(3000 + L));
                ++launches;
            }
            const int below = std::max(1, maxf - k - 1);
            const int nl = (below + kL21Rows - 1) / kL21Rows;
            const int ncol = (maxf + kL21Rows - 1) / kL21Rows;
            for (int qb = 0; qb < nq; qb += kMaxFrontsY) {
                k_l21_trsm<T><<<dim3(nl + ncol, std::min(nq - qb, kMaxFrontsY)), kL21Rows, 0,
                                s>>>(q0 + qb, k, nl, P->d_S, P->d_f, P->d_foff, P->d_voff, F,
                                     M->ipiv);
                if (qb > 0) ++launches;
            }
            V2D_TRY(mark(4000 + L));
            const int rem = std::max(1, maxf - k - 1);
            const int nt = (rem + kGemmTile - 1) / kGemmTile;
            // tiles of the larger of the two cases (narrow + row block, or
            // the super-panel's full update)
            const int ntile = nt * nt + nt;
            for (int qb = 0; qb < nq; qb += kMaxFrontsY) {
                k_gemm<T><<<dim3(ntile, std::min(nq - qb, kMaxFrontsY)), 256, tile_smem, s>>>(
                    q0 + qb, k, W, P->d_S, P->d_f, P->d_foff, P->d_voff, F, M->ipiv, M->perm,
                    M->flag);
                if (qb > 0) ++launches;
            }
            V2D_TRY(mark(6000 + L));
            launches += 2;
        }
        const int nbc = (P->lvl_maxS[L] + InvWidth<T>::v - 1) / InvWidth<T>::v;
        const size_t inv_bytes = (size_t)P->lvl_maxS[L] * (InvWidth<T>::v + 33) * sizeof(T);
        for (int qb = 0; qb < nq; qb += kMaxFrontsY) {
            const int nb = std::min(nq - qb, kMaxFrontsY);
            const bool blocked = P->lvl_maxS[L] >= kBlockedInvMinS &&
                                 (std::is_same<T, double>::value || inv_bytes <= kInvSmemMax);
            if (inv_bytes <= kInvSmemMax && !blocked) {
                const int nth = nbc * nb > kTrinvManyCtas ? kTrinvThreadsMany : kTrinvThreads;
                k_trinv<T><<<dim3(nbc, nb), nth, inv_bytes, s>>>(
                    q0 + qb, P->d_S, P->d_foff, P->d_f, P->d_toff, F, (T *)M->tmp);
            } else if (blocked) {
                // wide separators: blocked inversion on the tile engine (the
                // FP64 tensor cores; CUDA cores in FP32)
                const int nbk = (P->lvl_maxS[L] + kInvBlk - 1) / kInvBlk;
                k_trinv_diag<T><<<dim3(nbk, nb), kTrinvDiagThreads, trinv_diag_smem<T>(), s>>>(
                    q0 + qb, P->d_S, P->d_f, P->d_foff, P->d_toff, F, (T *)M->tmp);
                for (int st = nbk - 2; st >= 0; --st)
                    for (int phase = 0; phase < 2; ++phase) {
                        const int half = nbk - st - 1;
                        k_trinv_step<T><<<dim3(2 * half, nb), 256, tile_smem, s>>>(
                            q0 + qb, st, phase, half, P->d_S, P->d_f, P->d_foff, P->d_toff, F,
                            (T *)M->tmp);
                        ++launches;
                    }
            } else {
                k_trinv_g<T><<<dim3(nbc, nb), kTrinvThreadsG, 0, s>>>(
                    q0 + qb, P->d_S, P->d_foff, P->d_f, P->d_toff, F, (T *)M->tmp,
                    (T *)M->inv_g, (long long)P->lvl_maxS[L] * (InvWidth<T>::v + 33));
            }
            if (qb > 0) ++launches;
        }
        V2D_TRY(mark(7000 + L));
        const long long ss = (long long)P->lvl_maxS[L] * P->lvl_maxS[L];
        const int gcp = (int)std::max(1LL, std::min<long long>((ss + 255) / 256, 256));
        for (int qb = 0; qb < nq; qb += kMaxFrontsY) {
            k_trcopy<T><<<dim3(gcp, std::min(nq - qb, kMaxFrontsY)), 256, 0, s>>>(
                q0 + qb, P->d_S, P->d_f, P->d_foff, P->d_toff, (const T *)M->tmp, F);
            if (qb > 0) ++launches;
        }
        V2D_TRY(mark(8000 + L));
        launches += 2;
        // G = L21 L11^-1, H = U11^-1 U12 (the solve's row products)
        if (P->lvl_maxm[L] > 0) {
            const int ts = (P->lvl_maxS[L] + kGemmTile - 1) / kGemmTile;
            const int tm = (P->lvl_maxm[L] + kGemmTile - 1) / kGemmTile;
            const long long sm = 2LL * P->lvl_maxS[L] * P->lvl_maxm[L];
            const int gcg = (int)std::max(1LL, std::min<long long>((sm + 255) / 256, 256));
            for (int qb = 0; qb < nq; qb += kMaxFrontsY) {
                k_gh<T><<<dim3(2 * ts * tm, std::min(nq - qb, kMaxFrontsY)), 256, tile_smem, s>>>(
                    q0 + qb, P->d_S, P->d_f, P->d_foff, P->d_goff, F, (T *)M->gh);
                if (qb > 0) ++launches;
            }
            V2D_TRY(mark(9000 + L));
            for (int qb = 0; qb < nq; qb += kMaxFrontsY) {
                k_ghcopy<T><<<dim3(gcg, std::min(nq - qb, kMaxFrontsY)), 256, 0, s>>>(
                    q0 + qb, P->d_S, P->d_f, P->d_foff, P->d_goff, (const T *)M->gh, F);
                if (qb > 0) ++launches;
            }
            V2D_TRY(mark(10000 + L));
            launches += 2;
        }
    }
    if (M->fact64) {   // FP64 factors rounded to FP32 for the solve
        k_round_f32<<<grid_for(P->ftotal, 256), 256, 0, s>>>((const double *)M->F,
                                                             (float *)M->F32, P->ftotal);
        V2D_TRY(mark(11000));
        ++launches;
    }
    V2D_CUDA_TRY(cudaGetLastError());
    if (nev_out) *nev_out = nev;
    if (!ev) M->launches_per_factor = launches;
    return V2D_OK;
}

int mf_factor(const MfPlan *P, MfFactor *M, const int *rowptr, const double *val, cudaStream_t s)
{
    if (!M->graph || M->graph_val != val || M->graph_rowptr != rowptr) {
        if (M->graph) cudaGraphExecDestroy(M->graph);
        M->graph = nullptr;
        cudaGraph_t g = nullptr;
        V2D_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int st = M->fp32 && !M->fact64 ? factor_launches<float>(P, M, rowptr, val, s)
                                       : factor_launches<double>(P, M, rowptr, val, s);
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (st != V2D_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) {
            set_error("mf_factor: graph capture failed: %s", cudaGetErrorString(e));
            return V2D_ECUDA;
        }
        e = cudaGraphInstantiate(&M->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error("mf_factor: graph instantiate failed: %s", cudaGetErrorString(e));
            return V2D_ECUDA;
        }
        M->graph_val = val;
        M->graph_rowptr = rowptr;
    }
    V2D_CUDA_TRY(cudaMemsetAsync(M->flag, 0, sizeof(int), s));
    V2D_CUDA_TRY(cudaGraphLaunch(M->graph, s));
    count_launches(M->launches_per_factor);
    return V2D_OK;
}

// Error of the launch just issued, named (the solve is usually issued inside
// a stream capture, where a failed launch invalidates the capture and later
// calls report only that).
static int solve_launch(const char *what, int L)
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return V2D_OK;
    set_error("LU solve: launch of %s (level %d) failed: %s", what, L, cudaGetErrorString(e));
    return V2D_ECUDA;
}

// Launch codes of the solve's kernels for per-launch timing (kind * 1000 + level).
enum { kCodeFwdLevel = 0, kCodeBwdLevel = 1, kCodeFlow = 2 };

template <class T>
static int apply_launches(const MfPlan *P, const MfFactor *M, const T *b, T *x, const int *stop_a,
                          const int *stop_b, cudaStream_t s, long long *n_launches,
                          cudaEvent_t *ev = nullptr, int *codes = nullptr, int cap = 0,
                          unsigned long long *trace = nullptr)
{
    // with ev: an event is recorded after each launch (at most cap launches)
    int nev = 0;
    auto mark = [&](int code) -> int {
        if (!ev) return V2D_OK;
        if (nev >= cap) {
            set_error("LU solve timing: more than %d launches", cap);
            return V2D_EARG;
        }
        codes[nev] = code;
        V2D_CUDA_TRY(cudaEventRecord(ev[nev], s));
        ++nev;
        return V2D_OK;
    };
    const MfDev D = mf_dev(P, M);
    const T *F = (const T *)(M->fact64 ? M->F32 : M->F);
    T *z = (T *)M->z, *upd = (T *)M->upd;
    const SolveItemDev *items = (const SolveItemDev *)P->d_items;
    const size_t smf = (size_t)(P->maxf + P->maxS) * sizeof(T);
    long long launches = 0;
    if (M->flow) {
        V2D_CUDA_TRY(cudaMemsetAsync(M->sctr, 0, (size_t)(P->nctr + kFlowSlots) * sizeof(int), s));
        auto upper = [&](int i0, int i1, int slot) {
            const int n = std::max(1, i1 - i0);
            if (M->flow_form == 1 && M->flow_grid1 > 0)
                k_solve_flow<T, RowRegs3<T>::v, 3><<<std::min(n, M->flow_grid1), kSolveThreads, smf,
                                                     s>>>(D, F, b, M->rs, z, upd, x, items, i0, i1,
                                                          P->maxf, M->sctr, P->nctr, slot, M->bar,
                                                          stop_a, stop_b, trace);
            else
                k_solve_flow<T, RowRegs<T>::v, 2><<<std::min(n, M->flow_grid), kSolveThreads, smf,
                                                    s>>>(D, F, b, M->rs, z, upd, x, items, i0, i1,
                                                         P->maxf, M->sctr, P->nctr, slot, M->bar,
                                                         stop_a, stop_b, trace);
        };
        auto lower = [&](int i0, int i1, int slot) {
            k_solve_flow<T, RowRegs<T>::v, kLowMinBlocks, kLowThreads>
                <<<std::max(1, std::min(i1 - i0, M->low_grid)), kLowThreads, M->low_smem, s>>>(
                    D, F, b, M->rs, z, upd, x, items, i0, i1, M->low_wcap, M->sctr, P->nctr, slot,
                    M->bar, stop_a, stop_b, trace);
        };
        const int Ls = M->split;
        if (Ls > 0 && Ls < P->nlevel && M->low_grid > 0) {
            lower(P->lvl_fwd[0], P->lvl_fwd[Ls], 0);
            V2D_TRY(solve_launch("k_solve_flow (lower levels, forward)", 0));
            V2D_TRY(mark(kCodeFlow * 1000));
            upper(P->lvl_fwd[Ls], P->lvl_bwd[Ls], 1);
            V2D_TRY(solve_launch("k_solve_flow (upper levels)", 0));
            V2D_TRY(mark(kCodeFlow * 1000 + 1));
            lower(P->lvl_bwd[Ls], P->nitems, 2);
            V2D_TRY(solve_launch("k_solve_flow (lower levels, backward)", 0));
            V2D_TRY(mark(kCodeFlow * 1000 + 2));
            launches = 3;
        } else {
            upper(0, P->nitems, 0);
            V2D_TRY(solve_launch("k_solve_flow", 0));
            V2D_TRY(mark(kCodeFlow * 1000));
            launches = 1;
        }
    } else {
        // a level's gather items (first in its range) are a launch of their own
        for (int L = 0; L < P->nlevel; ++L) {
            const int i0 = P->lvl_fwd[L], ni = P->lvl_fwd[L + 1] - i0, ng = P->lvl_fwd_g[L];
            for (const int part : {0, 1}) {
                const int a = part == 0 ? i0 : i0 + ng, n = part == 0 ? ng : ni - ng;
                if (n == 0) continue;
                k_solve_level<T><<<n, kSolveThreads, smf, s>>>(D, F, b, M->rs, z, upd, x, items,
                                                              a, stop_a, stop_b);
                V2D_TRY(solve_launch("k_solve_level (forward)", L));
                V2D_TRY(mark(kCodeFwdLevel * 1000 + L));
                ++launches;
            }
        }
        for (int L = P->nlevel - 1; L >= 0; --L) {
            const int i0 = P->lvl_bwd[L + 1], ni = P->lvl_bwd[L] - i0, ng = P->lvl_bwd_g[L];
            for (const int part : {0, 1}) {
                const int a = part == 0 ? i0 : i0 + ng, n = part == 0 ? ng : ni - ng;
                if (n == 0) continue;
                k_solve_level<T><<<n, kSolveThreads, smf, s>>>(D, F, b, M->rs, z, upd, x, items,
                                                              a, stop_a, stop_b);
                V2D_TRY(solve_launch("k_solve_level (backward)", L));
                V2D_TRY(mark(kCodeBwdLevel * 1000 + L));
                ++launches;
            }
        }
    }
    V2D_CUDA_TRY(cudaGetLastError());
    if (n_launches) *n_launches = ev ? nev : launches;
    return V2D_OK;
}

int mf_apply(const MfPlan *P, const MfFactor *M, const void *b, void *x, const int *stop_a,
             const int *stop_b, cudaStream_t s, long long *n_launches)
{
    if (M->fp32)
        return apply_launches<float>(P, M, (const float *)b, (float *)x, stop_a, stop_b, s,
                                     n_launches);
    return apply_launches<double>(P, M, (const double *)b, (double *)x, stop_a, stop_b, s,
                                  n_launches);
}

template <class T>
static int apply_transpose_launches(const MfPlan *P, MfFactor *M, const T *g, T *lam,
                                    cudaStream_t s, long long *launches)
{
    const MfDev D = mf_dev(P, M);
    const T *F = (const T *)(M->fact64 ? M->F32 : M->F);
    const size_t smf = (size_t)2 * P->maxf * sizeof(T);
    for (int L = 0; L < P->nlevel; ++L) {
        const int q0 = P->lvl_off[L], nq = P->lvl_off[L + 1] - q0;
        k_tup_front<T><<<nq, kSolveThreads, smf, s>>>(q0, D, F, g, (T *)M->z, (T *)M->upd);
    }
    for (int L = P->nlevel - 1; L >= 0; --L) {
        const int q0 = P->lvl_off[L], nq = P->lvl_off[L + 1] - q0;
        k_tdown_front<T><<<nq, kSolveThreads, smf, s>>>(q0, D, F, M->rs, (const T *)M->z,
                                                        (T *)M->wb, lam);
    }
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(2LL * P->nlevel);
    if (launches) *launches = 2LL * P->nlevel;
    return V2D_OK;
}

int mf_apply_transpose(const MfPlan *P, MfFactor *M, const void *g, void *lambda, cudaStream_t s,
                       long long *launches)
{
    if (M->fp32)
        return apply_transpose_launches<float>(P, M, (const float *)g, (float *)lambda, s,
                                               launches);
    return apply_transpose_launches<double>(P, M, (const double *)g, (double *)lambda, s,
                                            launches);
}

int mf_flag(const MfFactor *M, int *flag, cudaStream_t s)
{
    V2D_CUDA_TRY(cudaMemcpyAsync(flag, M->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    return V2D_OK;
}

int mf_set_split(const MfPlan *P, MfFactor *M, int split)
{
    V2D_ARG_CHECK(split >= 0 && split < P->nlevel, "lu split: level %d (0 .. %d)", split,
                  P->nlevel - 1);
    if (split == 0) {
        M->split = 0;
        return V2D_OK;
    }
    int wcap = 0, smax = 0;
    for (int L = 0; L < split; ++L) {
        wcap = std::max(wcap, P->lvl_maxf[L]);
        smax = std::max(smax, P->lvl_maxS[L]);
    }
    const size_t es = M->fp32 ? sizeof(float) : sizeof(double);
    const size_t bytes = (size_t)(wcap + smax) * es;
    const void *fn = M->fp32
                         ? (const void *)k_solve_flow<float, RowRegs<float>::v, kLowMinBlocks,
                                                      kLowThreads>
                         : (const void *)k_solve_flow<double, RowRegs<double>::v, kLowMinBlocks,
                                                      kLowThreads>;
    V2D_CUDA_TRY(raise_dyn_smem(fn, bytes));
    int dev = 0, nsm = 0, per_sm = 0;
    V2D_CUDA_TRY(cudaGetDevice(&dev));
    V2D_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    V2D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kLowThreads, bytes));
    V2D_ARG_CHECK(per_sm > 0, "lu split: no CTA of the lower-level launch fits on an SM");
    M->low_wcap = wcap;
    M->low_smem = bytes;
    M->low_grid = nsm * per_sm;
    M->split = split;
    return V2D_OK;
}

int mf_time_apply(const MfPlan *P, const MfFactor *M, int reps, size_t flush_bytes, cudaStream_t s,
                  double *ms_avg)
{
    const size_t es = M->fp32 ? sizeof(float) : sizeof(double);
    DevBuf<char> buf;
    V2D_TRY(buf.alloc(2 * P->n * es + flush_bytes + 256, s));
    V2D_CUDA_TRY(cudaMemsetAsync(buf.p, 0, 2 * P->n * es, s));
    char *fl = buf.p + 2 * P->n * es;
    cudaEvent_t e0, e1;
    V2D_CUDA_TRY(cudaEventCreate(&e0));
    V2D_CUDA_TRY(cudaEventCreate(&e1));
    double total = 0.0;
    int st = V2D_OK;
    for (int r = 0; r < reps && st == V2D_OK; ++r) {
        if (flush_bytes) cudaMemsetAsync(fl, r & 0xff, flush_bytes, s);
        cudaEventRecord(e0, s);
        st = mf_apply(P, M, buf.p, buf.p + P->n * es, nullptr, nullptr, s, nullptr);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = V2D_ECUDA;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != V2D_OK) return st;
    V2D_TRY(mf_check_barrier(const_cast<MfFactor *>(M), s));   // a solve that gave up is no time
    *ms_avg = total / reps;
    return V2D_OK;
}

// Measurement aid: one dataflow solve of a zero vector with a per-item
// trace (ns of the global timer at the ticket, at the end of the item's
// wait, after its done counters): ticks[3 i + k] for the n items (n <= cap).
int mf_trace_apply(const MfPlan *P, const MfFactor *M, cudaStream_t s, unsigned long long *ticks,
                   int cap, int *n)
{
    V2D_ARG_CHECK(M->flow, "LU solve trace: needs the dataflow solve");
    V2D_ARG_CHECK(cap >= P->nitems, "LU solve trace: %d items, room for %d", P->nitems, cap);
    const size_t es = M->fp32 ? sizeof(float) : sizeof(double);
    DevBuf<char> buf;
    V2D_TRY(buf.alloc(2 * P->n * es + 3 * (size_t)P->nitems * sizeof(unsigned long long) + 256, s));
    V2D_CUDA_TRY(cudaMemsetAsync(buf.p, 0, 2 * P->n * es, s));
    unsigned long long *tr = (unsigned long long *)(buf.p + ((2 * P->n * es + 15) / 16) * 16);
    V2D_CUDA_TRY(cudaMemsetAsync(tr, 0, 3 * (size_t)P->nitems * sizeof(unsigned long long), s));
    int st = M->fp32 ? apply_launches<float>(P, M, (const float *)buf.p,
                                             (float *)(buf.p + P->n * es), nullptr, nullptr, s,
                                             nullptr, nullptr, nullptr, 0, tr)
                     : apply_launches<double>(P, M, (const double *)buf.p,
                                              (double *)(buf.p + P->n * es), nullptr, nullptr, s,
                                              nullptr, nullptr, nullptr, 0, tr);
    V2D_TRY(st);
    V2D_CUDA_TRY(cudaMemcpyAsync(ticks, tr, 3 * (size_t)P->nitems * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    V2D_TRY(mf_check_barrier(const_cast<MfFactor *>(M), s));
    *n = P->nitems;
    return V2D_OK;
}

// Keeps the device busy for about `us` microseconds (bounded), so that the
// host can enqueue a whole solve before it starts and per-launch events then
// time the device, not the host's submission.
__global__ void k_delay(int us)
{
    for (int i = 0; i < us; ++i) __nanosleep(1000);
}

int mf_time_apply_launches(const MfPlan *P, const MfFactor *M, int reps, size_t flush_bytes,
                           cudaStream_t s, double *ms, int *codes, int cap, int *n)
{
    const size_t es = M->fp32 ? sizeof(float) : sizeof(double);
    DevBuf<char> buf;
    V2D_TRY(buf.alloc(2 * P->n * es + flush_bytes + 256, s));
    V2D_CUDA_TRY(cudaMemsetAsync(buf.p, 0, 2 * P->n * es, s));
    char *fl = buf.p + 2 * P->n * es;
    std::vector<cudaEvent_t> ev(cap + 1, nullptr);
    int st = V2D_OK;
    for (auto &e : ev)
        if (st == V2D_OK && cudaEventCreate(&e) != cudaSuccess) st = V2D_ECUDA;
    std::vector<double> acc(cap, 0.0);
    long long nl = 0;
    for (int r = 0; r < reps && st == V2D_OK; ++r) {
        if (flush_bytes) cudaMemsetAsync(fl, r & 0xff, flush_bytes, s);
        k_delay<<<1, 32, 0, s>>>(300);
        cudaEventRecord(ev[0], s);
        st = M->fp32 ? apply_launches<float>(P, M, (const float *)buf.p,
                                             (float *)(buf.p + P->n * es), nullptr, nullptr, s,
                                             &nl, ev.data() + 1, codes, cap)
                     : apply_launches<double>(P, M, (const double *)buf.p,
                                              (double *)(buf.p + P->n * es), nullptr, nullptr,
                                              s, &nl, ev.data() + 1, codes, cap);
        if (st == V2D_OK && cudaEventSynchronize(ev[nl]) != cudaSuccess) st = V2D_ECUDA;
        for (long long k = 0; k < nl && st == V2D_OK; ++k) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            acc[k] += t;
        }
    }
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (st != V2D_OK) return st;
    V2D_TRY(mf_check_barrier(const_cast<MfFactor *>(M), s));
    for (long long k = 0; k < nl; ++k) ms[k] = acc[k] / reps;
    *n = (int)nl;
    return V2D_OK;
}

int mf_time_factor_launches(const MfPlan *P, MfFactor *M, const int *rowptr, const double *val,
                            int reps, cudaStream_t s, double *ms, int *codes, int cap, int *n)
{
    std::vector<cudaEvent_t> ev(cap + 1, nullptr);
    int st = V2D_OK;
    for (auto &e : ev)
        if (st == V2D_OK && cudaEventCreate(&e) != cudaSuccess) st = V2D_ECUDA;
    std::vector<double> acc(cap, 0.0);
    int nl = 0;
    for (int r = 0; r < reps && st == V2D_OK; ++r) {
        k_delay<<<1, 32, 0, s>>>(2000);
        cudaEventRecord(ev[0], s);
        st = M->fp32 && !M->fact64
                 ? factor_launches<float>(P, M, rowptr, val, s, ev.data() + 1, codes, cap, &nl)
                 : factor_launches<double>(P, M, rowptr, val, s, ev.data() + 1, codes, cap, &nl);
        if (st == V2D_OK && cudaEventSynchronize(ev[nl]) != cudaSuccess) st = V2D_ECUDA;
        for (int k = 0; k < nl && st == V2D_OK; ++k) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            acc[k] += t;
        }
    }
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (st != V2D_OK) return st;
    for (int k = 0; k < nl; ++k) ms[k] = acc[k] / reps;
    *n = nl;
    return V2D_OK;
}

int mf_check_barrier(MfFactor *M, cudaStream_t s)
{
    if (!M->bar) return V2D_OK;
    int err = 0;
    V2D_CUDA_TRY(cudaMemcpyAsync(&err, &M->bar->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    if (err) {
        V2D_CUDA_TRY(cudaMemsetAsync(M->bar, 0, sizeof(MfBarrier), s));
        set_error("LU solve: a dependency wait of the dataflow solve timed out");
        return V2D_ETIMEOUT;
    }
    return V2D_OK;
}

}  // namespace v2d
