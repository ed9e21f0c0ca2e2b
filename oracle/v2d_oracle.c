/*
 * ORACLE -- test infrastructure only.
 *
 * CPU restatement of the vorti2d compute kernels (src/fortran/vorti2d_core.f90
 * of the reference).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load this library, and only as the
 * checker or the timed CPU baseline; the product path never calls it.
 *
 * Parity anchor: the reference Fortran cannot be compiled in this image (no
 * Fortran compiler), so this restatement is pinned by the reference's own
 * known-answer tests (boundary values, symmetry, Ingham drag, outflow ==
 * dirichlet drag, angle-of-attack far field, local == global metrics and
 * Newton update) and by the drag values the reference documents for the
 * 181x181 analytic grid.
 *
 * Arithmetic follows the Fortran expression order term by term (left to right
 * as written, x**2 as x*x) and must be compiled without FP contraction
 * (-ffp-contract=off), so the CUDA kernels built with -fmad=false reproduce it
 * bit for bit.
 *
 * Conventions (vorti2d_core.f90:10-19): 1-based node pointer
 * k = imax*(j-1) + i; arrays below are 0-based, so field[k-1].  COO indices are
 * emitted 0-based, in the same push order as the reference, so the COO
 * sequences are identical.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define V2D_ORACLE_OK 0
#define V2D_ORACLE_EOVERFLOW (-2)
#define V2D_ORACLE_EARG (-1)

/* vorti2d_core.f90:33-61 -- 1-based neighbour pointers with the branch-cut
 * wrap (i=1 west -> i=imax-1, i=imax east -> i=2). out = k,e,w,n,s,ne,nw,se,sw */
void v2d_oracle_node_neighbors(int i, int j, int imax, int *out)
{
    int k = imax * (j - 1) + i;
    int n = k + imax, s = k - imax;
    int e, w, ne, nw, se, sw;
    if (i == 1) {
        e = k + 1; w = k + imax - 2;
        ne = n + 1; nw = n + imax - 2;
        se = s + 1; sw = s + imax - 2;
    } else if (i == imax) {
        e = k - imax + 2; w = k - 1;
        ne = n - imax + 2; nw = n - 1;
        se = s - imax + 2; sw = s - 1;
    } else {
        e = k + 1; w = k - 1;
        ne = n + 1; nw = n - 1;
        se = s + 1; sw = s - 1;
    }
    out[0] = k; out[1] = e; out[2] = w; out[3] = n; out[4] = s;
    out[5] = ne; out[6] = nw; out[7] = se; out[8] = sw;
}

/* Final metric block shared by the global and local variants
 * (vorti2d_core.f90:164-182 and :472-486). */
static void metric_point(double xi, double yi, double xh, double yh,
                         double xii, double yii, double xhh, double yhh,
                         double xih, double yih,
                         double *jac, double *alfa, double *beta, double *gama,
                         double *pmet, double *qmet, double *detadx, double *detady)
{
    /* xi = dx/dksi, xh = dx/deta, xii = d2x/dksi2, xhh = d2x/deta2,
     * xih = d2x/dksi deta (same for y) */
    double J = 1.0 / (xi * yh - xh * yi);
    double dksidx = J * yh;
    double dksidy = -J * xh;
    double ex = -J * yi;
    double ey = J * xi;
    double a = dksidx * dksidx + dksidy * dksidy;
    double b = ex * ex + ey * ey;
    double g = dksidx * ex + dksidy * ey;
    *jac = J; *detadx = ex; *detady = ey;
    *alfa = a; *beta = b; *gama = g;
    *pmet = -(a * (xii * dksidx + yii * dksidy)
              + 2.0 * g * (xih * dksidx + yih * dksidy)
              + b * (xhh * dksidx + yhh * dksidy));
    *qmet = -(a * (xii * ex + yii * ey)
              + 2.0 * g * (xih * ex + yih * ey)
              + b * (xhh * ex + yhh * ey));
}

/* vorti2d_core.f90:66-189.  xg, yg are Fortran-ordered (imax, jmax): element
 * (i, j) at xg[(i-1) + imax*(j-1)], i.e. already in pointer order. */
int v2d_oracle_compute_metrics(int imax, int jmax, double dksi, double deta,
                               const double *xg, const double *yg,
                               double *jac, double *alfa, double *beta, double *gama,
                               double *pmet, double *qmet, double *detadx, double *detady,
                               double *xphys, double *yphys)
{
    if (imax < 4 || jmax < 4) return V2D_ORACLE_EARG;
    int N = imax * jmax;
    double *x = (double *)calloc((size_t)N * 12, sizeof(double));
    if (!x) return V2D_ORACLE_EARG;
    double *y = x + N;
    double *xi = y + N, *yi = xi + N, *xh = yi + N, *yh = xh + N;      /* d/dksi, d/deta */
    double *xii = yh + N, *yii = xii + N, *xhh = yii + N, *yhh = xhh + N;
    double *xih = yhh + N, *yih = xih + N;
    int nb[9];
    const double two_dk = 2.0 * dksi, two_de = 2.0 * deta;
    const double dk2 = dksi * dksi, de2 = deta * deta;

    for (int k = 0; k < N; ++k) { x[k] = xg[k]; y[k] = yg[k]; }

    /* interior eta range (:104-116) */
    for (int j = 2; j <= jmax - 1; ++j)
        for (int i = 1; i <= imax; ++i) {
            v2d_oracle_node_neighbors(i, j, imax, nb);
            int k = nb[0] - 1, e = nb[1] - 1, w = nb[2] - 1, n = nb[3] - 1, s = nb[4] - 1;
            xi[k] = (x[e] - x[w]) / two_dk;
            yi[k] = (y[e] - y[w]) / two_dk;
            xh[k] = (x[n] - x[s]) / two_de;
            yh[k] = (y[n] - y[s]) / two_de;
            xii[k] = (x[e] - 2.0 * x[k] + x[w]) / dk2;
            yii[k] = (y[e] - 2.0 * y[k] + y[w]) / dk2;
            xhh[k] = (x[n] - 2.0 * x[k] + x[s]) / de2;
            yhh[k] = (y[n] - 2.0 * y[k] + y[s]) / de2;
        }
    /* wall j=1, one-sided forward in eta (:119-134) */
    for (int i = 1; i <= imax; ++i) {
        v2d_oracle_node_neighbors(i, 1, imax, nb);
        int k = nb[0] - 1, e = nb[1] - 1, w = nb[2] - 1;
        int k1 = i - 1, k2 = imax + i - 1, k3 = 2 * imax + i - 1, k4 = 3 * imax + i - 1;
        xi[k] = (x[e] - x[w]) / two_dk;
        yi[k] = (y[e] - y[w]) / two_dk;
        xii[k] = (x[e] - 2.0 * x[k] + x[w]) / dk2;
        yii[k] = (y[e] - 2.0 * y[k] + y[w]) / dk2;
        xh[k] = (-3.0 * x[k1] + 4.0 * x[k2] - x[k3]) / two_de;
        yh[k] = (-3.0 * y[k1] + 4.0 * y[k2] - y[k3]) / two_de;
        xhh[k] = (2.0 * x[k1] - 5.0 * x[k2] + 4.0 * x[k3] - x[k4]) / de2;
        yhh[k] = (2.0 * y[k1] - 5.0 * y[k2] + 4.0 * y[k3] - y[k4]) / de2;
    }
    /* far field j=jmax, one-sided backward in eta (:137-152) */
    for (int i = 1; i <= imax; ++i) {
        v2d_oracle_node_neighbors(i, jmax, imax, nb);
        int k = nb[0] - 1, e = nb[1] - 1, w = nb[2] - 1;
        int k1 = imax * (jmax - 1) + i - 1, k2 = imax * (jmax - 2) + i - 1;
        int k3 = imax * (jmax - 3) + i - 1, k4 = imax * (jmax - 4) + i - 1;
        xi[k] = (x[e] - x[w]) / two_dk;
        yi[k] = (y[e] - y[w]) / two_dk;
        xii[k] = (x[e] - 2.0 * x[k] + x[w]) / dk2;
        yii[k] = (y[e] - 2.0 * y[k] + y[w]) / dk2;
        xh[k] = (3.0 * x[k1] - 4.0 * x[k2] + x[k3]) / two_de;
        yh[k] = (3.0 * y[k1] - 4.0 * y[k2] + y[k3]) / two_de;
        xhh[k] = (2.0 * x[k1] - 5.0 * x[k2] + 4.0 * x[k3] - x[k4]) / de2;
        yhh[k] = (2.0 * y[k1] - 5.0 * y[k2] + 4.0 * y[k3] - y[k4]) / de2;
    }
    /* cross derivative = ksi-central of d/deta (:155-161) */
    for (int j = 1; j <= jmax; ++j)
        for (int i = 1; i <= imax; ++i) {
            v2d_oracle_node_neighbors(i, j, imax, nb);
            int k = nb[0] - 1, e = nb[1] - 1, w = nb[2] - 1;
            xih[k] = (xh[e] - xh[w]) / two_dk;
            yih[k] = (yh[e] - yh[w]) / two_dk;
        }
    for (int k = 0; k < N; ++k)
        metric_point(xi[k], yi[k], xh[k], yh[k], xii[k], yii[k], xhh[k], yhh[k],
                     xih[k], yih[k], &jac[k], &alfa[k], &beta[k], &gama[k], &pmet[k],
                     &qmet[k], &detadx[k], &detady[k]);
    for (int k = 0; k < N; ++k) { xphys[k] = x[k]; yphys[k] = y[k]; }
    free(x);
    return V2D_ORACLE_OK;
}

/* vorti2d_core.f90:392-495.  Ghosted local block gxm x jmax, owned 1-based
 * columns [il0, il1], no wrap.  Outputs are zero outside the owned columns
 * (xphys/yphys hold the whole local mesh). */
int v2d_oracle_compute_metrics_local(int gxm, int jmax, int il0, int il1,
                                     double dksi, double deta,
                                     const double *xgl, const double *ygl,
                                     double *jac, double *alfa, double *beta, double *gama,
                                     double *pmet, double *qmet, double *detadx,
                                     double *detady, double *xphys, double *yphys)
{
    if (jmax < 4 || il0 < 2 || il1 > gxm - 1 || il0 > il1) return V2D_ORACLE_EARG;
    int N = gxm * jmax;
    double *x = (double *)calloc((size_t)N * 4, sizeof(double));
    if (!x) return V2D_ORACLE_EARG;
    double *y = x + N, *xh = y + N, *yh = xh + N;
    const double two_dk = 2.0 * dksi, two_de = 2.0 * deta;
    const double dk2 = dksi * dksi, de2 = deta * deta;
    for (int k = 0; k < N; ++k) {
        x[k] = xgl[k]; y[k] = ygl[k];
        jac[k] = alfa[k] = beta[k] = gama[k] = 0.0;
        pmet[k] = qmet[k] = detadx[k] = detady[k] = 0.0;
    }
    /* d/deta on every column (:431-444) */
    for (int il = 1; il <= gxm; ++il) {
        for (int j = 2; j <= jmax - 1; ++j) {
            int k = gxm * (j - 1) + il - 1;
            xh[k] = (x[k + gxm] - x[k - gxm]) / two_de;
            yh[k] = (y[k + gxm] - y[k - gxm]) / two_de;
        }
        int k1 = il - 1, k2 = gxm + il - 1, k3 = 2 * gxm + il - 1;
        xh[k1] = (-3.0 * x[k1] + 4.0 * x[k2] - x[k3]) / two_de;
        yh[k1] = (-3.0 * y[k1] + 4.0 * y[k2] - y[k3]) / two_de;
        k1 = gxm * (jmax - 1) + il - 1; k2 = gxm * (jmax - 2) + il - 1;
        k3 = gxm * (jmax - 3) + il - 1;
        xh[k1] = (3.0 * x[k1] - 4.0 * x[k2] + x[k3]) / two_de;
        yh[k1] = (3.0 * y[k1] - 4.0 * y[k2] + y[k3]) / two_de;
    }
    /* owned columns (:447-488) */
    for (int il = il0; il <= il1; ++il)
        for (int j = 1; j <= jmax; ++j) {
            int k = gxm * (j - 1) + il - 1, e = k + 1, w = k - 1;
            double xi = (x[e] - x[w]) / two_dk;
            double yi = (y[e] - y[w]) / two_dk;
            double xii = (x[e] - 2.0 * x[k] + x[w]) / dk2;
            double yii = (y[e] - 2.0 * y[k] + y[w]) / dk2;
            double xhh, yhh;
            if (j >= 2 && j <= jmax - 1) {
                int n = k + gxm, s = k - gxm;
                xhh = (x[n] - 2.0 * x[k] + x[s]) / de2;
                yhh = (y[n] - 2.0 * y[k] + y[s]) / de2;
            } else if (j == 1) {
                int k1 = il - 1, k2 = gxm + il - 1, k3 = 2 * gxm + il - 1, k4 = 3 * gxm + il - 1;
                xhh = (2.0 * x[k1] - 5.0 * x[k2] + 4.0 * x[k3] - x[k4]) / de2;
                yhh = (2.0 * y[k1] - 5.0 * y[k2] + 4.0 * y[k3] - y[k4]) / de2;
            } else {
                int k1 = gxm * (jmax - 1) + il - 1, k2 = gxm * (jmax - 2) + il - 1;
                int k3 = gxm * (jmax - 3) + il - 1, k4 = gxm * (jmax - 4) + il - 1;
                xhh = (2.0 * x[k1] - 5.0 * x[k2] + 4.0 * x[k3] - x[k4]) / de2;
                yhh = (2.0 * y[k1] - 5.0 * y[k2] + 4.0 * y[k3] - y[k4]) / de2;
            }
            double xih = (xh[e] - xh[w]) / two_dk;
            double yih = (yh[e] - yh[w]) / two_dk;
            metric_point(xi, yi, xh[k], yh[k], xii, yii, xhh, yhh, xih, yih,
                         &jac[k], &alfa[k], &beta[k], &gama[k], &pmet[k], &qmet[k],
                         &detadx[k], &detady[k]);
        }
    for (int k = 0; k < N; ++k) { xphys[k] = x[k]; yphys[k] = y[k]; }
    free(x);
    return V2D_ORACLE_OK;
}

/* COO append; the reference's push (:664-674) has no capacity check, here an
 * overflow is reported instead of writing past the buffers. */
#define PUSH(gi, gj, val)                                                   \
    do {                                                                    \
        if (m >= maxnnz) { status = V2D_ORACLE_EOVERFLOW; goto done; }      \
        ci[m] = (gi); cj[m] = (gj); cv[m] = (val); ++m;                     \
    } while (0)

/* Field arrays of one assembly call, in the reference argument order. */
typedef struct {
    const double *jac, *alfa, *beta, *gama, *pmet, *qmet, *detadx, *detady, *xphys, *yphys;
    const double *psi, *ome, *omeold, *omeoldold;
} v2d_fields;

/* vorti2d_core.f90:219-383 -- field-blocked global assembly of rows [r0, r1). */
int v2d_oracle_assemble_coo(int imax, int jmax, double re, double invdtau, double inv2dt,
                            double urot, double dksi, double deta,
                            const double *jac, const double *alfa, const double *beta,
                            const double *gama, const double *pmet, const double *qmet,
                            const double *detadx, const double *detady,
                            const double *xphys, const double *yphys,
                            const double *psi, const double *ome, const double *omeold,
                            const double *omeoldold, int r0, int r1, int maxnnz, int ff_bc,
                            double ca, double sa, int *ci, int *cj, double *cv, int *nnz,
                            double *bvec)
{
    const int ndof = imax * jmax, pblk = 0, oblk = ndof;
    int m = 0, status = V2D_ORACLE_OK;
    int nb[9];
    if (imax < 4 || jmax < 4 || r0 < 0 || r1 > 2 * ndof || r0 > r1) return V2D_ORACLE_EARG;
    for (int r = r0; r < r1; ++r) bvec[r - r0] = 0.0;

    for (int r = r0; r < r1; ++r) {
        int lr = r - r0;
        if (r < ndof) {
            int k = r + 1, j = (k - 1) / imax + 1, i = k - imax * (j - 1);
            int K = k - 1; /* 0-based */
            if (j == jmax) {
                if (ff_bc >= 2 && (ca * detadx[K] + sa * detady[K]) > 0.0) {
                    int ks = K - imax, ks2 = K - 2 * imax;
                    PUSH(r, pblk + K, 1.0);
                    PUSH(r, pblk + ks, -2.0);
                    PUSH(r, pblk + ks2, 1.0);
                    bvec[lr] = -(psi[K] - 2.0 * psi[ks] + psi[ks2]);
                } else {
                    PUSH(r, pblk + K, 1.0);
                    bvec[lr] = (ca * yphys[K] - sa * xphys[K]) - psi[K];
                }
            } else if (j == 1) {
                PUSH(r, pblk + K, 1.0);
                bvec[lr] = 0.0 - psi[K];
            } else {
                v2d_oracle_node_neighbors(i, j, imax, nb);
                int e = nb[1] - 1, w = nb[2] - 1, n = nb[3] - 1, s = nb[4] - 1;
                int ne = nb[5] - 1, nw = nb[6] - 1, se = nb[7] - 1, sw = nb[8] - 1;
                double cgam = (2.0 * gama[K]) / (4.0 * re * dksi * deta);
                PUSH(r, pblk + K,
                     invdtau + ((2.0 * alfa[K]) / (dksi * dksi) + (2.0 * beta[K]) / (deta * deta)) / re);
                PUSH(r, pblk + e, -(alfa[K] / (re * (dksi * dksi)) + pmet[K] / (2.0 * re * dksi)));
                PUSH(r, pblk + w, (-alfa[K] / (re * (dksi * dksi)) + pmet[K] / (2.0 * re * dksi)));
                PUSH(r, pblk + n, -(beta[K] / (re * (deta * deta)) + qmet[K] / (2.0 * re * deta)));
                PUSH(r, pblk + s, (-beta[K] / (re * (deta * deta)) + qmet[K] / (2.0 * re * deta)));
                PUSH(r, pblk + ne, -cgam);
                PUSH(r, pblk + nw, cgam);
                PUSH(r, pblk + se, cgam);
                PUSH(r, pblk + sw, -cgam);
                PUSH(r, oblk + K, -1.0 / re);
                double Pp = (alfa[K] / re) * ((psi[e] - 2.0 * psi[K] + psi[w]) / (dksi * dksi));
                double Qq = 2.0 * (gama[K] / re) *
                            ((psi[ne] - psi[nw] - psi[se] + psi[sw]) / (4.0 * deta * dksi));
                double Rr = (beta[K] / re) * ((psi[n] - 2.0 * psi[K] + psi[s]) / (deta * deta));
                double Ss = (pmet[K] / re) * ((psi[e] - psi[w]) / (2.0 * dksi));
                double Tt = (qmet[K] / re) * ((psi[n] - psi[s]) / (2.0 * deta));
                bvec[lr] = Pp + Qq + Rr + Ss + Tt + ome[K] / re;
            }
        } else {
            int k = r - ndof + 1, j = (k - 1) / imax + 1, i = k - imax * (j - 1);
            int K = k - 1;
            if (j == jmax) {
                if (ff_bc >= 1 && (ca * detadx[K] + sa * detady[K]) > 0.0) {
                    int ks = K - imax, ks2 = K - 2 * imax;
                    PUSH(r, oblk + K, 1.0);
                    PUSH(r, oblk + ks, -4.0 / 3.0);
                    PUSH(r, oblk + ks2, 1.0 / 3.0);
                    bvec[lr] = (4.0 * ome[ks] - ome[ks2]) / 3.0 - ome[K];
                } else {
                    PUSH(r, oblk + K, 1.0);
                    bvec[lr] = 0.0 - ome[K];
                }
            } else if (j == 1) {
                int n = imax + i - 1, nn = 2 * imax + i - 1;
                double bw = beta[K] / (deta * deta);
                PUSH(r, oblk + K, -1.0);
                PUSH(r, pblk + K, (7.0 / 2.0) * bw);
                PUSH(r, pblk + n, -(8.0 / 2.0) * bw);
                PUSH(r, pblk + nn, (1.0 / 2.0) * bw);
                double rad = sqrt(xphys[K] * xphys[K] + yphys[K] * yphys[K]);
                double ct = xphys[K] / rad, st = yphys[K] / rad;
                bvec[lr] = ome[K] - (7.0 / 2.0) * bw * psi[K] + (8.0 / 2.0) * bw * psi[n]
                           - (1.0 / 2.0) * bw * psi[nn]
                           - ((qmet[K] - 3.0 * (beta[K] / deta)) *
                              (urot / (detadx[K] * ct + detady[K] * st)));
            } else {
                v2d_oracle_node_neighbors(i, j, imax, nb);
                int e = nb[1] - 1, w = nb[2] - 1, n = nb[3] - 1, s = nb[4] - 1;
                int ne = nb[5] - 1, nw = nb[6] - 1, se = nb[7] - 1, sw = nb[8] - 1;
                double Aa = (psi[n] - psi[s]) / (2.0 * deta);
                double Bb = (ome[e] - ome[w]) / (2.0 * dksi);
                double Cc = (psi[e] - psi[w]) / (2.0 * dksi);
                double Dd = (ome[n] - ome[s]) / (2.0 * deta);
                double Ee = (alfa[K] / re) * ((ome[e] - 2.0 * ome[K] + ome[w]) / (dksi * dksi));
                double Ff = 2.0 * (gama[K] / re) *
                            ((ome[ne] - ome[nw] - ome[se] + ome[sw]) / (4.0 * deta * dksi));
                double Gg = (beta[K] / re) * ((ome[n] - 2.0 * ome[K] + ome[s]) / (deta * deta));
                double Hh = (pmet[K] / re) * ((ome[e] - ome[w]) / (2.0 * dksi));
                double Ii = (qmet[K] / re) * ((ome[n] - ome[s]) / (2.0 * deta));
                double cab = alfa[K] / (re * (dksi * dksi));
                double cbt = beta[K] / (re * (deta * deta));
                double cgam = (2.0 * gama[K]) / (4.0 * re * dksi * deta);
                PUSH(r, oblk + K,
                     invdtau + (2.0 * alfa[K]) / (re * (dksi * dksi)) +
                         (2.0 * beta[K]) / (re * (deta * deta)) + 3.0 * inv2dt);
                PUSH(r, oblk + e, ((jac[K] * Aa) / (2.0 * dksi)) - cab - pmet[K] / (2.0 * re * dksi));
                PUSH(r, oblk + w, (-(jac[K] * Aa) / (2.0 * dksi)) - cab + pmet[K] / (2.0 * re * dksi));
                PUSH(r, oblk + n, (-(jac[K] * Cc) / (2.0 * deta)) - cbt - qmet[K] / (2.0 * re * deta));
                PUSH(r, oblk + s, ((jac[K] * Cc) / (2.0 * deta)) - cbt + qmet[K] / (2.0 * re * deta));
                PUSH(r, oblk + ne, -cgam);
                PUSH(r, oblk + nw, cgam);
                PUSH(r, oblk + se, cgam);
                PUSH(r, oblk + sw, -cgam);
                PUSH(r, pblk + n, (jac[K] * Bb) / (2.0 * deta));
                PUSH(r, pblk + s, -(jac[K] * Bb) / (2.0 * deta));
                PUSH(r, pblk + e, -(jac[K] * Dd) / (2.0 * dksi));
                PUSH(r, pblk + w, (jac[K] * Dd) / (2.0 * dksi));
                bvec[lr] = -(jac[K] * Aa * Bb) + (jac[K] * Cc * Dd) + Ee + Ff + Gg + Hh + Ii
                           - ((3.0 * ome[K] - 4.0 * omeold[K] + omeoldold[K]) * inv2dt);
            }
        }
    }
done:
    *nnz = m;
    return status;
}

/* vorti2d_core.f90:510-661 -- ghosted local block, node-interleaved global
 * dofs through lg (gdof(kk,c) = lg[2*(kk-1)+c], 0-based entries). */
int v2d_oracle_assemble_coo_local(int gxm, int jmax, int il0, int il1, double re,
                                  double invdtau, double inv2dt, double urot, double dksi,
                                  double deta, const double *jac, const double *alfa,
                                  const double *beta, const double *gama, const double *pmet,
                                  const double *qmet, const double *detadx,
                                  const double *detady, const double *xphys,
                                  const double *yphys, const double *psi, const double *ome,
                                  const double *omeold, const double *omeoldold, int r0,
                                  int nloc, const int *lg, int maxnnz, int ff_bc, double ca,
                                  double sa, int *ci, int *cj, double *cv, int *nnz,
                                  double *bvec)
{
    int m = 0, status = V2D_ORACLE_OK;
    if (jmax < 4 || il0 < 2 || il1 > gxm - 1 || il0 > il1) return V2D_ORACLE_EARG;
#define GD(kk, c) lg[2 * (kk) + (c)]
#define BROW(g) (((g) - r0) >= 0 && ((g) - r0) < nloc ? &bvec[(g) - r0] : &sink)
    double sink = 0.0;
    for (int t = 0; t < nloc; ++t) bvec[t] = 0.0;
    for (int jj = 1; jj <= jmax; ++jj)
        for (int il = il0; il <= il1; ++il) {
            int K = gxm * (jj - 1) + il - 1; /* 0-based local node */
            int gp = GD(K, 0), go = GD(K, 1);
            /* psi equation */
            if (jj == jmax) {
                if (ff_bc >= 2 && (ca * detadx[K] + sa * detady[K]) > 0.0) {
                    int ks = K - gxm, ks2 = K - 2 * gxm;
                    PUSH(gp, GD(K, 0), 1.0);
                    PUSH(gp, GD(ks, 0), -2.0);
                    PUSH(gp, GD(ks2, 0), 1.0);
                    *BROW(gp) = -(psi[K] - 2.0 * psi[ks] + psi[ks2]);
                } else {
                    PUSH(gp, GD(K, 0), 1.0);
                    *BROW(gp) = (ca * yphys[K] - sa * xphys[K]) - psi[K];
                }
            } else if (jj == 1) {
                PUSH(gp, GD(K, 0), 1.0);
                *BROW(gp) = 0.0 - psi[K];
            } else {
                int e = K + 1, w = K - 1, n = K + gxm, s = K - gxm;
                int ne = n + 1, nw = n - 1, se = s + 1, sw = s - 1;
                double cgam = (2.0 * gama[K]) / (4.0 * re * dksi * deta);
                PUSH(gp, GD(K, 0),
                     invdtau + ((2.0 * alfa[K]) / (dksi * dksi) + (2.0 * beta[K]) / (deta * deta)) / re);
                PUSH(gp, GD(e, 0), -(alfa[K] / (re * (dksi * dksi)) + pmet[K] / (2.0 * re * dksi)));
                PUSH(gp, GD(w, 0), (-alfa[K] / (re * (dksi * dksi)) + pmet[K] / (2.0 * re * dksi)));
                PUSH(gp, GD(n, 0), -(beta[K] / (re * (deta * deta)) + qmet[K] / (2.0 * re * deta)));
                PUSH(gp, GD(s, 0), (-beta[K] / (re * (deta * deta)) + qmet[K] / (2.0 * re * deta)));
                PUSH(gp, GD(ne, 0), -cgam);
                PUSH(gp, GD(nw, 0), cgam);
                PUSH(gp, GD(se, 0), cgam);
                PUSH(gp, GD(sw, 0), -cgam);
                PUSH(gp, GD(K, 1), -1.0 / re);
                double Pp = (alfa[K] / re) * ((psi[e] - 2.0 * psi[K] + psi[w]) / (dksi * dksi));
                double Qq = 2.0 * (gama[K] / re) *
                            ((psi[ne] - psi[nw] - psi[se] + psi[sw]) / (4.0 * deta * dksi));
                double Rr = (beta[K] / re) * ((psi[n] - 2.0 * psi[K] + psi[s]) / (deta * deta));
                double Ss = (pmet[K] / re) * ((psi[e] - psi[w]) / (2.0 * dksi));
                double Tt = (qmet[K] / re) * ((psi[n] - psi[s]) / (2.0 * deta));
                *BROW(gp) = Pp + Qq + Rr + Ss + Tt + ome[K] / re;
            }
            /* ome equation */
            if (jj == jmax) {
                if (ff_bc >= 1 && (ca * detadx[K] + sa * detady[K]) > 0.0) {
                    int ks = K - gxm, ks2 = K - 2 * gxm;
                    PUSH(go, GD(K, 1), 1.0);
                    PUSH(go, GD(ks, 1), -4.0 / 3.0);
                    PUSH(go, GD(ks2, 1), 1.0 / 3.0);
                    *BROW(go) = (4.0 * ome[ks] - ome[ks2]) / 3.0 - ome[K];
                } else {
                    PUSH(go, GD(K, 1), 1.0);
                    *BROW(go) = 0.0 - ome[K];
                }
            } else if (jj == 1) {
                int n2 = K + gxm, n3 = K + 2 * gxm;
                double bw = beta[K] / (deta * deta);
                PUSH(go, GD(K, 1), -1.0);
                PUSH(go, GD(K, 0), (7.0 / 2.0) * bw);
                PUSH(go, GD(n2, 0), -(8.0 / 2.0) * bw);
                PUSH(go, GD(n3, 0), (1.0 / 2.0) * bw);
                double rad = sqrt(xphys[K] * xphys[K] + yphys[K] * yphys[K]);
                double ct = xphys[K] / rad, st = yphys[K] / rad;
                *BROW(go) = ome[K] - (7.0 / 2.0) * bw * psi[K] + (8.0 / 2.0) * bw * psi[n2]
                            - (1.0 / 2.0) * bw * psi[n3]
                            - ((qmet[K] - 3.0 * (beta[K] / deta)) *
                               (urot / (detadx[K] * ct + detady[K] * st)));
            } else {
                int e = K + 1, w = K - 1, n = K + gxm, s = K - gxm;
                int ne = n + 1, nw = n - 1, se = s + 1, sw = s - 1;
                double Aa = (psi[n] - psi[s]) / (2.0 * deta);
                double Bb = (ome[e] - ome[w]) / (2.0 * dksi);
                double Cc = (psi[e] - psi[w]) / (2.0 * dksi);
                double Dd = (ome[n] - ome[s]) / (2.0 * deta);
                double Ee = (alfa[K] / re) * ((ome[e] - 2.0 * ome[K] + ome[w]) / (dksi * dksi));
                double Ff = 2.0 * (gama[K] / re) *
                            ((ome[ne] - ome[nw] - ome[se] + ome[sw]) / (4.0 * deta * dksi));
                double Gg = (beta[K] / re) * ((ome[n] - 2.0 * ome[K] + ome[s]) / (deta * deta));
                double Hh = (pmet[K] / re) * ((ome[e] - ome[w]) / (2.0 * dksi));
                double Ii = (qmet[K] / re) * ((ome[n] - ome[s]) / (2.0 * deta));
                double cab = alfa[K] / (re * (dksi * dksi));
                double cbt = beta[K] / (re * (deta * deta));
                double cgam = (2.0 * gama[K]) / (4.0 * re * dksi * deta);
                PUSH(go, GD(K, 1),
                     invdtau + (2.0 * alfa[K]) / (re * (dksi * dksi)) +
                         (2.0 * beta[K]) / (re * (deta * deta)) + 3.0 * inv2dt);
                PUSH(go, GD(e, 1), ((jac[K] * Aa) / (2.0 * dksi)) - cab - pmet[K] / (2.0 * re * dksi));
                PUSH(go, GD(w, 1), (-(jac[K] * Aa) / (2.0 * dksi)) - cab + pmet[K] / (2.0 * re * dksi));
                PUSH(go, GD(n, 1), (-(jac[K] * Cc) / (2.0 * deta)) - cbt - qmet[K] / (2.0 * re * deta));
                PUSH(go, GD(s, 1), ((jac[K] * Cc) / (2.0 * deta)) - cbt + qmet[K] / (2.0 * re * deta));
                PUSH(go, GD(ne, 1), -cgam);
                PUSH(go, GD(nw, 1), cgam);
                PUSH(go, GD(se, 1), cgam);
                PUSH(go, GD(sw, 1), -cgam);
                PUSH(go, GD(n, 0), (jac[K] * Bb) / (2.0 * deta));
                PUSH(go, GD(s, 0), -(jac[K] * Bb) / (2.0 * deta));
                PUSH(go, GD(e, 0), -(jac[K] * Dd) / (2.0 * dksi));
                PUSH(go, GD(w, 0), (jac[K] * Dd) / (2.0 * dksi));
                *BROW(go) = -(jac[K] * Aa * Bb) + (jac[K] * Cc * Dd) + Ee + Ff + Gg + Hh + Ii
                            - ((3.0 * ome[K] - 4.0 * omeold[K] + omeoldold[K]) * inv2dt);
            }
        }
#undef GD
#undef BROW
done:
    *nnz = m;
    return status;
}
