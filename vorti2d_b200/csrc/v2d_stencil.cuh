// Device-side statement of the vorti2d discretisation: Garmann metrics and the
// psi / ome rows of the coupled Newton system.  One definition serves the CSR
// pattern build, the COO seam kernels and the fused Newton assembly, so the
// pattern and the values can never disagree.
//
// Every expression keeps the reference's operand order
// (src/fortran/vorti2d_core.f90); translation units that include this header
// are compiled with -fmad=false so the results are bit-identical to the CPU
// restatement (no FMA contraction, IEEE division and sqrt).
#pragma once

#include "v2d_common.cuh"
#include "v2d_dual.cuh"

namespace v2d {

// Scalars of one assembly call (vorti2d_core.f90:219-227).
struct Coeffs {
    double re, invdtau, inv2dt, urot, dksi, deta, ca, sa;
    int ff_bc;
};

// Field arrays of one assembly call, reference argument order.
struct Fields {
    const double *jac, *alfa, *beta, *gama, *pmet, *qmet, *detadx, *detady, *xphys, *yphys;
    const double *psi, *ome, *omeold, *omeoldold;
};

// Replicated O-grid (vorti2d_core.f90:219-383): imax*jmax nodes including the
// duplicated seam column, neighbours wrap across the branch cut, dofs are
// field-blocked (psi K, ome N+K).
struct GlobalTopo {
    int imax, jmax, N;
    __device__ __forceinline__ int row_of(int K) const { return K / imax; }
    __device__ __forceinline__ int stride() const { return imax; }
    __device__ __forceinline__ Nbr nbrs(int K) const
    {
        int j = K / imax;
        return wrap_neighbors(K - j * imax, j, imax);
    }
    __device__ __forceinline__ int dof(int K, int c) const { return c ? N + K : K; }
};

// Ghosted local block (vorti2d_core.f90:510-661): gxm*jmax nodes, no wrap
// (ghost columns hold the wrapped neighbours), dofs through the
// local-to-global map lg (node-interleaved PETSc ordering).
struct LocalTopo {
    int gxm, jmax;
    const int *lg;
    __device__ __forceinline__ int row_of(int K) const { return K / gxm; }
    __device__ __forceinline__ int stride() const { return gxm; }
    __device__ __forceinline__ Nbr nbrs(int K) const
    {
        Nbr b;
        b.k = K; b.e = K + 1; b.w = K - 1; b.n = K + gxm; b.s = K - gxm;
        b.ne = b.n + 1; b.nw = b.n - 1; b.se = b.s + 1; b.sw = b.s - 1;
        return b;
    }
    __device__ __forceinline__ int dof(int K, int c) const { return lg[2 * K + c]; }
};

// ------------------------------------------------------------------ metrics
// The metric expressions are templates on the scalar type T (double, or the
// Dual numbers of the tangent derivatives) and on the coordinate accessor X
// (x[k] yields a T): the FP64 path instantiates them with T = double and
// plain pointers, which is the same arithmetic in the same order.
//
// d/deta and d2/deta2 of one coordinate along the column through node K (row
// j of jmax, row stride st).  Interior: central (vorti2d_core.f90:109-114);
// j=0: forward one-sided 3/4-point (:130-133); j=jmax-1: backward (:148-151).
template <class T, class X>
__device__ __forceinline__ T eta_d1_t(const X &x, int K, int j, int jmax, int st, double two_de)
{
    if (j == 0) {
        int k1 = K, k2 = K + st, k3 = K + 2 * st;
        return (-3.0 * x[k1] + 4.0 * x[k2] - x[k3]) / two_de;
    } else if (j == jmax - 1) {
        int k1 = K, k2 = K - st, k3 = K - 2 * st;
        return (3.0 * x[k1] - 4.0 * x[k2] + x[k3]) / two_de;
    }
    return (x[K + st] - x[K - st]) / two_de;
}

template <class T, class X>
__device__ __forceinline__ T eta_d2_t(const X &x, int K, int j, int jmax, int st, double de2)
{
    if (j == 0) {
        int k1 = K, k2 = K + st, k3 = K + 2 * st, k4 = K + 3 * st;
        return (2.0 * x[k1] - 5.0 * x[k2] + 4.0 * x[k3] - x[k4]) / de2;
    } else if (j == jmax - 1) {
        int k1 = K, k2 = K - st, k3 = K - 2 * st, k4 = K - 3 * st;
        return (2.0 * x[k1] - 5.0 * x[k2] + 4.0 * x[k3] - x[k4]) / de2;
    }
    return (x[K + st] - 2.0 * x[K] + x[K - st]) / de2;
}

__device__ __forceinline__ double eta_d1(const double *x, int K, int j, int jmax, int st,
                                         double two_de)
{
    return eta_d1_t<double>(x, K, j, jmax, st, two_de);
}

__device__ __forceinline__ double eta_d2(const double *x, int K, int j, int jmax, int st,
                                         double de2)
{
    return eta_d2_t<double>(x, K, j, jmax, st, de2);
}

template <class T>
struct MetricOutT {
    T jac, alfa, beta, gama, pmet, qmet, detadx, detady;
};
using MetricOut = MetricOutT<double>;

// Jacobian + transformation metrics (vorti2d_core.f90:164-182).
template <class T>
__device__ __forceinline__ MetricOutT<T> metric_point_t(T xi, T yi, T xh, T yh, T xii, T yii,
                                                        T xhh, T yhh, T xih, T yih)
{
    MetricOutT<T> m;
    T J = 1.0 / (xi * yh - xh * yi);
    T dksidx = J * yh;
    T dksidy = -J * xh;
    T ex = -J * yi;
    T ey = J * xi;
    T a = dksidx * dksidx + dksidy * dksidy;
    T b = ex * ex + ey * ey;
    T g = dksidx * ex + dksidy * ey;
    m.jac = J; m.detadx = ex; m.detady = ey; m.alfa = a; m.beta = b; m.gama = g;
    m.pmet = -(a * (xii * dksidx + yii * dksidy) + 2.0 * g * (xih * dksidx + yih * dksidy)
               + b * (xhh * dksidx + yhh * dksidy));
    m.qmet = -(a * (xii * ex + yii * ey) + 2.0 * g * (xih * ex + yih * ey)
               + b * (xhh * ex + yhh * ey));
    return m;
}

__device__ __forceinline__ MetricOut metric_point(double xi, double yi, double xh, double yh,
                                                  double xii, double yii, double xhh,
                                                  double yhh, double xih, double yih)
{
    return metric_point_t<double>(xi, yi, xh, yh, xii, yii, xhh, yhh, xih, yih);
}

// Metrics at node K with east/west neighbours e, w on the same row j.
template <class T, class X>
__device__ __forceinline__ MetricOutT<T> metrics_at_t(const X &x, const X &y, int K, int e,
                                                      int w, int j, int jmax, int st,
                                                      double dksi, double deta)
{
    const double two_dk = 2.0 * dksi, two_de = 2.0 * deta;
    const double dk2 = dksi * dksi, de2 = deta * deta;
    T xi = (x[e] - x[w]) / two_dk;
    T yi = (y[e] - y[w]) / two_dk;
    T xii = (x[e] - 2.0 * x[K] + x[w]) / dk2;
    T yii = (y[e] - 2.0 * y[K] + y[w]) / dk2;
    T xh = eta_d1_t<T>(x, K, j, jmax, st, two_de);
    T yh = eta_d1_t<T>(y, K, j, jmax, st, two_de);
    T xhh = eta_d2_t<T>(x, K, j, jmax, st, de2);
    T yhh = eta_d2_t<T>(y, K, j, jmax, st, de2);
    // cross derivative = ksi-central of d/deta (vorti2d_core.f90:155-161):
    // d/deta at the e and w columns is recomputed here with the same formula
    T xih = (eta_d1_t<T>(x, e, j, jmax, st, two_de) - eta_d1_t<T>(x, w, j, jmax, st, two_de)) /
            two_dk;
    T yih = (eta_d1_t<T>(y, e, j, jmax, st, two_de) - eta_d1_t<T>(y, w, j, jmax, st, two_de)) /
            two_dk;
    return metric_point_t<T>(xi, yi, xh, yh, xii, yii, xhh, yhh, xih, yih);
}

__device__ __forceinline__ MetricOut metrics_at(const double *x, const double *y, int K, int e,
                                                int w, int j, int jmax, int st, double dksi,
                                                double deta)
{
    return metrics_at_t<double>(x, y, K, e, w, j, jmax, st, dksi, deta);
}

// ----------------------------------------------------------------- rows
constexpr int kPsiMax = 10;  // interior psi row: 9 psi + 1 ome entries
constexpr int kOmeMax = 13;  // interior ome row: 9 ome + 4 psi entries

// Right-hand sides b = -R of the rows whose values depend on the metrics,
// templates on the type T of the metric values (double, or Dual for the
// tangent derivatives; the state is FP64 either way).
// Interior psi row (vorti2d_core.f90:295-300).
template <class T>
__device__ __forceinline__ T psi_rhs_interior(double re, double dksi, double deta, T a, T bt,
                                              T g, T pm, T qm, const double *psi,
                                              const double *ome, int K, const Nbr &nb)
{
    T Pp = (a / re) * ((psi[nb.e] - 2.0 * psi[K] + psi[nb.w]) / (dksi * dksi));
    T Qq = 2.0 * (g / re) *
           ((psi[nb.ne] - psi[nb.nw] - psi[nb.se] + psi[nb.sw]) / (4.0 * deta * dksi));
    T Rr = (bt / re) * ((psi[nb.n] - 2.0 * psi[K] + psi[nb.s]) / (deta * deta));
    T Ss = (pm / re) * ((psi[nb.e] - psi[nb.w]) / (2.0 * dksi));
    T Tt = (qm / re) * ((psi[nb.n] - psi[nb.s]) / (2.0 * deta));
    return Pp + Qq + Rr + Ss + Tt + ome[K] / re;
}

// Far-field psi row, Dirichlet form (vorti2d_core.f90:266-269).
template <class T>
__device__ __forceinline__ T psi_rhs_far(double ca, double sa, T xk, T yk, double psik)
{
    return (ca * yk - sa * xk) - psik;
}

// Wall omega row, Thom type with the rotation term (vorti2d_core.f90:322-339).
template <class T>
__device__ __forceinline__ T ome_rhs_wall(double deta, double urot, T beta, T qmet, T detadx,
                                          T detady, T xk, T yk, const double *psi,
                                          const double *ome, int K, int n, int nn)
{
    T bw = beta / (deta * deta);
    T rad = tsqrt(xk * xk + yk * yk);
    T ct = xk / rad, sn = yk / rad;
    return ome[K] - (7.0 / 2.0) * bw * psi[K] + (8.0 / 2.0) * bw * psi[n]
           - (1.0 / 2.0) * bw * psi[nn]
           - ((qmet - 3.0 * (beta / deta)) * (urot / (detadx * ct + detady * sn)));
}

// Interior omega row (vorti2d_core.f90:341-378).
template <class T>
__device__ __forceinline__ T ome_rhs_interior(double re, double dksi, double deta, double inv2dt,
                                              T J, T a, T bt, T g, T pm, T qm,
                                              const double *psi, const double *ome,
                                              const double *omeold, const double *omeoldold,
                                              int K, const Nbr &nb)
{
    double Aa = (psi[nb.n] - psi[nb.s]) / (2.0 * deta);
    double Bb = (ome[nb.e] - ome[nb.w]) / (2.0 * dksi);
    double Cc = (psi[nb.e] - psi[nb.w]) / (2.0 * dksi);
    double Dd = (ome[nb.n] - ome[nb.s]) / (2.0 * deta);
    T Ee = (a / re) * ((ome[nb.e] - 2.0 * ome[K] + ome[nb.w]) / (dksi * dksi));
    T Ff = 2.0 * (g / re) *
           ((ome[nb.ne] - ome[nb.nw] - ome[nb.se] + ome[nb.sw]) / (4.0 * deta * dksi));
    T Gg = (bt / re) * ((ome[nb.n] - 2.0 * ome[K] + ome[nb.s]) / (deta * deta));
    T Hh = (pm / re) * ((ome[nb.e] - ome[nb.w]) / (2.0 * dksi));
    T Ii = (qm / re) * ((ome[nb.n] - ome[nb.s]) / (2.0 * deta));
    return -(J * Aa * Bb) + (J * Cc * Dd) + Ee + Ff + Gg + Hh + Ii
           - ((3.0 * ome[K] - 4.0 * omeold[K] + omeoldold[K]) * inv2dt);
}

__device__ __forceinline__ bool outflow_arc(const Coeffs &c, const Fields &f, int K)
{
    return (c.ca * f.detadx[K] + c.sa * f.detady[K]) > 0.0;
}

// Entry count of the psi row of node K (pattern only needs detadx/detady).
template <class Topo>
__device__ __forceinline__ int psi_row_count(const Topo &T, const Coeffs &c, const Fields &f,
                                             int K)
{
    int j = T.row_of(K);
    if (j == T.jmax - 1) return (c.ff_bc >= 2 && outflow_arc(c, f, K)) ? 3 : 1;
    if (j == 0) return 1;
    return kPsiMax;
}

template <class Topo>
__device__ __forceinline__ int ome_row_count(const Topo &T, const Coeffs &c, const Fields &f,
                                             int K)
{
    int j = T.row_of(K);
    if (j == T.jmax - 1) return (c.ff_bc >= 1 && outflow_arc(c, f, K)) ? 3 : 1;
    if (j == 0) return 4;
    return kOmeMax;
}

// psi row of node K in push order (vorti2d_core.f90:251-301).  VAL=false fills
// only the columns (pattern build).  Returns the entry count.
template <bool VAL, class Topo>
__device__ __forceinline__ int psi_row(const Topo &T, const Coeffs &c, const Fields &f, int K,
                                       int *col, double *val, double *b)
{
    const int j = T.row_of(K), st = T.stride();
    const double re = c.re, dksi = c.dksi, deta = c.deta;
    if (j == T.jmax - 1) {
        if (c.ff_bc >= 2 && outflow_arc(c, f, K)) {
            int ks = K - st, ks2 = K - 2 * st;
            col[0] = T.dof(K, 0); col[1] = T.dof(ks, 0); col[2] = T.dof(ks2, 0);
            if (VAL) {
                val[0] = 1.0; val[1] = -2.0; val[2] = 1.0;
                *b = -(f.psi[K] - 2.0 * f.psi[ks] + f.psi[ks2]);
            }
            return 3;
        }
        col[0] = T.dof(K, 0);
        if (VAL) {
            val[0] = 1.0;
            *b = psi_rhs_far<double>(c.ca, c.sa, f.xphys[K], f.yphys[K], f.psi[K]);
        }
        return 1;
    }
    if (j == 0) {
        col[0] = T.dof(K, 0);
        if (VAL) {
            val[0] = 1.0;
            *b = 0.0 - f.psi[K];
        }
        return 1;
    }
    const Nbr nb = T.nbrs(K);
    col[0] = T.dof(K, 0); col[1] = T.dof(nb.e, 0); col[2] = T.dof(nb.w, 0);
    col[3] = T.dof(nb.n, 0); col[4] = T.dof(nb.s, 0); col[5] = T.dof(nb.ne, 0);
    col[6] = T.dof(nb.nw, 0); col[7] = T.dof(nb.se, 0); col[8] = T.dof(nb.sw, 0);
    col[9] = T.dof(K, 1);
    if (VAL) {
        const double a = f.alfa[K], bt = f.beta[K], g = f.gama[K], pm = f.pmet[K], qm = f.qmet[K];
        const double *psi = f.psi;
        double cgam = (2.0 * g) / (4.0 * re * dksi * deta);
        val[0] = c.invdtau + ((2.0 * a) / (dksi * dksi) + (2.0 * bt) / (deta * deta)) / re;
        val[1] = -(a / (re * (dksi * dksi)) + pm / (2.0 * re * dksi));
        val[2] = (-a / (re * (dksi * dksi)) + pm / (2.0 * re * dksi));
        val[3] = -(bt / (re * (deta * deta)) + qm / (2.0 * re * deta));
        val[4] = (-bt / (re * (deta * deta)) + qm / (2.0 * re * deta));
        val[5] = -cgam;
        val[6] = cgam;
        val[7] = cgam;
        val[8] = -cgam;
        val[9] = -1.0 / re;
        *b = psi_rhs_interior<double>(re, dksi, deta, a, bt, g, pm, qm, psi, f.ome, K, nb);
    }
    return kPsiMax;
}

// ome row of node K in push order (vorti2d_core.f90:303-379).
template <bool VAL, class Topo>
__device__ __forceinline__ int ome_row(const Topo &T, const Coeffs &c, const Fields &f, int K,
                                       int *col, double *val, double *b)
{
    const int j = T.row_of(K), st = T.stride();
    const double re = c.re, dksi = c.dksi, deta = c.deta;
    if (j == T.jmax - 1) {
        if (c.ff_bc >= 1 && outflow_arc(c, f, K)) {
            int ks = K - st, ks2 = K - 2 * st;
            col[0] = T.dof(K, 1); col[1] = T.dof(ks, 1); col[2] = T.dof(ks2, 1);
            if (VAL) {
                val[0] = 1.0; val[1] = -4.0 / 3.0; val[2] = 1.0 / 3.0;
                *b = (4.0 * f.ome[ks] - f.ome[ks2]) / 3.0 - f.ome[K];
            }
            return 3;
        }
        col[0] = T.dof(K, 1);
        if (VAL) {
            val[0] = 1.0;
            *b = 0.0 - f.ome[K];
        }
        return 1;
    }
    if (j == 0) {
        // wall vorticity, Thom type, psi-coupled (vorti2d_core.f90:322-339)
        int n = K + st, nn = K + 2 * st;
        col[0] = T.dof(K, 1); col[1] = T.dof(K, 0); col[2] = T.dof(n, 0); col[3] = T.dof(nn, 0);
        if (VAL) {
            const double *psi = f.psi;
            double bw = f.beta[K] / (deta * deta);
            val[0] = -1.0;
            val[1] = (7.0 / 2.0) * bw;
            val[2] = -(8.0 / 2.0) * bw;
            val[3] = (1.0 / 2.0) * bw;
            *b = ome_rhs_wall<double>(deta, c.urot, f.beta[K], f.qmet[K], f.detadx[K],
                                      f.detady[K], f.xphys[K], f.yphys[K], psi, f.ome, K, n,
                                      nn);
        }
        return 4;
    }
    const Nbr nb = T.nbrs(K);
    col[0] = T.dof(K, 1); col[1] = T.dof(nb.e, 1); col[2] = T.dof(nb.w, 1);
    col[3] = T.dof(nb.n, 1); col[4] = T.dof(nb.s, 1); col[5] = T.dof(nb.ne, 1);
    col[6] = T.dof(nb.nw, 1); col[7] = T.dof(nb.se, 1); col[8] = T.dof(nb.sw, 1);
    col[9] = T.dof(nb.n, 0); col[10] = T.dof(nb.s, 0); col[11] = T.dof(nb.e, 0);
    col[12] = T.dof(nb.w, 0);
    if (VAL) {
        const double *psi = f.psi, *ome = f.ome;
        const double a = f.alfa[K], bt = f.beta[K], g = f.gama[K], pm = f.pmet[K], qm = f.qmet[K];
        const double J = f.jac[K];
        double Aa = (psi[nb.n] - psi[nb.s]) / (2.0 * deta);
        double Bb = (ome[nb.e] - ome[nb.w]) / (2.0 * dksi);
        double Cc = (psi[nb.e] - psi[nb.w]) / (2.0 * dksi);
        double Dd = (ome[nb.n] - ome[nb.s]) / (2.0 * deta);
        double cab = a / (re * (dksi * dksi));
        double cbt = bt / (re * (deta * deta));
        double cgam = (2.0 * g) / (4.0 * re * dksi * deta);
        val[0] = c.invdtau + (2.0 * a) / (re * (dksi * dksi)) + (2.0 * bt) / (re * (deta * deta))
                 + 3.0 * c.inv2dt;
        val[1] = ((J * Aa) / (2.0 * dksi)) - cab - pm / (2.0 * re * dksi);
        val[2] = (-(J * Aa) / (2.0 * dksi)) - cab + pm / (2.0 * re * dksi);
        val[3] = (-(J * Cc) / (2.0 * deta)) - cbt - qm / (2.0 * re * deta);
        val[4] = ((J * Cc) / (2.0 * deta)) - cbt + qm / (2.0 * re * deta);
        val[5] = -cgam;
        val[6] = cgam;
        val[7] = cgam;
        val[8] = -cgam;
        val[9] = (J * Bb) / (2.0 * deta);
        val[10] = -(J * Bb) / (2.0 * deta);
        val[11] = -(J * Dd) / (2.0 * dksi);
        val[12] = (J * Dd) / (2.0 * dksi);
        *b = ome_rhs_interior<double>(re, dksi, deta, c.inv2dt, J, a, bt, g, pm, qm, psi, ome,
                                      f.omeold, f.omeoldold, K, nb);
    }
    return kOmeMax;
}

// Position of entry e inside its canonical (column-sorted) CSR row: the number
// of the row's columns smaller than col[e].  Rows hold no duplicate columns
// for imax, jmax >= 4, so ranks are a permutation of 0..cnt-1.
template <int MAXE>
__device__ __forceinline__ int col_rank(const int *col, int cnt, int e)
{
    int r = 0;
#pragma unroll
    for (int f = 0; f < MAXE; ++f)
        if (f < cnt && col[f] < col[e]) ++r;
    return r;
}

}  // namespace v2d
