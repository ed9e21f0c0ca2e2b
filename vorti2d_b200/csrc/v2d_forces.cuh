// Force / moment coefficients of one block (reference vorti2d/forces.py:82-194),
// a template on the scalar type T (double, or Dual for tangent derivatives)
// and on the wall accessor W: W.node(w) returns the wall node w's
// coordinates and metrics (x, y, beta, gama, detadx, detady of type T).
//
// The block walks the P = imax-1 distinct wall nodes (j = 0; i = imax-1 is the
// seam duplicate of i = 0): wall-normal vorticity gradient
// (gamma*omega_xi + beta*omega_eta)/sqrt(beta) with omega_xi periodic-central
// and omega_eta one-sided into the domain, periodic-trapezoid arc weights,
// pressure force by parts, friction from the wall vorticity, moment about
// (x0, y0), and the arc-weighted mean-radius reference length when none is
// given.  Sums use fixed-order block reductions.
#pragma once

#include "v2d_dual.cuh"
#include "v2d_util.cuh"

namespace v2d {

template <class T>
struct WallNode {
    T x, y, beta, gama, detadx, detady;
};

__device__ __forceinline__ double block_sum_t(double v, double *red) { return block_sum(v, red); }
__device__ __forceinline__ Dual block_sum_t(Dual v, double *red)
{
    const double a = block_sum(v.v, red);
    return {a, block_sum(v.d, red)};
}

// out10 (thread 0) = cd, cl, cm, cdp, cdf, clp, clf, cmp, cmf, ref_length.
template <class T, class W>
__device__ __forceinline__ void force_block(int imax, double dksi, double deta, const W &wall,
                                            const double *ome, double re, double ref_length,
                                            double x0, double y0, T *out10)
{
    __shared__ double red[32];
    const int P = imax - 1;
    const T zero = tconst<T>(0.0);
    T s_fxp = zero, s_fyp = zero, s_fxf = zero, s_fyf = zero, s_mzp = zero, s_mzf = zero;
    T s_w = zero, s_xw = zero, s_yw = zero;
    for (int w = threadIdx.x; w < P; w += blockDim.x) {
        const int wp = (w + 1) % P, wm = (w + P - 1) % P;
        const WallNode<T> a = wall.node(w), ap = wall.node(wp), am = wall.node(wm);
        const T xw = a.x, yw = a.y, bw = a.beta, gw = a.gama;
        const double ow = ome[w];
        const T inv_gn = 1.0 / tsqrt(bw);
        const T nx = a.detadx * inv_gn, ny = a.detady * inv_gn;
        const T tx = ny, ty = -nx;
        const double ome_xi = (ome[wp] - ome[wm]) / (2.0 * dksi);
        const double ome_eta = (-3.0 * ow + 4.0 * ome[imax + w] - ome[2 * imax + w]) / (2.0 * deta);
        const T dwdn = (gw * ome_xi + bw * ome_eta) * inv_gn;
        const T segf = tsqrt((ap.x - xw) * (ap.x - xw) + (ap.y - yw) * (ap.y - yw));
        const T segb = tsqrt((xw - am.x) * (xw - am.x) + (yw - am.y) * (yw - am.y));
        const T ds = 0.5 * (segf + segb);
        const double fric = (1.0 / re) * ow;
        const T rx = xw - x0, ry = yw - y0;
        s_fxp += yw * dwdn * ds;
        s_fyp += xw * dwdn * ds;
        s_fxf += -fric * tx * ds;
        s_fyf += -fric * ty * ds;
        s_mzp += (rx * rx + ry * ry) * dwdn * ds;
        s_mzf += (rx * (-fric * ty) - ry * (-fric * tx)) * ds;
        s_w += ds;
        s_xw += xw * ds;
        s_yw += yw * ds;
    }
    s_fxp = block_sum_t(s_fxp, red);
    s_fyp = block_sum_t(s_fyp, red);
    s_fxf = block_sum_t(s_fxf, red);
    s_fyf = block_sum_t(s_fyf, red);
    s_mzp = block_sum_t(s_mzp, red);
    s_mzf = block_sum_t(s_mzf, red);
    s_w = block_sum_t(s_w, red);
    s_xw = block_sum_t(s_xw, red);
    s_yw = block_sum_t(s_yw, red);
    T d = tconst<T>(ref_length);
    if (!(ref_length > 0.0)) {
        const T cx = s_xw / s_w, cy = s_yw / s_w;
        T s_r = zero;
        for (int w = threadIdx.x; w < P; w += blockDim.x) {
            const int wp = (w + 1) % P, wm = (w + P - 1) % P;
            const WallNode<T> a = wall.node(w), ap = wall.node(wp), am = wall.node(wm);
            const T xw = a.x, yw = a.y;
            const T segf = tsqrt((ap.x - xw) * (ap.x - xw) + (ap.y - yw) * (ap.y - yw));
            const T segb = tsqrt((xw - am.x) * (xw - am.x) + (yw - am.y) * (yw - am.y));
            s_r += tsqrt((xw - cx) * (xw - cx) + (yw - cy) * (yw - cy)) * (0.5 * (segf + segb));
        }
        s_r = block_sum_t(s_r, red);
        d = 2.0 * (s_r / s_w);
    }
    if (threadIdx.x == 0) {
        const T fxp = (1.0 / re) * s_fxp, fyp = -(1.0 / re) * s_fyp;
        const T mzp = -(1.0 / (2.0 * re)) * s_mzp;
        const T cdp = 2.0 * fxp / d, cdf = 2.0 * s_fxf / d;
        const T clp = 2.0 * fyp / d, clf = 2.0 * s_fyf / d;
        const T cmp = 2.0 * mzp / (d * d), cmf = 2.0 * s_mzf / (d * d);
        out10[0] = cdp + cdf; out10[1] = clp + clf; out10[2] = cmp + cmf;
        out10[3] = cdp; out10[4] = cdf; out10[5] = clp; out10[6] = clf; out10[7] = cmp;
        out10[8] = cmf; out10[9] = d;
    }
}

}  // namespace v2d
