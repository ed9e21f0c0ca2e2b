// Force / moment coefficients on the device (reference vorti2d/forces.py:82-194).
//
// One block walks the P = imax-1 distinct wall nodes (j = 0; i = imax-1 is the
// seam duplicate of i = 0): wall-normal vorticity gradient
// (gamma*omega_xi + beta*omega_eta)/sqrt(beta) with omega_xi periodic-central
// and omega_eta one-sided into the domain, periodic-trapezoid arc weights,
// pressure force by parts, friction from the wall vorticity, moment about
// (x0, y0), and the arc-weighted mean-radius reference length when none is
// given.  Sums use fixed-order block reductions in FP64.
#include "v2d_internal.cuh"

namespace v2d {

constexpr int kForceThreads = 256;

__global__ void __launch_bounds__(kForceThreads) k_forces(int imax, double dksi, double deta,
                                                          const double *beta, const double *gama,
                                                          const double *detadx, const double *detady,
                                                          const double *xp, const double *yp,
                                                          const double *ome, double re,
                                                          double ref_length, double x0, double y0,
                                                          double *out)
{
    __shared__ double red[32];
    const int P = imax - 1;
    double s_fxp = 0, s_fyp = 0, s_fxf = 0, s_fyf = 0, s_mzp = 0, s_mzf = 0;
    double s_w = 0, s_xw = 0, s_yw = 0;
    for (int w = threadIdx.x; w < P; w += blockDim.x) {
        const int wp = (w + 1) % P, wm = (w + P - 1) % P;
        const double xw = xp[w], yw = yp[w], ow = ome[w], bw = beta[w], gw = gama[w];
        const double inv_gn = 1.0 / sqrt(bw);
        const double nx = detadx[w] * inv_gn, ny = detady[w] * inv_gn;
        const double tx = ny, ty = -nx;
        const double ome_xi = (ome[wp] - ome[wm]) / (2.0 * dksi);
        const double ome_eta = (-3.0 * ow + 4.0 * ome[imax + w] - ome[2 * imax + w]) / (2.0 * deta);
        const double dwdn = (gw * ome_xi + bw * ome_eta) * inv_gn;
        const double segf = sqrt((xp[wp] - xw) * (xp[wp] - xw) + (yp[wp] - yw) * (yp[wp] - yw));
        const double segb = sqrt((xw - xp[wm]) * (xw - xp[wm]) + (yw - yp[wm]) * (yw - yp[wm]));
        const double ds = 0.5 * (segf + segb);
        const double fric = (1.0 / re) * ow;
        const double rx = xw - x0, ry = yw - y0;
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
    s_fxp = block_sum(s_fxp, red);
    s_fyp = block_sum(s_fyp, red);
    s_fxf = block_sum(s_fxf, red);
    s_fyf = block_sum(s_fyf, red);
    s_mzp = block_sum(s_mzp, red);
    s_mzf = block_sum(s_mzf, red);
    s_w = block_sum(s_w, red);
    s_xw = block_sum(s_xw, red);
    s_yw = block_sum(s_yw, red);
    double d = ref_length;
    if (!(d > 0.0)) {
        const double cx = s_xw / s_w, cy = s_yw / s_w;
        double s_r = 0.0;
        for (int w = threadIdx.x; w < P; w += blockDim.x) {
            const int wp = (w + 1) % P, wm = (w + P - 1) % P;
            const double xw = xp[w], yw = yp[w];
            const double segf = sqrt((xp[wp] - xw) * (xp[wp] - xw) + (yp[wp] - yw) * (yp[wp] - yw));
            const double segb = sqrt((xw - xp[wm]) * (xw - xp[wm]) + (yw - yp[wm]) * (yw - yp[wm]));
            s_r += sqrt((xw - cx) * (xw - cx) + (yw - cy) * (yw - cy)) * (0.5 * (segf + segb));
        }
        s_r = block_sum(s_r, red);
        d = 2.0 * (s_r / s_w);
    }
    if (threadIdx.x == 0) {
        const double fxp = (1.0 / re) * s_fxp, fyp = -(1.0 / re) * s_fyp;
        const double mzp = -(1.0 / (2.0 * re)) * s_mzp;
        const double cdp = 2.0 * fxp / d, cdf = 2.0 * s_fxf / d;
        const double clp = 2.0 * fyp / d, clf = 2.0 * s_fyf / d;
        const double cmp = 2.0 * mzp / (d * d), cmf = 2.0 * s_mzf / (d * d);
        out[0] = cdp + cdf; out[1] = clp + clf; out[2] = cmp + cmf;
        out[3] = cdp; out[4] = cdf; out[5] = clp; out[6] = clf; out[7] = cmp; out[8] = cmf;
        out[9] = d;
    }
}

int launch_forces(const GridDev &g, double re, double ref_length, double x0, double y0,
                  double *d_out10, cudaStream_t s)
{
    k_forces<<<1, kForceThreads, 0, s>>>(g.imax, g.dksi, g.deta, g.met[2], g.met[3], g.met[6],
                                         g.met[7], g.met[8], g.met[9], g.ome, re, ref_length, x0,
                                         y0, d_out10);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    return V2D_OK;
}

}  // namespace v2d

using namespace v2d;

extern "C" int v2d_force_coeffs(int imax, int jmax, double re, double dksi, double deta,
                                const double *beta, const double *gama, const double *detadx,
                                const double *detady, const double *xphys, const double *yphys,
                                const double *ome, double ref_length, double x0, double y0,
                                double *out10)
{
    V2D_ARG_CHECK(imax >= 4 && jmax >= 3, "force_coeffs: mesh %d x %d too small", imax, jmax);
    V2D_ARG_CHECK(beta && gama && detadx && detady && xphys && yphys && ome && out10,
                  "force_coeffs: null pointer");
    cudaStream_t s = 0;
    const size_t N = (size_t)imax * jmax;
    DevBuf<double> buf;
    V2D_TRY(buf.alloc(7 * N + 16, s));
    const double *h[7] = {beta, gama, detadx, detady, xphys, yphys, ome};
    for (int q = 0; q < 7; ++q)
        V2D_CUDA_TRY(cudaMemcpyAsync(buf.p + q * N, h[q], N * sizeof(double), cudaMemcpyHostToDevice, s));
    double *d = buf.p;
    k_forces<<<1, kForceThreads, 0, s>>>(imax, dksi, deta, d, d + N, d + 2 * N, d + 3 * N,
                                         d + 4 * N, d + 5 * N, d + 6 * N, re, ref_length, x0, y0,
                                         d + 7 * N);
    V2D_CUDA_TRY(cudaGetLastError());
    V2D_CUDA_TRY(cudaMemcpyAsync(out10, d + 7 * N, 10 * sizeof(double), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    return V2D_OK;
}
