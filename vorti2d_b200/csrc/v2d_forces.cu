// Force / moment coefficients on the device (reference vorti2d/forces.py:82-194):
// one block evaluates force_block (v2d_forces.cuh) over the wall nodes of the
// metric arrays.
#include "v2d_internal.cuh"
#include "v2d_forces.cuh"

namespace v2d {

constexpr int kForceThreads = 256;

// Wall nodes from the metric arrays (the first imax entries: row j = 0).
struct WallArrays {
    const double *beta, *gama, *detadx, *detady, *xp, *yp;
    __device__ __forceinline__ WallNode<double> node(int w) const
    {
        return {xp[w], yp[w], beta[w], gama[w], detadx[w], detady[w]};
    }
};

__global__ void __launch_bounds__(kForceThreads) k_forces(int imax, double dksi, double deta,
                                                          const double *beta, const double *gama,
                                                          const double *detadx, const double *detady,
                                                          const double *xp, const double *yp,
                                                          const double *ome, double re,
                                                          double ref_length, double x0, double y0,
                                                          double *out)
{
    const WallArrays wall{beta, gama, detadx, detady, xp, yp};
    force_block<double>(imax, dksi, deta, wall, ome, re, ref_length, x0, y0, out);
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
