// Cartesian velocity from the streamfunction on the device (reference
// vorti2d/velocity.py:38-93), built with -fmad=false: every expression keeps
// the reference's operand order, so the result equals the reference's NumPy
// evaluation bit for bit.
//
//   xi_x = (gamma eta_x + J eta_y) / beta,  xi_y = (gamma eta_y - J eta_x) / beta
//   u = psi_xi xi_y + psi_eta eta_y,        v = -(psi_xi xi_x + psi_eta eta_x)
//
// psi_xi is central with the O-grid branch-cut wrap (i = 0 and i = imax-1
// take i = 1 and i = imax-2 as neighbours); psi_eta is central in the
// interior and second-order one-sided at the wall and the far field.
#include <cmath>

#include "v2d_internal.cuh"

namespace v2d {

__global__ void __launch_bounds__(256) k_velocity(int imax, int jmax, double dksi, double deta,
                                                  const double *__restrict__ jac,
                                                  const double *__restrict__ beta,
                                                  const double *__restrict__ gama,
                                                  const double *__restrict__ detadx,
                                                  const double *__restrict__ detady,
                                                  const double *__restrict__ psi, double *u,
                                                  double *v, double *vmag)
{
    const int N = imax * jmax;
    V2D_GRID_STRIDE(t, N)
    {
        const int K = (int)t;
        const int j = K / imax, i = K - j * imax;
        const double xix = (gama[K] * detadx[K] + jac[K] * detady[K]) / beta[K];
        const double xiy = (gama[K] * detady[K] - jac[K] * detadx[K]) / beta[K];
        const int ie = (i == 0 || i == imax - 1) ? 1 : i + 1;
        const int iw = (i == 0 || i == imax - 1) ? imax - 2 : i - 1;
        const int row = j * imax;
        const double psi_xi = (psi[row + ie] - psi[row + iw]) / (2.0 * dksi);
        double psi_eta;
        if (j == 0)
            psi_eta = (-3.0 * psi[K] + 4.0 * psi[K + imax] - psi[K + 2 * imax]) / (2.0 * deta);
        else if (j == jmax - 1)
            psi_eta = (3.0 * psi[K] - 4.0 * psi[K - imax] + psi[K - 2 * imax]) / (2.0 * deta);
        else
            psi_eta = (psi[K + imax] - psi[K - imax]) / (2.0 * deta);
        const double uu = psi_xi * xiy + psi_eta * detady[K];
        const double vv = -(psi_xi * xix + psi_eta * detadx[K]);
        u[K] = uu;
        v[K] = vv;
        if (vmag) vmag[K] = sqrt(uu * uu + vv * vv);
    }
}

int launch_velocity(int imax, int jmax, double dksi, double deta, const double *jac,
                    const double *beta, const double *gama, const double *detadx,
                    const double *detady, const double *psi, double *u, double *v, double *vmag,
                    cudaStream_t s)
{
    k_velocity<<<grid_for((long long)imax * jmax, 256), 256, 0, s>>>(
        imax, jmax, dksi, deta, jac, beta, gama, detadx, detady, psi, u, v, vmag);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(1);
    return V2D_OK;
}

}  // namespace v2d

using namespace v2d;

extern "C" int v2d_compute_velocity(int imax, int jmax, double dksi, double deta,
                                    const double *jac, const double *beta, const double *gama,
                                    const double *detadx, const double *detady,
                                    const double *psi, double *u, double *v, double *vmag)
{
    V2D_ARG_CHECK(imax >= 4 && jmax >= 3, "compute_velocity: mesh %d x %d too small", imax, jmax);
    V2D_ARG_CHECK(jac && beta && gama && detadx && detady && psi && u && v,
                  "compute_velocity: null pointer");
    cudaStream_t s = 0;
    const size_t N = (size_t)imax * jmax;
    DevBuf<double> buf;
    V2D_TRY(buf.alloc(9 * N, s));
    const double *h[6] = {jac, beta, gama, detadx, detady, psi};
    for (int q = 0; q < 6; ++q)
        V2D_CUDA_TRY(cudaMemcpyAsync(buf.p + q * N, h[q], N * sizeof(double), cudaMemcpyHostToDevice, s));
    double *d = buf.p;
    V2D_TRY(launch_velocity(imax, jmax, dksi, deta, d, d + N, d + 2 * N, d + 3 * N, d + 4 * N,
                            d + 5 * N, d + 6 * N, d + 7 * N, vmag ? d + 8 * N : nullptr, s));
    V2D_CUDA_TRY(cudaMemcpyAsync(u, d + 6 * N, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaMemcpyAsync(v, d + 7 * N, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (vmag)
        V2D_CUDA_TRY(cudaMemcpyAsync(vmag, d + 8 * N, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    V2D_CUDA_TRY(cudaStreamSynchronize(s));
    return V2D_OK;
}
