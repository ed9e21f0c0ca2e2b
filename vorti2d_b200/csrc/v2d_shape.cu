// Tangent (forward-mode) derivatives of the residual and of the wall force
// integrals with respect to wall-normal shape displacements, for the shape
// gradients of the steady adjoint.
//
// Direction i (i < P = imax-1) moves grid line i -- and the seam line
// imax-1 with i = 0, its duplicate -- by (nx[i], ny[i]) * phi, phi the
// deformation weight of every node (1 at the wall, 0 at the far field).  The
// metrics (vorti2d_core.f90:66-189) are evaluated in Dual numbers whose
// derivative part is the coordinates' derivative along that direction, and
// the residual rows (vorti2d_core.f90:219-381) and the force integrals
// (vorti2d/forces.py:82-194) propagate it: the same expressions as the FP64
// path (v2d_stencil.cuh, v2d_forces.cuh), instantiated on Dual.  Exact
// derivatives of the discrete residual and forces; no finite-difference step.
//
// A node's rows use only its own metrics, and its metrics only the nodes of
// its own column and the two neighbouring ones, so direction i changes the
// rows of at most four columns: one CTA per direction walks those.
#include "v2d_internal.cuh"
#include "v2d_forces.cuh"
#include "v2d_stencil.cuh"

namespace v2d {

namespace {

constexpr int kShapeThreads = 256;

// Coordinates with the derivative of direction i: x[k] + t n phi[k] on the
// displaced columns c0 (and c1, -1 for none).
struct ShapeCoord {
    const double *x, *phi;
    double n;
    int imax, c0, c1;
    __device__ __forceinline__ Dual operator[](int k) const
    {
        const int i = k % imax;
        return {x[k], (i == c0 || i == c1) ? n * phi[k] : 0.0};
    }
};

__device__ __forceinline__ bool moved(int col, int c0, int c1) { return col == c0 || col == c1; }

// dots[i] = lambda . db/dd_i (b = -R, the residual of the handle's system at
// its state; the far-field outflow arcs as at the undisplaced mesh).
__global__ void __launch_bounds__(kShapeThreads) k_shape_residual_tangent(
    GlobalTopo T, Coeffs c, const double *x, const double *y, const double *phi, const double *nx,
    const double *ny, Fields f, const double *lam, double *dots)
{
    __shared__ double red[32];
    const int imax = T.imax, jmax = T.jmax, N = T.N;
    const int i = blockIdx.x;
    const int c0 = i, c1 = i == 0 ? imax - 1 : -1;
    const ShapeCoord X{x, phi, nx[i], imax, c0, c1}, Y{y, phi, ny[i], imax, c0, c1};
    // columns whose stencil (w, self, e) can meet a displaced column, each once
    const int cand[7] = {i - 1, i, i + 1, 0, 1, imax - 2, imax - 1};
    double acc = 0.0;
    for (int t = threadIdx.x; t < 7 * jmax; t += blockDim.x) {
        const int u = t / jmax, j = t - u * jmax, col = cand[u];
        if (col < 0 || col >= imax) continue;
        bool dup = false;
        for (int v = 0; v < u; ++v) dup = dup || cand[v] == col;
        if (dup) continue;
        const Nbr nb = wrap_neighbors(col, j, imax);
        if (!moved(col, c0, c1) && !moved(nb.e % imax, c0, c1) && !moved(nb.w % imax, c0, c1))
            continue;
        const int K = nb.k;
        const MetricOutT<Dual> m =
            metrics_at_t<Dual>(X, Y, K, nb.e, nb.w, j, jmax, imax, c.dksi, c.deta);
        Dual bpsi = tconst<Dual>(0.0), bome = tconst<Dual>(0.0);
        if (j == jmax - 1) {
            const bool arc = (c.ca * m.detadx.v + c.sa * m.detady.v) > 0.0;
            if (!(c.ff_bc >= 2 && arc)) bpsi = psi_rhs_far<Dual>(c.ca, c.sa, X[K], Y[K], f.psi[K]);
        } else if (j == 0) {
            bome = ome_rhs_wall<Dual>(c.deta, c.urot, m.beta, m.qmet, m.detadx, m.detady, X[K],
                                      Y[K], f.psi, f.ome, K, K + imax, K + 2 * imax);
        } else {
            bpsi = psi_rhs_interior<Dual>(c.re, c.dksi, c.deta, m.alfa, m.beta, m.gama, m.pmet,
                                          m.qmet, f.psi, f.ome, K, nb);
            bome = ome_rhs_interior<Dual>(c.re, c.dksi, c.deta, c.inv2dt, m.jac, m.alfa, m.beta,
                                          m.gama, m.pmet, m.qmet, f.psi, f.ome, f.omeold,
                                          f.omeoldold, K, nb);
        }
        acc += lam[K] * bpsi.d + lam[N + K] * bome.d;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) dots[i] = acc;
}

// Wall nodes with Dual coordinates and metrics of direction i.
struct WallTangent {
    ShapeCoord X, Y;
    int imax, jmax;
    double dksi, deta;
    __device__ __forceinline__ WallNode<Dual> node(int w) const
    {
        const Nbr nb = wrap_neighbors(w, 0, imax);
        const MetricOutT<Dual> m =
            metrics_at_t<Dual>(X, Y, w, nb.e, nb.w, 0, jmax, imax, dksi, deta);
        return {X[w], Y[w], m.beta, m.gama, m.detadx, m.detady};
    }
};

// dforces[10 i + c] = d(force value c)/dd_i (the 10 values of v2d_force_coeffs).
__global__ void __launch_bounds__(kShapeThreads) k_shape_force_tangent(
    int imax, int jmax, double dksi, double deta, const double *x, const double *y,
    const double *phi, const double *nx, const double *ny, const double *ome, double re,
    double ref_length, double x0, double y0, double *dforces)
{
    __shared__ Dual out[10];
    const int i = blockIdx.x;
    const int c1 = i == 0 ? imax - 1 : -1;
    const WallTangent wall{ShapeCoord{x, phi, nx[i], imax, i, c1},
                           ShapeCoord{y, phi, ny[i], imax, i, c1}, imax, jmax, dksi, deta};
    force_block<Dual>(imax, dksi, deta, wall, ome, re, ref_length, x0, y0, out);
    __syncthreads();
    if (threadIdx.x < 10) dforces[10 * i + threadIdx.x] = out[threadIdx.x].d;
}

}  // namespace

int launch_shape_tangent(const GridDev &g, const AsmParams &p, const double *phi,
                         const double *nx, const double *ny, const double *lam, double ref_length,
                         double x0, double y0, double *dots, double *dforces, cudaStream_t s)
{
    const int P = g.imax - 1;
    GlobalTopo T{g.imax, g.jmax, g.N};
    Coeffs c{p.re, p.invdtau, p.inv2dt, p.urot, g.dksi, g.deta, p.ca, p.sa, p.ff_bc};
    Fields f;
    f.jac = g.met[0]; f.alfa = g.met[1]; f.beta = g.met[2]; f.gama = g.met[3];
    f.pmet = g.met[4]; f.qmet = g.met[5]; f.detadx = g.met[6]; f.detady = g.met[7];
    f.xphys = g.met[8]; f.yphys = g.met[9];
    f.psi = g.psi; f.ome = g.ome; f.omeold = g.omeold; f.omeoldold = g.omeoldold;
    k_shape_residual_tangent<<<P, kShapeThreads, 0, s>>>(T, c, g.x, g.y, phi, nx, ny, f, lam,
                                                         dots);
    V2D_CUDA_TRY(cudaGetLastError());
    k_shape_force_tangent<<<P, kShapeThreads, 0, s>>>(g.imax, g.jmax, g.dksi, g.deta, g.x, g.y,
                                                      phi, nx, ny, g.ome, p.re, ref_length, x0,
                                                      y0, dforces);
    V2D_CUDA_TRY(cudaGetLastError());
    count_launches(2);
    return V2D_OK;
}

}  // namespace v2d
