// Internal interfaces between the translation units of libvorti2d_b200.
#pragma once

#include "v2d_util.cuh"

namespace v2d {

// One replicated O-grid in HBM.  Every array is SoA in pointer order
// K = imax*j + i (i fastest); the Newton system is the field-blocked 2N
// system of the reference (psi rows [0,N), ome rows [N,2N)) in canonical CSR.
struct GridDev {
    int imax = 0, jmax = 0, N = 0, n = 0;
    double dksi = 0, deta = 0;
    double *x = nullptr, *y = nullptr;   // mesh, pointer order
    double *met[10] = {};                // jac alfa beta gama pmet qmet detadx detady xphys yphys
    double *psi = nullptr, *ome = nullptr, *omeold = nullptr, *omeoldold = nullptr;
    int *rowptr = nullptr, *colind = nullptr;
    long long nnz = 0;
    double *val = nullptr;               // FP64 values, canonical CSR order
    float *val32 = nullptr;              // FP32 copy (mixed precision)
    double *b = nullptr;                 // right-hand side
    double *dinv = nullptr;              // 2x2 block inverses, 4 x N (i00 i01 i10 i11)
    float *dinv32 = nullptr;
};

struct AsmParams {
    double re, invdtau, inv2dt, urot, ca, sa;
    int ff_bc;
};

// v2d_assemble.cu
int build_pattern(GridDev &g, const AsmParams &p, cudaStream_t s);  // rowptr/colind/nnz
int launch_metrics(GridDev &g, cudaStream_t s);
int launch_assemble(GridDev &g, const AsmParams &p, bool want32, int *d_flag, cudaStream_t s);

// v2d_forces.cu
int launch_forces(const GridDev &g, double re, double ref_length, double x0, double y0,
                  double *d_out10, cudaStream_t s);

// ------------------------------------------------------------- Krylov
// A CSR operator with optional FP32 copy and 2x2 block inverse.
// layout: 0 point (dinv holds 1/a_rr in slot 0), 1 field-blocked pairs (q, q+n/2),
//         2 interleaved pairs (2q, 2q+1).
struct CsrOp {
    int n = 0;
    long long nnz = 0;
    const int *rowptr = nullptr, *colind = nullptr;
    const double *val = nullptr;
    const float *val32 = nullptr;
    const double *dinv = nullptr;
    const float *dinv32 = nullptr;
    int layout = 1;
    int nblk = 0;  // number of 2x2 blocks (or n for point layout)
};

struct KrylovWork;  // defined in v2d_krylov.cu

int krylov_create(KrylovWork **out, int n, int restart, cudaStream_t s);
void krylov_destroy(KrylovWork *w);
// Solves A x = b (x is overwritten, starting from zero).  d_b, d_x device.
int krylov_solve(KrylovWork *w, const CsrOp &A, const double *d_b, double *d_x,
                 const v2d_krylov_params &prm, v2d_lin_stats *st, cudaStream_t s);

int time_spmv(const CsrOp &A, bool fp32, int reps, size_t flush_bytes, cudaStream_t s,
              double *ms_avg);

// 2x2 block inverse of a CSR operator (generic layouts).
int launch_block_inverse(CsrOp &A, double *dinv, float *dinv32, int *d_flag, cudaStream_t s);

}  // namespace v2d
