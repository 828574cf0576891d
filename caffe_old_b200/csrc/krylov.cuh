// Krylov solvers on the device: operators, workspace and launchers.
#pragma once
#include "common.cuh"

namespace cb {

// Immersed-boundary ghost rows in ELL-9 form, sorted by cell (IbPiso.cpp:119-190):
// col[9g + 0] is the ghost cell itself, col[9g + 1..8] the interpolation stencil (-1 for a
// dropped column), val[9g + m] the coefficients; bits marks ghost cells (one bit per cell).
struct GhostRows {
    int n;
    const int* cell;
    const int* col;
    const double* val;
    const uint32_t* bits;
};

// Non-symmetric 7-point operator: 7 per-cell coefficient arrays (momentum, Simple.cpp:162-171).
struct Op7 {
    const double* a[7];
    long long nI, nIJ;
    GhostRows gh;
};

// Symmetric 7-point operator: diagonal plus east/north/top coefficients per cell; the
// west/south/bottom coefficient of a cell is the east/north/top one of that neighbour
// (pressure correction, Simple.cpp:241-265).
struct OpSym {
    const double* aP;
    const double* aE;
    const double* aN;
    const double* aT;
    long long nI, nIJ;
    GhostRows gh;
};

// General sparse operator in compressed rows: the AIJ matrix SparseMatrix assembles row by row
// (src/Math/SparseMatrix.cpp:49-83).  diag[r] is the position of row r's diagonal entry in
// col / val, -1 when the row has none.
struct OpCSR {
    const int* ptr;
    const int* col;
    const double* val;
    const int* diag;
};

struct KspOut {
    int iters[3];
    double relres[3];
    int status[3];      // 0 converged, 1 maxit, 2 breakdown, 3 non-finite
    int cascades;       // learned solve only: 1 when its network stage handed over to the pyramid stage
    int net_iters;      // learned solve only: inner iterations run with the network in the preconditioner
};

// Workspace for up to NR = 3 right-hand sides; every array is a halo-padded cell array of
// 3 planes (the single right-hand-side CG also uses plane 1 of r as a second buffer).
struct KspWork {
    double* r;
    double* rp;
    double* p[2];
    double* v[2];
    double* t;
    double* invD;     // one plane
    double* partials; // grid x 8 doubles
    KspOut* out;      // device
    // single-precision workspace of the mixed-precision solver (halo-padded float cell arrays)
    float* fr[2];
    float* fw[2];
    float* fs[2];
    float* fp;
    float* fe;
    float* finvD;
    float* fA[4];     // aP aE aN aT in FP32
    float* fv[2];     // extra vectors of the FP32 BiCGStab inner solver
    float* ft;
};

// Every solve stops once ||b - A x|| <= max(rtol ||b||, atol) in the FP64 true residual (the
// convergence test of PETSc's KSP, rtol and atol; atol = 0 leaves the relative test alone).
int ksp_bicgstab(const Op7& A, int nr, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                 cudaStream_t st, double atol = 0.);
// project != 0: remove the mean of b first (b is modified), for singular all-Neumann systems
int ksp_bicgstab_sym(const OpSym& A, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                     cudaStream_t st, int project = 0, double atol = 0.);
int ksp_cg(const OpSym& A, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit, cudaStream_t st,
           int project = 0, double atol = 0.);
int ksp_cg7(const Op7& A, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit, cudaStream_t st,
            double atol = 0.);
// FP64 iterative refinement around FP32 inner solves on the symmetric p' operator: CG inner
// (method CAFFE_KSP_CG_JACOBI, symmetric systems) or BiCGStab inner (ghost rows).
// inner_rtol: relative reduction each inner solve aims for.  out->iters counts inner
// iterations; the outer count goes to *outer_iters (device int, may be null).
int ksp_mixed_sym(const OpSym& A, int method, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                  double inner_rtol, cudaStream_t st, int project, double atol = 0.);
// Plain FP64 re-solve that runs only when *status is non-zero (the fallback of a mixed or
// learned solve), decided on the device without a host round trip.
int ksp_fallback_sym(const OpSym& A, int method, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                     cudaStream_t st, int project, const int* status, int* fallbacks, double atol = 0.);
// Krylov solve of an n-row compressed-row system (vectors of n doubles, no halo): BiCGStab or CG
// with Jacobi preconditioning, the same persistent kernels as the lattice solves.
int ksp_csr(const OpCSR& A, int method, long long n, const double* b, double* x, const KspWork& w, double rtol, int maxit,
            cudaStream_t st, double atol = 0.);
// Blocks of the cooperative grid a solve launches: 0 BiCGStab on 3 right-hand sides (Op7),
// 1 BiCGStab (OpSym), 2 CG (OpSym), 3 BiCGStab (Op7), 4 CG (Op7), 5 BiCGStab (OpCSR), 6 CG (OpCSR).  The block partials of a
// solve take 2 x grid x 8 doubles.
int krylov_grid_size(int which);

}  // namespace cb
