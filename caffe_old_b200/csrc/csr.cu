// General sparse systems through the C ABI: the matrix a caller assembles row by row, as the
// reference's SparseMatrix does over PETSc's AIJ format (src/Math/SparseMatrix.cpp:49-106), handed
// over once in compressed rows and solved by the persistent Jacobi-preconditioned Krylov kernels
// (krylov.cu) on the device.  Used by the host layer's SparseMatrix / SparseVector classes.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/caffe_b200.h"
#include "common.cuh"
#include "krylov.cuh"

namespace cb {
namespace {

// position of each row's diagonal entry (-1 when the row has none)
__global__ void csr_diag_kernel(long long n, const int* ptr, const int* col, int* diag) {
    long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= n) return;
    int d = -1;
    for (int p = ptr[r]; p < ptr[r + 1]; ++p)
        if (col[p] == r) { d = p; break; }
    diag[r] = d;
}

// y = A x, one row per thread
__global__ void csr_matvec_kernel(long long m, const int* ptr, const int* col, const double* val, const double* x, double* y) {
    long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= m) return;
    double s = 0.;
    for (int p = ptr[r]; p < ptr[r + 1]; ++p) s += val[p] * x[col[p]];
    y[r] = s;
}

// row pointers start at 0 and never decrease; every column lies in [0, ncols)
bool check_csr(int m, int ncols, const int* ptr, const int* col) {
    if (ptr[0] != 0) { set_error("row_ptr[0] must be 0"); return false; }
    for (int r = 0; r < m; ++r)
        if (ptr[r + 1] < ptr[r]) { set_error("row_ptr must not decrease (row " + std::to_string(r) + ")"); return false; }
    for (int p = 0; p < ptr[m]; ++p)
        if (col[p] < 0 || col[p] >= ncols) {
            set_error("column index " + std::to_string(col[p]) + " out of range at entry " + std::to_string(p));
            return false;
        }
    return true;
}

struct DevBufs {
    std::vector<void*> v;
    template <class T>
    T* get(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, count * sizeof(T) + 16) != cudaSuccess) return nullptr;
        v.push_back(p);
        return static_cast<T*>(p);
    }
    ~DevBufs() {
        cudaDeviceSynchronize();
        for (void* p : v) cudaFree(p);
    }
};

}  // namespace
}  // namespace cb

using namespace cb;

extern "C" int caffe_csr_solve(int n, const int* row_ptr, const int* col, const double* val, const double* b, double* x,
                               int method, double rtol, double atol, int maxit, int* iters, double* rel_res) {
    clear_error();
    if (n < 1 || !row_ptr || !b || !x || ((!col || !val) && row_ptr[n] > 0)) { set_error("invalid arguments"); return 1; }
    if (maxit < 1) { set_error("maxit must be >= 1"); return 1; }
    if (!(rtol >= 0.) || !(atol >= 0.)) { set_error("tolerances must be >= 0"); return 1; }
    if (method == CAFFE_KSP_BICGSTAB_SGS) {
        set_error("BiCGStab with symmetric Gauss-Seidel (the reference's PETSc PCSOR) is a sequential sweep and is not "
                  "implemented on the device: choose CAFFE_KSP_BICGSTAB_JACOBI or CAFFE_KSP_CG_JACOBI");
        return 1;
    }
    if (method != CAFFE_KSP_BICGSTAB_JACOBI && method != CAFFE_KSP_CG_JACOBI) { set_error("invalid Krylov method"); return 1; }
    if (!check_csr(n, n, row_ptr, col)) return 1;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { set_error("no CUDA device available"); return 1; }
    const long long nnz = row_ptr[n];
    DevBufs d;
    int* dptr = d.get<int>(n + 1);
    int* dcol = d.get<int>(nnz > 0 ? nnz : 1);
    double* dval = d.get<double>(nnz > 0 ? nnz : 1);
    int* ddiag = d.get<int>(n);
    double* db = d.get<double>(n);
    double* dx = d.get<double>(n);
    KspWork w;
    std::memset(&w, 0, sizeof(w));
    w.r = d.get<double>(2 * (size_t)n);   // the CG keeps its second r buffer one vector on
    w.rp = d.get<double>(n);
    w.p[0] = d.get<double>(n); w.p[1] = d.get<double>(n);
    w.v[0] = d.get<double>(n); w.v[1] = d.get<double>(n);
    w.t = d.get<double>(n);
    w.invD = d.get<double>(n);
    w.partials = d.get<double>((size_t)2 * 8 * 8 * 1024);
    w.out = d.get<KspOut>(1);
    bool ok = dptr && dcol && dval && ddiag && db && dx && w.r && w.rp && w.p[0] && w.p[1] && w.v[0] && w.v[1] && w.t && w.invD &&
              w.partials && w.out;
    if (!ok) { set_error("device allocation failed"); return 1; }
    cudaStream_t st = nullptr;
    CB_CUDA(cudaMemcpy(dptr, row_ptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    if (nnz > 0) {
        CB_CUDA(cudaMemcpy(dcol, col, sizeof(int) * nnz, cudaMemcpyHostToDevice));
        CB_CUDA(cudaMemcpy(dval, val, sizeof(double) * nnz, cudaMemcpyHostToDevice));
    }
    CB_CUDA(cudaMemcpy(db, b, sizeof(double) * n, cudaMemcpyHostToDevice));
    csr_diag_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, dptr, dcol, ddiag);
    CB_CHECK_LAUNCH();
    OpCSR A;
    A.ptr = dptr; A.col = dcol; A.val = dval; A.diag = ddiag;
    if (ksp_csr(A, method, n, db, dx, w, rtol, maxit, st, atol)) return 1;
    KspOut o;
    CB_CUDA(cudaMemcpy(&o, w.out, sizeof(KspOut), cudaMemcpyDeviceToHost));
    CB_CUDA(cudaMemcpy(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (iters) *iters = o.iters[0];
    if (rel_res) *rel_res = o.relres[0];
    switch (o.status[0]) {
        case 0: return 0;
        case 1: set_error("the solve reached maxit before the tolerance"); return 2;
        case 2: set_error("Krylov breakdown"); return 3;
        default: set_error("non-finite residual"); return 4;
    }
}

extern "C" int caffe_csr_matvec(int m, int n, const int* row_ptr, const int* col, const double* val, const double* x, double* y) {
    clear_error();
    if (m < 1 || n < 1 || !row_ptr || !x || !y || ((!col || !val) && row_ptr[m] > 0)) { set_error("invalid arguments"); return 1; }
    if (!check_csr(m, n, row_ptr, col)) return 1;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { set_error("no CUDA device available"); return 1; }
    const long long nnz = row_ptr[m];
    DevBufs d;
    int* dptr = d.get<int>(m + 1);
    int* dcol = d.get<int>(nnz > 0 ? nnz : 1);
    double* dval = d.get<double>(nnz > 0 ? nnz : 1);
    double* dx = d.get<double>(n);
    double* dy = d.get<double>(m);
    if (!dptr || !dcol || !dval || !dx || !dy) { set_error("device allocation failed"); return 1; }
    CB_CUDA(cudaMemcpy(dptr, row_ptr, sizeof(int) * (m + 1), cudaMemcpyHostToDevice));
    if (nnz > 0) {
        CB_CUDA(cudaMemcpy(dcol, col, sizeof(int) * nnz, cudaMemcpyHostToDevice));
        CB_CUDA(cudaMemcpy(dval, val, sizeof(double) * nnz, cudaMemcpyHostToDevice));
    }
    CB_CUDA(cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice));
    csr_matvec_kernel<<<grid_for(m, 256), 256>>>(m, dptr, dcol, dval, dx, dy);
    CB_CHECK_LAUNCH();
    CB_CUDA(cudaMemcpy(y, dy, sizeof(double) * m, cudaMemcpyDeviceToHost));
    return 0;
}
