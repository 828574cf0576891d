// Sparse matrix of the host layer's linear-algebra interface (reference: src/Math/SparseMatrix.h:
// 34-81 over PETSc's AIJ matrix and KSP).  Rows are assembled on the host with the reference's
// semantics -- setValue / setRow insert (a later value replaces an earlier one), negative row or
// column indices are ignored, zeroEntries keeps the structure -- and solve() hands the matrix over
// once in compressed rows to the device's Krylov solver (caffe_csr_solve), from a zero initial
// guess, returning the iteration count.
//
// The reference solves with PETSc's KSPBCGS + PCSOR (SparseMatrix.cpp:95-100).  A lexicographic
// SOR sweep is sequential, so the device solves with Jacobi-preconditioned BiCGStab by default
// (CG on request, setKspMethod), stopping at ||b - A x|| <= max(rtol ||b||, atol) on the true
// residual with PETSc's defaults (rtol 1e-5, atol 1e-50, 10000 iterations) unless given.  As with
// PETSc in the reference, a solve that stops at the iteration limit still returns its count;
// invalid input and device errors raise (Output::raiseException).
#pragma once
#include <map>
#include <string>
#include <vector>

#include "SparseVector.h"

// stands for PETSC_DEFAULT in the constructor's arguments
constexpr double CAFFE_SPARSE_DEFAULT = -2.;

class SparseMatrix {
public:
    enum ReuseMatrix { TRUE, FALSE };

    SparseMatrix(double rToler = CAFFE_SPARSE_DEFAULT, double absToler = CAFFE_SPARSE_DEFAULT,
                 int maxIters = (int)CAFFE_SPARSE_DEFAULT);
    SparseMatrix(int m, int n, int nnz);

    void allocate(int m, int n, int nnz);
    void deallocate();
    void setValue(int i, int j, double value);
    void setRow(int rowNo, int nCols, int colNos[], double values[]);
    void zeroEntries();

    int solve(const SparseVector& b, SparseVector& x);
    void assemble() {}

    int iLower() const { return 0; }
    int iUpper() const { return m_; }

    void print();
    void writeASCII(const std::string& filename);

    // extension: the device Krylov method (caffe_ksp: CAFFE_KSP_BICGSTAB_JACOBI or CAFFE_KSP_CG_JACOBI)
    void setKspMethod(int method) { method_ = method; }
    double lastRelativeResidual() const { return lastRelRes_; }
    // compressed rows of the current values (row_ptr, col, val)
    void compressedRows(std::vector<int>& ptr, std::vector<int>& col, std::vector<double>& val) const;

    int nRows() const { return m_; }
    int nCols() const { return n_; }

    friend void multiply(const SparseMatrix& A, const SparseMatrix& B, SparseMatrix& C);
    friend void multiply(const SparseMatrix& A, const SparseVector& x, SparseVector& b);
    friend void multiplyAdd(const SparseMatrix& A, const SparseVector& x1, const SparseVector& x2, SparseVector& b);
    friend void scale(double alpha, SparseMatrix& A);

private:
    int m_ = 0, n_ = 0;
    std::vector<std::map<int, double>> rows_;
    double rToler_, absToler_;
    int maxIters_;
    int method_;
    double lastRelRes_ = 0.;
};

void multiply(const SparseMatrix& A, const SparseMatrix& B, SparseMatrix& C);
void multiply(const SparseMatrix& A, const SparseVector& x, SparseVector& b);
void multiplyAdd(const SparseMatrix& A, const SparseVector& x1, const SparseVector& x2, SparseVector& b);
void scale(double alpha, SparseMatrix& A);
