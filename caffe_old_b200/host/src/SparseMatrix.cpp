// SparseMatrix / SparseVector of the host layer over the device library's compressed-row entry
// points (caffe_csr_solve, caffe_csr_matvec).  Reference: src/Math/SparseMatrix.cpp,
// src/Math/SparseVector.cpp.
#include "SparseMatrix.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>

#include "Output.h"
#include "caffe_b200.h"

// ---------------------------------------------------------------- SparseVector
void SparseVector::allocate(int m) { v_.assign(m > 0 ? m : 0, 0.); }
void SparseVector::allocate(const SparseVector& other) { v_.assign(other.v_.size(), 0.); }
void SparseVector::deallocate() { v_.clear(); v_.shrink_to_fit(); }
void SparseVector::setValue(int i, double value) {
    if (i < 0) return;
    if (i >= (int)v_.size()) Output::raiseException("SparseVector", "setValue", "index " + std::to_string(i) + " out of range");
    v_[i] = value;
}
void SparseVector::zeroEntries() { std::fill(v_.begin(), v_.end(), 0.); }
double SparseVector::operator()(int i) {
    if (i < 0 || i >= (int)v_.size()) Output::raiseException("SparseVector", "operator()", "index " + std::to_string(i) + " out of range");
    return v_[i];
}
double SparseVector::l1Norm() {
    double s = 0.;
    for (double v : v_) s += std::fabs(v);
    return s;
}
double SparseVector::l2Norm() {
    double s = 0.;
    for (double v : v_) s += v * v;
    return std::sqrt(s);
}
double SparseVector::infNorm() {
    double s = 0.;
    for (double v : v_) s = std::max(s, std::fabs(v));
    return s;
}
void SparseVector::print() {
    for (size_t i = 0; i < v_.size(); ++i) std::printf("%zu %.17g\n", i, v_[i]);
}
void scale(double alpha, SparseVector& vec) {
    for (double& v : vec.v_) v *= alpha;
}

// ---------------------------------------------------------------- SparseMatrix
SparseMatrix::SparseMatrix(double rToler, double absToler, int maxIters)
    : rToler_(rToler == CAFFE_SPARSE_DEFAULT ? 1e-5 : rToler),
      absToler_(absToler == CAFFE_SPARSE_DEFAULT ? 1e-50 : absToler),
      maxIters_(maxIters == (int)CAFFE_SPARSE_DEFAULT ? 10000 : maxIters),
      method_(CAFFE_KSP_BICGSTAB_JACOBI) {}

SparseMatrix::SparseMatrix(int m, int n, int nnz) : SparseMatrix() { allocate(m, n, nnz); }

void SparseMatrix::allocate(int m, int n, int /*nnz: a per-row hint*/) {
    if (m < 0 || n < 0) Output::raiseException("SparseMatrix", "allocate", "negative size");
    m_ = m;
    n_ = n;
    rows_.assign(m, {});
}

void SparseMatrix::deallocate() {
    rows_.clear();
    rows_.shrink_to_fit();
    m_ = n_ = 0;
}

void SparseMatrix::setValue(int i, int j, double value) {
    if (i < 0 || j < 0) return;   // PETSc ignores negative indices
    if (i >= m_ || j >= n_)
        Output::raiseException("SparseMatrix", "setValue", "entry (" + std::to_string(i) + ", " + std::to_string(j) + ") out of range");
    rows_[i][j] = value;
}

void SparseMatrix::setRow(int rowNo, int nCols, int colNos[], double values[]) {
    for (int q = 0; q < nCols; ++q) setValue(rowNo, colNos[q], values[q]);
}

void SparseMatrix::zeroEntries() {
    for (auto& r : rows_)
        for (auto& e : r) e.second = 0.;
}

void SparseMatrix::compressedRows(std::vector<int>& ptr, std::vector<int>& col, std::vector<double>& val) const {
    ptr.assign(m_ + 1, 0);
    col.clear();
    val.clear();
    for (int r = 0; r < m_; ++r) {
        for (const auto& e : rows_[r]) {
            col.push_back(e.first);
            val.push_back(e.second);
        }
        ptr[r + 1] = (int)col.size();
    }
}

int SparseMatrix::solve(const SparseVector& b, SparseVector& x) {
    if (m_ != n_) Output::raiseException("SparseMatrix", "solve", "the matrix is not square");
    if (b.size() != m_) Output::raiseException("SparseMatrix", "solve", "right-hand side of the wrong size");
    if (m_ == 0) return 0;
    std::vector<int> ptr, col;
    std::vector<double> val;
    compressedRows(ptr, col, val);
    x.allocate(m_);
    int iters = 0;
    double rr = 0.;
    int rc = caffe_csr_solve(m_, ptr.data(), col.data(), val.data(), b.values().data(), x.values().data(), method_, rToler_, absToler_,
                             maxIters_, &iters, &rr);
    if (rc == 1) Output::raiseException("SparseMatrix", "solve", std::string("device solve failed: ") + caffe_last_error());
    lastRelRes_ = rr;
    return iters;
}

void SparseMatrix::print() {
    for (int r = 0; r < m_; ++r) {
        std::printf("row %d:", r);
        for (const auto& e : rows_[r]) std::printf(" (%d, %.17g)", e.first, e.second);
        std::printf("\n");
    }
}

void SparseMatrix::writeASCII(const std::string& filename) {
    std::ofstream f(filename);
    if (!f) Output::raiseException("SparseMatrix", "writeASCII", "cannot open \"" + filename + "\"");
    f.precision(17);
    for (int r = 0; r < m_; ++r) {
        f << "row " << r << ":";
        for (const auto& e : rows_[r]) f << " (" << e.first << ", " << e.second << ")";
        f << "\n";
    }
}

void multiply(const SparseMatrix& A, const SparseMatrix& B, SparseMatrix& C) {
    if (A.n_ != B.m_) Output::raiseException("SparseMatrix", "multiply", "inner dimensions differ");
    C.allocate(A.m_, B.n_, 0);
    for (int r = 0; r < A.m_; ++r)
        for (const auto& a : A.rows_[r])
            for (const auto& b : B.rows_[a.first]) C.rows_[r][b.first] += a.second * b.second;
}

void multiply(const SparseMatrix& A, const SparseVector& x, SparseVector& b) {
    if (x.size() != A.n_) Output::raiseException("SparseMatrix", "multiply", "vector of the wrong size");
    std::vector<int> ptr, col;
    std::vector<double> val;
    A.compressedRows(ptr, col, val);
    b.allocate(A.m_);
    if (A.m_ == 0) return;
    if (caffe_csr_matvec(A.m_, A.n_, ptr.data(), col.data(), val.data(), x.values().data(), b.values().data()) != 0)
        Output::raiseException("SparseMatrix", "multiply", std::string("device product failed: ") + caffe_last_error());
}

void multiplyAdd(const SparseMatrix& A, const SparseVector& x1, const SparseVector& x2, SparseVector& b) {
    if (x2.size() != A.m_) Output::raiseException("SparseMatrix", "multiplyAdd", "vector of the wrong size");
    SparseVector y;
    multiply(A, x1, y);
    b.allocate(A.m_);
    for (int i = 0; i < A.m_; ++i) b.values()[i] = y.values()[i] + x2.values()[i];
}

void scale(double alpha, SparseMatrix& A) {
    for (auto& r : A.rows_)
        for (auto& e : r) e.second *= alpha;
}
