// Vector of the host layer's linear-algebra interface (reference: src/Math/SparseVector.h:8-43,
// a PETSc Vec).  One process owns every entry, so the values live in host memory and travel to
// the device once per SparseMatrix::solve / multiply.
#pragma once
#include <vector>

class SparseMatrix;

class SparseVector {
public:
    SparseVector() = default;
    explicit SparseVector(int m) { allocate(m); }

    void allocate(int m);
    void allocate(const SparseVector& other);
    void deallocate();
    void setValue(int i, double value);   // INSERT semantics; a negative index is ignored
    void zeroEntries();
    double operator()(int i);

    double l1Norm();
    double l2Norm();
    double infNorm();

    void print();

    int size() const { return (int)v_.size(); }
    const std::vector<double>& values() const { return v_; }
    std::vector<double>& values() { return v_; }

    friend class SparseMatrix;
    friend void scale(double alpha, SparseVector& vec);

private:
    std::vector<double> v_;
};

void scale(double alpha, SparseVector& vec);
