// Check program for the host layer's SparseMatrix / SparseVector (the reference's linear-algebra
// interface, src/Math/SparseMatrix.h:34-81, SparseVector.h:8-43).  "semantics": host-side rules
// only (no device call); "solve": assembles a non-symmetric system row by row with setRow (dropping
// negative columns, overwriting re-inserted entries), solves it on the device and checks the true
// residual with multiply(); prints one line per check and exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "SparseMatrix.h"
#include "caffe_b200.h"

static int fail(const char* what) {
    std::printf("FAIL %s\n", what);
    return 1;
}

static int semantics() {
    SparseMatrix A(3, 3, 3);
    int cols[3] = {0, -1, 2};
    double vals[3] = {4., 99., 1.};
    A.setRow(0, 3, cols, vals);          // column -1 is ignored
    A.setValue(0, 2, 2.);                // INSERT: replaces the 1
    A.setValue(-1, 0, 5.);               // negative row ignored
    A.setValue(1, 1, 3.);
    A.setValue(2, 2, 5.);
    std::vector<int> ptr, col;
    std::vector<double> val;
    A.compressedRows(ptr, col, val);
    if (!(ptr == std::vector<int>{0, 2, 3, 4})) return fail("row structure");
    if (!(col == std::vector<int>{0, 2, 1, 2})) return fail("columns");
    if (!(val == std::vector<double>{4., 2., 3., 5.})) return fail("insert semantics");
    A.zeroEntries();                     // values zeroed, structure kept
    A.compressedRows(ptr, col, val);
    if (col.size() != 4 || val != std::vector<double>(4, 0.)) return fail("zeroEntries");
    SparseVector v(4);
    v.setValue(0, -3.); v.setValue(3, 4.); v.setValue(-2, 7.);
    if (v.l1Norm() != 7. || v.l2Norm() != 5. || v.infNorm() != 4.) return fail("norms");
    scale(2., v);
    if (v(3) != 8.) return fail("vector scale");
    SparseMatrix B(2, 2, 2), C;
    B.setValue(0, 0, 1.); B.setValue(0, 1, 2.); B.setValue(1, 1, 3.);
    multiply(B, B, C);                   // [[1, 8], [0, 9]]
    C.compressedRows(ptr, col, val);
    if (!(val == std::vector<double>{1., 8., 9.})) return fail("matrix product");
    if (B.iLower() != 0 || B.iUpper() != 2) return fail("ownership range");
    std::printf("OK semantics\n");
    return 0;
}

// convection-diffusion rows on an n x n grid (upwind, so the matrix is not symmetric), assembled
// the way the reference's solvers do: 5 columns per row, out-of-grid neighbours as column -1
static int solve(int n) {
    const int N = n * n;
    SparseMatrix A(1e-10, 0., 20000);
    A.allocate(N, N, 5);
    SparseVector b(N), x;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            int r = j * n + i;
            int cols[5] = {r, i + 1 < n ? r + 1 : -1, i > 0 ? r - 1 : -1, j + 1 < n ? r + n : -1, j > 0 ? r - n : -1};
            double vals[5] = {4.6, -0.7, -1.3, -0.9, -1.1};
            A.setRow(r, 5, cols, vals);
            b.setValue(r, std::sin(0.37 * r) + 0.5);
        }
    int iters = A.solve(b, x);
    SparseVector Ax, r(N);
    multiply(A, x, Ax);
    for (int q = 0; q < N; ++q) r.setValue(q, b(q) - Ax(q));
    double rel = r.l2Norm() / b.l2Norm();
    std::printf("solve iterations %d rel_res %.3e reported %.3e\n", iters, rel, A.lastRelativeResidual());
    if (!(iters > 0) || !(rel <= 1e-9)) return fail("bicgstab solve");
    // multiplyAdd: A x + b
    SparseVector y;
    multiplyAdd(A, x, b, y);
    for (int q = 0; q < N; ++q)
        if (std::fabs(y(q) - (Ax(q) + b(q))) > 1e-12 * (1. + std::fabs(y(q)))) return fail("multiplyAdd");
    // a symmetric positive definite system with CG
    SparseMatrix S(1e-10, 0., 20000);
    S.allocate(N, N, 5);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            int rr = j * n + i;
            int cols[5] = {rr, i + 1 < n ? rr + 1 : -1, i > 0 ? rr - 1 : -1, j + 1 < n ? rr + n : -1, j > 0 ? rr - n : -1};
            double vals[5] = {4.2, -1., -1., -1., -1.};
            S.setRow(rr, 5, cols, vals);
        }
    S.setKspMethod(CAFFE_KSP_CG_JACOBI);
    iters = S.solve(b, x);
    multiply(S, x, Ax);
    for (int q = 0; q < N; ++q) r.setValue(q, b(q) - Ax(q));
    rel = r.l2Norm() / b.l2Norm();
    std::printf("cg iterations %d rel_res %.3e\n", iters, rel);
    if (!(rel <= 1e-9)) return fail("cg solve");
    std::printf("OK solve\n");
    return 0;
}

int main(int argc, char** argv) {
    try {
        if (argc > 1 && std::strcmp(argv[1], "solve") == 0) return solve(argc > 2 ? std::atoi(argv[2]) : 40);
        return semantics();
    } catch (const char* msg) {
        std::printf("EXCEPTION %s\n", msg);
        return 2;
    }
}
