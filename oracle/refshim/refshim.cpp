// Implementations behind the stand-in headers in refshim/include (test infrastructure only):
// the PETSc, MPI, LAPACKE and Boost calls of the reference's solver path, so that its own
// sources (src/Solvers, src/Domains, src/Schemes, src/Math, src/RunControl, src/Parallel)
// compile and run here unchanged and pin the CPU oracle.
//
// KSPSolve does not restate PETSc's KSPBCGS + PCSOR: it records the system (rows as assembled
// by MatSetValues, right-hand side) and solves it tightly with restarted GMRES (Saad & Schultz
// 1986; modified Gram-Schmidt, Givens rotations) right-preconditioned by ILU(0), stopping on
// the true residual ||b - A x|| <= rtol ||b|| (rtol set by the driver; the reference's
// tolerances only shape PETSc's own stopping point, which is not what is being pinned).  A
// matrix whose every row sums to zero (the all-Neumann pressure correction) has the constants
// as null space: its right-hand side is projected onto the range and the solution returned
// with zero mean, as any consistent solve of that system must be chosen.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <boost/property_tree/info_parser.hpp>
#include <lapacke/lapacke.h>
#include <mpi.h>
#include <petsc.h>

#include "refshim.h"

// ------------------------------------------------------------------ objects
struct RefshimMat {
    int m = 0, n = 0;
    std::vector<std::map<int, double>> rows;
};
struct RefshimVec {
    std::vector<double> v;
};
struct RefshimKsp {
    Mat A = nullptr;
    int iters = 0;
};
struct RefshimViewer {
    int unused = 0;
};

namespace {
std::set<void*> g_live;   // handles created here; destroy calls on others (never-allocated members) are ignored
template <class T>
T* make() {
    T* p = new T();
    g_live.insert(p);
    return p;
}
template <class T>
void destroy(T** p) {
    if (p && *p && g_live.erase(*p)) delete *p;
    if (p) *p = nullptr;
}
std::vector<std::vector<double>> g_inject;   // solutions KSPSolve returns, in order, instead of solving
size_t g_injectNext = 0;
double g_rtol = 1e-13;
int g_maxit = 200000;
bool g_record = false;
std::vector<refshim::System> g_systems;
}  // namespace

namespace refshim {
void set_solve_tolerance(double rtol, int maxit) { g_rtol = rtol; g_maxit = maxit; }
void set_recording(bool on) { g_record = on; }
void inject(const double* x, int n) { g_inject.emplace_back(x, x + n); }
void clear_injected() { g_inject.clear(); g_injectNext = 0; }
int injected_left() { return (int)(g_inject.size() - g_injectNext); }
std::vector<System>& systems() { return g_systems; }
}  // namespace refshim

PetscErrorCode PetscInitializeNoArguments(void) { return 0; }

PetscErrorCode MatCreate(PetscComm, Mat* A) { *A = make<RefshimMat>(); return 0; }
PetscErrorCode MatSetSizes(Mat A, PetscInt, PetscInt, PetscInt M, PetscInt N) {
    A->m = M; A->n = N; A->rows.assign(M > 0 ? M : 0, {});
    return 0;
}
PetscErrorCode MatSetType(Mat, MatType) { return 0; }
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt*, PetscInt, const PetscInt*) { return 0; }
PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt*) { return 0; }
PetscErrorCode MatSetUp(Mat) { return 0; }
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt* lo, PetscInt* hi) { *lo = 0; *hi = A->m; return 0; }
PetscErrorCode MatDestroy(Mat* A) { destroy(A); return 0; }
PetscErrorCode MatSetValues(Mat A, PetscInt nr, const PetscInt* rows, PetscInt nc, const PetscInt* cols, const PetscScalar* v,
                            InsertMode mode) {
    for (int a = 0; a < nr; ++a) {
        int r = rows[a];
        if (r < 0) continue;   // negative indices are ignored, as in PETSc
        if (r >= A->m) { std::fprintf(stderr, "refshim: row %d out of range\n", r); std::abort(); }
        for (int b = 0; b < nc; ++b) {
            int c = cols[b];
            if (c < 0) continue;
            if (c >= A->n) { std::fprintf(stderr, "refshim: column %d out of range\n", c); std::abort(); }
            double val = v[(size_t)a * nc + b];
            if (mode == ADD_VALUES) A->rows[r][c] += val; else A->rows[r][c] = val;
        }
    }
    return 0;
}
PetscErrorCode MatZeroEntries(Mat A) {
    for (auto& r : A->rows) for (auto& e : r) e.second = 0.;
    return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatView(Mat A, PetscViewer) {
    for (int r = 0; r < A->m; ++r) {
        std::printf("row %d:", r);
        for (auto& e : A->rows[r]) std::printf(" (%d, %.17g)", e.first, e.second);
        std::printf("\n");
    }
    return 0;
}
PetscErrorCode MatMatMult(Mat A, Mat B, MatReuse, PetscReal, Mat* C) {
    *C = make<RefshimMat>();
    (*C)->m = A->m; (*C)->n = B->n; (*C)->rows.assign(A->m, {});
    for (int r = 0; r < A->m; ++r)
        for (auto& e : A->rows[r])
            for (auto& f : B->rows[e.first]) (*C)->rows[r][f.first] += e.second * f.second;
    return 0;
}
PetscErrorCode MatMult(Mat A, Vec x, Vec y) {
    std::vector<double> out(A->m, 0.);
    for (int r = 0; r < A->m; ++r) for (auto& e : A->rows[r]) out[r] += e.second * x->v[e.first];
    y->v = out;
    return 0;
}
PetscErrorCode MatMultAdd(Mat A, Vec x, Vec y, Vec z) {
    std::vector<double> out(y->v);
    for (int r = 0; r < A->m; ++r) for (auto& e : A->rows[r]) out[r] += e.second * x->v[e.first];
    z->v = out;
    return 0;
}
PetscErrorCode MatScale(Mat A, PetscScalar a) {
    for (auto& r : A->rows) for (auto& e : r) e.second *= a;
    return 0;
}

PetscErrorCode KSPCreate(PetscComm, KSP* k) { *k = make<RefshimKsp>(); return 0; }
PetscErrorCode KSPDestroy(KSP* k) { destroy(k); return 0; }
PetscErrorCode KSPSetOperators(KSP k, Mat A, Mat) { k->A = A; return 0; }
PetscErrorCode KSPGetPC(KSP k, PC* pc) { *pc = k; return 0; }
PetscErrorCode PCSetType(PC, PCType) { return 0; }
PetscErrorCode PCSORSetIterations(PC, PetscInt, PetscInt) { return 0; }
PetscErrorCode KSPSetTolerances(KSP, PetscReal, PetscReal, PetscReal, PetscInt) { return 0; }
PetscErrorCode KSPSetType(KSP, KSPType) { return 0; }
PetscErrorCode KSPGetIterationNumber(KSP k, PetscInt* it) { *it = k->iters; return 0; }

PetscErrorCode PetscViewerASCIIOpen(PetscComm, const char*, PetscViewer* v) { *v = make<RefshimViewer>(); return 0; }
PetscErrorCode PetscViewerDestroy(PetscViewer* v) { destroy(v); return 0; }

PetscErrorCode VecCreate(PetscComm, Vec* x) { *x = make<RefshimVec>(); return 0; }
PetscErrorCode VecSetSizes(Vec x, PetscInt, PetscInt N) { x->v.assign(N > 0 ? N : 0, 0.); return 0; }
PetscErrorCode VecSetType(Vec, VecType) { return 0; }
PetscErrorCode VecGetOwnershipRange(Vec x, PetscInt* lo, PetscInt* hi) { *lo = 0; *hi = (int)x->v.size(); return 0; }
PetscErrorCode VecDuplicate(Vec x, Vec* y) { *y = make<RefshimVec>(); (*y)->v.assign(x->v.size(), 0.); return 0; }
PetscErrorCode VecDestroy(Vec* x) { destroy(x); return 0; }
PetscErrorCode VecSetValues(Vec x, PetscInt n, const PetscInt* ix, const PetscScalar* y, InsertMode mode) {
    for (int q = 0; q < n; ++q) {
        if (ix[q] < 0) continue;
        if (mode == ADD_VALUES) x->v[ix[q]] += y[q]; else x->v[ix[q]] = y[q];
    }
    return 0;
}
PetscErrorCode VecZeroEntries(Vec x) { std::fill(x->v.begin(), x->v.end(), 0.); return 0; }
PetscErrorCode VecGetValues(Vec x, PetscInt n, const PetscInt* ix, PetscScalar* y) {
    for (int q = 0; q < n; ++q) y[q] = x->v[ix[q]];
    return 0;
}
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal* out) {
    double s = 0.;
    for (double v : x->v) {
        if (t == NORM_1) s += std::fabs(v);
        else if (t == NORM_INFINITY) s = std::max(s, std::fabs(v));
        else s += v * v;
    }
    *out = (t == NORM_2 || t == NORM_FROBENIUS) ? std::sqrt(s) : s;
    return 0;
}
PetscErrorCode VecView(Vec x, PetscViewer) {
    for (size_t q = 0; q < x->v.size(); ++q) std::printf("%zu %.17g\n", q, x->v[q]);
    return 0;
}
PetscErrorCode VecScale(Vec x, PetscScalar a) { for (double& v : x->v) v *= a; return 0; }
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }

// ------------------------------------------------------------------ the tight solve
namespace {

struct Csr {
    int n = 0;
    std::vector<int> ptr, col, diag;
    std::vector<double> val;
};

Csr to_csr(const RefshimMat& A) {
    Csr C;
    C.n = A.m;
    C.ptr.assign(A.m + 1, 0);
    C.diag.assign(A.m, -1);
    for (int r = 0; r < A.m; ++r) {
        for (auto& e : A.rows[r]) {
            if (e.first == r) C.diag[r] = (int)C.col.size();
            C.col.push_back(e.first);
            C.val.push_back(e.second);
        }
        C.ptr[r + 1] = (int)C.col.size();
    }
    return C;
}

void spmv(const Csr& C, const std::vector<double>& x, std::vector<double>& y) {
    y.assign(C.n, 0.);
    for (int r = 0; r < C.n; ++r) {
        double s = 0.;
        for (int p = C.ptr[r]; p < C.ptr[r + 1]; ++p) s += C.val[p] * x[C.col[p]];
        y[r] = s;
    }
}

double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.;
    for (size_t q = 0; q < a.size(); ++q) s += a[q] * b[q];
    return s;
}

// ILU(0) on the matrix's own sparsity pattern (rows sorted by column); shift > 0 lifts the
// diagonal of the factor only (a singular matrix would otherwise leave a zero last pivot)
struct Ilu0 {
    Csr F;
    void build(const Csr& A, double shift) {
        F = A;
        for (int r = 0; r < F.n; ++r)
            if (F.diag[r] >= 0) F.val[F.diag[r]] *= 1. + shift;
        for (int i = 0; i < F.n; ++i) {
            for (int p = F.ptr[i]; p < F.ptr[i + 1] && F.col[p] < i; ++p) {
                int k = F.col[p];
                double dk = F.diag[k] >= 0 ? F.val[F.diag[k]] : 0.;
                if (dk == 0.) continue;
                F.val[p] /= dk;
                double lik = F.val[p];
                int q = p + 1, s = F.diag[k] + 1;
                while (q < F.ptr[i + 1] && s < F.ptr[k + 1]) {
                    if (F.col[q] == F.col[s]) { F.val[q] -= lik * F.val[s]; ++q; ++s; }
                    else if (F.col[q] < F.col[s]) ++q;
                    else ++s;
                }
            }
        }
    }
    void apply(const std::vector<double>& r, std::vector<double>& z) const {
        z = r;
        for (int i = 0; i < F.n; ++i)
            for (int p = F.ptr[i]; p < F.ptr[i + 1] && F.col[p] < i; ++p) z[i] -= F.val[p] * z[F.col[p]];
        for (int i = F.n - 1; i >= 0; --i) {
            double s = z[i];
            int p = F.diag[i] >= 0 ? F.diag[i] + 1 : F.ptr[i + 1];
            for (; p < F.ptr[i + 1]; ++p) s -= F.val[p] * z[F.col[p]];
            double d = F.diag[i] >= 0 ? F.val[F.diag[i]] : 1.;
            z[i] = d != 0. ? s / d : s;
        }
    }
};

int gmres_solve(const Csr& A, const std::vector<double>& b, std::vector<double>& x, double rtol, int maxit, bool singular) {
    const int n = A.n, m = 60;
    Ilu0 M;
    M.build(A, singular ? 1e-10 : 0.);
    x.assign(n, 0.);
    double bn = std::sqrt(dot(b, b));
    if (bn == 0.) return 0;
    std::vector<std::vector<double>> V(m + 1, std::vector<double>(n)), Z(m, std::vector<double>(n));
    std::vector<double> r(n), w(n), H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    int it = 0;
    while (it < maxit) {
        spmv(A, x, r);
        for (int q = 0; q < n; ++q) r[q] = b[q] - r[q];
        double beta = std::sqrt(dot(r, r));
        if (beta <= rtol * bn) break;
        for (int q = 0; q < n; ++q) V[0][q] = r[q] / beta;
        std::fill(g.begin(), g.end(), 0.);
        g[0] = beta;
        int j = 0;
        for (; j < m && it < maxit; ++j, ++it) {
            M.apply(V[j], Z[j]);
            spmv(A, Z[j], w);
            for (int i = 0; i <= j; ++i) {
                double h = dot(w, V[i]);
                H[(size_t)j * (m + 1) + i] = h;
                for (int q = 0; q < n; ++q) w[q] -= h * V[i][q];
            }
            double hn = std::sqrt(dot(w, w));
            H[(size_t)j * (m + 1) + j + 1] = hn;
            if (hn > 0.) for (int q = 0; q < n; ++q) V[j + 1][q] = w[q] / hn;
            for (int i = 0; i < j; ++i) {
                double a = H[(size_t)j * (m + 1) + i], c = H[(size_t)j * (m + 1) + i + 1];
                H[(size_t)j * (m + 1) + i] = cs[i] * a + sn[i] * c;
                H[(size_t)j * (m + 1) + i + 1] = -sn[i] * a + cs[i] * c;
            }
            double a = H[(size_t)j * (m + 1) + j], c = H[(size_t)j * (m + 1) + j + 1];
            double rr = std::sqrt(a * a + c * c);
            cs[j] = rr > 0. ? a / rr : 1.;
            sn[j] = rr > 0. ? c / rr : 0.;
            H[(size_t)j * (m + 1) + j] = rr;
            H[(size_t)j * (m + 1) + j + 1] = 0.;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            if (std::fabs(g[j + 1]) <= 0.1 * rtol * bn || !(hn > 0.)) { ++j; ++it; break; }
        }
        for (int i = j - 1; i >= 0; --i) {
            double s = g[i];
            for (int k = i + 1; k < j; ++k) s -= H[(size_t)k * (m + 1) + i] * y[k];
            double d = H[(size_t)i * (m + 1) + i];
            y[i] = d != 0. ? s / d : 0.;
        }
        for (int i = 0; i < j; ++i) for (int q = 0; q < n; ++q) x[q] += y[i] * Z[i][q];
    }
    return it;
}

}  // namespace

PetscErrorCode KSPSolve(KSP k, Vec b, Vec x) {
    Csr A = to_csr(*k->A);
    std::vector<double> rhs(b->v);
    // all rows summing to zero: the constants span the null space
    bool singular = A.n > 0;
    for (int r = 0; r < A.n && singular; ++r) {
        double s = 0., a = 0.;
        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) { s += A.val[p]; a += std::fabs(A.val[p]); }
        if (std::fabs(s) > 1e-12 * a) singular = false;
    }
    if (singular) {
        double mean = 0.;
        for (double v : rhs) mean += v;
        mean /= (double)rhs.size();
        for (double& v : rhs) v -= mean;
    }
    std::vector<double> sol;
    if (g_injectNext < g_inject.size()) {
        // a solution handed in by the driver (the oracle's): the reference's code continues from
        // exactly the numbers the oracle continues from, so everything outside the Krylov solves
        // can be compared bit for bit
        sol = g_inject[g_injectNext++];
        if ((int)sol.size() != A.n) { std::fprintf(stderr, "refshim: injected solution of the wrong size\n"); std::abort(); }
        x->v = sol;
        k->iters = 0;
        if (g_record) {
            refshim::System s;
            s.n = A.n; s.ptr = A.ptr; s.col = A.col; s.val = A.val; s.b = b->v; s.x = sol;
            g_systems.push_back(std::move(s));
        }
        return 0;
    }
    k->iters = gmres_solve(A, rhs, sol, g_rtol, g_maxit, singular);
    if (singular) {
        double mean = 0.;
        for (double v : sol) mean += v;
        mean /= (double)sol.size();
        for (double& v : sol) v -= mean;
    }
    x->v = sol;
    if (g_record) {
        refshim::System s;
        s.n = A.n;
        s.ptr = A.ptr; s.col = A.col; s.val = A.val;
        s.b = b->v;
        s.x = sol;
        g_systems.push_back(std::move(s));
    }
    return 0;
}

// ------------------------------------------------------------------ MPI, one process
namespace MPI {
const Datatype INT{(int)sizeof(int)}, DOUBLE{(int)sizeof(double)}, CHAR{1};
const Op SUM{0}, MIN{1}, MAX{2};
Intracomm COMM_WORLD;
void Init() {}
void Finalize() {}
void Intracomm::Allreduce(const void* in, void* out, int count, const Datatype& t, const Op&) const {
    std::memmove(out, in, (size_t)count * t.bytes);
}
void Intracomm::Allgather(const void* in, int count, const Datatype& t, void* out, int, const Datatype&) const {
    std::memmove(out, in, (size_t)count * t.bytes);
}
[[noreturn]] static void no_peer() {
    std::fprintf(stderr, "refshim: point-to-point message with a single process\n");
    std::abort();
}
void Intracomm::Send(const void*, int, const Datatype&, int, int) const { no_peer(); }
void Intracomm::Recv(void*, int, const Datatype&, int, int) const { no_peer(); }
Request Intracomm::Isend(const void*, int, const Datatype&, int, int) const { no_peer(); }
Request Intracomm::Irecv(void*, int, const Datatype&, int, int) const { no_peer(); }
}  // namespace MPI

// ------------------------------------------------------------------ LAPACKE (row major)
lapack_int LAPACKE_dgetrf(int, lapack_int m, lapack_int n, double* a, lapack_int lda, lapack_int* ipiv) {
    int info = 0;
    for (int k = 0; k < std::min(m, n); ++k) {
        int p = k;
        for (int i = k + 1; i < m; ++i) if (std::fabs(a[(size_t)i * lda + k]) > std::fabs(a[(size_t)p * lda + k])) p = i;
        ipiv[k] = p + 1;
        if (p != k) for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * lda + j], a[(size_t)p * lda + j]);
        double d = a[(size_t)k * lda + k];
        if (d == 0.) { if (!info) info = k + 1; continue; }
        for (int i = k + 1; i < m; ++i) {
            double l = a[(size_t)i * lda + k] / d;
            a[(size_t)i * lda + k] = l;
            for (int j = k + 1; j < n; ++j) a[(size_t)i * lda + j] -= l * a[(size_t)k * lda + j];
        }
    }
    return info;
}
lapack_int LAPACKE_dgetri(int, lapack_int n, double* a, lapack_int lda, const lapack_int* ipiv) {
    // columns of the inverse: solve L U X = P I, then X overwrites a
    std::vector<double> inv((size_t)n * n, 0.), e(n);
    for (int c = 0; c < n; ++c) {
        std::fill(e.begin(), e.end(), 0.);
        e[c] = 1.;
        for (int k = 0; k < n; ++k) std::swap(e[k], e[ipiv[k] - 1]);
        for (int i = 0; i < n; ++i) for (int j = 0; j < i; ++j) e[i] -= a[(size_t)i * lda + j] * e[j];
        for (int i = n - 1; i >= 0; --i) {
            for (int j = i + 1; j < n; ++j) e[i] -= a[(size_t)i * lda + j] * e[j];
            e[i] /= a[(size_t)i * lda + i];
        }
        for (int i = 0; i < n; ++i) inv[(size_t)i * n + c] = e[i];
    }
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) a[(size_t)i * lda + j] = inv[(size_t)i * n + j];
    return 0;
}
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double* a, lapack_int lda, lapack_int* ipiv, double* b,
                         lapack_int ldb) {
    int info = LAPACKE_dgetrf(layout, n, n, a, lda, ipiv);
    for (int c = 0; c < nrhs; ++c) {
        for (int k = 0; k < n; ++k) std::swap(b[(size_t)k * ldb + c], b[(size_t)(ipiv[k] - 1) * ldb + c]);
        for (int i = 0; i < n; ++i) for (int j = 0; j < i; ++j) b[(size_t)i * ldb + c] -= a[(size_t)i * lda + j] * b[(size_t)j * ldb + c];
        for (int i = n - 1; i >= 0; --i) {
            for (int j = i + 1; j < n; ++j) b[(size_t)i * ldb + c] -= a[(size_t)i * lda + j] * b[(size_t)j * ldb + c];
            b[(size_t)i * ldb + c] /= a[(size_t)i * lda + i];
        }
    }
    return info;
}
lapack_int LAPACKE_dgels(int, char, lapack_int m, lapack_int n, lapack_int nrhs, double* a, lapack_int lda, double* b, lapack_int ldb) {
    // Householder QR of the m x n matrix (m >= n), then R x = Q^T b in the first n rows of b
    for (int k = 0; k < n && k < m; ++k) {
        double nrm = 0.;
        for (int i = k; i < m; ++i) nrm += a[(size_t)i * lda + k] * a[(size_t)i * lda + k];
        nrm = std::sqrt(nrm);
        if (nrm == 0.) continue;
        double alpha = a[(size_t)k * lda + k] > 0. ? -nrm : nrm;
        std::vector<double> v(m - k);
        for (int i = k; i < m; ++i) v[i - k] = a[(size_t)i * lda + k];
        v[0] -= alpha;
        double vv = 0.;
        for (double t : v) vv += t * t;
        if (vv == 0.) continue;
        for (int j = k; j < n; ++j) {
            double s = 0.;
            for (int i = k; i < m; ++i) s += v[i - k] * a[(size_t)i * lda + j];
            s = 2. * s / vv;
            for (int i = k; i < m; ++i) a[(size_t)i * lda + j] -= s * v[i - k];
        }
        for (int c = 0; c < nrhs; ++c) {
            double s = 0.;
            for (int i = k; i < m; ++i) s += v[i - k] * b[(size_t)i * ldb + c];
            s = 2. * s / vv;
            for (int i = k; i < m; ++i) b[(size_t)i * ldb + c] -= s * v[i - k];
        }
    }
    for (int c = 0; c < nrhs; ++c)
        for (int i = n - 1; i >= 0; --i) {
            double s = b[(size_t)i * ldb + c];
            for (int j = i + 1; j < n; ++j) s -= a[(size_t)i * lda + j] * b[(size_t)j * ldb + c];
            b[(size_t)i * ldb + c] = s / a[(size_t)i * lda + i];
        }
    return 0;
}

// ------------------------------------------------------------------ BLAS dgemm (column major)
// C := alpha op(A) op(B) + beta C with the loop order of the reference BLAS (netlib): for every
// entry of C a dot product over K, accumulated in order.  Matrix.cpp:259-268 calls it.
extern "C" void dgemm_(char* ta, char* tb, int* M, int* N, int* K, double* alpha, double* A, int* lda, double* B, int* ldb,
                       double* beta, double* C, int* ldc) {
    const bool tA = *ta == 'T' || *ta == 't' || *ta == 'C' || *ta == 'c';
    const bool tB = *tb == 'T' || *tb == 't' || *tb == 'C' || *tb == 'c';
    for (int j = 0; j < *N; ++j)
        for (int i = 0; i < *M; ++i) {
            double t = 0.;
            for (int l = 0; l < *K; ++l) {
                double a = tA ? A[(size_t)i * *lda + l] : A[(size_t)l * *lda + i];
                double b = tB ? B[(size_t)l * *ldb + j] : B[(size_t)j * *ldb + l];
                t += a * b;
            }
            double& c = C[(size_t)j * *ldc + i];
            c = *beta == 0. ? *alpha * t : *alpha * t + *beta * c;
        }
}

// ------------------------------------------------------------------ INFO files
namespace boost {
namespace property_tree {
namespace info_parser {

static std::vector<std::string> tokens(const std::string& line) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < line.size()) {
        char c = line[i];
        if (c == ';') break;
        if (std::isspace((unsigned char)c)) { ++i; continue; }
        if (c == '{' || c == '}') { out.emplace_back(1, c); ++i; continue; }
        std::string t;
        if (c == '"') {
            ++i;
            while (i < line.size() && line[i] != '"') t.push_back(line[i++]);
            ++i;
        } else {
            while (i < line.size() && !std::isspace((unsigned char)line[i]) && line[i] != '{' && line[i] != '}' && line[i] != ';')
                t.push_back(line[i++]);
        }
        out.push_back(t);
    }
    return out;
}

void read_info(const std::string& filename, ptree& pt) {
    std::ifstream f(filename);
    if (!f) throw std::runtime_error("cannot open file " + filename);
    std::vector<ptree*> stack{&pt};
    ptree* last = nullptr;
    std::string line;
    while (std::getline(f, line)) {
        std::vector<std::string> t = tokens(line);
        size_t q = 0;
        while (q < t.size()) {
            if (t[q] == "{") {
                if (!last) throw std::runtime_error("unexpected '{' in " + filename);
                stack.push_back(last);
                last = nullptr;
                ++q;
            } else if (t[q] == "}") {
                if (stack.size() < 2) throw std::runtime_error("unbalanced '}' in " + filename);
                stack.pop_back();
                last = nullptr;
                ++q;
            } else {
                ptree* parent = stack.back();
                parent->children.emplace_back(t[q], ptree());
                last = &parent->children.back().second;
                ++q;
                if (q < t.size() && t[q] != "{" && t[q] != "}") { last->data = t[q]; ++q; }
                while (q < t.size() && t[q] != "{" && t[q] != "}") ++q;   // the rest of a line is not part of the value
            }
        }
    }
}

}  // namespace info_parser
}  // namespace property_tree
}  // namespace boost
