// Driver of the reference's own solver code (test infrastructure): src/Solvers/Simple.cpp,
// Piso.cpp, IbPiso.cpp, Coupled.cpp and Diffusion.cpp with the mesh, fields, schemes and math they
// use, compiled from the
// reference's sources where they lie (oracle/Makefile, target refsolver) against the stand-in
// headers in refshim/include.  A case is set up the way the reference's module mains do it
// (Modules/caffeSimple.cpp:13-30): Input reads case/case.info, the mesh is built from a node
// array (HexaFvmMesh::initialize(const Array3D<Point3D>&)), the solver is constructed from both
// and Solver::solve(timeStep) is called once per step.  Fields are read back through a class
// derived from the solver (its fields are protected members); every linear system the solver
// assembles is recorded by the stand-in KSPSolve.  Exposed to ctypes by tests/ and the golden
// fixture script; nothing in the product links it.
#include <unistd.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "Coupled.h"
#include "Diffusion.h"
#include "IbPiso.h"
#include "Interpolation.h"
#include "Parallel.h"
#include "Piso.h"
#include "Simple.h"

#include "refshim/refshim.h"

namespace {

template <class B>
struct Open : B {
    Open(const Input& in, const HexaFvmMesh& m) : B(in, m) {}
    Field<Vector3D>& u() { return this->uField_; }
    Field<double>& p() { return this->pField_; }
    Field<double>& pc() { return this->pCorrField_; }
    Field<double>& d() { return this->dField_; }
    Field<double>& mf() { return this->massFlowField_; }
    Field<Vector3D>& gradP() { return this->gradPField_; }
};

// the Coupled and Diffusion solvers' fields (protected members)
struct OpenCoupled : Coupled {
    OpenCoupled(const Input& in, const HexaFvmMesh& m) : Coupled(in, m) {}
    Field<Vector3D>& u() { return uField_; }
    Field<double>& p() { return pField_; }
    Field<double>& d() { return dField_; }
    Field<double>& mf() { return massFlowField_; }
    Field<Vector3D>& gradP() { return gradPField_; }
    Field<Vector3D>& h() { return hField_; }
};
struct OpenDiffusion : Diffusion {
    OpenDiffusion(const Input& in, const HexaFvmMesh& m) : Diffusion(in, m) {}
    Field<double>& phi() { return phiField_; }
    Field<Vector3D>& gradPhi() { return gradPhiField_; }
};

struct Run {
    std::unique_ptr<Input> input;
    std::unique_ptr<HexaFvmMesh> mesh;
    std::unique_ptr<Solver> solver;
    int kind = 0;
    int nI = 0, nJ = 0, nK = 0;
    template <class F>
    auto with(F&& f) {   // kinds 0-2: the flow solvers
        if (kind == 0) return f(*static_cast<Open<Simple>*>(solver.get()));
        if (kind == 1) return f(*static_cast<Open<Piso>*>(solver.get()));
        return f(*static_cast<Open<IbPiso>*>(solver.get()));
    }
};

std::string g_err;
bool g_parallel = false;

}  // namespace

extern "C" {

const char* refsolver_last_error(void) { return g_err.c_str(); }

void refsolver_set_tolerance(double rtol, int maxit) { refshim::set_solve_tolerance(rtol, maxit); }
void refsolver_record(int on) { refshim::set_recording(on != 0); refshim::systems().clear(); }
int refsolver_nsystems(void) { return (int)refshim::systems().size(); }
void refsolver_inject(const double* x, int n) { refshim::inject(x, n); }
void refsolver_clear_injected(void) { refshim::clear_injected(); }
int refsolver_injected_left(void) { return refshim::injected_left(); }

// sizes of recorded system k: rows and stored entries
int refsolver_system_size(int k, int* n, int* nnz) {
    auto& s = refshim::systems();
    if (k < 0 || k >= (int)s.size()) return 1;
    *n = s[k].n;
    *nnz = (int)s[k].col.size();
    return 0;
}
int refsolver_system(int k, int* ptr, int* col, double* val, double* b, double* x) {
    auto& s = refshim::systems();
    if (k < 0 || k >= (int)s.size()) return 1;
    const refshim::System& q = s[k];
    std::memcpy(ptr, q.ptr.data(), sizeof(int) * q.ptr.size());
    std::memcpy(col, q.col.data(), sizeof(int) * q.col.size());
    std::memcpy(val, q.val.data(), sizeof(double) * q.val.size());
    std::memcpy(b, q.b.data(), sizeof(double) * q.b.size());
    std::memcpy(x, q.x.data(), sizeof(double) * q.x.size());
    return 0;
}

// casedir holds case/case.info and case/initialConditions.info; nodes are (nNK, nNJ, nNI, 3)
void* refsolver_create(const char* casedir, const double* nodes, int nNI, int nNJ, int nNK, int kind) {
    g_err.clear();
    if (!g_parallel) { Parallel::initialize(); g_parallel = true; }
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) { g_err = "getcwd failed"; return nullptr; }
    if (chdir(casedir) != 0) { g_err = std::string("cannot enter ") + casedir; return nullptr; }
    Run* r = new Run();
    r->kind = kind;
    try {
        r->input.reset(new Input());
        Array3D<Point3D> pts(nNI, nNJ, nNK);
        for (int k = 0; k < nNK; ++k)
            for (int j = 0; j < nNJ; ++j)
                for (int i = 0; i < nNI; ++i) {
                    const double* p = nodes + 3 * (((size_t)k * nNJ + j) * nNI + i);
                    pts(i, j, k) = Point3D(p[0], p[1], p[2]);
                }
        r->mesh.reset(new HexaFvmMesh());
        r->mesh->initialize(pts);
        if (kind == 0) r->solver.reset(new Open<Simple>(*r->input, *r->mesh));
        else if (kind == 1) r->solver.reset(new Open<Piso>(*r->input, *r->mesh));
        else if (kind == 2) r->solver.reset(new Open<IbPiso>(*r->input, *r->mesh));
        else if (kind == 3) r->solver.reset(new OpenCoupled(*r->input, *r->mesh));
        else r->solver.reset(new OpenDiffusion(*r->input, *r->mesh));
        r->nI = nNI - 1; r->nJ = nNJ - 1; r->nK = nNK - 1;
    } catch (const char* msg) {
        g_err = msg;
    } catch (const std::exception& e) {
        g_err = e.what();
    }
    if (chdir(cwd) != 0 && g_err.empty()) g_err = "cannot return to the working directory";
    if (!g_err.empty()) { delete r; return nullptr; }
    return r;
}

void refsolver_destroy(void* h) { delete static_cast<Run*>(h); }

// The reference reads uninitialised memory when it sets up the pressure boundary conditions:
// PrimitiveBoundaryCondition<double>::refValues_[6] (PrimitiveBoundaryCondition.h:42) is never
// initialised, and FlowBoundaryConditions (FlowBoundaryConditions.cpp:44-71) configures the faces
// in order with changeType, which for a FIXED type (an outlet's pressure) copies all six
// refValues_ into the patches of every face whose type is still the constructor's FIXED
// (PrimitiveBoundaryCondition.tpp:257-294).  The faces configured after an outlet therefore
// start with arbitrary patch values, which the first step's Rhie-Chow fluxes read before the
// first setBoundaries() replaces them.  This sets such a face's pressure patch and boundary
// faces to 0, the value zero-initialised memory gives (and the oracle and device use), so that
// the reference's first step is deterministic.
int refsolver_zero_pressure_patch(void* h, int face) {
    Run* r = static_cast<Run*>(h);
    if (face < 0 || face > 5) return 1;
    if (r->kind == 3) {
        Field<double>& p = static_cast<OpenCoupled*>(r->solver.get())->p();
        Array3D<double>* patch[6] = {&p.eastBoundaryPatch, &p.westBoundaryPatch, &p.northBoundaryPatch,
                                     &p.southBoundaryPatch, &p.topBoundaryPatch, &p.bottomBoundaryPatch};
        patch[face]->assign(0.);
        switch (face) {
            case 0: p.setEastFacesFromPatch(); break;
            case 1: p.setWestFacesFromPatch(); break;
            case 2: p.setNorthFacesFromPatch(); break;
            case 3: p.setSouthFacesFromPatch(); break;
            case 4: p.setTopFacesFromPatch(); break;
            default: p.setBottomFacesFromPatch(); break;
        }
        return 0;
    }
    if (r->kind > 3) return 1;
    return r->with([&](auto& s) -> int {
        Field<double>& p = s.p();
        Array3D<double>* patch[6] = {&p.eastBoundaryPatch, &p.westBoundaryPatch, &p.northBoundaryPatch,
                                     &p.southBoundaryPatch, &p.topBoundaryPatch, &p.bottomBoundaryPatch};
        patch[face]->assign(0.);
        switch (face) {
            case 0: p.setEastFacesFromPatch(); break;
            case 1: p.setWestFacesFromPatch(); break;
            case 2: p.setNorthFacesFromPatch(); break;
            case 3: p.setSouthFacesFromPatch(); break;
            case 4: p.setTopFacesFromPatch(); break;
            default: p.setBottomFacesFromPatch(); break;
        }
        return 0;
    });
}

// one Solver::solve(timeStep); returns its value (the continuity error), NaN on an exception
double refsolver_solve(void* h, double dt) {
    g_err.clear();
    try {
        return static_cast<Run*>(h)->solver->solve(dt);
    } catch (const char* msg) {
        g_err = msg;
    } catch (const std::exception& e) {
        g_err = e.what();
    }
    return std::nan("");
}

// "u" (N x 3), "gradP" (N x 3), "p", "pCorr", "d", "massFlow" (cells), "massFlowI/J/K" (faces); the
// Coupled solver: "u", "gradP", "h", "p", "d", "massFlowI/J/K"; Diffusion: "phi", "gradPhi", "phiFaceI/J/K"
long refsolver_field(void* h, const char* name, double* out, long count) {
    Run* r = static_cast<Run*>(h);
    std::string n(name);
    const int nI = r->nI, nJ = r->nJ, nK = r->nK;
    auto cells = [&](auto& f, int comps) -> long {
        long need = (long)nI * nJ * nK * comps;
        if (out && count >= need)
            for (int k = 0; k < nK; ++k)
                for (int j = 0; j < nJ; ++j)
                    for (int i = 0; i < nI; ++i) {
                        long c = ((long)k * nJ + j) * nI + i;
                        const auto& v = f(i, j, k);
                        double* o = out + comps * c;
                        if constexpr (std::is_same<std::decay_t<decltype(v)>, Vector3D>::value) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }
                        else o[0] = v;
                    }
        return need;
    };
    auto faces = [&](Field<double>& f, int dir) -> long {
        int a = nI + (dir == 0), b = nJ + (dir == 1), c = nK + (dir == 2);
        long need = (long)a * b * c;
        if (out && count >= need)
            for (int k = 0; k < c; ++k)
                for (int j = 0; j < b; ++j)
                    for (int i = 0; i < a; ++i) {
                        double v = dir == 0 ? f.faceI(i, j, k) : (dir == 1 ? f.faceJ(i, j, k) : f.faceK(i, j, k));
                        out[((long)k * b + j) * a + i] = v;
                    }
        return need;
    };
    if (r->kind == 3) {
        OpenCoupled& s = *static_cast<OpenCoupled*>(r->solver.get());
        if (n == "u") return cells(s.u(), 3);
        if (n == "gradP") return cells(s.gradP(), 3);
        if (n == "h") return cells(s.h(), 3);
        if (n == "p") return cells(s.p(), 1);
        if (n == "d") return cells(s.d(), 1);
        if (n == "massFlowI") return faces(s.mf(), 0);
        if (n == "massFlowJ") return faces(s.mf(), 1);
        if (n == "massFlowK") return faces(s.mf(), 2);
        return -1L;
    }
    if (r->kind == 4) {
        OpenDiffusion& s = *static_cast<OpenDiffusion*>(r->solver.get());
        if (n == "phi") return cells(s.phi(), 1);
        if (n == "gradPhi") return cells(s.gradPhi(), 3);
        if (n == "phiFaceI") return faces(s.phi(), 0);
        if (n == "phiFaceJ") return faces(s.phi(), 1);
        if (n == "phiFaceK") return faces(s.phi(), 2);
        return -1L;
    }
    return r->with([&](auto& s) -> long {
        if (n == "u") return cells(s.u(), 3);
        if (n == "gradP") return cells(s.gradP(), 3);
        if (n == "p") return cells(s.p(), 1);
        if (n == "pCorr") return cells(s.pc(), 1);
        if (n == "d") return cells(s.d(), 1);
        if (n == "massFlow") return cells(s.mf(), 1);
        if (n == "massFlowI") return faces(s.mf(), 0);
        if (n == "massFlowJ") return faces(s.mf(), 1);
        if (n == "massFlowK") return faces(s.mf(), 2);
        return -1L;
    });
}

// Interpolation::computeTrilinearCoeffs (src/Math/Interpolation.cpp:135-180) for 8 points
// (p24, x y z each) and an interpolation point: beta (8 values)
int refsolver_trilinear(const double* p24, const double* ip, double* beta) {
    g_err.clear();
    try {
        Point3D pts[8];
        for (int q = 0; q < 8; ++q) pts[q] = Point3D(p24[3 * q], p24[3 * q + 1], p24[3 * q + 2]);
        Matrix m = Interpolation::computeTrilinearCoeffs(pts, 8, Point3D(ip[0], ip[1], ip[2]));
        for (int q = 0; q < 8; ++q) beta[q] = m(0, q);
    } catch (const char* msg) {
        g_err = msg;
        return 1;
    }
    return 0;
}

}  // extern "C"
