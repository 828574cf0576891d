// Solvers of the host layer over the device library's C ABI (include/caffe_b200.h).
// caseFromInput reads the keys of case/case.info that Solver / Simple / Piso / IbPiso read in
// the reference (Solver.cpp:8, Simple.cpp:61-67,104-108, Piso.cpp:9,
// FlowBoundaryConditions.cpp:25-40, IbPiso.cpp:37-38), plus optional keys for what the
// reference leaves to PETSc defaults or does not have:
//   Solver.convectionScheme            upwind (the reference) | central
//   Solver.nonOrthogonalCorrection     OFF (the reference) | ON
//   LinearSolvers.momentum / .pressureCorrection   bicgstab_jacobi | cg_jacobi
//   LinearSolvers.tolerance            relative true residual (default 1e-8)
//   LinearSolvers.absoluteTolerance    absolute floor of ||b - A x|| (PETSc's atol; default 0)
//   LinearSolvers.maxIterations        (default 20000)
//   LinearSolvers.pressureCorrectionForm   fp64 | mixed | learned | learned_mixed
//   LearnedPreconditioner.mode         levels | network | jacobi
//   LearnedPreconditioner.parameters   file of caffe_precond_param_count() floats (raw or .npy)
//   LearnedPreconditioner.firstNetworkLevel   first pyramid level that runs the network (1)
//   LearnedPreconditioner.lastNetworkLevel    last pyramid level that runs the network (all)
//   LearnedPreconditioner.innerMethod  auto | fcg | bicgstab | fgmres
//   LearnedPreconditioner.restart      FGMRES cycle length (40)
#include "Solver.h"

#include <cstring>
#include <fstream>
#include <iostream>

#include "Coupled.h"
#include "Diffusion.h"
#include "IbPiso.h"
#include "MultiphasePiso.h"
#include "InitialConditions.h"
#include "Output.h"
#include "Piso.h"
#include "Simple.h"

namespace {

int face_type(const std::string& t) {
    if (t == "inlet") return CAFFE_INLET;
    if (t == "outlet") return CAFFE_OUTLET;
    if (t == "wall") return CAFFE_WALL;
    if (t == "empty") return CAFFE_EMPTY;
    if (t == "zeroGradient") return CAFFE_ZERO_GRADIENT;
    Output::raiseException("FlowBoundaryConditions", "FlowBoundaryConditions", "unrecognized boundary type \"" + t + "\".");
    return -1;
}

int ksp_method(const std::string& m) {
    if (m == "bicgstab_jacobi") return CAFFE_KSP_BICGSTAB_JACOBI;
    if (m == "cg_jacobi") return CAFFE_KSP_CG_JACOBI;
    if (m == "bicgstab_sgs") return CAFFE_KSP_BICGSTAB_SGS;
    Output::raiseException("Solver", "caseFromInput", "unknown linear solver \"" + m + "\"");
    return -1;
}

int p_form(const std::string& f) {
    if (f == "fp64") return CAFFE_P_FP64;
    if (f == "mixed") return CAFFE_P_MIXED;
    if (f == "learned") return CAFFE_P_LEARNED;
    if (f == "learned_mixed") return CAFFE_P_LEARNED_MIXED;
    Output::raiseException("Solver", "caseFromInput", "unknown pressure-correction form \"" + f + "\"");
    return -1;
}

// raw float32 file or NumPy .npy (version 1-3, little-endian float32, C order)
std::vector<float> read_params(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) Output::raiseException("Solver", "readParams", "cannot open \"" + path + "\"");
    std::vector<char> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t off = 0;
    if (bytes.size() >= 10 && std::memcmp(bytes.data(), "\x93NUMPY", 6) == 0) {
        int major = (unsigned char)bytes[6];
        size_t hlen = major == 1 ? (size_t)(unsigned char)bytes[8] | ((size_t)(unsigned char)bytes[9] << 8)
                                 : (size_t)(unsigned char)bytes[8] | ((size_t)(unsigned char)bytes[9] << 8) |
                                       ((size_t)(unsigned char)bytes[10] << 16) | ((size_t)(unsigned char)bytes[11] << 24);
        off = (major == 1 ? 10 : 12) + hlen;
        std::string header(bytes.data() + (major == 1 ? 10 : 12), hlen);
        if (header.find("<f4") == std::string::npos) Output::raiseException("Solver", "readParams", "\"" + path + "\" is not float32");
    }
    size_t n = (bytes.size() - off) / 4;
    std::vector<float> p(n);
    if (n) std::memcpy(p.data(), bytes.data() + off, n * 4);
    return p;
}

}  // namespace

caffe_case Solver::caseFromInput(const Input& input, int kind) {
    const InfoTree& c = input.caseParameters;
    caffe_case cs;
    std::memset(&cs, 0, sizeof(cs));
    cs.kind = kind;
    static const char* faces[6] = {"east", "west", "north", "south", "top", "bottom"};
    for (int f = 0; f < 6; ++f) {
        std::string b = std::string("Boundaries.") + faces[f];
        cs.bc_type[f] = face_type(c.get<std::string>(b + ".type"));
        cs.ref_val[f] = c.get<double>(b + ".refValue");
        Vector3D v = std::stov(c.get<std::string>(b + ".refVector"));
        cs.ref_vec[f][0] = v.x; cs.ref_vec[f][1] = v.y; cs.ref_vec[f][2] = v.z;
    }
    cs.time_accurate = c.get<std::string>("Solver.timeAccurate") == "ON" ? 1 : 0;
    cs.n_inner = cs.time_accurate ? c.get<int>("Solver.numberOfInnerIterations") : 1;
    cs.omega_u = c.get<double>("Solver.relaxationFactorMomentum");
    cs.omega_p = c.get<double>("Solver.relaxationFactorPCorr");
    cs.rho = c.get<double>("Solver.rho");
    cs.mu = c.get<double>("Solver.mu");
    cs.n_pcorr = kind == CAFFE_SIMPLE ? 1 : c.get<int>("Solver.numberOfPressureCorrections");
    std::string conv = c.get<std::string>("Solver.convectionScheme", std::string("upwind"));
    if (conv != "upwind" && conv != "central") Output::raiseException("Solver", "caseFromInput", "unknown convection scheme \"" + conv + "\"");
    cs.convection = conv == "central" ? 1 : 0;
    cs.nonorth = c.get<std::string>("Solver.nonOrthogonalCorrection", std::string("OFF")) == "ON" ? 1 : 0;
    cs.mom_method = ksp_method(c.get<std::string>("LinearSolvers.momentum", std::string("bicgstab_jacobi")));
    cs.p_method = ksp_method(c.get<std::string>("LinearSolvers.pressureCorrection", std::string("bicgstab_jacobi")));
    cs.mom_rtol = cs.p_rtol = c.get<double>("LinearSolvers.tolerance", 1e-8);
    cs.mom_atol = cs.p_atol = c.get<double>("LinearSolvers.absoluteTolerance", 0.);
    cs.maxit = c.get<int>("LinearSolvers.maxIterations", 20000);
    cs.p_form = p_form(c.get<std::string>("LinearSolvers.pressureCorrectionForm", std::string("fp64")));
    if (kind == CAFFE_IBPISO) {
        cs.ib_radius = c.get<double>("ImmersedBoundaries.Sphere.radius");
        Vector3D ctr = std::stov(c.get<std::string>("ImmersedBoundaries.Sphere.center"));
        cs.ib_center[0] = ctr.x; cs.ib_center[1] = ctr.y; cs.ib_center[2] = ctr.z;
    }
    // uniform initial conditions go into the case record; others are uploaded after creation
    const InfoTree& ic = input.initialConditions;
    if (ic.get<std::string>("u.type", std::string("uniform")) == "uniform" && ic.has("u.value")) {
        Vector3D u = std::stov(ic.get<std::string>("u.value"));
        cs.u_init[0] = u.x; cs.u_init[1] = u.y; cs.u_init[2] = u.z;
    }
    if (ic.get<std::string>("p.type", std::string("uniform")) == "uniform" && ic.has("p.value")) cs.p_init = ic.get<double>("p.value");
    return cs;
}

Solver::Solver(const Input& input, const HexaFvmMesh& mesh, int kind) : mesh_(mesh) {
    case_ = caseFromInput(input, kind);
    const int nI1 = mesh.nCellsI() + 1, nJ1 = mesh.nCellsJ() + 1, nK1 = mesh.nCellsK() + 1;
    if (caffe_dev_create(mesh.nodes().data(), nI1, nJ1, nK1, &case_, 0, &h_) != 0)
        Output::raiseException("Solver", "Solver", std::string("device set-up failed: ") + caffe_last_error());
    // non-uniform initial conditions: evaluated at the cell centroids on the host, uploaded
    InitialConditions ics(input);
    const long N = (long)mesh.nCells();
    for (const char* fname : {"u", "p"}) {
        if (!ics.has(fname) || input.initialConditions.get<std::string>(std::string(fname) + ".type") == "uniform") continue;
        std::vector<double> cc(3 * N);
        if (caffe_dev_array(h_, "cc", cc.data(), (long)cc.size(), 2) < 0)
            Output::raiseException("Solver", "Solver", std::string("cannot read cell centroids: ") + caffe_last_error());
        setField(fname, ics.values(fname, std::strcmp(fname, "u") == 0 ? 3 : 1, cc));
    }
    // learned pressure-correction options
    if (case_.p_form == CAFFE_P_LEARNED || case_.p_form == CAFFE_P_LEARNED_MIXED) {
        const InfoTree& c = input.caseParameters;
        std::string mode = c.get<std::string>("LearnedPreconditioner.mode", std::string("levels"));
        int m = mode == "network" ? CAFFE_NET_NETWORK : (mode == "jacobi" ? CAFFE_NET_JACOBI : CAFFE_NET_LEVELS);
        if (c.has("LearnedPreconditioner.parameters")) {
            std::vector<float> p = read_params(c.get<std::string>("LearnedPreconditioner.parameters"));
            if ((int)p.size() != caffe_precond_param_count())
                Output::raiseException("Solver", "Solver", "learned-preconditioner parameter file has the wrong size");
            if (caffe_dev_set_precond(h_, p.data()) != 0)
                Output::raiseException("Solver", "Solver", std::string("cannot set the network parameters: ") + caffe_last_error());
        }
        if (caffe_dev_set_precond_mode(h_, m) != 0)
            Output::raiseException("Solver", "Solver", std::string("cannot set the preconditioner mode: ") + caffe_last_error());
        std::string inner = c.get<std::string>("LearnedPreconditioner.innerMethod", std::string("auto"));
        int im = inner == "fcg" ? 1 : (inner == "bicgstab" ? 2 : (inner == "fgmres" ? 3 : 0));
        if (inner != "auto" && im == 0) Output::raiseException("Solver", "Solver", "unknown inner method \"" + inner + "\"");
        int netFrom = c.get<int>("LearnedPreconditioner.firstNetworkLevel", 1);
        int restart = c.get<int>("LearnedPreconditioner.restart", 40);
        if (caffe_dev_set_precond_options(h_, im, netFrom, restart) != 0)
            Output::raiseException("Solver", "Solver", std::string("cannot set the preconditioner options: ") + caffe_last_error());
        int netTo = c.get<int>("LearnedPreconditioner.lastNetworkLevel", -1);
        if (caffe_dev_set_precond_net_levels(h_, netFrom, netTo) != 0)
            Output::raiseException("Solver", "Solver", std::string("cannot set the network levels: ") + caffe_last_error());
    }
    mesh.attachSolver(this);
}

Solver::Solver(const HexaFvmMesh& mesh, const char* name) : mesh_(mesh) {
    std::memset(&case_, 0, sizeof(case_));
    name_ = name;
    mesh.attachSolver(this);
}

Solver::~Solver() {
    mesh_.detachSolver(this);
    if (h_) caffe_dev_destroy(h_);
}

double Solver::step(double timeStep) {
    int rc = caffe_dev_solve(h_, timeStep, &stats_);
    if (rc != 0) Output::raiseException(name_, "solve", std::string("device step failed: ") + caffe_last_error());
    return stats_.continuity;
}

void Solver::displayUpdateMessage() {
    Output::print(name_, "completed iteration.");
    Output::print(name_, "Krylov iterations (p') : " + std::to_string(stats_.p_iters_total));
    Output::print(name_, "Max continuity error   : " + std::to_string(stats_.continuity));
    if (case_.kind != CAFFE_IBPISO) Output::print(name_, "Max Courant number     : " + std::to_string(stats_.courant));
    Output::printLine();
}

std::vector<double> Solver::field(const std::string& name) const {
    long n = caffe_dev_array(h_, name.c_str(), nullptr, 0, 0);
    if (n < 0) Output::raiseException(name_, "field", "unknown field \"" + name + "\"");
    std::vector<double> out((size_t)n);
    if (caffe_dev_array(h_, name.c_str(), out.data(), n, 2) < 0)
        Output::raiseException(name_, "field", std::string("read failed: ") + caffe_last_error());
    return out;
}

void Solver::setField(const std::string& name, const std::vector<double>& values) {
    if (caffe_dev_array(h_, name.c_str(), const_cast<double*>(values.data()), (long)values.size(), 3) < 0)
        Output::raiseException(name_, "setField", std::string("write failed: ") + caffe_last_error());
}

Simple::Simple(const Input& input, const HexaFvmMesh& mesh) : Simple(input, mesh, CAFFE_SIMPLE) {}
Simple::Simple(const Input& input, const HexaFvmMesh& mesh, int kind) : Solver(input, mesh, kind) { name_ = "Simple"; }
double Simple::solve(double timeStep) { return step(timeStep); }

Piso::Piso(const Input& input, const HexaFvmMesh& mesh) : Piso(input, mesh, CAFFE_PISO) {}
Piso::Piso(const Input& input, const HexaFvmMesh& mesh, int kind) : Simple(input, mesh, kind) { name_ = "Piso"; }
double Piso::solve(double timeStep) { return step(timeStep); }

IbPiso::IbPiso(const Input& input, const HexaFvmMesh& mesh) : Piso(input, mesh, CAFFE_IBPISO) { name_ = "IbPiso"; }
double IbPiso::solve(double timeStep) { return step(timeStep); }

MultiphasePiso::MultiphasePiso(const Input& input, const HexaFvmMesh& mesh) : Piso(input, mesh, CAFFE_PISO) { name_ = "MultiphasePiso"; }
double MultiphasePiso::solve(double timeStep) { return step(timeStep); }

// ---------------------------------------------------------------------------- Coupled
namespace {

// an interleaved N x c host array from the device library as c planes of N
std::vector<double> to_planes(const std::vector<double>& a, int comps) {
    if (comps == 1) return a;
    const size_t n = a.size() / comps;
    std::vector<double> out(a.size());
    for (size_t q = 0; q < n; ++q)
        for (int c = 0; c < comps; ++c) out[c * n + q] = a[q * comps + c];
    return out;
}
std::vector<double> to_interleaved(const std::vector<double>& a, int comps) {
    if (comps == 1) return a;
    const size_t n = a.size() / comps;
    std::vector<double> out(a.size());
    for (size_t q = 0; q < n; ++q)
        for (int c = 0; c < comps; ++c) out[q * comps + c] = a[c * n + q];
    return out;
}
int vector_components(const std::string& name) { return name == "u" || name == "u0" || name == "gradP" || name == "h" || name == "gradPhi" || name == "cc" ? 3 : 1; }

}  // namespace

Coupled::Coupled(const Input& input, const HexaFvmMesh& mesh) : Solver(mesh, "Coupled") {
    const InfoTree& c = input.caseParameters;
    static const char* faces[6] = {"east", "west", "north", "south", "top", "bottom"};
    for (int f = 0; f < 6; ++f) {
        std::string b = std::string("Boundaries.") + faces[f];
        case_.bc_type[f] = face_type(c.get<std::string>(b + ".type"));
        case_.ref_val[f] = c.get<double>(b + ".refValue");
        Vector3D v = std::stov(c.get<std::string>(b + ".refVector"));
        case_.ref_vec[f][0] = v.x; case_.ref_vec[f][1] = v.y; case_.ref_vec[f][2] = v.z;
    }
    case_.kind = CAFFE_SIMPLE;
    case_.time_accurate = c.get<std::string>("Solver.timeAccurate") == "ON" ? 1 : 0;
    case_.n_inner = case_.time_accurate ? c.get<int>("Solver.numberOfInnerIterations") : 1;
    case_.omega_u = c.get<double>("Solver.relaxationFactorMomentum");
    case_.omega_p = 1.;
    case_.rho = c.get<double>("Solver.rho");
    case_.mu = c.get<double>("Solver.mu");
    case_.mom_method = ksp_method(c.get<std::string>("LinearSolvers.momentum", std::string("bicgstab_jacobi")));
    case_.p_method = case_.mom_method;
    case_.mom_rtol = case_.p_rtol = c.get<double>("LinearSolvers.tolerance", 1e-8);
    case_.mom_atol = case_.p_atol = c.get<double>("LinearSolvers.absoluteTolerance", 0.);
    case_.maxit = c.get<int>("LinearSolvers.maxIterations", 20000);
    const int nI1 = mesh.nCellsI() + 1, nJ1 = mesh.nCellsJ() + 1, nK1 = mesh.nCellsK() + 1;
    if (caffe_coupled_create(mesh.nodes().data(), nI1, nJ1, nK1, &case_, 0, &hc_) != 0)
        Output::raiseException("Coupled", "Coupled", std::string("device set-up failed: ") + caffe_last_error());
}

Coupled::~Coupled() {
    if (hc_) caffe_coupled_destroy(hc_);
}

double Coupled::solve(double timeStep) {
    if (caffe_coupled_solve(hc_, timeStep, &continuity_) != 0)
        Output::raiseException("Coupled", "solve", std::string("device step failed: ") + caffe_last_error());
    return continuity_;
}

void Coupled::displayUpdateMessage() {
    int iters = 0, status = 0;
    double relres = 0.;
    caffe_coupled_stats(hc_, &iters, &relres, &status);
    Output::print("Coupled", "completed iteration.");
    Output::print("Coupled", "Krylov iterations (block system) : " + std::to_string(iters));
    Output::print("Coupled", "Max continuity error             : " + std::to_string(continuity_));
    Output::printLine();
}

std::vector<double> Coupled::field(const std::string& name) const {
    if (name == "massFlow") return std::vector<double>((size_t)mesh_.nCells(), 0.);
    long n = caffe_coupled_array(hc_, name.c_str(), nullptr, 0, 0);
    if (n < 0) Output::raiseException("Coupled", "field", "unknown field \"" + name + "\"");
    std::vector<double> out((size_t)n);
    if (caffe_coupled_array(hc_, name.c_str(), out.data(), n, 0) < 0)
        Output::raiseException("Coupled", "field", std::string("read failed: ") + caffe_last_error());
    return to_planes(out, vector_components(name));
}

void Coupled::setField(const std::string& name, const std::vector<double>& values) {
    std::vector<double> v = to_interleaved(values, vector_components(name));
    if (caffe_coupled_array(hc_, name.c_str(), v.data(), (long)v.size(), 1) < 0)
        Output::raiseException("Coupled", "setField", std::string("write failed: ") + caffe_last_error());
}

// ---------------------------------------------------------------------------- Diffusion
Diffusion::Diffusion(const Input& input, const HexaFvmMesh& mesh) : Solver(mesh, "Diffusion") {
    const InfoTree& c = input.caseParameters;
    static const char* faces[6] = {"east", "west", "north", "south", "top", "bottom"};
    int types[6];
    double refs[6];
    for (int f = 0; f < 6; ++f) {
        std::string b = std::string("Boundaries.") + faces[f];
        const std::string t = c.get<std::string>(b + ".type");
        if (t == "fixed") types[f] = 0;
        else if (t == "zeroGradient") types[f] = 1;
        else if (t == "empty") types[f] = 2;
        else Output::raiseException("FlowBoundaryCondition", "FlowBoundaryCondition", "invalid boundary type \"" + t + "\".");
        refs[f] = c.get<double>(b + ".refValue");
    }
    case_.time_accurate = c.get<std::string>("Solver.timeAccurate") == "ON" ? 1 : 0;
    const int method = ksp_method(c.get<std::string>("LinearSolvers.diffusion", std::string("bicgstab_jacobi")));
    const double rtol = c.get<double>("LinearSolvers.tolerance", 1e-8);
    const int maxit = c.get<int>("LinearSolvers.maxIterations", 20000);
    // a uniform phi goes in at creation; other initial conditions are evaluated at the centroids
    InitialConditions ics(input);
    double phi0 = 0.;
    const bool uniform = !ics.has("phi") || input.initialConditions.get<std::string>("phi.type") == "uniform";
    if (uniform && input.initialConditions.has("phi.value")) phi0 = input.initialConditions.get<double>("phi.value");
    const int nI1 = mesh.nCellsI() + 1, nJ1 = mesh.nCellsJ() + 1, nK1 = mesh.nCellsK() + 1;
    if (caffe_diffusion_create(mesh.nodes().data(), nI1, nJ1, nK1, types, refs, case_.time_accurate, phi0, method, rtol, maxit, 0, &hd_) != 0)
        Output::raiseException("Diffusion", "Diffusion", std::string("device set-up failed: ") + caffe_last_error());
    if (!uniform) setField("phi", ics.values("phi", 1, field("cc")));
}

Diffusion::~Diffusion() {
    if (hd_) caffe_diffusion_destroy(hd_);
}

double Diffusion::solve(double timeStep) {
    if (caffe_diffusion_solve(hd_, timeStep, &residual_, &iters_, &relres_) != 0)
        Output::raiseException("Diffusion", "solve", std::string("device solve failed: ") + caffe_last_error());
    return residual_;
}

void Diffusion::displayUpdateMessage() {
    Output::print("Diffusion", "completed iteration.");
    Output::print("Diffusion", "Krylov iterations : " + std::to_string(iters_));
    Output::print("Diffusion", "||A x - b||_inf   : " + std::to_string(residual_));
    Output::printLine();
}

std::vector<double> Diffusion::field(const std::string& name) const {
    long n = caffe_diffusion_array(hd_, name.c_str(), nullptr, 0, 0);
    if (n < 0) Output::raiseException("Diffusion", "field", "unknown field \"" + name + "\"");
    std::vector<double> out((size_t)n);
    if (caffe_diffusion_array(hd_, name.c_str(), out.data(), n, 0) < 0)
        Output::raiseException("Diffusion", "field", std::string("read failed: ") + caffe_last_error());
    return to_planes(out, vector_components(name));
}

void Diffusion::setField(const std::string& name, const std::vector<double>& values) {
    std::vector<double> v = to_interleaved(values, vector_components(name));
    if (caffe_diffusion_array(hd_, name.c_str(), v.data(), (long)v.size(), 1) < 0)
        Output::raiseException("Diffusion", "setField", std::string("write failed: ") + caffe_last_error());
}
