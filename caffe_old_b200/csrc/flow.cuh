// Views passed to the finite-volume kernels and their host launchers.
#pragma once
#include "common.cuh"

namespace cb {

struct FlowFields {
    double* u;        // 3 planes
    const double* u0; // 3 planes (may alias u)
    double* gradP;    // 3 planes
    double* gradPC;   // 3 planes
    double* gradU;    // 9 planes, only with the non-orthogonal extension
    double* p;
    double* pc;       // p'
    double* d;
    double* mfc;      // net mass flux per cell (massFlowField_ cell values)
    double* F[3];     // face mass fluxes, +i/+j/+k oriented
    double* Fout[3];  // second buffer written by the correct kernel
    double* pPatch[6];
    const uint8_t* status;   // nullptr when every cell is active
    int nonorth;
};

struct MomSys {
    double* a[7];     // aP aE aW aN aS aT aB, per cell
    double* b;        // 3 planes
};

struct PcSys {
    double* aP;       // per cell
    double* aE;       // per cell: coefficient of the east neighbour (= west coefficient of that neighbour)
    double* aN;       // per cell: north
    double* aT;       // per cell: top
    double* b;
};

struct FlowParams {
    double rho, mu, omega_u, omega_p;
    int unsteady;
    int convection;
};

int compute_metrics(const Lat& L, const double* d_xyz, double* vol, double* cc, double* S[3], double* fc[3],
                    double* D[3], double* cv[3], cudaStream_t st);
int launch_momentum_assemble(const Geo& g, const Bc& bc, const FlowFields& f, const MomSys& m, const FlowParams& P, double dt,
                             cudaStream_t st);
int launch_rhie_chow(const Geo& g, const Bc& bc, const FlowFields& f, const FlowParams& P, cudaStream_t st);
int launch_pcorr_assemble(const Geo& g, const Bc& bc, const FlowFields& f, const PcSys& s, const FlowParams& P, cudaStream_t st);
int launch_correct(const Geo& g, const Bc& bc, const FlowFields& f, const FlowParams& P, cudaStream_t st);
// gradU = false leaves grad u (non-orthogonal extension) to launch_grad_u, for a slab whose u
// halo planes must be exchanged in between
int launch_correct_post(const Geo& g, const Bc& bc, const FlowFields& f, cudaStream_t st, bool gradU = true);
int launch_grad_u(const Geo& g, const Bc& bc, const FlowFields& f, cudaStream_t st);
// max over the cells [c0, c1); c1 < 0: all cells
int launch_courant(const Geo& g, const FlowFields& f, double dt, unsigned long long* d_out, cudaStream_t st, long long c0 = 0,
                   long long c1 = -1);
int launch_continuity(const Lat& L, const double* mfc, const double* vol, const uint8_t* status, double* chunkMax, double* d_out,
                      cudaStream_t st);

}  // namespace cb
