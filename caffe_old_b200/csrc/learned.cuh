// Learned-preconditioner solve and training (learned.cu).
#pragma once
#include "cnn.cuh"
#include "krylov.cuh"

namespace cb {

constexpr int LEARN_MAX_LEVELS = 12;

// FP32 copy of the symmetric 7-point p' operator (plus the FP64 ghost rows)
struct OpSymF32 {
    const float* aP;
    const float* aE;
    const float* aN;
    const float* aT;
    long long nI, nIJ;
    GhostRows gh;
};

// Level l of the coarsening pyramid (l = 0 is the cell lattice itself).
struct Level {
    int n[3];            // cells along i, j, k
    long long N;
    float rscale;        // restriction = rscale * P^T (cell average)
    float gain;          // output gain of the level's term (4^l)
    float chan;          // constant level channel fed to the network
    float* u = nullptr;  // restricted Jacobi-scaled residual (training: adjoint of w)
    float* w = nullptr;  // prolongation accumulator (training: dL/dy)
    float* mask = nullptr;   // fraction of active cells
    NetBuffers net;      // activations of this level for the input x; weights shared with level 1
    NetBuffers netNeg;   // activations for the input -x (the network term is odd: (net(x) - net(-x)) / 2)
    float* w2 = nullptr; // training: dL/dy of the -x evaluation
};

enum { NET_MODE_JACOBI = 0, NET_MODE_NETWORK = 1, NET_MODE_LEVELS = 2 };
// inner Krylov method: automatic = flexible CG for a symmetric operator; for a non-symmetric
// one, FGMRES when the network runs (a preconditioner that varies between applications) and
// BiCGStab otherwise (a fixed linear preconditioner)
enum { LEARN_INNER_AUTO = 0, LEARN_INNER_FCG = 1, LEARN_INNER_BICGSTAB = 2, LEARN_INNER_FGMRES = 3 };
constexpr int FGMRES_MAX_RESTART = 64;

struct LearnedWork {
    Lat L;
    float* r = nullptr;
    float* z = nullptr;
    float* e = nullptr;
    float* p[2] = {nullptr, nullptr};
    float* q[2] = {nullptr, nullptr};
    float* t = nullptr;
    float* rh = nullptr;
    float* invD = nullptr;
    float* A[4] = {nullptr, nullptr, nullptr, nullptr};
    double* part = nullptr;
    double* mean = nullptr;
    void* scal = nullptr;        // device scalar record
    void* hostScal = nullptr;    // pinned copy
    int nLev = 0;                // levels 1 .. nLev-1 form the pyramid
    Level lev[LEARN_MAX_LEVELS];
    NetBuffers* weights = nullptr;   // the level whose NetBuffers own params / packed weights / grad
    bool masksReady = false;
    bool haveParams = false;
    int netFrom = 1;             // first level that runs the network (finer levels: identity)
    int netTo = 1 << 20;         // last level that runs the network (coarser levels: identity)
    int inner = LEARN_INNER_AUTO;
    int restart = 40;            // FGMRES cycle length (one cycle per FP64 refinement pass)
    // FGMRES basis (restart + 1 planes) and preconditioned vectors (restart planes), one
    // allocation each, planes PS apart; scalar record and dot partials
    float* fgV = nullptr;
    float* fgZ = nullptr;
    int fgCap = 0;
    void* fgScal = nullptr;
    double* fgPart = nullptr;
    void* (*alloc)(size_t, void*) = nullptr;
    void* allocCtx = nullptr;
    int lastIters = 0, lastOuter = 0;
    int* rtErr = nullptr;        // set by the TMA-staged restriction when a wait ran out
    unsigned* ctr = nullptr;     // finished-block counter of the kernels that end with their own reduction
    float* u1 = nullptr;         // D^-1 x on active cells of the vector being preconditioned (restriction input)
};

int learned_alloc(LearnedWork& lw, const Lat& L, void* (*alloc)(size_t, void*), void* ctx);
void learned_free_host(LearnedWork& lw);
// FP64 refinement around an FP32 inner Krylov solve (flexible CG for the symmetric operator;
// FGMRES or BiCGStab when immersed-boundary ghost rows make it non-symmetric) with
//   M(r) = D^-1 r + sum_l P_l (gain_l s y_l),  y_l = net(R_l D^-1 r / s) (mode NETWORK),
//   y_l = R_l D^-1 r / s (mode LEVELS), nothing (mode JACOBI).
// Writes iterations / outer passes / relative residual / status to *out (device).
int learned_solve(LearnedWork& lw, const OpSym& A, const uint8_t* status, const double* b, double* x, const Lat& L, double rtol,
                  int maxit, double eta, int project, int mode, KspOut* out, cudaStream_t st, double atol = 0.);
// Train the network on pairs (b, x*) stored as FP32 halo-padded planes [n][PS] in device memory.
int learned_train(LearnedWork& lw, const OpSym& A, const uint8_t* status, const Lat& L, const float* pairsB, const float* pairsX,
                  int nPairs, int steps, int batch, float lr, unsigned seed, float* lossHost, cudaStream_t st);
// Training pair of an intermediate iterate xk of a solve with solution xstar: (b - A xk, xstar - xk) in FP32.
int learned_snapshot_pair(const OpSym& A, const Lat& L, const double* b, const double* xstar, const double* xk, float* pb, float* px,
                          cudaStream_t st);
// n synthetic pairs (A e, e): e = seeded uniform noise on pyramid level q mod levels,
// prolonged to the cell lattice (zero off the active cells): smooth at every scale the
// pyramid spans.  Written to FP32 halo-padded planes [n][PS].
int learned_random_pairs(LearnedWork& lw, const OpSym& A, const uint8_t* status, const Lat& L, int nPairs, unsigned seed, float* pairsB,
                         float* pairsX, cudaStream_t st);
// Energy-norm loss of one application M(b) against x* for each of n pairs (mode as above).
int learned_eval(LearnedWork& lw, const OpSym& A, const uint8_t* status, const Lat& L, const float* pairsB, const float* pairsX,
                 int nPairs, int mode, float* lossHost, cudaStream_t st);

}  // namespace cb
