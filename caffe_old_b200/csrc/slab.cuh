// One slab of a k-slab decomposition: the phases of a distributed Krylov solve that run on
// the slab's own cells.
//
// A slab's handle holds the cells of its owned k-planes plus one halo plane on each side
// that has a neighbouring slab (its lattice is the global lattice's planes [k0-1, k1+1)
// clipped to the domain), so every finite-volume kernel runs unchanged on it and computes
// the owned cells exactly as on the whole lattice once the halo planes hold the neighbours'
// values.  The Krylov solves cannot run that way: their dot products span every slab.  They
// are split at each reduction into phases; a phase sweeps the owned cells [o0, o1), and,
// where it reduces, leaves its slab's sums in `red` for the caller to sum over the slabs.
// Every phase that applies A reads the halo plane of the vector it applies, which the
// caller exchanges right before it.
//
// The phases restate the persistent single-lattice solvers (krylov.cu): the same
// right-preconditioned Jacobi BiCGStab (van der Vorst 1992) and the same Chronopoulos-Gear
// Jacobi CG, with the same true-residual checks and restarts, taken by the caller.
#pragma once
#include "krylov.cuh"

namespace cb {

struct SlabKsp {
    Lat L;
    long long o0, o1;   // owned cells [o0, o1): whole k-planes
    double* b;          // nr planes (modified only by the mean projection)
    double* x;          // nr planes
    KspWork w;
    double* ph;         // nr planes: D^-1 p (BiCGStab), D^-1 r (CG); exchanged before A is applied to it
    double* sh;         // nr planes: D^-1 s (BiCGStab); exchanged before A is applied to it
    double* part;       // block partials, SLAB_MAX_BLOCKS x 8 doubles
    double* red;        // the phase's sums (<= 8 doubles, device)
};

// Scalars of one phase, per right-hand side q (the caller's Krylov state)
struct SlabScal {
    double alpha[3], beta[3], omega[3];
    int flags[3];
};
enum { SF_RUN = 1, SF_FRESH = 2, SF_TRUE = 4 };

enum SlabPhase {
    // BiCGStab
    SB_INIT = 0,   // x = 0, r = rp = b, D^-1;                       sums (b, b)
    SB_P = 1,      // p = r + beta (p - omega v) (fresh: p = rp = r), ph = D^-1 p
    SB_V = 2,      // v = A ph;                                     sums (rp, v)
    SB_S = 3,      // sh = D^-1 (r - alpha v)
    SB_T = 4,      // t = A sh;                                     sums (t, s), (t, t)
    SB_X = 5,      // x += alpha ph + omega sh, r = s - omega t;    sums (r, rp), (r, r)
    SB_TRUE = 6,   // r = b - A x where flagged;                    sums (r, r)
    // CG (one right-hand side)
    SC_INIT = 10,     // x = 0, r = b, D^-1, ph = D^-1 r, s = p = 0
    SC_W = 11,        // w = A ph;                                  sums (r, ph), (w, ph), (r, r)
    SC_UPD = 12,      // s = w + beta s, p = ph + beta p, x += alpha p, r -= alpha s, ph = D^-1 r
    SC_TRUE = 13,     // r = b - A x;                               sums (r, r)
    SC_RESTART = 14,  // ph = D^-1 r, s = p = 0
    // mean projection of a singular (all-Neumann) system
    SS_SUM_B = 20,    // sums (b)
    SS_SUB_B = 21,    // b -= alpha[0] on the owned cells
    SS_SUM_X = 22,    // sums (x)
    SS_SUB_X = 23,    // x -= alpha[0] on the owned cells and the halo planes
};

constexpr int SLAB_MAX_BLOCKS = 1184;   // 8 blocks per SM on 148 SMs

// Runs one phase on the handle's stream; returns the number of sums written to k.red (0 for
// a phase that reduces nothing), or -1 with the error set.
int slab_ksp_phase(const Op7& A, int nr, int phase, const SlabKsp& k, const SlabScal& s, cudaStream_t st);
int slab_ksp_phase(const OpSym& A, int nr, int phase, const SlabKsp& k, const SlabScal& s, cudaStream_t st);

}  // namespace cb
