// Finite-volume kernels of one SIMPLE / PISO iteration on the device.
//
// Each kernel restates one loop of src/Solvers/Simple.cpp and keeps its operand order;
// the file is compiled with --fmad=false so results are bit-identical to the CPU
// oracle (and to the reference's own CPU arithmetic) outside the Krylov solves.
//
// B200 layout choices (the loops they replace walk cells with bounds-checked
// accessors and keep separate face arrays for every field):
//   * face values of d, h, p, p' are not stored.  The reference refreshes them
//     (zero-gradient patch copy + volume-weighted interpolation, FvScheme.tpp:12-40,
//     Field.tpp:518-558) immediately after the cell values change and reads them
//     before the cells change again, so each kernel recomputes the face value it
//     needs from the two cell values with the same formula;
//   * h = u + d grad p is not stored either: Rhie-Chow forms it per cell on the fly;
//   * only p keeps explicit boundary patches, because its patch is refreshed at the
//     end of correct() while Rhie-Chow reads it at the start of the next iteration;
//   * mass fluxes live on faces (one array per direction) and are double-buffered
//     in correct(), so that a cell can recompute its west neighbour's correction
//     instead of waiting for it.
#include "common.cuh"
#include "flow.cuh"

namespace cb {

__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }  // std::max

// volume weight of the upper neighbour's side: gE(P) = V_E / (V_E + V_P) (HexaFvmMesh.cpp:886-914)
__device__ __forceinline__ double gw(double vNb, double vP) { return vNb / (vNb + vP); }
// reference interpolation g*phi_P + (1-g)*phi_nb (FvScheme.tpp:29-36)
__device__ __forceinline__ double interp(double g, double phiP, double phiN) { return g * phiP + (1. - g) * phiN; }

// ---------------------------------------------------------------------------
// Momentum assembly: Simple::computeMomentum assembly loop (Simple.cpp:117-179) with the
// boundary folding of PrimitiveBoundaryCondition::setImplicitBoundaryCoefficients
// (PrimitiveBoundaryCondition.tpp:145-255).  Writes the 7 coefficients with dropped
// (out-of-domain) columns zeroed, the 3 right-hand sides and d = V / a_P.
// ---------------------------------------------------------------------------
template <bool UNSTEADY, int CONV, bool IB>
__global__ void __launch_bounds__(256) momentum_assemble_kernel(Geo g, Bc bc, FlowFields f, MomSys m, double rho, double mu,
                                                                double om, double dt) {
    const Lat& L = g.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    if (IB) {
        uint8_t st = f.status[c];
        if (st != ST_ACTIVE) {
            // inactive rows are identity rows with zero right-hand side; ghost rows keep
            // the diagonal written by the immersed-boundary kernel
            if (st == ST_INACTIVE) m.a[0][c] = 1.;
            for (int q = 1; q < 7; ++q) m.a[q][c] = 0.;
            m.b[c] = 0.; m.b[c + L.PS] = 0.; m.b[c + 2 * L.PS] = 0.;
            return;
        }
    }
    long long fW = L.fiI(i, j, k), fE = fW + 1;
    long long fS = L.fiJ(i, j, k), fN = fS + L.nI;
    long long fB = c, fT = c + L.nIJ;
    double FE = f.F[0][fE], FW = f.F[0][fW], FN = f.F[1][fN], FS = f.F[1][fS], FT = f.F[2][fT], FB = f.F[2][fB];
    double DE = g.D[0][fE], DW = g.D[0][fW], DN = g.D[1][fN], DS = g.D[1][fS], DT = g.D[2][fT], DB = g.D[2][fB];
    double V = g.vol[c];
    double a0P = UNSTEADY ? rho * V / dt : 0.;
    double a[7];
    if (CONV == 0) {
        a[1] = smin(FE, 0.) - mu * DE;
        a[2] = -smax(FW, 0.) - mu * DW;
        a[3] = smin(FN, 0.) - mu * DN;
        a[4] = -smax(FS, 0.) - mu * DS;
        a[5] = smin(FT, 0.) - mu * DT;
        a[6] = -smax(FB, 0.) - mu * DB;
        a[0] = (smax(FE, 0.) + mu * DE - smin(FW, 0.) + mu * DW + smax(FN, 0.) + mu * DN - smin(FS, 0.) + mu * DS
                + smax(FT, 0.) + mu * DT - smin(FB, 0.) + mu * DB + a0P) / om;
    } else {
        // implicit volume-weighted central differencing (extension; g of cell P per face,
        // zero at a boundary face as in HexaFvmMesh::computeMeshMetrics)
        double gE = i < L.nI - 1 ? gw(g.vol[c + 1], V) : 0.;
        double gW = i > 0 ? gw(g.vol[c - 1], V) : 0.;
        double gN = j < L.nJ - 1 ? gw(g.vol[c + L.nI], V) : 0.;
        double gS = j > 0 ? gw(g.vol[c - L.nI], V) : 0.;
        double gT = k < L.nK - 1 ? gw(g.vol[c + L.nIJ], V) : 0.;
        double gB = k > 0 ? gw(g.vol[c - L.nIJ], V) : 0.;
        a[1] = FE * (1. - gE) - mu * DE;
        a[2] = -FW * (1. - gW) - mu * DW;
        a[3] = FN * (1. - gN) - mu * DN;
        a[4] = -FS * (1. - gS) - mu * DS;
        a[5] = FT * (1. - gT) - mu * DT;
        a[6] = -FB * (1. - gB) - mu * DB;
        a[0] = (FE * gE + mu * DE - FW * gW + mu * DW + FN * gN + mu * DN - FS * gS + mu * DS
                + FT * gT + mu * DT - FB * gB + mu * DB + a0P) / om;
    }
    long long N = L.PS;   // plane stride of cell vectors
    double u0x = f.u0[c], u0y = f.u0[c + N], u0z = f.u0[c + 2 * N];
    double ux = f.u[c], uy = f.u[c + N], uz = f.u[c + 2 * N];
    double gpx = f.gradP[c], gpy = f.gradP[c + N], gpz = f.gradP[c + 2 * N];
    double bx = u0x * a0P, by = u0y * a0P, bz = u0z * a0P;
    double mV = -V;
    bx = bx + gpx * mV; by = by + gpy * mV; bz = bz + gpz * mV;
    double rl = (1. - om) * a[0];
    bx = bx + ux * rl; by = by + uy * rl; bz = bz + uz * rl;
    if (f.nonorth) {
        // (extension) sum_f mu (grad u)_f . c_f with volume-weighted face gradients
        const double* G = f.gradU;   // 9 planes, row-major (xx xy xz yx ...)
        auto gU = [&](long long cc_, int q) { return G[cc_ + q * N]; };
        for (int face = 0; face < 6; ++face) {
            // face tensor: interior -> g-interpolation of the two cells; boundary -> the cell's own
            int dir = face >> 1;
            bool upper = (face & 1) == 0;
            int idx = dir == 0 ? i : (dir == 1 ? j : k);
            int n = dir == 0 ? L.nI : (dir == 1 ? L.nJ : L.nK);
            long long stride = dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ);
            bool boundary = upper ? idx == n - 1 : idx == 0;
            long long fidx = dir == 0 ? (upper ? fE : fW) : (dir == 1 ? (upper ? fN : fS) : (upper ? fT : fB));
            long long nF = dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK);
            double cvx = g.cv[dir][fidx], cvy = g.cv[dir][fidx + nF], cvz = g.cv[dir][fidx + 2 * nF];
            if (!upper) { cvx = -cvx; cvy = -cvy; cvz = -cvz; }
            double T[9];
            if (boundary) {
                for (int q = 0; q < 9; ++q) T[q] = gU(c, q);
            } else {
                long long lo = upper ? c : c - stride, hi = upper ? c + stride : c;
                double gg = gw(g.vol[hi], g.vol[lo]);
                for (int q = 0; q < 9; ++q) T[q] = interp(gg, gU(lo, q), gU(hi, q));
            }
            bx = bx + (T[0] * cvx + T[1] * cvy + T[2] * cvz) * mu;
            by = by + (T[3] * cvx + T[4] * cvy + T[5] * cvz) * mu;
            bz = bz + (T[6] * cvx + T[7] * cvy + T[8] * cvz) * mu;
        }
    }
    // boundary folding, in the reference's order E, W, N, S, T, B
    if (i == L.nI - 1) {
        if (bc.uType[0] == P_FIXED) { bx = bx - bc.uRef[0][0] * a[1]; by = by - bc.uRef[0][1] * a[1]; bz = bz - bc.uRef[0][2] * a[1]; }
        else { a[0] += a[1]; a[1] = 0.; }
    }
    if (i == 0) {
        if (bc.uType[1] == P_FIXED) { bx = bx - bc.uRef[1][0] * a[2]; by = by - bc.uRef[1][1] * a[2]; bz = bz - bc.uRef[1][2] * a[2]; }
        else { a[0] += a[2]; a[2] = 0.; }
    }
    if (j == L.nJ - 1) {
        if (bc.uType[2] == P_FIXED) { bx = bx - bc.uRef[2][0] * a[3]; by = by - bc.uRef[2][1] * a[3]; bz = bz - bc.uRef[2][2] * a[3]; }
        else { a[0] += a[3]; a[3] = 0.; }
    }
    if (j == 0) {
        if (bc.uType[3] == P_FIXED) { bx = bx - bc.uRef[3][0] * a[4]; by = by - bc.uRef[3][1] * a[4]; bz = bz - bc.uRef[3][2] * a[4]; }
        else { a[0] += a[4]; a[4] = 0.; }
    }
    if (k == L.nK - 1) {
        if (bc.uType[4] == P_FIXED) { bx = bx - bc.uRef[4][0] * a[5]; by = by - bc.uRef[4][1] * a[5]; bz = bz - bc.uRef[4][2] * a[5]; }
        else { a[0] += a[5]; a[5] = 0.; }
    }
    if (k == 0) {
        if (bc.uType[5] == P_FIXED) { bx = bx - bc.uRef[5][0] * a[6]; by = by - bc.uRef[5][1] * a[6]; bz = bz - bc.uRef[5][2] * a[6]; }
        else { a[0] += a[6]; a[6] = 0.; }
    }
    m.a[0][c] = a[0];
    m.a[1][c] = i == L.nI - 1 ? 0. : a[1];
    m.a[2][c] = i == 0 ? 0. : a[2];
    m.a[3][c] = j == L.nJ - 1 ? 0. : a[3];
    m.a[4][c] = j == 0 ? 0. : a[4];
    m.a[5][c] = k == L.nK - 1 ? 0. : a[5];
    m.a[6][c] = k == 0 ? 0. : a[6];
    m.b[c] = bx; m.b[c + N] = by; m.b[c + 2 * N] = bz;
    f.d[c] = V / a[0];
}

// ---------------------------------------------------------------------------
// h = u + d grad p (Simple.cpp:198-203): active cells; ghost cells use u; inactive cells
// were never written by the reference and hold zero.
// ---------------------------------------------------------------------------
template <bool IB>
__device__ __forceinline__ void h_of(const FlowFields& f, long long N, long long c, double& hx, double& hy, double& hz) {
    if (IB) {
        uint8_t st = f.status[c];
        if (st == ST_INACTIVE) { hx = hy = hz = 0.; return; }
        if (st == ST_GHOST) { hx = f.u[c]; hy = f.u[c + N]; hz = f.u[c + 2 * N]; return; }
    }
    double dd = f.d[c];
    hx = f.u[c] + dd * f.gradP[c];
    hy = f.u[c + N] + dd * f.gradP[c + N];
    hz = f.u[c + 2 * N] + dd * f.gradP[c + 2 * N];
}

// ---------------------------------------------------------------------------
// Rhie-Chow face fluxes: Simple::rhieChowInterpolateFaces (Simple.cpp:410-449), after the
// BC refresh of u, d, h and their face interpolation (Simple.cpp:213-218).  One thread
// per cell writes the faces that cell owns: east, north, top, plus west/south/bottom on
// the low boundary.
// ---------------------------------------------------------------------------
template <bool IB>
__global__ void __launch_bounds__(256) rhie_chow_kernel(Geo g, Bc bc, FlowFields f, double rho) {
    const Lat& L = g.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    if (IB && f.status[c] == ST_INACTIVE) return;
    long long N = L.PS;   // plane stride of cell vectors
    double hPx, hPy, hPz;
    h_of<IB>(f, N, c, hPx, hPy, hPz);
    double dP = f.d[c], pP = f.p[c], VP = g.vol[c];
    // --- upper faces E, N, T
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        int n = dir == 0 ? L.nI : (dir == 1 ? L.nJ : L.nK);
        long long stride = dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ);
        long long nF = dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK);
        long long fu = dir == 0 ? L.fiI(i, j, k) + 1 : (dir == 1 ? L.fiJ(i, j, k) + L.nI : c + L.nIJ);
        int pf = 2 * dir;   // patch index of the upper face
        double hx, hy, hz, df, pN;
        if (idx < n - 1) {
            long long cn = c + stride;
            double gg = gw(g.vol[cn], VP);
            double hNx, hNy, hNz;
            h_of<IB>(f, N, cn, hNx, hNy, hNz);
            hx = hPx * gg + hNx * (1. - gg);
            hy = hPy * gg + hNy * (1. - gg);
            hz = hPz * gg + hNz * (1. - gg);
            df = interp(gg, dP, f.d[cn]);
            pN = f.p[cn];
        } else {
            if (bc.uType[pf] == P_FIXED) { hx = bc.uRef[pf][0]; hy = bc.uRef[pf][1]; hz = bc.uRef[pf][2]; }
            else { hx = hPx; hy = hPy; hz = hPz; }
            df = dP;
            long long pi = dir == 0 ? (long long)k * L.nJ + j : (dir == 1 ? (long long)k * L.nI + i : (long long)j * L.nI + i);
            pN = f.pPatch[pf][pi];
        }
        double sx = g.S[dir][fu], sy = g.S[dir][fu + nF], sz = g.S[dir][fu + 2 * nF];
        double F = hx * sx + hy * sy + hz * sz - df * (pN - pP) * g.D[dir][fu];
        f.F[dir][fu] = F * rho;
    }
    // --- lower boundary faces W, S, B
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        if (idx != 0) continue;
        long long nF = dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK);
        long long fl = dir == 0 ? L.fiI(i, j, k) : (dir == 1 ? L.fiJ(i, j, k) : c);
        int pf = 2 * dir + 1;
        double hx, hy, hz;
        if (bc.uType[pf] == P_FIXED) { hx = bc.uRef[pf][0]; hy = bc.uRef[pf][1]; hz = bc.uRef[pf][2]; }
        else { hx = hPx; hy = hPy; hz = hPz; }
        long long pi = dir == 0 ? (long long)k * L.nJ + j : (dir == 1 ? (long long)k * L.nI + i : (long long)j * L.nI + i);
        double pW = f.pPatch[pf][pi];
        // S_W = -S: dot(h, S_W) = -(dot(h, S)) exactly
        double sx = -g.S[dir][fl], sy = -g.S[dir][fl + nF], sz = -g.S[dir][fl + 2 * nF];
        double F = -(hx * sx + hy * sy + hz * sz) + dP * (pW - pP) * g.D[dir][fl];
        f.F[dir][fl] = F * rho;
    }
}

// ---------------------------------------------------------------------------
// Pressure-correction assembly: Simple::computePCorr assembly loop (Simple.cpp:230-269).
// The matrix is symmetric (a_E(P) and a_W(E) use the same face d and D), so it is kept as
// the diagonal plus the east, north and top coefficients of every cell; the west
// coefficient of a cell is the east one of its west neighbour (a_W(c) = a_E(c-1), which
// is also right on the west boundary because a_E of the last cell of a row is zero).
// A coefficient is zero on the boundary (its column is outside the domain and is dropped)
// and where neither side is an active cell.  Ghost rows are owned by the immersed-
// boundary kernel.
// ---------------------------------------------------------------------------
template <bool IB>
__global__ void __launch_bounds__(256) pcorr_assemble_kernel(Geo g, Bc bc, FlowFields f, PcSys s, double rho) {
    const Lat& L = g.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    uint8_t st = IB ? f.status[c] : (uint8_t)ST_ACTIVE;
    double dP = f.d[c], VP = g.vol[c];
    double a[7];
    long long fidx[6];
    fidx[0] = L.fiI(i, j, k) + 1; fidx[1] = fidx[0] - 1;
    fidx[2] = L.fiJ(i, j, k) + L.nI; fidx[3] = fidx[2] - L.nI;
    fidx[4] = c + L.nIJ; fidx[5] = c;
#pragma unroll
    for (int face = 0; face < 6; ++face) {
        int dir = face >> 1;
        bool upper = (face & 1) == 0;
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        int n = dir == 0 ? L.nI : (dir == 1 ? L.nJ : L.nK);
        long long stride = dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ);
        double df;
        bool boundary = upper ? idx == n - 1 : idx == 0;
        if (boundary) df = dP;
        else if (upper) df = interp(gw(g.vol[c + stride], VP), dP, f.d[c + stride]);
        else { long long cw = c - stride; df = interp(gw(VP, g.vol[cw]), f.d[cw], dP); }
        a[face + 1] = rho * df * g.D[dir][fidx[face]];
    }
    if (st == ST_ACTIVE) {
        a[0] = -(a[1] + a[2] + a[3] + a[4] + a[5] + a[6]);
        double b = f.F[0][fidx[0]] - f.F[0][fidx[1]] + f.F[1][fidx[2]] - f.F[1][fidx[3]] + f.F[2][fidx[4]] - f.F[2][fidx[5]];
        // folding with p' types (reference value 0: a FIXED face leaves b unchanged)
        if (i == L.nI - 1 && bc.pType[0] != P_FIXED) { a[0] += a[1]; }
        if (i == 0 && bc.pType[1] != P_FIXED) { a[0] += a[2]; }
        if (j == L.nJ - 1 && bc.pType[2] != P_FIXED) { a[0] += a[3]; }
        if (j == 0 && bc.pType[3] != P_FIXED) { a[0] += a[4]; }
        if (k == L.nK - 1 && bc.pType[4] != P_FIXED) { a[0] += a[5]; }
        if (k == 0 && bc.pType[5] != P_FIXED) { a[0] += a[6]; }
        s.aP[c] = a[0];
        s.b[c] = b;
    } else {
        if (st == ST_INACTIVE) s.aP[c] = 1.;
        s.b[c] = 0.;
    }
    double* up[3] = {s.aE, s.aN, s.aT};
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        int n = dir == 0 ? L.nI : (dir == 1 ? L.nJ : L.nK);
        long long stride = dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ);
        double val = 0.;
        if (idx < n - 1) {
            bool any = st == ST_ACTIVE;
            if (IB && !any) any = f.status[c + stride] == ST_ACTIVE;
            val = any ? a[2 * dir + 1] : 0.;
        }
        up[dir][c] = val;
    }
}

// ---------------------------------------------------------------------------
// Simple::correct cell loop (Simple.cpp:303-346), preceded by the p' boundary refresh,
// face interpolation and divergence-theorem gradient of computePCorr
// (Simple.cpp:295-298, FvScalarScheme.cpp:48-66).  Reads fluxes from Fin, writes every
// face to Fout (corrected where the reference corrects it, copied otherwise).
// ---------------------------------------------------------------------------
template <bool IB>
__global__ void __launch_bounds__(256) correct_kernel(Geo g, Bc bc, FlowFields f, double rho, double omp) {
    const Lat& L = g.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    long long N = L.PS;   // plane stride of cell vectors
    bool inact = IB && f.status[c] == ST_INACTIVE;
    long long fidx[6];
    fidx[0] = L.fiI(i, j, k) + 1; fidx[1] = fidx[0] - 1;
    fidx[2] = L.fiJ(i, j, k) + L.nI; fidx[3] = fidx[2] - L.nI;
    fidx[4] = c + L.nIJ; fidx[5] = c;
    if (inact) {
        for (int dir = 0; dir < 3; ++dir) {
            f.Fout[dir][fidx[2 * dir]] = f.F[dir][fidx[2 * dir]];
            int idx = dir == 0 ? i : (dir == 1 ? j : k);
            if (idx == 0) f.Fout[dir][fidx[2 * dir + 1]] = f.F[dir][fidx[2 * dir + 1]];
        }
    }
    double pcP = f.pc[c], dP = f.d[c], VP = g.vol[c];
    double gsx = 0., gsy = 0., gsz = 0.;
    double Fn[6];
#pragma unroll
    for (int face = 0; face < 6; ++face) {
        int dir = face >> 1;
        bool upper = (face & 1) == 0;
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        int n = dir == 0 ? L.nI : (dir == 1 ? L.nJ : L.nK);
        long long stride = dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ);
        long long nF = dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK);
        long long fi = fidx[face];
        bool boundary = upper ? idx == n - 1 : idx == 0;
        double pcF, df, pcNb;
        bool nbInactive = false;
        if (boundary) {
            // p' patch: zero-gradient -> the cell's own value; fixed -> 0
            pcNb = bc.pType[face] == P_FIXED ? 0. : pcP;
            pcF = pcNb;
            df = dP;
        } else if (upper) {
            long long cn = c + stride;
            double gg = gw(g.vol[cn], VP);
            pcNb = f.pc[cn];
            pcF = interp(gg, pcP, pcNb);
            df = interp(gg, dP, f.d[cn]);
        } else {
            long long cn = c - stride;
            double gg = gw(VP, g.vol[cn]);   // the west cell's gE
            pcNb = f.pc[cn];
            pcF = interp(gg, pcNb, pcP);
            df = interp(gg, f.d[cn], dP);
            if (IB) nbInactive = f.status[cn] == ST_INACTIVE;
        }
        double sx = g.S[dir][fi], sy = g.S[dir][fi + nF], sz = g.S[dir][fi + 2 * nF];
        if (!upper) { sx = -sx; sy = -sy; sz = -sz; }
        gsx = gsx + sx * pcF; gsy = gsy + sy * pcF; gsz = gsz + sz * pcF;
        if (inact) continue;   // grad p' is formed for every cell; the rest only for non-inactive cells
        double Fold = f.F[dir][fi];
        double DF = g.D[dir][fi];
        double Fnew = Fold;
        if (upper) {
            bool corr = !boundary || bc.flow[face] == F_OUTLET;
            if (corr) Fnew = Fold + -rho * df * (pcNb - pcP) * DF;
        } else if (boundary) {
            if (bc.flow[face] == F_OUTLET) Fnew = Fold + rho * df * (pcNb - pcP) * DF;
        } else {
            // the west/south/bottom neighbour corrects this face as its east face
            if (!nbInactive) Fnew = Fold + -rho * df * (pcP - pcNb) * DF;
        }
        Fn[face] = Fnew;
        if (upper || boundary) f.Fout[dir][fi] = Fnew;
    }
    double rv = 1. / VP;
    double gx = gsx * rv, gy = gsy * rv, gz = gsz * rv;
    f.gradPC[c] = gx; f.gradPC[c + N] = gy; f.gradPC[c + 2 * N] = gz;
    if (inact) return;
    f.mfc[c] = Fn[0] - Fn[1] + Fn[2] - Fn[3] + Fn[4] - Fn[5];
    f.p[c] = f.p[c] + omp * pcP;
    double md = -dP;
    f.u[c] = f.u[c] + gx * md;
    f.u[c + N] = f.u[c + N] + gy * md;
    f.u[c + 2 * N] = f.u[c + 2 * N] + gz * md;
}

// ---------------------------------------------------------------------------
// End of Simple::correct (Simple.cpp:348-355): p boundary refresh and the divergence-
// theorem gradient of p for every cell.  (u's faces and grad u feed only the
// non-orthogonal term, which the reference never activates; they are formed here only
// when that extension is on.)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) correct_post_kernel(Geo g, Bc bc, FlowFields f) {
    const Lat& L = g.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    long long N = L.PS;   // plane stride of cell vectors
    double pP = f.p[c], VP = g.vol[c];
    double sx0 = 0., sy0 = 0., sz0 = 0.;
    long long fidx[6];
    fidx[0] = L.fiI(i, j, k) + 1; fidx[1] = fidx[0] - 1;
    fidx[2] = L.fiJ(i, j, k) + L.nI; fidx[3] = fidx[2] - L.nI;
    fidx[4] = c + L.nIJ; fidx[5] = c;
#pragma unroll
    for (int face = 0; face < 6; ++face) {
        int dir = face >> 1;
        bool upper = (face & 1) == 0;
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        int n = dir == 0 ? L.nI : (dir == 1 ? L.nJ : L.nK);
        long long stride = dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ);
        long long nF = dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK);
        long long fi = fidx[face];
        bool boundary = upper ? idx == n - 1 : idx == 0;
        double pF;
        if (boundary) {
            long long pi = dir == 0 ? (long long)k * L.nJ + j : (dir == 1 ? (long long)k * L.nI + i : (long long)j * L.nI + i);
            if (bc.pType[face] == P_FIXED) pF = f.pPatch[face][pi];
            else { pF = pP; f.pPatch[face][pi] = pP; }
        } else if (upper) {
            pF = interp(gw(g.vol[c + stride], VP), pP, f.p[c + stride]);
        } else {
            long long cn = c - stride;
            pF = interp(gw(VP, g.vol[cn]), f.p[cn], pP);
        }
        double sx = g.S[dir][fi], sy = g.S[dir][fi + nF], sz = g.S[dir][fi + 2 * nF];
        if (!upper) { sx = -sx; sy = -sy; sz = -sz; }
        sx0 = sx0 + sx * pF; sy0 = sy0 + sy * pF; sz0 = sz0 + sz * pF;
    }
    double rv = 1. / VP;
    f.gradP[c] = sx0 * rv; f.gradP[c + N] = sy0 * rv; f.gradP[c + 2 * N] = sz0 * rv;
}

// grad u by the divergence theorem (FvVectorScheme.cpp:56-74) with u faces from the u
// boundary conditions; only for the non-orthogonal extension.
__global__ void __launch_bounds__(256) grad_u_kernel(Geo g, Bc bc, FlowFields f) {
    const Lat& L = g.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    long long N = L.PS;   // plane stride of cell vectors
    double VP = g.vol[c];
    double uP[3] = {f.u[c], f.u[c + N], f.u[c + 2 * N]};
    double T[9];
    for (int q = 0; q < 9; ++q) T[q] = 0.;
    long long fidx[6];
    fidx[0] = L.fiI(i, j, k) + 1; fidx[1] = fidx[0] - 1;
    fidx[2] = L.fiJ(i, j, k) + L.nI; fidx[3] = fidx[2] - L.nI;
    fidx[4] = c + L.nIJ; fidx[5] = c;
    for (int face = 0; face < 6; ++face) {
        int dir = face >> 1;
        bool upper = (face & 1) == 0;
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        int n = dir == 0 ? L.nI : (dir == 1 ? L.nJ : L.nK);
        long long stride = dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ);
        long long nF = dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK);
        long long fi = fidx[face];
        bool boundary = upper ? idx == n - 1 : idx == 0;
        double uf[3];
        if (boundary) {
            for (int q = 0; q < 3; ++q) uf[q] = bc.uType[face] == P_FIXED ? bc.uRef[face][q] : uP[q];
        } else if (upper) {
            double gg = gw(g.vol[c + stride], VP);
            for (int q = 0; q < 3; ++q) uf[q] = uP[q] * gg + f.u[c + stride + q * N] * (1. - gg);
        } else {
            long long cn = c - stride;
            double gg = gw(VP, g.vol[cn]);
            for (int q = 0; q < 3; ++q) uf[q] = f.u[cn + q * N] * gg + uP[q] * (1. - gg);
        }
        double s[3] = {g.S[dir][fi], g.S[dir][fi + nF], g.S[dir][fi + 2 * nF]};
        if (!upper) { s[0] = -s[0]; s[1] = -s[1]; s[2] = -s[2]; }
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) T[3 * r + q] = T[3 * r + q] + uf[r] * s[q];
    }
    for (int q = 0; q < 9; ++q) f.gradU[c + q * N] = T[q] / VP;
}

// ---------------------------------------------------------------------------
// Courant number (Simple.cpp:382-408): max over the cells [c0, c1) (all cells, or a slab's own).  Non-negative doubles order
// like their bit patterns, so the maximum is an atomicMax on the bits.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) courant_kernel(Geo g, FlowFields f, double dt, unsigned long long* out, long long c0,
                                                      long long c1) {
    const Lat& L = g.L;
    long long c = c0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double co = 0.;
    if (c < c1) {
        int i, j, k;
        L.ijk(c, i, j, k);
        long long N = L.PS;   // plane stride of cell vectors
        double ccx = g.cc[c], ccy = g.cc[c + N], ccz = g.cc[c + 2 * N];
        double ux = f.u[c], uy = f.u[c + N], uz = f.u[c + 2 * N];
        double acc = 0.;
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
            long long nF = dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK);
            long long fl = dir == 0 ? L.fiI(i, j, k) : (dir == 1 ? L.fiJ(i, j, k) : c);
            long long fu = fl + (dir == 0 ? 1 : (dir == 1 ? L.nI : L.nIJ));
            const double* F = g.fc[dir];
            double ex = F[fu] - ccx, ey = F[fu + nF] - ccy, ez = F[fu + 2 * nF] - ccz;
            double wx = F[fl] - ccx, wy = F[fl + nF] - ccy, wz = F[fl + 2 * nF] - ccz;
            double rx = ex - wx, ry = ey - wy, rz = ez - wz;
            double m = sqrt(rx * rx + ry * ry + rz * rz);
            double inv = 1. / m;
            double uu = fabs(ux * (inv * rx) + uy * (inv * ry) + uz * (inv * rz));
            acc = dir == 0 ? uu / m : acc + uu / m;
        }
        co = dt * acc;
    }
    // block max
    __shared__ double sm[256];
    sm[threadIdx.x] = (co > 0.) ? co : 0.;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) { double o = sm[threadIdx.x + s]; if (o > sm[threadIdx.x]) sm[threadIdx.x] = o; }
        __syncthreads();
    }
    if (threadIdx.x == 0 && sm[0] > 0.) atomicMax(out, (unsigned long long)__double_as_longlong(sm[0]));
}

// ---------------------------------------------------------------------------
// Continuity error (Simple.cpp:358-380).  The reference scans active cells in k-j-i
// order and, whenever |m| exceeds the running value, replaces the running value by
// |m| / V.  That scan is reproduced exactly: a parallel pass takes the max |m| of every
// 1024-cell chunk; one block then walks the chunks in order, skipping every chunk whose
// max cannot exceed the running value and scanning the others cell by cell.
// ---------------------------------------------------------------------------
constexpr int CONT_CHUNK = 1024;

template <bool IB>
__global__ void __launch_bounds__(1024) continuity_chunk_kernel(Lat L, const double* mfc, const uint8_t* status, double* chunkMax) {
    long long c = blockIdx.x * (long long)CONT_CHUNK + threadIdx.x;
    double v = -1.;
    if (c < L.N && (!IB || status[c] == ST_ACTIVE)) {
        double a = fabs(mfc[c]);
        v = (a == a) ? a : -1.;   // NaN never passes the reference's test
    }
    __shared__ double sm[32];
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = sm[threadIdx.x];
        for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
        if (threadIdx.x == 0) chunkMax[blockIdx.x] = v;
    }
}

__device__ __forceinline__ int block_min_int(int v, int* sm) {
    for (int off = 16; off > 0; off >>= 1) v = min(v, __shfl_down_sync(0xffffffffu, v, off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = sm[threadIdx.x];
        for (int off = 16; off > 0; off >>= 1) v = min(v, __shfl_down_sync(0xffffffffu, v, off));
        if (threadIdx.x == 0) sm[0] = v;
    }
    __syncthreads();
    int r = sm[0];
    __syncthreads();
    return r;
}

template <bool IB>
__global__ void __launch_bounds__(1024) continuity_walk_kernel(Lat L, const double* mfc, const double* vol, const uint8_t* status,
                                                               const double* chunkMax, int nChunks, double* out) {
    __shared__ int smi[32];
    __shared__ double sval;
    const int BIG = 0x7fffffff;
    double s = 0.;
    int q0 = 0;
    while (q0 < nChunks) {
        // first chunk at or after q0 whose max exceeds s
        int first = BIG;
        for (int base = q0; base < nChunks && first == BIG; base += blockDim.x) {
            int q = base + threadIdx.x;
            int cand = (q < nChunks && chunkMax[q] > s) ? q : BIG;
            first = block_min_int(cand, smi);
        }
        if (first == BIG) break;
        // scan that chunk cell by cell
        long long c0 = (long long)first * CONT_CHUNK;
        int cur = 0;
        while (true) {
            long long c = c0 + threadIdx.x;
            int cand = BIG;
            if ((int)threadIdx.x >= cur && c < L.N && (!IB || status[c] == ST_ACTIVE) && fabs(mfc[c]) > s) cand = threadIdx.x;
            int hit = block_min_int(cand, smi);
            if (hit == BIG) break;
            if (threadIdx.x == 0) sval = fabs(mfc[c0 + hit]) / vol[c0 + hit];
            __syncthreads();
            s = sval;
            __syncthreads();
            cur = hit + 1;
        }
        q0 = first + 1;
    }
    if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
int launch_momentum_assemble(const Geo& g, const Bc& bc, const FlowFields& f, const MomSys& m, const FlowParams& P, double dt,
                             cudaStream_t st) {
    const int B = 256;
    int G = grid_for(g.L.N, B);
    bool ib = f.status != nullptr;
#define MA(U, C, I) momentum_assemble_kernel<U, C, I><<<G, B, 0, st>>>(g, bc, f, m, P.rho, P.mu, P.omega_u, dt)
    if (P.unsteady) {
        if (P.convection == 0) { if (ib) MA(true, 0, true); else MA(true, 0, false); }
        else { if (ib) MA(true, 1, true); else MA(true, 1, false); }
    } else {
        if (P.convection == 0) { if (ib) MA(false, 0, true); else MA(false, 0, false); }
        else { if (ib) MA(false, 1, true); else MA(false, 1, false); }
    }
#undef MA
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_rhie_chow(const Geo& g, const Bc& bc, const FlowFields& f, const FlowParams& P, cudaStream_t st) {
    const int B = 256;
    int G = grid_for(g.L.N, B);
    if (f.status) rhie_chow_kernel<true><<<G, B, 0, st>>>(g, bc, f, P.rho);
    else rhie_chow_kernel<false><<<G, B, 0, st>>>(g, bc, f, P.rho);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_pcorr_assemble(const Geo& g, const Bc& bc, const FlowFields& f, const PcSys& s, const FlowParams& P, cudaStream_t st) {
    const int B = 256;
    int G = grid_for(g.L.N, B);
    if (f.status) pcorr_assemble_kernel<true><<<G, B, 0, st>>>(g, bc, f, s, P.rho);
    else pcorr_assemble_kernel<false><<<G, B, 0, st>>>(g, bc, f, s, P.rho);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_correct(const Geo& g, const Bc& bc, const FlowFields& f, const FlowParams& P, cudaStream_t st) {
    const int B = 256;
    int G = grid_for(g.L.N, B);
    if (f.status) correct_kernel<true><<<G, B, 0, st>>>(g, bc, f, P.rho, P.omega_p);
    else correct_kernel<false><<<G, B, 0, st>>>(g, bc, f, P.rho, P.omega_p);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_correct_post(const Geo& g, const Bc& bc, const FlowFields& f, cudaStream_t st, bool gradU) {
    const int B = 256;
    int G = grid_for(g.L.N, B);
    correct_post_kernel<<<G, B, 0, st>>>(g, bc, f);
    if (f.nonorth && gradU) grad_u_kernel<<<G, B, 0, st>>>(g, bc, f);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_grad_u(const Geo& g, const Bc& bc, const FlowFields& f, cudaStream_t st) {
    if (!f.nonorth) return 0;
    const int B = 256;
    grad_u_kernel<<<grid_for(g.L.N, B), B, 0, st>>>(g, bc, f);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_courant(const Geo& g, const FlowFields& f, double dt, unsigned long long* d_out, cudaStream_t st, long long c0,
                   long long c1) {
    CB_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st));
    if (c1 < 0) c1 = g.L.N;
    if (c1 <= c0) return 0;
    const int B = 256;
    courant_kernel<<<grid_for(c1 - c0, B), B, 0, st>>>(g, f, dt, d_out, c0, c1);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_continuity(const Lat& L, const double* mfc, const double* vol, const uint8_t* status, double* chunkMax, double* d_out,
                      cudaStream_t st) {
    int nChunks = (int)((L.N + CONT_CHUNK - 1) / CONT_CHUNK);
    if (status) {
        continuity_chunk_kernel<true><<<nChunks, CONT_CHUNK, 0, st>>>(L, mfc, status, chunkMax);
        continuity_walk_kernel<true><<<1, 1024, 0, st>>>(L, mfc, vol, status, chunkMax, nChunks, d_out);
    } else {
        continuity_chunk_kernel<false><<<nChunks, CONT_CHUNK, 0, st>>>(L, mfc, status, chunkMax);
        continuity_walk_kernel<false><<<1, 1024, 0, st>>>(L, mfc, vol, status, chunkMax, nChunks, d_out);
    }
    CB_CHECK_LAUNCH();
    return 0;
}

}  // namespace cb
