/*
 * caffe_b200.h -- C ABI of the B200 device library for CAFFE's finite-volume hot path.
 *
 * One handle holds one structured hexahedral mesh and the solver state of one
 * Simple / Piso / IbPiso instance, resident in HBM, plus one CUDA stream on which
 * every kernel of that handle runs.  All entry points return 0 on success and a
 * non-zero status otherwise; caffe_last_error() gives the message of the last
 * failure on the calling thread.  Plain pointers and sizes only: host arrays are
 * float64, i-fastest (index (k*nJ + j)*nI + i), the layout of Array3D
 * (src/DataStructures/Array3D.tpp:41-48 in the reference).
 *
 * Face order in every 6-array is east, west, north, south, top, bottom
 * (HexaFvmMesh::Direction, src/Domains/HexaFvmMesh/HexaFvmMesh.h:44).
 */
#ifndef CAFFE_B200_H
#define CAFFE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary types: FlowBoundaryConditions::Type (src/Domains/Field/FlowBoundaryConditions.h:10). */
enum caffe_flow_bc { CAFFE_INLET = 0, CAFFE_OUTLET = 1, CAFFE_WALL = 2, CAFFE_EMPTY = 3, CAFFE_ZERO_GRADIENT = 4 };
/* Solver classes: Simple (src/Solvers/Simple.h:33), Piso (Piso.h:6), IbPiso (IbPiso.h:33). */
enum caffe_solver_kind { CAFFE_SIMPLE = 0, CAFFE_PISO = 1, CAFFE_IBPISO = 2 };
/* Krylov methods.  The reference uses PETSc KSPBCGS + PCSOR (src/Math/SparseMatrix.cpp:95-100);
 * the device implements BiCGStab and CG with Jacobi preconditioning. */
enum caffe_ksp { CAFFE_KSP_BICGSTAB_SGS = 0, CAFFE_KSP_BICGSTAB_JACOBI = 1, CAFFE_KSP_CG_JACOBI = 2 };
/* Form of the pressure-correction solve: plain FP64, FP32 inner solves inside FP64
 * iterative refinement, learned preconditioner, or both. */
enum caffe_p_form { CAFFE_P_FP64 = 0, CAFFE_P_MIXED = 1, CAFFE_P_LEARNED = 2, CAFFE_P_LEARNED_MIXED = 3 };

/* Case parameters: the keys Simple / Piso / IbPiso read from case/case.info
 * (Solver.cpp:8, Simple.cpp:61-67,104-108, Piso.cpp:9, FlowBoundaryConditions.cpp:25-40,
 * IbPiso.cpp:37-38) plus the linear-solver settings the reference leaves to PETSc. */
typedef struct caffe_case {
    int kind;               /* caffe_solver_kind */
    int bc_type[6];         /* caffe_flow_bc per face */
    double ref_vec[6][3];   /* Boundaries.<face>.refVector */
    double ref_val[6];      /* Boundaries.<face>.refValue */
    double rho, mu;         /* Solver.rho, Solver.mu */
    int time_accurate;      /* Solver.timeAccurate ON (1) / OFF (0) */
    double omega_u, omega_p;/* Solver.relaxationFactorMomentum / relaxationFactorPCorr */
    int n_inner, n_pcorr;   /* Solver.numberOfInnerIterations / numberOfPressureCorrections */
    int convection;         /* 0 upwind (the reference), 1 volume-weighted central */
    int nonorth;            /* 0 off (the reference), 1 non-orthogonal diffusion correction */
    int mom_method, p_method;   /* caffe_ksp */
    double mom_rtol, p_rtol;    /* relative true-residual tolerance ||b - Ax|| / ||b|| */
    int maxit;
    double ib_radius;       /* ImmersedBoundaries.Sphere.radius */
    double ib_center[3];    /* ImmersedBoundaries.Sphere.center */
    double u_init[3];       /* uniform initial u (InitialConditions, uniform) */
    double p_init;          /* uniform initial p */
    int p_form;             /* caffe_p_form */
    /* Absolute floors of the momentum and p' solves: a solve stops once
     * ||b - A x||_2 <= max(rtol ||b||_2, atol), the convergence test of PETSc's KSP, whose
     * defaults the reference keeps (atol 1e-50, src/Math/SparseMatrix.cpp:95-105).  0 leaves
     * the relative test alone.  A right-hand side that is round-off noise (the second PISO
     * corrector of a converged first one) meets a floor at its round-off level at once. */
    double mom_atol, p_atol;
} caffe_case;

/* Per-step statistics (what Simple::displayUpdateMessage prints, Simple.cpp:93-100, plus
 * solver diagnostics). */
typedef struct caffe_step_stats {
    double continuity;      /* return value of Solver::solve: max continuity error */
    double courant;         /* max Courant number (not computed by IbPiso) */
    int mom_iters[3];       /* Krylov iterations of the last momentum solve, per component */
    int p_iters_last;       /* iterations of the last pressure-correction solve */
    int p_iters_total;      /* summed over all pressure-correction solves of the step */
    int p_solves;
    double p_res_max;       /* worst true relative residual of the step's p' solves */
    double mom_res_max;     /* worst true relative residual of the step's momentum solves */
    int status;             /* 0 ok; 1 a solve hit maxit; 2 breakdown; 3 non-finite residual */
    int fallbacks;          /* p' solves that fell back to the plain FP64 method */
    int n_ghost;            /* immersed-boundary ghost cells */
    int n_rows;             /* unknowns per system (active + ghost cells) */
    double p_ms, mom_ms, step_ms;   /* device time of the step's phases (CUDA events) */
    int cascades;           /* learned p' solves whose network stage stalled and that finished with
                             * the pyramid alone (an identity in place of the network) */
    int net_iters;          /* inner iterations of the step's learned p' solves run with the network
                             * in the preconditioner (the rest ran with the pyramid alone) */
} caffe_step_stats;

typedef struct caffe_dev caffe_dev;

/* Last error message of the calling thread (empty when none). */
const char* caffe_last_error(void);

/* Build the device state: mesh metrics from the node array, fields, matrices and solver
 * workspaces.  nodes: (nNodesK, nNodesJ, nNodesI, 3) float64 host array, i fastest.
 * Replaces HexaFvmMesh::initialize (src/Domains/HexaFvmMesh/HexaFvmMesh.cpp:51-58,
 * 615-624) followed by the Simple / Piso / IbPiso constructors (Simple.cpp:34-74,
 * Piso.cpp:3-10, IbPiso.cpp:32-39).  device: CUDA ordinal to use. */
int caffe_dev_create(const double* nodes, int nNodesI, int nNodesJ, int nNodesK,
                     const caffe_case* cs, int device, caffe_dev** out);
int caffe_dev_destroy(caffe_dev* h);

/* One call of Solver::solve(timeStep) (src/Solvers/Solver.h:20): Simple::solve
 * (Simple.cpp:78-91), Piso::solve (Piso.cpp:12-29) or IbPiso::solve (IbPiso.cpp:43-61).
 * Asynchronous on the handle's stream unless stats != NULL, in which case it waits for
 * the step and fills stats. */
int caffe_dev_solve(caffe_dev* h, double dt, caffe_step_stats* stats);

/* Run one named phase of the solver on the device (for tests and fine-grained callers):
 * "save_u0", "assemble_momentum", "solve_momentum", "momentum_post" (BCs + face
 * interpolation + Rhie-Chow), "assemble_pcorr", "solve_pcorr", "correct", "continuity",
 * "courant", "ib_field", "ib_coeffs".  Names follow Simple.h:44-51 and IbPiso.h:46-47. */
int caffe_dev_phase(caffe_dev* h, const char* name, double dt);

/* Copy a named array between host and device, synchronously.  dir bit 0 gives the
 * direction (0: device -> host, 1: host -> device); bit 1 selects the host layout of
 * multi-component arrays (0: N x components interleaved, 2: one plane of N per component).
 * So dir 0 / 1 read / write interleaved vectors, dir 2 / 3 read / write planes.  Returns the
 * element count of the array in doubles (so a call with host == NULL queries the size), or
 * -1 for an unknown name, a host buffer smaller than that count, or a write to a read-only
 * array.  Names: fields "u", "u0", "p", "pCorr", "d", "gradP", "gradPCorr", "gradU" (9
 * components; non-orthogonal correction only), "massFlow" (cell mass imbalance),
 * "massFlowI/J/K" (face fluxes), "pPatch0".."pPatch5"; systems "momA" (N x 7, read-only),
 * "momB" (N x 3), "pcA" (N x 7, read-only), "pcB"; read-only metrics "vol", "cc",
 * "SI/SJ/SK", "fcI/fcJ/fcK", "DI/DJ/DK", "cvI/cvJ/cvK"; immersed boundary (read-only)
 * "status", "ibCell", "ibCol", "ibValMom", "ibValP".
 * Field access of the reference: Field.h:53-61, HexaFvmMesh.h:66-142. */
long caffe_dev_array(caffe_dev* h, const char* name, double* host, long count, int dir);

/* Fill a copy of the last step's statistics without running anything. */
int caffe_dev_stats(caffe_dev* h, caffe_step_stats* stats);

/* The handle's CUDA stream (a cudaStream_t), so callers can order their own work and
 * events with the solver's kernels. */
void* caffe_dev_stream(caffe_dev* h);
int caffe_dev_synchronize(caffe_dev* h);
/* Run the handle's work on the caller's CUDA stream from now on (after finishing what the
 * handle's own stream holds); the caller keeps ownership of the stream and must keep it
 * alive until caffe_dev_destroy. */
int caffe_dev_set_stream(caffe_dev* h, void* stream);

/* ---- k-slab decomposition (replaces ParallelHexaFvmMesh::initializeSubDomains,
 * src/Domains/HexaFvmMesh/ParallelHexaFvmMesh.cpp:119-307, the halo exchange of
 * PrimitiveBoundaryCondition::setBoundaries for PARALLEL faces,
 * src/Domains/Field/PrimitiveBoundaryCondition.tpp:54-141, and the Parallel::sum / max
 * reductions of src/Parallel/Parallel.cpp).
 *
 * One rank owns the cell planes [k0, k1) of the global lattice.  Its handle is created by
 * caffe_dev_create on the node planes of the cells [max(k0-1, 0), min(k1+1, nK)): the owned
 * planes plus one halo plane on each side that has a neighbouring slab, with the global case
 * (its six boundary types and values) unchanged.  Every finite-volume phase then runs on the
 * slab exactly as on the whole lattice for the owned cells, provided the halo planes hold the
 * neighbours' values of the arrays the phase reads; the caller exchanges them with
 * caffe_slab_halo (through NCCL, or any transport) and runs the linear solves as distributed
 * Krylov phases (caffe_slab_ksp) whose sums it adds over the ranks.  Plain FP64 solves of
 * Simple and Piso only (no immersed boundary, no mixed or learned pressure solve). */

/* Declare the owned planes [k0, k1) in the handle's own k numbering.  From then on the handle's
 * step runs through the caffe_slab_* calls; caffe_dev_solve refuses it. */
int caffe_slab_set_owned(caffe_dev* h, int k0, int k1);

/* Copy one plane of `planes` planes of a cell array between the slab and a device buffer
 * of planes x nI*nJ doubles, on the handle's stream.  side 0: the plane below the owned
 * ones; side 1: above.  dir 0 packs the owned boundary plane into buf; dir 1 unpacks buf into
 * the halo plane.  Arrays: "u", "p", "pCorr", "d", "gradP", "gradPCorr", "gradU", and the
 * Krylov vectors "kspPh", "kspSh".  planes 0 means all of the array's.  Returns the buffer's
 * length in doubles (buf == NULL only queries it), -1 on error. */
long caffe_slab_halo(caffe_dev* h, const char* name, int planes, int side, int dir, double* buf);

/* One phase of a distributed Krylov solve on the owned cells (sys 0: the momentum system,
 * three right-hand sides, solution u; sys 1: the pressure correction, solution p').  Phases:
 * BiCGStab 0 init, 1 p, 2 v = A D^-1 p, 3 s, 4 t = A D^-1 s, 5 update, 6 true residual;
 * CG 10 init, 11 w = A D^-1 r, 12 update, 13 true residual, 14 restart; mean projection
 * 20 sum b, 21 b -= c, 22 sum x, 23 x -= c.  scal: 12 host doubles (alpha, beta, omega,
 * flags per right-hand side; flags 1 run, 2 fresh start, 4 true residual).  red: device
 * buffer of 8 doubles that receives this slab's sums.  Returns how many sums it wrote, -1
 * on error.  Replaces SparseMatrix::solve (src/Math/SparseMatrix.cpp:86-106) on one rank. */
int caffe_slab_ksp(caffe_dev* h, int sys, int phase, const double* scal, double* red);

/* The phases of the step that run on the slab without a reduction, asynchronously on its
 * stream: "save_u0", "assemble_momentum", "momentum_post", "assemble_pcorr", "correct"
 * (without grad u) and "grad_u" (non-orthogonal extension). */
int caffe_slab_phase(caffe_dev* h, const char* name, double dt);

/* This slab's share of a step's reductions into red[0] (device): "continuity", the
 * reference's scan over the owned cells (Simple.cpp:358-380; ranks combine by max, as its
 * Parallel::max does), or "courant", the max over the owned cells (Simple.cpp:382-408). */
int caffe_slab_reduce(caffe_dev* h, const char* what, double dt, double* red);

/* Stand-alone Krylov solve of a 7-point system on an nI x nJ x nK lattice: coef7 holds
 * 7 host arrays of N = nI*nJ*nK doubles (aP, aE, aW, aN, aS, aT, aB; a coefficient whose
 * neighbour lies outside the lattice must be zero), b and x are host arrays of N.
 * x starts from zero.  Replaces SparseMatrix::solve (src/Math/SparseMatrix.cpp:86-106),
 * which returns the iteration count. */
int caffe_ksp7_solve(int nI, int nJ, int nK, const double* coef7, const double* b, double* x,
                     int method, double rtol, int maxit, int* iters, double* rel_res);

/* Device-pointer variant of caffe_ksp7_solve for callers that keep the system in HBM:
 * d_coef7 (7*N), d_b, d_x are device pointers; stream is a cudaStream_t (NULL for the
 * legacy default stream).  Workspace is allocated per call. */
int caffe_ksp7_solve_device(int nI, int nJ, int nK, const double* d_coef7, const double* d_b, double* d_x,
                            int method, double rtol, int maxit, void* stream, int* iters, double* rel_res);

/* Krylov solve of a general sparse system of n rows in compressed-row form (host arrays: row_ptr
 * n + 1 entries from 0, col / val row_ptr[n] entries, every column in [0, n)), b and x n doubles, x
 * from zero.  Replaces SparseMatrix::solve over PETSc's AIJ matrix (src/Math/SparseMatrix.cpp:86-106)
 * for any row structure; the host layer's SparseMatrix class calls it.  Stops once
 * ||b - A x|| <= max(rtol ||b||, atol) (PETSc's rtol / atol test, on the true residual).
 * Returns 0 when converged, 1 on invalid input or a device error, 2 at maxit, 3 on a breakdown,
 * 4 on a non-finite residual (iters, rel_res and x filled for 0, 2, 3 and 4). */
int caffe_csr_solve(int n, const int* row_ptr, const int* col, const double* val, const double* b, double* x,
                    int method, double rtol, double atol, int maxit, int* iters, double* rel_res);
/* y = A x for an m x n compressed-row matrix (host arrays): MatMult behind the reference's
 * multiply(const SparseMatrix&, const SparseVector&, SparseVector&) (src/Math/SparseMatrix.cpp:132-135). */
int caffe_csr_matvec(int m, int n, const int* row_ptr, const int* col, const double* val, const double* x, double* y);

/* Scalar diffusion with unit diffusivity on one block: the reference's Diffusion solver
 * (src/Solvers/Diffusion.cpp:35-131), its coefficients as written there (a_nb = +D_f,
 * a_P = -sum D_f + V/dt, b = (V/dt) phi0).  bc_type per face (east, west, north, south, top,
 * bottom): 0 fixed, 1 zeroGradient, 2 empty (PrimitiveBoundaryCondition::Type), ref_val the
 * faces' reference values; phi starts at phi0.  caffe_diffusion_solve is Diffusion::solve: assemble,
 * Krylov solve (method / rtol / maxit as for caffe_ksp7_solve), phi and its faces and gradient,
 * and ||A x - b||_inf (its return value in the reference).  caffe_diffusion_phase runs one part:
 * "assemble", "solve" (the linear solve into x) or "post" (everything after it).
 * caffe_diffusion_array: "phi", "x" (writable), "b", "A" (N x 7: aP aE aW aN aS aT aB), "phiFaceI/J/K",
 * "phiPatch0".."phiPatch5", "gradPhi", "cc" (cell centroids) (N x 3); same conventions as caffe_dev_array. */
typedef struct caffe_diffusion caffe_diffusion;
int caffe_diffusion_create(const double* nodes, int nNodesI, int nNodesJ, int nNodesK, const int* bc_type, const double* ref_val,
                           int time_accurate, double phi0, int method, double rtol, int maxit, int device, caffe_diffusion** out);
int caffe_diffusion_destroy(caffe_diffusion* h);
int caffe_diffusion_solve(caffe_diffusion* h, double dt, double* residual_inf, int* iters, double* rel_res);
int caffe_diffusion_phase(caffe_diffusion* h, const char* name, double dt);
long caffe_diffusion_array(caffe_diffusion* h, const char* name, double* host, long count, int dir);

/* Momentum and continuity solved as one block system: the reference's Coupled solver
 * (src/Solvers/Coupled.cpp:5-339).  Unknowns u_x, u_y, u_z, p, each numbered like the cells
 * (4 N rows); momentum rows hold 14 entries, continuity rows 28.  The case fields used are
 * bc_type, ref_vec, ref_val, rho, mu, omega_u, time_accurate, n_inner, mom_method, mom_rtol,
 * mom_atol and maxit; u and p start at zero, as in the reference.  caffe_coupled_solve is
 * Coupled::solve (u0 = u, n_inner iterations of assembly, block solve and Rhie-Chow fluxes when
 * time-accurate, one otherwise) and returns the continuity error max |net face flux| / V.
 * caffe_coupled_phase runs one part: "save_u0", "assemble" ("assemble_momentum" then
 * "assemble_continuity"), "solve" (the block solve into x), "post" (u, p, grad p, h, face fluxes)
 * or "continuity".  caffe_coupled_stats gives the last block solve's iterations, true relative
 * residual and status (0 converged, 1 maxit, 2 breakdown, 3 non-finite).
 * caffe_coupled_system copies the block matrix out in compressed rows (row_ptr 4N + 1, col and
 * val nnz; any may be NULL) and returns nnz; the entries of each row are in the reference's
 * insertion order.  caffe_coupled_array: "u", "u0", "gradP", "h" (N x 3), "p", "d" (N),
 * "massFlowI/J/K" (faces), "b", "x" (4N); u, u0, p, gradP, massFlow* and x are writable. */
typedef struct caffe_coupled caffe_coupled;
int caffe_coupled_create(const double* nodes, int nNodesI, int nNodesJ, int nNodesK, const caffe_case* cs, int device,
                         caffe_coupled** out);
int caffe_coupled_destroy(caffe_coupled* h);
int caffe_coupled_solve(caffe_coupled* h, double dt, double* continuity);
int caffe_coupled_phase(caffe_coupled* h, const char* name, double dt);
int caffe_coupled_stats(caffe_coupled* h, int* iters, double* rel_res, int* status);
long long caffe_coupled_system(caffe_coupled* h, int* row_ptr, int* col, double* val);
long caffe_coupled_array(caffe_coupled* h, const char* name, double* host, long count, int dir);

/* Learned preconditioner network (an extension; the reference has no learned component):
 * a 4-layer 3-D convolutional network with 3x3x3 kernels and 16 channels, BF16 weights and
 * activations, FP32 accumulation on the tensor cores.  Parameters are FP32, layer by layer:
 * W[27 taps][16 out][16 in] then b[16]; tap = 9*(dk+1) + 3*(dj+1) + (di+1).  Layer 4 writes
 * output channel 0.  The host-data entry points below feed input channels 0 and 1; inside the
 * p' solve a third channel carries the pyramid level. */
int caffe_precond_param_count(void);
/* Apply the network to a 2-channel input x2 (host, nI*nJ*nK x 2 floats); y receives the
 * output channel (host, nI*nJ*nK floats). */
int caffe_precond_net_apply(int nI, int nJ, int nK, const float* params, const float* x2, float* y);
/* Forward plus backward: y as above and dparams = d(sum dy*y)/d(params) (host arrays). */
int caffe_precond_net_grad(int nI, int nJ, int nK, const float* params, const float* x2, const float* dy,
                           float* y, float* dparams);

/* Learned preconditioner of the p' solve (p_form CAFFE_P_LEARNED or CAFFE_P_LEARNED_MIXED):
 * an FP32 flexible Krylov solve inside FP64 refinement, preconditioned by
 *     M(r) = D^-1 r + sum_l P_l (4^l s y_l),   y_l = (net(x_l) - net(-x_l)) / 2,
 *     x_l = (R_l D^-1 r / s, active fraction, level / 8)  (the sign flips the first channel only)
 * on a pyramid of coarsened lattices (l >= 1), with one network (above) serving every level;
 * s is the RMS of D^-1 r over the active cells.
 * No counterpart in the reference: the reference solves p' with its Krylov library only
 * (src/Math/SparseMatrix.cpp:95-100).  Every solve still reaches p_rtol in the FP64 true
 * residual; the plain FP64 solve re-runs on the device when the learned one does not.
 * Parameters: caffe_precond_param_count() floats; NULL removes them (the solve then uses the
 * Jacobi part alone). */
int caffe_dev_set_precond(caffe_dev* h, const float* params);
int caffe_dev_get_precond(caffe_dev* h, float* params);
/* CAFFE_NET_JACOBI: M = D^-1 (the method without the network); CAFFE_NET_NETWORK (default);
 * CAFFE_NET_LEVELS: the pyramid with an identity in place of the network. */
enum { CAFFE_NET_JACOBI = 0, CAFFE_NET_NETWORK = 1, CAFFE_NET_LEVELS = 2 };
int caffe_dev_set_precond_mode(caffe_dev* h, int mode);
/* inner_method: 0 automatic (flexible CG for a symmetric p' matrix; with immersed-boundary
 * ghost rows, FGMRES when the network runs and BiCGStab otherwise), 1 flexible CG,
 * 2 BiCGStab (right-preconditioned; needs a fixed linear preconditioner), 3 FGMRES.
 * net_from_level: first pyramid level (>= 1) that runs the network; finer levels use the
 * identity.  restart: FGMRES cycle length, 1..64 (one cycle per FP64 refinement pass; it
 * cannot grow after the handle's first FGMRES solve). */
int caffe_dev_set_precond_options(caffe_dev* h, int inner_method, int net_from_level, int restart);
/* The pyramid levels that run the network: first_level .. last_level (last_level < 0: every
 * level from first_level down to the coarsest); the others use the identity. */
int caffe_dev_set_precond_net_levels(caffe_dev* h, int first_level, int last_level);
/* Training pairs (b, x) with A x = b, kept on the device in FP32.  record_pairs(capacity > 0)
 * stores the right-hand side and solution of every following p' solve until `capacity` pairs
 * are held, plus `snapshots` residual/correction pairs (b - A x_k, x - x_k) per solve from
 * plain re-solves truncated after k = 8, 32, 128, ... iterations; capacity 0 stops recording.
 * add_pairs uploads host pairs, arrays [n_pairs][nI*nJ*nK]; copy_pairs appends another
 * handle's pairs (same lattice and device). */
int caffe_dev_record_pairs(caffe_dev* h, int capacity, int snapshots);
int caffe_dev_pair_count(caffe_dev* h);
int caffe_dev_add_pairs(caffe_dev* h, const float* b_pairs, const float* x_pairs, int n_pairs);
int caffe_dev_copy_pairs(caffe_dev* dst, caffe_dev* src);
/* Append n_pairs synthetic pairs (A e, e) built with the handle's current p' operator: e is
 * seeded noise on pyramid level (pair mod levels), prolonged to the cell lattice, so the
 * pairs cover every scale the pyramid spans (inputs like the Krylov vectors the network
 * meets inside a solve, not only right-hand sides). */
int caffe_dev_add_random_pairs(caffe_dev* h, int n_pairs, unsigned seed);
/* Train on the handle's pairs with its current p' operator, on the device: loss per pair
 * ||M(b) - x||^2_E / ||x||^2_E in the energy norm of the (negated, positive) p' matrix, on its
 * active-cell block with an immersed body; Adam with learning rate lr, `steps` updates of
 * `batch` random pairs.  params_inout holds the starting parameters and receives the trained
 * ones; loss_hist (optional) receives the mean loss of each step.  Afterwards the handle's
 * solves use the trained parameters. */
int caffe_dev_train_precond(caffe_dev* h, int steps, int batch, float lr, unsigned seed, float* params_inout, float* loss_hist);
/* Loss of one application M(b) for every stored pair, in the given mode: loss[pair_count]. */
int caffe_dev_eval_precond(caffe_dev* h, int mode, float* loss);

/* Number of kernel launches this library has issued in this process (all handles). */
long long caffe_launch_count(void);

/* caffe_ksp7_solve_device without any device allocation.  It has no counterpart in the
 * reference.  For callers that cannot call cudaMalloc/cudaFree from inside a solve -- a program
 * whose own allocator already owns nearly all of HBM, or a time loop that cannot take the
 * device-wide synchronisation cudaFree implies -- the workspace lives in one 16 MiB __device__
 * array inside this library (held on every GPU that loads it, until exit).  Same arguments and
 * results as caffe_ksp7_solve_device (d_coef7, d_b, d_x are the caller's device arrays); lattices
 * whose workspace, 11 halo-padded planes of nI*nJ*nK + 2*ceil32(nI*nJ) doubles plus 128 KiB,
 * exceeds 16 MiB (about 180 thousand cells) are rejected with an error.  Calls share the array:
 * each clears the part it uses on entry, and calls that overlap on the GPU race.  The first call
 * on a device looks up the array's address (cudaGetSymbolAddress); make it before any stream
 * capture. */
int caffe_ksp7_solve_device_noalloc(int nI, int nJ, int nK, const double* d_coef7, const double* d_b, double* d_x,
                                    int method, double rtol, int maxit, void* stream, int* iters, double* rel_res);

#ifdef __cplusplus
}
#endif

#endif /* CAFFE_B200_H */
