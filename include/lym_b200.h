/*
 * lym_b200.h -- C ABI of the B200 (sm_100a) Wilson / Wilson-clover operator and
 * Krylov-solver library.  Drop-in boundary for LeonardYM's fermion hot path.
 *
 * Plain C: opaque context, plain pointers and sizes, no CUDA or torch types.
 * Every entry point returns an int status: 0 success, 1 solver not converged,
 * < 0 error (see lym_status); lym_last_error() gives the message.  No entry point
 * calls exit().  One CUDA stream per context; calls on one context are
 * serialised by a mutex (thread safe per context).
 *
 * Host vectors use the reference's raw memory layout (Lattice<T,LocalLayout>::
 * getRawData(), MPILattice/Lattice.h:228-234; LatticeDefinitions.h:86-161):
 *   spinor  reduced_dirac_vector_t : double[V][4 spin][3 colour][re,im]
 *   links   extended_fermion_lattice_t : per site 4 links, Eigen column-major,
 *           complex double[3][3] (SU(3) fundamental) or double[3][3] (SU(2) adjoint)
 *   site    t + Lt*(z + Lz*(y + Ly*x))            (MPILattice/LocalLayout.h:149-163)
 * "_device" variants take device pointers with the same layout.  The context's stream does
 * not wait for other streams: device inputs must be fully written before the call (for
 * example, synchronise the stream that produced them); every call has finished with its
 * device outputs when it returns.
 */
#ifndef LYM_B200_H
#define LYM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lym_context lym_context;

enum lym_status {
    LYM_OK = 0,
    LYM_NOT_CONVERGED = 1,
    LYM_ERR_ARGUMENT = -1,
    LYM_ERR_CUDA = -2,
    LYM_ERR_MEMORY = -3,
    LYM_ERR_UNSUPPORTED = -4,
    LYM_ERR_BREAKDOWN = -5,
    LYM_ERR_NOT_FOUND = -6,
    LYM_ERR_TIMEOUT = -7,
    LYM_ERR_NUMERIC = -8
};

/* Representations: the compile-time NUMCOLORS / ADJOINT choices of the reference
 * (MatrixTypedef.h:73-90) become a run-time choice. */
enum lym_rep {
    LYM_REP_SU3_FUNDAMENTAL = 0,  /* NUMCOLORS=3: FermionicGroup = complex 3x3 */
    LYM_REP_SU2_ADJOINT = 1       /* NUMCOLORS=2 -DADJOINT: FermionicGroup = real 3x3 */
};

/* Operator kinds: the names DiracOperator::getInstance registers
 * (dirac_operators/DiracOperator.cpp:20-165) and the even-odd operator. */
enum lym_operator_kind {
    LYM_OP_DIRAC_WILSON = 0,            /* DiracWilsonOperator                      */
    LYM_OP_IMPROVED = 1,                /* ImprovedDiracWilsonOperator              */
    LYM_OP_EVEN_ODD_IMPROVED = 2,       /* EvenOddImprovedDiracWilsonOperator       */
    LYM_OP_SQUARE_DIRAC_WILSON = 3,     /* SquareDiracWilsonOperator                */
    LYM_OP_SQUARE_IMPROVED = 4,         /* SquareImprovedDiracWilsonOperator        */
    LYM_OP_SQUARE_EVEN_ODD_IMPROVED = 5 /* SquareEvenOddImprovedDiracWilsonOperator */
};

enum lym_boundary {
    LYM_BC_PERIODIC = 0,           /* "fermion_periodic"     */
    LYM_BC_ANTIPERIODIC = 1        /* "fermion_antiperiodic" (LatticeBoundaryConditions.h:8-14) */
};

enum lym_solver {
    LYM_SOLVER_CG = 0,               /* ConjugateGradient::solve (inverters/ConjugateGradient.cpp:10-74)   */
    LYM_SOLVER_BICGSTAB = 1,         /* BiConjugateGradient::solve (inverters/BiConjugateGradient.cpp:321-507) */
    LYM_SOLVER_EO_BICGSTAB = 2,      /* PreconditionedBiCGStab::solve (inverters/PreconditionedBiCGStab.cpp:33-100) */
    LYM_SOLVER_EO_CG = 3,            /* even-odd Schur CG on (g5 S)^2, D x = b, FP64 throughout          */
    LYM_SOLVER_EO_CG_MIXED_SINGLE = 4, /* same, FP32 stencil inner iterations, FP64 reliable updates     */
    LYM_SOLVER_EO_CG_MIXED_HALF = 5,   /* same, FP16 spinor storage (per-site norm) inner iterations     */
    /* BiCGStab (inverters/BiConjugateGradient.cpp:321-507) on the even-odd Schur operator S
     * itself (not squared): D x = b, FP32 or FP16 inner iterations, FP64 reliable updates that
     * restart from the true residual; no initial guess */
    LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE = 6,
    LYM_SOLVER_EO_BICGSTAB_MIXED_HALF = 7
};

enum lym_multishift_solver {
    LYM_MULTISHIFT_ME = 0,    /* "mass_estrapolation": MEMultishiftSolver (inverters/MEMultishiftSolver.cpp:10-143) */
    LYM_MULTISHIFT_MMMR = 1,  /* "minimal_residual": MMMRMultishiftSolver (inverters/MMMRMultishiftSolver.cpp:42-198) */
    LYM_MULTISHIFT_CG = 2,    /* multishift CG (no reference counterpart; a new MultishiftSolver subclass) */
    /* "chronological_mass_estrapolation": ChronologicalMultishiftSolver
     * (inverters/ChronologicalMultishiftSolver.cpp:11-194); solutions[i], i >= 1, hold the
     * chronological guess of shift i on entry (zeros for none) */
    LYM_MULTISHIFT_CHRONOLOGICAL = 3,
    /* multishift CG for RHMC (no reference counterpart) on the squared even-odd operator with
     * gamma5 (SquareEvenOddImprovedDiracWilsonOperator, the operator of
     * actions/NFlavorFermionAction.cpp:76-96): FP32 / FP16-with-norms directions and operator,
     * FP32 residual and solution accumulators, FP64 shift recurrences, inner products and
     * reliable updates of the base system, then mixed-precision CG per shift until every
     * |b - (A + shifts[i]) x_i|^2 < precision in FP64 (stats->true_residual: the largest,
     * relative to |b|; stats->steps: iterations of the shared Krylov space, stats->iterations:
     * those plus the per-shift refinement; max_steps bounds the sum); other operator kinds:
     * LYM_ERR_UNSUPPORTED */
    LYM_MULTISHIFT_CG_MIXED_SINGLE = 4,
    LYM_MULTISHIFT_CG_MIXED_HALF = 5
};

typedef struct {
    int steps;             /* Solver::getLastSteps semantics (inverters/Solver.h:53-55)          */
    int iterations;        /* operator applications of the Krylov recursion                        */
    int reliable_updates;  /* FP64 residual recomputations (mixed precision)                       */
    int converged;
    double last_error;     /* Solver::getLastError semantics: last squared residual of the recursion */
    double true_residual;  /* ||b - A x|| / ||b|| recomputed in FP64 after the solve                */
    double seconds;        /* device time of the solve                                             */
} lym_solve_stats;

/* ---- context: one lattice geometry and representation on one GPU --------------
 * Replaces the process-global LocalLayout::initialize (MPILattice/LocalLayout.h:34-110). */
int lym_context_create(const int dims[4], int rep, int device, lym_context **ctx);
void lym_context_destroy(lym_context *ctx);
const char *lym_last_error(lym_context *ctx);
int lym_context_volume(lym_context *ctx);
/* bytes of device memory held by the context (gauge fields, clover terms, work vectors,
 * and the idle cached buffers below) */
size_t lym_context_device_bytes(lym_context *ctx);
/* Frees the context's cache of idle work spinors, host-transfer staging buffers and the
 * per-call buffers of the block solves (batch vectors, staging rings, scratch), which are kept
 * for the next call of the same size; they are allocated again when needed.  A device
 * allocation that fails trims the cache and retries once by itself. */
int lym_context_trim(lym_context *ctx);
int lym_synchronize(lym_context *ctx);

/* ---- gauge fields, resident by id ----------------------------------------------
 * lym_gauge_upload takes the fermion link field exactly as
 * DiracOperator::setLattice(const extended_fermion_lattice_t&) receives it
 * (dirac_operators/DiracOperator.h:125, DiracOperator.cpp:332-334).
 * lym_gauge_upload_fundamental builds the fermion links from fundamental gauge links
 * as Environment::synchronize does (Environment.cpp:21-79): adjoint map for SU(2)
 * (utils/ConvertLattice.h:24-34) and the boundary condition folded into U_t. */
int lym_gauge_upload(lym_context *ctx, int gauge_id, const double *fermion_links);
int lym_gauge_upload_device(lym_context *ctx, int gauge_id, const double *fermion_links_device);
int lym_gauge_upload_fundamental(lym_context *ctx, int gauge_id, const double *gauge_links, int boundary);
int lym_gauge_evict(lym_context *ctx, int gauge_id);

/* ---- operators ------------------------------------------------------------------
 * DiracOperator::getInstance(name, power, ...) + setKappa/setCSW/setGamma5/setLattice
 * (DiracOperator.cpp:20-165, DiracOperator.h:107-127, ImprovedDiracWilsonOperator.h:34-35).
 * The clover term F (ImprovedDiracWilsonOperator.cpp:502-523) and the even-even
 * inverse (EvenOddImprovedDiracWilsonOperator.cpp:285-317) are built on the GPU in
 * FP64 when first needed. */
int lym_operator_create(lym_context *ctx, int gauge_id, int kind, double kappa, double csw, int gamma5, int *op_id);
int lym_operator_set_gamma5(lym_context *ctx, int op_id, int gamma5);
int lym_operator_set_kappa(lym_context *ctx, int op_id, double kappa);
int lym_operator_set_csw(lym_context *ctx, int op_id, double csw);
int lym_operator_set_gauge(lym_context *ctx, int op_id, int gauge_id);
int lym_operator_destroy(lym_context *ctx, int op_id);

/* ---- operator application -------------------------------------------------------
 * DiracOperator::multiply(output, input) (DiracOperator.h:90) and
 * multiplyAdd(output, v1, v2, alpha) = Op v1 + alpha v2 (DiracOperator.h:99).
 * EvenOddImprovedDiracWilsonOperator::multiplyAdd is not implemented in the
 * reference (EvenOddImprovedDiracWilsonOperator.cpp:49-52): LYM_ERR_UNSUPPORTED. */
int lym_multiply(lym_context *ctx, int op_id, double *out, const double *in);
int lym_multiply_add(lym_context *ctx, int op_id, double *out, const double *v1, const double *v2, double alpha_re,
                     double alpha_im);
int lym_multiply_device(lym_context *ctx, int op_id, double *out, const double *in);
int lym_multiply_add_device(lym_context *ctx, int op_id, double *out, const double *v1, const double *v2,
                            double alpha_re, double alpha_im);
/* No counterpart in the reference.  Applies an EvenOddImproved operator like
 * lym_multiply_device, but allocates no device memory: for callers that cannot call
 * cudaMalloc, such as a process whose device memory all belongs to one pre-reserved arena
 * or framework allocator, or a hot path that must not take the device-wide
 * synchronisation of cudaMalloc / cudaFree.  `in` and `out` are caller-owned device
 * vectors in the reference layout and must not overlap.  The operator's one intermediate
 * vector (the even-site half spinor) lives in a fixed 12 MiB array inside the library,
 * held by every GPU that loads it until exit, which limits the lattice to 131072 sites
 * (for example 16^3 x 32); larger lattices get LYM_ERR_ARGUMENT.  The clover term must
 * have been built by an earlier ordinary use of the operator (lym_multiply /
 * lym_multiply_device), else LYM_ERR_ARGUMENT.  The first call on a device looks up the
 * array's device address, so make that call before any stream capture.  All calls share
 * the array (it keeps the last call's contents; nothing in it needs clearing): calls that
 * overlap on the GPU, from several contexts on one device, race.  Returns after the result
 * is complete. */
int lym_multiply_device_noalloc(lym_context *ctx, int op_id, double *out, const double *in);
/* storage precision of the single-precision / half-precision operator path, for
 * parity tests of the sloppy stencils: prec 0 FP64, 1 FP32 (12-real links), 2 FP16 */
int lym_multiply_precision(lym_context *ctx, int op_id, int prec, double *out, const double *in);

/* field strength F_{mu nu} of an operator's gauge field, reference layout
 * (reduced_field_strength_lattice_t: V x 6 x 3x3 complex column-major) */
int lym_field_strength(lym_context *ctx, int op_id, double *F);

/* ---- solvers ---------------------------------------------------------------------
 * Solver::solve(DiracOperator*, source, solution, guess) -> bool (inverters/Solver.h:13).
 * `precision` is the reference's absolute threshold on the squared residual norm
 * (ConjugateGradient.cpp:50, BiConjugateGradient.cpp:489).  For the even-odd CG
 * solvers, `precision` <= 0 selects the relative criterion ||b - D x|| <= `tol` ||b||
 * with tol = -precision (0 -> 1e-10). guess may be NULL. */
int lym_solve(lym_context *ctx, int op_id, int solver, double precision, int max_steps, const double *source,
              double *solution, const double *guess, lym_solve_stats *stats);
int lym_solve_device(lym_context *ctx, int op_id, int solver, double precision, int max_steps, const double *source,
                     double *solution, const double *guess, lym_solve_stats *stats);
/* BiConjugateGradient::solve(dirac, source, solution, shift, guess): (A + shift) x = b
 * (BiConjugateGradient.cpp:510-690) */
int lym_solve_shifted(lym_context *ctx, int op_id, double shift_re, double shift_im, double precision, int max_steps,
                      const double *source, double *solution, const double *guess, lym_solve_stats *stats);
/* BiCGStab(l): BiConjugateGradient::solve(dirac, source, solution, int l, guess)
 * (inverters/BiConjugateGradient.cpp:130-317), FP64, 1 <= l <= 16 */
int lym_solve_bicgstab_l(lym_context *ctx, int op_id, int l, double precision, int max_steps, const double *source,
                         double *solution, const double *guess, lym_solve_stats *stats);
/* BiCGStab with a preconditioner operator: BiConjugateGradient::solve(dirac, source,
 * solution, preconditioner, guess) (inverters/BiConjugateGradient.cpp:11-128), FP64, with the
 * reference's steps as they are (t = A s, convergence only after step 5: its result solves
 * A x = b only where the preconditioner commutes with that choice, e.g. P = 1) */
int lym_solve_preconditioned(lym_context *ctx, int op_id, int preconditioner_op_id, double precision,
                             int max_steps, const double *source, double *solution, const double *guess,
                             lym_solve_stats *stats);

/* ---- many right-hand sides (no reference counterpart: the reference solves point and
 * noise sources one by one, correlators/MesonCorrelator.cpp:92-98,
 * fermion_measurements/ChiralCondensate.cpp:86-105) ----------------------------------
 * Solves D x_j = b_j for nrhs sources with the mixed-precision even-odd CG
 * (LYM_SOLVER_EO_CG_MIXED_SINGLE or _HALF) or BiCGStab (LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE
 * or _HALF), `batch` right-hand sides at a time (a power of two <= 32, at least 2; 0 selects
 * 16) through one batched stencil: links and clover are read once
 * per site for the whole batch.  Each right-hand side keeps its own scalars, convergence
 * mask and FP64 reliable updates, so its result does not depend on its batch mates beyond
 * rounding.  stats (nrhs entries) may be NULL. */
int lym_solve_block(lym_context *ctx, int op_id, int solver, double precision, int max_steps, int nrhs,
                    const double *const *sources, double *const *solutions, int batch, lym_solve_stats *stats);
int lym_solve_block_device(lym_context *ctx, int op_id, int solver, double precision, int max_steps, int nrhs,
                           const double *const *sources, double *const *solutions, int batch,
                           lym_solve_stats *stats);

/* ---- multishift -------------------------------------------------------------------
 * MultishiftSolver::solve(dirac, source, solutions, shifts) -> bool
 * (inverters/MultishiftSolver.h:28); the operator must be Hermitian positive
 * definite (a Square* kind).  solutions[i] receives (A + shifts[i])^{-1} source. */
int lym_multishift(lym_context *ctx, int op_id, int algorithm, int nshift, const double *shifts, double precision,
                   int max_steps, const double *source, double **solutions, lym_solve_stats *stats);
int lym_multishift_device(lym_context *ctx, int op_id, int algorithm, int nshift, const double *shifts,
                          double precision, int max_steps, const double *source, double **solutions,
                          lym_solve_stats *stats);

/* ---- RHMC consumers of the multishift (dirac_functions/RationalApproximation.cpp,
 * actions/NFlavorFermionAction.cpp) -----------------------------------------------------
 * RationalApproximation::evaluate(dirac, output, input) (RationalApproximation.cpp:18-42):
 * output = sum_i alphas[i] (A + betas[i])^{-1} input with the multishift `algorithm` (a
 * lym_multishift_solver value; precision and max_steps as the approximation's
 * setPrecision / setMaximumRecursion), solutions and their combination on the device. */
int lym_rational_evaluate(lym_context *ctx, int op_id, int algorithm, int n, const double *alphas,
                          const double *betas, double precision, int max_steps, const double *input,
                          double *output, lym_solve_stats *stats);
int lym_rational_evaluate_device(lym_context *ctx, int op_id, int algorithm, int n, const double *alphas,
                                 const double *betas, double precision, int max_steps, const double *input,
                                 double *output, lym_solve_stats *stats);
/* The solves of NFlavorFermionAction::updateForce (NFlavorFermionAction.cpp:76-96) for one
 * pseudofermion phi: x[i] = (A + betas[i])^{-1} phi with the multishift on square_op_id, then
 * y[i] = D x[i] with dirac_op_id (DiracOperator::multiply); both operators on one gauge field.
 * x[i], y[i]: n caller buffers of full spinors (device pointers for the _device form). */
int lym_rhmc_force_solves(lym_context *ctx, int square_op_id, int dirac_op_id, int algorithm, int n,
                          const double *betas, double precision, int max_steps, const double *phi, double **x,
                          double **y, lym_solve_stats *stats);
int lym_rhmc_force_solves_device(lym_context *ctx, int square_op_id, int dirac_op_id, int algorithm, int n,
                                 const double *betas, double precision, int max_steps, const double *phi,
                                 double **x, double **y, lym_solve_stats *stats);

/* FermionForce::derivative (hmc_forces/FermionForce.cpp:11-20) for the operator op_id:
 * force[x][mu] -= weight * F_mu(x), F the per-link matrix of ImprovedFermionForce
 * (hmc_forces/ImprovedFermionForce.cpp:11-223: the clover-leaf terms / 4 plus the Wilson part;
 * the kinds with a clover term, at the operator's kappa and c_sw) or DiracWilsonFermionForce
 * (hmc_forces/DiracWilsonFermionForce.cpp:10-53; DiracWilson kinds), from the spinors X, Y
 * (NFlavorFermionAction's x_i and y_i = D x_i) on the operator's gauge field.  force: the
 * fermion force field in the reference's layout, double[V][4][3][3][2] (complex 3x3 matrices,
 * column-major), read and updated in place.  _device: device pointers. */
int lym_fermion_force(lym_context *ctx, int op_id, const double *X, const double *Y, double weight, double *force);
int lym_fermion_force_device(lym_context *ctx, int op_id, const double *X, const double *Y, double weight,
                             double *force);
/* The same for n pairs at once, force -= sum_i weights[i] F(X[i], Y[i]) (NFlavorFermionAction's
 * sum over the shifts, NFlavorFermionAction.cpp:53-75): the link products of each clover leaf
 * are formed once for all pairs. */
int lym_fermion_force_multi(lym_context *ctx, int op_id, int n, const double *const *X, const double *const *Y,
                            const double *weights, double *force);
int lym_fermion_force_multi_device(lym_context *ctx, int op_id, int n, const double *const *X,
                                   const double *const *Y, const double *weights, double *force);

/* ---- propagator consumers (correlators/MesonCorrelator.cpp,
 * fermion_measurements/ChiralCondensate.cpp) ---------------------------------------------
 * The connected contractions of MesonCorrelator::execute (MesonCorrelator.cpp:98-157) of
 * the 12 point-source propagators (propagators[c * 4 + alpha]: the solution of D x = b for
 * the source of spin alpha and colour c at the origin, StochasticEstimator.cpp:100-112), in
 * the reference's layout: per time slice t the summator results pion[t], scalar[t], ps[t]
 * (Lt doubles each; the reference's output multiplies them by 4 kappa^2, :163).  Both
 * representations have 3 colour components.  _device: device pointers. */
int lym_meson_contractions(lym_context *ctx, const double *const *propagators, double *pion, double *scalar,
                           double *ps);
int lym_meson_contractions_device(lym_context *ctx, const double *const *propagators, double *pion,
                                  double *scalar, double *ps);
/* out[2k], out[2k+1] = <a[k], b[k]> (gamma5 = 0, AlgebraUtils::dot, AlgebraUtils.h:17-27) or
 * <a[k], gamma5 b[k]> (gamma5 = 1, AlgebraUtils::gamma5dot, :219-238) for n pairs of full
 * spinors in device memory (the dot products of ChiralCondensate::execute, :92-105); out on
 * the host. */
int lym_dots_device(lym_context *ctx, int n, const double *const *a, const double *const *b, int gamma5,
                    double *out);
/* Real Z2 noise (StochasticEstimator::generateRandomNoise, StochasticEstimator.h:16-31: every
 * spin-colour component +-1) from a counter-based generator instead of the reference's
 * time-seeded one: component j of vector `stream` is +1 when the top bit of
 * splitmix64(seed + 0x9E3779B97F4A7C15 (stream 12 V + j + 1)) is set, else -1.  out: a full
 * AoS spinor in device memory. */
int lym_noise_z2_device(lym_context *ctx, unsigned long long seed, unsigned long long stream, double *out);
/* MesonCorrelator::execute (MesonCorrelator.cpp:22-157) for the operator op_id (a
 * DiracWilson / Improved kind, gamma5 off as the reference sets it): the 12 point sources
 * solved with the block solver `solver` (lym_solve_block's solvers, precision and batch as
 * there), then lym_meson_contractions; stats: 12 entries or NULL.  Without the reference's
 * stout smearing, source shift and stochastic disconnected part. */
int lym_meson_correlator(lym_context *ctx, int op_id, int solver, double precision, int max_steps, int batch,
                         double *pion, double *scalar, double *ps, lym_solve_stats *stats);
/* ChiralCondensate::execute (ChiralCondensate.cpp:84-118) for n stochastic estimators:
 * eta_k = lym_noise_z2_device(seed, k), x_k = D^-1 eta_k and with `connected` y_k = D^-1 x_k
 * (block solver `solver`); out[8k .. 8k+7] = <eta,x>/V, <eta,gamma5 x>/V, <x,x>/V,
 * <eta,y>/V as (re, im) (the last pair 0 without `connected`); stats: n (2n with
 * `connected`) entries or NULL. */
int lym_chiral_condensate(lym_context *ctx, int op_id, int solver, double precision, int max_steps, int batch,
                          int n, unsigned long long seed, int connected, double *out, lym_solve_stats *stats);

/* ---- gauge-configuration files (io/OutputSweep.cpp, starters/ReadStartGaugeConfiguration.cpp)
 * Fundamental links (nc = 3: SU(3); nc = 2: SU(2)) in the layout of lym_gauge_upload_fundamental.
 * LYM_GAUGE_LEONARD ("leonard_format", ReadStartGaugeConfiguration.cpp:51-130): the text
 * descriptor <directory><name>_<number>.descriptor.txt (extents, process grid, processes,
 * sites per process, plaquette) and one XDR file <directory><name>_<number>_<proc>.txt per
 * process (per site x y z t and U(i,j) row by row as double pairs).  LYM_GAUGE_MUENSTER
 * ("muenster_format"): SU(2) <directory>0:<number>:<name> (U^+ as float pairs plus the
 * run-parameter trailer, :131-300), SU(3) <directory><name>.config-<number> (two columns of
 * U^* as float pairs, re-orthonormalised on reading, :300-480).  Readers return
 * LYM_ERR_NOT_FOUND for a missing file and LYM_ERR_ARGUMENT for other extents or a short
 * file; plaquette (may be NULL) receives the value stored in the file.  Writers write one
 * process's files (OutputSweep.cpp:32-440); beta and kappa go into the muenster trailers.
 * Host code: usable without a GPU. */
enum lym_gauge_format { LYM_GAUGE_LEONARD = 0, LYM_GAUGE_MUENSTER = 1 };
int lym_gauge_file_read(int format, const int dims[4], int nc, const char *directory, const char *name, int number,
                        double *links, double *plaquette);
int lym_gauge_file_write(int format, const int dims[4], int nc, const double *links, const char *directory,
                         const char *name, int number, double plaquette, double beta, double kappa);
/* ReadStartGaugeConfiguration::readConfiguration then Environment::synchronize: read a file
 * of the context's extents and make its fermion links resident under gauge_id, as
 * lym_gauge_upload_fundamental with `boundary`. */
int lym_gauge_read(lym_context *ctx, int gauge_id, int format, const char *directory, const char *name, int number,
                   int boundary, double *plaquette);

/* ---- solve server (no reference counterpart: the reference has no serving mode) -------
 * Keeps gauge fields resident by key (one context, CUDA stream and worker thread per
 * field, so work on different fields overlaps on the device) and serves solve requests
 * D x_k = b_k (an Improved operator: kappa, c_sw; 1..n sources; relative tolerance on the
 * true residual) with the block mixed-precision even-odd solvers: `solver` is
 * LYM_SOLVER_EO_CG_MIXED_SINGLE / _HALF or LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE / _HALF (1 and 2
 * are accepted for the two CG solvers; with BiCGStab, a source on which it breaks down is
 * solved again with CG on the same lane).  Sources of all requests on a
 * field are continuously batched: they enter free slots of the running batch as earlier
 * ones finish, whatever their kappa.  A request's clover term is built when its first
 * source is admitted and freed with its last; a new clover term is admitted only while
 * the server's device memory stays within hbm_budget_bytes (0 = no limit).  Each field's
 * lane copies sources in and solutions out on a second thread through 4 + 4 device staging
 * buffers (one full FP64 spinor each, counted in the server's device bytes), so the copies
 * overlap the solves.  Host source / solution buffers must stay valid until
 * lym_server_wait returns for the ticket. */
typedef struct lym_server lym_server;
typedef struct {
    double latency_s;          /* submit -> last solution written                   */
    double queue_s;            /* submit -> first source admitted into a slot       */
    int nsrc;
    int max_iterations;        /* over the request's sources                        */
    double max_true_residual;  /* ||b - D x|| / ||b|| re-measured in FP64, worst source */
    int converged;
    int status;                /* lym_status of the request                         */
} lym_request_stats;
int lym_server_create(int device, size_t hbm_budget_bytes, int batch, int solver, lym_server **server);
void lym_server_destroy(lym_server *server);
const char *lym_server_last_error(lym_server *server);
size_t lym_server_device_bytes(lym_server *server);
int lym_server_add_gauge(lym_server *server, int key, const int dims[4], int rep, const double *fermion_links);
int lym_server_submit(lym_server *server, int key, double kappa, double csw, int nsrc, const double *const *sources,
                      double *const *solutions, double tol, int max_steps, long long *ticket);
int lym_server_wait(lym_server *server, long long ticket, double timeout_s, lym_request_stats *stats);
int lym_server_poll(lym_server *server, long long ticket, int *done);

/* ---- layout self-checks (no reference counterpart: test hooks for the layout) --------
 * reference-order neighbour tables sup/sdn [V][4] (LocalLayout.h:34-110, Lattice.h:201-207)
 * and the stencil's computed indices [2][V/2][9] (own site, 8 neighbour half-indices). */
int lym_neighbour_tables(lym_context *ctx, int *sup, int *sdn);
int lym_stencil_indices(lym_context *ctx, int *out);

/* ---- measurement hooks (no reference counterpart) ----------------------------------
 * kernels this context has enqueued (a CUDA-graph replay counts its kernel nodes), and
 * the device time of one stencil launch on the context's stream (CUDA events, after 3
 * warm-up launches): which 0 = odd-parity output with the clover term and xpay epilogue
 * (second half of the Schur operator), 1 = even-parity output with T_ee^-1 (first half). */
unsigned long long lym_context_kernel_launches(lym_context *ctx);
/* where the block solves of this context spent their host wall time so far (seconds, and
 * counts as doubles): out[0] iterating (graph replays of the batched loop, host waiting),
 * out[1] reliable updates and restarts of parked slots, out[2] adding sources (Schur source,
 * first true residual), out[3] collecting solutions (reconstruction, true residual,
 * download), out[4] graph replays, out[5] loop pauses, out[6] reliable updates, out[7]
 * iterations of the batched loop, out[8] the slots' iterations summed over the slots (out[8]
 * / (out[7] * batch width) is how full the batch was); n = 9 */
int lym_context_engine_stats(lym_context *ctx, double *out, int n);
int lym_time_stencil(lym_context *ctx, int op_id, int prec, int which, int iters, double *ms_per_launch);
/* the same for the batched stencil of the block solves (prec 1 or 2, batch a power of 2,
 * 2 <= batch <= 32), in the configuration the autotuner picks (tuned on first use) */
int lym_time_stencil_batch(lym_context *ctx, int op_id, int prec, int which, int batch, int iters,
                           double *ms_per_launch);

/* ---- batched stencil, one application (no reference counterpart: a test and tuning
 * hook) ---------------------------------------------------------------------------
 * out[j] = EvenOddImprovedDiracWilsonOperator::multiply(in[j]) of operator op_ids[j]
 * (EvenOddImprovedDiracWilsonOperator.cpp:26-47) for nrhs <= 32 full host spinors at
 * once, through the batched stencil with prec 1 (FP32) or 2 (FP16 + norms) storage.
 * The operators share the gauge field and the gamma5 flag; kappa and c_sw may differ. */
int lym_multiply_batch(lym_context *ctx, int prec, int nrhs, const int *op_ids, const double *const *in,
                       double *const *out);

/* ---- batched-stencil autotuner (no reference counterpart) --------------------------
 * The block solves time every traversal column and kernel variant of the batched
 * stencil on first use per (precision, batch width, clover) and keep the fastest.  A
 * column is by * bz sites of the (y, z) plane, walked x first and t fastest inside
 * (by = 0: plain half-site order, x slowest); minb selects the kernel variant: 1, 3
 * or 4 = direct loads with that register budget (minimum resident blocks per SM), 19
 * or 20 = neighbour spinors staged through shared memory by per-thread cp.async with 3
 * or 4 blocks per SM, 35 or 36 = the same staged by bulk copies completing on mbarriers
 * (FP32 batches; not timed by the autotuner), 83 or 84 = 19 or 20 reading SU(3) links in
 * all 18 reals instead of 12 reals and a sign bit.  lym_set_batch_tile forces a
 * configuration for the context (by < 0 returns to tuning); lym_get_batch_tile reports
 * the one in use (LYM_ERR_NOT_FOUND before the first tuning of that key). */
int lym_set_batch_tile(lym_context *ctx, int by, int bz, int minb);
int lym_get_batch_tile(lym_context *ctx, int prec, int batch, int has_clover, int *by, int *bz, int *minb);

/* ---- FP32 link format (the north star's optional 12- or 8-real gauge reconstruction) ----
 * The FP32 single-RHS stencils (the inner iterations of the mixed-precision solvers) read
 * SU(3) links as 12 reals (rows 0 and 1, row 2 from their cross product; the default) or
 * 8 reals (a2, a3, b1 and the phases of a1, c1; the rest from unitarity), both with the
 * sign table that keeps antiperiodic links exact.  8 reals move 256 instead of 384 link bytes
 * per half-site at the price of two sincos, two square roots and a division per link;
 * their rounding grows as |U_00| nears 1.  Applies to every gauge field of the context;
 * SU(2) adjoint links keep their 6-real format (LYM_ERR_UNSUPPORTED for 8).  The batched
 * stencil reads 12 reals. */
int lym_set_link_format(lym_context *ctx, int reals);

/* ---- fault injection on the host (no reference counterpart: a test hook) -----------
 * The next n device allocations of the context (of the server lane holding gauge field
 * `key`) report failure as a cudaMalloc that returned cudaErrorMemoryAllocation would:
 * the call that needed the memory returns LYM_ERR_MEMORY.  No device memory or kernel is
 * involved.  A server lane fails only the request whose admission met the failure. */
int lym_context_inject_alloc_failures(lym_context *ctx, int n);
int lym_server_inject_alloc_failures(lym_server *server, int key, int n);
/* The next host check of the word in which the bulk-copy variant of the batched stencil
 * (lym_set_batch_tile codes 35, 36) records a copy wait that gave up reads it as set: the
 * call that ran the variant returns LYM_ERR_TIMEOUT and the word is cleared.  The kernels
 * run as usual; only the host's reading of their status is faked. */
int lym_context_inject_copy_wait_timeout(lym_context *ctx);

/* ---- pinned host memory for callers that want fast transfers ---------------------- */
void *lym_host_alloc(size_t bytes);
void lym_host_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
