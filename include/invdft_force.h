/*
 * invdft_force.h -- C ABI of the B200 force evaluation of invDFT.
 *
 * The library replaces, for one GPU, the reference's
 *   InverseDFTSolverFunction<p,pe,mem>          (include/InverseDFTSolverFunction.h:51-384)
 *   MultiVectorAdjointLinearSolverProblem<mem>  (include/MultiVectorAdjointLinearSolverProblem.h:15-214)
 * behind plain pointers and sizes.  All arithmetic on the path is FP64 by
 * default.  With INVDFT_PRECISION_MIXED the early Chebyshev passes run FP32
 * cell products until the residual reaches mixed_residual_floor, and the
 * adjoint block MINRES runs on FP32 cell products inside an FP64 iterative
 * refinement (FP64 true residuals, FP64 Lanczos scalars); Rayleigh-Ritz,
 * Cholesky, densities, transfers and the force stay FP64.
 *
 * Vectors ("multi-vectors") are row-major [n_nodes][B]: node index slowest,
 * vector index fastest, as the reference's dftfe::linearAlgebra::MultiVector
 * (MultiVectorAdjointLinearSolverProblem.cpp:638).  Every node of the mesh owns a
 * row, constrained nodes included, like the deal.II vectors of the reference.
 *
 * Entry points that take "d_" pointers expect device memory of the current
 * CUDA device; all others take host memory.  No entry point aborts: failures
 * are reported through invdft_status and invdft_last_error().
 * One context per stream; a context is not thread-safe.
 */
#ifndef INVDFT_FORCE_H
#define INVDFT_FORCE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  INVDFT_OK = 0,
  INVDFT_MAXITER = 1,    /* an iteration cap was reached (results are returned) */
  INVDFT_NONFINITE = 2,  /* NaN/Inf in an input or produced on the device */
  INVDFT_BREAKDOWN = 3,  /* Cholesky/Lanczos breakdown in the eigensolver */
  INVDFT_OOM = 4,
  INVDFT_BAD_ARG = 5,
  INVDFT_CUDA_ERROR = 6,
  INVDFT_NOT_READY = 7   /* call order violated (e.g. compute_rhs before update_psi) */
} invdft_status;

typedef enum { INVDFT_PRECISION_FP64 = 0, INVDFT_PRECISION_MIXED = 1 } invdft_precision;

typedef struct invdft_ctx invdft_ctx;

/* Constraint set in closed CSR form: node rows[r] = sum_k weights[k] * x[masters[k]]
 * for k in [ptr[r], ptr[r+1]); an empty row is a homogeneous Dirichlet node.
 * (dealii::AffineConstraints after close(); dftUtils::constraintMatrixInfo.) */
typedef struct {
  int64_t n_rows;
  const int64_t *rows;
  const int64_t *ptr;     /* n_rows + 1 */
  const int64_t *masters;
  const double *weights;
} invdft_constraints;

/* Everything InverseDFTSolverFunction::reinit receives
 * (InverseDFTSolverFunction.cpp:110-450), for one spin channel at the Gamma point. */
typedef struct {
  /* parent (wavefunction) mesh: cubic cells, order-p GLL elements, n1 = p+1 */
  int32_t p;
  int64_t n_cells;
  int64_t n_nodes;
  const int64_t *cell_nodes;   /* [n_cells][n1^3], lexicographic x fastest */
  const double *cell_h;        /* [n_cells] edge length */
  const double *gll_nodes;     /* [n1] on [0,1] */
  const double *gll_weights;   /* [n1] */
  const double *gauss_points;  /* [n1] on [0,1] */
  const double *gauss_weights; /* [n1] */
  invdft_constraints cons_psi; /* hanging + zero boundary */
  invdft_constraints cons_adj; /* hanging + rho_target < tol (InverseDFTEngine.cpp:1502-1573) */
  /* parent quadrature data, [n_cells][n1^3] */
  const double *jxw;
  const double *v_base;        /* nuclear + Hartree */
  const double *v_lda;         /* LDA v_xc of the target (scaled by factor_lda) */
  const double *rho_target_up; /* spin-up target density */
  const double *weight;        /* loss weights */
  /* child (Q1 v_xc) mesh, nested in the parent cells */
  int64_t n_child_cells;
  int64_t n_child_nodes;
  const int64_t *child_cell_nodes; /* [n_child_cells][8] */
  const double *child_jxw;         /* [n_child_cells][8] */
  invdft_constraints cons_child;   /* hanging only */
  const int64_t *child_parent;     /* [n_child_cells], non-decreasing */
  const double *child_offset;      /* [n_child_cells][3] lower corner in parent ref coords */
  const double *child_scale;       /* [n_child_cells] child size / parent size */
  const int64_t *pq_child;         /* [n_cells*n1^3] child cell of each parent quad point */
  const double *pq_xi;             /* [n_cells*n1^3][3] its coordinates in that child */
  /* physics */
  int32_t n_states;
  double n_electrons;
  double temperature;
} invdft_problem_desc;

/* Hot-path knobs (inverseDFTParameters.cpp:369-445 names in comments). */
typedef struct {
  int32_t cheb_degree;            /* CHEBYSHEV POLYNOMIAL DEGREE (0: ceil(3 sqrt(upper bound)) in [24,500]) */
  int32_t max_cheb_passes;        /* MAX CHEBYSHEV PASSES */
  double cheby_tol;               /* CHEBYSHEV FILTER TOLERANCE */
  double initial_tol_cheb;        /* INITIAL TOL FOR CHEBYSHEV FILTERING */
  double adaptive_factor_cheb;    /* ADAPTIVE FACTOR FOR CHEBYSHEV FILTERING */
  double adjoint_initial_tol;     /* INITIAL TOL FOR ADJOINT PROBLEM */
  double adaptive_factor_adjoint; /* ADAPTIVE FACTOR FOR ADJOINT */
  int32_t adjoint_max_iter;       /* MAX ITERATIONS FOR ADJOINT PROBLEM */
  double degeneracy_tol;          /* TOL FOR DEGENERACY */
  double frac_occ_tol;            /* TOL FOR FRACTIONAL OCCUPANCY */
  int32_t additional_states;      /* Solve Additional States During Cheb Filtering */
  int32_t block_size;             /* CHEBY WFC BLOCK SIZE (0 = all states) */
  int32_t inter_block_size;       /* BLOCK SIZE OF INTERPOLATE */
  double factor_lda;              /* FACTOR FOR LDA VXC */
  int32_t lanczos_steps;          /* steps of the spectrum-bound Lanczos run */
  int32_t precision;              /* invdft_precision */
  double mixed_residual_floor;    /* MIXED: filter with FP32 cell products until the max
                                     residual falls below this or stalls, then in FP64 */
  double mixed_inner_tol;         /* MIXED: relative tolerance of each FP32-operator MINRES solve
                                     inside the FP64 iterative refinement of the adjoint problem */
  int32_t mixed_max_refine;       /* MIXED: refinement steps at most (each computes the FP64 true residual) */
} invdft_params;

typedef struct {
  int32_t passes;            /* Chebyshev passes of this evaluation */
  double max_residual;       /* final max residual over the tracked states */
  double cheb_tol;
  double adjoint_tol;
  double loss;               /* sum drho^2 w JxW (InverseDFTSolverFunction.cpp:893-900) */
  double loss_unweighted;
  double l1_error;           /* sum |drho| JxW (half of int |rho - rho*|) */
  double int_rho_veff;
  double fermi_energy;
  int32_t minres_iters_max;  /* largest per-column MINRES iteration count */
  int64_t minres_iters_sum;
  int32_t n_blocks;
  int32_t n_hx_calls;        /* Hamiltonian applications issued */
  int64_t n_hx_columns;      /* sum of their block widths */
  double ms_eigen, ms_density, ms_adjoint, ms_transfer; /* device time per stage */
  /* filled when profiling is on: CUDA-event time of the cell-matrix GEMM
   * launches (the dominant kernel) and their algorithmic bytes and flops */
  int32_t n_cell_gemm;
  double ms_cell_gemm;
  double cell_gemm_bytes;
  double cell_gemm_flops;
  int64_t n_launches;        /* kernels this evaluation launched */
  int32_t degree;            /* Chebyshev filter degree used */
  double upper_bound;        /* Lanczos upper bound of the spectrum */
  double device_bytes;       /* device memory held by the library after the evaluation */
  double device_bytes_peak;  /* its high-water mark */
  int32_t passes_low;        /* Chebyshev passes filtered with FP32-stored cell matrices */
  int64_t generation;        /* state generation of the forward half this evaluation ran (see
                                invdft_force_backward_at) */
  int32_t refine_steps;      /* MIXED: FP64 refinement steps of the adjoint solves */
} invdft_force_stats;

/* Defaults of the reference's parameters. */
void invdft_default_params(invdft_params *params);

/* InverseDFTSolverFunction::reinit (InverseDFTSolverFunction.cpp:110) plus
 * MultiVectorAdjointLinearSolverProblem::reinit/computeDiagonalA
 * (MultiVectorAdjointLinearSolverProblem.cpp:476-585): uploads the problem,
 * builds the gather/scatter maps, mass and stiffness diagonals. */
invdft_status invdft_force_create(const invdft_problem_desc *desc,
                                  const invdft_params *params, invdft_ctx **ctx);
void invdft_force_destroy(invdft_ctx *ctx);
const char *invdft_last_error(const invdft_ctx *ctx);
invdft_status invdft_set_params(invdft_ctx *ctx, const invdft_params *params);

/* Record CUDA events around every cell-matrix GEMM launch of the following
 * evaluations (enable != 0) so that invdft_force_stats reports their device time. */
invdft_status invdft_set_profiling(invdft_ctx *ctx, int32_t enable);

/* Start subspace of the eigensolver (Lowdin coefficients, host [n_nodes][n_states]).
 * Without it the first evaluation starts from a fixed hash-generated block. */
invdft_status invdft_set_subspace(invdft_ctx *ctx, const double *X);

/* InverseDFTSolverFunction::getForceVector (InverseDFTSolverFunction.cpp:657-1311),
 * one spin.  pot [n_child_nodes] is distributed on entry and its constrained
 * entries are zeroed on exit (:671-676, :1295-1298); force [n_child_nodes] is
 * overwritten with its constrained entries zero (:1246); *loss receives L. */
invdft_status invdft_force_eval(invdft_ctx *ctx, double *pot, double *force,
                                double *loss, invdft_force_stats *stats);

/* InverseDFTSolverFunction::dotProduct with blockSize 1 (:1693-1705). */
invdft_status invdft_dot(invdft_ctx *ctx, const double *a, const double *b,
                         int64_t n, double *out);
/* InverseDFTSolverFunction::dotProduct (:1693-1705) with any blockSize:
 * out[j] = sum over i with i % block_size == j of a[i] b[i], accumulated in
 * entry order, out [block_size].  Host arrays. */
invdft_status invdft_dot_blocks(invdft_ctx *ctx, const double *a, const double *b,
                                int64_t n, int32_t block_size, double *out);

/* Results of the last evaluation (host copies). */
invdft_status invdft_get_eigen(invdft_ctx *ctx, double *eig, double *occ, double *fermi);
invdft_status invdft_get_psi(invdft_ctx *ctx, double *psi);           /* nodal [n_nodes][N] */
invdft_status invdft_get_density(invdft_ctx *ctx, double *rho);       /* [n_cells*n1^3] total */
invdft_status invdft_get_child_quad_products(invdft_ctx *ctx, double *S); /* [n_child_cells*8] */

/* Forward half of getForceVector: distribute v_xc, solveEigen (:1315-1477),
 * computeRhoFromPSI (:748-758), drho and the loss (:776-912); stats->loss
 * receives L.  The eigenvectors stay in the context (stored once) for
 * invdft_force_backward.  pot's constrained entries are zeroed on exit. */
invdft_status invdft_solve_eigen(invdft_ctx *ctx, double *pot, invdft_force_stats *stats);
/* Backward half of getForceVector for the last invdft_solve_eigen: the block
 * adjoint solves and the projection (:914-1246) giving force = dL/dv_xc
 * [n_child_nodes].  invdft_solve_eigen + invdft_force_backward ==
 * invdft_force_eval.  NOT_READY when no forward half ran, or when
 * invdft_set_potential changed the Hamiltonian since. */
invdft_status invdft_force_backward(invdft_ctx *ctx, double *force, invdft_force_stats *stats);
/* The same for the forward half whose stats->generation was `generation`:
 * NOT_READY when any later forward half (invdft_solve_eigen, invdft_force_eval,
 * invdft_bfgs_solve) or invdft_set_potential has changed the state since, so a
 * caller that keeps several forward results (an autograd tape) never receives
 * dL/dv_xc at another v_xc. */
invdft_status invdft_force_backward_at(invdft_ctx *ctx, int64_t generation, double *force,
                                       invdft_force_stats *stats);

/* --- building blocks, exposed for the adjoint interface and for tests --- */

/* v_KS = v_base + v_xc(child -> parent quad) + factor_lda v_lda and the cell
 * Hamiltonians (setVEff + computeCellHamiltonianMatrix, :1367-1388).  Ends the
 * validity of the last forward half for invdft_force_backward. */
invdft_status invdft_set_potential(invdft_ctx *ctx, const double *pot);

/* POST_PROCESS projection of v_xc to the parent mesh (InverseDFTEngine::
 * projectVxcToParentMesh, InverseDFTEngine.cpp:3462-3545, called from
 * interpolateVxc :3241-3248): vxc_child [n_child_nodes] (child constraints are
 * distributed first), parent_nodal [n_nodes] = lumped-mass L2 projection of
 * v_xc + factorForLDAVxc * v_LDA at the parent quadrature points, with the psi
 * constraints distributed.  Host arrays; pot and force state are untouched. */
invdft_status invdft_project_vxc_to_parent(invdft_ctx *ctx, const double *vxc_child, double *parent_nodal);

/* A parent nodal field at points (the writeToPoints branch of
 * InverseDFTEngine::interpolateVxc, InverseDFTEngine.cpp:3275-3456): point i
 * lies in parent cell cells[i] at reference coordinates xi[3i..3i+2] in
 * [0, 1]^3 (x, y, z); out[i] = sum_l parent_nodal[node(cell, l)] N_l(xi).
 * Host arrays. */
invdft_status invdft_evaluate_parent_field(invdft_ctx *ctx, const double *parent_nodal, int64_t npts,
                                           const int64_t *cells, const double *xi, double *out);

/* Lowdin HX on device blocks: d_y = M^-1/2 C^T sum_e H_e (C M^-1/2 d_x)_e
 * (KohnShamDFTBaseOperator::HXWithLowdinOrthonormalisedInput as called at
 * MultiVectorAdjointLinearSolverProblem.cpp:1353).  B in [1, 64]. */
invdft_status invdft_hx(invdft_ctx *ctx, const double *d_x, double *d_y, int32_t B);

/* MultiVectorAdjointLinearSolverProblem::updateInputPsi (:818-910).
 * d_psi [n_nodes][B] nodal, occ/eig [B] host, d_u [n_cells*n1^3] = drho * w,
 * degeneracy in CSR (deg_ptr [B+1], deg_idx), mu = Fermi energy. */
invdft_status invdft_adjoint_update_psi(invdft_ctx *ctx, const double *d_psi,
                                        const double *occ, const double *d_u,
                                        const int32_t *deg_ptr, const int32_t *deg_idx,
                                        double mu, const double *eig, int32_t B);
/* computeRhs (:616-812): d_rhs [n_nodes][B]. */
invdft_status invdft_adjoint_compute_rhs(invdft_ctx *ctx, double *d_rhs);
/* vmult (:1346-1367): d_Ax = Ht d_x - eps .* d_x; zeroes constrained rows of d_x and d_Ax. */
invdft_status invdft_adjoint_vmult(invdft_ctx *ctx, double *d_Ax, double *d_x);
/* precondition_Jacobi / precondition_JacobiSqrt (:588-612); omega is unused as in the reference. */
invdft_status invdft_adjoint_precondition_jacobi(invdft_ctx *ctx, double *d_dst,
                                                 const double *d_src, double omega);
invdft_status invdft_adjoint_precondition_jacobi_sqrt(invdft_ctx *ctx, double *d_dst,
                                                      const double *d_src, double omega);
/* distributeX (:1003-1141) on the block solution d_x (in place). */
invdft_status invdft_adjoint_distribute_x(invdft_ctx *ctx, double *d_x);
/* Block MINRES of DFT-FE's MultiVectorMinResSolver::solve as called at
 * InverseDFTSolverFunction.cpp:1106-1112 (zero start, distributeX at the end);
 * iters [B] receives per-column iteration counts. */
invdft_status invdft_adjoint_solve(invdft_ctx *ctx, double *d_x, double tol, int32_t max_iter,
                                   int32_t *iters);

/* The base potential v_base on the GPU: InverseDFTEngine::setPotBasePoissonNuclear
 * (InverseDFTEngine.cpp:2459-2571) with solvePhiTotalAllElectronNonPeriodic
 * (:2573-2621).  Solves, on the parent mesh with its psi constraints (hanging
 * nodes, zero boundary), the Poisson problem of the total electrostatic
 * potential of the density rho_quad [n_cells*n1^3] (host, total at the parent
 * quadrature points) and n_atoms point nuclei of charge Z[a] in cell
 * atom_cell[a] at reference coordinates atom_xi[3a..3a+2] in [0, 1]^3:
 *   -lap phi = 4 pi (rho - sum_a Z_a delta_a),
 * by Jacobi-preconditioned CG with the matrix-free Laplacian until the
 * residual falls below rel_tol times the right-hand side (2-norms, in the
 * Lowdin-scaled unknowns) or max_iter.  phi_quad [n_cells*n1^3] receives phi at
 * the quadrature points and phi_nodal [n_nodes] (may be NULL) the nodal
 * solution; *iters and *rel_res (may be NULL) the CG iterations and final
 * relative residual.  install != 0 makes phi_quad the context's v_base for the
 * following evaluations (and ends the validity of the last forward half).
 * MAXITER when max_iter ran out (results are returned). */
invdft_status invdft_poisson_total_potential(invdft_ctx *ctx, const double *rho_quad, int32_t n_atoms,
                                             const double *Z, const int64_t *atom_cell, const double *atom_xi,
                                             double rel_tol, int32_t max_iter, int32_t install,
                                             double *phi_quad, double *phi_nodal, int32_t *iters,
                                             double *rel_res);

/* One launch of each kernel of the evaluation on the context's full-size
 * buffers, for kernel profiles (needs invdft_set_potential first): the Lowdin
 * HX chain on the start block, the density, psi.p at the child quadrature
 * points, the force projection, the adjoint rhs chain and one MINRES update
 * pair.  Results are meaningless; ends the validity of the last forward half. */
invdft_status invdft_kernel_probe(invdft_ctx *ctx);

/* The initial v_xc guess on the GPU: InverseDFTEngine::setInitialPotL2Proj
 * (InverseDFTEngine.cpp:1046-1498).  From the total target density rho_quad
 * [n_cells*n1^3] (host, parent quadrature points) and, for LB94 exchange, its
 * |grad rho|^2 sigma_quad (NULL: LDA exchange), forms at the quadrature points
 *   v = (1 - p) v_x + p (v_x + v_c),  p = rho / (rho + tau_vx),
 * with the Fermi-Amaldi far field v = q v - (1 - q) factor_fa / N_e v_H,
 * q = rho / (rho + tau_fa), when fermi_amaldi_bc != 0 (v_H: the Hartree
 * potential of rho solved on the GPU, boundary values hartree_bc [n_nodes] on
 * the Dirichlet rows of the psi constraints, as computeHartreePotOnParentQuad
 * sets them, :1790-2118).  v is L2-projected onto the parent nodes (lumped
 * mass, psi constraints distributed), evaluated at the child Gauss points,
 * scaled by 1 - factor_lda and L2-projected onto the child nodes, whose
 * constrained entries are set to zero.  vxc_child [n_child_nodes] receives the
 * guess; vxc_parent [n_nodes] and vh_quad [n_cells*n1^3] (may be NULL) the
 * parent nodal field and v_H. */
typedef struct {
  double tau_vx;               /* TAU FOR WEIGHTS FOR SETTING VX BC (reference default 1e-2) */
  double tau_fa;               /* TAU FOR WEIGHTS FOR SETTING FABC (1e-2) */
  int32_t fermi_amaldi_bc;     /* SET FERMIAMALDI IN THE FAR FIELD AS INPUT (0) */
  double factor_fa;            /* FACTOR FOR FERMIAMALDI (1) */
  double hartree_rel_tol;      /* CG tolerance of the Hartree solve (relative residual) */
  int32_t hartree_max_iter;
} invdft_initial_guess_options;
invdft_status invdft_initial_guess(invdft_ctx *ctx, const double *rho_quad, const double *sigma_quad,
                                   const double *hartree_bc, const invdft_initial_guess_options *opts,
                                   double *vxc_child, double *vxc_parent, double *vh_quad);

/* Integer index data the library built on the device from the descriptor,
 * downloaded as int32 for exact comparison with the caller's (the reference's
 * cell->DoF maps of computeCellLocalIndexSetMap and the constraint indexing of
 * dftUtils::constraintMatrixInfo, InverseDFTSolverFunction.cpp:281-283 and
 * MultiVectorAdjointLinearSolverProblem.cpp:476-538).  `n` must equal the
 * map's length (BAD_ARG otherwise, with the length in the message).
 *   CELL_NODES   [n_cells*n1^3] node of each cell entry
 *   CELL_GATHER  [n_cells*n1^3] that node when it is free, else -(1 + r), r its
 *                row in the psi constraints (the gather of the Lowdin HX)
 *   CELL_SLOTS   [n_cells*n1^3] slot of the entry in the cell-result layout
 *                (-1: a Dirichlet row, dropped)
 *   *_ROWS/_PTR/_MASTERS  closed CSR of the psi, adjoint and child constraints
 *   CHILD_CELL_NODES [n_child_cells*8], PQ_CHILD [n_cells*n1^3] */
enum {
  INVDFT_MAP_CELL_NODES = 0, INVDFT_MAP_CELL_GATHER = 1, INVDFT_MAP_CELL_SLOTS = 2,
  INVDFT_MAP_PSI_ROWS = 3, INVDFT_MAP_PSI_PTR = 4, INVDFT_MAP_PSI_MASTERS = 5,
  INVDFT_MAP_ADJ_ROWS = 6, INVDFT_MAP_ADJ_PTR = 7, INVDFT_MAP_ADJ_MASTERS = 8,
  INVDFT_MAP_CHILD_ROWS = 9, INVDFT_MAP_CHILD_PTR = 10, INVDFT_MAP_CHILD_MASTERS = 11,
  INVDFT_MAP_CHILD_CELL_NODES = 12, INVDFT_MAP_PQ_CHILD = 13
};
invdft_status invdft_get_index_map(invdft_ctx *ctx, int32_t which, int32_t *out, int64_t n);

/* L-BFGS driver of BFGSInverseDFTSolver::solve with the CP line search
 * (BFGSInverseDFTSolver.cpp:467-627).  pot is updated in place; losses
 * [2*max_iter+1] (may be NULL) receives the loss of each force evaluation
 * (one per iteration plus one per line-search probe). */
invdft_status invdft_bfgs_solve(invdft_ctx *ctx, double *pot, int32_t max_iter, double tol,
                                int32_t line_search_iters, double line_search_tol,
                                int32_t history, double *losses, int32_t *n_evals);

/* The same L-BFGS driver with a stop on the density error, for runs to a
 * fixed int |rho - rho*| (the reference stops on the force norm and the
 * iteration cap only).  After each accepted iterate (and at the start) the run
 * stops once int |rho - rho*| = 2 stats.l1_error <= density_l1_target (0: off).
 * losses and density_l1 (may be NULL) receive, per force evaluation, L and
 * int |rho - rho*|, up to `capacity` entries. */
typedef struct {
  int32_t max_iter;
  double tol;                 /* force-norm tolerance */
  int32_t line_search_iters;
  double line_search_tol;
  int32_t history;
  double density_l1_target;
} invdft_bfgs_options;
typedef struct {
  int32_t n_iters;            /* accepted iterates */
  int32_t n_evals;            /* force evaluations, line-search probes included */
  double final_loss;
  double final_density_l1;    /* int |rho - rho*| at the last evaluation */
  int32_t reached;            /* 1 when the density target stopped the run */
} invdft_bfgs_report;
invdft_status invdft_bfgs_run(invdft_ctx *ctx, double *pot, const invdft_bfgs_options *opts, double *losses,
                              double *density_l1, int32_t capacity, invdft_bfgs_report *report);

/* Per-column dot products out[j] = sum_i a[i*B+j] b[i*B+j] of device blocks
 * [n][B], computed on `stream` (a cudaStream_t, NULL = default stream) without
 * allocating anything.  No counterpart in the reference: it serves callers that
 * must not let a library allocate device memory while they run (an outer
 * L-BFGS or Krylov driver whose vectors live in its own device pool).  Needs no
 * context.  Scratch is a static device array of 296 x 64 doubles held by every
 * GPU that loads the library, so B must be in [1, 64] (BAD_ARG otherwise, with
 * the reason in invdft_last_error(NULL)).  The library's device code is loaded
 * lazily: the first call on a device loads the module, which reserves the
 * array and the kernels' own device memory, so a caller that owns its device
 * pool makes one warm-up call on each device before handing the device to its
 * pool; later calls allocate nothing.  Every call
 * looks up the array's device address with the device current (no allocation
 * once the module is loaded), so the address stays right after a device reset.
 * Calls share the array: calls that overlap on the GPU race.  Asynchronous
 * with respect to the host; d_out [B] is device memory. */
invdft_status invdft_coldot_noalloc(const double *d_a, const double *d_b, int64_t n, int32_t B,
                                    double *d_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* INVDFT_FORCE_H */
