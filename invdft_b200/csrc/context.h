// Context of the B200 force evaluation: device-resident problem, state and
// the host orchestration mirroring InverseDFTSolverFunction and
// MultiVectorAdjointLinearSolverProblem.
#pragma once
#include <string>
#include <vector>

#include "../../include/invdft_force.h"
#include "kernels.cuh"

namespace invdft {

constexpr double C_KB = 3.166811429e-06;  // Ha/K
int auto_degree(double upper_bound);

struct Cons {                      // device copy of a closed constraint set
  int n = 0;
  DevBuf<int> rows, ptr, masters;
  DevBuf<double> w;
  std::vector<int64_t> h_rows;     // host copy of the constrained rows
  int64_t h_nnz = 0;               // master entries
  std::vector<int64_t> h_ptr, h_masters;  // host copy of the CSR
  std::vector<double> h_w;
};

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
};

class Context {
 public:
  Context(const invdft_problem_desc *d, const invdft_params *p);
  ~Context();

  invdft_params prm;
  std::string last_error;
  cudaStream_t stream = nullptr;

  // sizes
  int p = 0, n1 = 0, nd = 0, nq = 0, N = 0;
  int64_t nc = 0, nn = 0, ncc = 0, ncn = 0;
  double n_electrons = 0, temperature = 0, kT = 0;

  // parent data
  DevBuf<double> phi, Kref, cell_h, jxw, v_base, v_lda, rho_t, weight;
  DevBuf<int> cell_nodes, cell_map;
  DevBuf<int> cell_map_sf;               // the matrix-free kernel's gather map (compact constrained rows)
  DevBuf<int> cell_map_t, d_slot_of_t;   // [nd][nc] copies (narrow blocks of the matrix-free kernel)
  Cons cpsi, cadj, cchild;
  DevBuf<double> cons_gw;
  DevBuf<int> d_slot_of, d_dptr, d_err, d_zptr;
  int nhang = 0;
  int ldh = 0;
  // cell products: 3 matrix-free sum factorisation (default), 0 FP64 tensor core
  // on stored cell matrices (mma.sync f64), 1 row-stream DFMA, 2 bulk-staged DFMA
  int hx_variant = 3;
  int sf_tune = -1;                // launch shape of the matrix-free kernel (-1: autotuned per width)
  bool minres_fused = true;        // MINRES update1 + reductions + scalars, update2 + v, in two launches
  bool minres_graph = false;       // INVDFT_MINRES_GRAPH=1: fused MINRES segments replayed from CUDA graphs
  bool capturing = false;          // a CUDA graph capture is in progress (no profiling events)
  struct SegGraph {                // one captured MINRES segment
    std::vector<uintptr_t> key;    // width, precision, tolerance bits and every buffer it touches
    cudaGraphExec_t exec;
    long long launches;            // kernels per replay
  };
  std::vector<SegGraph> seg_graphs;
  void release_graphs();
  bool trace = false;              // per-pass lines of the eigensolver on stderr
  int sf_tuned[65];                // autotuned shape per block width (-1: not measured yet)
  int sf_shape(const double *d_x, int Bw);
  SfMats sfm{};                    // reference-element matrices of the matrix-free variant
  SfMatsT<float> sfm32{};          // the same in FP32 (low rungs of the precision ladder)
  SfMatsT<Tf32Operand> sfm_tf32{}; // ... with TF32- / BF16-rounded products (ladder_operands 1 / 2)
  SfMatsT<Bf16Operand> sfm_bf16{};
  int ladder_operands = 0;         // filter products of the low rungs: 0 FP32, 1 TF32 operands, 2 BF16 operands
  bool in_filter = false;          // a Chebyshev filter pass is running
  DevBuf<double> vj;               // [nc][nq] v_KS * JxW (matrix-free variant)
  DevBuf<int> d_mslot;             // [nmast] the slot of each master that holds its hanging contributions
  int64_t n_slots = 0;             // result slots of a cell product (per column)
  int n_masters = 0;
  // constraint groups (rows with identical master lists) and master pair lists
  DevBuf<int> d_g_rptr, d_g_hrow, d_g_m0, d_g_nm, d_g_poff, d_mp_ptr, d_mp_idx;
  DevBuf<double> d_gpart;          // [npairs][64] per-(group, master) partial sums
  DevBuf<int64_t> d_g_woff;        // per-group start of its weight block
  DevBuf<double> d_g_w, d_g_wt;    // distinct group weight blocks, [row][master] and [master][row]
  int n_weight_blocks = 0;
  DevBuf<double> d_hvg;            // [nhang+1][64] pre-gathered hanging rows and a zero row (matrix-free variant)
  bool needs_cell_matrices() const;
  void check_device_error();
  DevBuf<double> sqrtM, invsqrtM, diagA, diagSqrtA;
  std::vector<double> h_invsqrtM;  // host copy of M^-1/2 (0 on constrained rows)
  std::vector<char> h_free;        // unconstrained psi rows
  // child data
  DevBuf<int> ch_nodes, ch_parent, pq_child, ch_sc_ptr, ch_sc_src, work_parent, work_c0, work_c1;
  DevBuf<double> ch_jxw, ch_offset, ch_scale, pq_xi, ch_sc_w, gll, g2;
  int nwork = 0;
  FeView fe{};
  ChildView cv{};

  // eigensolver state
  DevBuf<double> H;                // [nc][nd][nd] column-major cells
  DevBuf<double> X, Yb, Zb, Wb;    // [nn][N]
  DevBuf<double> Ycell;            // [nc][nd][maxB]
  DevBuf<double> vks, rho, u, psi, S, pot_d, force_d;
  DevBuf<double> partial, small, lz_v, lz_w, lz_p;
  std::vector<double> eig, occ;
  double mu = 0.0;
  bool have_eig = false;
  bool have_H = false;
  int counter = 0;
  double tol_cheb = 1e-8, loss_prev = 0.0, adjoint_tol = 0.0;
  int nblocks_red = 1184;
  // statistics of the current evaluation
  int n_hx = 0;
  int64_t n_hx_cols = 0;
  // optional per-launch timing of the cell GEMM
  bool profile = false;
  std::vector<cudaEvent_t> ev_pool;
  int ev_used = 0;
  double prof_bytes = 0.0, prof_flops = 0.0;
  void cell_gemm(const double *d_x, int Bw, bool low = false);
  DevBuf<float> H32;               // FP32 copy of the cell matrices (mixed precision)
  bool have_H32 = false;
  void profile_begin();
  void profile_end(invdft_force_stats *st);

  // adjoint problem state (MultiVectorAdjointLinearSolverProblem)
  int B = 0;
  bool psi_ready = false;
  DevBuf<double> a_psi, a_ujxw, a_Mu, a_occ4, a_eig, a_coef, a_Q1, a_Q2;
  std::vector<double> h_occ, h_eig, h_Mu;
  double a_mu = 0.0, a_eta = 0.0;
  std::vector<int> pairs, pair_ptr, pair_j;
  DevBuf<int> d_pairs, d_pair_ptr, d_pair_j;
  // MINRES buffers
  DevBuf<double> m_r1, m_r2, m_y, m_v, m_w, m_w2, m_yn, m_b, m_x, m_p, m_xc, m_tmp;
  DevBuf<double> m_scal;           // 16 * maxB doubles
  DevBuf<int> m_flags;             // 3 * maxB ints
  DevBuf<unsigned> m_ticket;       // CTA ticket of the fused MINRES update (0 between launches)
  std::vector<int> last_iters;

  // ---- operations ----
  void set_params(const invdft_params *p);
  void set_subspace(const double *Xh);
  void hx(const double *d_x, double *d_y, int Bw);
  // POST_PROCESS: child v_xc -> parent nodal field (lumped-mass L2 projection of
  // v_xc + factor_lda v_LDA at the parent quadrature points); host arrays
  void project_vxc_to_parent(const double *h_vxc, double *h_out);
  // a parent nodal field at points (cell, reference coordinates); host arrays
  void evaluate_parent_field(const double *h_u, int64_t npts, const int64_t *h_cells, const double *h_xi,
                             double *h_out);
  DevBuf<double> pp_pot, pp_q, pp_y, pp_xi, pp_out;   // post-processing scratch
  DevBuf<int64_t> pp_cells;
  void set_potential_device(double *d_pot);   // distributes d_pot in place
  void lanczos_bounds(double &lo, double &hi);
  void chfsi_pass(double a, double b, double a0, std::vector<double> &res, bool low = false);
  void solve_eigen(double *d_pot, invdft_force_stats *st);
  void density_and_loss(double out4[4]);
  // adjoint
  void adj_update_psi(const double *d_psi_in, int64_t ld, int col0, const double *occ, const double *d_u,
                      const std::vector<std::vector<int>> &degen, double mu, const double *e, int Bw);
  void adj_mu(const std::vector<double> &occv, std::vector<double> &Mu_out);
  void adj_compute_rhs(double *d_rhs);
  void adj_vmult(double *d_Ax, double *d_x);
  void adj_precondition(double *d_dst, const double *d_src, bool sqrt_version);
  void adj_distribute_x(double *d_x);
  void adj_minres(double *d_x, double tol, int maxit, std::vector<int> &iters);
  void minres_core(const double *d_rhs, double *d_x, double tol, int maxit, std::vector<int> &iters, bool low);
  void minres_refined(const double *d_b, double *d_x, double tol, int maxit, std::vector<int> &iters);
  int refine_steps = 0;            // FP64 refinement steps of the adjoint solves of this evaluation
  // full evaluation = forward half + backward half
  void forward(double *pot, invdft_force_stats *st);
  // expected_generation < 0: the current forward half, whichever it is
  void backward(double *force, invdft_force_stats *st, int64_t expected_generation = -1);
  void eval(double *pot, double *force, double *loss, invdft_force_stats *st);
  bool have_forward = false;
  // Bumped by every forward half and by every call that changes what the
  // backward half reads (the potential); a backward for an older forward is
  // refused instead of returning dL/dv_xc at another v_xc.
  int64_t generation = 0;
  void invalidate_forward() { have_forward = false; ++generation; }
  double last_loss = 0.0;
  long long fwd_launches0 = 0;
  void accumulate_child_products(const double *d_psi, const double *d_p, int Bw);
  // v_base = total electrostatic potential of a density and point nuclei
  // (InverseDFTEngine::setPotBasePoissonNuclear), by preconditioned CG on the
  // GPU with the matrix-free Laplacian; host arrays
  void poisson_total(const double *h_rho_quad, int n_atoms, const double *Z, const int64_t *atom_cell,
                     const double *atom_xi, double rel_tol, int max_iter, bool install, double *h_phi_quad,
                     double *h_phi_nodal, int *iters, double *rel_res);
  void poisson_solve(const double *h_rho, int n_atoms, const double *Z, const int64_t *atom_cell,
                     const double *atom_xi, const double *h_bc, double rel_tol, int max_iter, DevBuf<double> &phi,
                     int &it, double &res);
  // initial v_xc guess (InverseDFTEngine::setInitialPotL2Proj); host arrays
  void initial_guess(const double *h_rho, const double *h_sigma, const double *h_bc,
                     const invdft_initial_guess_options &o, double *h_vxc_child, double *h_vxc_parent,
                     double *h_vh_quad);
  DevBuf<double> vj_zero;          // zero potential term: the cell products of the Laplacian
  void kernel_probe();             // one launch of each kernel (profiling)

 private:
  void alloc_state();
  void ensure_adjoint(int Bw);
};

}  // namespace invdft
