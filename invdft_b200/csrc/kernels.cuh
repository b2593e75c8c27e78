// Device kernels of the force evaluation (declarations + small device helpers).
#pragma once
#include "common.cuh"

namespace invdft {

// Device-side view of the parent finite-element data.
struct FeView {
  int n1, nd, nq;
  int ldh;                  // leading dimension of a cell matrix column (nd rounded up to even)
  int64_t nc, nnodes;
  const double *phi;        // [n1][n1]: phi[q*n1+a] = l_a(gauss_q)
  const double *cell_h;     // [nc]
  const int *cell_nodes;    // [nc*nd]
  const int *cell_map;      // [nc*nd]: node (free) or -(1+constraint row)
  const int *cons_ptr;      // [ncons+1]
  const int *cons_masters;
  const double *cons_gw;    // weights * M^-1/2[master] (Lowdin gather)
  int ncons;
  // slot layout of cell results: row (cell, local) of a cell product is written
  // to slot slot_of[cell*nd+local] (-1: Dirichlet row, dropped).  Free nodes own
  // the contiguous slots [dptr[n], dptr[n+1]), a master of hanging nodes one
  // more (the last, for its hanging contributions); rows of hanging nodes live
  // in slots after those, contiguous per hanging node in hanging-index order,
  // and reach their masters through the constraint groups below.
  const int *slot_of;       // [nc*nd]
  // the matrix-free kernel's gather map (cell_map_sf) and the slot map
  // transposed, [nd][nc]: for blocks narrower than 16 columns a CTA of the
  // matrix-free kernel holds several cells, whose entries for one local index
  // are then contiguous
  const int *cell_map_t;
  const int *slot_of_t;
  // the matrix-free kernel's row-major gather map: node, or -(1 + row of hvg)
  // for a constrained entry (the hanging index, or nhang for the zero row of
  // the Dirichlet entries)
  const int *cell_map_sf;
  const int *dptr;          // [nnodes+1]
  const int *zptr;          // [nhang+1] slot ranges of the hanging nodes' rows
  int nhang;
  int nmast;
  const int *mslot;         // [nmast] the last slot of each master's range: its summed hanging contributions
  // constraint rows grouped by identical (ordered) master lists: group g owns
  // the rows g_rptr[g] .. g_rptr[g+1] of the group order, whose hanging indices
  // g_hrow are consecutive (-1 for Dirichlet rows) and whose masters are
  // cons_masters[g_m0[g] ..][0, g_nm[g]); groups [0, ngroup_h) have masters,
  // the rest are Dirichlet rows.  Pair (g, t) of a hanging group is partial
  // row g_poff[g] + t; master i sums the partial rows mp_idx[mp_ptr[i] .. mp_ptr[i+1]).
  int ngroup, ngroup_h, g_maxnm, g_maxnr;
  int g_stage;              // shared staging per group, doubles; larger groups read global memory
  const int *g_rptr, *g_hrow, *g_m0, *g_nm, *g_poff;
  // the plain weights of group g's rows from g_woff[g]: [row q][master t]
  // (g_w, for the transpose) and [t][q] (g_wt, for the gather); groups with
  // identical weight blocks share one copy
  const int64_t *g_woff;
  const double *g_w, *g_wt;
  const int *mp_ptr, *mp_idx;
  double *gpart;            // [npairs][B] scratch: per (group, master) partial sums
  double *hvg;              // [nhang+1][B] scratch: Lowdin-gathered hanging rows, then a zero row
  int *err;                 // device error word (bounded waits that gave up)
  const double *inv_sqrt_mass, *sqrt_mass;
};

constexpr int kGroupRows = 64;     // constraint rows per group at most
constexpr int kGroupStage = 12288; // default shared staging per constraint group (96 KB of doubles)

// Gather modes of the cell GEMM.
enum GatherMode { GATHER_LOWDIN = 0, GATHER_PLAIN = 1 };

// ---- launches (implemented in kernels.cu) ----
long long launch_count();  // kernels launched by this library so far
void count_launch();       // for launches made outside kernels.cu
void count_launches(long long n);   // the kernels of a replayed CUDA graph
void launch_build_cell_h(const FeView &fe, const double *vks, const double *jxw, const double *Kref,
                         double *H, cudaStream_t s);
void launch_hx_cell_gemm(const FeView &fe, const double *H, const double *x, double *Ycell, int B,
                         int gather_mode, cudaStream_t s);
// FP64 tensor-core (mma.sync m8n8k4 f64) variant
void launch_hx_cell_dmma(const FeView &fe, const double *H, const double *x, double *Ycell, int B,
                         int gather_mode, cudaStream_t s);
// same with cell matrices stored in FP32 (products still accumulated in FP64)
void launch_hx_cell_dmma_f32(const FeView &fe, const float *H32, const double *x, double *Ycell, int B,
                             int gather_mode, cudaStream_t s);
void launch_narrow(const double *src, float *dst, int64_t n, cudaStream_t s);
// Reference-element matrices of the matrix-free variant (passed by value, so
// every launch carries its own copy): phi[q*n1+a] = l_a(g_q) on the GLL basis,
// dq[q*n1+r] = derivative at g_q of the Lagrange basis on the Gauss points,
// w = 1D Gauss weights on [0, 1].
constexpr int kSfMaxN = 8;
constexpr int kSfMaxH = kSfMaxN / 2;
template <typename T> struct SfMatsT {
  T phi[kSfMaxN * kSfMaxN];
  T dq[kSfMaxN * kSfMaxN];
  T w[kSfMaxN];
  // even n1: even-odd halves [q*h + a] (h = n1/2) of the four 1D operators,
  // applied as out[q] = E + O, out[n1-1-q] = E - O (Phi, Phi^T: centro-
  // symmetric) or O - E (Dq, Dq^T: centro-antisymmetric), with
  // E = sum_a Xe[q][a] (in[a] + in[n1-1-a]), O = sum_a Xo[q][a] (in[a] - in[n1-1-a])
  T phe[kSfMaxH * kSfMaxH], pho[kSfMaxH * kSfMaxH];   // Phi
  T dqe[kSfMaxH * kSfMaxH], dqo[kSfMaxH * kSfMaxH];   // Dq
  T pte[kSfMaxH * kSfMaxH], pto[kSfMaxH * kSfMaxH];   // Phi^T
  T dte[kSfMaxH * kSfMaxH], dto[kSfMaxH * kSfMaxH];   // Dq^T

  // the same matrices rounded to another type
  template <typename U> SfMatsT<U> as() const {
    SfMatsT<U> o;
    for (int i = 0; i < kSfMaxN * kSfMaxN; ++i) { o.phi[i] = U(phi[i]); o.dq[i] = U(dq[i]); }
    for (int i = 0; i < kSfMaxN; ++i) o.w[i] = U(w[i]);
    for (int i = 0; i < kSfMaxH * kSfMaxH; ++i) {
      o.phe[i] = U(phe[i]); o.pho[i] = U(pho[i]); o.dqe[i] = U(dqe[i]); o.dqo[i] = U(dqo[i]);
      o.pte[i] = U(pte[i]); o.pto[i] = U(pto[i]); o.dte[i] = U(dte[i]); o.dto[i] = U(dto[i]);
    }
    return o;
  }
};
using SfMats = SfMatsT<double>;

// FP32 arithmetic whose products take their operands rounded to the input
// format of a tensor-core MMA: M = 1 TF32 (cvt.rna.tf32.f32, 10-bit mantissa),
// M = 2 BF16 (round to nearest even, 7-bit mantissa).  The 1D operator
// applications (the GEMM-shaped part of the cell product) round both operands
// and accumulate in FP32, as tcgen05.mma kind::tf32 / kind::f16 with an FP32
// accumulator do; sums, the weights and the potential product (the element-wise
// epilogue of such a kernel) stay plain FP32.  It measures what those tensor-core
// products would do to the filter's convergence, at FP32 speed.
template <int M> struct TcOperand {
  float v;
  TcOperand() = default;
  __host__ __device__ constexpr TcOperand(float x) : v(x) {}
  __host__ __device__ constexpr TcOperand(double x) : v(float(x)) {}
  __host__ __device__ constexpr TcOperand(int x) : v(float(x)) {}
  __host__ __device__ explicit operator double() const { return v; }
  __host__ __device__ TcOperand &operator*=(TcOperand o) { v *= o.v; return *this; }
};
template <int M> __host__ __device__ inline TcOperand<M> operator+(TcOperand<M> a, TcOperand<M> b) { return a.v + b.v; }
template <int M> __host__ __device__ inline TcOperand<M> operator-(TcOperand<M> a, TcOperand<M> b) { return a.v - b.v; }
template <int M> __host__ __device__ inline TcOperand<M> operator*(TcOperand<M> a, TcOperand<M> b) { return a.v * b.v; }
using Tf32Operand = TcOperand<1>;
using Bf16Operand = TcOperand<2>;
// matrix-free variant: vj = v_KS * JxW at the parent quadrature points, twice:
// [nc][nq] followed by its transpose [nq][nc] (read by blocks narrower than 16);
// tune 0: one CTA per SM allowed the registers it wants, 1: two CTAs per SM,
// 2: two CTAs per SM with the derivative lines held in shared memory (order 5)
void launch_hx_cell_sf(const FeView &fe, const SfMats &mt, const double *vj, const double *x, double *Ycell,
                       int B, int gather_mode, int tune, cudaStream_t s);
// the same with FP32 arithmetic (FP64 block in, FP64 cell results out): the
// low rungs of the mixed-precision Chebyshev ladder
void launch_hx_cell_sf_f32(const FeView &fe, const SfMatsT<float> &mt, const double *vj, const double *x,
                           double *Ycell, int B, int gather_mode, cudaStream_t s);
// ... with the 1D operator products on TF32- or BF16-rounded operands (FE orders
// 2, 4 and 5): the numerics of a tensor-core cell product
void launch_hx_cell_sf_tc(const FeView &fe, const SfMatsT<Tf32Operand> &mt, const double *vj, const double *x,
                          double *Ycell, int B, int gather_mode, cudaStream_t s);
void launch_hx_cell_sf_tc(const FeView &fe, const SfMatsT<Bf16Operand> &mt, const double *vj, const double *x,
                          double *Ycell, int B, int gather_mode, cudaStream_t s);
// out[c][q] = a[q][c] (rows x cols -> cols x rows)
void launch_transpose(const double *a, double *out, int64_t rows, int64_t cols, cudaStream_t s);
// out[i] = a[i] * b[i]
void launch_mul(const double *a, const double *b, double *out, int64_t n, cudaStream_t s);
// out[i] = a x[i] + b y[i] + c z[i] (y, z may be null); out may alias x, y or z
void launch_axpbypcz(double *out, double a, const double *x, double b, const double *y, double c, const double *z,
                     int64_t n, cudaStream_t s);
// bulk-asynchronous staged variant (persistent CTAs, shared-memory panel ring)
void launch_hx_cell_gemm_bulk(const FeView &fe, const double *H, const double *x, double *Yslot, int B,
                              int gather_mode, cudaStream_t s);

// Epilogue selector for the assembly kernel.
struct AsmEpilogue {
  enum Kind { STORE = 0, CHEB = 1, VMULT = 2, RHS = 3, MINRES = 4 } kind = STORE;
  double alpha = 1.0, c = 0.0, beta = 0.0;   // CHEB: out = alpha*(acc - c*in) - beta*prev
  const double *in = nullptr;                // CHEB input block / VMULT x / MINRES v
  const double *prev = nullptr;              // CHEB previous block / MINRES r1
  const double *eps = nullptr;               // VMULT/MINRES shifts (eps_b, added as -eps_b x)
  const double *occ4 = nullptr;              // RHS: 4 f_b
  const double *Mu = nullptr;                // RHS: Mu[k*B+b]
  const double *psi = nullptr;               // RHS: distributed nodal psi
  const double *minres_coef = nullptr;       // MINRES: beta/oldb per column (0 at itn 1)
  double *dot_partial = nullptr;             // MINRES: per-block column partials of v.y
  double *dot_out = nullptr;                 // MINRES: if set with dot_ticket, the last CTA reduces the
  unsigned *dot_ticket = nullptr;            //   partials into dot_out[B] (ticket zero on entry and exit)
};
int assemble_blocks(const FeView &fe, int B);  // CTAs of launch_hx_assemble for width B
// returns the number of CTAs (= MINRES dot partials written), or 0 when the
// launch has already reduced them into epi.dot_out
int launch_hx_assemble(const FeView &fe, const double *Ycell, double *out, int B,
                       const AsmEpilogue &epi, int dot_blocks, cudaStream_t s);

void launch_scale_rows(const double *d, const double *x, double *y, int64_t n, int B, cudaStream_t s);
void launch_distribute(const int *rows, const int *ptr, const int *masters, const double *w, int nrows,
                       double *x, int B, cudaStream_t s);
void launch_set_zero(const int *rows, int nrows, double *x, int B, cudaStream_t s);

// Tall-skinny products, deterministic: C = A^T B, N x N (N <= 64)
void launch_gram(const double *A, const double *Bm, int64_t n, int N, double *partial, int nblocks,
                 double *out, cudaStream_t s);
// Z = Y T (T N x N)
void launch_rotate(const double *Y, const double *T, double *Z, int64_t n, int N, cudaStream_t s);
// X = Y Q, R = HY Q - X diag(eps): column sums of R^2 into out [N]
void launch_rotate_residual(const double *Y, const double *HY, const double *Q, const double *eps,
                            double *X, int64_t n, int N, double *partial, int nblocks, double *out,
                            cudaStream_t s);
// per-column dot products a.b over n rows -> out [B] (deterministic)
void launch_coldot(const double *a, const double *b, int64_t n, int B, double *partial, int nblocks,
                   double *out, cudaStream_t s);
void launch_reduce_partials(const double *partial, int nparts, int width, double *out, cudaStream_t s);

// Interpolation of nodal blocks to parent quadrature points: out [nc][nq][B]
void launch_interp_to_quad(const FeView &fe, const double *x, double *out, int B, cudaStream_t s);
// per-cell pair sums: partial[e*npairs + k] = fac(k) * sum_q w[e,q] Qa[e,q,i_k] Qb[e,q,j_k]
void launch_pair_quad_sums(const FeView &fe, const double *Qa, const double *Qb, const double *w, int B,
                           const int *pairs, int npairs, double *partial, cudaStream_t s);
// sum_e R_e x_e with R_e = N^T diag(wq) N: Ycell [nc][nd][B]
void launch_r_cell(const FeView &fe, const double *x, const double *wq, double *Ycell, int B,
                   cudaStream_t s);
// cell right-hand sides of an L2 projection: Ycell[slot(e,l)] = sum_q N_l(q) fw[e,q] (width 1)
void launch_quad_rhs(const FeView &fe, const double *fw, double *Ycell, cudaStream_t s);
// out[i] = parent nodal field u at (cells[i], xi[3i..3i+2]) (reference coordinates in [0,1]^3)
void launch_eval_points(const FeView &fe, const double *gll, const double *u, int64_t npts, const int64_t *cells,
                        const double *xi, double *out, cudaStream_t s);
// density rho = 2 sum f psi^2 at parent quad points + drho/u/loss partials
void launch_density(const FeView &fe, const double *psi, const double *occ, int N, const double *rho_t,
                    const double *weight, const double *jxw, const double *vks, double *rho,
                    double *u, double *partial4, cudaStream_t s);
// x[:, i] += sum_{k in pairs with i_k = i} coef_k psi[:, j_k]
void launch_nullspace_update(double *x, const double *psi, int64_t n, int B, const int *pair_ptr,
                             const int *pair_j, const double *coef, cudaStream_t s);

// MINRES building blocks (per-column masked, scalars on device)
struct MinresState {
  double *beta, *oldb, *dbar, *epsln, *phibar, *cs, *sn;
  double *alfa, *beta2;            // reduced dots
  double *coef1;                   // beta/oldb (0 at the first iteration)
  double *oldeps, *delta, *denom, *phi;
  int *active, *commit, *iters;
  double tol;
};
void launch_minres_v(const double *y, const MinresState &st, double *v, int64_t n, int B, cudaStream_t s);
void launch_minres_update1(double *r1, double *r2, double *y, const double *yn, const double *diagA,
                           const MinresState &st, int64_t n, int B, double *partial, int nblocks,
                           cudaStream_t s);
void launch_minres_scalars(const MinresState &st, int B, int itn, cudaStream_t s);
void launch_minres_update2(double *x, double *w, double *w2, const double *v, const MinresState &st,
                           int64_t n, int B, cudaStream_t s);
void launch_minres_init(const double *b, const double *diagA, double *r1, double *r2, double *y,
                        int64_t n, int B, double *partial, int nblocks, cudaStream_t s);
void launch_minres_init_scalars(const MinresState &st, const double *beta1_sq, int B, cudaStream_t s);
// update1 + the reduction of beta2 + the scalar update in one launch (the last
// CTA reduces and updates; *ticket must be 0 before, and is 0 after).  The new
// r2 = yn - (alfa/beta) r2 is written over yn; the caller then rotates the
// buffers (r1, r2, yn) <- (r2, yn, r1) instead of copying r2 into r1.
void launch_minres_update1_fused(const double *r2, double *yn, double *y, const double *diagA,
                                 const MinresState &st, int64_t n, int B, double *partial, int nblocks,
                                 unsigned *ticket, cudaStream_t s);
// update2 + the next iteration's v = y / beta in one launch (v in place).  The
// new w is written over w2; the caller then swaps the buffers w and w2.
void launch_minres_update2v(double *x, const double *w, double *w2, double *v, const double *y,
                            const MinresState &st, int64_t n, int B, cudaStream_t s);

// Child mesh transfers
struct ChildView {
  int64_t ncc, nchild_nodes;
  const int *cell_nodes;      // [ncc*8]
  const double *jxw;          // [ncc*8]
  const int *parent;          // [ncc]
  const double *offset;       // [ncc*3]
  const double *scale;        // [ncc]
  const int *pq_child;        // [nc*nq]
  const double *pq_xi;        // [nc*nq*3]
  const int *sc_ptr, *sc_src; // scatter CSR over child nodes (entry = cell*8 + k)
  const double *sc_w;
  const int *work_parent, *work_c0, *work_c1; // transfer work items
  int nwork;
  const double *gll;          // [n1] parent GLL nodes
  const double *g2;           // [2] Gauss points of the child rule
};
// vks = v_base (optional, may be null) + child potential at parent quad points + factor_lda * v_lda
void launch_child_to_parent_quad(const ChildView &cv, const double *pot, const double *v_base,
                                 const double *v_lda, double factor_lda, double *vks, int64_t nqtot,
                                 cudaStream_t s);
void launch_psi_adjoint_child(const FeView &fe, const ChildView &cv, const double *psi, const double *p,
                              int B, double *S, cudaStream_t s);
void launch_force_project(const ChildView &cv, const double *S, double *force, cudaStream_t s);

}  // namespace invdft
