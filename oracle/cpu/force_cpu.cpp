// CPU restatement of invDFT's force evaluation in C++17 + OpenMP, FP64.
//
// TEST INFRASTRUCTURE ONLY: the tests use it as a fast checker on meshes too
// large for the numpy oracle, and the benchmark times it as the CPU baseline
// (the reference itself needs DFT-FE, deal.II and MPI, none of which exist
// here).  The product never links or calls it.
//
// It restates, operation by operation, the numpy oracle in oracle/*.py, which
// in turn follows the reference:
//   getForceVector           src/InverseDFTSolverFunction.cpp:657-1311
//   solveEigen               src/InverseDFTSolverFunction.cpp:1315-1477
//   evaluateDegeneracyMap    src/InverseDFTSolverFunction.cpp:37-77
//   integrateWithShapeFunctionsForChildData  :1611-1674
//   computeRhs / vmult / precondition_Jacobi / distributeX / updateInputPsi
//                            src/MultiVectorAdjointLinearSolverProblem.cpp:541-1367
// and restates from the mathematics what the reference delegates to DFT-FE:
// the Lowdin Hamiltonian of GLL spectral elements (here applied matrix-free by
// sum factorisation instead of the oracle's stored cell matrices -- the same
// operator, since the (p+1)-point Gauss rule integrates the stiffness
// exactly), Chebyshev-filtered subspace iteration with Cholesky
// orthonormalisation and Rayleigh-Ritz, Paige-Saunders block MINRES with
// per-column masks, and the Fermi-Dirac occupancies.
//
// Layouts follow the reference: multi-vectors [node][B] with the vector index
// fastest, parent quadrature data [cell][q], child quadrature data [cell][8].
// Every reduction is split into a fixed number of chunks summed in chunk
// order, so results do not depend on the thread count.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/invdft_force.h"

namespace ocpu {

using std::int64_t;
using std::vector;

constexpr double kKb = 3.166811429e-06;  // Ha/K
constexpr int kChunks = 512;             // fixed reduction chunks

thread_local std::string g_err;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// ---------------------------------------------------------------------------
// small dense helpers (N <= 64)
// ---------------------------------------------------------------------------
double hash_uniform(uint64_t i, uint64_t salt) {
  // the oracle's reproducible generator (oracle/eigen.py hash_uniform)
  uint64_t h = (i * 2654435761ull + salt * 40503ull) & 0xFFFFFFFFull;
  h ^= h >> 15;
  h = (h * 2246822519ull) & 0xFFFFFFFFull;
  h ^= h >> 13;
  return (double)h / 4294967296.0 - 0.5;
}

// symmetric eigenproblem by cyclic Jacobi rotations; ascending eigenvalues,
// eigenvector columns signed so that their largest-magnitude entry is positive
void sym_eig(int n, vector<double> A, vector<double> &w, vector<double> &V) {
  vector<double> Q((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) (i == j ? diag : off) += A[(size_t)i * n + j] * A[(size_t)i * n + j];
    if (off == 0.0 || off < 1e-30 * diag) break;
    for (int p = 0; p + 1 < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double tau = (A[(size_t)q * n + q] - A[(size_t)p * n + p]) / (2.0 * apq);
        const double t = std::copysign(1.0, tau) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double x = A[(size_t)k * n + p], y = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * x - s * y;
          A[(size_t)k * n + q] = s * x + c * y;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double x = A[(size_t)p * n + k], y = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * x - s * y;
          A[(size_t)q * n + k] = s * x + c * y;
        }
        for (int k = 0; k < n; ++k) {
          const double x = Q[(size_t)k * n + p], y = Q[(size_t)k * n + q];
          Q[(size_t)k * n + p] = c * x - s * y;
          Q[(size_t)k * n + q] = s * x + c * y;
        }
      }
  }
  vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int a, int b) { return A[(size_t)a * n + a] < A[(size_t)b * n + b]; });
  w.resize(n);
  V.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    const int c = ord[j];
    w[j] = A[(size_t)c * n + c];
    int im = 0;
    for (int i = 1; i < n; ++i)
      if (std::fabs(Q[(size_t)i * n + c]) > std::fabs(Q[(size_t)im * n + c])) im = i;
    const double sg = Q[(size_t)im * n + c] < 0.0 ? -1.0 : 1.0;
    for (int i = 0; i < n; ++i) V[(size_t)i * n + j] = sg * Q[(size_t)i * n + c];
  }
}

double occupancy(double e, double mu, double kT) {
  const double x = (e - mu) / kT;
  return x >= 0 ? std::exp(-x) / (1.0 + std::exp(-x)) : 1.0 / (1.0 + std::exp(x));
}
double occupancy_der(double e, double mu, double kT) {
  const double x = (e - mu) / kT, t = std::exp(-std::fabs(x));
  return -t / (kT * (1.0 + t) * (1.0 + t));
}
double fermi_level(const vector<double> &e, double ne, double kT) {
  double lo = *std::min_element(e.begin(), e.end()) - 1.0, hi = *std::max_element(e.begin(), e.end()) + 1.0;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    double n = 0.0;
    for (double v : e) n += occupancy(v, mid, kT);
    if (2.0 * n > ne) hi = mid;
    else lo = mid;
    if (hi - lo < 1e-15 * std::max(1.0, std::fabs(mid))) break;
  }
  return 0.5 * (lo + hi);
}

vector<double> lagrange(const vector<double> &nodes, double x) {
  const int n = (int)nodes.size();
  vector<double> v(n, 1.0);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      if (b != a) v[a] *= (x - nodes[b]) / (nodes[a] - nodes[b]);
  return v;
}
vector<double> lagrange_d(const vector<double> &nodes, double x) {
  const int n = (int)nodes.size();
  vector<double> v(n, 0.0);
  for (int a = 0; a < n; ++a)
    for (int m = 0; m < n; ++m) {
      if (m == a) continue;
      double t = 1.0 / (nodes[a] - nodes[m]);
      for (int b = 0; b < n; ++b)
        if (b != a && b != m) t *= (x - nodes[b]) / (nodes[a] - nodes[b]);
      v[a] += t;
    }
  return v;
}

// ---------------------------------------------------------------------------
// constraints (closed: masters are never constrained)
// ---------------------------------------------------------------------------
struct Cons {
  int64_t n = 0;
  vector<int64_t> rows, ptr, masters;
  vector<double> w;
  // transpose over master nodes, entries in (row, k) order
  vector<int64_t> tnode, tptr, tslave;
  vector<double> tw;

  void load(const invdft_constraints &c, int64_t nnodes) {
    n = c.n_rows;
    rows.assign(c.rows, c.rows + n);
    ptr.assign(c.ptr, c.ptr + n + 1);
    const int64_t nm = n ? ptr[n] : 0;
    masters.assign(c.masters, c.masters + nm);
    w.assign(c.weights, c.weights + nm);
    for (int64_t r = 0; r < n; ++r)
      if (rows[r] < 0 || rows[r] >= nnodes) throw Error(INVDFT_BAD_ARG, "constraint row out of range");
    std::map<int64_t, vector<std::pair<int64_t, double>>> t;
    for (int64_t r = 0; r < n; ++r)
      for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) {
        if (masters[k] < 0 || masters[k] >= nnodes) throw Error(INVDFT_BAD_ARG, "constraint master out of range");
        t[masters[k]].push_back({rows[r], w[k]});
      }
    tptr.assign(1, 0);
    for (auto &kv : t) {
      tnode.push_back(kv.first);
      for (auto &e : kv.second) {
        tslave.push_back(e.first);
        tw.push_back(e.second);
      }
      tptr.push_back((int64_t)tslave.size());
    }
  }
  // x[s] = sum_k w x[m] (Dirichlet rows become zero)
  void distribute(double *x, int B) const {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r)
      for (int b = 0; b < B; ++b) {
        double v = 0.0;
        for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) v += w[k] * x[masters[k] * B + b];
        x[rows[r] * B + b] = v;
      }
  }
  // x[m] += w x[s]; then x[s] = 0
  void slave_to_master(double *x, int B) const {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)tnode.size(); ++i)
      for (int b = 0; b < B; ++b) {
        double v = x[tnode[i] * B + b];
        for (int64_t k = tptr[i]; k < tptr[i + 1]; ++k) v += tw[k] * x[tslave[k] * B + b];
        x[tnode[i] * B + b] = v;
      }
    set_zero(x, B);
  }
  void set_zero(double *x, int B) const {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r)
      for (int b = 0; b < B; ++b) x[rows[r] * B + b] = 0.0;
  }
};

// column dot products of [n][B] blocks, chunked deterministic reduction
void coldots(const double *a, const double *b, int64_t n, int B, double *out) {
  vector<double> part((size_t)kChunks * B, 0.0);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < kChunks; ++c) {
    const int64_t r0 = n * c / kChunks, r1 = n * (c + 1) / kChunks;
    double *p = &part[(size_t)c * B];
    for (int64_t r = r0; r < r1; ++r)
      for (int j = 0; j < B; ++j) p[j] += a[r * B + j] * b[r * B + j];
  }
  for (int j = 0; j < B; ++j) out[j] = 0.0;
  for (int c = 0; c < kChunks; ++c)
    for (int j = 0; j < B; ++j) out[j] += part[(size_t)c * B + j];
}

// growable buffer whose contents are not initialised (no memset per call)
struct Scratch {
  std::unique_ptr<double[]> p;
  size_t n = 0;
  double *get(size_t count) {
    if (count > n) {
      p.reset(new double[count]);
      n = count;
    }
    return p.get();
  }
};

// ---------------------------------------------------------------------------
// the context
// ---------------------------------------------------------------------------
struct Ctx {
  invdft_params prm{};
  int p = 0, n1 = 0, nd = 0, N = 0;
  int64_t nc = 0, nn = 0, ncc = 0, ncn = 0;
  double ne = 0, kT = 0;
  vector<double> phi, dq, wq, gll;     // phi[q*n1+a], dq[q*n1+r]: collocation derivative on the Gauss points
  vector<int64_t> cell_nodes;          // [nc][nd]
  vector<double> cell_h, jxw, v_base, v_lda, rho_t, weight;
  Cons cpsi, cadj, cchild;
  vector<double> mass, sqm, isqm, diagA;
  vector<char> free_row;
  vector<int64_t> aptr, aent;          // node -> entries e*nd + l (assembly)
  // child mesh
  vector<int64_t> ch_nodes, ch_parent, pq_child, cptr, cent;
  vector<double> ch_jxw, ch_off, ch_scale, pq_xi;
  // state
  vector<double> X, psi, eig, occ, vks, vj, rho, u;
  double mu = 0.0, tol_cheb = 1e-8, loss_prev = 0.0, adjoint_tol = 0.0;
  bool have_eig = false;
  int counter = 0;
  int64_t n_hx = 0, n_hx_cols = 0;
  Scratch s_t;

  vector<double> w3;                   // [nq] products of the 1D Gauss weights
  vector<int64_t> color_ptr, color_cells;  // cells by colour: no two cells of a colour share a node
  void cells(int op, const double *x, int B, double *y, const double *wf) const;
  void hx(const double *x, double *y, int B);
  void set_potential(const double *pot_distributed);
  void to_quad(const double *x, int B, double *q) const;           // [nc][nq][B]
  void r_times(const double *x, const double *wq_field, int B, double *y) const;
};

// ---------------------------------------------------------------------------
// cell kernels by sum factorisation on tiles of BT columns, [n1^3][BT] layout,
// the order N = n1 and the tile width compile-time constants
// ---------------------------------------------------------------------------
// a tile row of BT columns as one value: a GCC vector of BT doubles (8-byte
// aligned, so any row of a buffer can be loaded), a plain double for BT = 1
template <int BT> struct Row {
  typedef double type __attribute__((vector_size(BT * 8), aligned(8)));
};
template <> struct Row<1> {
  typedef double type;
};

// out[.., q, ..] (+)= sum_a M(q, a) in[.., a, ..] along direction DIR, with
// M(q, a) = A[q*N+a] (or A[a*N+q] when TR).  For even N the operators of the
// GLL/Gauss element are centro-symmetric (Phi) or centro-antisymmetric (the
// collocation derivative), M(N-1-q, N-1-a) = +-M(q, a), because both point
// sets are symmetric about 1/2: the product then splits into even and odd
// halves, (N/2)^2 multiply-adds each instead of N^2.
template <int N, int BT, int DIR, bool TR, bool ACC, bool ANTI>
static inline void ap1(const double *__restrict A, const double *__restrict in, double *__restrict out) {
  typedef typename Row<BT>::type V;
  constexpr int S = DIR == 0 ? 1 : (DIR == 1 ? N : N * N);
  constexpr int N2 = N * N;
  constexpr int H = N / 2;
  const V *vin = reinterpret_cast<const V *>(in);
  V *vout = reinterpret_cast<V *>(out);
  double M[N][N];
  for (int q = 0; q < N; ++q)
    for (int a = 0; a < N; ++a) M[q][a] = TR ? A[a * N + q] : A[q * N + a];
  if constexpr (N % 2 == 0) {
    double Me[H][H], Mo[H][H];
    for (int q = 0; q < H; ++q)
      for (int a = 0; a < H; ++a) {
        Me[q][a] = 0.5 * (M[q][a] + M[q][N - 1 - a]);
        Mo[q][a] = 0.5 * (M[q][a] - M[q][N - 1 - a]);
      }
    for (int line = 0; line < N2; ++line) {
      const int i0 = line % N, i1 = line / N;
      const int base = DIR == 0 ? N * i0 + N2 * i1 : (DIR == 1 ? i0 + N2 * i1 : i0 + N * i1);
      V e[H], o[H];
#pragma GCC unroll 8
      for (int a = 0; a < H; ++a) {
        const V lo = vin[base + a * S], hi = vin[base + (N - 1 - a) * S];
        e[a] = lo + hi;
        o[a] = lo - hi;
      }
#pragma GCC unroll 8
      for (int q = 0; q < H; ++q) {
        V E = e[0] * Me[q][0], O = o[0] * Mo[q][0];
#pragma GCC unroll 8
        for (int a = 1; a < H; ++a) {
          E += Me[q][a] * e[a];
          O += Mo[q][a] * o[a];
        }
        const V lo = E + O, hi = ANTI ? O - E : E - O;
        if (ACC) {
          vout[base + q * S] += lo;
          vout[base + (N - 1 - q) * S] += hi;
        } else {
          vout[base + q * S] = lo;
          vout[base + (N - 1 - q) * S] = hi;
        }
      }
    }
  } else {
    for (int line = 0; line < N2; ++line) {
      const int i0 = line % N, i1 = line / N;
      const int base = DIR == 0 ? N * i0 + N2 * i1 : (DIR == 1 ? i0 + N2 * i1 : i0 + N * i1);
      V v[N];
#pragma GCC unroll 8
      for (int a = 0; a < N; ++a) v[a] = vin[base + a * S];
#pragma GCC unroll 8
      for (int q = 0; q < N; ++q) {
        V acc = ACC ? vout[base + q * S] : v[0] * 0.0;
#pragma GCC unroll 8
        for (int a = 0; a < N; ++a) acc += M[q][a] * v[a];
        vout[base + q * S] = acc;
      }
    }
  }
}

// y = (f K_ref + N^T diag(vJ) N) x on one tile: Gauss-point values, their
// collocation derivatives weighted by f W3, and the transposes
template <int N, int BT>
static void cell_tile(const double *phi, const double *dq, const double *w3f, const double *vje,
                      const double *x, double *y, double *work) {
  constexpr int ND = N * N * N;
  double *t1 = work, *t2 = work + ND * BT, *uq = work + 2 * ND * BT, *g = work + 3 * ND * BT,
         *r = work + 4 * ND * BT;
  ap1<N, BT, 0, false, false, false>(phi, x, t1);
  ap1<N, BT, 1, false, false, false>(phi, t1, t2);
  ap1<N, BT, 2, false, false, false>(phi, t2, uq);
  for (int q = 0; q < ND; ++q)
    for (int b = 0; b < BT; ++b) r[q * BT + b] = vje[q] * uq[q * BT + b];
  ap1<N, BT, 0, false, false, true>(dq, uq, g);
  for (int q = 0; q < ND; ++q)
    for (int b = 0; b < BT; ++b) g[q * BT + b] *= w3f[q];
  ap1<N, BT, 0, true, true, true>(dq, g, r);
  ap1<N, BT, 1, false, false, true>(dq, uq, g);
  for (int q = 0; q < ND; ++q)
    for (int b = 0; b < BT; ++b) g[q * BT + b] *= w3f[q];
  ap1<N, BT, 1, true, true, true>(dq, g, r);
  ap1<N, BT, 2, false, false, true>(dq, uq, g);
  for (int q = 0; q < ND; ++q)
    for (int b = 0; b < BT; ++b) g[q * BT + b] *= w3f[q];
  ap1<N, BT, 2, true, true, true>(dq, g, r);
  ap1<N, BT, 2, true, false, false>(phi, r, t1);
  ap1<N, BT, 1, true, false, false>(phi, t1, t2);
  ap1<N, BT, 0, true, false, false>(phi, t2, y);
}

// values at the Gauss points (interp) or N^T diag(wf) N x (rmat)
template <int N, int BT>
static void quad_tile(const double *phi, const double *wf, const double *x, double *y, double *work, bool rmat) {
  constexpr int ND = N * N * N;
  double *t1 = work, *t2 = work + ND * BT, *t3 = work + 2 * ND * BT;
  ap1<N, BT, 0, false, false, false>(phi, x, t1);
  ap1<N, BT, 1, false, false, false>(phi, t1, t2);
  if (!rmat) {
    ap1<N, BT, 2, false, false, false>(phi, t2, y);
    return;
  }
  ap1<N, BT, 2, false, false, false>(phi, t2, t3);
  for (int q = 0; q < ND; ++q)
    for (int b = 0; b < BT; ++b) t3[q * BT + b] *= wf[q];
  ap1<N, BT, 2, true, false, false>(phi, t3, t1);
  ap1<N, BT, 1, true, false, false>(phi, t1, t2);
  ap1<N, BT, 0, true, false, false>(phi, t2, y);
}

enum TileOp { OP_H = 0, OP_R = 1, OP_Q = 2 };

template <int N, int BT>
static void tile_op(int op, const double *phi, const double *dq, const double *w3f, const double *wf,
                    const double *x, double *y, double *work) {
  if (op == OP_H) cell_tile<N, BT>(phi, dq, w3f, wf, x, y, work);
  else quad_tile<N, BT>(phi, wf, x, y, work, op == OP_R);
}

template <int BT>
static void tile_dispatch(int n1, int op, const double *phi, const double *dq, const double *w3f, const double *wf,
                          const double *x, double *y, double *work) {
  switch (n1) {
    case 2: tile_op<2, BT>(op, phi, dq, w3f, wf, x, y, work); break;
    case 3: tile_op<3, BT>(op, phi, dq, w3f, wf, x, y, work); break;
    case 4: tile_op<4, BT>(op, phi, dq, w3f, wf, x, y, work); break;
    case 5: tile_op<5, BT>(op, phi, dq, w3f, wf, x, y, work); break;
    case 6: tile_op<6, BT>(op, phi, dq, w3f, wf, x, y, work); break;
    case 7: tile_op<7, BT>(op, phi, dq, w3f, wf, x, y, work); break;
    case 8: tile_op<8, BT>(op, phi, dq, w3f, wf, x, y, work); break;
    default: throw Error(INVDFT_BAD_ARG, "FE order outside 1..7");
  }
}

static int tile_width(int B) { return B >= 6 ? 8 : (B >= 2 ? 4 : 1); }

// Per-cell operator over all columns of a [node][B] block, in column tiles.
// OP_H and OP_R scatter-add into y[node][B] (cells of one colour share no
// node, so colours run one after another and cells of a colour in parallel);
// OP_Q writes the cell's [nq][B] Gauss-point values to y + e*nq*B.
void Ctx::cells(int op, const double *x, int B, double *y, const double *wf) const {
  const int BT = tile_width(B);
  const int64_t ndl = nd;
  if (op != OP_Q) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nn; ++i)
      for (int b = 0; b < B; ++b) y[i * B + b] = 0.0;
  }
  const int ncol = (int)color_ptr.size() - 1;
  for (int col = 0; col < (op == OP_Q ? 1 : ncol); ++col) {
    const int64_t k0 = op == OP_Q ? 0 : color_ptr[col], k1 = op == OP_Q ? nc : color_ptr[col + 1];
#pragma omp parallel
    {
      vector<double> xe((size_t)nd * BT), ye((size_t)nd * BT), work((size_t)5 * nd * BT), w3f(nd);
#pragma omp for schedule(static)
      for (int64_t k = k0; k < k1; ++k) {
        const int64_t e = op == OP_Q ? k : color_cells[k];
        const int64_t *cn = &cell_nodes[e * ndl];
        if (op == OP_H)
          for (int q = 0; q < nd; ++q) w3f[q] = 0.5 * cell_h[e] * w3[q];
        for (int b0 = 0; b0 < B; b0 += BT) {
          const int w = std::min(BT, B - b0);
          for (int l = 0; l < nd; ++l)
            for (int b = 0; b < BT; ++b) xe[(size_t)l * BT + b] = b < w ? x[cn[l] * B + b0 + b] : 0.0;
          const double *wfe = op == OP_H ? &vj[e * ndl] : (wf ? wf + e * ndl : nullptr);
          if (BT == 8) tile_dispatch<8>(n1, op, phi.data(), dq.data(), w3f.data(), wfe, xe.data(), ye.data(), work.data());
          else if (BT == 4) tile_dispatch<4>(n1, op, phi.data(), dq.data(), w3f.data(), wfe, xe.data(), ye.data(), work.data());
          else tile_dispatch<1>(n1, op, phi.data(), dq.data(), w3f.data(), wfe, xe.data(), ye.data(), work.data());
          if (op == OP_Q) {
            double *o = y + (size_t)e * nd * B;
            for (int q = 0; q < nd; ++q)
              for (int b = 0; b < w; ++b) o[(size_t)q * B + b0 + b] = ye[(size_t)q * BT + b];
          } else {
            for (int l = 0; l < nd; ++l)
              for (int b = 0; b < w; ++b) y[cn[l] * B + b0 + b] += ye[(size_t)l * BT + b];
          }
        }
      }
    }
  }
}

// Lowdin HX: y = M^-1/2 C^T sum_e H_e (C M^-1/2 x)_e
void Ctx::hx(const double *x, double *y, int B) {
  double *t = s_t.get((size_t)nn * B);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nn; ++i)
    for (int b = 0; b < B; ++b) t[i * B + b] = isqm[i] * x[i * B + b];
  cpsi.distribute(t, B);
  cells(OP_H, t, B, y, nullptr);
  cpsi.slave_to_master(y, B);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nn; ++i)
    for (int b = 0; b < B; ++b) y[i * B + b] *= isqm[i];
  ++n_hx;
  n_hx_cols += B;
}

void Ctx::to_quad(const double *x, int B, double *q) const { cells(OP_Q, x, B, q, nullptr); }

// sum_e A_e R_e x_e with R_e = N^T diag(wf) N (wf a quadrature field)
void Ctx::r_times(const double *x, const double *wf, int B, double *y) const { cells(OP_R, x, B, y, wf); }

// child v_xc (already distributed) -> v_KS at the parent quadrature points
void Ctx::set_potential(const double *pot) {
  const int64_t nqt = nc * nd;
  vks.resize(nqt);
  vj.resize(nqt);
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < nqt; ++q) {
    const int64_t c = pq_child[q];
    const double x = pq_xi[3 * q], y = pq_xi[3 * q + 1], z = pq_xi[3 * q + 2];
    double v = 0.0;
    for (int k = 0; k < 8; ++k) {
      const double wx = (k & 1) ? x : 1.0 - x, wy = (k & 2) ? y : 1.0 - y, wz = (k & 4) ? z : 1.0 - z;
      v += wx * wy * wz * pot[ch_nodes[c * 8 + k]];
    }
    vks[q] = v_base[q] + v + prm.factor_lda * v_lda[q];
    vj[q] = vks[q] * jxw[q];
  }
}

int auto_degree(double b) {
  return (int)std::min(500.0, std::max(24.0, std::ceil(3.0 * std::sqrt(std::max(b, 0.0)))));
}

// ---------------------------------------------------------------------------
// eigensolver (solveEigen, InverseDFTSolverFunction.cpp:1315-1477)
// ---------------------------------------------------------------------------
struct Eigen {
  Ctx &c;
  explicit Eigen(Ctx &cc) : c(cc) {}

  void bounds(double &lo, double &hi) {
    const int64_t n = c.nn;
    vector<double> v(n), vp(n, 0.0), w(n);
    double nrm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      v[i] = c.free_row[i] ? hash_uniform((uint64_t)i, 7) : 0.0;
      nrm += v[i] * v[i];
    }
    nrm = std::sqrt(nrm);
    for (auto &t : v) t /= nrm;
    vector<double> al, be;
    double beta = 0.0;
    for (int it = 0; it < c.prm.lanczos_steps; ++it) {
      c.hx(v.data(), w.data(), 1);
      double a;
      coldots(v.data(), w.data(), n, 1, &a);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i) w[i] = w[i] - a * v[i] - beta * vp[i];
      double b2;
      coldots(w.data(), w.data(), n, 1, &b2);
      beta = std::sqrt(std::max(b2, 0.0));
      al.push_back(a);
      be.push_back(beta);
      if (!std::isfinite(a) || !std::isfinite(beta)) throw Error(INVDFT_NONFINITE, "non-finite Lanczos step");
      if (beta == 0.0) break;
      vp = v;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i) v[i] = w[i] / beta;
    }
    const int k = (int)al.size();
    vector<double> T((size_t)k * k, 0.0), ev, V;
    for (int i = 0; i < k; ++i) {
      T[(size_t)i * k + i] = al[i];
      if (i + 1 < k) T[(size_t)i * k + i + 1] = T[(size_t)(i + 1) * k + i] = be[i];
    }
    sym_eig(k, T, ev, V);
    lo = ev.front();
    hi = ev.back() + std::fabs(be.back());
  }

  // one filter + Cholesky-GS + Rayleigh-Ritz + residual pass
  void pass(int m, double a, double b, double a0, vector<double> &res) {
    const int N = c.N;
    const int64_t n = c.nn;
    const double e = (b - a) / 2.0, cc = (b + a) / 2.0;
    double sigma = e / (a0 - cc);
    const double sigma1 = sigma, gamma = 2.0 / sigma1;
    vector<double> X0 = c.X, Y((size_t)n * N), HY((size_t)n * N);
    c.hx(X0.data(), HY.data(), N);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n * N; ++i) Y[i] = (HY[i] - cc * X0[i]) * (sigma1 / e);
    for (int k = 2; k <= m; ++k) {
      const double sigma2 = 1.0 / (gamma - sigma);
      c.hx(Y.data(), HY.data(), N);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n * N; ++i) {
        const double yn = (HY[i] - cc * Y[i]) * (2.0 * sigma2 / e) - (sigma * sigma2) * X0[i];
        X0[i] = Y[i];
        Y[i] = yn;
      }
      sigma = sigma2;
    }
    // S = Y^T Y, Cholesky, Y <- Y L^-T
    vector<double> S = gram(Y.data(), Y.data());
    vector<double> L((size_t)N * N, 0.0);
    for (int j = 0; j < N; ++j) {
      double d = S[(size_t)j * N + j];
      for (int k = 0; k < j; ++k) d -= L[(size_t)j * N + k] * L[(size_t)j * N + k];
      if (!(d > 0.0)) throw Error(INVDFT_BREAKDOWN, "overlap matrix not positive definite");
      L[(size_t)j * N + j] = std::sqrt(d);
      for (int i = j + 1; i < N; ++i) {
        double s = S[(size_t)i * N + j];
        for (int k = 0; k < j; ++k) s -= L[(size_t)i * N + k] * L[(size_t)j * N + k];
        L[(size_t)i * N + j] = s / L[(size_t)j * N + j];
      }
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
      double *y = &Y[r * N];
      for (int j = 0; j < N; ++j) {
        double s = y[j];
        for (int k = 0; k < j; ++k) s -= L[(size_t)j * N + k] * y[k];
        y[j] = s / L[(size_t)j * N + j];
      }
    }
    c.hx(Y.data(), HY.data(), N);
    vector<double> Hp = gram(Y.data(), HY.data());
    for (int i = 0; i < N; ++i)
      for (int j = i + 1; j < N; ++j) {
        const double v = 0.5 * (Hp[(size_t)i * N + j] + Hp[(size_t)j * N + i]);
        Hp[(size_t)i * N + j] = Hp[(size_t)j * N + i] = v;
      }
    vector<double> w, Q;
    sym_eig(N, Hp, w, Q);
    vector<double> part((size_t)kChunks * N, 0.0);
#pragma omp parallel for schedule(static)
    for (int ch = 0; ch < kChunks; ++ch) {
      const int64_t r0 = n * ch / kChunks, r1 = n * (ch + 1) / kChunks;
      vector<double> xr(N), hr(N);
      for (int64_t r = r0; r < r1; ++r) {
        for (int j = 0; j < N; ++j) {
          double xs = 0.0, hs = 0.0;
          for (int k = 0; k < N; ++k) {
            xs += Y[r * N + k] * Q[(size_t)k * N + j];
            hs += HY[r * N + k] * Q[(size_t)k * N + j];
          }
          xr[j] = xs;
          hr[j] = hs;
        }
        for (int j = 0; j < N; ++j) {
          c.X[r * N + j] = xr[j];
          const double rr = hr[j] - w[j] * xr[j];
          part[(size_t)ch * N + j] += rr * rr;
        }
      }
    }
    res.assign(N, 0.0);
    for (int ch = 0; ch < kChunks; ++ch)
      for (int j = 0; j < N; ++j) res[j] += part[(size_t)ch * N + j];
    for (auto &r : res) r = std::sqrt(std::max(r, 0.0));
    c.eig = w;
    c.have_eig = true;
  }

  vector<double> gram(const double *A, const double *Bm) const {
    const int N = c.N;
    const int64_t n = c.nn;
    vector<double> part((size_t)kChunks * N * N, 0.0);
#pragma omp parallel for schedule(static)
    for (int ch = 0; ch < kChunks; ++ch) {
      const int64_t r0 = n * ch / kChunks, r1 = n * (ch + 1) / kChunks;
      double *p = &part[(size_t)ch * N * N];
      for (int64_t r = r0; r < r1; ++r)
        for (int i = 0; i < N; ++i) {
          const double ai = A[r * N + i];
          for (int j = 0; j < N; ++j) p[i * N + j] += ai * Bm[r * N + j];
        }
    }
    vector<double> S((size_t)N * N, 0.0);
    for (int ch = 0; ch < kChunks; ++ch)
      for (int k = 0; k < N * N; ++k) S[k] += part[(size_t)ch * N * N + k];
    return S;
  }

  void solve(const double *pot, invdft_force_stats *st) {
    const invdft_params &P = c.prm;
    if (c.counter > 3) {
      const double prev = c.tol_cheb;
      c.tol_cheb = std::min(P.cheby_tol, c.loss_prev / P.adaptive_factor_cheb);
      c.tol_cheb = std::min(c.tol_cheb, prev);
    } else {
      c.tol_cheb = std::min(P.cheby_tol, P.initial_tol_cheb);
    }
    c.set_potential(pot);
    double lo, b;
    bounds(lo, b);
    const int m = P.cheb_degree > 0 ? P.cheb_degree : auto_degree(b);
    int passes = 0;
    double maxres = 0.0;
    vector<double> res;
    for (;;) {
      double a, a0;
      if (!c.have_eig) {
        a0 = lo;
        a = lo + 0.1 * (b - lo);
      } else {
        a0 = c.eig.front();
        a = c.eig.back();
      }
      pass(m, a, b, a0, res);
      c.mu = fermi_level(c.eig, c.ne, c.kT);
      c.occ.resize(c.N);
      int homo = 0;
      for (int i = 0; i < c.N; ++i) {
        c.occ[i] = occupancy(c.eig[i], c.mu, c.kT);
        if (c.eig[i] < c.mu + 1e-3 && homo < i) homo = i;
      }
      maxres = 0.0;
      for (int i = 0; i < c.N; ++i)
        if (c.occ[i] > P.frac_occ_tol || i <= homo + P.additional_states) maxres = std::max(maxres, res[i]);
      ++passes;
      if (!(maxres > c.tol_cheb && passes < P.max_cheb_passes)) break;
    }
    // nodal eigenvectors psi = C M^-1/2 X
    c.psi.resize((size_t)c.nn * c.N);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < c.nn; ++i)
      for (int j = 0; j < c.N; ++j) c.psi[i * c.N + j] = c.isqm[i] * c.X[i * c.N + j];
    c.cpsi.distribute(c.psi.data(), c.N);
    if (st) {
      st->passes = passes;
      st->max_residual = maxres;
      st->cheb_tol = c.tol_cheb;
      st->degree = m;
      st->upper_bound = b;
      st->fermi_energy = c.mu;
    }
  }
};

// ---------------------------------------------------------------------------
// adjoint problem (MultiVectorAdjointLinearSolverProblem) and block MINRES
// ---------------------------------------------------------------------------
struct Adjoint {
  Ctx &c;
  int B = 0;
  vector<double> psi, occ, eig, ujxw;
  vector<std::pair<int, int>> pairs;
  double mu = 0.0, eta = 0.0;
  explicit Adjoint(Ctx &cc) : c(cc) {}

  // updateInputPsi (:818-910)
  void update(const double *psi_block, int bw, const double *f, const double *e, double mu_in,
              const vector<vector<int>> &degen, const double *u) {
    B = bw;
    psi.assign(psi_block, psi_block + (size_t)c.nn * B);
    c.cpsi.distribute(psi.data(), B);
    occ.assign(f, f + B);
    eig.assign(e, e + B);
    mu = mu_in;
    pairs.clear();
    for (int i = 0; i < B; ++i)
      for (int j : degen[i]) pairs.push_back({i, j});
    ujxw.resize(c.nc * c.nd);
    for (int64_t q = 0; q < c.nc * c.nd; ++q) ujxw[q] = u[q] * c.jxw[q];
  }

  // per-pair sums over cells of sum_q w Q1[i] Q2[j], chunked over cells
  vector<double> pair_sums(const double *Q1, const double *Q2, const double *w) const {
    const int np = (int)pairs.size();
    const int64_t nq = c.nd;
    vector<double> part((size_t)kChunks * np, 0.0);
#pragma omp parallel for schedule(static)
    for (int ch = 0; ch < kChunks; ++ch) {
      const int64_t e0 = c.nc * ch / kChunks, e1 = c.nc * (ch + 1) / kChunks;
      for (int64_t e = e0; e < e1; ++e)
        for (int k = 0; k < np; ++k) {
          double s = 0.0;
          for (int64_t q = 0; q < nq; ++q) {
            const int64_t g = e * nq + q;
            s += Q1[g * B + pairs[k].first] * Q2[g * B + pairs[k].second] * w[g];
          }
          part[(size_t)ch * np + k] += s;
        }
    }
    vector<double> out(np, 0.0);
    for (int ch = 0; ch < kChunks; ++ch)
      for (int k = 0; k < np; ++k) out[k] += part[(size_t)ch * np + k];
    return out;
  }

  vector<double> mu_matrix(const vector<double> &f) const {
    vector<double> Q((size_t)c.nc * c.nd * B);
    c.to_quad(psi.data(), B, Q.data());
    const vector<double> v = pair_sums(Q.data(), Q.data(), ujxw.data());
    vector<double> Mu((size_t)B * B, 0.0);
    for (size_t k = 0; k < pairs.size(); ++k)
      Mu[(size_t)pairs[k].first * B + pairs[k].second] += 2.0 * f[pairs[k].first] * v[k];
    return Mu;
  }

  // computeRhs (:616-812)
  vector<double> rhs() const {
    const int64_t n = c.nn;
    vector<double> t(psi);
    c.cpsi.distribute(t.data(), B);
    for (int64_t i = 0; i < n; ++i)
      for (int b = 0; b < B; ++b) t[i * B + b] *= c.sqm[i];
    const vector<double> Mu = mu_matrix(occ);
    vector<double> r((size_t)n * B);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
      for (int j = 0; j < B; ++j) {
        double s = 0.0;
        for (int k = 0; k < B; ++k) s += t[i * B + k] * Mu[(size_t)k * B + j];
        r[i * B + j] = -2.0 * s;
      }
    for (int64_t i = 0; i < n; ++i)
      for (int b = 0; b < B; ++b) t[i * B + b] *= c.isqm[i];
    c.cpsi.distribute(t.data(), B);
    vector<double> t2((size_t)n * B);
    c.r_times(t.data(), ujxw.data(), B, t2.data());
    c.cpsi.slave_to_master(t2.data(), B);
    c.cpsi.distribute(t2.data(), B);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
      for (int b = 0; b < B; ++b) t2[i * B + b] *= c.isqm[i];
    c.cpsi.distribute(t2.data(), B);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n * B; ++i) r[i] += t2[i] * 4.0 * occ[i % B];
    c.cpsi.set_zero(r.data(), B);
    return r;
  }

  // vmult (:1346-1367): Ax = Ht x - eps x, constrained entries of x and Ax zero
  void vmult(double *x, double *Ax) {
    c.hx(x, Ax, B);
    c.cpsi.set_zero(x, B);
    c.cpsi.set_zero(Ax, B);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < c.nn * B; ++i) Ax[i] -= eig[i % B] * x[i];
  }

  // distributeX (:1003-1141)
  void distribute_x(double *x) {
    const int64_t n = c.nn;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
      for (int b = 0; b < B; ++b) x[i * B + b] *= c.isqm[i];
    c.cpsi.distribute(x, B);
    vector<double> Q1((size_t)c.nc * c.nd * B), Q2((size_t)c.nc * c.nd * B);
    c.to_quad(x, B, Q1.data());
    c.to_quad(psi.data(), B, Q2.data());
    const vector<double> dots = pair_sums(Q1.data(), Q2.data(), c.jxw.data());
    const vector<double> MuU = mu_matrix(vector<double>(B, 1.0));
    double sum_d = 0.0, eta_rhs = 0.0;
    for (int i = 0; i < B; ++i) {
      const double dfi = -occupancy_der(eig[i], mu, c.kT);
      sum_d += dfi;
      eta_rhs += dfi * MuU[(size_t)i * B + i];
    }
    eta = std::fabs(eta_rhs) < 1e-16 ? 0.0 : eta_rhs / sum_d;
    vector<double> coef(pairs.size());
    for (size_t k = 0; k < pairs.size(); ++k) {
      const int i = pairs[k].first, j = pairs[k].second;
      const double der = occupancy_der(eig[i], mu, c.kT);
      double corr = -der * MuU[(size_t)i * B + j];
      if (i == j) corr += der * eta;
      coef[k] = -dots[k] + corr;
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r)
      for (size_t k = 0; k < pairs.size(); ++k)
        x[r * B + pairs[k].first] += coef[k] * psi[r * B + pairs[k].second];
  }

  // preconditioned block MINRES, independent per column, zero start
  vector<int> minres(double *x, double tol, int maxit) {
    const int64_t n = c.nn;
    const size_t v = (size_t)n * B;
    vector<double> b = rhs();
    vector<double> r1(b), r2(b), y(v), w(v, 0.0), w2(v, 0.0), vv(v), yn(v);
    std::fill(x, x + v, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
      for (int j = 0; j < B; ++j) y[i * B + j] = c.diagA[i] * r1[i * B + j];
    vector<double> beta1(B);
    coldots(r1.data(), y.data(), n, B, beta1.data());
    vector<double> oldb(B, 0.0), beta(B), dbar(B, 0.0), epsln(B, 0.0), phibar(B), cs(B, -1.0), sn(B, 0.0);
    vector<char> active(B);
    vector<int> iters(B, 0);
    for (int j = 0; j < B; ++j) {
      beta1[j] = std::sqrt(std::max(beta1[j], 0.0));
      beta[j] = phibar[j] = beta1[j];
      active[j] = phibar[j] >= tol;
    }
    const double epsm = 2.220446049250313e-16;
    vector<double> alfa(B), betan2(B), s(B), c1(B), c2(B), phi(B), gam(B), oldeps(B), delta(B);
    vector<double> r2n(v), yp(v);
    for (int itn = 1; itn <= maxit; ++itn) {
      bool any = false;
      for (int j = 0; j < B; ++j) any = any || active[j];
      if (!any) break;
      for (int j = 0; j < B; ++j) s[j] = active[j] ? 1.0 / (beta[j] > 0 ? beta[j] : 1.0) : 0.0;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)v; ++i) vv[i] = y[i] * s[i % B];
      vmult(vv.data(), yn.data());
      if (itn >= 2) {
        for (int j = 0; j < B; ++j) c1[j] = beta[j] / (oldb[j] > 0 ? oldb[j] : 1.0);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)v; ++i) yn[i] -= c1[i % B] * r1[i];
      }
      coldots(vv.data(), yn.data(), n, B, alfa.data());
      for (int j = 0; j < B; ++j) c2[j] = alfa[j] / (beta[j] > 0 ? beta[j] : 1.0);
      // the new r2 (yn - alfa/beta r2) and its preconditioned copy
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i)
        for (int j = 0; j < B; ++j) {
          const double t = yn[i * B + j] - c2[j] * r2[i * B + j];
          r2n[i * B + j] = t;
          yp[i * B + j] = c.diagA[i] * t;
        }
      coldots(r2n.data(), yp.data(), n, B, betan2.data());
      vector<double> bn(B), epn(B), dbn(B), csn(B), snn(B), phbn(B);
      for (int j = 0; j < B; ++j) {
        bn[j] = std::sqrt(std::max(betan2[j], 0.0));
        oldeps[j] = epsln[j];
        delta[j] = cs[j] * dbar[j] + sn[j] * alfa[j];
        const double gbar = sn[j] * dbar[j] - cs[j] * alfa[j];
        epn[j] = sn[j] * bn[j];
        dbn[j] = -cs[j] * bn[j];
        gam[j] = std::max(std::sqrt(gbar * gbar + bn[j] * bn[j]), epsm);
        csn[j] = gbar / gam[j];
        snn[j] = bn[j] / gam[j];
        phi[j] = csn[j] * phibar[j];
        phbn[j] = snn[j] * phibar[j];
      }
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i)
        for (int j = 0; j < B; ++j) {
          if (!active[j]) continue;
          const size_t k = (size_t)i * B + j;
          const double wn = (vv[k] - oldeps[j] * w2[k] - delta[j] * w[k]) / gam[j];
          x[k] += phi[j] * wn;
          w2[k] = w[k];
          w[k] = wn;
          r1[k] = r2[k];
          r2[k] = r2n[k];
          y[k] = yp[k];
        }
      for (int j = 0; j < B; ++j) {
        if (!active[j]) continue;
        oldb[j] = beta[j];
        beta[j] = bn[j];
        epsln[j] = epn[j];
        dbar[j] = dbn[j];
        cs[j] = csn[j];
        sn[j] = snn[j];
        phibar[j] = phbn[j];
        iters[j] += 1;
        active[j] = phibar[j] >= tol;
      }
    }
    return iters;
  }
};

vector<vector<int>> degeneracy_map(const vector<double> &ev, double tol) {
  // InverseDFTSolverFunction.cpp:37-77
  const int n = (int)ev.size();
  std::map<int, std::set<int>> groups;
  std::map<int, int> group_of;
  int count = 0;
  for (int i = 0; i < n; ++i) {
    auto it = group_of.find(i);
    const int g = it != group_of.end() ? it->second : count;
    if (it == group_of.end()) {
      groups[g].insert(i);
      group_of[i] = g;
      ++count;
    }
    for (int j = 0; j < n; ++j)
      if (std::fabs(ev[i] - ev[j]) < tol) {
        groups[g].insert(j);
        group_of[j] = g;
      }
  }
  vector<vector<int>> out(n);
  for (int i = 0; i < n; ++i) {
    const auto &s = groups[group_of[i]];
    out[i].assign(s.begin(), s.end());
  }
  return out;
}

// ---------------------------------------------------------------------------
// getForceVector (InverseDFTSolverFunction.cpp:657-1311)
// ---------------------------------------------------------------------------
struct Force {
  Ctx &c;
  explicit Force(Ctx &cc) : c(cc) {}

  // psi (cols of block) and p at the child Gauss points; S += sum_i psi_i p_i
  void child_products(const double *psi, const double *pv, int B, vector<double> &S) {
    const int n1 = c.n1, nd = c.nd;
    const double g2[2] = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)};
#pragma omp parallel
    {
      vector<double> ue((size_t)nd * B), pe((size_t)nd * B);
      int64_t cur = -1;
#pragma omp for schedule(static)
      for (int64_t ch = 0; ch < c.ncc; ++ch) {
        const int64_t e = c.ch_parent[ch];
        if (e != cur) {
          for (int l = 0; l < nd; ++l)
            for (int b = 0; b < B; ++b) {
              ue[(size_t)l * B + b] = psi[c.cell_nodes[e * nd + l] * B + b];
              pe[(size_t)l * B + b] = pv[c.cell_nodes[e * nd + l] * B + b];
            }
          cur = e;
        }
        double L[3][2][16];
        for (int d = 0; d < 3; ++d)
          for (int t = 0; t < 2; ++t) {
            const double xi = c.ch_off[ch * 3 + d] + c.ch_scale[ch] * g2[t];
            for (int a = 0; a < n1; ++a) {
              double v = 1.0;
              for (int b2 = 0; b2 < n1; ++b2)
                if (b2 != a) v *= (xi - c.gll[b2]) / (c.gll[a] - c.gll[b2]);
              L[d][t][a] = v;
            }
          }
        for (int q = 0; q < 8; ++q) {
          const double *lx = L[0][q & 1], *ly = L[1][(q >> 1) & 1], *lz = L[2][(q >> 2) & 1];
          double acc = 0.0;
          for (int b = 0; b < B; ++b) {
            double su = 0.0, sp = 0.0;
            for (int k3 = 0; k3 < n1; ++k3)
              for (int k2 = 0; k2 < n1; ++k2) {
                const double wyz = ly[k2] * lz[k3];
                for (int k1 = 0; k1 < n1; ++k1) {
                  const int l = k1 + n1 * (k2 + n1 * k3);
                  su += lx[k1] * wyz * ue[(size_t)l * B + b];
                  sp += lx[k1] * wyz * pe[(size_t)l * B + b];
                }
              }
            acc += su * sp;
          }
          S[ch * 8 + q] += acc;
        }
      }
    }
  }

  // integrateWithShapeFunctionsForChildData (:1611-1674) + child condensation
  void project(const vector<double> &S, double *force) {
    const double g2[2] = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)};
    double Nq[8][8];
    for (int q = 0; q < 8; ++q)
      for (int k = 0; k < 8; ++k) {
        const double gx = g2[q & 1], gy = g2[(q >> 1) & 1], gz = g2[(q >> 2) & 1];
        Nq[q][k] = ((k & 1) ? gx : 1.0 - gx) * ((k & 2) ? gy : 1.0 - gy) * ((k & 4) ? gz : 1.0 - gz);
      }
    vector<double> local((size_t)c.ncc * 8);
#pragma omp parallel for schedule(static)
    for (int64_t ch = 0; ch < c.ncc; ++ch)
      for (int k = 0; k < 8; ++k) {
        double s = 0.0;
        for (int q = 0; q < 8; ++q) s += S[ch * 8 + q] * c.ch_jxw[ch * 8 + q] * Nq[q][k];
        local[ch * 8 + k] = s;
      }
#pragma omp parallel for schedule(static)
    for (int64_t nidx = 0; nidx < c.ncn; ++nidx) {
      double s = 0.0;
      for (int64_t k = c.cptr[nidx]; k < c.cptr[nidx + 1]; ++k) s += local[c.cent[k]];
      force[nidx] = s;
    }
    c.cchild.slave_to_master(force, 1);
  }

  void eval(double *pot, double *force, double *loss, invdft_force_stats *st) {
    const invdft_params &P = c.prm;
    std::memset(st, 0, sizeof(*st));
    c.n_hx = c.n_hx_cols = 0;
    for (int64_t i = 0; i < c.ncn; ++i)
      if (!std::isfinite(pot[i])) throw Error(INVDFT_NONFINITE, "non-finite entry in the potential");
    c.cchild.distribute(pot, 1);
    Eigen eg(c);
    eg.solve(pot, st);
    // density, drho, loss (:748-912)
    const int64_t nqt = c.nc * c.nd;
    const int N = c.N;
    vector<double> Q((size_t)nqt * N);
    c.to_quad(c.psi.data(), N, Q.data());
    c.rho.resize(nqt);
    c.u.resize(nqt);
    double sums[4] = {0, 0, 0, 0};
    {
      vector<double> part((size_t)kChunks * 4, 0.0);
#pragma omp parallel for schedule(static)
      for (int ch = 0; ch < kChunks; ++ch) {
        const int64_t q0 = nqt * ch / kChunks, q1 = nqt * (ch + 1) / kChunks;
        for (int64_t q = q0; q < q1; ++q) {
          double r = 0.0;
          for (int i = 0; i < N; ++i) r += 2.0 * c.occ[i] * Q[q * N + i] * Q[q * N + i];
          c.rho[q] = r;
          const double d = c.rho_t[q] - 0.5 * r;
          c.u[q] = d * c.weight[q];
          part[ch * 4 + 0] += d * d * c.weight[q] * c.jxw[q];
          part[ch * 4 + 1] += d * d * c.jxw[q];
          part[ch * 4 + 2] += std::fabs(d * c.jxw[q]);
          part[ch * 4 + 3] += c.vks[q] * r * c.jxw[q];
        }
      }
      for (int ch = 0; ch < kChunks; ++ch)
        for (int k = 0; k < 4; ++k) sums[k] += part[ch * 4 + k];
    }
    st->loss = sums[0];
    st->loss_unweighted = sums[1];
    st->l1_error = sums[2];
    st->int_rho_veff = sums[3];
    // adjoint blocks
    vector<double> S((size_t)c.ncc * 8, 0.0);
    const int block = P.block_size > 0 ? P.block_size : N;
    int jvec = 0, itmax = 0, nblk = 0;
    int64_t itsum = 0;
    Adjoint ad(c);
    while (jvec < N) {
      int bs = std::min(block, N - jvec);
      for (;;) {
        const int last = jvec + bs - 1;
        if (last + 1 != N && std::fabs(c.eig[last] - c.eig[last + 1]) < P.degeneracy_tol) --bs;
        else break;
      }
      if (bs < 1) throw Error(INVDFT_BAD_ARG, "degenerate group wider than the block size");
      vector<double> shifts(c.eig.begin() + jvec, c.eig.begin() + jvec + bs);
      vector<double> focc(c.occ.begin() + jvec, c.occ.begin() + jvec + bs);
      vector<double> pb((size_t)c.nn * bs);
      for (int64_t i = 0; i < c.nn; ++i)
        for (int j = 0; j < bs; ++j) pb[i * bs + j] = c.psi[i * N + jvec + j];
      ad.update(pb.data(), bs, focc.data(), shifts.data(), c.mu, degeneracy_map(shifts, P.degeneracy_tol),
                c.u.data());
      c.adjoint_tol = std::min(c.adjoint_tol, c.tol_cheb / P.adaptive_factor_adjoint);
      vector<double> x((size_t)c.nn * bs);
      const vector<int> its = ad.minres(x.data(), c.adjoint_tol, P.adjoint_max_iter);
      ad.distribute_x(x.data());
      for (int i : its) {
        itmax = std::max(itmax, i);
        itsum += i;
      }
      c.cadj.distribute(x.data(), bs);
      child_products(ad.psi.data(), x.data(), bs, S);
      jvec += bs;
      ++nblk;
    }
    project(S, force);
    c.cchild.set_zero(force, 1);
    c.cchild.set_zero(pot, 1);
    *loss = sums[0];
    c.loss_prev = sums[0];
    ++c.counter;
    st->adjoint_tol = c.adjoint_tol;
    st->minres_iters_max = itmax;
    st->minres_iters_sum = itsum;
    st->n_blocks = nblk;
    st->n_hx_calls = (int32_t)c.n_hx;
    st->n_hx_columns = c.n_hx_cols;
  }
};

Ctx *create(const invdft_problem_desc *d, const invdft_params *pp) {
  if (!d || !pp) throw Error(INVDFT_BAD_ARG, "null problem or parameters");
  auto c = std::make_unique<Ctx>();
  c->prm = *pp;
  c->p = d->p;
  c->n1 = d->p + 1;
  c->nd = c->n1 * c->n1 * c->n1;
  c->nc = d->n_cells;
  c->nn = d->n_nodes;
  c->ncc = d->n_child_cells;
  c->ncn = d->n_child_nodes;
  c->N = d->n_states;
  c->ne = d->n_electrons;
  c->kT = kKb * d->temperature;
  if (c->N < 1 || c->N > 64) throw Error(INVDFT_BAD_ARG, "n_states must be in [1, 64]");
  const int n1 = c->n1, nd = c->nd;
  c->gll.assign(d->gll_nodes, d->gll_nodes + n1);
  vector<double> gp(d->gauss_points, d->gauss_points + n1);
  c->wq.assign(d->gauss_weights, d->gauss_weights + n1);
  vector<double> wg(d->gll_weights, d->gll_weights + n1);
  c->phi.resize(n1 * n1);
  c->dq.resize(n1 * n1);
  vector<double> dphi(n1 * n1);
  for (int q = 0; q < n1; ++q) {
    const vector<double> v = lagrange(c->gll, gp[q]), dv = lagrange_d(gp, gp[q]), dl = lagrange_d(c->gll, gp[q]);
    for (int a = 0; a < n1; ++a) {
      c->phi[q * n1 + a] = v[a];
      c->dq[q * n1 + a] = dv[a];
      dphi[q * n1 + a] = dl[a];
    }
  }
  c->cell_nodes.assign(d->cell_nodes, d->cell_nodes + c->nc * nd);
  for (int64_t t = 0; t < c->nc * nd; ++t)
    if (c->cell_nodes[t] < 0 || c->cell_nodes[t] >= c->nn) throw Error(INVDFT_BAD_ARG, "cell node out of range");
  const int64_t nqt = c->nc * nd;
  c->cell_h.assign(d->cell_h, d->cell_h + c->nc);
  c->jxw.assign(d->jxw, d->jxw + nqt);
  c->v_base.assign(d->v_base, d->v_base + nqt);
  if (d->v_lda) c->v_lda.assign(d->v_lda, d->v_lda + nqt);
  else c->v_lda.assign(nqt, 0.0);
  c->rho_t.assign(d->rho_target_up, d->rho_target_up + nqt);
  c->weight.assign(d->weight, d->weight + nqt);
  c->cpsi.load(d->cons_psi, c->nn);
  c->cadj.load(d->cons_adj, c->nn);
  c->cchild.load(d->cons_child, c->ncn);
  // lumped mass and stiffness diagonal, condensed
  vector<double> M1(n1 * n1, 0.0), S1(n1 * n1, 0.0);
  for (int a = 0; a < n1; ++a)
    for (int b = 0; b < n1; ++b)
      for (int q = 0; q < n1; ++q) {
        M1[a * n1 + b] += c->phi[q * n1 + a] * c->wq[q] * c->phi[q * n1 + b];
        S1[a * n1 + b] += dphi[q * n1 + a] * c->wq[q] * dphi[q * n1 + b];
      }
  c->mass.assign(c->nn, 0.0);
  vector<double> kd(c->nn, 0.0);
  for (int64_t e = 0; e < c->nc; ++e) {
    const double h = c->cell_h[e];
    for (int l = 0; l < nd; ++l) {
      const int a = l % n1, b = (l / n1) % n1, cc = l / (n1 * n1);
      const double kll = S1[a * n1 + a] * M1[b * n1 + b] * M1[cc * n1 + cc] +
                         M1[a * n1 + a] * S1[b * n1 + b] * M1[cc * n1 + cc] +
                         M1[a * n1 + a] * M1[b * n1 + b] * S1[cc * n1 + cc];
      const int64_t nidx = c->cell_nodes[e * nd + l];
      c->mass[nidx] += h * h * h * wg[a] * wg[b] * wg[cc];
      kd[nidx] += h * kll;
    }
  }
  c->cpsi.slave_to_master(c->mass.data(), 1);
  c->cpsi.slave_to_master(kd.data(), 1);
  c->sqm.resize(c->nn);
  c->isqm.resize(c->nn);
  c->diagA.resize(c->nn);
  for (int64_t i = 0; i < c->nn; ++i) {
    const double m = c->mass[i];
    c->sqm[i] = std::sqrt(m);
    c->isqm[i] = m > 0.0 ? 1.0 / std::sqrt(m) : 0.0;
    const double ik = kd[i] > 0.0 ? 1.0 / kd[i] : 0.0;
    c->diagA[i] = (1.0 / 0.5) * ik * c->sqm[i] * c->sqm[i];
  }
  c->free_row.assign(c->nn, 1);
  for (int64_t r : c->cpsi.rows) c->free_row[r] = 0;
  // assembly CSR: node -> cell entries in entry order
  {
    vector<int64_t> cnt(c->nn + 1, 0);
    for (int64_t t = 0; t < nqt; ++t) cnt[c->cell_nodes[t] + 1]++;
    for (int64_t i = 0; i < c->nn; ++i) cnt[i + 1] += cnt[i];
    c->aptr = cnt;
    c->aent.resize(nqt);
    vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t t = 0; t < nqt; ++t) c->aent[fill[c->cell_nodes[t]]++] = t;
  }
  // greedy colouring of the cells: two cells that share a node differ in colour
  {
    vector<int> color(c->nc, -1);
    vector<int64_t> stamp(64, -1);
    int ncol = 0;
    for (int64_t e = 0; e < c->nc; ++e) {
      for (int l = 0; l < nd; ++l) {
        const int64_t nidx = c->cell_nodes[e * nd + l];
        for (int64_t k = c->aptr[nidx]; k < c->aptr[nidx + 1]; ++k) {
          const int co = color[c->aent[k] / nd];
          if (co >= 0) {
            if (co >= (int)stamp.size()) stamp.resize(co + 1, -1);
            stamp[co] = e;
          }
        }
      }
      int co = 0;
      while (co < (int)stamp.size() && stamp[co] == e) ++co;
      color[e] = co;
      ncol = std::max(ncol, co + 1);
      if (co >= (int)stamp.size()) stamp.resize(co + 1, -1);
    }
    c->color_ptr.assign(ncol + 1, 0);
    for (int64_t e = 0; e < c->nc; ++e) c->color_ptr[color[e] + 1]++;
    for (int k = 0; k < ncol; ++k) c->color_ptr[k + 1] += c->color_ptr[k];
    c->color_cells.resize(c->nc);
    vector<int64_t> fill(c->color_ptr.begin(), c->color_ptr.end() - 1);
    for (int64_t e = 0; e < c->nc; ++e) c->color_cells[fill[color[e]]++] = e;
  }
  c->w3.resize(nd);
  for (int q = 0; q < nd; ++q) c->w3[q] = c->wq[q % n1] * c->wq[(q / n1) % n1] * c->wq[q / (n1 * n1)];
  // child mesh
  c->ch_nodes.assign(d->child_cell_nodes, d->child_cell_nodes + c->ncc * 8);
  c->ch_parent.assign(d->child_parent, d->child_parent + c->ncc);
  c->ch_jxw.assign(d->child_jxw, d->child_jxw + c->ncc * 8);
  c->ch_off.assign(d->child_offset, d->child_offset + c->ncc * 3);
  c->ch_scale.assign(d->child_scale, d->child_scale + c->ncc);
  c->pq_child.assign(d->pq_child, d->pq_child + nqt);
  c->pq_xi.assign(d->pq_xi, d->pq_xi + nqt * 3);
  for (int64_t t = 0; t < c->ncc * 8; ++t)
    if (c->ch_nodes[t] < 0 || c->ch_nodes[t] >= c->ncn) throw Error(INVDFT_BAD_ARG, "child node out of range");
  for (int64_t q = 0; q < nqt; ++q)
    if (c->pq_child[q] < 0 || c->pq_child[q] >= c->ncc) throw Error(INVDFT_BAD_ARG, "pq_child out of range");
  {
    vector<int64_t> cnt(c->ncn + 1, 0);
    for (int64_t t = 0; t < c->ncc * 8; ++t) cnt[c->ch_nodes[t] + 1]++;
    for (int64_t i = 0; i < c->ncn; ++i) cnt[i + 1] += cnt[i];
    c->cptr = cnt;
    c->cent.resize(c->ncc * 8);
    vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t t = 0; t < c->ncc * 8; ++t) c->cent[fill[c->ch_nodes[t]]++] = t;
  }
  // start subspace X[i][j] = hash_uniform(i N + j, 11) on free rows
  c->X.assign((size_t)c->nn * c->N, 0.0);
  for (int64_t i = 0; i < c->nn; ++i)
    if (c->free_row[i])
      for (int j = 0; j < c->N; ++j) c->X[i * c->N + j] = hash_uniform((uint64_t)(i * c->N + j), 11);
  c->adjoint_tol = c->prm.adjoint_initial_tol;
  return c.release();
}

}  // namespace ocpu

// ---------------------------------------------------------------------------
// C ABI of the CPU restatement (plain pointers, status codes of invdft_status)
// ---------------------------------------------------------------------------
template <class F> static int ocpu_guard(F &&f) {
  try {
    f();
    return 0;
  } catch (const ocpu::Error &e) {
    ocpu::g_err = e.what();
    return e.code;
  } catch (const std::exception &e) {
    ocpu::g_err = e.what();
    return INVDFT_BAD_ARG;
  }
}

extern "C" {

const char *ocpu_last_error(void) { return ocpu::g_err.c_str(); }

void ocpu_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}
int ocpu_max_threads(void) { return omp_get_max_threads(); }


int ocpu_create(const invdft_problem_desc *d, const invdft_params *p, void **ctx) {
  return ocpu_guard([&] { *ctx = ocpu::create(d, p); });
}

void ocpu_destroy(void *ctx) { delete static_cast<ocpu::Ctx *>(ctx); }

int ocpu_force_eval(void *ctx, double *pot, double *force, double *loss, invdft_force_stats *st) {
  return ocpu_guard([&] {
    invdft_force_stats local;
    ocpu::Force f(*static_cast<ocpu::Ctx *>(ctx));
    f.eval(pot, force, loss, st ? st : &local);
  });
}

// forward half only: distribute pot, solveEigen, psi kept in the context
int ocpu_solve_eigen(void *ctx, double *pot, invdft_force_stats *st) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    c.cchild.distribute(pot, 1);
    invdft_force_stats local{};
    ocpu::Eigen(c).solve(pot, st ? st : &local);
  });
}

// the evaluation state a caller hands over from another implementation, so
// that the next evaluation repeats exactly the work that one did next: the
// start subspace from nodal eigenvectors psi [n_nodes][N] (X = M^1/2 psi on
// free rows) with its Ritz values eig [N], the evaluation counter and last
// loss of the adaptive Chebyshev tolerance (:1336-1347) and the tolerances
// reached so far
int ocpu_set_state(void *ctx, const double *psi, const double *eig, int counter, double loss_prev,
                   double tol_cheb, double adjoint_tol) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    if (psi) {
      for (int64_t i = 0; i < c.nn; ++i)
        for (int j = 0; j < c.N; ++j) c.X[i * c.N + j] = c.free_row[i] ? c.sqm[i] * psi[i * c.N + j] : 0.0;
      c.have_eig = false;
    }
    if (eig) {   // Ritz values of that subspace: the filter bounds of the next pass
      c.eig.assign(eig, eig + c.N);
      c.have_eig = true;
    }
    c.counter = counter;
    c.loss_prev = loss_prev;
    if (tol_cheb > 0.0) c.tol_cheb = tol_cheb;
    if (adjoint_tol > 0.0) c.adjoint_tol = adjoint_tol;
  });
}

// the spectrum bounds of solveEigen's Lanczos run with `steps` steps at the
// current potential (set_potential first)
int ocpu_lanczos_bounds(void *ctx, int steps, double *lo, double *hi) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    if (c.vj.empty()) throw ocpu::Error(INVDFT_NOT_READY, "no potential set");
    const int keep = c.prm.lanczos_steps;
    c.prm.lanczos_steps = steps;
    ocpu::Eigen(c).bounds(*lo, *hi);
    c.prm.lanczos_steps = keep;
  });
}

int ocpu_set_potential(void *ctx, const double *pot) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    std::vector<double> v(pot, pot + c.ncn);
    c.cchild.distribute(v.data(), 1);
    c.set_potential(v.data());
  });
}

int ocpu_hx(void *ctx, const double *x, double *y, int B) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    if (c.vj.empty()) throw ocpu::Error(INVDFT_NOT_READY, "no potential set");
    if (B < 1 || B > 64) throw ocpu::Error(INVDFT_BAD_ARG, "B must be in [1, 64]");
    c.hx(x, y, B);
  });
}

int ocpu_get_eigen(void *ctx, double *eig, double *occ, double *mu) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    if (!c.have_eig) throw ocpu::Error(INVDFT_NOT_READY, "no eigensolve yet");
    std::copy(c.eig.begin(), c.eig.end(), eig);
    if (occ && !c.occ.empty()) std::copy(c.occ.begin(), c.occ.end(), occ);
    if (mu) *mu = c.mu;
  });
}

int ocpu_get_psi(void *ctx, double *psi) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    if (c.psi.empty()) throw ocpu::Error(INVDFT_NOT_READY, "no eigensolve yet");
    std::copy(c.psi.begin(), c.psi.end(), psi);
  });
}

// total density at the parent quadrature points of the current psi
int ocpu_density(void *ctx, double *rho) {
  return ocpu_guard([&] {
    ocpu::Ctx &c = *static_cast<ocpu::Ctx *>(ctx);
    if (c.psi.empty()) throw ocpu::Error(INVDFT_NOT_READY, "no eigensolve yet");
    const int64_t nqt = c.nc * c.nd;
    std::vector<double> Q((size_t)nqt * c.N);
    c.to_quad(c.psi.data(), c.N, Q.data());
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < nqt; ++q) {
      double r = 0.0;
      for (int i = 0; i < c.N; ++i) r += 2.0 * c.occ[i] * Q[q * c.N + i] * Q[q * c.N + i];
      rho[q] = r;
    }
  });
}

}  // extern "C"
