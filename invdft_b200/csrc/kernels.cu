// Device kernels of the invDFT force evaluation, FP64 path, sm_100a.
//
// Layout conventions: multi-vectors are [node][B] (B fastest); cell blocks are
// [cell][local node][B]; quadrature blocks are [cell][q][B]; cell matrices are
// stored column-major per cell, H[e][j][i], so that thread i of a CTA streams
// column j of H_e with unit stride.
#include "kernels.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <string>
#include <atomic>

namespace invdft {

namespace {
constexpr int NT = 256;

__device__ __forceinline__ double mat1d(const double *A, bool trans, int n1, int q, int a) {
  return trans ? A[a * n1 + q] : A[q * n1 + a];
}

// Three-pass tensor-product contraction on a [n1^3][CH] block held in shared
// memory: out = (A (x) A (x) A) in, or with A^T when trans.  Result lands in t1.
__device__ void tensor3(const double *A, bool trans, const double *in, double *t1, double *t2,
                        int n1, int CH) {
  const int n2 = n1 * n1, n3 = n2 * n1, tot = n3 * CH;
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int k = idx % CH, pt = idx / CH, q = pt % n1, bc = pt / n1;
    double s = 0.0;
    for (int a = 0; a < n1; ++a) s = fma(mat1d(A, trans, n1, q, a), in[(a + n1 * bc) * CH + k], s);
    t1[idx] = s;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int k = idx % CH, pt = idx / CH, q1 = pt % n1, q2 = (pt / n1) % n1, c = pt / n2;
    double s = 0.0;
    for (int b = 0; b < n1; ++b) s = fma(mat1d(A, trans, n1, q2, b), t1[(q1 + n1 * b + n2 * c) * CH + k], s);
    t2[idx] = s;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int k = idx % CH, pt = idx / CH, q12 = pt % n2, q3 = pt / n2;
    double s = 0.0;
    for (int c = 0; c < n1; ++c) s = fma(mat1d(A, trans, n1, q3, c), t2[(q12 + n2 * c) * CH + k], s);
    t1[idx] = s;
  }
  __syncthreads();
}


// One entry of the cell block X_e (row l, column b) of the gather: the
// Lowdin-scaled and hanging-distributed value, or the plain nodal value.
__device__ __forceinline__ double gather_value(const FeView &fe, const double *__restrict__ x, int64_t e, int l,
                                               int b, int B, int mode) {
  const int nd = fe.nd;
  if (mode == GATHER_PLAIN) return x[(int64_t)fe.cell_nodes[e * nd + l] * B + b];
  const int m = fe.cell_map[e * nd + l];
  if (m >= 0) return x[(int64_t)m * B + b] * fe.inv_sqrt_mass[m];
  const int r = -m - 1;
  double v = 0.0;
  for (int k = fe.cons_ptr[r]; k < fe.cons_ptr[r + 1]; ++k)
    v = fma(fe.cons_gw[k], x[(int64_t)fe.cons_masters[k] * B + b], v);
  return v;
}

// X_e into shared memory as [rows][ld] (rows >= nd, columns >= B zero), with
// eight independent load chains in flight per thread.
__device__ __forceinline__ void gather_cell_block(const FeView &fe, const double *__restrict__ x, int64_t e,
                                                  int B, int ld, int rows, int mode, double *xs) {
  constexpr int U = 8;
  const int total = rows * ld;
  for (int base = threadIdx.x; base < total; base += blockDim.x * U) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base + u * blockDim.x;
      const int l = idx / ld, b = idx - l * ld;
      v[u] = (idx < total && b < B && l < fe.nd) ? gather_value(fe, x, e, l, b, B, mode) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base + u * blockDim.x;
      if (idx < total) xs[idx] = v[u];
    }
  }
}

// dst[0..n) = src[0..n) with eight loads in flight per thread
template <typename T>
__device__ __forceinline__ void stage_copy(T *dst, const T *__restrict__ src, int n) {
  constexpr int U = 8;
  for (int base = threadIdx.x; base < n; base += blockDim.x * U) {
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = base + u * blockDim.x;
      v[u] = i < n ? src[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = base + u * blockDim.x;
      if (i < n) dst[i] = v[u];
    }
  }
}

// ---------------------------------------------------------------------------
// Cell Hamiltonian H_e = 1/2 h K_ref + N^T diag(v JxW) N by sum factorisation.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) build_cell_h_kernel(int n1, int ldh, const double *__restrict__ phi,
                                                          const double *__restrict__ vks,
                                                          const double *__restrict__ jxw,
                                                          const double *__restrict__ Kref,
                                                          const double *__restrict__ cell_h,
                                                          double *__restrict__ H) {
  extern __shared__ double sm[];
  const int n2 = n1 * n1, nq = n2 * n1, nd = nq;
  double *w = sm;
  double *P = w + nq;            // [cc'][q]
  double *T1 = P + n2 * n1;      // [(q1 n1 + q2)][cc']
  double *T2 = T1 + n2 * n2;     // [(q1 n2 + bb')][cc']
  const int64_t e = blockIdx.x;
  for (int q = threadIdx.x; q < nq; q += blockDim.x) w[q] = vks[e * nq + q] * jxw[e * nq + q];
  for (int t = threadIdx.x; t < n2 * n1; t += blockDim.x) {
    const int cc = t / n1, q = t % n1;
    P[t] = phi[q * n1 + cc / n1] * phi[q * n1 + cc % n1];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < n2 * n2; t += blockDim.x) {
    const int q12 = t / n2, cc = t % n2, q1 = q12 / n1, q2 = q12 % n1;
    double s = 0.0;
    for (int q3 = 0; q3 < n1; ++q3) s = fma(P[cc * n1 + q3], w[q1 + n1 * q2 + n2 * q3], s);
    T1[t] = s;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < n1 * n2 * n2; t += blockDim.x) {
    const int cc = t % n2, r = t / n2, bb = r % n2, q1 = r / n2;
    double s = 0.0;
    for (int q2 = 0; q2 < n1; ++q2) s = fma(P[bb * n1 + q2], T1[(q1 * n1 + q2) * n2 + cc], s);
    T2[t] = s;
  }
  __syncthreads();
  const double hh = 0.5 * cell_h[e];
  double *He = H + e * (int64_t)((nd + 1) >> 1) * 2 * ldh;
  for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) {
    const int j = t / nd, i = t % nd;
    const int a = i % n1, b = (i / n1) % n1, c = i / n2;
    const int ap = j % n1, bp = (j / n1) % n1, cp = j / n2;
    const int aa = a * n1 + ap, bb = b * n1 + bp, cc = c * n1 + cp;
    double s = 0.0;
    for (int q1 = 0; q1 < n1; ++q1) s = fma(P[aa * n1 + q1], T2[(q1 * n2 + bb) * n2 + cc], s);
    He[(int64_t)(j >> 1) * 2 * ldh + 2 * i + (j & 1)] = fma(hh, Kref[t], s);
  }
  // zero the padding row (i = nd) and, for odd nd, the padding column (j = nd)
  if (ldh > nd)
    for (int j = threadIdx.x; j < nd; j += blockDim.x) He[(int64_t)(j >> 1) * 2 * ldh + 2 * nd + (j & 1)] = 0.0;
  if (nd & 1)
    for (int i = threadIdx.x; i < ldh; i += blockDim.x) He[(int64_t)(nd >> 1) * 2 * ldh + 2 * i + 1] = 0.0;
}

// ---------------------------------------------------------------------------
// HX, part 1: Y_e = H_e X_e with the constrained gather fused in.
// One CTA per cell; thread i owns row i and BC accumulators.
// ---------------------------------------------------------------------------
template <int BC, int R>
__global__ void __launch_bounds__(NT) hx_cell_gemm_kernel(FeView fe, const double *__restrict__ H,
                                                          const double *__restrict__ x,
                                                          double *__restrict__ Ycell, int B, int mode) {
  // Thread t owns rows R*t .. R*t+R-1 of H_e (register blocking: every vector
  // value read from shared memory feeds R*2 FMAs per column pair) and streams
  // them as 16-byte column-pair loads, R*16 contiguous bytes per thread.
  extern __shared__ double xs[];  // [2*ncp][BC], rows beyond nd zero
  const int nd = fe.nd;
  const int ncp = (nd + 1) >> 1;
  const int64_t e = blockIdx.x;
  for (int idx = threadIdx.x; idx < 2 * ncp * BC; idx += blockDim.x) {
    const int l = idx / BC, b = idx - l * BC;
    double v = 0.0;
    if (b < B && l < nd) {
      if (mode == GATHER_PLAIN) {
        const int m = fe.cell_nodes[e * nd + l];
        v = x[(int64_t)m * B + b];
      } else {
        const int m = fe.cell_map[e * nd + l];
        if (m >= 0) {
          v = x[(int64_t)m * B + b] * fe.inv_sqrt_mass[m];
        } else {
          const int r = -m - 1;
          for (int k = fe.cons_ptr[r]; k < fe.cons_ptr[r + 1]; ++k)
            v = fma(fe.cons_gw[k], x[(int64_t)fe.cons_masters[k] * B + b], v);
        }
      }
    }
    xs[idx] = v;
  }
  __syncthreads();
  const int r0 = R * threadIdx.x;
  if (r0 >= nd) return;
  double acc[R][BC];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int b = 0; b < BC; ++b) acc[r][b] = 0.0;
  // rows r0..r0+R-1 are < ldh (ldh >= nd rounded up to even, R divides the
  // padded row count handled below), so the loads stay inside the cell block
  const double2 *Hc = reinterpret_cast<const double2 *>(H + e * (int64_t)ncp * 2 * fe.ldh) + r0;
#pragma unroll 2
  for (int jp = 0; jp < ncp; ++jp) {
    double2 h[R];
#pragma unroll
    for (int r = 0; r < R; ++r) h[r] = (r0 + r < fe.ldh) ? __ldcs(Hc + (int64_t)jp * fe.ldh + r) : make_double2(0.0, 0.0);
    const double *xr = xs + 2 * jp * BC;
#pragma unroll
    for (int b = 0; b < BC; b += 2) {
      const double2 x0 = *reinterpret_cast<const double2 *>(xr + b);
      const double2 x1 = *reinterpret_cast<const double2 *>(xr + BC + b);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        acc[r][b] = fma(h[r].x, x0.x, acc[r][b]);
        acc[r][b + 1] = fma(h[r].x, x0.y, acc[r][b + 1]);
        acc[r][b] = fma(h[r].y, x1.x, acc[r][b]);
        acc[r][b + 1] = fma(h[r].y, x1.y, acc[r][b + 1]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = r0 + r;
    if (i < nd) {
      const int sl = fe.slot_of[e * nd + i];
      if (sl >= 0) {
        double *yo = Ycell + (int64_t)sl * B;
#pragma unroll
        for (int b = 0; b < BC; ++b)
          if (b < B) yo[b] = acc[r][b];
      }
    }
  }
}


// ---------------------------------------------------------------------------
// HX, part 1, FP64 tensor-core variant: Y_e = H_e X_e with mma.sync m8n8k4 f64
// (the FP64 tensor path of sm_100a; tcgen05 has no f64 kind).  One CTA per
// cell, warp w owns 8-row tiles m = w, w+nwarps, ...; for every k-step of 4
// columns each thread loads one double of H_e (a warp reads two contiguous
// 128-byte column-pair segments) and one double of X_e from shared memory.
// ---------------------------------------------------------------------------
template <int NTILE, typename MT>
__global__ void __launch_bounds__(NT) hx_cell_dmma_kernel(FeView fe, const MT *__restrict__ H,
                                                          const double *__restrict__ x,
                                                          double *__restrict__ Ycell, int B, int mode) {
  extern __shared__ double xs[];  // [kpad][BP] with BP = 8*NTILE, zero padded
  constexpr int BP = 8 * NTILE;
  const int nd = fe.nd, ldh = fe.ldh;
  const int ncol = 2 * ((nd + 1) >> 1);          // stored columns (pair layout)
  const int ksteps = (nd + 3) >> 2;
  const int kpad = 4 * ksteps;
  const int64_t e = blockIdx.x;
  gather_cell_block(fe, x, e, B, BP, kpad, mode, xs);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const MT *He = H + e * (int64_t)(ncol >> 1) * 2 * ldh;
  const int mtiles = (nd + 7) >> 3;
  for (int mt = warp; mt < mtiles; mt += nwarps) {
    const int row = 8 * mt + g;
    const bool row_ok = row < ldh;
    double c[NTILE][2];
#pragma unroll
    for (int n = 0; n < NTILE; ++n) c[n][0] = c[n][1] = 0.0;
    // two-stage register pipeline: the next U k-steps of H are in flight while
    // the current U feed the tensor core
    constexpr int U = 8;
    auto load_a = [&](int ks) -> double {
      const int k = 4 * ks + t;
      return (row_ok && ks < ksteps && k < ncol)
                 ? (double)__ldcs(He + (int64_t)(k >> 1) * 2 * ldh + 2 * row + (k & 1))
                 : 0.0;
    };
    double a0[U], a1[U];
#pragma unroll
    for (int u = 0; u < U; ++u) a0[u] = load_a(u);
    for (int ks0 = 0; ks0 < ksteps; ks0 += U) {
#pragma unroll
      for (int u = 0; u < U; ++u) a1[u] = load_a(ks0 + U + u);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = 4 * (ks0 + u) + t;
        if (ks0 + u < ksteps) {
#pragma unroll
          for (int n = 0; n < NTILE; ++n) {
            const double bv = xs[k * BP + 8 * n + g];   // B[t][g] = X_e[k][8n+g]
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                         : "+d"(c[n][0]), "+d"(c[n][1])
                         : "d"(a0[u]), "d"(bv));
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) a0[u] = a1[u];
    }
    if (row < nd) {
      const int sl = fe.slot_of[e * nd + row];
      if (sl >= 0) {
        double *yo = Ycell + (int64_t)sl * B;
#pragma unroll
        for (int n = 0; n < NTILE; ++n) {
          const int col = 8 * n + 2 * t;
          if (col < B) yo[col] = c[n][0];
          if (col + 1 < B) yo[col + 1] = c[n][1];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// HX, part 1, matrix-free variant: Y_e = H_e X_e by sum factorisation, never
// forming H_e.  With u the cell values on the GLL nodes, Gauss-point values
// uq = (phi (x) phi (x) phi) u, collocation derivatives g_d = Dq_d uq, and
// per-point weights, H_e u = phi3^T (vJ uq) + 1/2 h sum_d phi3^T Dq_d^T (W3 g_d),
// which equals (1/2 h K_ref + N^T diag(v JxW) N) u in exact arithmetic (the
// (p+1)-point Gauss rule integrates every product in the stiffness exactly).
// 12 N^4 FMAs per (cell, column) instead of 2 N^6, and no cell-matrix traffic:
// the kernel is bound by the FP64 pipes and shared memory, not by HBM.
//
// A CTA holds 16 (cell, column) pairs: C columns of 16/C consecutive cells.
// Shared arrays are [point][pair], so a warp (16 pairs x 2 tensor lines)
// touches two 128-byte rows per access, free of bank conflicts.  Thread
// (pair p, line L) owns tensor line L in every stage; the direction of the
// line changes between stages.
// ---------------------------------------------------------------------------
template <int N, int DIR>
__device__ __forceinline__ int sf_point(int L, int k) {
  if (DIR == 0) return k + N * L;                              // x-line, L = j + N k
  if (DIR == 1) return (L % N) + N * k + N * N * (L / N);      // y-line, L = i + N k
  return L + N * N * k;                                        // z-line, L = i + N j
}

__device__ __forceinline__ double sf_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float sf_fma(float a, float b, float c) { return fmaf(a, b, c); }
// Products that feed an addition are written as __dmul_rn / __fmul_rn so the
// compiler cannot contract them into an FMA with that addition: every launch
// shape of the cell kernel then rounds identically, whatever its code layout.
__device__ __forceinline__ double sf_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float sf_mul(float a, float b) { return __fmul_rn(a, b); }
template <int M> __device__ __forceinline__ TcOperand<M> sf_mul(TcOperand<M> a, TcOperand<M> b) {
  return __fmul_rn(a.v, b.v);
}
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
__device__ __forceinline__ Tf32Operand sf_fma(Tf32Operand a, Tf32Operand b, Tf32Operand c) {
  return fmaf(tf32_round(a.v), tf32_round(b.v), c.v);
}
__device__ __forceinline__ Bf16Operand sf_fma(Bf16Operand a, Bf16Operand b, Bf16Operand c) {
  return fmaf(__bfloat162float(__float2bfloat16_rn(a.v)), __bfloat162float(__float2bfloat16_rn(b.v)), c.v);
}

template <int N, int DIR, typename T>
__device__ __forceinline__ void sf_load(const T *a, int L, int p, T (&r)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) r[k] = a[sf_point<N, DIR>(L, k) * 16 + p];
}
template <int N, int DIR, typename T>
__device__ __forceinline__ void sf_store(T *a, int L, int p, const T (&r)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) a[sf_point<N, DIR>(L, k) * 16 + p] = r[k];
}
// out[q] = sum_a M[q][a] in[a]  (M row-major N x N)
template <int N, typename T>
__device__ __forceinline__ void sf_apply(const T *M, const T (&in)[N], T (&out)[N]) {
#pragma unroll
  for (int q = 0; q < N; ++q) {
    T s = T(0);
#pragma unroll
    for (int a = 0; a < N; ++a) s = sf_fma(M[q * N + a], in[a], s);
    out[q] = s;
  }
}
// out[a] += sum_q M[q][a] in[q]
template <int N, typename T>
__device__ __forceinline__ void sf_apply_t(const T *M, const T (&in)[N], T (&out)[N]) {
#pragma unroll
  for (int a = 0; a < N; ++a) {
    T s = out[a];
#pragma unroll
    for (int q = 0; q < N; ++q) s = sf_fma(M[q * N + a], in[q], s);
    out[a] = s;
  }
}

// Even-odd application of a centro-symmetric (ANTI: centro-antisymmetric) 1D
// operator from its halves: 2 (N/2)^2 FMAs instead of N^2.  ACC adds into out.
template <int N, bool ANTI, bool ACC, typename T>
__device__ __forceinline__ void sf_eo(const T *Xe, const T *Xo, const T (&in)[N], T (&out)[N]) {
  constexpr int H = N / 2;
  T e[H], o[H];
#pragma unroll
  for (int a = 0; a < H; ++a) {
    e[a] = in[a] + in[N - 1 - a];
    o[a] = in[a] - in[N - 1 - a];
  }
#pragma unroll
  for (int q = 0; q < H; ++q) {
    T E = T(0), O = T(0);
#pragma unroll
    for (int a = 0; a < H; ++a) {
      E = sf_fma(Xe[q * H + a], e[a], E);
      O = sf_fma(Xo[q * H + a], o[a], O);
    }
    const T lo = E + O, hi = ANTI ? O - E : E - O;
    out[q] = ACC ? out[q] + lo : lo;
    out[N - 1 - q] = ACC ? out[N - 1 - q] + hi : hi;
  }
}
// The four 1D operators of the cell product: even orders of N use the
// even-odd halves, odd N the full matrices.
template <int N, typename T>
__device__ __forceinline__ void sf_phi(const SfMatsT<T> &mt, const T (&in)[N], T (&out)[N]) {
  if constexpr (N % 2 == 0) sf_eo<N, false, false>(mt.phe, mt.pho, in, out);
  else sf_apply<N>(mt.phi, in, out);
}
template <int N, typename T>
__device__ __forceinline__ void sf_dq(const SfMatsT<T> &mt, const T (&in)[N], T (&out)[N]) {
  if constexpr (N % 2 == 0) sf_eo<N, true, false>(mt.dqe, mt.dqo, in, out);
  else sf_apply<N>(mt.dq, in, out);
}
template <int N, typename T>   // out += Dq^T in
__device__ __forceinline__ void sf_dqt_add(const SfMatsT<T> &mt, const T (&in)[N], T (&out)[N]) {
  if constexpr (N % 2 == 0) sf_eo<N, true, true>(mt.dte, mt.dto, in, out);
  else sf_apply_t<N>(mt.dq, in, out);
}
template <int N, typename T>   // out = Phi^T in
__device__ __forceinline__ void sf_phit(const SfMatsT<T> &mt, const T (&in)[N], T (&out)[N]) {
  if constexpr (N % 2 == 0) {
    sf_eo<N, false, false>(mt.pte, mt.pto, in, out);
  } else {
#pragma unroll
    for (int a = 0; a < N; ++a) out[a] = T(0);
    sf_apply_t<N>(mt.phi, in, out);
  }
}

// Asynchronous 8- and 4-byte global -> shared copies (cp.async, zero-filled
// when `valid` is false), completed by cp_async_wait_all in the same thread.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sa), "l"(gmem), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(sa), "l"(gmem), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int N, int MINB, bool GXS, typename T = double, bool PRE = false>
__global__ void __launch_bounds__(16 * N * N, MINB) hx_cell_sf_kernel(FeView fe, SfMatsT<T> mt, const double *__restrict__ vj,
                                                                const double *__restrict__ x,
                                                                double *__restrict__ Ycell, int B, int C, int mode) {
  // GXS: the weighted x-derivative lines wait in a fourth shared array instead
  // of registers between the forward and the backward x pass.  T is the
  // arithmetic type (double; float for the low rungs of the precision ladder):
  // the gathered values and v JxW are rounded to T, the results widened to
  // double in the cell-result slots.  PRE: the potential values and, once
  // those are used, the slot indices of the thread's z-line are copied into a
  // further shared array with cp.async at the start, so their global latency
  // hides behind the first stages instead of stalling the stages that use them.
  constexpr int N2 = N * N, N3 = N2 * N;
  extern __shared__ __align__(16) unsigned char sf_smem[];
  T *sm = reinterpret_cast<T *>(sf_smem);
  T *A = sm, *Bs = sm + N3 * 16, *Cs = sm + 2 * N3 * 16, *Gs = sm + 3 * N3 * 16;
  double *Vs = reinterpret_cast<double *>(sm + (GXS ? 4 : 3) * N3 * 16);   // PRE: [point][pair]
  const int p = threadIdx.x & 15, L = threadIdx.x >> 4;
  const int G = 16 / C;
  const int g = p / C, c = p - g * C;
  const int64_t e = (int64_t)blockIdx.x * G + g;
  const int b = blockIdx.y * C + c;
  const bool act = e < fe.nc && b < B;
  // index of (cell e, local l) in the per-cell arrays: [nd][nc] (transposed
  // copies, contiguous over the CTA's cells) when the CTA holds several cells
  const bool trn = G > 1;
  auto at = [&](int l) -> int64_t { return trn ? (int64_t)l * fe.nc + e : e * N3 + l; };
  const double *vjv = trn ? vj + fe.nc * N3 : vj;
  if (PRE) {
#pragma unroll
    for (int k = 0; k < N; ++k)
      cp_async8(&Vs[sf_point<N, 2>(L, k) * 16 + p], act ? &vjv[at(L + N2 * k)] : vj, act);
    cp_async_commit();
  }
  const T hh = act ? T(0.5 * fe.cell_h[e]) : T(0);
  T wa = T(0), wb = T(0);   // weights of the two coordinates off the line (compile-time indices)
#pragma unroll
  for (int k = 0; k < N; ++k) {
    if (L % N == k) wa = mt.w[k];
    if (L / N == k) wb = mt.w[k];
  }
  const T f = sf_mul(sf_mul(hh, wa), wb);
  T r[N], s[N], gx[N];
  // gather of the z-line L straight into registers: all N node indices, then
  // all 2N independent value loads, then the (rare) hanging rows; phi along z
  {
    int m[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const int l = L + N2 * k;
      m[k] = act ? (mode == GATHER_PLAIN ? fe.cell_nodes[e * N3 + l] : (trn ? fe.cell_map_t : fe.cell_map_sf)[at(l)]) : 0;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const bool direct = act && m[k] >= 0;
      const double xv = direct ? x[(int64_t)m[k] * B + b] : 0.0;
      const double sc = (direct && mode != GATHER_PLAIN) ? fe.inv_sqrt_mass[m[k]] : 1.0;
      r[k] = T(__dmul_rn(xv, sc));
    }
#pragma unroll
    for (int k = 0; k < N; ++k)   // constrained rows: pre-gathered by group_gather_kernel
      if (act && m[k] < 0) r[k] = T(fe.hvg[(int64_t)(-m[k] - 1) * B + b]);
  }
  sf_phi<N>(mt, r, s);
  sf_store<N, 2>(A, L, p, s);
  __syncthreads();
  sf_load<N, 1>(A, L, p, r);             // phi along y
  sf_phi<N>(mt, r, s);
  sf_store<N, 1>(Bs, L, p, s);
  __syncthreads();
  sf_load<N, 0>(Bs, L, p, r);            // phi along x: Gauss-point values, then d/dx
  sf_phi<N>(mt, r, s);
  sf_store<N, 0>(A, L, p, s);
  sf_dq<N>(mt, s, gx);
#pragma unroll
  for (int q = 0; q < N; ++q) gx[q] = sf_mul(gx[q], sf_mul(f, mt.w[q]));
  if (GXS) sf_store<N, 0>(Gs, L, p, gx);
  __syncthreads();
  sf_load<N, 1>(A, L, p, r);             // d/dy, weighted, kept for the y back pass
  sf_dq<N>(mt, r, s);
#pragma unroll
  for (int q = 0; q < N; ++q) s[q] = sf_mul(s[q], sf_mul(f, mt.w[q]));
  sf_store<N, 1>(Cs, L, p, s);
  {
    T v[N];
    if (PRE) {
      cp_async_wait_all();
#pragma unroll
      for (int k = 0; k < N; ++k) v[k] = T(Vs[sf_point<N, 2>(L, k) * 16 + p]);
      // the slot indices of the output, into the low half of each used entry
#pragma unroll
      for (int k = 0; k < N; ++k)
        cp_async4(&Vs[sf_point<N, 2>(L, k) * 16 + p], act ? &(trn ? fe.slot_of_t : fe.slot_of)[at(L + N2 * k)] : fe.slot_of,
                  act);
      cp_async_commit();
    } else {
#pragma unroll
      for (int k = 0; k < N; ++k) v[k] = act ? T(vjv[at(L + N2 * k)]) : T(0);
    }
    sf_load<N, 2>(A, L, p, r);           // d/dz, the z back pass and the potential term
    sf_dq<N>(mt, r, s);
#pragma unroll
    for (int q = 0; q < N; ++q) {
      s[q] = sf_mul(s[q], sf_mul(f, mt.w[q]));
      r[q] = sf_mul(r[q], v[q]);
    }
    sf_dqt_add<N>(mt, s, r);
    sf_store<N, 2>(Bs, L, p, r);
  }
  __syncthreads();
  sf_load<N, 1>(Bs, L, p, r);            // y back pass of the derivative term
  sf_load<N, 1>(Cs, L, p, s);
  sf_dqt_add<N>(mt, s, r);
  sf_store<N, 1>(A, L, p, r);
  __syncthreads();
  sf_load<N, 0>(A, L, p, r);             // x back pass, then phi^T along x
  if (GXS) sf_load<N, 0>(Gs, L, p, gx);
  sf_dqt_add<N>(mt, gx, r);
  sf_phit<N>(mt, r, s);
  sf_store<N, 0>(Bs, L, p, s);
  __syncthreads();
  sf_load<N, 1>(Bs, L, p, r);            // phi^T along y
  sf_phit<N>(mt, r, s);
  sf_store<N, 1>(A, L, p, s);
  __syncthreads();
  sf_load<N, 2>(A, L, p, r);             // phi^T along z, straight to the cell-result slots
  sf_phit<N>(mt, r, s);
  if (PRE) cp_async_wait_all();
  if (act) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const int sl = PRE ? *reinterpret_cast<const int *>(&Vs[sf_point<N, 2>(L, k) * 16 + p])
                         : (trn ? fe.slot_of_t : fe.slot_of)[at(L + N2 * k)];
      if (sl >= 0) Ycell[(int64_t)sl * B + b] = double(s[k]);
    }
  }
}

// Two (cell, column) pairs per thread: the same stages as hx_cell_sf_kernel
// (FP64), with thread (pair couple pp, tensor line L) carrying pairs 2pp and
// 2pp+1 through every stage.  The pairs sit next to each other in the
// [point][pair] arrays, so each shared access is one 16-byte load or store for
// both, and each 1D operator coefficient serves two FMA chains; half the
// threads, twice the independent work per thread.  When a CTA holds one cell
// per two or more columns (C >= 2) both pairs share the cell, and its gather
// indices, potential values and slots are loaded once.  Every value is
// computed by the same operations in the same order as in hx_cell_sf_kernel,
// so the results are bitwise identical.
template <int N, int DIR>
__device__ __forceinline__ void sf_load2(const double *a, int L, int pp, double (&r0)[N], double (&r1)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const double2 v = *reinterpret_cast<const double2 *>(&a[sf_point<N, DIR>(L, k) * 16 + 2 * pp]);
    r0[k] = v.x;
    r1[k] = v.y;
  }
}
template <int N, int DIR>
__device__ __forceinline__ void sf_store2(double *a, int L, int pp, const double (&r0)[N], const double (&r1)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k)
    *reinterpret_cast<double2 *>(&a[sf_point<N, DIR>(L, k) * 16 + 2 * pp]) = make_double2(r0[k], r1[k]);
}

template <int N, int MINB>
__global__ void __launch_bounds__(8 * N * N, MINB) hx_cell_sf2_kernel(FeView fe, SfMats mt, const double *__restrict__ vj,
                                                                const double *__restrict__ x,
                                                                double *__restrict__ Ycell, int B, int C, int mode) {
  constexpr int N2 = N * N, N3 = N2 * N;
  extern __shared__ __align__(16) unsigned char sf_smem[];
  double *A = reinterpret_cast<double *>(sf_smem), *Bs = A + N3 * 16, *Cs = A + 2 * N3 * 16;
  const int pp = threadIdx.x & 7, L = threadIdx.x >> 3;
  const int G = 16 / C;
  const bool trn = G > 1, same = C >= 2;
  int64_t e[2];
  int bc[2];
  bool act[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int p = 2 * pp + u, g = p / C, c = p - g * C;
    e[u] = (int64_t)blockIdx.x * G + g;
    bc[u] = blockIdx.y * C + c;
    act[u] = e[u] < fe.nc && bc[u] < B;
  }
  auto at = [&](int u, int l) -> int64_t { return trn ? (int64_t)l * fe.nc + e[u] : e[u] * N3 + l; };
  const double *vjv = trn ? vj + fe.nc * N3 : vj;
  double wa = 0.0, wb = 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    if (L % N == k) wa = mt.w[k];
    if (L / N == k) wb = mt.w[k];
  }
  double f[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) f[u] = sf_mul(sf_mul(act[u] ? 0.5 * fe.cell_h[e[u]] : 0.0, wa), wb);
  double r[2][N], s[2][N], gx[2][N];
  {
    int m[2][N];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const int l = L + N2 * k;
        if (u == 1 && same) {
          m[1][k] = act[1] ? m[0][k] : 0;
        } else {
          m[u][k] = act[u] ? (mode == GATHER_PLAIN ? fe.cell_nodes[e[u] * N3 + l]
                                                   : (trn ? fe.cell_map_t : fe.cell_map_sf)[at(u, l)])
                           : 0;
        }
      }
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const bool direct = act[u] && m[u][k] >= 0;
        const double xv = direct ? x[(int64_t)m[u][k] * B + bc[u]] : 0.0;
        const double sc = (direct && mode != GATHER_PLAIN) ? fe.inv_sqrt_mass[m[u][k]] : 1.0;
        r[u][k] = __dmul_rn(xv, sc);
      }
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (act[u] && m[u][k] < 0) r[u][k] = fe.hvg[(int64_t)(-m[u][k] - 1) * B + bc[u]];
  }
#pragma unroll
  for (int u = 0; u < 2; ++u) sf_phi<N>(mt, r[u], s[u]);
  sf_store2<N, 2>(A, L, pp, s[0], s[1]);
  __syncthreads();
  sf_load2<N, 1>(A, L, pp, r[0], r[1]);   // phi along y
#pragma unroll
  for (int u = 0; u < 2; ++u) sf_phi<N>(mt, r[u], s[u]);
  sf_store2<N, 1>(Bs, L, pp, s[0], s[1]);
  __syncthreads();
  sf_load2<N, 0>(Bs, L, pp, r[0], r[1]);  // phi along x: Gauss-point values, then d/dx
#pragma unroll
  for (int u = 0; u < 2; ++u) sf_phi<N>(mt, r[u], s[u]);
  sf_store2<N, 0>(A, L, pp, s[0], s[1]);
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    sf_dq<N>(mt, s[u], gx[u]);
#pragma unroll
    for (int q = 0; q < N; ++q) gx[u][q] = sf_mul(gx[u][q], sf_mul(f[u], mt.w[q]));
  }
  __syncthreads();
  sf_load2<N, 1>(A, L, pp, r[0], r[1]);   // d/dy, weighted, kept for the y back pass
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    sf_dq<N>(mt, r[u], s[u]);
#pragma unroll
    for (int q = 0; q < N; ++q) s[u][q] = sf_mul(s[u][q], sf_mul(f[u], mt.w[q]));
  }
  sf_store2<N, 1>(Cs, L, pp, s[0], s[1]);
  {
    double v[2][N];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int k = 0; k < N; ++k)
        v[u][k] = (u == 1 && same) ? (act[1] ? v[0][k] : 0.0) : (act[u] ? vjv[at(u, L + N2 * k)] : 0.0);
    sf_load2<N, 2>(A, L, pp, r[0], r[1]); // d/dz, the z back pass and the potential term
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      sf_dq<N>(mt, r[u], s[u]);
#pragma unroll
      for (int q = 0; q < N; ++q) {
        s[u][q] = sf_mul(s[u][q], sf_mul(f[u], mt.w[q]));
        r[u][q] = sf_mul(r[u][q], v[u][q]);
      }
      sf_dqt_add<N>(mt, s[u], r[u]);
    }
    sf_store2<N, 2>(Bs, L, pp, r[0], r[1]);
  }
  __syncthreads();
  sf_load2<N, 1>(Bs, L, pp, r[0], r[1]);  // y back pass of the derivative term
  sf_load2<N, 1>(Cs, L, pp, s[0], s[1]);
#pragma unroll
  for (int u = 0; u < 2; ++u) sf_dqt_add<N>(mt, s[u], r[u]);
  sf_store2<N, 1>(A, L, pp, r[0], r[1]);
  __syncthreads();
  sf_load2<N, 0>(A, L, pp, r[0], r[1]);   // x back pass, then phi^T along x
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    sf_dqt_add<N>(mt, gx[u], r[u]);
    sf_phit<N>(mt, r[u], s[u]);
  }
  sf_store2<N, 0>(Bs, L, pp, s[0], s[1]);
  __syncthreads();
  sf_load2<N, 1>(Bs, L, pp, r[0], r[1]);  // phi^T along y
#pragma unroll
  for (int u = 0; u < 2; ++u) sf_phit<N>(mt, r[u], s[u]);
  sf_store2<N, 1>(A, L, pp, s[0], s[1]);
  __syncthreads();
  sf_load2<N, 2>(A, L, pp, r[0], r[1]);   // phi^T along z, straight to the cell-result slots
#pragma unroll
  for (int u = 0; u < 2; ++u) sf_phit<N>(mt, r[u], s[u]);
  int sl[2][N];
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int k = 0; k < N; ++k)
      sl[u][k] = (u == 1 && same) ? sl[0][k]
                                  : (act[u] ? (trn ? fe.slot_of_t : fe.slot_of)[at(u, L + N2 * k)] : -1);
#pragma unroll
  for (int u = 0; u < 2; ++u)
    if (act[u]) {
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (sl[u][k] >= 0) Ycell[(int64_t)sl[u][k] * B + bc[u]] = s[u][k];
    }
}

// ---------------------------------------------------------------------------
// HX, part 1, bulk-asynchronous variant.  Persistent CTAs walk their cells;
// thread 0 streams contiguous column panels of H_e (PW columns x ldh doubles)
// with cp.async.bulk into an S-stage shared-memory ring completed through
// mbarriers, S-1 panels ahead of the consumers.  Every wait is bounded: a wait
// that gives up sets fe.err and the CTA stops computing (it never hangs).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
constexpr long long kWaitLimit = 1ll << 22;

template <int BC>
__global__ void __launch_bounds__(NT, 1) hx_gemm_bulk_kernel(FeView fe, const double *__restrict__ H,
                                                             const double *__restrict__ x,
                                                             double *__restrict__ Yslot, int B, int mode,
                                                             int S, int PW) {
  extern __shared__ __align__(128) unsigned char smraw[];
  const int nd = fe.nd, ldh = fe.ldh;
  const int np = (nd + PW - 1) / PW;
  double *stages = reinterpret_cast<double *>(smraw);
  double *xs = stages + (size_t)S * PW * ldh;
  uint64_t *bars = reinterpret_cast<uint64_t *>(xs + (size_t)(nd + 1) * BC);
  const int tid = threadIdx.x;
  if (blockIdx.x >= fe.nc) return;
  const int64_t ncell = (fe.nc - 1 - blockIdx.x) / gridDim.x + 1;
  const int64_t total = ncell * np;
  if (tid == 0) {
    for (int st = 0; st < S; ++st) mbar_init(&bars[st], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int64_t sq) {
    const int64_t t = sq / np;
    const int k = (int)(sq - t * np);
    const int64_t e = blockIdx.x + t * gridDim.x;
    const int c0 = k * PW;
    const int ncol = min(PW, 2 * ((nd + 1) >> 1) - c0);   // even: whole column pairs
    const uint32_t bytes = (uint32_t)ncol * ldh * 8u;
    uint64_t *bar = &bars[sq % S];
    mbar_expect_tx(bar, bytes);
    bulk_g2s(stages + (sq % S) * (int64_t)PW * ldh,
             H + e * (int64_t)((nd + 1) >> 1) * 2 * ldh + (int64_t)c0 * ldh, bytes, bar);
  };
  int64_t n_issued = 0;     // thread 0: panels issued so far
  int64_t first_open = -1;  // thread 0: first panel its own wait gave up on
  if (tid == 0)
    for (int64_t sq = 0; sq < min((int64_t)S, total); ++sq) issue(sq), n_issued = sq + 1;
  bool ok = true;
  const int i = tid;
  for (int64_t t = 0; t < ncell; ++t) {
    const int64_t e = blockIdx.x + t * gridDim.x;
    for (int idx = tid; idx < (nd + 1) * BC; idx += blockDim.x) {
      const int l = idx / BC, b = idx - l * BC;
      double v = 0.0;
      if (b < B && l < nd) {
        if (mode == GATHER_PLAIN) {
          v = x[(int64_t)fe.cell_nodes[e * nd + l] * B + b];
        } else {
          const int m = fe.cell_map[e * nd + l];
          if (m >= 0) {
            v = x[(int64_t)m * B + b] * fe.inv_sqrt_mass[m];
          } else {
            const int r = -m - 1;
            for (int k = fe.cons_ptr[r]; k < fe.cons_ptr[r + 1]; ++k)
              v = fma(fe.cons_gw[k], x[(int64_t)fe.cons_masters[k] * B + b], v);
          }
        }
      }
      xs[idx] = v;
    }
    __syncthreads();
    double acc[BC];
#pragma unroll
    for (int b = 0; b < BC; ++b) acc[b] = 0.0;
    for (int k = 0; k < np; ++k) {
      const int64_t sq = t * np + k;
      const int st = (int)(sq % S);
      const uint32_t par = (uint32_t)((sq / S) & 1);
      if (ok) {
        long long it = 0;
        while (!mbar_try_wait(&bars[st], par)) {
          if (++it > kWaitLimit) {
            ok = false;
            atomicExch(fe.err, 1);
            if (tid == 0) first_open = sq;
            break;
          }
        }
      }
      const int c0 = k * PW;
      const int ncol = min(PW, 2 * ((nd + 1) >> 1) - c0);
      if (ok && i < nd) {
        const double2 *Hs = reinterpret_cast<const double2 *>(stages + (int64_t)st * PW * ldh) + i;
        const double *xr = xs + (int64_t)c0 * BC;
        for (int cp = 0; cp < (ncol + 1) / 2; ++cp) {
          const double2 h = Hs[cp * ldh];
#pragma unroll
          for (int b = 0; b < BC; b += 2) {
            const double2 x0 = *reinterpret_cast<const double2 *>(xr + 2 * cp * BC + b);
            const double2 x1 = *reinterpret_cast<const double2 *>(xr + (2 * cp + 1) * BC + b);
            acc[b] = fma(h.x, x0.x, acc[b]);
            acc[b + 1] = fma(h.x, x0.y, acc[b + 1]);
            acc[b] = fma(h.y, x1.x, acc[b]);
            acc[b + 1] = fma(h.y, x1.y, acc[b + 1]);
          }
        }
      }
      __syncthreads();
      if (tid == 0 && ok && sq + S < total) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(sq + S);
        n_issued = sq + S + 1;
      }
    }
    if (ok && i < nd) {
      const int sl = fe.slot_of[e * nd + i];
      if (sl >= 0) {
        double *yo = Yslot + (int64_t)sl * B;
#pragma unroll
        for (int b = 0; b < BC; ++b)
          if (b < B) yo[b] = acc[b];
      }
    }
  }
  // after a wait gave up, copies issued from there on may still be writing
  // this CTA's shared memory: thread 0 waits for them (bounded again) before
  // the CTA retires and its shared memory can be handed to another CTA.  Thread
  // 0 stops issuing once its own wait fails, so each stage holds at most one
  // such copy, with the parity of its panel.
  if (tid == 0 && first_open >= 0) {
    for (int64_t sq = first_open; sq < n_issued; ++sq) {
      long long it = 0;
      while (!mbar_try_wait(&bars[sq % S], (uint32_t)((sq / S) & 1)) && ++it <= kWaitLimit) {
      }
    }
  }
}

// The last CTA of a grid-wide reduction: out[c] = sum over g < nparts of
// partial[g*B + c] for c < B (B <= NT).  Every thread of the CTA takes part:
// thread (group k, column c) sums the partials k, k + R, ... (R = NT / B), then
// the R group sums of each column are added by a halving tree.  The order is
// fixed by B and nparts alone, so the result is deterministic.
__device__ void cta_column_sums(const double *partial, int nparts, int B, double *out, double *red) {
  const int R = NT / B;
  const int c = threadIdx.x % B, k = threadIdx.x / B;
  double v = 0.0;
  if (k < R)
    for (int g = k; g < nparts; g += R) v += __ldcg(&partial[(int64_t)g * B + c]);
  red[threadIdx.x] = v;
  __syncthreads();
  int span = 1;
  while (span < R) span <<= 1;
  for (int h = span >> 1; h > 0; h >>= 1) {
    if (k < h && k + h < R) red[k * B + c] += red[(k + h) * B + c];
    __syncthreads();
  }
  if (threadIdx.x < B) out[threadIdx.x] = red[threadIdx.x];
  __syncthreads();
}

// One tile of the assembly: node rows r0 .. r0+rows-1 with their slots read
// from segp[sl*B + j - a0] (a shared-memory copy of the tile's slot segment, or
// the cell results themselves with a0 = 0) -- a master of hanging nodes has its
// summed hanging contributions in its last slot -- their slot ranges from dp,
// M^-1/2 from ism and the epilogue inputs from t_in/t_prev (all tile-local, row
// stride B for blocks).  Thread (rr, j) handles column j of rows rr, rr+RR, ...
// in a fixed order.
template <int KIND>
__device__ __forceinline__ void assemble_tile_rows_k(const FeView &fe, const double *segp, int64_t a0,
                                                     const int *dp, const double *ism,
                                                     const double *t_in, const double *t_prev, int64_t r0, int rows,
                                                     double *__restrict__ out, int B, const AsmEpilogue &epi,
                                                     double &dot) {
  const int RR = NT / B;
  const int j = threadIdx.x % B, rr = threadIdx.x / B;
  if (rr >= RR) return;
  const double *sj = segp + j;
  for (int lr = rr; lr < rows; lr += RR) {
    const int64_t n = r0 + lr;
    const int d0 = dp[lr], d1 = dp[lr + 1];
    double acc = 0.0;   // a master's hanging contributions are its last slot
    for (int sl = d0; sl < d1; ++sl) acc += sj[(int64_t)sl * B - a0];
    acc *= ism[lr];
    const int64_t idx = n * B + j;
    const int li = lr * B + j;
    if constexpr (KIND == AsmEpilogue::STORE) {
      out[idx] = acc;
    } else if constexpr (KIND == AsmEpilogue::CHEB) {
      double v = epi.alpha * (acc - epi.c * t_in[li]);
      if (epi.prev) v -= epi.beta * t_prev[li];
      out[idx] = v;
    } else if constexpr (KIND == AsmEpilogue::VMULT) {
      out[idx] = acc - epi.eps[j] * t_in[li];
    } else if constexpr (KIND == AsmEpilogue::RHS) {
      double v = 0.0;
      if (d1 > d0 && ism[lr] != 0.0) {
        double mu = 0.0;
        for (int k = 0; k < B; ++k) mu = fma(epi.Mu[k * B + j], epi.psi[n * B + k], mu);
        v = epi.occ4[j] * acc - 2.0 * fe.sqrt_mass[n] * mu;
      }
      out[idx] = v;
    } else {
      const double vv = t_in[li];
      const double yn = acc - epi.eps[j] * vv - epi.minres_coef[j] * t_prev[li];
      out[idx] = yn;
      dot = fma(vv, yn, dot);
    }
  }
}
// the same with the epilogue chosen at run time (the bulk-pipelined variant)
__device__ __forceinline__ void assemble_tile_rows(const FeView &fe, const double *segp, int64_t a0,
                                                   const int *dp, const double *ism,
                                                   const double *t_in, const double *t_prev, int64_t r0, int rows,
                                                   double *__restrict__ out, int B, const AsmEpilogue &epi,
                                                   double &dot) {
  switch (epi.kind) {
    case AsmEpilogue::STORE:
      assemble_tile_rows_k<AsmEpilogue::STORE>(fe, segp, a0, dp, ism, t_in, t_prev, r0, rows, out, B, epi, dot);
      break;
    case AsmEpilogue::CHEB:
      assemble_tile_rows_k<AsmEpilogue::CHEB>(fe, segp, a0, dp, ism, t_in, t_prev, r0, rows, out, B, epi, dot);
      break;
    case AsmEpilogue::VMULT:
      assemble_tile_rows_k<AsmEpilogue::VMULT>(fe, segp, a0, dp, ism, t_in, t_prev, r0, rows, out, B, epi, dot);
      break;
    case AsmEpilogue::RHS:
      assemble_tile_rows_k<AsmEpilogue::RHS>(fe, segp, a0, dp, ism, t_in, t_prev, r0, rows, out, B, epi, dot);
      break;
    default:
      assemble_tile_rows_k<AsmEpilogue::MINRES>(fe, segp, a0, dp, ism, t_in, t_prev, r0, rows, out, B, epi, dot);
  }
}

constexpr int kAsmRow = 3;   // per-thread shares of the staged node rows (TR + 1 <= 3 NT)
constexpr int kAsmBlk = 4;   // ... of an epilogue block (TR B <= 4 NT)
constexpr int kAsmSeg = 8;   // ... of a staged slot segment (cap B = 2 TR B <= 8 NT)

// ---------------------------------------------------------------------------
// HX, part 2 (tiled): a CTA owns TR consecutive nodes, whose slots form one
// contiguous segment [dptr[r0], dptr[r0+TR]).  The segment is streamed into
// shared memory with coalesced loads and the per-node sums are taken from
// there; a master of hanging nodes finds its pre-summed contribution in its
// last slot, written by the master-sum pass.  Thread (rr, j) handles column j of nodes r0+rr,
// r0+rr+RR, ... (fixed order), so the MINRES dot partials are deterministic.
// ---------------------------------------------------------------------------
template <int KIND>
__global__ void __launch_bounds__(NT, 4) hx_assemble_tile_kernel(FeView fe, const double *__restrict__ Ycell,
                                                              double *__restrict__ out, int B, AsmEpilogue epi,
                                                              int TR, int cap_slots) {
  // shared layout: seg [cap][B] | s_in [TR][B] | s_prev [TR][B] | ism [TR] | dp [TR+1]
  extern __shared__ double sm_asm[];
  double *seg = sm_asm;
  double *s_in = seg + (size_t)cap_slots * B;
  double *s_prev = s_in + (size_t)TR * B;
  double *ism = s_prev + (size_t)TR * B;
  int *dp = reinterpret_cast<int *>(ism + TR);
  __shared__ double red[NT];
  __shared__ bool last;
  const int64_t r0 = (int64_t)blockIdx.x * TR;
  // the grid is sized by the caller (ceil(nnodes / TR)), so rows >= 1
  const int rows = (int)max((int64_t)0, min((int64_t)TR, fe.nnodes - r0));
  constexpr bool need_in = KIND == AsmEpilogue::CHEB || KIND == AsmEpilogue::VMULT || KIND == AsmEpilogue::MINRES;
  const bool need_prev = (KIND == AsmEpilogue::CHEB && epi.prev) || KIND == AsmEpilogue::MINRES;
  // one round of loads: the slot bounds of the tile first, then every staged
  // array into fixed per-thread register shares (the launcher keeps
  // TR*B <= kAsmBlk*NT and 2*TR*B <= kAsmSeg*NT), then all stores
  const int s0 = fe.dptr[r0], s1 = fe.dptr[r0 + rows];
  const bool staged = (s1 - s0) <= cap_slots;
  const int tid = threadIdx.x, nb = rows * B, ns = (s1 - s0) * B;
  int v_dp[kAsmRow];
  double v_ism[kAsmRow], v_in[kAsmBlk], v_pr[kAsmBlk], v_sg[kAsmSeg];
#pragma unroll
  for (int u = 0; u < kAsmRow; ++u) {
    const int i = tid + u * NT;
    v_dp[u] = i <= rows ? fe.dptr[r0 + i] : 0;
    v_ism[u] = i < rows ? fe.inv_sqrt_mass[r0 + i] : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kAsmBlk; ++u) {
    const int i = tid + u * NT;
    v_in[u] = (need_in && i < nb) ? epi.in[r0 * B + i] : 0.0;
    v_pr[u] = (need_prev && i < nb) ? epi.prev[r0 * B + i] : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kAsmSeg; ++u) {
    const int i = tid + u * NT;
    v_sg[u] = (staged && i < ns) ? Ycell[(int64_t)s0 * B + i] : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kAsmRow; ++u) {
    const int i = tid + u * NT;
    if (i <= rows) dp[i] = v_dp[u];
    if (i < rows) ism[i] = v_ism[u];
  }
#pragma unroll
  for (int u = 0; u < kAsmBlk; ++u) {
    const int i = tid + u * NT;
    if (i < nb) {
      if (need_in) s_in[i] = v_in[u];
      if (need_prev) s_prev[i] = v_pr[u];
    }
  }
#pragma unroll
  for (int u = 0; u < kAsmSeg; ++u) {
    const int i = tid + u * NT;
    if (staged && i < ns) seg[i] = v_sg[u];
  }
  __syncthreads();
  double dot = 0.0;
  assemble_tile_rows_k<KIND>(fe, staged ? seg : Ycell, staged ? (int64_t)s0 * B : 0, dp, ism, s_in, s_prev, r0,
                             rows, out, B, epi, dot);
  if constexpr (KIND == AsmEpilogue::MINRES) {
    const int RR = NT / B;
    red[threadIdx.x] = dot;
    __syncthreads();
    if (threadIdx.x < B) {
      double sum = 0.0;
      for (int q = 0; q < RR; ++q) sum += red[q * B + threadIdx.x];
      epi.dot_partial[(int64_t)blockIdx.x * B + threadIdx.x] = sum;
    }
    if (epi.dot_ticket) {
      // the last CTA to finish (ticket taken after a fence) reduces the
      // partials, each column by one warp in a fixed order
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) last = atomicAdd(epi.dot_ticket, 1u) == gridDim.x - 1;
      __syncthreads();
      if (!last) return;
      __threadfence();
      cta_column_sums(epi.dot_partial, (int)gridDim.x, B, epi.dot_out, red);
      if (threadIdx.x == 0) *epi.dot_ticket = 0u;
    }
  }
}

// ---------------------------------------------------------------------------
// HX, part 2, bulk-pipelined: persistent CTAs walk the full tiles of TR nodes
// (tile blockIdx.x + i*gridDim.x).  Everything a tile reads is contiguous in
// HBM -- its slot ranges, master indices, M^-1/2, the epilogue inputs and its
// slot segment of the cell results -- so thread 0 streams tile i+1 into the
// other of two shared-memory stages with cp.async.bulk (one mbarrier per
// stage) while the CTA reduces tile i.  The slot segment is copied from its
// 16-byte-aligned start (offset a0 kept in shared memory); a segment longer
// than the stage holds is read from HBM directly.  Waits are bounded and
// voted across the CTA: a wait that gives up sets fe.err, thread 0 drains
// the other stage (bounded again) and the CTA returns.  The last, partial
// tile is reduced with direct loads by one CTA after the loop.
// ---------------------------------------------------------------------------
struct AsmStage {
  double *seg, *in, *prev, *ism;
  int *dp;
};

__device__ __forceinline__ AsmStage asm_stage(unsigned char *base, int st, int TR, int cap, int B) {
  const size_t seg_n = (size_t)cap * B + 2, blk = (size_t)TR * B;
  const size_t stage_bytes = 8 * (seg_n + 2 * blk + TR) + 4 * ((size_t)TR + 4);
  double *p = reinterpret_cast<double *>(base + (size_t)st * ((stage_bytes + 127) & ~(size_t)127));
  AsmStage s;
  s.seg = p;
  s.in = p + seg_n;
  s.prev = s.in + blk;
  s.ism = s.prev + blk;
  s.dp = reinterpret_cast<int *>(s.ism + TR);
  return s;
}

__global__ void __launch_bounds__(NT) hx_assemble_bulk_kernel(FeView fe, const double *__restrict__ Ycell,
                                                              double *__restrict__ out, int B, AsmEpilogue epi,
                                                              int TR, int cap) {
  extern __shared__ __align__(128) unsigned char sm_ab[];
  __shared__ uint64_t bars[2];
  __shared__ double red[NT];
  const int64_t nfull = fe.nnodes / TR;
  const int64_t G = gridDim.x;
  const int64_t cnt = blockIdx.x < nfull ? (nfull - 1 - blockIdx.x) / G + 1 : 0;
  const bool need_in = epi.kind == AsmEpilogue::CHEB || epi.kind == AsmEpilogue::VMULT ||
                       epi.kind == AsmEpilogue::MINRES;
  const bool need_prev = (epi.kind == AsmEpilogue::CHEB && epi.prev) || epi.kind == AsmEpilogue::MINRES;
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // thread 0: stream tile i (slot bounds s0, s1 already loaded) into stage i & 1
  auto issue = [&](int64_t i, int s0, int s1) {
    const int64_t r0 = (blockIdx.x + i * G) * TR;
    AsmStage S = asm_stage(sm_ab, (int)(i & 1), TR, cap, B);
    uint64_t *bar = &bars[i & 1];
    uint32_t bytes = 4u * (uint32_t)(TR + 4) + 8u * (uint32_t)TR;
    if (need_in) bytes += 8u * (uint32_t)TR * B;
    if (need_prev) bytes += 8u * (uint32_t)TR * B;
    const bool staged = s1 - s0 <= cap;
    const int64_t a0 = ((int64_t)s0 * B) & ~(int64_t)1, a1 = ((int64_t)s1 * B + 1) & ~(int64_t)1;
    if (staged) bytes += 8u * (uint32_t)(a1 - a0);
    mbar_expect_tx(bar, bytes);
    bulk_g2s(S.dp, fe.dptr + r0, 4u * (TR + 4), bar);
    bulk_g2s(S.ism, fe.inv_sqrt_mass + r0, 8u * TR, bar);
    if (need_in) bulk_g2s(S.in, epi.in + r0 * B, 8u * TR * B, bar);
    if (need_prev) bulk_g2s(S.prev, epi.prev + r0 * B, 8u * TR * B, bar);
    if (staged && a1 > a0) bulk_g2s(S.seg, Ycell + a0, 8u * (uint32_t)(a1 - a0), bar);
  };
  auto bounds = [&](int64_t i, int &s0, int &s1) {
    const int64_t r0 = (blockIdx.x + i * G) * TR;
    s0 = fe.dptr[r0];
    s1 = fe.dptr[r0 + TR];
  };
  int pre0 = 0, pre1 = 0;   // thread 0: slot bounds of tile i+2
  if (threadIdx.x == 0) {
    int s0, s1;
    if (cnt > 0) { bounds(0, s0, s1); issue(0, s0, s1); }
    if (cnt > 1) { bounds(1, s0, s1); issue(1, s0, s1); }
  }
  double dot = 0.0;
  for (int64_t i = 0; i < cnt; ++i) {
    if (threadIdx.x == 0 && i + 2 < cnt) bounds(i + 2, pre0, pre1);   // in flight during this tile
    bool ok = true;
    {
      long long it = 0;
      while (!mbar_try_wait(&bars[i & 1], (uint32_t)((i >> 1) & 1))) {
        if (++it > kWaitLimit) { ok = false; break; }
      }
    }
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) {
        atomicExch(fe.err, 1);
        if (i + 1 < cnt) {   // drain the other stage's copies before the CTA leaves
          long long it = 0;
          while (!mbar_try_wait(&bars[(i + 1) & 1], (uint32_t)(((i + 1) >> 1) & 1)) && ++it <= kWaitLimit) {
          }
        }
      }
      return;
    }
    const int64_t r0 = (blockIdx.x + i * G) * TR;
    AsmStage S = asm_stage(sm_ab, (int)(i & 1), TR, cap, B);
    const int s0 = S.dp[0], s1 = S.dp[TR];
    const bool staged = s1 - s0 <= cap;
    const int64_t a0 = staged ? (((int64_t)s0 * B) & ~(int64_t)1) : 0;
    assemble_tile_rows(fe, staged ? S.seg : Ycell, a0, S.dp, S.ism, S.in, S.prev, r0, TR, out, B, epi, dot);
    __syncthreads();
    if (threadIdx.x == 0 && i + 2 < cnt) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(i + 2, pre0, pre1);
    }
  }
  // the partial last tile, direct loads, on the CTA next in the round robin
  const int64_t rt = nfull * TR;
  if (rt < fe.nnodes && blockIdx.x == nfull % G) {
    const int rows = (int)(fe.nnodes - rt);
    assemble_tile_rows(fe, Ycell, 0, fe.dptr + rt, fe.inv_sqrt_mass + rt,
                       need_in ? epi.in + rt * B : nullptr, need_prev ? epi.prev + rt * B : nullptr, rt, rows,
                       out, B, epi, dot);
  }
  if (epi.kind == AsmEpilogue::MINRES) {
    const int RR = NT / B;
    red[threadIdx.x] = dot;
    __syncthreads();
    if (threadIdx.x < B) {
      double sum = 0.0;
      for (int q = 0; q < RR; ++q) sum += red[q * B + threadIdx.x];
      epi.dot_partial[(int64_t)blockIdx.x * B + threadIdx.x] = sum;
    }
  }
}

// z[h][j] = sum of the cell rows of hanging node h (its contiguous slots), in slot order
__device__ __forceinline__ double hanging_row_sum(const FeView &fe, const double *__restrict__ Ycell, int h, int j,
                                                  int B) {
  double acc = 0.0;
  for (int sl = fe.zptr[h]; sl < fe.zptr[h + 1]; ++sl) acc += Ycell[(int64_t)sl * B + j];
  return acc;
}

// What C^T adds to the masters of hanging nodes, in two passes.  One CTA per
// hanging constraint group sums the cell rows of the group's hanging nodes (z,
// each hanging node belongs to one group) into shared memory, stages the
// group's weights, and writes gpart[g_poff[g] + t][j] = sum_q w[row q, t] z[row q][j]
// for each of its masters t; then master_sum_kernel sums master i's (group,
// master) partials into the master's last slot.  Both in a fixed order.
__global__ void __launch_bounds__(NT) group_partial_kernel(FeView fe, const double *__restrict__ Ycell, int B,
                                                           int cap) {
  extern __shared__ double sp[];   // zr [nr][B] | wm [nr][nmp] (rows padded to 4 with zeros)
  const int g = blockIdx.x;
  const int nm = fe.g_nm[g], rp0 = fe.g_rptr[g], nr = fe.g_rptr[g + 1] - rp0;
  const int nmp = (nm + 3) & ~3;
  const int h0 = fe.g_hrow[rp0];   // the group's rows have consecutive hanging indices
  const int64_t po = fe.g_poff[g];
  const double *w = fe.g_w + fe.g_woff[g];
  if ((int64_t)nr * (B + nmp) > cap) {   // too large to stage: z summed per use from the cell results
    for (int i = threadIdx.x; i < nm * B; i += blockDim.x) {
      const int t = i / B, j = i - t * B;
      double acc = 0.0;
      for (int q = 0; q < nr; ++q) acc = fma(w[q * nm + t], hanging_row_sum(fe, Ycell, (h0 + q), j, B), acc);
      fe.gpart[(po + t) * B + j] = acc;
    }
    return;
  }
  double *zr = sp, *wm = sp + (size_t)nr * B;
  for (int i = threadIdx.x; i < nr * B; i += blockDim.x) {
    const int q = i / B, j = i - q * B;
    zr[i] = hanging_row_sum(fe, Ycell, (h0 + q), j, B);
  }
  for (int i = threadIdx.x; i < nr * nmp; i += blockDim.x) {
    const int q = i / nmp, t = i - q * nmp;
    wm[i] = t < nm ? w[q * nm + t] : 0.0;
  }
  __syncthreads();
  if (B >= 8) {
    // four masters per thread: each staged z value serves four FMA chains
    for (int i = threadIdx.x; i < (nmp >> 2) * B; i += blockDim.x) {
      const int t0 = (i / B) << 2, j = i % B;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      for (int q = 0; q < nr; ++q) {
        const double z = zr[q * B + j];
        const double *wr = wm + q * nmp + t0;
        a0 = fma(wr[0], z, a0);
        a1 = fma(wr[1], z, a1);
        a2 = fma(wr[2], z, a2);
        a3 = fma(wr[3], z, a3);
      }
      const double aa[4] = {a0, a1, a2, a3};
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (t0 + u < nm) fe.gpart[(po + t0 + u) * B + j] = aa[u];
    }
  } else {
    for (int i = threadIdx.x; i < nm * B; i += blockDim.x) {
      const int t = i / B, j = i - t * B;
      double acc = 0.0;
      for (int q = 0; q < nr; ++q) acc = fma(wm[q * nmp + t], zr[q * B + j], acc);
      fe.gpart[(po + t) * B + j] = acc;
    }
  }
}

__global__ void master_sum_kernel(FeView fe, int B, double *__restrict__ Ycell) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)fe.nmast * B) return;
  const int i = (int)(idx / B), j = (int)(idx - (int64_t)i * B);
  double acc = 0.0;
  for (int q = fe.mp_ptr[i]; q < fe.mp_ptr[i + 1]; ++q) acc += fe.gpart[(int64_t)fe.mp_idx[q] * B + j];
  Ycell[(int64_t)fe.mslot[i] * B + j] = acc;
}

__global__ void scale_rows_kernel(const double *d, const double *x, double *y, int64_t n, int B) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx < n * B) y[idx] = d[idx / B] * x[idx];
}

__global__ void distribute_kernel(const int *rows, const int *ptr, const int *masters, const double *w,
                                  int nrows, double *x, int B) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nrows * B) return;
  const int r = (int)(idx / B), b = (int)(idx % B);
  double v = 0.0;
  for (int k = ptr[r]; k < ptr[r + 1]; ++k) v = fma(w[k], x[(int64_t)masters[k] * B + b], v);
  x[(int64_t)rows[r] * B + b] = v;
}

__global__ void set_zero_kernel(const int *rows, int nrows, double *x, int B) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nrows * B) return;
  x[(int64_t)rows[idx / B] * B + idx % B] = 0.0;
}

// ---------------------------------------------------------------------------
// Tall-skinny products
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(NT) gram_kernel(const double *__restrict__ A, const double *__restrict__ Bm,
                                                  int64_t n, int N, int64_t rows_per_block,
                                                  double *__restrict__ partial) {
  __shared__ double As[32 * 64], Bs[32 * 64];
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1 = min(n, r0 + rows_per_block);
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (int64_t rb = r0; rb < r1; rb += 32) {
    const int nr = (int)min((int64_t)32, r1 - rb);
    for (int idx = threadIdx.x; idx < nr * N; idx += blockDim.x) {
      As[idx] = A[rb * N + idx];
      Bs[idx] = Bm[rb * N + idx];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int o = threadIdx.x + k * NT;
      if (o < N * N) {
        const int i = o / N, jj = o % N;
        double s = 0.0;
        for (int r = 0; r < nr; ++r) s = fma(As[r * N + i], Bs[r * N + jj], s);
        acc[k] += s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int o = threadIdx.x + k * NT;
    if (o < N * N) partial[(int64_t)blockIdx.x * N * N + o] = acc[k];
  }
}

// out[o] = sum_g partial[g*width + o]; one CTA per output, fixed summation
// order (strided thread sums, then a fixed tree), so results are reproducible.
__global__ void __launch_bounds__(NT) reduce_partials_kernel(const double *partial, int nparts, int width,
                                                             double *out) {
  __shared__ double red[32];
  const int o = blockIdx.x;
  double s = 0.0;
  for (int g = threadIdx.x; g < nparts; g += blockDim.x) s += partial[(int64_t)g * width + o];
  s = block_sum<NT>(s, red);
  if (threadIdx.x == 0) out[o] = s;
}

__global__ void __launch_bounds__(NT) rotate_kernel(const double *__restrict__ Y, const double *__restrict__ T,
                                                    double *__restrict__ Z, int64_t n, int N) {
  __shared__ double Ts[64 * 64];
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) Ts[i] = T[i];
  __syncthreads();
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= n * N) return;
  const int64_t r = idx / N;
  const int j = (int)(idx % N);
  const double *yr = Y + r * N;
  double s = 0.0;
  for (int k = 0; k < N; ++k) s = fma(yr[k], Ts[k * N + j], s);
  Z[idx] = s;
}

__global__ void __launch_bounds__(NT) rotate_residual_kernel(const double *__restrict__ Y,
                                                             const double *__restrict__ HY,
                                                             const double *__restrict__ Q,
                                                             const double *__restrict__ eps,
                                                             double *__restrict__ X, int64_t n, int N,
                                                             int64_t rows_per_block,
                                                             double *__restrict__ partial) {
  __shared__ double Qs[64 * 64];
  __shared__ double red[NT];
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) Qs[i] = Q[i];
  __syncthreads();
  const int RR = NT / N;
  const int j = threadIdx.x % N, rr = threadIdx.x / N;
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1 = min(n, r0 + rows_per_block);
  double acc = 0.0;
  if (rr < RR) {
    for (int64_t r = r0 + rr; r < r1; r += RR) {
      double xs = 0.0, hs = 0.0;
      for (int k = 0; k < N; ++k) {
        xs = fma(Y[r * N + k], Qs[k * N + j], xs);
        hs = fma(HY[r * N + k], Qs[k * N + j], hs);
      }
      X[r * N + j] = xs;
      const double res = hs - eps[j] * xs;
      acc = fma(res, res, acc);
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < N) {
    double s = 0.0;
    for (int q = 0; q < RR; ++q) s += red[q * N + threadIdx.x];
    partial[(int64_t)blockIdx.x * N + threadIdx.x] = s;
  }
}

__global__ void __launch_bounds__(NT) coldot_kernel(const double *__restrict__ a, const double *__restrict__ b,
                                                    int64_t n, int B, int64_t rows_per_block,
                                                    double *__restrict__ partial) {
  __shared__ double red[NT];
  const int RR = NT / B;
  const int j = threadIdx.x % B, rr = threadIdx.x / B;
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1 = min(n, r0 + rows_per_block);
  double acc = 0.0;
  if (rr < RR)
    for (int64_t r = r0 + rr; r < r1; r += RR) acc = fma(a[r * B + j], b[r * B + j], acc);
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < B) {
    double s = 0.0;
    for (int q = 0; q < RR; ++q) s += red[q * B + threadIdx.x];
    partial[(int64_t)blockIdx.x * B + threadIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// Cell-local interpolation kernels (column chunks of CH)
// ---------------------------------------------------------------------------
constexpr int CH = 16;

__global__ void __launch_bounds__(NT) interp_to_quad_kernel(FeView fe, const double *__restrict__ x,
                                                            double *__restrict__ out, int B) {
  extern __shared__ double sm[];
  const int n1 = fe.n1, nd = fe.nd;
  double *A = sm;
  double *b0 = A + n1 * n1, *b1 = b0 + nd * CH, *b2 = b1 + nd * CH;
  for (int i = threadIdx.x; i < n1 * n1; i += blockDim.x) A[i] = fe.phi[i];
  const int64_t e = blockIdx.x;
  for (int c0 = 0; c0 < B; c0 += CH) {
    const int w = min(CH, B - c0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nd * CH; idx += blockDim.x) {
      const int l = idx / CH, k = idx % CH;
      b0[idx] = (k < w) ? x[(int64_t)fe.cell_nodes[e * nd + l] * B + c0 + k] : 0.0;
    }
    __syncthreads();
    tensor3(A, false, b0, b1, b2, n1, CH);
    for (int idx = threadIdx.x; idx < nd * CH; idx += blockDim.x) {
      const int q = idx / CH, k = idx % CH;
      if (k < w) out[(e * nd + q) * B + c0 + k] = b1[idx];
    }
  }
}

__global__ void __launch_bounds__(NT) r_cell_kernel(FeView fe, const double *__restrict__ x,
                                                    const double *__restrict__ wq, double *__restrict__ Ycell,
                                                    int B) {
  extern __shared__ double sm[];
  const int n1 = fe.n1, nd = fe.nd;
  double *A = sm;
  double *b0 = A + n1 * n1, *b1 = b0 + nd * CH, *b2 = b1 + nd * CH;
  for (int i = threadIdx.x; i < n1 * n1; i += blockDim.x) A[i] = fe.phi[i];
  const int64_t e = blockIdx.x;
  for (int c0 = 0; c0 < B; c0 += CH) {
    const int w = min(CH, B - c0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nd * CH; idx += blockDim.x) {
      const int l = idx / CH, k = idx % CH;
      b0[idx] = (k < w) ? x[(int64_t)fe.cell_nodes[e * nd + l] * B + c0 + k] : 0.0;
    }
    __syncthreads();
    tensor3(A, false, b0, b1, b2, n1, CH);
    for (int idx = threadIdx.x; idx < nd * CH; idx += blockDim.x) b1[idx] *= wq[e * nd + idx / CH];
    __syncthreads();
    tensor3(A, true, b1, b0, b2, n1, CH);
    for (int idx = threadIdx.x; idx < nd * CH; idx += blockDim.x) {
      const int l = idx / CH, k = idx % CH;
      const int sl = fe.slot_of[e * nd + l];
      if (k < w && sl >= 0) Ycell[(int64_t)sl * B + c0 + k] = b0[idx];
    }
  }
}

// Ycell[slot(e, l)] = sum_q N_l(q) fw[e*nq + q]: the cell right-hand sides of
// an L2 projection of a quadrature field (fw = f * JxW), by sum factorisation
// with Phi^T along the three directions.
__global__ void __launch_bounds__(NT) quad_rhs_kernel(FeView fe, const double *__restrict__ fw,
                                                      double *__restrict__ Ycell) {
  extern __shared__ double sm[];
  const int n1 = fe.n1, nd = fe.nd;
  double *A = sm;
  double *b0 = A + n1 * n1, *b1 = b0 + nd, *b2 = b1 + nd;
  for (int i = threadIdx.x; i < n1 * n1; i += blockDim.x) A[i] = fe.phi[i];
  const int64_t e = blockIdx.x;
  for (int q = threadIdx.x; q < nd; q += blockDim.x) b0[q] = fw[e * nd + q];
  __syncthreads();
  tensor3(A, true, b0, b1, b2, n1, 1);
  for (int l = threadIdx.x; l < nd; l += blockDim.x) {
    const int sl = fe.slot_of[e * nd + l];
    if (sl >= 0) Ycell[sl] = b1[l];
  }
}

// out[i] = sum_l u[node(cell_i, l)] N_l(xi_i): a parent nodal field at points
// given by their cell and reference coordinates in [0, 1]^3; the Lagrange
// basis on the GLL nodes is evaluated on the fly.
__global__ void eval_points_kernel(FeView fe, const double *__restrict__ gll, const double *__restrict__ u,
                                   int64_t npts, const int64_t *__restrict__ cells,
                                   const double *__restrict__ xi, double *__restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const int n1 = fe.n1;
  double l[3][kSfMaxN];
  for (int d = 0; d < 3; ++d) {
    const double t = xi[3 * i + d];
    for (int a = 0; a < n1; ++a) {
      double v = 1.0;
      for (int b = 0; b < n1; ++b)
        if (b != a) v *= (t - gll[b]) / (gll[a] - gll[b]);
      l[d][a] = v;
    }
  }
  const int64_t e = cells[i];
  const int *cn = fe.cell_nodes + e * fe.nd;
  double acc = 0.0;
  for (int c = 0; c < n1; ++c)
    for (int b = 0; b < n1; ++b) {
      const double wbc = l[1][b] * l[2][c];
      for (int a = 0; a < n1; ++a) acc = fma(l[0][a] * wbc, u[cn[a + n1 * (b + n1 * c)]], acc);
    }
  out[i] = acc;
}

__global__ void __launch_bounds__(NT) density_kernel(FeView fe, const double *__restrict__ psi,
                                                     const double *__restrict__ occ, int N,
                                                     const double *__restrict__ rho_t,
                                                     const double *__restrict__ weight,
                                                     const double *__restrict__ jxw,
                                                     const double *__restrict__ vks, double *__restrict__ rho,
                                                     double *__restrict__ u, double *__restrict__ partial4) {
  extern __shared__ double sm[];
  const int n1 = fe.n1, nd = fe.nd, nq = fe.nq;
  double *A = sm;
  double *b0 = A + n1 * n1, *b1 = b0 + nd * CH, *b2 = b1 + nd * CH, *rs = b2 + nd * CH;
  __shared__ double red[32];
  for (int i = threadIdx.x; i < n1 * n1; i += blockDim.x) A[i] = fe.phi[i];
  for (int q = threadIdx.x; q < nq; q += blockDim.x) rs[q] = 0.0;
  const int64_t e = blockIdx.x;
  for (int c0 = 0; c0 < N; c0 += CH) {
    const int w = min(CH, N - c0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nd * CH; idx += blockDim.x) {
      const int l = idx / CH, k = idx % CH;
      b0[idx] = (k < w) ? psi[(int64_t)fe.cell_nodes[e * nd + l] * N + c0 + k] : 0.0;
    }
    __syncthreads();
    tensor3(A, false, b0, b1, b2, n1, CH);
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
      double s = rs[q];
      for (int k = 0; k < w; ++k) {
        const double v = b1[q * CH + k];
        s = fma(2.0 * occ[c0 + k] * v, v, s);
      }
      rs[q] = s;
    }
  }
  __syncthreads();
  double pl = 0.0, plu = 0.0, pl1 = 0.0, piv = 0.0;
  for (int q = threadIdx.x; q < nq; q += blockDim.x) {
    const int64_t g = e * nq + q;
    const double r = rs[q];
    const double d = rho_t[g] - 0.5 * r;
    rho[g] = r;
    u[g] = d * weight[g];
    pl += d * d * weight[g] * jxw[g];
    plu += d * d * jxw[g];
    pl1 += fabs(d * jxw[g]);
    piv += vks[g] * r * jxw[g];
  }
  pl = block_sum<NT>(pl, red);
  plu = block_sum<NT>(plu, red);
  pl1 = block_sum<NT>(pl1, red);
  piv = block_sum<NT>(piv, red);
  if (threadIdx.x == 0) {
    partial4[e * 4 + 0] = pl;
    partial4[e * 4 + 1] = plu;
    partial4[e * 4 + 2] = pl1;
    partial4[e * 4 + 3] = piv;
  }
}

__global__ void __launch_bounds__(NT) pair_quad_sums_kernel(int nq, const double *__restrict__ Qa,
                                                            const double *__restrict__ Qb,
                                                            const double *__restrict__ w, int B,
                                                            const int *__restrict__ pairs, int npairs,
                                                            double *__restrict__ partial) {
  const int64_t e = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int k = warp; k < npairs; k += nw) {
    const int i = pairs[2 * k], j = pairs[2 * k + 1];
    double s = 0.0;
    for (int q = lane; q < nq; q += 32) {
      const int64_t g = e * nq + q;
      s = fma(w[g] * Qa[g * B + i], Qb[g * B + j], s);
    }
    s = warp_sum(s);
    if (lane == 0) partial[e * npairs + k] = s;
  }
}

__global__ void nullspace_update_kernel(double *x, const double *psi, int64_t n, int B, const int *pair_ptr,
                                        const int *pair_j, const double *coef) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= n * B) return;
  const int64_t r = idx / B;
  const int i = (int)(idx % B);
  double acc = x[idx];
  for (int k = pair_ptr[i]; k < pair_ptr[i + 1]; ++k) acc = fma(coef[k], psi[r * B + pair_j[k]], acc);
  x[idx] = acc;
}

// ---------------------------------------------------------------------------
// MINRES kernels (per-column masks; scalars live on the device)
// ---------------------------------------------------------------------------
__global__ void minres_v_kernel(const double *y, const double *beta, double *v, int64_t n, int B) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= n * B) return;
  const double bt = beta[idx % B];
  v[idx] = bt > 0.0 ? y[idx] / bt : 0.0;
}

__global__ void __launch_bounds__(NT) minres_init_kernel(const double *__restrict__ b, const double *__restrict__ diagA,
                                                         double *r1, double *r2, double *y, int64_t n, int B,
                                                         int64_t rows_per_block, double *partial) {
  __shared__ double red[NT];
  const int RR = NT / B;
  const int j = threadIdx.x % B, rr = threadIdx.x / B;
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1e = min(n, r0 + rows_per_block);
  double acc = 0.0;
  if (rr < RR)
    for (int64_t r = r0 + rr; r < r1e; r += RR) {
      const int64_t idx = r * B + j;
      const double bv = b[idx];
      const double yv = diagA[r] * bv;
      r1[idx] = bv;
      r2[idx] = bv;
      y[idx] = yv;
      acc = fma(bv, yv, acc);
    }
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < B) {
    double s = 0.0;
    for (int q = 0; q < RR; ++q) s += red[q * B + threadIdx.x];
    partial[(int64_t)blockIdx.x * B + threadIdx.x] = s;
  }
}

__global__ void minres_init_scalars_kernel(MinresState st, const double *beta1_sq, int B) {
  const int b = threadIdx.x;
  if (b >= B) return;
  const double b1 = sqrt(fmax(beta1_sq[b], 0.0));
  st.beta[b] = b1;
  st.oldb[b] = 0.0;
  st.dbar[b] = 0.0;
  st.epsln[b] = 0.0;
  st.phibar[b] = b1;
  st.cs[b] = -1.0;
  st.sn[b] = 0.0;
  st.coef1[b] = 0.0;
  st.active[b] = (b1 >= st.tol) ? 1 : 0;
  st.commit[b] = 0;
  st.iters[b] = 0;
}

__global__ void __launch_bounds__(NT) minres_update1_kernel(double *__restrict__ r1, double *__restrict__ r2,
                                                            double *__restrict__ y, const double *__restrict__ yn,
                                                            const double *__restrict__ diagA, MinresState st,
                                                            int64_t n, int B, int64_t rows_per_block,
                                                            double *__restrict__ partial) {
  __shared__ double red[NT];
  const int RR = NT / B;
  const int j = threadIdx.x % B, rr = threadIdx.x / B;
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1e = min(n, r0 + rows_per_block);
  double acc = 0.0;
  if (rr < RR && st.active[j]) {
    const double a = st.alfa[j] / st.beta[j];
    for (int64_t r = r0 + rr; r < r1e; r += RR) {
      const int64_t idx = r * B + j;
      const double r2o = r2[idx];
      const double ynv = yn[idx] - a * r2o;
      const double yv = diagA[r] * ynv;
      r1[idx] = r2o;
      r2[idx] = ynv;
      y[idx] = yv;
      acc = fma(ynv, yv, acc);
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < B) {
    double s = 0.0;
    for (int q = 0; q < RR; ++q) s += red[q * B + threadIdx.x];
    partial[(int64_t)blockIdx.x * B + threadIdx.x] = s;
  }
}

// One column's Paige-Saunders scalar update of an iteration (beta2 = the new
// |r2|_D^2 and alfa already reduced); shared by the scalar kernel and the
// fused update below.
__device__ __forceinline__ void minres_column_scalars(const MinresState &st, int b);

__global__ void minres_scalars_kernel(MinresState st, int B) {
  const int b = threadIdx.x;
  if (b >= B) return;
  minres_column_scalars(st, b);
}

// update1 with the reduction of its dot partials and the scalar update fused
// in: the last CTA to finish (a ticket taken after a fence) sums the partials
// of all CTAs -- one warp per column, lanes over the CTAs in a fixed order --
// into beta2 and runs the scalars; it then resets the ticket.  The sum order
// does not depend on which CTA is last, so results are reproducible.
__global__ void __launch_bounds__(NT) minres_update1_fused_kernel(const double *__restrict__ r2,
                                                                  double *__restrict__ yn,
                                                                  double *__restrict__ y,
                                                                  const double *__restrict__ diagA, MinresState st,
                                                                  int64_t n, int B, int64_t rows_per_block,
                                                                  double *__restrict__ partial,
                                                                  unsigned *__restrict__ ticket) {
  __shared__ double red[NT];
  __shared__ bool last;
  const int RR = NT / B;
  const int j = threadIdx.x % B, rr = threadIdx.x / B;
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1e = min(n, r0 + rows_per_block);
  double acc = 0.0;
  if (rr < RR && st.active[j]) {
    const double a = st.alfa[j] / st.beta[j];
    int64_t r = r0 + rr;
    // four rows in flight per thread (their loads issue together); the dot
    // accumulates in row order, as the one-row loop below does
    for (; r + 3 * RR < r1e; r += 4 * RR) {
      double ynv[4], yv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t ru = r + u * RR, idx = ru * B + j;
        ynv[u] = yn[idx] - a * r2[idx];
        yv[u] = diagA[ru] * ynv[u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t idx = (r + u * RR) * B + j;
        yn[idx] = ynv[u];   // the new r2
        y[idx] = yv[u];
        acc = fma(ynv[u], yv[u], acc);
      }
    }
    for (; r < r1e; r += RR) {
      const int64_t idx = r * B + j;
      const double ynv = yn[idx] - a * r2[idx];
      const double yv = diagA[r] * ynv;
      yn[idx] = ynv;   // the new r2
      y[idx] = yv;
      acc = fma(ynv, yv, acc);
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < B) {
    double sum = 0.0;
    for (int q = 0; q < RR; ++q) sum += red[q * B + threadIdx.x];
    partial[(int64_t)blockIdx.x * B + threadIdx.x] = sum;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  cta_column_sums(partial, (int)gridDim.x, B, st.beta2, red);
  if (threadIdx.x < B) minres_column_scalars(st, threadIdx.x);
  if (threadIdx.x == 0) *ticket = 0u;
}

// update2 (w, w2, x of the committed columns) fused with the next iteration's
// v = y / beta (beta already the new one): each element is read and written by
// one thread, so v is updated in place after its old value is used.
__global__ void minres_update2v_kernel(double *__restrict__ x, const double *__restrict__ w,
                                       double *__restrict__ w2, double *__restrict__ v,
                                       const double *__restrict__ y, MinresState st, int64_t n, int B) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= n * B) return;
  const int b = (int)(idx % B);
  const double vo = v[idx];
  if (st.commit[b]) {
    const double wo = w[idx], w2o = w2[idx];
    const double wn = (vo - st.oldeps[b] * w2o - st.delta[b] * wo) * st.denom[b];
    w2[idx] = wn;   // the new w; the caller swaps w and w2
    x[idx] = fma(st.phi[b], wn, x[idx]);
  }
  const double bt = st.beta[b];
  v[idx] = bt > 0.0 ? y[idx] / bt : 0.0;
}

__device__ __forceinline__ void minres_column_scalars(const MinresState &st, int b) {
  if (!st.active[b]) {
    st.commit[b] = 0;
    return;
  }
  const double beta = st.beta[b];
  const double betan = sqrt(fmax(st.beta2[b], 0.0));
  const double alfa = st.alfa[b];
  const double cs = st.cs[b], sn = st.sn[b], dbar = st.dbar[b];
  const double oldeps = st.epsln[b];
  const double delta = cs * dbar + sn * alfa;
  const double gbar = sn * dbar - cs * alfa;
  const double epsln = sn * betan;
  const double dbarn = -cs * betan;
  double gamma = sqrt(gbar * gbar + betan * betan);
  gamma = fmax(gamma, 2.220446049250313e-16);
  const double csn = gbar / gamma, snn = betan / gamma;
  const double phibar = st.phibar[b];
  const double phi = csn * phibar;
  const double phibarn = snn * phibar;
  st.oldb[b] = beta;
  st.beta[b] = betan;
  st.epsln[b] = epsln;
  st.dbar[b] = dbarn;
  st.cs[b] = csn;
  st.sn[b] = snn;
  st.phibar[b] = phibarn;
  st.oldeps[b] = oldeps;
  st.delta[b] = delta;
  st.denom[b] = 1.0 / gamma;
  st.phi[b] = phi;
  st.coef1[b] = beta > 0.0 ? betan / beta : 0.0;
  st.commit[b] = 1;
  st.iters[b] += 1;
  st.active[b] = (phibarn >= st.tol) ? 1 : 0;
}

__global__ void minres_update2_kernel(double *__restrict__ x, double *__restrict__ w, double *__restrict__ w2,
                                      const double *__restrict__ v, MinresState st, int64_t n, int B) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= n * B) return;
  const int b = (int)(idx % B);
  if (!st.commit[b]) return;
  const double wo = w[idx], w2o = w2[idx];
  const double wn = (v[idx] - st.oldeps[b] * w2o - st.delta[b] * wo) * st.denom[b];
  w2[idx] = wo;
  w[idx] = wn;
  x[idx] = fma(st.phi[b], wn, x[idx]);
}

// ---------------------------------------------------------------------------
// Child mesh transfers
// ---------------------------------------------------------------------------
__global__ void child_to_parent_quad_kernel(ChildView cv, const double *__restrict__ pot,
                                            const double *__restrict__ v_base,
                                            const double *__restrict__ v_lda, double factor_lda,
                                            double *__restrict__ vks, int64_t nqtot) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nqtot) return;
  const int c = cv.pq_child[q];
  const double x = cv.pq_xi[3 * q], y = cv.pq_xi[3 * q + 1], z = cv.pq_xi[3 * q + 2];
  const int *nodes = cv.cell_nodes + (int64_t)c * 8;
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double wx = (k & 1) ? x : 1.0 - x;
    const double wy = (k & 2) ? y : 1.0 - y;
    const double wz = (k & 4) ? z : 1.0 - z;
    v = fma(wx * wy * wz, pot[nodes[k]], v);
  }
  vks[q] = (v_base ? v_base[q] : 0.0) + v + factor_lda * v_lda[q];
}

// One CTA per work item (parent cell, range of its child cells); one warp per
// child cell; lane = state column.  S[c*8+q] += sum_i psi_i(q) p_i(q).
__global__ void __launch_bounds__(NT) psi_adjoint_child_kernel(FeView fe, ChildView cv,
                                                               const double *__restrict__ psi,
                                                               const double *__restrict__ p, int B,
                                                               double *__restrict__ S) {
  extern __shared__ double sm[];
  const int n1 = fe.n1, nd = fe.nd, n2 = n1 * n1;
  double *Us = sm;                  // [nd][32]
  double *Ps = Us + nd * 32;        // [nd][32]
  double *gl = Ps + nd * 32;        // [n1] GLL nodes
  double *inv = gl + n1;            // [n1] inverse denominators
  double *Lw = inv + n1;            // per warp [3][2][n1]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int e = cv.work_parent[blockIdx.x];
  const int c0 = cv.work_c0[blockIdx.x], c1 = cv.work_c1[blockIdx.x];
  if (threadIdx.x < n1) {
    const double xa = cv.gll[threadIdx.x];
    double d = 1.0;
    for (int b = 0; b < n1; ++b)
      if (b != (int)threadIdx.x) d *= (xa - cv.gll[b]);
    gl[threadIdx.x] = xa;
    inv[threadIdx.x] = 1.0 / d;
  }
  double *L = Lw + warp * 6 * n1;
  for (int cb = 0; cb < B; cb += 32) {
    const int wcols = min(32, B - cb);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nd * 32; idx += blockDim.x) {
      const int l = idx >> 5, k = idx & 31;
      const int64_t node = fe.cell_nodes[(int64_t)e * nd + l];
      Us[idx] = (k < wcols) ? psi[node * B + cb + k] : 0.0;
      Ps[idx] = (k < wcols) ? p[node * B + cb + k] : 0.0;
    }
    __syncthreads();
    for (int c = c0 + warp; c < c1; c += nw) {
      for (int t = lane; t < 6 * n1; t += 32) {
        const int dim = t / (2 * n1), pt = (t / n1) % 2, a = t % n1;
        const double xi = cv.offset[(int64_t)c * 3 + dim] + cv.scale[c] * cv.g2[pt];
        double v = inv[a];
        for (int b = 0; b < n1; ++b)
          if (b != a) v *= (xi - gl[b]);
        L[t] = v;   // L[(dim*2 + pt)*n1 + a]
      }
      __syncwarp();
      const double *Lx = L, *Ly = L + 2 * n1, *Lz = L + 4 * n1;
      double op[8], oa[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) { op[q] = 0.0; oa[q] = 0.0; }
      for (int cz = 0; cz < n1; ++cz) {
        double tp[4] = {0, 0, 0, 0}, ta[4] = {0, 0, 0, 0};
        for (int by = 0; by < n1; ++by) {
          double xp0 = 0, xp1 = 0, xa0 = 0, xa1 = 0;
          const int base = (n1 * by + n2 * cz) * 32 + lane;
          for (int a = 0; a < n1; ++a) {
            const double uv = Us[base + a * 32], pv = Ps[base + a * 32];
            xp0 = fma(Lx[a], uv, xp0);
            xp1 = fma(Lx[n1 + a], uv, xp1);
            xa0 = fma(Lx[a], pv, xa0);
            xa1 = fma(Lx[n1 + a], pv, xa1);
          }
          const double ly0 = Ly[by], ly1 = Ly[n1 + by];
          tp[0] = fma(ly0, xp0, tp[0]); tp[1] = fma(ly0, xp1, tp[1]);
          tp[2] = fma(ly1, xp0, tp[2]); tp[3] = fma(ly1, xp1, tp[3]);
          ta[0] = fma(ly0, xa0, ta[0]); ta[1] = fma(ly0, xa1, ta[1]);
          ta[2] = fma(ly1, xa0, ta[2]); ta[3] = fma(ly1, xa1, ta[3]);
        }
        const double lz0 = Lz[cz], lz1 = Lz[n1 + cz];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          op[q] = fma(lz0, tp[q], op[q]);
          op[4 + q] = fma(lz1, tp[q], op[4 + q]);
          oa[q] = fma(lz0, ta[q], oa[q]);
          oa[4 + q] = fma(lz1, ta[q], oa[4 + q]);
        }
      }
      double prod[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) prod[q] = warp_sum(lane < wcols ? op[q] * oa[q] : 0.0);
      if (lane < 8) {
        double pv = prod[0];
#pragma unroll
        for (int q = 1; q < 8; ++q)
          if (lane == q) pv = prod[q];
        S[(int64_t)c * 8 + lane] += pv;
      }
      __syncwarp();
    }
  }
}

__global__ void force_project_kernel(ChildView cv, const double *__restrict__ S, double *__restrict__ force) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= cv.nchild_nodes) return;
  const double g0 = cv.g2[0], g1 = cv.g2[1];
  double f = 0.0;
  for (int k = cv.sc_ptr[n]; k < cv.sc_ptr[n + 1]; ++k) {
    const int src = cv.sc_src[k];
    const int c = src >> 3, kk = src & 7;
    double loc = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double gx = (q & 1) ? g1 : g0, gy = (q & 2) ? g1 : g0, gz = (q & 4) ? g1 : g0;
      const double nk = ((kk & 1) ? gx : 1.0 - gx) * ((kk & 2) ? gy : 1.0 - gy) * ((kk & 4) ? gz : 1.0 - gz);
      const int64_t g = (int64_t)c * 8 + q;
      loc = fma(nk * cv.jxw[g], S[g], loc);
    }
    f = fma(cv.sc_w[k], loc, f);
  }
  force[n] = f;
}

std::atomic<long long> g_launches{0};

}  // namespace

long long launch_count() { return g_launches.load(); }
void count_launch() { g_launches.fetch_add(1); }
void count_launches(long long n) { g_launches.fetch_add(n); }

// ---------------------------------------------------------------------------
// launch wrappers (each counts its launches)
// ---------------------------------------------------------------------------
#undef INVDFT_LAUNCH_CHECK
#define INVDFT_LAUNCH_CHECK()              \
  do {                                     \
    g_launches.fetch_add(1);               \
    INVDFT_CUDA(cudaGetLastError());       \
  } while (0)
void launch_build_cell_h(const FeView &fe, const double *vks, const double *jxw, const double *Kref,
                         double *H, cudaStream_t s) {
  const int n1 = fe.n1, n2 = n1 * n1;
  const size_t smem = sizeof(double) * (size_t)(n2 * n1 + n2 * n1 + n2 * n2 + n1 * n2 * n2);
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(build_cell_h_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  build_cell_h_kernel<<<(unsigned)fe.nc, NT, smem, s>>>(n1, fe.ldh, fe.phi, vks, jxw, Kref, fe.cell_h, H);
  INVDFT_LAUNCH_CHECK();
}

template <int BC, int R>
static void hx_gemm_bc(const FeView &fe, const double *H, const double *x, double *Ycell, int B, int mode,
                       cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(hx_cell_gemm_kernel<BC, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
    attr = true;
  }
  const int rows = (fe.nd + R - 1) / R;
  const int threads = ((rows + 31) / 32) * 32;
  if (threads > NT) throw StatusError(5, "cell too large for the FP64 HX kernel");
  const size_t smem = sizeof(double) * (size_t)(fe.nd + 1) * BC;
  hx_cell_gemm_kernel<BC, R><<<(unsigned)fe.nc, threads, smem, s>>>(fe, H, x, Ycell, B, mode);
  INVDFT_LAUNCH_CHECK();
}

void launch_hx_cell_gemm(const FeView &fe, const double *H, const double *x, double *Ycell, int B,
                         int gather_mode, cudaStream_t s) {
  if (B <= 2) hx_gemm_bc<2, 1>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 4) hx_gemm_bc<4, 1>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 8) hx_gemm_bc<8, 1>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 16) hx_gemm_bc<16, 1>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 32) hx_gemm_bc<32, 1>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 64) hx_gemm_bc<64, 1>(fe, H, x, Ycell, B, gather_mode, s);
  else throw StatusError(5, "block width above 64");
}


template <int NTILE, typename MT>
static void hx_dmma_nt(const FeView &fe, const MT *H, const double *x, double *Ycell, int B, int mode,
                       cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(hx_cell_dmma_kernel<NTILE, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
    attr = true;
  }
  const int mtiles = (fe.nd + 7) / 8;
  const int threads = std::min(NT, 32 * std::max(1, std::min(8, mtiles)));
  const int kpad = 4 * ((fe.nd + 3) / 4);
  const size_t smem = sizeof(double) * (size_t)kpad * 8 * NTILE;
  hx_cell_dmma_kernel<NTILE, MT><<<(unsigned)fe.nc, threads, smem, s>>>(fe, H, x, Ycell, B, mode);
  INVDFT_LAUNCH_CHECK();
}

template <typename MT>
static void dmma_dispatch(const FeView &fe, const MT *H, const double *x, double *Ycell, int B, int gather_mode,
                          cudaStream_t s) {
  if (B <= 8) hx_dmma_nt<1, MT>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 16) hx_dmma_nt<2, MT>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 24) hx_dmma_nt<3, MT>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 32) hx_dmma_nt<4, MT>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 48) hx_dmma_nt<6, MT>(fe, H, x, Ycell, B, gather_mode, s);
  else if (B <= 64) hx_dmma_nt<8, MT>(fe, H, x, Ycell, B, gather_mode, s);
  else throw StatusError(5, "block width above 64");
}

void launch_hx_cell_dmma(const FeView &fe, const double *H, const double *x, double *Ycell, int B,
                         int gather_mode, cudaStream_t s) {
  dmma_dispatch<double>(fe, H, x, Ycell, B, gather_mode, s);
}

void launch_hx_cell_dmma_f32(const FeView &fe, const float *H32, const double *x, double *Ycell, int B,
                             int gather_mode, cudaStream_t s) {
  dmma_dispatch<float>(fe, H32, x, Ycell, B, gather_mode, s);
}

// hvg[h][b] = sum_t w_t (M^-1/2 x)[master_t][b] for every hanging row h (compact
// hanging index), and hvg[nhang][b] = 0 for the Dirichlet entries: the Lowdin
// gather of the constrained rows, so the matrix-free kernel reads each with one
// load.  One CTA per hanging constraint group: the group's master values,
// scaled by M^-1/2, are staged once in shared memory and serve all of its
// rows; the weights are read from the group's (shared, [master][row]) block.
__global__ void __launch_bounds__(NT) group_gather_kernel(FeView fe, const double *__restrict__ x, int B,
                                                          int cap) {
  extern __shared__ double sg[];   // xm [nm][B] | wt [nm][nrp] (rows padded to 4 with zeros)
  const int g = blockIdx.x;
  if (g == 0 && threadIdx.x < B) fe.hvg[(int64_t)fe.nhang * B + threadIdx.x] = 0.0;
  if (g >= fe.ngroup_h) return;   // the launch with no hanging group: the zero row only
  const int nm = fe.g_nm[g], m0 = fe.g_m0[g];
  const int rp0 = fe.g_rptr[g], nr = fe.g_rptr[g + 1] - rp0;
  const int nrp = (nr + 3) & ~3;
  const int h0 = fe.g_hrow[rp0];   // the group's rows have consecutive hanging indices
  const double *wt = fe.g_wt + fe.g_woff[g];
  if ((int64_t)nm * (B + nrp) > cap) {
    // a group too large for the shared staging (rows with hundreds of masters
    // after constraint closure): the same sums, read from global memory
    for (int i = threadIdx.x; i < nr * B; i += blockDim.x) {
      const int q = i / B, j = i - q * B;
      double v = 0.0;
      for (int t = 0; t < nm; ++t) {
        const int mt = fe.cons_masters[m0 + t];
        v = fma(wt[t * nr + q], __dmul_rn(x[(int64_t)mt * B + j], fe.inv_sqrt_mass[mt]), v);
      }
      fe.hvg[(int64_t)(h0 + q) * B + j] = v;
    }
    return;
  }
  double *ws = sg + (size_t)nm * B;
  for (int i = threadIdx.x; i < nm * B; i += blockDim.x) {
    const int t = i / B, j = i - t * B;
    const int mt = fe.cons_masters[m0 + t];
    sg[i] = __dmul_rn(x[(int64_t)mt * B + j], fe.inv_sqrt_mass[mt]);
  }
  for (int i = threadIdx.x; i < nm * nrp; i += blockDim.x) {
    const int t = i / nrp, q = i - t * nrp;
    ws[i] = q < nr ? wt[t * nr + q] : 0.0;
  }
  __syncthreads();
  if (B >= 8) {
    // four rows per thread: each staged master value serves four FMA chains
    for (int i = threadIdx.x; i < (nrp >> 2) * B; i += blockDim.x) {
      const int q0 = (i / B) << 2, j = i % B;
      double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
      for (int t = 0; t < nm; ++t) {
        const double xs = sg[t * B + j];
        const double *wr = ws + t * nrp + q0;
        v0 = fma(wr[0], xs, v0);
        v1 = fma(wr[1], xs, v1);
        v2 = fma(wr[2], xs, v2);
        v3 = fma(wr[3], xs, v3);
      }
      const double vv[4] = {v0, v1, v2, v3};
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (q0 + u < nr) fe.hvg[(int64_t)(h0 + q0 + u) * B + j] = vv[u];
    }
  } else {
    for (int i = threadIdx.x; i < nr * B; i += blockDim.x) {
      const int q = i / B, j = i - q * B;
      double v = 0.0;
      for (int t = 0; t < nm; ++t) v = fma(ws[t * nrp + q], sg[t * B + j], v);
      fe.hvg[(int64_t)(h0 + q) * B + j] = v;
    }
  }
}

template <int N, int MINB, bool GXS = false, typename T = double, bool PRE = false>
static void hx_sf_n(const FeView &fe, const SfMatsT<T> &mt, const double *vj, const double *x, double *Ycell, int B,
                    int mode, cudaStream_t s) {
  constexpr int threads = 16 * N * N;
  const size_t smem = sizeof(T) * (GXS ? 4 : 3) * (size_t)N * N * N * 16 + (PRE ? sizeof(double) * N * N * N * 16 : 0);
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(hx_cell_sf_kernel<N, MINB, GXS, T, PRE>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  // C columns of 16/C cells per CTA; C = the smallest power of two >= B, at most 16
  int C = 1;
  while (C < B && C < 16) C <<= 1;
  const int G = 16 / C;
  const dim3 grid((unsigned)((fe.nc + G - 1) / G), (unsigned)((B + C - 1) / C));
  hx_cell_sf_kernel<N, MINB, GXS, T, PRE><<<grid, threads, smem, s>>>(fe, mt, vj, x, Ycell, B, C, mode);
  INVDFT_LAUNCH_CHECK();
}

template <int N, int MINB>
static void hx_sf2_n(const FeView &fe, const SfMats &mt, const double *vj, const double *x, double *Ycell, int B,
                     int mode, cudaStream_t s) {
  constexpr int threads = 8 * N * N;
  const size_t smem = sizeof(double) * 3 * (size_t)N * N * N * 16;
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(hx_cell_sf2_kernel<N, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    attr = true;
  }
  int C = 1;
  while (C < B && C < 16) C <<= 1;
  const int G = 16 / C;
  const dim3 grid((unsigned)((fe.nc + G - 1) / G), (unsigned)((B + C - 1) / C));
  hx_cell_sf2_kernel<N, MINB><<<grid, threads, smem, s>>>(fe, mt, vj, x, Ycell, B, C, mode);
  INVDFT_LAUNCH_CHECK();
}

template <int MINB>
static void hx_sf_dispatch(const FeView &fe, const SfMats &mt, const double *vj, const double *x, double *Ycell,
                           int B, int mode, cudaStream_t s) {
  switch (fe.n1) {
    case 2: hx_sf_n<2, MINB>(fe, mt, vj, x, Ycell, B, mode, s); break;
    case 3: hx_sf_n<3, MINB>(fe, mt, vj, x, Ycell, B, mode, s); break;
    case 4: hx_sf_n<4, MINB>(fe, mt, vj, x, Ycell, B, mode, s); break;
    case 5: hx_sf_n<5, MINB>(fe, mt, vj, x, Ycell, B, mode, s); break;
    case 6: hx_sf_n<6, MINB>(fe, mt, vj, x, Ycell, B, mode, s); break;
    case 7: if (MINB == 1) { hx_sf_n<7, 1>(fe, mt, vj, x, Ycell, B, mode, s); break; }
      [[fallthrough]];
    default: throw StatusError(5, "matrix-free HX: FE order outside the compiled launch shapes");
  }
}

static void launch_group_gather(const FeView &fe, const double *x, int B, int gather_mode, cudaStream_t s) {
  if (gather_mode != GATHER_PLAIN && fe.ngroup > 0) {
    // staging capacity: the largest group's need, at most fe.g_stage doubles
    const int cap = (int)std::min<int64_t>((int64_t)std::max(fe.g_maxnm, 1) * (B + ((fe.g_maxnr + 3) & ~3)),
                                           fe.g_stage);
    static bool attr = false;
    if (!attr) {
      INVDFT_CUDA(cudaFuncSetAttribute(group_gather_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      attr = true;
    }
    // the hanging groups; block 0 also writes the zero row.  (64-thread CTAs
    // for narrow blocks were measured slower at c1: B = 1 HX 0.186 vs 0.169 ms)
    group_gather_kernel<<<std::max(fe.ngroup_h, 1), NT, sizeof(double) * (size_t)cap, s>>>(fe, x, B, cap);
    INVDFT_LAUNCH_CHECK();
  }
}

void launch_hx_cell_sf_f32(const FeView &fe, const SfMatsT<float> &mt, const double *vj, const double *x,
                           double *Ycell, int B, int gather_mode, cudaStream_t s) {
  launch_group_gather(fe, x, B, gather_mode, s);
  switch (fe.n1) {
    case 2: hx_sf_n<2, 2, false, float>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 3: hx_sf_n<3, 2, false, float>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 4: hx_sf_n<4, 2, false, float>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 5: hx_sf_n<5, 2, false, float>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 6: hx_sf_n<6, 2, false, float>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 7: hx_sf_n<7, 1, false, float>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 8: hx_sf_n<8, 1, false, float>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    default: throw StatusError(5, "matrix-free HX supports FE orders 1..7");
  }
}

template <typename T>
static void hx_sf_tc(const FeView &fe, const SfMatsT<T> &mt, const double *vj, const double *x, double *Ycell,
                     int B, int gather_mode, cudaStream_t s) {
  launch_group_gather(fe, x, B, gather_mode, s);
  switch (fe.n1) {
    case 3: hx_sf_n<3, 2, false, T>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 5: hx_sf_n<5, 2, false, T>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    case 6: hx_sf_n<6, 2, false, T>(fe, mt, vj, x, Ycell, B, gather_mode, s); break;
    default: throw StatusError(5, "tensor-core operand rounding is built for FE orders 2, 4 and 5");
  }
}
void launch_hx_cell_sf_tc(const FeView &fe, const SfMatsT<Tf32Operand> &mt, const double *vj, const double *x,
                          double *Ycell, int B, int gather_mode, cudaStream_t s) {
  hx_sf_tc(fe, mt, vj, x, Ycell, B, gather_mode, s);
}
void launch_hx_cell_sf_tc(const FeView &fe, const SfMatsT<Bf16Operand> &mt, const double *vj, const double *x,
                          double *Ycell, int B, int gather_mode, cudaStream_t s) {
  hx_sf_tc(fe, mt, vj, x, Ycell, B, gather_mode, s);
}

void launch_hx_cell_sf(const FeView &fe, const SfMats &mt, const double *vj, const double *x, double *Ycell,
                       int B, int gather_mode, int tune, cudaStream_t s) {
  launch_group_gather(fe, x, B, gather_mode, s);
  if (tune == 2 && fe.n1 == 6) {   // two CTAs per SM, derivative lines in shared memory
    hx_sf_n<6, 2, true>(fe, mt, vj, x, Ycell, B, gather_mode, s);
    return;
  }
  if (tune == 3 && fe.n1 == 6) {   // two CTAs per SM, potential and slot indices prefetched by cp.async
    hx_sf_n<6, 2, false, double, true>(fe, mt, vj, x, Ycell, B, gather_mode, s);
    return;
  }
  if (tune == 3 && fe.n1 == 5) {
    hx_sf_n<5, 2, false, double, true>(fe, mt, vj, x, Ycell, B, gather_mode, s);
    return;
  }
  if (tune == 4 && fe.n1 == 6) {   // two pairs per thread, two CTAs per SM
    hx_sf2_n<6, 2>(fe, mt, vj, x, Ycell, B, gather_mode, s);
    return;
  }
  if (tune == 4 && fe.n1 == 5) {
    hx_sf2_n<5, 2>(fe, mt, vj, x, Ycell, B, gather_mode, s);
    return;
  }
  if (tune >= 1 && fe.n1 <= 6) {
    hx_sf_dispatch<2>(fe, mt, vj, x, Ycell, B, gather_mode, s);
    return;
  }
  if (fe.n1 == 8) {
    hx_sf_n<8, 1>(fe, mt, vj, x, Ycell, B, gather_mode, s);
    return;
  }
  hx_sf_dispatch<1>(fe, mt, vj, x, Ycell, B, gather_mode, s);
}

__global__ void transpose_kernel(const double *__restrict__ a, double *__restrict__ out, int64_t rows,
                                 int64_t cols) {
  __shared__ double t[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int64_t r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[i][threadIdx.x] = a[r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int64_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = t[threadIdx.x][i];
  }
}

void launch_transpose(const double *a, double *out, int64_t rows, int64_t cols, cudaStream_t s) {
  if (rows * cols == 0) return;
  const dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(a, out, rows, cols);
  INVDFT_LAUNCH_CHECK();
}

__global__ void mul_kernel(const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ out,
                           int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] * b[i];
}

__global__ void axpbypcz_kernel(double *__restrict__ out, double a, const double *__restrict__ x, double b,
                                const double *__restrict__ y, double c, const double *__restrict__ z, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = a * x[i];
  if (y) v = fma(b, y[i], v);
  if (z) v = fma(c, z[i], v);
  out[i] = v;
}

void launch_axpbypcz(double *out, double a, const double *x, double b, const double *y, double c, const double *z,
                     int64_t n, cudaStream_t s) {
  if (n == 0) return;
  axpbypcz_kernel<<<ceil_div(n, NT), NT, 0, s>>>(out, a, x, b, y, c, z, n);
  INVDFT_LAUNCH_CHECK();
}

void launch_mul(const double *a, const double *b, double *out, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  mul_kernel<<<ceil_div(n, NT), NT, 0, s>>>(a, b, out, n);
  INVDFT_LAUNCH_CHECK();
}

__global__ void narrow_kernel(const double *__restrict__ src, float *__restrict__ dst, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __double2float_rn(src[i]);
}

void launch_narrow(const double *src, float *dst, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  narrow_kernel<<<ceil_div(n, NT), NT, 0, s>>>(src, dst, n);
  INVDFT_LAUNCH_CHECK();
}

template <int BC>
static void hx_gemm_bulk_bc(const FeView &fe, const double *H, const double *x, double *Yslot, int B, int mode,
                            cudaStream_t s) {
  static bool attr = false;
  static int nsm = 0;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(hx_gemm_bulk_kernel<BC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     210 * 1024));
    int dev = 0;
    INVDFT_CUDA(cudaGetDevice(&dev));
    INVDFT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    attr = true;
  }
  const int threads = ((fe.nd + 31) / 32) * 32;
  if (threads > NT) throw StatusError(5, "cell too large for the FP64 HX kernel");
  const int PW = 16;
  const size_t stage = (size_t)PW * fe.ldh * 8;
  const size_t xsb = (size_t)(fe.nd + 1) * BC * 8;
  const size_t budget = 200 * 1024;
  if (xsb + 2 * stage + 64 > budget) throw StatusError(5, "block too wide for the staged HX kernel");
  int S = (int)((budget - xsb - 64) / stage);
  if (S > 8) S = 8;
  const size_t smem = (size_t)S * stage + xsb + (size_t)S * 8;
  const int grid = (int)std::min<int64_t>(fe.nc, nsm);
  hx_gemm_bulk_kernel<BC><<<grid, threads, smem, s>>>(fe, H, x, Yslot, B, mode, S, PW);
  INVDFT_LAUNCH_CHECK();
}

void launch_hx_cell_gemm_bulk(const FeView &fe, const double *H, const double *x, double *Yslot, int B,
                              int gather_mode, cudaStream_t s) {
  if (B <= 2) hx_gemm_bulk_bc<2>(fe, H, x, Yslot, B, gather_mode, s);
  else if (B <= 4) hx_gemm_bulk_bc<4>(fe, H, x, Yslot, B, gather_mode, s);
  else if (B <= 8) hx_gemm_bulk_bc<8>(fe, H, x, Yslot, B, gather_mode, s);
  else if (B <= 16) hx_gemm_bulk_bc<16>(fe, H, x, Yslot, B, gather_mode, s);
  else if (B <= 32) hx_gemm_bulk_bc<32>(fe, H, x, Yslot, B, gather_mode, s);
  else if (B <= 64) hx_gemm_bulk_bc<64>(fe, H, x, Yslot, B, gather_mode, s);
  else throw StatusError(5, "block width above 64");
}

static void assemble_shape(int B, int &TR, int &cap) {
  TR = std::max(8, std::min(B <= 4 ? 512 : 128, 1024 / B));   // every thread busy at small widths
  cap = 2 * TR;   // ~1.6 slots per node on average
}

// launch shape of the bulk-pipelined assembly: TR nodes per tile (a multiple
// of 4), 2 TR slots per stage, two stages; persistent grid of as many CTAs as
// fit on the SMs, at most one per full tile
struct AsmBulkShape {
  int TR, cap, grid;
  size_t smem;
};
static AsmBulkShape asm_bulk_shape(const FeView &fe, int B) {
  AsmBulkShape sh;
  sh.TR = std::max(16, std::min(256, 1024 / B)) & ~3;
  sh.cap = 2 * sh.TR;
  const size_t seg_n = (size_t)sh.cap * B + 2, blk = (size_t)sh.TR * B;
  const size_t stage = 8 * (seg_n + 2 * blk + sh.TR) + 4 * ((size_t)sh.TR + 4);
  sh.smem = 2 * ((stage + 127) & ~(size_t)127);
  static int nsm = 0;
  static int occ[257] = {};
  if (!nsm) {
    int dev = 0;
    INVDFT_CUDA(cudaGetDevice(&dev));
    INVDFT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    INVDFT_CUDA(cudaFuncSetAttribute(hx_assemble_bulk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
  }
  if (!occ[B]) {
    int o = 0;
    INVDFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, hx_assemble_bulk_kernel, NT, sh.smem));
    occ[B] = std::max(o, 1);
  }
  const int64_t nfull = fe.nnodes / sh.TR;
  sh.grid = (int)std::max<int64_t>(1, std::min<int64_t>(nfull, (int64_t)occ[B] * nsm));
  return sh;
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

int assemble_blocks(const FeView &fe, int B) {
  int TR, cap;
  assemble_shape(B, TR, cap);
  const int tiled = (int)((fe.nnodes + TR - 1) / TR);
  return std::max(tiled, asm_bulk_shape(fe, B).grid);
}

int launch_hx_assemble(const FeView &fe, const double *Ycell, double *out, int B, const AsmEpilogue &epi,
                       int dot_blocks, cudaStream_t s) {
  (void)dot_blocks;
  if (B > NT) throw StatusError(5, "block width above 256");
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(hx_assemble_tile_kernel<AsmEpilogue::STORE>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    INVDFT_CUDA(cudaFuncSetAttribute(hx_assemble_tile_kernel<AsmEpilogue::CHEB>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    INVDFT_CUDA(cudaFuncSetAttribute(hx_assemble_tile_kernel<AsmEpilogue::VMULT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    INVDFT_CUDA(cudaFuncSetAttribute(hx_assemble_tile_kernel<AsmEpilogue::RHS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    INVDFT_CUDA(cudaFuncSetAttribute(hx_assemble_tile_kernel<AsmEpilogue::MINRES>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    attr = true;
  }
  int TR, cap;
  assemble_shape(B, TR, cap);
  if (TR + 1 > kAsmRow * NT || TR * B > kAsmBlk * NT || cap * B > kAsmSeg * NT)
    throw StatusError(5, "assembly tile larger than its staging shares");
  const int nb = (int)((fe.nnodes + TR - 1) / TR);   // one tile of TR nodes per CTA
  if (fe.nmast > 0) {
    const int cap = (int)std::min<int64_t>((int64_t)std::max(fe.g_maxnr, 1) * (B + ((std::max(fe.g_maxnm, 1) + 3) & ~3)),
                                           fe.g_stage);
    static bool attr = false;
    if (!attr) {
      INVDFT_CUDA(cudaFuncSetAttribute(group_partial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      attr = true;
    }
    group_partial_kernel<<<fe.ngroup_h, NT, sizeof(double) * (size_t)cap, s>>>(fe, Ycell, B, cap);
    INVDFT_LAUNCH_CHECK();
    master_sum_kernel<<<ceil_div((int64_t)fe.nmast * B, NT), NT, 0, s>>>(fe, B, const_cast<double *>(Ycell));
    INVDFT_LAUNCH_CHECK();
  }
  // one tile per CTA by default; INVDFT_ASM_KERNEL=bulk selects the
  // bulk-pipelined persistent variant
  static const bool want_bulk = [] {
    const char *v = std::getenv("INVDFT_ASM_KERNEL");
    return v && std::string(v) == "bulk";
  }();
  const bool bulk_ok = want_bulk && aligned16(Ycell) && aligned16(fe.dptr) &&
                       aligned16(fe.inv_sqrt_mass) && (!epi.in || aligned16(epi.in)) &&
                       (!epi.prev || aligned16(epi.prev));
  if (bulk_ok) {
    const AsmBulkShape sh = asm_bulk_shape(fe, B);
    hx_assemble_bulk_kernel<<<sh.grid, NT, sh.smem, s>>>(fe, Ycell, out, B, epi, sh.TR, sh.cap);
    INVDFT_LAUNCH_CHECK();
    return sh.grid;
  }
  const size_t smem = sizeof(double) * ((size_t)cap * B + 2 * (size_t)TR * B + TR) + sizeof(int) * (TR + 1);
  // the last CTA reduces the MINRES dot partials itself only while they are
  // few (at most 32 per thread); more go to the B-CTA reduction kernel
  AsmEpilogue e2 = epi;
  const bool fuse_dot = epi.kind == AsmEpilogue::MINRES && epi.dot_ticket && (int64_t)nb * B <= 32 * NT;
  if (!fuse_dot) e2.dot_ticket = nullptr;
  switch (epi.kind) {
    case AsmEpilogue::STORE:
      hx_assemble_tile_kernel<AsmEpilogue::STORE><<<nb, NT, smem, s>>>(fe, Ycell, out, B, e2, TR, cap);
      break;
    case AsmEpilogue::CHEB:
      hx_assemble_tile_kernel<AsmEpilogue::CHEB><<<nb, NT, smem, s>>>(fe, Ycell, out, B, e2, TR, cap);
      break;
    case AsmEpilogue::VMULT:
      hx_assemble_tile_kernel<AsmEpilogue::VMULT><<<nb, NT, smem, s>>>(fe, Ycell, out, B, e2, TR, cap);
      break;
    case AsmEpilogue::RHS:
      hx_assemble_tile_kernel<AsmEpilogue::RHS><<<nb, NT, smem, s>>>(fe, Ycell, out, B, e2, TR, cap);
      break;
    default:
      hx_assemble_tile_kernel<AsmEpilogue::MINRES><<<nb, NT, smem, s>>>(fe, Ycell, out, B, e2, TR, cap);
  }
  INVDFT_LAUNCH_CHECK();
  return fuse_dot ? 0 : nb;
}

void launch_scale_rows(const double *d, const double *x, double *y, int64_t n, int B, cudaStream_t s) {
  if (n * B == 0) return;
  scale_rows_kernel<<<ceil_div(n * B, NT), NT, 0, s>>>(d, x, y, n, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_distribute(const int *rows, const int *ptr, const int *masters, const double *w, int nrows,
                       double *x, int B, cudaStream_t s) {
  if ((int64_t)nrows * B == 0) return;
  distribute_kernel<<<ceil_div((int64_t)nrows * B, NT), NT, 0, s>>>(rows, ptr, masters, w, nrows, x, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_set_zero(const int *rows, int nrows, double *x, int B, cudaStream_t s) {
  if ((int64_t)nrows * B == 0) return;
  set_zero_kernel<<<ceil_div((int64_t)nrows * B, NT), NT, 0, s>>>(rows, nrows, x, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_reduce_partials(const double *partial, int nparts, int width, double *out, cudaStream_t s) {
  if (width <= 0) return;
  reduce_partials_kernel<<<width, NT, 0, s>>>(partial, nparts, width, out);
  INVDFT_LAUNCH_CHECK();
}

void launch_gram(const double *A, const double *Bm, int64_t n, int N, double *partial, int nblocks,
                 double *out, cudaStream_t s) {
  if (N > 64) throw StatusError(5, "subspace wider than 64");
  const int64_t rpb = (n + nblocks - 1) / nblocks;
  const int K = (N * N + NT - 1) / NT;
  if (K <= 1) gram_kernel<1><<<nblocks, NT, 0, s>>>(A, Bm, n, N, rpb, partial);
  else if (K <= 4) gram_kernel<4><<<nblocks, NT, 0, s>>>(A, Bm, n, N, rpb, partial);
  else gram_kernel<16><<<nblocks, NT, 0, s>>>(A, Bm, n, N, rpb, partial);
  INVDFT_LAUNCH_CHECK();
  launch_reduce_partials(partial, nblocks, N * N, out, s);
}

void launch_rotate(const double *Y, const double *T, double *Z, int64_t n, int N, cudaStream_t s) {
  rotate_kernel<<<ceil_div(n * N, NT), NT, 0, s>>>(Y, T, Z, n, N);
  INVDFT_LAUNCH_CHECK();
}

void launch_rotate_residual(const double *Y, const double *HY, const double *Q, const double *eps, double *X,
                            int64_t n, int N, double *partial, int nblocks, double *out, cudaStream_t s) {
  const int64_t rpb = (n + nblocks - 1) / nblocks;
  rotate_residual_kernel<<<nblocks, NT, 0, s>>>(Y, HY, Q, eps, X, n, N, rpb, partial);
  INVDFT_LAUNCH_CHECK();
  launch_reduce_partials(partial, nblocks, N, out, s);
}

void launch_coldot(const double *a, const double *b, int64_t n, int B, double *partial, int nblocks,
                   double *out, cudaStream_t s) {
  const int64_t rpb = (n + nblocks - 1) / nblocks;
  coldot_kernel<<<nblocks, NT, 0, s>>>(a, b, n, B, rpb, partial);
  INVDFT_LAUNCH_CHECK();
  launch_reduce_partials(partial, nblocks, B, out, s);
}

static size_t interp_smem(const FeView &fe, int extra) {
  return sizeof(double) * ((size_t)fe.n1 * fe.n1 + 3 * (size_t)fe.nd * CH + extra);
}

void launch_interp_to_quad(const FeView &fe, const double *x, double *out, int B, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(interp_to_quad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  interp_to_quad_kernel<<<(unsigned)fe.nc, NT, interp_smem(fe, 0), s>>>(fe, x, out, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_pair_quad_sums(const FeView &fe, const double *Qa, const double *Qb, const double *w, int B,
                           const int *pairs, int npairs, double *partial, cudaStream_t s) {
  if (npairs == 0) return;
  pair_quad_sums_kernel<<<(unsigned)fe.nc, NT, 0, s>>>(fe.nq, Qa, Qb, w, B, pairs, npairs, partial);
  INVDFT_LAUNCH_CHECK();
}

void launch_r_cell(const FeView &fe, const double *x, const double *wq, double *Ycell, int B, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(r_cell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  r_cell_kernel<<<(unsigned)fe.nc, NT, interp_smem(fe, 0), s>>>(fe, x, wq, Ycell, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_quad_rhs(const FeView &fe, const double *fw, double *Ycell, cudaStream_t s) {
  const size_t smem = sizeof(double) * ((size_t)fe.n1 * fe.n1 + 3 * (size_t)fe.nd);
  quad_rhs_kernel<<<(unsigned)fe.nc, NT, smem, s>>>(fe, fw, Ycell);
  INVDFT_LAUNCH_CHECK();
}

void launch_eval_points(const FeView &fe, const double *gll, const double *u, int64_t npts, const int64_t *cells,
                        const double *xi, double *out, cudaStream_t s) {
  if (npts == 0) return;
  eval_points_kernel<<<ceil_div(npts, NT), NT, 0, s>>>(fe, gll, u, npts, cells, xi, out);
  INVDFT_LAUNCH_CHECK();
}

void launch_density(const FeView &fe, const double *psi, const double *occ, int N, const double *rho_t,
                    const double *weight, const double *jxw, const double *vks, double *rho, double *u,
                    double *partial4, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(density_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  density_kernel<<<(unsigned)fe.nc, NT, interp_smem(fe, fe.nq), s>>>(fe, psi, occ, N, rho_t, weight, jxw, vks,
                                                                     rho, u, partial4);
  INVDFT_LAUNCH_CHECK();
}

void launch_nullspace_update(double *x, const double *psi, int64_t n, int B, const int *pair_ptr,
                             const int *pair_j, const double *coef, cudaStream_t s) {
  nullspace_update_kernel<<<ceil_div(n * B, NT), NT, 0, s>>>(x, psi, n, B, pair_ptr, pair_j, coef);
  INVDFT_LAUNCH_CHECK();
}

void launch_minres_v(const double *y, const MinresState &st, double *v, int64_t n, int B, cudaStream_t s) {
  minres_v_kernel<<<ceil_div(n * B, NT), NT, 0, s>>>(y, st.beta, v, n, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_minres_init(const double *b, const double *diagA, double *r1, double *r2, double *y, int64_t n,
                        int B, double *partial, int nblocks, cudaStream_t s) {
  const int64_t rpb = (n + nblocks - 1) / nblocks;
  minres_init_kernel<<<nblocks, NT, 0, s>>>(b, diagA, r1, r2, y, n, B, rpb, partial);
  INVDFT_LAUNCH_CHECK();
}

void launch_minres_init_scalars(const MinresState &st, const double *beta1_sq, int B, cudaStream_t s) {
  minres_init_scalars_kernel<<<1, 64, 0, s>>>(st, beta1_sq, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_minres_update1(double *r1, double *r2, double *y, const double *yn, const double *diagA,
                           const MinresState &st, int64_t n, int B, double *partial, int nblocks,
                           cudaStream_t s) {
  const int64_t rpb = (n + nblocks - 1) / nblocks;
  minres_update1_kernel<<<nblocks, NT, 0, s>>>(r1, r2, y, yn, diagA, st, n, B, rpb, partial);
  INVDFT_LAUNCH_CHECK();
  launch_reduce_partials(partial, nblocks, B, st.beta2, s);
}

void launch_minres_update1_fused(const double *r2, double *yn, double *y, const double *diagA,
                                 const MinresState &st, int64_t n, int B, double *partial, int nblocks,
                                 unsigned *ticket, cudaStream_t s) {
  const int64_t rpb = (n + nblocks - 1) / nblocks;
  minres_update1_fused_kernel<<<nblocks, NT, 0, s>>>(r2, yn, y, diagA, st, n, B, rpb, partial, ticket);
  INVDFT_LAUNCH_CHECK();
}

void launch_minres_update2v(double *x, const double *w, double *w2, double *v, const double *y,
                            const MinresState &st, int64_t n, int B, cudaStream_t s) {
  minres_update2v_kernel<<<ceil_div(n * B, NT), NT, 0, s>>>(x, w, w2, v, y, st, n, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_minres_scalars(const MinresState &st, int B, int itn, cudaStream_t s) {
  (void)itn;
  minres_scalars_kernel<<<1, 64, 0, s>>>(st, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_minres_update2(double *x, double *w, double *w2, const double *v, const MinresState &st,
                           int64_t n, int B, cudaStream_t s) {
  minres_update2_kernel<<<ceil_div(n * B, NT), NT, 0, s>>>(x, w, w2, v, st, n, B);
  INVDFT_LAUNCH_CHECK();
}

void launch_child_to_parent_quad(const ChildView &cv, const double *pot, const double *v_base,
                                 const double *v_lda, double factor_lda, double *vks, int64_t nqtot,
                                 cudaStream_t s) {
  child_to_parent_quad_kernel<<<ceil_div(nqtot, NT), NT, 0, s>>>(cv, pot, v_base, v_lda, factor_lda, vks, nqtot);
  INVDFT_LAUNCH_CHECK();
}

void launch_psi_adjoint_child(const FeView &fe, const ChildView &cv, const double *psi, const double *p, int B,
                              double *S, cudaStream_t s) {
  if (cv.nwork == 0) return;
  static bool attr = false;
  if (!attr) {
    INVDFT_CUDA(cudaFuncSetAttribute(psi_adjoint_child_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
    attr = true;
  }
  const size_t smem = sizeof(double) * ((size_t)fe.nd * 64 + 2 * fe.n1 + (NT / 32) * 6 * fe.n1);
  psi_adjoint_child_kernel<<<cv.nwork, NT, smem, s>>>(fe, cv, psi, p, B, S);
  INVDFT_LAUNCH_CHECK();
}

void launch_force_project(const ChildView &cv, const double *S, double *force, cudaStream_t s) {
  force_project_kernel<<<ceil_div(cv.nchild_nodes, NT), NT, 0, s>>>(cv, S, force);
  INVDFT_LAUNCH_CHECK();
}

}  // namespace invdft
