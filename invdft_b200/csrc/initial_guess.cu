// Initial v_xc guess on the GPU: InverseDFTEngine::setInitialPotL2Proj
// (src/InverseDFTEngine.cpp:1046-1498).
//
// At the parent quadrature points, from the total target density rho:
//   v_x      LDA exchange, or LB94 exchange when |grad rho|^2 is given
//            (:1183-1199; libxc XC_LDA_X / XC_GGA_X_LB),
//   v_c      Perdew-Wang 1992 correlation (:1200-1206; libxc XC_LDA_C_PW),
//   v        = (1 - p) v_x + p (v_x + v_c),  p = rho / (rho + tau_vx)   (:1255-1270)
//   with the Fermi-Amaldi far field (:1272-1289):
//   v        = q v + (1 - q) (-factor_fa / N_e) v_H,  q = rho / (rho + tau_fa),
// v_H the Hartree potential of rho with the boundary values of
// computeHartreePotOnParentQuad (:1790-2118).  v is projected onto the parent
// nodes (l2ProjectionQuadToNodal with the psi constraints, :1311-1320, then
// distributed), evaluated at the Gauss points of the child (v_xc) cells
// (:1415-1419), scaled by 1 - factorForLDAVxc (:1421-1427) and projected onto
// the child nodes (:1429-1433) whose constrained entries are zeroed (:1434).
// The L2 projections use the lumped (row-sum) mass of each space, as the
// POST_PROCESS projection of this library does.
//
// The exchange-correlation forms are the published ones, written here:
// Slater exchange v_x = -(3 rho / pi)^(1/3); PW92 correlation
// e_c = -2A(1 + a1 rs) ln(1 + 1 / (2A (b1 rs^1/2 + b2 rs + b3 rs^3/2 + b4 rs^2)))
// with v_c = e_c - rs/3 de_c/drs; LB94 (van Leeuwen and Baerends 1994) per
// spin, v_x,s = v_x^LDA(rho_s) - beta rho_s^1/3 x_s^2 / (1 + 3 beta x_s asinh(x_s)),
// x_s = |grad rho_s| / rho_s^4/3, beta = 0.05, rho_s = rho / 2.
#include <cmath>

#include "context.h"

namespace invdft {

namespace {

__device__ double pw92_vc(double rho) {
  const double A = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
  const double rs = cbrt(3.0 / (4.0 * M_PI * rho));
  const double sr = sqrt(rs);
  const double q0 = -2.0 * A * (1.0 + a1 * rs);
  const double q1 = 2.0 * A * (b1 * sr + b2 * rs + b3 * rs * sr + b4 * rs * rs);
  const double q1p = A * (b1 / sr + 2.0 * b2 + 3.0 * b3 * sr + 4.0 * b4 * rs);
  const double lg = log1p(1.0 / q1);
  const double ec = q0 * lg;
  const double dec = -2.0 * A * a1 * lg - q0 * q1p / (q1 * q1 + q1);
  return ec - rs / 3.0 * dec;
}

__global__ void initial_guess_quad_kernel(const double *__restrict__ rho, const double *__restrict__ sigma,
                                          const double *__restrict__ vh, int64_t n, double tau_vx, double tau_fa,
                                          int fa_bc, double fa_scale, double *__restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r = fmax(rho[i], 1e-30);
  double vx = -cbrt(3.0 * r / M_PI);
  if (sigma) {
    const double rs = 0.5 * r, gs = 0.5 * sqrt(fmax(sigma[i], 0.0));
    const double x = gs / pow(rs, 4.0 / 3.0);
    const double beta = 0.05;
    vx -= beta * cbrt(rs) * x * x / (1.0 + 3.0 * beta * x * asinh(x));
  }
  const double vc = pw92_vc(r);
  const double p = rho[i] / (rho[i] + tau_vx);
  double v = (1.0 - p) * vx + p * (vx + vc);
  if (fa_bc) {
    const double q = rho[i] / (rho[i] + tau_fa);
    v = q * v + (1.0 - q) * fa_scale * vh[i];
  }
  out[i] = v;
}

// value of the parent nodal field u at the 2x2x2 Gauss points of every child
// cell, with the parent's Lagrange basis evaluated on the fly; out [ncc*8]
__global__ void parent_field_child_quad_kernel(FeView fe, ChildView cv, const double *__restrict__ u, double scale,
                                               double *__restrict__ out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= cv.ncc * 8) return;
  const int64_t c = t >> 3;
  const int qp = (int)(t & 7);
  const int n1 = fe.n1;
  const int64_t e = cv.parent[c];
  double l[3][kSfMaxN];
  for (int d = 0; d < 3; ++d) {
    const double xi = cv.offset[c * 3 + d] + cv.scale[c] * cv.g2[(qp >> d) & 1];
    for (int a = 0; a < n1; ++a) {
      double v = 1.0;
      for (int b = 0; b < n1; ++b)
        if (b != a) v *= (xi - cv.gll[b]) / (cv.gll[a] - cv.gll[b]);
      l[d][a] = v;
    }
  }
  const int *cn = fe.cell_nodes + e * fe.nd;
  double acc = 0.0;
  for (int k3 = 0; k3 < n1; ++k3)
    for (int k2 = 0; k2 < n1; ++k2) {
      const double w = l[1][k2] * l[2][k3];
      for (int k1 = 0; k1 < n1; ++k1) acc = fma(l[0][k1] * w, u[cn[k1 + n1 * (k2 + n1 * k3)]], acc);
    }
  out[t] = scale * acc;
}

__global__ void divide_free_kernel(const double *__restrict__ r, const double *__restrict__ m, double *__restrict__ out,
                                   int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = m[i] > 0.0 ? r[i] / m[i] : 0.0;
}

}  // namespace

void Context::initial_guess(const double *h_rho, const double *h_sigma, const double *h_bc,
                            const invdft_initial_guess_options &o, double *h_vxc_child, double *h_vxc_parent,
                            double *h_vh_quad) {
  if (!(o.tau_vx > 0.0) || !(o.tau_fa > 0.0)) throw StatusError(INVDFT_BAD_ARG, "tau_vx and tau_fa must be > 0");
  const int64_t nqt = nc * nq;
  for (int64_t q = 0; q < nqt; ++q)
    if (!std::isfinite(h_rho[q]) || h_rho[q] < 0.0) throw StatusError(INVDFT_NONFINITE, "bad density value");
  // the Hartree potential of rho (no nuclei) with the caller's boundary values
  DevBuf<double> vh_quad(nqt), rho_d, sig_d, vq(nqt);
  if (o.fermi_amaldi_bc || h_vh_quad) {
    DevBuf<double> phi;
    int it = 0;
    double res = 0.0;
    poisson_solve(h_rho, 0, nullptr, nullptr, nullptr, h_bc, o.hartree_rel_tol, o.hartree_max_iter, phi, it, res);
    if (res >= o.hartree_rel_tol) throw StatusError(INVDFT_MAXITER, "Hartree CG reached max_iter before its tolerance");
    INVDFT_CUDA(cudaMemcpyAsync(vh_quad.p, pp_q.p, sizeof(double) * nqt, cudaMemcpyDeviceToDevice, stream));
  } else {
    vh_quad.zero(stream);
  }
  rho_d.upload(h_rho, (size_t)nqt, stream);
  if (h_sigma) sig_d.upload(h_sigma, (size_t)nqt, stream);
  initial_guess_quad_kernel<<<ceil_div(nqt, 256), 256, 0, stream>>>(
      rho_d.p, h_sigma ? sig_d.p : nullptr, vh_quad.p, nqt, o.tau_vx, o.tau_fa, o.fermi_amaldi_bc ? 1 : 0,
      -o.factor_fa / n_electrons, vq.p);
  INVDFT_LAUNCH_CHECK();
  count_launch();
  // lumped-mass L2 projection onto the parent nodes, psi constraints distributed
  DevBuf<double> parent(nn);
  launch_mul(vq.p, jxw.p, vq.p, nqt, stream);
  launch_quad_rhs(fe, vq.p, Ycell.p, stream);
  AsmEpilogue epi;
  epi.kind = AsmEpilogue::STORE;
  launch_hx_assemble(fe, Ycell.p, parent.p, 1, epi, 0, stream);
  launch_scale_rows(invsqrtM.p, parent.p, parent.p, nn, 1, stream);
  launch_distribute(cpsi.rows.p, cpsi.ptr.p, cpsi.masters.p, cpsi.w.p, cpsi.n, parent.p, 1, stream);
  // at the child Gauss points, scaled by 1 - factorForLDAVxc
  DevBuf<double> cq((size_t)ncc * 8), ones((size_t)ncc * 8), r(ncn), m(ncn);
  parent_field_child_quad_kernel<<<ceil_div(ncc * 8, 256), 256, 0, stream>>>(fe, cv, parent.p, 1.0 - prm.factor_lda,
                                                                              cq.p);
  INVDFT_LAUNCH_CHECK();
  count_launch();
  // lumped-mass L2 projection onto the child nodes: r = C^T int N f, m = C^T int N
  std::vector<double> h1((size_t)ncc * 8, 1.0);
  ones.upload(h1, stream);
  launch_force_project(cv, cq.p, r.p, stream);
  launch_force_project(cv, ones.p, m.p, stream);
  divide_free_kernel<<<ceil_div(ncn, 256), 256, 0, stream>>>(r.p, m.p, r.p, ncn);
  INVDFT_LAUNCH_CHECK();
  count_launch();
  launch_set_zero(cchild.rows.p, cchild.n, r.p, 1, stream);
  r.download(h_vxc_child, (size_t)ncn, stream);
  if (h_vxc_parent) parent.download(h_vxc_parent, (size_t)nn, stream);
  if (h_vh_quad) vh_quad.download(h_vh_quad, (size_t)nqt, stream);
  INVDFT_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace invdft
