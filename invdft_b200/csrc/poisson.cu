// Base potential of the force evaluation on the GPU: the total electrostatic
// potential of the target density and the point nuclei.
//
// InverseDFTEngine::setPotBasePoissonNuclear (src/InverseDFTEngine.cpp:
// 2459-2571) forms the total target density at the parent quadrature points,
// solvePhiTotalAllElectronNonPeriodic (:2573-2621) solves DFT-FE's
// all-electron non-periodic Poisson problem for it with CG, and the nodal
// solution interpolated to the quadrature points becomes v_base (:2523-2541).
// Restated here for the order-p GLL elements of the wavefunctions:
//
//   sum_e int grad N_i . grad N_j phi_j = 4 pi int N_i rho - 4 pi sum_a Z_a N_i(R_a)
//
// condensed with the psi constraints (hanging nodes, zero boundary).  The
// Laplacian needs no stored matrix: it is the kinetic half of the Hamiltonian
// with a zero potential, so in the Lowdin-scaled unknown u = M^1/2 phi the
// system is  2 Ht0 u = M^-1/2 C^T b,  Ht0 the matrix-free Lowdin HX with
// v = 0, whose right-hand side is exactly what the cell-rhs kernel and the
// tiled assembly produce.  Jacobi-preconditioned CG (diag(2 Ht0) = kd/m, the
// inverse of the adjoint problem's D/2) runs on the device with the library's
// deterministic reductions; phi = C M^-1/2 u.
#include <cmath>

#include "context.h"

namespace invdft {

namespace {

// local Lagrange basis on the GLL nodes at reference coordinate t
void gll_basis(const std::vector<double> &nodes, double t, std::vector<double> &out) {
  const int n = (int)nodes.size();
  out.assign(n, 1.0);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      if (b != a) out[a] *= (t - nodes[b]) / (nodes[a] - nodes[b]);
}

}  // namespace

void Context::poisson_total(const double *h_rho, int n_atoms, const double *Z, const int64_t *atom_cell,
                            const double *atom_xi, double rel_tol, int max_iter, bool install,
                            double *h_phi_quad, double *h_phi_nodal, int *iters, double *rel_res) {
  DevBuf<double> phi;
  int it = 0;
  double res = 0.0;
  poisson_solve(h_rho, n_atoms, Z, atom_cell, atom_xi, nullptr, rel_tol, max_iter, phi, it, res);
  if (install) {
    INVDFT_CUDA(cudaMemcpyAsync(v_base.p, pp_q.p, sizeof(double) * nc * nq, cudaMemcpyDeviceToDevice, stream));
    invalidate_forward();   // the Hamiltonian of the next evaluation changes
    have_H = false;
  }
  if (h_phi_quad) pp_q.download(h_phi_quad, (size_t)nc * nq, stream);
  if (h_phi_nodal) phi.download(h_phi_nodal, (size_t)nn, stream);
  INVDFT_CUDA(cudaStreamSynchronize(stream));
  if (iters) *iters = it;
  if (rel_res) *rel_res = res;
  if (res >= rel_tol) throw StatusError(INVDFT_MAXITER, "Poisson CG reached max_iter before rel_tol");
}

// The Poisson solve shared by the base potential and the Hartree potential of
// the initial guess: nodal phi (constraints distributed) into `phi`, its values
// at the parent quadrature points into pp_q.  h_bc (may be null) holds
// boundary values on the Dirichlet rows of the psi constraints (zero
// otherwise); they enter through the lift g: phi = phi0 + g with phi0 zero on
// the boundary and A phi0 = b - K g.
void Context::poisson_solve(const double *h_rho, int n_atoms, const double *Z, const int64_t *atom_cell,
                            const double *atom_xi, const double *h_bc, double rel_tol, int max_iter,
                            DevBuf<double> &phi, int &it_out, double &res_out) {
  if (n_atoms < 0) throw StatusError(INVDFT_BAD_ARG, "negative atom count");
  if (!(rel_tol > 0.0) || max_iter < 1) throw StatusError(INVDFT_BAD_ARG, "rel_tol must be > 0, max_iter >= 1");
  const int64_t nqt = nc * nq;
  for (int64_t q = 0; q < nqt; ++q)
    if (!std::isfinite(h_rho[q])) throw StatusError(INVDFT_NONFINITE, "non-finite density");
  // point charges: -4 pi Z N_l(R_a) on the nodes of the nucleus' cell,
  // condensed through the constraints, in the Lowdin-scaled form M^-1/2 C^T
  std::vector<double> pc(nn, 0.0);
  {
    std::vector<double> nodes(n1);
    INVDFT_CUDA(cudaMemcpy(nodes.data(), gll.p, sizeof(double) * n1, cudaMemcpyDeviceToHost));
    std::vector<int64_t> crow(nn, -1);
    for (int64_t r = 0; r < cpsi.n; ++r) crow[cpsi.h_rows[r]] = r;
    std::vector<int> hcn((size_t)nc * nd);
    INVDFT_CUDA(cudaMemcpy(hcn.data(), cell_nodes.p, sizeof(int) * nc * nd, cudaMemcpyDeviceToHost));
    std::vector<double> lx, ly, lz;
    for (int a = 0; a < n_atoms; ++a) {
      if (atom_cell[a] < 0 || atom_cell[a] >= nc) throw StatusError(INVDFT_BAD_ARG, "atom cell out of range");
      for (int d = 0; d < 3; ++d)
        if (!(atom_xi[3 * a + d] >= -1e-12 && atom_xi[3 * a + d] <= 1.0 + 1e-12))
          throw StatusError(INVDFT_BAD_ARG, "atom reference coordinate outside [0, 1]");
      gll_basis(nodes, atom_xi[3 * a], lx);
      gll_basis(nodes, atom_xi[3 * a + 1], ly);
      gll_basis(nodes, atom_xi[3 * a + 2], lz);
      for (int l = 0; l < nd; ++l) {
        const double v = -4.0 * M_PI * Z[a] * lx[l % n1] * ly[(l / n1) % n1] * lz[l / (n1 * n1)];
        const int64_t node = hcn[(size_t)atom_cell[a] * nd + l];
        const int64_t r = crow[node];
        if (r < 0) {
          pc[node] += v;
        } else {
          for (int64_t k = cpsi.h_ptr[r]; k < cpsi.h_ptr[r + 1]; ++k) pc[cpsi.h_masters[k]] += cpsi.h_w[k] * v;
        }
      }
    }
    for (int64_t i = 0; i < nn; ++i) pc[i] *= h_invsqrtM[i];
  }
  // boundary lift g: the values on the Dirichlet rows, hanging rows
  // interpolated from their masters, zero elsewhere
  std::vector<double> g;
  if (h_bc) {
    g.assign(nn, 0.0);
    for (int64_t r = 0; r < cpsi.n; ++r)
      if (cpsi.h_ptr[r + 1] == cpsi.h_ptr[r]) {
        const double v = h_bc[cpsi.h_rows[r]];
        if (!std::isfinite(v)) throw StatusError(INVDFT_NONFINITE, "non-finite boundary value");
        g[cpsi.h_rows[r]] = v;
      }
    for (int64_t r = 0; r < cpsi.n; ++r)
      if (cpsi.h_ptr[r + 1] > cpsi.h_ptr[r]) {
        double v = 0.0;
        for (int64_t k = cpsi.h_ptr[r]; k < cpsi.h_ptr[r + 1]; ++k) v += cpsi.h_w[k] * g[cpsi.h_masters[k]];
        g[cpsi.h_rows[r]] = v;
      }
  }
  // right-hand side bt = M^-1/2 C^T (4 pi int N rho + point charges - K g)
  DevBuf<double> bt(nn), r(nn), z(nn), pd(nn), q(nn), tmp(nn);
  DevBuf<double> &x = phi;
  x.alloc(nn);
  pp_q.ensure((size_t)nqt);
  pp_q.upload(h_rho, (size_t)nqt, stream);
  launch_mul(pp_q.p, jxw.p, pp_q.p, nqt, stream);
  launch_quad_rhs(fe, pp_q.p, Ycell.p, stream);
  AsmEpilogue epi;
  epi.kind = AsmEpilogue::STORE;
  launch_hx_assemble(fe, Ycell.p, bt.p, 1, epi, 0, stream);
  tmp.upload(pc, stream);
  launch_axpbypcz(bt.p, 4.0 * M_PI, bt.p, 1.0, tmp.p, 0.0, nullptr, nn, stream);
  // the Laplacian: the matrix-free cell product with a zero potential
  if (vj_zero.n < 2 * (size_t)nqt) {   // both layouts of the (zero) potential term
    vj_zero.alloc(2 * (size_t)nqt);
    vj_zero.zero(stream);
  }
  auto apply = [&](const double *in, double *out) {   // out = 2 Ht0 in
    launch_hx_cell_sf(fe, sfm, vj_zero.p, in, Ycell.p, 1, GATHER_LOWDIN, 0, stream);
    launch_hx_assemble(fe, Ycell.p, out, 1, epi, 0, stream);
    launch_axpbypcz(out, 2.0, out, 0.0, nullptr, 0.0, nullptr, nn, stream);
  };
  DevBuf<double> gd;
  if (h_bc) {   // bt -= M^-1/2 C^T K g: the plain gather reads g as it is
    gd.upload(g, stream);
    launch_hx_cell_sf(fe, sfm, vj_zero.p, gd.p, Ycell.p, 1, GATHER_PLAIN, 0, stream);
    launch_hx_assemble(fe, Ycell.p, tmp.p, 1, epi, 0, stream);
    launch_axpbypcz(bt.p, 1.0, bt.p, -2.0, tmp.p, 0.0, nullptr, nn, stream);
  }
  auto dot = [&](const double *a, const double *b) {
    double v = 0.0;
    launch_coldot(a, b, nn, 1, partial.p, nblocks_red, small.p, stream);
    INVDFT_CUDA(cudaMemcpyAsync(&v, small.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
    INVDFT_CUDA(cudaStreamSynchronize(stream));
    return v;
  };
  // preconditioned CG from u = 0; P = diag(2 Ht0)^-1 = D / 2 (0 on constrained rows)
  x.zero(stream);
  INVDFT_CUDA(cudaMemcpyAsync(r.p, bt.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, stream));
  launch_scale_rows(diagA.p, r.p, z.p, nn, 1, stream);
  launch_axpbypcz(z.p, 0.5, z.p, 0.0, nullptr, 0.0, nullptr, nn, stream);
  INVDFT_CUDA(cudaMemcpyAsync(pd.p, z.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, stream));
  const double bnorm = std::sqrt(dot(bt.p, bt.p));
  double rz = dot(r.p, z.p), res = bnorm > 0.0 ? 1.0 : 0.0;
  int it = 0;
  while (bnorm > 0.0 && it < max_iter) {
    apply(pd.p, q.p);
    const double pq = dot(pd.p, q.p);
    if (!std::isfinite(pq) || pq <= 0.0) throw StatusError(INVDFT_BREAKDOWN, "Poisson CG: p^T A p not positive");
    const double alpha = rz / pq;
    launch_axpbypcz(x.p, 1.0, x.p, alpha, pd.p, 0.0, nullptr, nn, stream);
    launch_axpbypcz(r.p, 1.0, r.p, -alpha, q.p, 0.0, nullptr, nn, stream);
    ++it;
    res = std::sqrt(dot(r.p, r.p)) / bnorm;
    if (!std::isfinite(res)) throw StatusError(INVDFT_NONFINITE, "Poisson CG: non-finite residual");
    if (res < rel_tol) break;
    launch_scale_rows(diagA.p, r.p, z.p, nn, 1, stream);
    launch_axpbypcz(z.p, 0.5, z.p, 0.0, nullptr, 0.0, nullptr, nn, stream);
    const double rz_new = dot(r.p, z.p);
    launch_axpbypcz(pd.p, 1.0, z.p, rz_new / rz, pd.p, 0.0, nullptr, nn, stream);
    rz = rz_new;
  }
  // phi = C M^-1/2 u + g, then its values at the parent quadrature points
  launch_scale_rows(invsqrtM.p, x.p, x.p, nn, 1, stream);
  launch_distribute(cpsi.rows.p, cpsi.ptr.p, cpsi.masters.p, cpsi.w.p, cpsi.n, x.p, 1, stream);
  if (h_bc) launch_axpbypcz(x.p, 1.0, x.p, 1.0, gd.p, 0.0, nullptr, nn, stream);
  launch_interp_to_quad(fe, x.p, pp_q.p, 1, stream);
  INVDFT_CUDA(cudaStreamSynchronize(stream));
  it_out = it;
  res_out = res;
}

}  // namespace invdft
