// L-BFGS driver of BFGSInverseDFTSolver::solve with the CP secant line search
// (src/BFGSInverseDFTSolver.cpp:68-118, 185-303, 467-627), one spin component.
// The vectors live on the host like the reference's distributedCPUVec; every
// force evaluation goes through invdft_force_eval.
#include <cmath>
#include <deque>
#include <vector>

#include "../../include/invdft_force.h"

namespace invdft {

int64_t child_node_count(invdft_ctx *ctx);

namespace {
double dot(const std::vector<double> &a, const std::vector<double> &b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
}  // namespace

invdft_status bfgs_run(invdft_ctx *ctx, double *pot, const invdft_bfgs_options &o, double *losses,
                       double *density_l1, int cap, invdft_bfgs_report *rep) {
  const int max_iter = o.max_iter, ls_iters = o.line_search_iters, history = o.history;
  const double tol = o.tol, ls_tol = o.line_search_tol;
  invdft_force_stats st;
  double L = 0.0;
  int iters_done = 0;
  bool reached = false;
  std::vector<double> x, g, p, s, y, xnew, gtmp;
  std::deque<std::vector<double>> Ys, Ss;
  std::deque<double> rhos;
  int k = 0, evals = 0;
  const int64_t n = child_node_count(ctx);
  if (n <= 0) return INVDFT_BAD_ARG;
  x.assign(pot, pot + n);
  g.assign(n, 0.0);
  // the evaluation distributes and then zeroes the constrained entries of its
  // potential in place, as getForceVector does with the BFGS iterate
  auto eval = [&](std::vector<double> &xin, std::vector<double> &gout, double &Lout) -> invdft_status {
    invdft_status rc = invdft_force_eval(ctx, xin.data(), gout.data(), &Lout, &st);
    if (losses && evals < cap) losses[evals] = Lout;
    // int |rho - rho*| = 2 sum |rho*_up - rho/2| JxW in the spin-unpolarised case
    if (density_l1 && evals < cap) density_l1[evals] = 2.0 * st.l1_error;
    ++evals;
    return rc;
  };
  // the density target, checked at the accepted iterates (not at line-search probes)
  auto at_target = [&]() { return o.density_l1_target > 0.0 && 2.0 * st.l1_error <= o.density_l1_target; };
  invdft_status rc = INVDFT_OK;
  for (int iter = 0; iter < max_iter; ++iter) {
    if (iter == 0) {
      rc = eval(x, g, L);
      if (rc != INVDFT_OK) break;
      if (at_target()) {
        reached = true;
        break;
      }
    }
    const double gnorm = std::sqrt(dot(g, g));
    // two-loop recursion (:68-118)
    std::vector<double> q(g);
    double gamma = 1.0;
    if (!Ys.empty()) gamma = dot(Ss.back(), Ys.back()) / dot(Ys.back(), Ys.back());
    std::vector<double> alpha(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
      alpha[i] = rhos[i] * dot(Ss[i], q);
      for (int64_t t = 0; t < n; ++t) q[t] -= alpha[i] * Ys[i][t];
    }
    p = q;
    for (auto &v : p) v *= gamma;
    for (int i = 0; i < k; ++i) {
      const double beta = rhos[i] * dot(Ys[i], p);
      for (int64_t t = 0; t < n; ++t) p[t] += (alpha[i] - beta) * Ss[i][t];
    }
    for (auto &v : p) v = -v;
    if (gnorm < tol) break;
    // CP line search (:217-303)
    std::vector<double> lam = {0.0, 1.0}, f = {dot(g, p)};
    for (int it = 0; it < ls_iters; ++it) {
      const double l0 = lam[lam.size() - 2], l1 = lam.back();
      const double f0 = f.back();
      if (std::sqrt(std::fabs(f0)) < ls_tol) {
        lam.pop_back();
        break;
      }
      xnew = x;
      for (int64_t t = 0; t < n; ++t) xnew[t] += l1 * p[t];
      gtmp.assign(n, 0.0);
      double Lp = 0.0;
      rc = eval(xnew, gtmp, Lp);
      if (rc != INVDFT_OK) break;
      const double f1 = dot(gtmp, p);
      f.push_back(f1);
      if (std::sqrt(std::fabs(f1)) < ls_tol) break;
      if (std::fabs((f1 - f0) / f1) < 1e-15) {
        rc = INVDFT_BREAKDOWN;
        break;
      }
      double sl = (f1 - f0) / (l1 - l0);
      if (sl > 0.0) sl = -sl;
      double nxt = l1 - f1 / sl;
      if (nxt < 0.0) nxt = l1 + f1 / sl;
      lam.push_back(nxt);
    }
    if (rc != INVDFT_OK) break;
    const double lamopt = lam.back() > 0.0 ? lam.back() : 1.0;
    s = p;
    for (auto &v : s) v *= lamopt;
    for (int64_t t = 0; t < n; ++t) x[t] += s[t];
    y = g;
    for (auto &v : y) v = -v;
    rc = eval(x, g, L);
    if (rc != INVDFT_OK) break;
    iters_done = iter + 1;
    const double l1_now = 2.0 * st.l1_error;
    for (int64_t t = 0; t < n; ++t) y[t] += g[t];
    const double curv = dot(y, s);
    if (curv > 0.0) {
      Ys.push_back(y);
      Ss.push_back(s);
      rhos.push_back(1.0 / curv);
      ++k;
    }
    if (k > history) {
      k = history;
      Ys.pop_front();
      Ss.pop_front();
      rhos.pop_front();
    }
    if (o.density_l1_target > 0.0 && l1_now <= o.density_l1_target) {
      reached = true;
      break;
    }
  }
  for (int64_t t = 0; t < n; ++t) pot[t] = x[t];
  if (rep) {
    rep->n_iters = iters_done;
    rep->n_evals = evals;
    rep->final_loss = L;
    rep->final_density_l1 = 2.0 * st.l1_error;
    rep->reached = reached ? 1 : 0;
  }
  return rc;
}

invdft_status bfgs_solve(invdft_ctx *ctx, double *pot, int max_iter, double tol, int ls_iters, double ls_tol,
                         int history, double *losses, int *n_evals) {
  invdft_bfgs_options o{};
  o.max_iter = max_iter;
  o.tol = tol;
  o.line_search_iters = ls_iters;
  o.line_search_tol = ls_tol;
  o.history = history;
  o.density_l1_target = 0.0;
  invdft_bfgs_report rep{};
  const invdft_status rc = bfgs_run(ctx, pot, o, losses, nullptr, 2 * max_iter + 1, &rep);
  if (n_evals) *n_evals = rep.n_evals;
  return rc;
}

}  // namespace invdft
