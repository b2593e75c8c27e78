// extern "C" entry points of include/invdft_force.h.  Every call is wrapped so
// that no C++ exception or CUDA error crosses the ABI: failures become an
// invdft_status and a message retrievable with invdft_last_error().
#include <cmath>
#include <cstring>
#include <memory>
#include <string>

#include "context.h"

struct invdft_ctx {
  std::unique_ptr<invdft::Context> c;
  std::string err;
};

namespace {
thread_local std::string g_create_error;

template <class F> invdft_status guard(invdft_ctx *ctx, F &&f) {
  if (!ctx || !ctx->c) return INVDFT_BAD_ARG;
  try {
    f(*ctx->c);
    ctx->err.clear();
    return INVDFT_OK;
  } catch (const invdft::StatusError &e) {
    ctx->err = e.what();
    return (invdft_status)e.status;
  } catch (const invdft::CudaError &e) {
    ctx->err = e.what();
    return INVDFT_CUDA_ERROR;
  } catch (const std::bad_alloc &) {
    ctx->err = "host allocation failed";
    return INVDFT_OOM;
  } catch (const std::exception &e) {
    ctx->err = e.what();
    return INVDFT_BAD_ARG;
  }
}
}  // namespace

namespace invdft {
int64_t child_node_count(invdft_ctx *ctx) { return (ctx && ctx->c) ? ctx->c->ncn : -1; }
void set_thread_error(const std::string &msg) { g_create_error = msg; }
// Implemented in bfgs.cpp
invdft_status bfgs_solve(invdft_ctx *ctx, double *pot, int max_iter, double tol, int ls_iters, double ls_tol,
                         int history, double *losses, int *n_evals);
invdft_status bfgs_run(invdft_ctx *ctx, double *pot, const invdft_bfgs_options &o, double *losses,
                       double *density_l1, int cap, invdft_bfgs_report *rep);
}

extern "C" {

void invdft_default_params(invdft_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->cheb_degree = 50;
  p->max_cheb_passes = 100;
  p->cheby_tol = 1e-6;
  p->initial_tol_cheb = 1e-6;
  p->adaptive_factor_cheb = 100.0;
  p->adjoint_initial_tol = 1e-11;
  p->adaptive_factor_adjoint = 1000.0;
  p->adjoint_max_iter = 5000;
  p->degeneracy_tol = 0.002;
  p->frac_occ_tol = 1e-8;
  p->additional_states = 0;
  p->block_size = 0;
  p->inter_block_size = 10;
  p->factor_lda = 0.0;
  p->lanczos_steps = 20;
  p->precision = INVDFT_PRECISION_FP64;
  p->mixed_residual_floor = 1e-4;
  p->mixed_inner_tol = 1e-4;
  p->mixed_max_refine = 12;
}

invdft_status invdft_force_create(const invdft_problem_desc *desc, const invdft_params *params,
                                  invdft_ctx **ctx) {
  if (!ctx) return INVDFT_BAD_ARG;
  *ctx = nullptr;
  try {
    auto h = std::make_unique<invdft_ctx>();
    h->c = std::make_unique<invdft::Context>(desc, params);
    *ctx = h.release();
    g_create_error.clear();
    return INVDFT_OK;
  } catch (const invdft::StatusError &e) {
    g_create_error = e.what();
    return (invdft_status)e.status;
  } catch (const invdft::CudaError &e) {
    g_create_error = e.what();
    return INVDFT_CUDA_ERROR;
  } catch (const std::bad_alloc &) {
    g_create_error = "host allocation failed";
    return INVDFT_OOM;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    return INVDFT_BAD_ARG;
  }
}

void invdft_force_destroy(invdft_ctx *ctx) { delete ctx; }

const char *invdft_last_error(const invdft_ctx *ctx) {
  if (!ctx) return g_create_error.c_str();
  return ctx->err.c_str();
}

invdft_status invdft_set_params(invdft_ctx *ctx, const invdft_params *params) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!params) throw invdft::StatusError(INVDFT_BAD_ARG, "null params");
    c.set_params(params);
  });
}

invdft_status invdft_set_profiling(invdft_ctx *ctx, int32_t enable) {
  return guard(ctx, [&](invdft::Context &c) { c.profile = enable != 0; });
}

invdft_status invdft_set_subspace(invdft_ctx *ctx, const double *X) {
  return guard(ctx, [&](invdft::Context &c) { c.set_subspace(X); });
}

invdft_status invdft_force_eval(invdft_ctx *ctx, double *pot, double *force, double *loss,
                                invdft_force_stats *stats) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!pot || !force || !loss) throw invdft::StatusError(INVDFT_BAD_ARG, "null argument");
    c.eval(pot, force, loss, stats);
  });
}

invdft_status invdft_dot(invdft_ctx *ctx, const double *a, const double *b, int64_t n, double *out) {
  return invdft_dot_blocks(ctx, a, b, n, 1, out);
}

invdft_status invdft_dot_blocks(invdft_ctx *ctx, const double *a, const double *b, int64_t n, int32_t block_size,
                                double *out) {
  return guard(ctx, [&](invdft::Context &) {
    if (!a || !b || !out || n < 0 || block_size < 1)
      throw invdft::StatusError(INVDFT_BAD_ARG, "bad dot arguments (null array, n < 0 or block_size < 1)");
    // entry i accumulates into out[i % block_size], in entry order
    for (int32_t j = 0; j < block_size; ++j) out[j] = 0.0;
    for (int64_t i = 0; i < n; ++i) out[i % block_size] += a[i] * b[i];
  });
}

invdft_status invdft_get_eigen(invdft_ctx *ctx, double *eig, double *occ, double *fermi) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!c.have_eig) throw invdft::StatusError(INVDFT_NOT_READY, "no eigensolve yet");
    if (eig) std::memcpy(eig, c.eig.data(), sizeof(double) * c.N);
    if (occ && !c.occ.empty()) std::memcpy(occ, c.occ.data(), sizeof(double) * c.N);
    if (fermi) *fermi = c.mu;
  });
}

invdft_status invdft_get_psi(invdft_ctx *ctx, double *psi) {
  return guard(ctx, [&](invdft::Context &c) {
    c.psi.download(psi, (size_t)c.nn * c.N, c.stream);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_get_density(invdft_ctx *ctx, double *rho) {
  return guard(ctx, [&](invdft::Context &c) {
    c.rho.download(rho, (size_t)c.nc * c.nq, c.stream);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_get_child_quad_products(invdft_ctx *ctx, double *S) {
  return guard(ctx, [&](invdft::Context &c) {
    c.S.download(S, (size_t)c.ncc * 8, c.stream);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_solve_eigen(invdft_ctx *ctx, double *pot, invdft_force_stats *stats) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!pot) throw invdft::StatusError(INVDFT_BAD_ARG, "null potential");
    invdft_force_stats local{};
    invdft_force_stats *st = stats ? stats : &local;
    std::memset(st, 0, sizeof(*st));
    c.forward(pot, st);
  });
}

invdft_status invdft_force_backward(invdft_ctx *ctx, double *force, invdft_force_stats *stats) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!force) throw invdft::StatusError(INVDFT_BAD_ARG, "null force");
    invdft_force_stats local{};
    invdft_force_stats *st = stats ? stats : &local;
    c.backward(force, st);
  });
}

invdft_status invdft_force_backward_at(invdft_ctx *ctx, int64_t generation, double *force,
                                       invdft_force_stats *stats) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!force || generation < 0) throw invdft::StatusError(INVDFT_BAD_ARG, "null force or negative generation");
    invdft_force_stats local{};
    invdft_force_stats *st = stats ? stats : &local;
    c.backward(force, st, generation);
  });
}

invdft_status invdft_set_potential(invdft_ctx *ctx, const double *pot) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!pot) throw invdft::StatusError(INVDFT_BAD_ARG, "null potential");
    c.invalidate_forward();   // the backward half would run with this Hamiltonian
    c.pot_d.upload(pot, c.ncn, c.stream);
    c.set_potential_device(c.pot_d.p);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_project_vxc_to_parent(invdft_ctx *ctx, const double *vxc_child, double *parent_nodal) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!vxc_child || !parent_nodal) throw invdft::StatusError(INVDFT_BAD_ARG, "null array");
    c.project_vxc_to_parent(vxc_child, parent_nodal);
  });
}

invdft_status invdft_evaluate_parent_field(invdft_ctx *ctx, const double *parent_nodal, int64_t npts,
                                           const int64_t *cells, const double *xi, double *out) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!parent_nodal || npts < 0 || (npts > 0 && (!cells || !xi || !out)))
      throw invdft::StatusError(INVDFT_BAD_ARG, "null array or negative point count");
    c.evaluate_parent_field(parent_nodal, npts, cells, xi, out);
  });
}

invdft_status invdft_hx(invdft_ctx *ctx, const double *d_x, double *d_y, int32_t B) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!d_x || !d_y || B < 1 || B > 64) throw invdft::StatusError(INVDFT_BAD_ARG, "bad hx arguments (B in [1, 64])");
    c.hx(d_x, d_y, B);
    c.check_device_error();
  });
}

invdft_status invdft_adjoint_update_psi(invdft_ctx *ctx, const double *d_psi, const double *occ, const double *d_u,
                                        const int32_t *deg_ptr, const int32_t *deg_idx, double mu,
                                        const double *eig, int32_t B) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!d_psi || !occ || !d_u || !deg_ptr || !deg_idx || !eig || B < 1)
      throw invdft::StatusError(INVDFT_BAD_ARG, "bad update_psi arguments");
    std::vector<std::vector<int>> degen(B);
    for (int i = 0; i < B; ++i) degen[i].assign(deg_idx + deg_ptr[i], deg_idx + deg_ptr[i + 1]);
    c.adj_update_psi(d_psi, B, 0, occ, d_u, degen, mu, eig, B);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_adjoint_compute_rhs(invdft_ctx *ctx, double *d_rhs) {
  return guard(ctx, [&](invdft::Context &c) {
    c.adj_compute_rhs(d_rhs);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_adjoint_vmult(invdft_ctx *ctx, double *d_Ax, double *d_x) {
  return guard(ctx, [&](invdft::Context &c) {
    c.adj_vmult(d_Ax, d_x);
    c.check_device_error();
  });
}

invdft_status invdft_adjoint_precondition_jacobi(invdft_ctx *ctx, double *d_dst, const double *d_src, double) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!c.psi_ready) throw invdft::StatusError(INVDFT_NOT_READY, "updateInputPsi has not been called");
    c.adj_precondition(d_dst, d_src, false);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_adjoint_precondition_jacobi_sqrt(invdft_ctx *ctx, double *d_dst, const double *d_src,
                                                      double) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!c.psi_ready) throw invdft::StatusError(INVDFT_NOT_READY, "updateInputPsi has not been called");
    c.adj_precondition(d_dst, d_src, true);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_adjoint_distribute_x(invdft_ctx *ctx, double *d_x) {
  return guard(ctx, [&](invdft::Context &c) {
    c.adj_distribute_x(d_x);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_adjoint_solve(invdft_ctx *ctx, double *d_x, double tol, int32_t max_iter, int32_t *iters) {
  return guard(ctx, [&](invdft::Context &c) {
    std::vector<int> its;
    c.adj_minres(d_x, tol, max_iter, its);
    c.check_device_error();
    if (iters)
      for (size_t i = 0; i < its.size(); ++i) iters[i] = its[i];
  });
}

invdft_status invdft_poisson_total_potential(invdft_ctx *ctx, const double *rho_quad, int32_t n_atoms,
                                             const double *Z, const int64_t *atom_cell, const double *atom_xi,
                                             double rel_tol, int32_t max_iter, int32_t install,
                                             double *phi_quad, double *phi_nodal, int32_t *iters,
                                             double *rel_res) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!rho_quad || (n_atoms > 0 && (!Z || !atom_cell || !atom_xi)))
      throw invdft::StatusError(INVDFT_BAD_ARG, "null density or atom arrays");
    int it = 0;
    double res = 0.0;
    try {
      c.poisson_total(rho_quad, n_atoms, Z, atom_cell, atom_xi, rel_tol, max_iter, install != 0, phi_quad,
                      phi_nodal, &it, &res);
    } catch (...) {
      if (iters) *iters = it;
      if (rel_res) *rel_res = res;
      throw;
    }
    if (iters) *iters = it;
    if (rel_res) *rel_res = res;
  });
}

invdft_status invdft_initial_guess(invdft_ctx *ctx, const double *rho_quad, const double *sigma_quad,
                                   const double *hartree_bc, const invdft_initial_guess_options *opts,
                                   double *vxc_child, double *vxc_parent, double *vh_quad) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!rho_quad || !opts || !vxc_child) throw invdft::StatusError(INVDFT_BAD_ARG, "null density, options or output");
    if (opts->fermi_amaldi_bc && !hartree_bc)
      throw invdft::StatusError(INVDFT_BAD_ARG, "the Fermi-Amaldi far field needs the Hartree boundary values");
    c.initial_guess(rho_quad, sigma_quad, hartree_bc, *opts, vxc_child, vxc_parent, vh_quad);
  });
}

invdft_status invdft_kernel_probe(invdft_ctx *ctx) {
  return guard(ctx, [&](invdft::Context &c) { c.kernel_probe(); });
}

invdft_status invdft_get_index_map(invdft_ctx *ctx, int32_t which, int32_t *out, int64_t n) {
  return guard(ctx, [&](invdft::Context &c) {
    if (!out || n < 0) throw invdft::StatusError(INVDFT_BAD_ARG, "null output or negative length");
    const invdft::DevBuf<int> *src = nullptr;
    int64_t len = 0;
    auto cons = [&](const invdft::Cons &k, int part) {
      if (part == 0) { src = &k.rows; len = k.n; }
      else if (part == 1) { src = &k.ptr; len = k.n + 1; }
      else { src = &k.masters; len = k.n ? (int64_t)k.h_nnz : 0; }
    };
    switch (which) {
      case INVDFT_MAP_CELL_NODES: src = &c.cell_nodes; len = c.nc * c.nd; break;
      case INVDFT_MAP_CELL_GATHER: src = &c.cell_map; len = c.nc * c.nd; break;
      case INVDFT_MAP_CELL_SLOTS: src = &c.d_slot_of; len = c.nc * c.nd; break;
      case INVDFT_MAP_PSI_ROWS: cons(c.cpsi, 0); break;
      case INVDFT_MAP_PSI_PTR: cons(c.cpsi, 1); break;
      case INVDFT_MAP_PSI_MASTERS: cons(c.cpsi, 2); break;
      case INVDFT_MAP_ADJ_ROWS: cons(c.cadj, 0); break;
      case INVDFT_MAP_ADJ_PTR: cons(c.cadj, 1); break;
      case INVDFT_MAP_ADJ_MASTERS: cons(c.cadj, 2); break;
      case INVDFT_MAP_CHILD_ROWS: cons(c.cchild, 0); break;
      case INVDFT_MAP_CHILD_PTR: cons(c.cchild, 1); break;
      case INVDFT_MAP_CHILD_MASTERS: cons(c.cchild, 2); break;
      case INVDFT_MAP_CHILD_CELL_NODES: src = &c.ch_nodes; len = c.ncc * 8; break;
      case INVDFT_MAP_PQ_CHILD: src = &c.pq_child; len = c.nc * c.nq; break;
      default: throw invdft::StatusError(INVDFT_BAD_ARG, "unknown index map");
    }
    if (n != len)
      throw invdft::StatusError(INVDFT_BAD_ARG, "index map length is " + std::to_string(len) + ", not " +
                                                    std::to_string(n));
    if (len) src->download(out, (size_t)len, c.stream);
    INVDFT_CUDA(cudaStreamSynchronize(c.stream));
  });
}

invdft_status invdft_bfgs_solve(invdft_ctx *ctx, double *pot, int32_t max_iter, double tol,
                                int32_t line_search_iters, double line_search_tol, int32_t history,
                                double *losses, int32_t *n_evals) {
  if (!ctx || !ctx->c || !pot || max_iter < 0 || history < 1) return INVDFT_BAD_ARG;
  return invdft::bfgs_solve(ctx, pot, max_iter, tol, line_search_iters, line_search_tol, history, losses,
                            n_evals);
}

invdft_status invdft_bfgs_run(invdft_ctx *ctx, double *pot, const invdft_bfgs_options *opts, double *losses,
                              double *density_l1, int32_t capacity, invdft_bfgs_report *report) {
  if (!ctx || !ctx->c || !pot || !opts || opts->max_iter < 0 || opts->history < 1 || capacity < 0)
    return INVDFT_BAD_ARG;
  return invdft::bfgs_run(ctx, pot, *opts, losses, density_l1, capacity, report);
}

}  // extern "C"
