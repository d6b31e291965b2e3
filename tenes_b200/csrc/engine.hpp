// The per-context engine: device-resident iTPS state and the CTMRG driver.
#pragma once

#include <cusolverDn.h>

#include <array>
#include <string>
#include <vector>

#include "common.hpp"
#include "dtensor.hpp"
#include "lattice.hpp"

namespace tg {

struct Engine {
  virtual ~Engine() = default;
  virtual void set_site_tensor(int site, const double* host) = 0;
  virtual void get_site_tensor(int site, double* host) = 0;
  virtual void set_lambda(int site, int leg, const double* host) = 0;
  virtual void get_lambda(int site, int leg, double* host) = 0;
  virtual void set_env(int which, int site, const double* host) = 0;
  virtual void get_env(int which, int site, double* host) = 0;
  virtual void ctm_init() = 0;
  virtual void ctm_move(int dir, int line) = 0;
  virtual void ctm_sweep() = 0;
  virtual void check_convergence(int* converged, double* sig_max) = 0;
  virtual void ctm_run(int initialize, int* iterations, int* converged, double* sig_max) = 0;
  virtual void corner_spectrum(int which, int site, double* host) = 0;
  virtual void measure_onesite(int site, const double* op, double* out) = 0;
  virtual void measure_bond_op12(int source, int dx, int dy, const double* op, double* out) = 0;
  virtual void measure_bond_rdm(int source, int dx, int dy, double* out) = 0;
  virtual void measure_correlation(int left, int dir, int r_max, const double* left_op, int nright,
                                   const double* right_ops, double* out) = 0;
  virtual void measure_window(int source, int nrow, int ncol, int source_row, int source_col, int nops,
                              const int* op_row, const int* op_col, const double* ops, double* out) = 0;
  virtual void tm_eigenvalues(int dir, int fixed, int num_eigvals, int maxdim_dense, int maxdim, int restartdim,
                              int maxiter, double rtol, double* out, int* nev_out) = 0;
  virtual void su_onesite(int site, const double* op) = 0;
  virtual void su_bond(int source, int leg, const double* op) = 0;
  virtual void su_bonds(int n, const int* sources, const int* legs, const double* const* ops) = 0;
  virtual void fu_bond(int source, int leg, const double* op, const tg_fu_params* params, int* iterations,
                       int* converged) = 0;
  virtual void su_fix_gauge(int maxiter, double eps, int* sweeps, double* score) = 0;
  virtual void init_tensors(int seed, const double* dirs, const int* dir_len, const double* noises) = 0;
  virtual void energy_grad(int nterms, const tg_window_term* terms, int iterations, int checkpoint_every,
                           double svd_broadening, double* energy, double* grad) = 0;
  // counters of the exact truncated SVD of the full-SVD projectors:
  // solves, subspace iterations, Rayleigh-Ritz checks, dense fallbacks
  virtual void svd_stats(int64_t* out) = 0;
  virtual void sync() = 0;
  virtual void* stream() = 0;
};

Engine* make_engine(const tg_lattice_desc* lat, const tg_params* p, int is_complex, int device);

}  // namespace tg
