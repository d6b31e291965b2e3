// C ABI of libtenes_gpu (declared in include/tenes_gpu.h).  Every entry point
// converts C++ exceptions into tg_status codes; nothing is thrown across it.
#include <cmath>
#include <cstring>
#include <exception>
#include <string>

#include "engine.hpp"
#include "kernels.cuh"
#include "tenes_gpu.h"

struct tg_ctx {
  tg::Engine* eng = nullptr;
};

namespace {

thread_local std::string g_last_error;

template <typename F>
tg_status guard(F&& f) {
  try {
    f();
    return TG_OK;
  } catch (const tg::Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return TG_E_RUNTIME;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return TG_E_RUNTIME;
  } catch (...) {
    g_last_error = "unknown error";
    return TG_E_RUNTIME;
  }
}

tg::Engine* E(tg_ctx* c) {
  if (!c || !c->eng) tg::fail(TG_E_STATE, "null context");
  return c->eng;
}

void need(const void* p, const char* what) {
  if (!p) tg::fail(TG_E_INPUT, std::string("null pointer: ") + what);
}

}  // namespace

namespace tg {
void set_last_error(const std::string& m) { g_last_error = m; }
}  // namespace tg

extern "C" {

void tg_params_default(tg_params* p) {
  if (!p) return;
  p->chi = 2;
  p->inverse_projector_cut = 1e-12;
  p->ctm_convergence_epsilon = 1e-6;
  p->max_ctm_iteration = 100;
  p->projector_corner = 1;
  p->use_rsvd = 0;
  p->rsvd_oversampling_factor = 2.0;
  p->rsvd_oversample_abs = -1;
  p->rsvd_power_iters = 2;
  p->rsvd_seed = 0;
  p->inverse_lambda_cut = 1e-12;
  p->mixed = 0;
  p->cuda_graph = 1;
  p->svd_solver = 0;
  p->density = 0;
}

const char* tg_last_error(void) { return g_last_error.c_str(); }

const char* tg_version(void) { return "tenes_gpu 0.1.0 (sm_100a)"; }

tg_status tg_ctx_create(const tg_lattice_desc* lattice, const tg_params* params, int is_complex, int device,
                        tg_ctx** out) {
  return guard([&] {
    need(out, "out");
    *out = nullptr;
    auto* c = new tg_ctx;
    try {
      c->eng = tg::make_engine(lattice, params, is_complex, device);
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

tg_status tg_ctx_destroy(tg_ctx* ctx) {
  return guard([&] {
    if (!ctx) return;
    delete ctx->eng;
    delete ctx;
  });
}

tg_status tg_set_site_tensor(tg_ctx* ctx, int site, const double* host) {
  return guard([&] {
    need(host, "host");
    E(ctx)->set_site_tensor(site, host);
  });
}
tg_status tg_get_site_tensor(tg_ctx* ctx, int site, double* host) {
  return guard([&] {
    need(host, "host");
    E(ctx)->get_site_tensor(site, host);
  });
}
tg_status tg_set_lambda(tg_ctx* ctx, int site, int leg, const double* host) {
  return guard([&] {
    need(host, "host");
    E(ctx)->set_lambda(site, leg, host);
  });
}
tg_status tg_get_lambda(tg_ctx* ctx, int site, int leg, double* host) {
  return guard([&] {
    need(host, "host");
    E(ctx)->get_lambda(site, leg, host);
  });
}
tg_status tg_set_env(tg_ctx* ctx, int which, int site, const double* host) {
  return guard([&] {
    need(host, "host");
    E(ctx)->set_env(which, site, host);
  });
}
tg_status tg_get_env(tg_ctx* ctx, int which, int site, double* host) {
  return guard([&] {
    need(host, "host");
    E(ctx)->get_env(which, site, host);
  });
}
tg_status tg_ctm_init(tg_ctx* ctx) {
  return guard([&] { E(ctx)->ctm_init(); });
}
tg_status tg_ctm_move(tg_ctx* ctx, int dir, int line) {
  return guard([&] {
    E(ctx)->ctm_move(dir, line);
    E(ctx)->sync();
  });
}
tg_status tg_ctm_sweep(tg_ctx* ctx) {
  return guard([&] { E(ctx)->ctm_sweep(); });
}
tg_status tg_ctm_check_convergence(tg_ctx* ctx, int* converged, double* sig_max) {
  return guard([&] { E(ctx)->check_convergence(converged, sig_max); });
}
tg_status tg_projector_svd_stats(tg_ctx* ctx, int64_t* out) {
  return guard([&] {
    need(out, "out");
    E(ctx)->svd_stats(out);
  });
}
tg_status tg_ctm_run(tg_ctx* ctx, int initialize, int* iterations, int* converged, double* sig_max) {
  return guard([&] { E(ctx)->ctm_run(initialize, iterations, converged, sig_max); });
}
tg_status tg_corner_spectrum(tg_ctx* ctx, int which, int site, double* host) {
  return guard([&] {
    need(host, "host");
    E(ctx)->corner_spectrum(which, site, host);
  });
}
tg_status tg_measure_onesite(tg_ctx* ctx, int site, const double* op, double* out) {
  return guard([&] {
    need(op, "op");
    need(out, "out");
    E(ctx)->measure_onesite(site, op, out);
  });
}
tg_status tg_measure_bond_op12(tg_ctx* ctx, int source, int dx, int dy, const double* op, double* out) {
  return guard([&] {
    need(op, "op");
    need(out, "out");
    E(ctx)->measure_bond_op12(source, dx, dy, op, out);
  });
}
tg_status tg_measure_bond_rdm(tg_ctx* ctx, int source, int dx, int dy, double* out) {
  return guard([&] {
    need(out, "out");
    E(ctx)->measure_bond_rdm(source, dx, dy, out);
  });
}
tg_status tg_measure_correlation(tg_ctx* ctx, int left, int dir, int r_max, const double* left_op, int nright,
                                 const double* right_ops, double* out) {
  return guard([&] {
    need(left_op, "left_op");
    need(right_ops, "right_ops");
    need(out, "out");
    E(ctx)->measure_correlation(left, dir, r_max, left_op, nright, right_ops, out);
  });
}
tg_status tg_measure_window(tg_ctx* ctx, int source, int nrow, int ncol, int source_row, int source_col, int nops,
                            const int* op_row, const int* op_col, const double* ops, double* out) {
  return guard([&] {
    need(out, "out");
    if (nops > 0) {
      need(op_row, "op_row");
      need(op_col, "op_col");
      need(ops, "ops");
    }
    E(ctx)->measure_window(source, nrow, ncol, source_row, source_col, nops, op_row, op_col, ops, out);
  });
}
tg_status tg_tm_eigenvalues(tg_ctx* ctx, int dir, int fixed, int num_eigvals, int maxdim_dense, int arnoldi_maxdim,
                            int arnoldi_restartdim, int arnoldi_maxiter, double arnoldi_rtol, double* out,
                            int* nev) {
  return guard([&] {
    need(out, "out");
    if (num_eigvals < 1 || arnoldi_maxdim < 2 || arnoldi_maxiter < 1) tg::fail(TG_E_INPUT, "bad transfer-matrix parameters");
    E(ctx)->tm_eigenvalues(dir, fixed, num_eigvals, maxdim_dense, arnoldi_maxdim, arnoldi_restartdim,
                           arnoldi_maxiter, arnoldi_rtol, out, nev);
  });
}
tg_status tg_su_onesite(tg_ctx* ctx, int site, const double* op) {
  return guard([&] {
    need(op, "op");
    E(ctx)->su_onesite(site, op);
  });
}
tg_status tg_su_bond(tg_ctx* ctx, int source, int source_leg, const double* op) {
  return guard([&] {
    need(op, "op");
    E(ctx)->su_bond(source, source_leg, op);
  });
}
tg_status tg_su_bonds(tg_ctx* ctx, int n, const int* sources, const int* source_legs, const double* const* ops) {
  return guard([&] {
    if (n > 0) {
      need(sources, "sources");
      need(source_legs, "source_legs");
      need(ops, "ops");
    }
    E(ctx)->su_bonds(n, sources, source_legs, ops);
  });
}
tg_status tg_init_tensors(tg_ctx* ctx, int seed, const double* initial_dirs, const int* dir_len,
                          const double* noises) {
  return guard([&] {
    need(initial_dirs, "initial_dirs");
    need(dir_len, "dir_len");
    need(noises, "noises");
    E(ctx)->init_tensors(seed, initial_dirs, dir_len, noises);
  });
}
tg_status tg_energy_grad(tg_ctx* ctx, int nterms, const tg_window_term* terms, int iterations, int checkpoint_every,
                         double svd_broadening, double* energy, double* grad) {
  return guard([&] {
    need(terms, "terms");
    need(energy, "energy");
    E(ctx)->energy_grad(nterms, terms, iterations, checkpoint_every, svd_broadening, energy, grad);
  });
}
void tg_fu_params_default(tg_fu_params* p) {
  if (!p) return;
  p->inverse_env_cut = 1e-12;
  p->inverse_precision = 1e-12;
  p->convergence_epsilon = 1e-6;
  p->max_iteration = 100;
  p->gauge_fix = 1;
}
tg_status tg_fu_bond(tg_ctx* ctx, int source, int source_leg, const double* op, const tg_fu_params* params,
                     int* iterations, int* converged) {
  return guard([&] {
    need(op, "op");
    need(params, "params");
    E(ctx)->fu_bond(source, source_leg, op, params, iterations, converged);
  });
}
tg_status tg_su_fix_gauge(tg_ctx* ctx, int maxiter, double eps, int* sweeps, double* score) {
  return guard([&] { E(ctx)->su_fix_gauge(maxiter, eps, sweeps, score); });
}
tg_status tg_sync(tg_ctx* ctx) {
  return guard([&] { E(ctx)->sync(); });
}
uint64_t tg_kernel_launch_count(void) { return tg::launch_count(); }

tg_status tg_ctx_stream(tg_ctx* ctx, void** stream) {
  return guard([&] {
    need(stream, "stream");
    *stream = E(ctx)->stream();
  });
}
tg_status tg_profile_enable(int on) {
  return guard([&] { tg::profile_enable(on != 0); });
}
tg_status tg_profile_reset(void) {
  return guard([&] { tg::profile_reset(); });
}
tg_status tg_profile_query(int kind, uint64_t* launches, double* ms, double* flops, double* bytes) {
  return guard([&] { tg::profile_query(kind, launches, ms, flops, bytes); });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Microbenchmark of the contraction kernel on one product shape (device
// buffers allocated and freed here; not used by the CTMRG path).
extern "C" tg_status tg_gemm_host(int64_t M, int64_t N, int64_t K, const double* A, int64_t sAm, int64_t sAk,
                                  const double* B, int64_t sBk, int64_t sBn, double* C, int64_t sCm, int64_t sCn,
                                  int prec) {
  return guard([&] {
    if (M < 1 || N < 1 || K < 1 || !A || !B || !C) tg::fail(TG_E_INPUT, "bad gemm arguments");
    if ((sAm != 1 && sAk != 1) || (sBk != 1 && sBn != 1) || sAm < 1 || sAk < 1 || sBk < 1 || sBn < 1 || sCm < 1 ||
        sCn < 1)
      tg::fail(TG_E_INPUT, "gemm: one unit stride per operand required");
    if (prec != 0 && prec != 1) tg::fail(TG_E_INPUT, "prec must be 0 or 1");
    const int64_t na = (M - 1) * sAm + (K - 1) * sAk + 1, nb = (K - 1) * sBk + (N - 1) * sBn + 1,
                  nc = (M - 1) * sCm + (N - 1) * sCn + 1;
    cudaStream_t st;
    TG_CUDA(cudaStreamCreate(&st));
    double *dA = nullptr, *dB = nullptr, *dC = nullptr;
    TG_CUDA(cudaMalloc(&dA, sizeof(double) * na));
    TG_CUDA(cudaMalloc(&dB, sizeof(double) * nb));
    TG_CUDA(cudaMalloc(&dC, sizeof(double) * nc));
    TG_CUDA(cudaMemcpyAsync(dA, A, sizeof(double) * na, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(dB, B, sizeof(double) * nb, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(dC, C, sizeof(double) * nc, cudaMemcpyHostToDevice, st));
    tg::GemmDesc g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.batch = 1;
    g.sAm = sAm;
    g.sAk = sAk;
    g.sBk = sBk;
    g.sBn = sBn;
    g.sCm = sCm;
    g.sCn = sCn;
    g.prec = prec;
    tg::gemm<double>(dA, dB, dC, g, st);
    TG_CUDA(cudaMemcpyAsync(C, dC, sizeof(double) * nc, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    const bool fault = prec == 1 && tg::tc_fault_take();
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaStreamDestroy(st);
    if (fault) tg::fail(TG_E_RUNTIME, "tensor-core product stopped waiting for its MMAs");
  });
}

extern "C" tg_status tg_gemm_group_host(int n, const int64_t* mnk, const int* flags, int is_complex,
                                        const double* A, const double* B, double* C) {
  return guard([&] {
    if (n < 1 || !mnk || !A || !B || !C) tg::fail(TG_E_INPUT, "bad grouped gemm arguments");
    const int64_t w = is_complex ? 2 : 1;  // doubles per element
    std::vector<tg::GroupItem> items(static_cast<size_t>(n));
    std::vector<int64_t> oa(static_cast<size_t>(n)), ob(oa), oc(oa);  // element offsets
    int64_t na = 0, nb = 0, nc = 0;
    for (int i = 0; i < n; ++i) {
      const int64_t M = mnk[3 * i], N = mnk[3 * i + 1], K = mnk[3 * i + 2];
      if (M < 1 || N < 1 || K < 1) tg::fail(TG_E_INPUT, "grouped gemm: every M, N, K must be positive");
      const int f = flags ? flags[i] : 0;
      if ((f & ~15) || (!is_complex && (f & 12))) tg::fail(TG_E_INPUT, "grouped gemm: bad flags");
      tg::GroupItem& it = items[static_cast<size_t>(i)];
      it.M = M;
      it.N = N;
      it.K = K;
      it.sAm = (f & 1) ? 1 : K;
      it.sAk = (f & 1) ? M : 1;
      it.sBk = (f & 2) ? 1 : N;
      it.sBn = (f & 2) ? K : 1;
      it.sCm = N;
      it.sCn = 1;
      it.conjA = (f & 4) != 0;
      it.conjB = (f & 8) != 0;
      oa[static_cast<size_t>(i)] = na;
      ob[static_cast<size_t>(i)] = nb;
      oc[static_cast<size_t>(i)] = nc;
      na += M * K;
      nb += K * N;
      nc += M * N;
    }
    cudaStream_t st;
    TG_CUDA(cudaStreamCreate(&st));
    double *dA = nullptr, *dB = nullptr, *dC = nullptr;
    TG_CUDA(cudaMalloc(&dA, sizeof(double) * w * na));
    TG_CUDA(cudaMalloc(&dB, sizeof(double) * w * nb));
    TG_CUDA(cudaMalloc(&dC, sizeof(double) * w * nc));
    TG_CUDA(cudaMemcpyAsync(dA, A, sizeof(double) * w * na, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(dB, B, sizeof(double) * w * nb, cudaMemcpyHostToDevice, st));
    for (size_t i = 0; i < items.size(); ++i) {
      items[i].A = dA + w * oa[i];
      items[i].B = dB + w * ob[i];
      items[i].C = dC + w * oc[i];
    }
    if (is_complex) tg::gemm_group<tg::cplx>(items.data(), n, st);
    else tg::gemm_group<double>(items.data(), n, st);
    TG_CUDA(cudaMemcpyAsync(C, dC, sizeof(double) * w * nc, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaStreamDestroy(st);
  });
}

extern "C" tg_status tg_gemm_group_stats(int64_t* tuned, int64_t* wins, int nwins) {
  return guard([&] { tg::gemm_group_stats(tuned, wins, nwins); });
}

extern "C" tg_status tg_cholqr_host(int64_t n, int64_t k, double* Y, int passes, int* pivot_flag) {
  return guard([&] {
    if (n < 1 || k < 1 || k > n || passes < 1 || !Y) tg::fail(TG_E_INPUT, "bad CholeskyQR arguments");
    if (!tg::cholqr_cluster_supported(n, k)) tg::fail(TG_E_INPUT, "CholeskyQR panel shape not supported");
    cudaStream_t st;
    TG_CUDA(cudaStreamCreate(&st));
    double *dY = nullptr, *dscr = nullptr;
    int* dflag = nullptr;
    TG_CUDA(cudaMalloc(&dY, sizeof(double) * n * k));
    TG_CUDA(cudaMalloc(&dscr, sizeof(double) * tg::cholqr_scratch_doubles(k)));
    TG_CUDA(cudaMalloc(&dflag, sizeof(int)));
    TG_CUDA(cudaMemsetAsync(dflag, 0, sizeof(int), st));
    TG_CUDA(cudaMemcpyAsync(dY, Y, sizeof(double) * n * k, cudaMemcpyHostToDevice, st));
    tg::cholqr_cluster(dY, n, k, passes, 2, 1, 1e-14 / std::sqrt(static_cast<double>(n)), dscr, dflag, st);
    int flag = 0;
    TG_CUDA(cudaMemcpyAsync(Y, dY, sizeof(double) * n * k, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaMemcpyAsync(&flag, dflag, sizeof(int), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    cudaFree(dY);
    cudaFree(dscr);
    cudaFree(dflag);
    cudaStreamDestroy(st);
    if (pivot_flag) *pivot_flag = flag;
  });
}

extern "C" tg_status tg_bench_gemm(int64_t M, int64_t N, int64_t K, int layout, int prec, int iters,
                                   double* avg_ms) {
  return guard([&] {
    if (M < 1 || N < 1 || K < 1 || iters < 1 || !avg_ms) tg::fail(TG_E_INPUT, "bad gemm benchmark arguments");
    cudaStream_t st;
    TG_CUDA(cudaStreamCreate(&st));
    double *A = nullptr, *B = nullptr, *C = nullptr;
    TG_CUDA(cudaMalloc(&A, sizeof(double) * M * K));
    TG_CUDA(cudaMalloc(&B, sizeof(double) * K * N));
    TG_CUDA(cudaMalloc(&C, sizeof(double) * M * N));
    TG_CUDA(cudaMemset(A, 0, sizeof(double) * M * K));
    TG_CUDA(cudaMemset(B, 0, sizeof(double) * K * N));
    tg::GemmDesc g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.batch = 1;
    // layout 0: A row-major (M,K), B row-major (K,N); 1: B column-major (panel products)
    g.sAm = K;
    g.sAk = 1;
    if (layout == 1) {
      g.sBk = 1;
      g.sBn = K;
    } else {
      g.sBk = N;
      g.sBn = 1;
    }
    g.sCm = N;
    g.sCn = 1;
    g.prec = prec;
    tg::gemm<double>(A, B, C, g, st);
    cudaEvent_t e0, e1;
    TG_CUDA(cudaEventCreate(&e0));
    TG_CUDA(cudaEventCreate(&e1));
    TG_CUDA(cudaEventRecord(e0, st));
    for (int i = 0; i < iters; ++i) tg::gemm<double>(A, B, C, g, st);
    TG_CUDA(cudaEventRecord(e1, st));
    TG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    TG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *avg_ms = ms / iters;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(A);
    cudaFree(B);
    cudaFree(C);
    cudaStreamDestroy(st);
  });
}
