// CTMRG environment engine of libtenes_gpu.
//
// The driver mirrors src/iTPS/core/ctm.cpp contraction by contraction
// (same tensordot sequences, same leg orders), so every intermediate can be
// compared one to one with the reference algorithm.  All tensors stay on the
// device; contractions run on the hand-written DMMA kernels of kernels.cu,
// the dense projector SVD and the simple-update QR / SVD on cuSOLVER.
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <numeric>
#include <cstring>
#include <map>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "adjoint_device.hpp"
#include "full_update.hpp"
#include "local_gauge.hpp"
#include "dtensor.hpp"
#include "engine.hpp"
#include "kernels.cuh"

namespace tg {

namespace {

void check_sol(cusolverStatus_t s, const char* what) {
  if (s != CUSOLVER_STATUS_SUCCESS) fail(TG_E_CUDA, std::string(what) + ": cuSOLVER status " + std::to_string(static_cast<int>(s)));
}

using V = std::vector<int>;

}  // namespace

template <typename T>
struct EngineT final : Engine {
  static constexpr bool CPLX = is_cplx<T>::value;
  static constexpr int NW = CPLX ? 2 : 1;  // doubles per element

  Lattice lat;
  tg_params P;
  int dev = 0;
  cudaStream_t st = nullptr;
  cusolverDnHandle_t sol = nullptr;  // slot 0 (the main stream); see hsol()

  std::vector<DT<T>> Tn;
  std::vector<std::array<DT<T>, 3>> Trot;  // right (2,3,0,1,4), top (1,2,3,0,4), bottom (3,0,1,2,4)
  std::vector<bool> rot_ok;
  // iTPO (tg_params.density): Tn[i] holds the density tensor
  // (D,D,D,D,d,d) as (D,D,D,D,d*d); the CTMRG runs on the single-layer
  // network of Ts[i] = sum_p Tn[i][...,p,p] (Make_single_tensor_density,
  // ctm_single.cpp:43-50), stored (D,D,D,D,1).  Every double-layer
  // contraction of the engine then serves as the single-layer one with the
  // all-ones (1,1,1,1,1) tensor `bra1` in place of conj(Tn): the edges are
  // (chi,chi,D,1) and every "bra" leg has dimension 1.
  bool density = false;
  std::vector<DT<T>> Ts;
  DT<T> bra1, one1;  // (1,1,1,1,1) ones; the 1 x 1 operator [[1]]
  std::array<std::vector<DT<T>>, 4> C;  // C1..C4
  std::array<std::vector<DT<T>>, 4> E;  // eTt, eTr, eTb, eTl
  std::vector<std::array<std::vector<double>, 4>> lambda;
  bool env_ready = false;
  DT<double> spec_old;
  bool spec_old_ok = false;

  // The rows of a move are independent (ctm.cpp:577-593, 603-615): with rSVD
  // projectors each row runs on its own stream, forked from and joined back
  // into `st` with events (inside a captured sweep these become parallel
  // branches of the graph).  `st` and `slot` name the stream in use; every
  // stream slot has its own device scratch.
  static constexpr int kRowStreams = 4;
  cudaStream_t main_st = nullptr;
  cudaStream_t row_st[kRowStreams] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kRowStreams] = {}, ev_mid[kRowStreams] = {};
  // Row staggering: row r's rSVD waits for row r-1's first range-finder
  // product, so that the rows' latency-bound orthonormalisations fall on
  // each other's tensor-core products instead of coinciding.
  cudaEvent_t ev_stagger[kRowStreams] = {};
  bool stagger_rec[kRowStreams] = {};
  int cur_row = -1;
  int slot = 0;  // 0: main stream, 1..kRowStreams: row streams

  // cuSOLVER handles, one per stream slot (created on first use), so that
  // rows factorising on their own streams share no handle state
  cusolverDnHandle_t sol_slot[kRowStreams + 1] = {};
  cusolverDnHandle_t hsol() {
    cusolverDnHandle_t& h = sol_slot[slot];
    if (!h) check_sol(cusolverDnCreate(&h), "cusolverDnCreate");
    check_sol(cusolverDnSetStream(h, st), "cusolverDnSetStream");
    return h;
  }

  unsigned long long* d_max = nullptr;  // one per stream slot
  static constexpr int kInfoSlots = 4096;
  int* d_info = nullptr;  // one slot per cuSOLVER call, checked at sync points
  int info_used = 0;
  int* d_flag = nullptr;  // one per stream slot: set by device kernels on a numerical failure
  uint64_t noise_stream = 0;  // key sequence of the orthonormalisation perturbations
  int* d_cut = nullptr;
  // Simple-update weights on the device, [(site * 4 + leg) * lam_ld + j]: the
  // fused bond kernel reads and writes them there; `lambda` (host) is the
  // copy the other paths use.  Either side may be the newer one.
  double* d_lam = nullptr;
  int lam_ld = 1;
  bool lam_dev_stale = true, lam_host_stale = false;
  int* d_su_flag = nullptr;
  std::map<std::vector<double>, DT<T>> op_cache;  // evolution operators already on the device
  const T** d_ptrs = nullptr;
  const T** h_ptrs = nullptr;  // pinned
  double* h_sig = nullptr;     // pinned

  EngineT(const tg_lattice_desc* ld, const tg_params* p, int device) : P(*p), dev(device) {
    if (!ld || !ld->physical_dims || !ld->virtual_dims) fail(TG_E_INPUT, "lattice description is incomplete");
    lat = Lattice(ld->LX, ld->LY, ld->skew);
    lat.pdim.resize(lat.N);
    lat.vdim.resize(lat.N);
    for (int i = 0; i < lat.N; ++i) {
      lat.pdim[i] = ld->physical_dims[i];
      for (int l = 0; l < 4; ++l) lat.vdim[i][l] = ld->virtual_dims[4 * i + l];
    }
    lat.check_dims();
    if (P.chi < 1) fail(TG_E_INPUT, "chi must be positive");
    if (P.density) {
      // the single-layer environment starts at the bond dimensions
      // (ctm_single.cpp:752-960) and is kept padded to chi
      for (int i = 0; i < lat.N; ++i)
        for (int l = 0; l < 4; ++l)
          if (lat.vdim[i][l] > P.chi)
            fail(TG_E_INPUT, "an iTPO environment needs chi >= every bond dimension");
    }
    if (P.rsvd_oversampling_factor < 1.0) fail(TG_E_INPUT, "rsvd_oversampling_factor must be >= 1.0");
    if (P.mixed && CPLX) fail(TG_E_INPUT, "mixed precision is available for real tensors only");
    density = P.density != 0;
    abs_prec = P.mixed ? 1 : 0;
    TG_CUDA(cudaSetDevice(dev));
    TG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaMemPool_t pool;
    TG_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = UINT64_MAX;
    TG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    check_sol(cusolverDnCreate(&sol), "cusolverDnCreate");
    check_sol(cusolverDnSetStream(sol, st), "cusolverDnSetStream");
    sol_slot[0] = sol;
    main_st = st;
    for (int r = 0; r < kRowStreams; ++r) {
      TG_CUDA(cudaStreamCreateWithFlags(&row_st[r], cudaStreamNonBlocking));
      TG_CUDA(cudaEventCreateWithFlags(&ev_join[r], cudaEventDisableTiming));
      TG_CUDA(cudaEventCreateWithFlags(&ev_mid[r], cudaEventDisableTiming));
      TG_CUDA(cudaEventCreateWithFlags(&ev_stagger[r], cudaEventDisableTiming));
    }
    TG_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    TG_CUDA(cudaMalloc(&d_max, sizeof(unsigned long long) * (kRowStreams + 1)));
    TG_CUDA(cudaMalloc(&d_info, sizeof(int) * kInfoSlots));
    TG_CUDA(cudaMemset(d_info, 0, sizeof(int) * kInfoSlots));
    TG_CUDA(cudaMalloc(&d_flag, sizeof(int) * (kRowStreams + 1)));
    TG_CUDA(cudaMemset(d_flag, 0, sizeof(int) * (kRowStreams + 1)));
    TG_CUDA(cudaMalloc(&d_cut, sizeof(int) * (kRowStreams + 1)));
    for (int i = 0; i < lat.N; ++i)
      for (int l = 0; l < 4; ++l) lam_ld = std::max(lam_ld, lat.vdim[i][l]);
    TG_CUDA(cudaMalloc(&d_lam, sizeof(double) * 4 * lat.N * lam_ld));
    TG_CUDA(cudaMalloc(&d_su_flag, sizeof(int)));
    TG_CUDA(cudaMemset(d_su_flag, 0, sizeof(int)));
    TG_CUDA(cudaMalloc(&d_ptrs, sizeof(T*) * 4 * lat.N));
    TG_CUDA(cudaMallocHost(&h_ptrs, sizeof(T*) * 4 * lat.N));
    TG_CUDA(cudaMallocHost(&h_sig, sizeof(double) * 4 * lat.N));
    Tn.resize(lat.N);
    Trot.resize(lat.N);
    rot_ok.assign(lat.N, false);
    lambda.resize(lat.N);
    for (int i = 0; i < lat.N; ++i) {
      const auto& v = lat.vdim[i];
      Tn[i] = zeros<T>({v[0], v[1], v[2], v[3], tdim(i)}, st);
      for (int l = 0; l < 4; ++l) lambda[i][l].assign(v[l], 1.0);
    }
    if (density) {
      Ts.resize(lat.N);
      for (int i = 0; i < lat.N; ++i) {
        const auto& v = lat.vdim[i];
        Ts[i] = zeros<T>({v[0], v[1], v[2], v[3], 1}, st);
      }
      std::vector<double> h(NW, 0.0);
      h[0] = 1.0;
      bra1 = from_host({1, 1, 1, 1, 1}, h.data());
      one1 = from_host({1, 1}, h.data());
    }
    const int64_t chi = P.chi;
    for (int k = 0; k < 4; ++k) {
      C[k].resize(lat.N);
      E[k].resize(lat.N);
    }
    for (int i = 0; i < lat.N; ++i) {
      for (int k = 0; k < 4; ++k) C[k][i] = zeros<T>({chi, chi}, st);
      // eTt: vdim[1], eTr: vdim[2], eTb: vdim[3], eTl: vdim[0] (tensors.cpp:57-60)
      // (iTPO: the bra leg of dimension 1, tensors.cpp:155-158)
      const int64_t dt = lat.vdim[i][1], dr = lat.vdim[i][2], db = lat.vdim[i][3], dl = lat.vdim[i][0];
      E[0][i] = zeros<T>({chi, chi, dt, density ? 1 : dt}, st);
      E[1][i] = zeros<T>({chi, chi, dr, density ? 1 : dr}, st);
      E[2][i] = zeros<T>({chi, chi, db, density ? 1 : db}, st);
      E[3][i] = zeros<T>({chi, chi, dl, density ? 1 : dl}, st);
    }
    TG_CUDA(cudaStreamSynchronize(st));
  }

  ~EngineT() override {
    drop_graph();
    // release device tensors before the stream goes away
    Tn.clear();
    Trot.clear();
    Ts.clear();
    bra1 = DT<T>();
    one1 = DT<T>();
    for (auto& v : C) v.clear();
    for (auto& v : E) v.clear();
    spec_old = DT<double>();
    warm_v.clear();  // every device tensor is freed on `st`, so before it is destroyed below
    op_cache.clear();
    if (st) cudaStreamSynchronize(st);
    cudaDeviceGraphMemTrim(dev);
    if (gj_params) cusolverDnDestroyGesvdjInfo(gj_params);
    for (int r = 1; r <= kRowStreams; ++r)
      if (sol_slot[r]) cusolverDnDestroy(sol_slot[r]);
    if (sol) cusolverDnDestroy(sol);
    cudaFree(d_max);
    cudaFree(d_info);
    cudaFree(d_flag);
    cudaFree(d_cut);
    cudaFree(d_lam);
    cudaFree(d_su_flag);
    cudaFree(d_ptrs);
    cudaFreeHost(h_ptrs);
    cudaFreeHost(h_sig);
    for (int r = 0; r < kRowStreams; ++r) {
      if (row_st[r]) cudaStreamDestroy(row_st[r]);
      if (ev_join[r]) cudaEventDestroy(ev_join[r]);
      if (ev_mid[r]) cudaEventDestroy(ev_mid[r]);
      if (ev_stagger[r]) cudaEventDestroy(ev_stagger[r]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (st) cudaStreamDestroy(st);
  }

  // ---------------------------------------------------------------- helpers
  // precision of the contraction products issued now: the absorption
  // contractions of a move run in `abs_prec` (3xTF32 when params.mixed),
  // everything else (initialisation, measurements, simple update) in FP64
  int cur_prec = 0;
  int abs_prec = 0;
  struct PrecScope {
    EngineT* e;
    int saved;
    PrecScope(EngineT* e_, int p) : e(e_), saved(e_->cur_prec) { e->cur_prec = p; }
    ~PrecScope() { e->cur_prec = saved; }
  };

  DT<T> td(const DT<T>& a, const DT<T>& b, const V& x, const V& y, bool ca = false, bool cb = false) {
    return tensordot<T>(a, b, x, y, st, ca, cb, cur_prec);
  }
  DT<T> tr(const DT<T>& a, const V& p) { return transpose<T>(a, p, st); }
  void normalize(DT<T>& a) { normalize_max_abs<T>(a.p, a.p, a.size(), d_max + slot, st); }
  // dst = a / max|a|, written into the existing storage of dst
  void normalize_into(const DT<T>& a, DT<T>& dst) {
    if (dst.size() != a.size()) fail(TG_E_RUNTIME, "normalize_into: size mismatch");
    normalize_max_abs<T>(a.p, dst.p, a.size(), d_max + slot, st);
  }

  // Run body(r) for r = 0 .. n-1, row r on row stream r % kRowStreams when
  // `parallel`, else in order on the current stream.  Tensors that a row
  // creates and that outlive it must be handed to `st` with keep() before
  // they are released, so that their release is ordered after every row.
  template <typename F>
  void for_rows(int n, bool parallel, F&& body) {
    if (!parallel || n < 2) {
      for (int r = 0; r < n; ++r) body(r);
      return;
    }
    const int ns = std::min(n, kRowStreams);
    TG_CUDA(cudaEventRecord(ev_fork, st));
    for (int s = 0; s < ns; ++s) TG_CUDA(cudaStreamWaitEvent(row_st[s], ev_fork, 0));
    cudaStream_t saved = st;
    const int saved_slot = slot;
    const bool stagger = n <= kRowStreams;  // one stream per row
    for (int r = 0; r < kRowStreams; ++r) stagger_rec[r] = false;
    auto join = [&]() {
      st = saved;
      slot = saved_slot;
      cur_row = -1;
      for (int s = 0; s < ns; ++s) {
        cudaEventRecord(ev_join[s], row_st[s]);
        cudaStreamWaitEvent(st, ev_join[s], 0);
      }
    };
    try {
      for (int r = 0; r < n; ++r) {
        st = row_st[r % ns];
        slot = 1 + r % ns;
        cur_row = stagger ? r : -1;
        body(r);
      }
    } catch (...) {
      join();
      throw;
    }
    join();
    TG_CUDA(cudaGetLastError());
  }
  // row staggering (see ev_stagger): wait for the previous row's mark / set this row's
  void stagger_wait() {
    if (cur_row > 0 && stagger_rec[cur_row - 1]) TG_CUDA(cudaStreamWaitEvent(st, ev_stagger[cur_row - 1], 0));
  }
  void stagger_mark() {
    if (cur_row >= 0 && !stagger_rec[cur_row]) {
      TG_CUDA(cudaEventRecord(ev_stagger[cur_row], st));
      stagger_rec[cur_row] = true;
    }
  }
  // release `v`'s storage in stream order on `st` (after a join)
  void keep(std::vector<DT<T>>& v) {
    for (auto& t : v)
      if (t.mem) t.mem->st = st;
  }
  // Rows run on their own streams except under the per-kernel profiler,
  // whose attribution wants one launch at a time.  (Rows with full-SVD
  // projectors synchronise with the host at every residual check, so they
  // overlap only with the rows that follow them.)
  bool rows_parallel() const { return !profile_enabled(); }

  void upload(DT<T>& t, const double* host) {
    TG_CUDA(cudaMemcpyAsync(t.p, host, sizeof(T) * t.size(), cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));
  }
  void download(const DT<T>& t, double* host) {
    TG_CUDA(cudaMemcpyAsync(host, t.p, sizeof(T) * t.size(), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
  }
  T scalar(const DT<T>& t) {
    T v;
    TG_CUDA(cudaMemcpyAsync(&v, t.p, sizeof(T), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return v;
  }
  DT<T> from_host(const Shape& s, const double* host) {
    DT<T> t(s, st);
    TG_CUDA(cudaMemcpyAsync(t.p, host, sizeof(T) * t.size(), cudaMemcpyHostToDevice, st));
    return t;
  }

  void check_site(int site) const {
    if (site < 0 || site >= lat.N) fail(TG_E_INPUT, "site index out of range: " + std::to_string(site));
  }

  // last leg of a site tensor: d, or d*d for an iTPO
  int64_t tdim(int site) const {
    const int64_t d = lat.pdim[site];
    return density ? d * d : d;
  }
  // the conjugated layer of a double-layer contraction: the tensor itself,
  // or the all-ones unit tensor of the single-layer network
  const DT<T>& bra(const DT<T>& t) const { return density ? bra1 : t; }

  // an iTPO site tensor with the operator op (d x d, on the device) traced
  // in: sum_{p,q} op[p,q] Tn[...,p,q] as (D,D,D,D,1) -- the operator legs
  // of contract_density_ctm/ctm.cpp:103 and correlation.cpp:46; with op the
  // identity, Make_single_tensor_density (ctm_single.cpp:43-50)
  DT<T> traced(int site, const DT<T>& op) {
    const int64_t dd = tdim(site);
    if (op.size() != dd) fail(TG_E_INPUT, "operator size does not match the site");
    return td(Tn[site], reshape(op, {dd, 1}), {4}, {0});
  }
  void traced_into(int site, const DT<T>& op, DT<T>& out) {
    const DT<T> t = traced(site, op);
    TG_CUDA(cudaMemcpyAsync(out.p, t.p, sizeof(T) * t.size(), cudaMemcpyDeviceToDevice, st));
  }

  // the tensor the CTMRG moves absorb at a site (Tn, or the iTPO's Ts) and
  // its rotations for the right / top / bottom moves, refreshed whenever Tn
  // has changed
  const DT<T>& rot(int site, int which) {
    if (!rot_ok[site]) {
      if (density) traced_into(site, identity_op(site), Ts[site]);
      const DT<T>& src = density ? Ts[site] : Tn[site];
      static const std::vector<int> perms[3] = {{2, 3, 0, 1, 4}, {1, 2, 3, 0, 4}, {3, 0, 1, 2, 4}};
      for (int w = 0; w < 3; ++w) {
        if (Trot[site][w].empty()) {
          Shape s(5);
          for (int a = 0; a < 5; ++a) s[a] = src.dim(perms[w][a]);
          Trot[site][w] = DT<T>(s, st);  // allocated once, rewritten when Tn changes
        }
        permute<T>(src.p, Trot[site][w].p, src.sh, perms[w], false, st);
      }
      rot_ok[site] = true;
    }
    return Trot[site][which];
  }
  const DT<T>& mt(int site) { return density ? Ts[site] : Tn[site]; }
  void prepare_rotations() {
    for (int i = 0; i < lat.N; ++i) rot(i, 0);
  }

  // Singular value decomposition of a row-major m x n matrix A (consumed):
  // U (m x k), s (k), VT (k x n), k = min(m, n).  cuSOLVER gesvd works on
  // column-major data with rows >= cols; for m <= n the row-major buffer is
  // the column-major A^T and the factors of A^T give those of A without any
  // transposition (U_A = conj(V_{A^T}), VT_A = U_{A^T}^T).
  void svd(DT<T>& A, int64_t m, int64_t n, DT<T>& U, DT<double>& s, DT<T>& VT) {
    if (m > n) {
      // work on the transpose: A^T (n x m), n < m
      DT<T> At = tr(reshape(A, {m, n}), {1, 0});
      DT<T> Ut, VTt;
      svd(At, n, m, Ut, s, VTt);  // A^T = Ut s VTt  ->  A = VTt^T s Ut^T
      const int64_t k = n;
      // U_A = (VTt)^T (m x k) without conj; VT_A = (Ut)^T (k x n)
      U = tr(reshape(VTt, {k, m}), {1, 0});
      VT = tr(reshape(Ut, {n, k}), {1, 0});
      return;
    }
    const int64_t k = m;  // m <= n
    // column-major view: B = A^T is n x m (rows >= cols)
    const int rows = static_cast<int>(n), cols = static_cast<int>(m);
    ProfScope ps(PK_SOLVER, st, (CPLX ? 4.0 : 1.0) * 22.0 * static_cast<double>(m) * m * n, 0.0);
    s = DT<double>({k}, st);
    DT<T> Ub({k, n}, st);   // U_B: n x k column-major  == VT_A row-major (k x n)
    DT<T> VTb({k, k}, st);  // VT_B: k x k column-major == U_A row-major (m x k)
    int lwork = 0;
    if constexpr (CPLX) {
      check_sol(cusolverDnZgesvd_bufferSize(hsol(), rows, cols, &lwork), "Zgesvd_bufferSize");
      DT<T> work({static_cast<int64_t>(std::max(lwork, 1))}, st);
      DT<double> rwork({std::max<int64_t>(5 * k, 1)}, st);
      check_sol(cusolverDnZgesvd(hsol(), 'S', 'S', rows, cols, reinterpret_cast<cuDoubleComplex*>(A.p), rows, s.p,
                                 reinterpret_cast<cuDoubleComplex*>(Ub.p), rows,
                                 reinterpret_cast<cuDoubleComplex*>(VTb.p), cols,
                                 reinterpret_cast<cuDoubleComplex*>(work.p), lwork, rwork.p, info_slot()),
                "Zgesvd");
    } else {
      check_sol(cusolverDnDgesvd_bufferSize(hsol(), rows, cols, &lwork), "Dgesvd_bufferSize");
      DT<T> work({static_cast<int64_t>(std::max(lwork, 1))}, st);
      check_sol(cusolverDnDgesvd(hsol(), 'S', 'S', rows, cols, A.p, rows, s.p, Ub.p, rows, VTb.p, cols, work.p,
                                 lwork, nullptr, info_slot()),
                "Dgesvd");
    }
    U = reshape(VTb, {m, k});
    VT = reshape(Ub, {k, n});
    if constexpr (CPLX) {
      // U_A = conj(V_B) = (VT_B)^T read row-major without conj -> conj needed
      // only on the value: VT_B holds V_B^H, whose row-major reading is
      // conj(V_B) already; VT_A = U_B^T has no conjugation.
    }
  }

  // The same factors by cuSOLVER's Jacobi SVD (gesvdj, real matrices),
  // which takes any m, n and runs on the device without the host-side
  // bidiagonal iteration of gesvd; the energy gradient's projector SVDs use
  // it.  Singular vectors of vanishing values may be left incomplete, which
  // the gradient's SVD adjoint does not read.  The column-major view of the
  // row-major A is A^T = U' S V'^T, so VT = U'^T is U' read row-major and U
  // is the transpose of V' read row-major.
  gesvdjInfo_t gj_params = nullptr;
  void svd_jacobi(DT<T>& A, int64_t m, int64_t n, DT<T>& U, DT<double>& s, DT<T>& VT) {
    if constexpr (CPLX) {
      fail(TG_E_RUNTIME, "svd_jacobi: real matrices only");
    } else {
      if (!gj_params) {
        check_sol(cusolverDnCreateGesvdjInfo(&gj_params), "CreateGesvdjInfo");
        check_sol(cusolverDnXgesvdjSetSortEig(gj_params, 1), "gesvdjSetSortEig");
      }
      const int64_t k = std::min(m, n);
      const int rows = static_cast<int>(n), cols = static_cast<int>(m);
      ProfScope ps(PK_SOLVER, st, 22.0 * static_cast<double>(m) * n * k, 0.0);
      s = DT<double>({k}, st);
      DT<T> Ub({k, n}, st);  // U' (n x k column-major) = VT (k x n row-major)
      DT<T> Vb({k, m}, st);  // V' (m x k column-major) = U^T (k x m row-major)
      int lwork = 0;
      check_sol(cusolverDnDgesvdj_bufferSize(hsol(), CUSOLVER_EIG_MODE_VECTOR, 1, rows, cols, A.p, rows, s.p, Ub.p,
                                             rows, Vb.p, cols, &lwork, gj_params),
                "Dgesvdj_bufferSize");
      DT<T> work({static_cast<int64_t>(std::max(lwork, 1))}, st);
      check_sol(cusolverDnDgesvdj(hsol(), CUSOLVER_EIG_MODE_VECTOR, 1, rows, cols, A.p, rows, s.p, Ub.p, rows, Vb.p,
                                  cols, work.p, lwork, info_slot(), gj_params),
                "Dgesvdj");
      VT = reshape(Ub, {k, n});
      U = tr(reshape(Vb, {k, m}), {1, 0});
    }
  }

  int* info_slot() {
    if (info_used == kInfoSlots) check_infos();
    return d_info + info_used++;
  }
  // Every cuSOLVER call reports into its own device slot; a non-zero value
  // (illegal argument or non-convergence) is turned into an error here.
  void check_infos() {
    int flags[kRowStreams + 1] = {};
    TG_CUDA(cudaMemcpyAsync(flags, d_flag, sizeof(flags), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    int flag = 0;
    for (int f : flags) flag |= f;
    if (flag) {
      TG_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(flags), st));
      fail(TG_E_RUNTIME, "CholeskyQR orthonormalisation met a non-positive pivot (rank-deficient panel)");
    }
    TG_CUDA(cudaMemcpyAsync(&flag, d_su_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    if (flag) {
      TG_CUDA(cudaMemsetAsync(d_su_flag, 0, sizeof(int), st));
      fail(TG_E_RUNTIME, "simple update: the SVD of Theta did not converge (bond left unchanged)");
    }
    if (P.mixed && tc_fault_take())
      fail(TG_E_RUNTIME, "tensor-core product stopped waiting for its MMAs (results discarded)");
    if (info_used == 0) return;
    std::vector<int> h(static_cast<size_t>(info_used));
    TG_CUDA(cudaMemcpyAsync(h.data(), d_info, sizeof(int) * info_used, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    const int n = info_used;
    info_used = 0;
    for (int i = 0; i < n; ++i)
      if (h[static_cast<size_t>(i)] != 0) {
        TG_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int) * n, st));
        fail(TG_E_RUNTIME, "cuSOLVER factorisation failed, info = " + std::to_string(h[static_cast<size_t>(i)]));
      }
  }

  // QR of a row-major m x n matrix: Q (m x k), R (k x n), k = min(m, n)
  // (Householder, cuSOLVER geqrf + orgqr on a column-major copy).
  void qr(const DT<T>& A, int64_t m, int64_t n, DT<T>& Q, DT<T>& R) {
    const int64_t k = std::min(m, n);
    DT<T> Ac = tr(reshape(A, {m, n}), {1, 0});  // row-major (n, m) == column-major (m, n)
    ProfScope ps(PK_SOLVER, st, (CPLX ? 4.0 : 1.0) * 4.0 * static_cast<double>(m) * n * k, 0.0);
    DT<T> tau({std::max<int64_t>(k, 1)}, st);
    int lwork = 0, lwork2 = 0;
    const int im = static_cast<int>(m), in = static_cast<int>(n), ik = static_cast<int>(k);
    if constexpr (CPLX) {
      auto* a = reinterpret_cast<cuDoubleComplex*>(Ac.p);
      auto* t = reinterpret_cast<cuDoubleComplex*>(tau.p);
      check_sol(cusolverDnZgeqrf_bufferSize(hsol(), im, in, a, im, &lwork), "Zgeqrf_bufferSize");
      check_sol(cusolverDnZungqr_bufferSize(hsol(), im, ik, ik, a, im, t, &lwork2), "Zungqr_bufferSize");
      DT<T> work({static_cast<int64_t>(std::max(std::max(lwork, lwork2), 1))}, st);
      auto* w = reinterpret_cast<cuDoubleComplex*>(work.p);
      check_sol(cusolverDnZgeqrf(hsol(), im, in, a, im, t, w, std::max(lwork, lwork2), info_slot()), "Zgeqrf");
      // R: upper k x n of the factored matrix (column-major (m, n))
      R = DT<T>({n, k}, st);  // fill as row-major (n, k) == column-major (k, n)
      extract_r(Ac, m, n, k, R);
      check_sol(cusolverDnZungqr(hsol(), im, ik, ik, a, im, t, w, std::max(lwork, lwork2), info_slot()), "Zungqr");
    } else {
      check_sol(cusolverDnDgeqrf_bufferSize(hsol(), im, in, Ac.p, im, &lwork), "Dgeqrf_bufferSize");
      check_sol(cusolverDnDorgqr_bufferSize(hsol(), im, ik, ik, Ac.p, im, tau.p, &lwork2), "Dorgqr_bufferSize");
      DT<T> work({static_cast<int64_t>(std::max(std::max(lwork, lwork2), 1))}, st);
      check_sol(cusolverDnDgeqrf(hsol(), im, in, Ac.p, im, tau.p, work.p, std::max(lwork, lwork2), info_slot()), "Dgeqrf");
      R = DT<T>({n, k}, st);
      extract_r(Ac, m, n, k, R);
      check_sol(cusolverDnDorgqr(hsol(), im, ik, ik, Ac.p, im, tau.p, work.p, std::max(lwork, lwork2), info_slot()),
                "Dorgqr");
    }
    // Q: first k columns of the column-major (m, *) buffer -> row-major (m, k)
    DT<T> Qc = DT<T>({k, m}, st);
    TG_CUDA(cudaMemcpyAsync(Qc.p, Ac.p, sizeof(T) * k * m, cudaMemcpyDeviceToDevice, st));
    Q = tr(Qc, {1, 0});
    R = tr(R, {1, 0});  // column-major (k, n) -> row-major (k, n)
  }

  // copy the upper-trapezoidal k x n block of a column-major (m, n) matrix
  // into column-major (k, n) storage (row-major (n, k)), zeroing below the diagonal
  void extract_r(const DT<T>& Ac, int64_t m, int64_t n, int64_t k, DT<T>& R) {
    std::vector<T> h(static_cast<size_t>(m * n)), r(static_cast<size_t>(k * n));
    TG_CUDA(cudaMemcpyAsync(h.data(), Ac.p, sizeof(T) * m * n, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    for (int64_t c = 0; c < n; ++c)
      for (int64_t rr = 0; rr < k; ++rr) {
        T v = h[static_cast<size_t>(rr + c * m)];
        if (rr > c) std::memset(&v, 0, sizeof(T));
        r[static_cast<size_t>(rr + c * k)] = v;
      }
    TG_CUDA(cudaMemcpyAsync(R.p, r.data(), sizeof(T) * k * n, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));
  }

  // ------------------------------------------------------------ CTM pieces
  // LT = Tn1*(((C1*eT1)*eT8)*conj(Tn1)), legs (t12,t41,e12,e78,tc12,tc41)  (ctm.cpp:207-212)
  DT<T> block_LT(const DT<T>& C1, const DT<T>& eT1, const DT<T>& eT8, const DT<T>& T1) {
    DT<T> X = td(td(td(C1, eT1, {1}, {0}), eT8, {0}, {1}), bra(T1), {2, 5}, {1, 0}, false, true);
    return td(T1, X, {0, 1, 4}, {3, 1, 6});
  }
  // LB = Tn4*(((C4*eT7)*eT6)*conj(Tn4)), legs (t41,t34,e78,e56,tc41,tc34)  (ctm.cpp:222-227)
  DT<T> block_LB(const DT<T>& C4, const DT<T>& eT7, const DT<T>& eT6, const DT<T>& T4) {
    DT<T> X = td(td(td(C4, eT7, {1}, {0}), eT6, {0}, {1}), bra(T4), {2, 5}, {0, 3}, false, true);
    return td(T4, X, {0, 3, 4}, {1, 3, 6});
  }

  // ------------------------------------------------ matrix-view products
  // element (i, j) of a view is p[i*rs + j*cs]; one of rs / cs must be 1
  struct MV {
    const T* p;
    int64_t rows, cols, rs, cs;
    bool conj;
    // for a left operand: its TF32 split (rows x cols); for a right operand:
    // the split of its transpose (cols x rows).  Used by 3xTF32 products only.
    const SplitOperand* split = nullptr;
  };
  static MV rm(const T* p, int64_t r, int64_t c) { return MV{p, r, c, c, 1, false}; }      // row-major
  static MV cm(const T* p, int64_t r, int64_t c) { return MV{p, r, c, 1, r, false}; }      // column-major
  static MV tp(MV a) { return MV{a.p, a.cols, a.rows, a.cs, a.rs, a.conj}; }               // transpose
  static MV ht(MV a) { return MV{a.p, a.cols, a.rows, a.cs, a.rs, !a.conj}; }              // conj transpose
  static MV with_split(MV a, const SplitOperand* s) {
    a.split = s;
    return a;
  }
  // TF32 split of the left-operand view X (rows x cols), for reuse by several products
  struct Split {
    DT<float> buf;
    SplitOperand op;
  };
  Split split_of(const MV& X) {
    Split s;
    s.buf = DT<float>({split_operand_floats(X.rows, X.cols)}, st);
    split_operand(reinterpret_cast<const double*>(X.p), X.rows, X.cols, X.rs, X.cs, s.buf.p, &s.op, st);
    return s;
  }
  // C (rows x cols at C[i*crs + j*ccs]) = A B
  void mm(const MV& A, const MV& B, T* C, int64_t crs, int64_t ccs) {
    if (A.cols != B.rows) fail(TG_E_INPUT, "mm: inner dimensions differ");
    GemmDesc g{};
    g.M = A.rows;
    g.N = B.cols;
    g.K = A.cols;
    g.batch = 1;
    g.sAm = A.rs;
    g.sAk = A.cs;
    g.sBk = B.rs;
    g.sBn = B.cs;
    g.sCm = crs;
    g.sCn = ccs;
    g.conjA = A.conj;
    g.conjB = B.conj;
    g.accumulate = false;
    g.prec = cur_prec;
    if (cur_prec == 1) {
      g.preA = A.split;
      g.preB = B.split;
    }
    gemm<T>(A.p, B.p, C, g, st);
  }
  DT<T> mm_rm(const MV& A, const MV& B) {  // row-major result
    DT<T> C({A.rows, B.cols}, st);
    mm(A, B, C.p, B.cols, 1);
    return C;
  }
  DT<T> mm_cm(const MV& A, const MV& B) {  // column-major result (stored as (cols, rows) row-major)
    DT<T> C({B.cols, A.rows}, st);
    mm(A, B, C.p, 1, A.rows);
    return C;
  }

  // Householder QR of a column-major n x k panel, in place (cuSOLVER geqrf):
  // R in the upper triangle, reflectors below; tau returned.
  DT<T> geqrf_cm(DT<T>& Y, int64_t n, int64_t k) {
    DT<T> tau({std::max<int64_t>(k, 1)}, st);
    int lwork = 0;
    const int in = static_cast<int>(n), ik = static_cast<int>(k);
    ProfScope ps(PK_SOLVER, st, (CPLX ? 4.0 : 1.0) * 2.0 * n * k * k, 0.0);
    if constexpr (CPLX) {
      auto* a = reinterpret_cast<cuDoubleComplex*>(Y.p);
      check_sol(cusolverDnZgeqrf_bufferSize(hsol(), in, ik, a, in, &lwork), "Zgeqrf_bufferSize");
      DT<T> work({std::max<int64_t>(lwork, 1)}, st);
      check_sol(cusolverDnZgeqrf(hsol(), in, ik, a, in, reinterpret_cast<cuDoubleComplex*>(tau.p),
                                 reinterpret_cast<cuDoubleComplex*>(work.p), lwork, info_slot()),
                "Zgeqrf");
    } else {
      check_sol(cusolverDnDgeqrf_bufferSize(hsol(), in, ik, Y.p, in, &lwork), "Dgeqrf_bufferSize");
      DT<T> work({std::max<int64_t>(lwork, 1)}, st);
      check_sol(cusolverDnDgeqrf(hsol(), in, ik, Y.p, in, tau.p, work.p, lwork, info_slot()), "Dgeqrf");
    }
    return tau;
  }
  // form the explicit Q (n x k, column-major) from geqrf's output, in place
  void orgqr_cm(DT<T>& Y, int64_t n, int64_t k, const DT<T>& tau) {
    int lwork = 0;
    const int in = static_cast<int>(n), ik = static_cast<int>(k);
    ProfScope ps(PK_SOLVER, st, (CPLX ? 4.0 : 1.0) * 2.0 * n * k * k, 0.0);
    if constexpr (CPLX) {
      auto* a = reinterpret_cast<cuDoubleComplex*>(Y.p);
      auto* t = reinterpret_cast<const cuDoubleComplex*>(tau.p);
      check_sol(cusolverDnZungqr_bufferSize(hsol(), in, ik, ik, a, in, t, &lwork), "Zungqr_bufferSize");
      DT<T> work({std::max<int64_t>(lwork, 1)}, st);
      check_sol(cusolverDnZungqr(hsol(), in, ik, ik, a, in, t, reinterpret_cast<cuDoubleComplex*>(work.p), lwork,
                                 info_slot()),
                "Zungqr");
    } else {
      check_sol(cusolverDnDorgqr_bufferSize(hsol(), in, ik, ik, Y.p, in, tau.p, &lwork), "Dorgqr_bufferSize");
      DT<T> work({std::max<int64_t>(lwork, 1)}, st);
      check_sol(cusolverDnDorgqr(hsol(), in, ik, ik, Y.p, in, tau.p, work.p, lwork, info_slot()), "Dorgqr");
    }
  }
  void orth_cm(DT<T>& Y, int64_t n, int64_t k) {
    DT<T> tau = geqrf_cm(Y, n, k);
    orgqr_cm(Y, n, k, tau);
  }

  // Partial Gram matrices G_p = Y_p^H Y_p (k x k, row-major) of row chunks of
  // a column-major n x k panel (split-K DMMA products); sum_p G_p = Y^H Y.
  DT<T> gram_parts(const DT<T>& Y, int64_t n, int64_t k, int* nparts_out) {
    const int64_t chunk = std::max<int64_t>(64, (n + 63) / 64);
    const int64_t nfull = n / chunk, rem = n - nfull * chunk;
    const int nparts = static_cast<int>(nfull + (rem > 0 ? 1 : 0));
    DT<T> parts({nparts, k, k}, st);
    GemmDesc g{};
    g.M = k;
    g.N = k;
    g.sAm = n;  // A = Y^H: element (i, j) = conj(Y[j + i n])
    g.sAk = 1;
    g.sBk = 1;  // B = Y: element (j, c) = Y[j + c n]
    g.sBn = n;
    g.sCm = k;
    g.sCn = 1;
    g.conjA = true;
    g.conjB = false;
    g.accumulate = false;
    if (nfull > 0) {
      g.K = chunk;
      g.batch = nfull;
      g.bA = chunk;
      g.bB = chunk;
      g.bC = k * k;
      gemm<T>(Y.p, Y.p, parts.p, g, st);
    }
    if (rem > 0) {
      g.K = rem;
      g.batch = 1;
      gemm<T>(Y.p + nfull * chunk, Y.p + nfull * chunk, parts.p + nfull * k * k, g, st);
    }
    *nparts_out = nparts;
    return parts;
  }

  // Shifted CholeskyQR with column equilibration (Fukaya, Kannan,
  // Nakatsukasa, Yamamoto, Yanagisawa 2020): Gram / Cholesky / triangular
  // solve passes, orthonormal to O(u) for panels with condition number up to
  // ~1/u.  Y (column-major n x k) is replaced by an orthonormal Q.
  //
  // Only the span of Q is used.  A panel may be rank deficient (zero-padded
  // environment legs give exactly-zero rows), so after the first shifted pass
  // -- whose output has columns of norm <= 1 -- a counter-based Gaussian
  // perturbation of norm ~1e-14 per column is added: it turns the missing
  // directions into independent ones, which the following shifted pass and
  // two plain passes orthonormalise.  The perturbation moves the span by
  // ~1e-14, below the rounding of the products that produced the panel.
  //
  // passes = 4: two shifted and two plain passes, orthonormal to O(u): the
  // final range basis Q and the basis Qz of the Rayleigh-Ritz core.
  // passes = 2: the two shifted passes only, a basis of the same span with
  // condition number ~1e4 -- enough for the intermediate bases of the power
  // iteration, whose next product and orthonormalisation only use the span.
  // (One shifted pass is not enough: with weakly converged site tensors the
  // next panel's Gram matrix then met a non-positive pivot.)
  void orth_chol(DT<T>& Y, int64_t n, int64_t k, int passes = 4) {
    PrecScope fp64(this, 0);
    if constexpr (!CPLX) {
      if (cholqr_cluster_supported(n, k)) {
        DT<double> scratch({cholqr_scratch_doubles(k)}, st);
        cholqr_cluster(Y.p, n, k, passes, 2, ++noise_stream, 1e-14 / std::sqrt(static_cast<double>(n)), scratch.p,
                       d_flag + slot, st);
        return;
      }
    }
    for (int pass = 0; pass < passes; ++pass) {
      int nparts = 0;
      DT<T> parts = gram_parts(Y, n, k, &nparts);
      DT<T> G({k, k}, st);
      sum_partials<T>(parts.p, nparts, k * k, G.p, st);
      DT<T> Ri({k, k}, st);
      chol_rinv<T>(G.p, 1, k, n, pass <= 1 ? 1 : 0, Ri.p, d_flag + slot, st);
      Y = mm_cm(cm(Y.p, n, k), rm(Ri.p, k, k));
      if (pass == 0) add_noise<T>(Y.p, n * k, 1e-14 / std::sqrt(static_cast<double>(n)), ++noise_stream, st);
    }
  }

  // Randomized SVD of M = LTm * LBm (Halko, Martinsson & Tropp 2011,
  // Alg. 4.4 with q power iterations, then the SVD of B = Q^H M through a QR
  // of B^H and a one-sided Jacobi SVD of the k x k factor).  The test matrix
  // is the counter-based Gaussian stream shared with the CPU oracle.  Outputs
  // the truncated, 1/sqrt(s)-scaled factors Uc (nrow x w, row-major) and
  // Vc (ncol x w, row-major), w = min(k, chi); columns past `cut` are zero.
  // Stands in for mptensor::rsvd (src/iTPS/core/ctm.cpp:243-244).
  // lt, lb: LT, LB as row-major matrices; lth, lbh: their conjugate
  // transposes (the views may carry TF32 splits for 3xTF32 products)
  void rsvd_factors(const MV& lt, const MV& lth, const MV& lb, const MV& lbh, int64_t nrow, int64_t nmid,
                    int64_t ncol, int cut, int64_t k, DT<T>& Uc, DT<T>& Vc) {
    auto apply_M = [&](const DT<T>& Xcm) {  // (ncol x k) col-major -> (nrow x k) col-major
      DT<T> t = mm_cm(lb, cm(Xcm.p, ncol, k));
      return mm_cm(lt, cm(t.p, nmid, k));
    };
    auto apply_MH = [&](const DT<T>& Ycm) {  // (nrow x k) -> (ncol x k), both col-major
      DT<T> t = mm_cm(lth, cm(Ycm.p, nrow, k));
      return mm_cm(lbh, cm(t.p, nmid, k));
    };
    rsvd_run(apply_M, apply_MH, nrow, ncol, cut, k, Uc, Vc);
  }

  // The range finder, core SVD and truncation of rsvd_factors for any M
  // given by its products: apply_M maps a column-major (ncol x k) panel to
  // M times it (nrow x k, column-major), apply_MH the same for M^H.
  template <typename FM, typename FMH>
  void rsvd_run(FM&& apply_M, FMH&& apply_MH, int64_t nrow, int64_t ncol, int cut, int64_t k, DT<T>& Uc,
                DT<T>& Vc) {
    DT<T> Om({k, ncol}, st);
    counter_normal<T>(Om.p, ncol, k, P.rsvd_seed, 0, st);
    stagger_wait();
    DT<T> Q = apply_M(Om);
    stagger_mark();
    orth_chol(Q, nrow, k, P.rsvd_power_iters > 0 ? 2 : 4);
    for (int it = 0; it < P.rsvd_power_iters; ++it) {
      DT<T> Z = apply_MH(Q);
      orth_chol(Z, ncol, k, 2);
      Q = apply_M(Z);
      orth_chol(Q, nrow, k, it + 1 < P.rsvd_power_iters ? 2 : 4);
    }
    // B = Q^H M = Z^H with Z = M^H Q.  With Qz an orthonormal basis of
    // range(Z), B = (Z^H Qz) Qz^H, so the SVD of the k x k matrix T = Z^H Qz,
    // T = Ut S Wt^H, gives B = Ut S (Qz Wt)^H.
    DT<T> Z = apply_MH(Q);  // ncol x k, column-major
    DT<T> Qz = clone(Z, st);
    orth_chol(Qz, ncol, k);
    PrecScope fp64(this, 0);  // the core SVD and its basis changes stay FP64
    DT<T> Tm = mm_rm(ht(cm(Z.p, ncol, k)), cm(Qz.p, ncol, k));  // k x k row-major
    DT<T> Ur({k, k}, st), Wr({k, k}, st);
    DT<double> s({k}, st);
    // (The previous sweep's right singular vectors are no warm start here: T
    // is expressed in the CholeskyQR basis of Z, which rotates within the
    // kept subspace from sweep to sweep, so a cold start needs fewer sweeps.)
    jacobi_svd<T>(Tm.p, k, Ur.p, s.p, Wr.p, st);  // T Wr = Ur S
    DT<T> U = mm_rm(cm(Q.p, nrow, k), rm(Ur.p, k, k));
    DT<T> V = mm_rm(cm(Qz.p, ncol, k), rm(Wr.p, k, k));
    const int w = static_cast<int>(std::min<int64_t>(k, P.chi));
    DT<double> sinv({w}, st);
    truncation(s.p, k, cut, P.inverse_projector_cut, sinv.p, w, d_cut + slot, st);
    Uc = DT<T>({nrow, w}, st);
    scale_cols<T>(U.p, k, nrow, w, sinv.p, false, Uc.p, st);
    Vc = DT<T>({ncol, w}, st);
    scale_cols<T>(V.p, k, ncol, w, sinv.p, false, Vc.p, st);
  }

  // ------------------------------------------------ exact truncated SVD
  // The full-SVD projectors (ctm.cpp:273-302, 441-475) keep at most chi
  // singular triplets of an n x n matrix (n = chi D^2: 2592 at D = 6,
  // chi = 72), so the dense SVD of the whole matrix is not needed.  The kept
  // triplets come from block subspace iteration on M (alternating products
  // with M and M^H, i.e. orthogonal iteration on M^H M: Golub & Van Loan,
  // Matrix Computations, 4th ed., sec. 8.2.4) on a block of b > chi
  // columns, orthonormalised by the rSVD's shifted CholeskyQR.  A two-sided
  // Rayleigh-Ritz step -- the SVD of the b x b matrix T = Q^H M Qz, Qz an
  // orthonormal basis of M^H Q, by the one-CTA Jacobi kernel -- gives
  // approximate triplets (s_i, u_i = Q t_i, v_i = Qz w_i) for which
  // M^H u_i = s_i v_i holds exactly; they are accepted once every triplet
  // the truncation keeps also has || M v_i - s_i u_i || <= kExactTol s_0,
  // which bounds the angle between each kept vector and the exact one by
  // that residual over the gap to the rest of the spectrum.  The result
  // therefore matches the dense SVD's truncated factors to that accuracy.
  // The start block holds the basis that the same projector (move, line,
  // row) ended with in the previous sweep -- an almost converged guess once
  // the environment settles -- completed with counter-based Gaussian
  // columns.  If the residuals are not below the tolerance after
  // kExactMaxIters iterations (a flat spectrum at the block edge), the
  // dense SVD is used instead.
  static constexpr double kExactTol = 1e-13;
  static constexpr int kExactMaxIters = 80;
  std::map<int, DT<T>> warm_v;   // right basis (ncol x b, column-major) per projector
  int proj_key = -1;             // set by the moves before each projector
  int64_t exact_solves = 0, exact_iters = 0, exact_checks = 0, exact_dense = 0;

  // block size of the subspace iteration, or -1 where the dense SVD is the
  // better choice: a matrix whose smaller dimension a block would span gains
  // nothing from the iteration (and its first-sweep panels can be almost
  // entirely null space), and chi too close to the largest block leaves no
  // room for oversampling
  int exact_block(int64_t kmax) const {
    const int bmax = CPLX ? 84 : 96;  // CholeskyQR / Jacobi core sizes (one cluster, one CTA)
    const int64_t w = std::min<int64_t>(P.chi, kmax);
    if (kmax <= bmax) return -1;
    const int64_t b = std::min<int64_t>(bmax, std::max<int64_t>(w + 16, w + w / 3));
    return b >= w + 8 ? static_cast<int>(b) : -1;
  }

  // Truncated factors of M (views m = M, mh = M^H, nrow x ncol) as rsvd_run
  // returns them: Uc (nrow x w) and Vc (ncol x w), row-major, scaled by
  // 1/sqrt(s), zero past the cut.  Returns false when the dense SVD must be
  // used (block too small for chi, or no convergence).
  bool exact_factors(const MV& m, const MV& mh, int64_t nrow, int64_t ncol, DT<T>& Uc, DT<T>& Vc) {
    const int64_t kmax = std::min(nrow, ncol);
    const int b = exact_block(kmax);
    if (b < 1) return false;
    PrecScope fp64(this, 0);
    const int w = static_cast<int>(std::min<int64_t>(P.chi, kmax));
    ++exact_solves;
    // Attempt 0 orthonormalises by shifted CholeskyQR.  A matrix of rank below
    // the block (the padded environments of an iTPO, whose single-layer
    // matrices are narrow) can leave a Gram matrix that no shift makes
    // positive: the solve then starts again with Householder QR, which
    // yields orthonormal columns for any panel, before giving up for the
    // dense SVD.
    for (int attempt = 0; attempt < 2; ++attempt) {
      const bool householder = attempt == 1;
      auto orth = [&](DT<T>& X, int64_t n, int passes) {
        if (householder) orth_cm(X, n, b);
        else orth_chol(X, n, b, passes);
      };
      DT<T> Om({b, ncol}, st);  // column-major ncol x b
      int w0 = 0;
      auto hit = warm_v.find(proj_key);
      if (proj_key >= 0 && hit != warm_v.end() && hit->second.size() == static_cast<int64_t>(b) * ncol) {
        w0 = w;
        TG_CUDA(cudaMemcpyAsync(Om.p, hit->second.p, sizeof(T) * w0 * ncol, cudaMemcpyDeviceToDevice, st));
      }
      if (b > w0) counter_normal<T>(Om.p + static_cast<int64_t>(w0) * ncol, ncol, b - w0, P.rsvd_seed, 7, st);
      DT<T> Q = mm_cm(m, cm(Om.p, ncol, b));  // nrow x b, column-major
      int next_check = (w0 > 0 || b == kmax) ? 1 : 3;
      orth(Q, nrow, next_check == 1 ? 4 : 2);
      std::vector<double> hs(static_cast<size_t>(b)), hr(static_cast<size_t>(w));
      int prev_it = 0;
      double prev_ratio = 0.0;
      bool pivot_failed = false;
      for (int it = 1; it <= kExactMaxIters; ++it) {
        ++exact_iters;
        DT<T> Z = mm_cm(mh, cm(Q.p, nrow, b));  // M^H Q: ncol x b
        if (it < next_check) {
          orth(Z, ncol, 2);
          Q = mm_cm(m, cm(Z.p, ncol, b));
          orth(Q, nrow, it + 1 == next_check ? 4 : 2);
          continue;
        }
        ++exact_checks;
        DT<T> Qz = clone(Z, st);
        orth(Qz, ncol, 4);
        DT<T> Tm = mm_rm(ht(cm(Z.p, ncol, b)), cm(Qz.p, ncol, b));  // Q^H M Qz (b x b row-major)
        DT<T> Ur({b, b}, st), Wr({b, b}, st);
        DT<double> s({b}, st);
        jacobi_svd<T>(Tm.p, b, Ur.p, s.p, Wr.p, st);  // T Wr = Ur S
        DT<T> Y = mm_cm(m, cm(Qz.p, ncol, b));        // M Qz: nrow x b
        DT<T> MV1 = mm_cm(cm(Y.p, nrow, b), rm(Wr.p, b, b));  // M v_i
        DT<T> U1 = mm_cm(cm(Q.p, nrow, b), rm(Ur.p, b, b));   // u_i
        DT<double> r({w}, st);
        ritz_residual<T>(MV1.p, U1.p, s.p, nrow, w, r.p, st);
        int pivot_flag = 0;
        TG_CUDA(cudaMemcpyAsync(hs.data(), s.p, sizeof(double) * b, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaMemcpyAsync(hr.data(), r.p, sizeof(double) * w, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaMemcpyAsync(&pivot_flag, d_flag + slot, sizeof(int), cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
        if (pivot_flag) {  // an orthonormalisation met a non-positive pivot
          TG_CUDA(cudaMemsetAsync(d_flag + slot, 0, sizeof(int), st));
          pivot_failed = true;
          break;
        }
        // the kept triplets: the truncation rule of ctm.cpp:277-288
        int cut = w;
        for (int i = 0; i < w; ++i)
          if (!(hs[static_cast<size_t>(i)] > P.inverse_projector_cut * hs[0])) {
            cut = i;
            break;
          }
        double worst = 0.0;
        for (int i = 0; i < cut; ++i) worst = std::max(worst, hr[static_cast<size_t>(i)]);
        const double ratio = hs[0] > 0.0 ? worst / (kExactTol * hs[0]) : 0.0;
        if (ratio <= 1.0 || b == kmax) {
          DT<T> U = mm_rm(cm(Q.p, nrow, b), rm(Ur.p, b, b));   // nrow x b row-major
          DT<T> V = mm_rm(cm(Qz.p, ncol, b), rm(Wr.p, b, b));  // ncol x b row-major
          DT<double> sinv({w}, st);
          truncation(s.p, b, P.chi, P.inverse_projector_cut, sinv.p, w, d_cut + slot, st);
          Uc = DT<T>({nrow, w}, st);
          scale_cols<T>(U.p, b, nrow, w, sinv.p, false, Uc.p, st);
          Vc = DT<T>({ncol, w}, st);
          scale_cols<T>(V.p, b, ncol, w, sinv.p, false, Vc.p, st);
          if (proj_key >= 0) warm_v[proj_key] = mm_cm(cm(Qz.p, ncol, b), rm(Wr.p, b, b));
          return true;
        }
        // a stalled decay (a flat spectrum at the block edge): the dense SVD
        if (prev_it > 0 && it > 12 && ratio > 0.5 * prev_ratio) break;
        // iterations to the next check, from the decay seen between the last two
        int gap = 3;
        if (prev_it > 0 && ratio < prev_ratio) {
          const double f = std::pow(ratio / prev_ratio, 1.0 / (it - prev_it));
          gap = static_cast<int>(std::ceil(std::log(ratio) / -std::log(f)));
          gap = std::min(16, std::max(1, gap));
        }
        prev_it = it;
        prev_ratio = ratio;
        next_check = it + gap;
        Q = std::move(Y);
        orth(Q, nrow, next_check == it + 1 ? 4 : 2);
      }
      if (!pivot_failed) break;
    }
    ++exact_dense;
    return false;
  }

  // The SVD of a strongly rectangular M (nrow x ncol, row-major; the long
  // side at least 4 times the short one k, and k within the one-CTA Jacobi
  // kernel's limit) by R-SVD: a Householder QR of the tall one of M^H / M,
  // the Jacobi SVD of the k x k factor, and two products back -- in place of
  // cuSOLVER's gesvd, whose bidiagonalisation of the whole matrix is a chain
  // of hundreds of small launches (about 3 ms a call at 48 x 1200 complex:
  // the projectors of a line with a D = 1 leg are that narrow).  Outputs as
  // svd(): U (nrow x k), s (k, descending), VT (k x ncol), row-major.
  // Returns false (computing nothing) for other shapes, which keep gesvd.
  bool small_side_svd(const DT<T>& Min, int64_t nrow, int64_t ncol, DT<T>& U, DT<double>& s, DT<T>& VT) {
    const int64_t k = std::min(nrow, ncol);
    if (k < 2 || k > jacobi_svd_max_k<T>() || std::max(nrow, ncol) < 4 * k) return false;
    const DT<T> M = reshape(Min, {nrow, ncol});
    PrecScope fp64(this, 0);  // every product of the factorisation in FP64
    DT<T> Ub({k, k}, st), Wb({k, k}, st);
    s = DT<double>({k}, st);
    if (ncol >= nrow) {
      // Q R = M^H (ncol x k); B = M Q = R^H (k x k); B = Ub S Wb^H; M = Ub S (Q Wb)^H
      DT<T> Q = transpose<T>(M, {0, 1}, st, true);  // column-major view: M^H
      orth_cm(Q, ncol, k);
      DT<T> B = mm_rm(rm(M.p, nrow, ncol), cm(Q.p, ncol, k));
      jacobi_svd<T>(B.p, k, Ub.p, s.p, Wb.p, st);  // B Wb = Ub S
      U = Ub;
      VT = transpose<T>(mm_rm(cm(Q.p, ncol, k), rm(Wb.p, k, k)), {1, 0}, st, true);
    } else {
      // Q R = M (nrow x k); B = Q^H M = R (k x k); B = Ub S Wb^H; M = (Q Ub) S Wb^H
      DT<T> Q = transpose<T>(M, {1, 0}, st);  // column-major view: M
      orth_cm(Q, nrow, k);
      DT<T> B = mm_rm(ht(cm(Q.p, nrow, k)), rm(M.p, nrow, ncol));
      jacobi_svd<T>(B.p, k, Ub.p, s.p, Wb.p, st);
      U = mm_rm(cm(Q.p, nrow, k), rm(Ub.p, k, k));
      VT = transpose<T>(Wb, {1, 0}, st, true);
    }
    return true;
  }

  // Truncated projectors from M (nrow x ncol, consumed):
  // U_c (nrow x w), VT_c (w x ncol) scaled by 1/sqrt(s), w = min(k, chi)
  void truncated_factors(DT<T>& M, int64_t nrow, int64_t ncol, DT<T>& Uc, DT<T>& VTc) {
    if (P.svd_solver == 0) {
      const MV m = rm(M.p, nrow, ncol);
      DT<T> Vc;
      if (exact_factors(m, ht(m), nrow, ncol, Uc, Vc)) {
        VTc = transpose<T>(Vc, {1, 0}, st, true);  // VT_c = V_c^H (w x ncol)
        return;
      }
    }
    DT<T> U, VT;
    DT<double> s;
    if (!small_side_svd(M, nrow, ncol, U, s, VT)) svd(M, nrow, ncol, U, s, VT);
    const int64_t k = std::min(nrow, ncol);
    const int w = static_cast<int>(std::min<int64_t>(k, P.chi));
    DT<double> sinv({w}, st);
    truncation(s.p, k, P.chi, P.inverse_projector_cut, sinv.p, w, d_cut + slot, st);
    Uc = DT<T>({nrow, w}, st);
    scale_cols<T>(U.p, k, nrow, w, sinv.p, false, Uc.p, st);
    VTc = DT<T>({w, ncol}, st);
    scale_rows<T>(VT.p, ncol, ncol, w, sinv.p, false, VTc.p, st);
  }

  // Calc_projector_left_block (ctm.cpp:174-318)
  void proj_left_block(const DT<T>& C1, const DT<T>& C4, const DT<T>& eT1, const DT<T>& eT6,
                       const DT<T>& eT7, const DT<T>& eT8, const DT<T>& T1, const DT<T>& T4, DT<T>& PU,
                       DT<T>& PL) {
    const int64_t e12 = eT1.dim(1), e56 = eT6.dim(0), e78 = eT8.dim(0);
    const int64_t t12 = T1.dim(2), t41 = T1.dim(3), t34 = T4.dim(2);
    // the bra's bond dimensions: t.. again, or 1 in the single-layer network of an iTPO
    const int64_t b12 = bra(T1).dim(2), b41 = bra(T1).dim(3), b34 = bra(T4).dim(2);
    if (t41 != 1) {
      // LT as the matrix [(t12,e12,tc12), (t41,e78,tc41)], LB as [(t41,e78,tc41), (t34,e56,tc34)]:
      // M = LTm LBm is tensordot(LT, LB, Axes(1,3,5), Axes(0,2,4)) of ctm.cpp:273
      DT<T> LTm = tr(block_LT(C1, eT1, eT8, T1), {0, 2, 4, 1, 3, 5});
      DT<T> LBm = tr(block_LB(C4, eT7, eT6, T4), {0, 2, 4, 1, 3, 5});
      const int64_t nrow = t12 * e12 * b12, nmid = t41 * e78 * b41, ncol = t34 * e56 * b34;
      MV lt = rm(LTm.p, nrow, nmid), lb = rm(LBm.p, nmid, ncol);
      MV lth = ht(lt), lbh = ht(lb);
      // 3xTF32: LT, LB and their transposes are the left operands of every
      // product below (six range-finder products, PU, PL); split them once
      Split s_lt, s_lth, s_lb, s_lbh;
      if constexpr (!CPLX) {
        if (cur_prec == 1 && (t12 != 1 && t34 != 1) && P.use_rsvd) {
          s_lt = split_of(lt);
          s_lth = split_of(lth);
          s_lb = split_of(lb);
          s_lbh = split_of(lbh);
          lt.split = &s_lt.op;
          lth.split = &s_lth.op;
          lb.split = &s_lb.op;
          lbh.split = &s_lbh.op;
        }
      }
      DT<T> Uc, Vrow;  // Uc: nrow x w;  PU = LBm * Vc where Vc = (VT_c)^H
      MV vc{nullptr, 0, 0, 0, 0, false};
      if ((t12 != 1 && t34 != 1) && P.use_rsvd) {
        // cut = min(chi, e78 t41^2, e12 t12^2, e56 t34^2), k = factor * cut (ctm.cpp:242-244;
        // single layer: e78 t41, ..., ctm_single.cpp:200-203)
        const int cut = static_cast<int>(std::min<int64_t>(std::min<int64_t>(P.chi, nmid), std::min(nrow, ncol)));
        int64_t k = P.rsvd_oversample_abs >= 0 ? cut + P.rsvd_oversample_abs
                                               : static_cast<int64_t>(P.rsvd_oversampling_factor * cut);
        k = std::min<int64_t>(std::min(k, nrow), ncol);
        if (k > jacobi_svd_max_k<T>())
          fail(TG_E_INPUT, "rSVD sketch size " + std::to_string(k) + " exceeds " +
                               std::to_string(jacobi_svd_max_k<T>()) +
                               " (lower rsvd_oversampling_factor or set rsvd_oversample_abs)");
        rsvd_factors(lt, lth, lb, lbh, nrow, nmid, ncol, cut, k, Uc, Vrow);
        vc = rm(Vrow.p, ncol, Vrow.dim(1));
      } else {
        DT<T> M = mm_rm(lt, lb);
        truncated_factors(M, nrow, ncol, Uc, Vrow);  // Vrow = VT_c (w x ncol)
        vc = ht(rm(Vrow.p, Vrow.dim(0), ncol));
      }
      const int64_t w = Uc.dim(1);
      // PU = tensordot(LB, conj(VT_c), Axes(1,3,5), Axes(1,2,3)).transpose(1,0,2,3)  (ctm.cpp:263-266)
      PU = tr(reshape(mm_rm(lb, vc), {t41, e78, b41, w}), {1, 0, 2, 3});
      // PL = tensordot(LT, conj(U_c), Axes(0,2,4), Axes(0,1,2)).transpose(1,0,2,3)
      MV uc = rm(Uc.p, nrow, w);
      uc.conj = true;
      MV ltt = tp(lt);
      ltt.split = lth.split;  // real operands: transpose = conjugate transpose
      PL = tr(reshape(mm_rm(ltt, uc), {t41, e78, b41, w}), {1, 0, 2, 3});
    } else {
      PU = DT<T>({e78, 1, 1, e78}, st);
      identity<T>(PU.p, e78, st);
      PL = clone(PU, st);
    }
  }

  // rSVD branch of Calc_projector_updown_blocks (ctm.cpp:401-439).  The
  // matrix is M = RT^T LT LB RB over the row legs (t23,e34,tc23) of RT and
  // the column legs (t23,e34,tc23) of RB -- the product Mult_col_ud applies
  // (ctm.cpp:129-149) and R1 R2^T of the full-SVD branch -- and it is only
  // ever applied to panels, four products at a time, never formed.  With the
  // blocks as matrices (rows / columns = the legs named):
  //   RTm: (t12,e12,tc12) x (t23,e34,tc23)    LTm: (t12,e12,tc12) x (t41,e78,tc41)
  //   LBm: (t41,e78,tc41) x (t34,e56,tc34)    RBm: (t34,e56,tc34) x (t23,e34,tc23)
  // the projectors are PU = LBm RBm V_c and PL = LTm^T RTm conj(U_c), each
  // reshaped to (t41,e78,tc41,cut) and transposed (1,0,2,3) (ctm.cpp:434-439).
  void proj_updown_rsvd(const DT<T>& LT, const DT<T>& RT, const DT<T>& RB, const DT<T>& LB, int64_t e34,
                        int64_t t23, int64_t b23, int64_t e78, int64_t t41, int64_t b41, DT<T>& PU, DT<T>& PL) {
    DT<T> RTm = tr(RT, {0, 3, 4, 1, 2, 5});
    DT<T> LTm = tr(LT, {0, 2, 4, 1, 3, 5});
    DT<T> LBm = tr(LB, {0, 2, 4, 1, 3, 5});
    DT<T> RBm = tr(RB, {0, 2, 4, 1, 3, 5});
    const int64_t na = RT.dim(0) * RT.dim(3) * RT.dim(4), n = RT.dim(1) * RT.dim(2) * RT.dim(5);
    const int64_t nb = LT.dim(1) * LT.dim(3) * LT.dim(5), nc = LB.dim(1) * LB.dim(3) * LB.dim(5);
    if (RB.dim(1) * RB.dim(3) * RB.dim(5) != n || LT.dim(0) * LT.dim(2) * LT.dim(4) != na)
      fail(TG_E_RUNTIME, "proj_updown_rsvd: block shapes do not chain");
    const MV rtm = rm(RTm.p, na, n), ltm = rm(LTm.p, na, nb), lbm = rm(LBm.p, nb, nc), rbm = rm(RBm.p, nc, n);
    MV rtm_c = rtm;
    rtm_c.conj = true;
    // cut = min(chi, e34 t23^2), k = factor * cut (ctm.cpp:410-414; single layer:
    // e34 t23, ctm_single.cpp:362-365)
    const int cut = static_cast<int>(std::min<int64_t>(P.chi, e34 * t23 * b23));
    int64_t k = P.rsvd_oversample_abs >= 0 ? cut + P.rsvd_oversample_abs
                                           : static_cast<int64_t>(P.rsvd_oversampling_factor * cut);
    k = std::min<int64_t>(k, n);
    if (k > jacobi_svd_max_k<T>())
      fail(TG_E_INPUT, "rSVD sketch size " + std::to_string(k) + " exceeds " +
                           std::to_string(jacobi_svd_max_k<T>()) +
                           " (lower rsvd_oversampling_factor or set rsvd_oversample_abs)");
    auto apply_M = [&](const DT<T>& Xcm) {  // RTm^T (LTm (LBm (RBm X)))
      DT<T> a = mm_cm(rbm, cm(Xcm.p, n, k));
      DT<T> b = mm_cm(lbm, cm(a.p, nc, k));
      a = mm_cm(ltm, cm(b.p, nb, k));
      return mm_cm(tp(rtm), cm(a.p, na, k));
    };
    auto apply_MH = [&](const DT<T>& Ycm) {  // RBm^H (LBm^H (LTm^H (conj(RTm) Y)))
      DT<T> a = mm_cm(rtm_c, cm(Ycm.p, n, k));
      DT<T> b = mm_cm(ht(ltm), cm(a.p, na, k));
      a = mm_cm(ht(lbm), cm(b.p, nb, k));
      return mm_cm(ht(rbm), cm(a.p, nc, k));
    };
    DT<T> Uc, Vc;
    rsvd_run(apply_M, apply_MH, n, n, cut, k, Uc, Vc);
    const int64_t w = Uc.dim(1);
    DT<T> t = mm_rm(rbm, rm(Vc.p, n, w));  // (nc x w)
    PU = tr(reshape(mm_rm(lbm, rm(t.p, nc, w)), {t41, e78, b41, w}), {1, 0, 2, 3});
    MV uc = rm(Uc.p, n, w);
    uc.conj = true;
    t = mm_rm(rtm, uc);  // (na x w)
    PL = tr(reshape(mm_rm(tp(ltm), rm(t.p, na, w)), {t41, e78, b41, w}), {1, 0, 2, 3});
  }

  // Calc_projector_updown_blocks (ctm.cpp:320-491): full-SVD and rSVD branches
  void proj_updown(const DT<T>& C1, const DT<T>& C2, const DT<T>& C3, const DT<T>& C4, const DT<T>& eT1,
                   const DT<T>& eT2, const DT<T>& eT3, const DT<T>& eT4, const DT<T>& eT5, const DT<T>& eT6,
                   const DT<T>& eT7, const DT<T>& eT8, const DT<T>& T1, const DT<T>& T2, const DT<T>& T3,
                   const DT<T>& T4, DT<T>& PU, DT<T>& PL) {
    const int64_t e78 = eT7.dim(1), e34 = eT3.dim(1);
    const int64_t t23 = T2.dim(3), t41 = T4.dim(1);
    if (t41 != 1) {
      DT<T> LT = block_LT(C1, eT1, eT8, T1);
      DT<T> X = td(td(td(C2, eT3, {1}, {0}), eT2, {0}, {1}), bra(T2), {2, 5}, {2, 1}, false, true);
      DT<T> RT = td(T2, X, {1, 2, 4}, {3, 1, 6});
      X = td(td(td(C3, eT5, {1}, {0}), eT4, {0}, {1}), bra(T3), {2, 5}, {3, 2}, false, true);
      DT<T> RB = td(T3, X, {2, 3, 4}, {3, 1, 6});
      DT<T> LB = block_LB(C4, eT7, eT6, T4);
      if (t23 != 1 && P.use_rsvd) {
        proj_updown_rsvd(LT, RT, RB, LB, e34, t23, bra(T2).dim(3), e78, t41, bra(T4).dim(1), PU, PL);
        return;
      }
      DT<T> R1 = td(RT, LT, {0, 3, 4}, {0, 2, 4});
      DT<T> R2 = td(RB, LB, {0, 2, 4}, {1, 3, 5});
      DT<T> M = td(R1, R2, {3, 4, 5}, {3, 4, 5});
      const int64_t nrow = M.dim(0) * M.dim(1) * M.dim(2), ncol = M.dim(3) * M.dim(4) * M.dim(5);
      DT<T> Uc, VTc;
      const Shape ms = M.sh;
      truncated_factors(M, nrow, ncol, Uc, VTc);
      const int64_t w = Uc.dim(1);
      DT<T> VTc4 = reshape(VTc, {w, ms[3], ms[4], ms[5]});
      DT<T> Uc4 = reshape(Uc, {ms[0], ms[1], ms[2], w});
      PU = tr(td(R2, VTc4, {0, 1, 2}, {1, 2, 3}, false, true), {1, 0, 2, 3});
      PL = tr(td(R1, Uc4, {0, 1, 2}, {0, 1, 2}, false, true), {1, 0, 2, 3});
    } else {
      PU = DT<T>({e78, 1, 1, e78}, st);
      identity<T>(PU.p, e78, st);
      PL = clone(PU, st);
    }
  }

  // Pass 2 of a move, every line at once: Calc_Next_CTM (ctm.cpp:493-518,
  // the new corners, normalised by their largest element) and Calc_Next_eT
  // (ctm.cpp:520-552, the new edges) for all rows, stage by stage, each stage's products over all
  // rows in ONE grouped persistent launch (gemm_group; the 3xTF32 form runs
  // them one by one).  Stage 1 reads every corner and edge tensor the pass
  // needs; the new ones are written at the ends of stages 2 and 4, so no
  // row reads a tensor another row has already replaced -- on a skewed cell,
  // where one row's next line is another row's current one, this is what
  // the reference's C1_bak / C4_bak / eTl_bak copies (ctm.cpp:595-601)
  // provide.
  struct CtmAbs {
    const DT<T>*C1, *C4, *eT1, *eT6, *PU, *PL;
    DT<T>*C1o, *C4o;
  };
  struct EtAbs {
    const DT<T>*eT8, *T1, *PU, *PL;
    DT<T>* out;
  };
  // One stage of absorb: the tensordots `specs`, independent of each other.
  // The operand permutations run on the row streams; FP64 products without
  // a specialised kernel (gemm_specialised) then run as one grouped launch on
  // `st`, while the others -- and every 3xTF32 product -- run one by one on
  // the row streams, overlapping it.
  struct TdSpec {
    DT<T> a, b;
    V x, y;
    bool ca;
  };
  std::vector<DT<T>> td_stage(std::vector<TdSpec>& specs) {
    const int n = static_cast<int>(specs.size());
    std::vector<TdPlan<T>> plans(static_cast<size_t>(n));
    std::vector<char> alone(static_cast<size_t>(n), 0);
    const bool par = rows_parallel() && n > 1;
    const int ns = par ? std::min(n, kRowStreams) : 0;
    cudaStream_t home = st;
    if (par) {
      TG_CUDA(cudaEventRecord(ev_fork, home));
      for (int r = 0; r < ns; ++r) TG_CUDA(cudaStreamWaitEvent(row_st[r], ev_fork, 0));
    }
    auto on = [&](int q) { return par ? row_st[q % ns] : home; };
    auto make = [&](int q) {
      TdSpec& sp = specs[static_cast<size_t>(q)];
      plans[static_cast<size_t>(q)] = plan_tensordot<T>(sp.a, sp.b, sp.x, sp.y, on(q), sp.ca, false, cur_prec);
      const GemmDesc& g = plans[static_cast<size_t>(q)].g;
      alone[static_cast<size_t>(q)] = cur_prec != 0 || gemm_specialised<T>(g);
    };
    auto own = [&](int q) {
      TdPlan<T>& pl = plans[static_cast<size_t>(q)];
      if (pl.g.K > 0) gemm<T>(pl.A.p, pl.B.p, pl.C.p, pl.g, on(q));
    };
    // the grouped products' operands first on every row stream, then the lone products
    for (int q = 0; q < n; ++q) make(q);
    std::vector<TdPlan<T>> grouped;
    for (int q = 0; q < n; ++q)
      if (!alone[static_cast<size_t>(q)]) grouped.push_back(plans[static_cast<size_t>(q)]);
    if (par)
      for (int r = 0; r < ns; ++r) TG_CUDA(cudaEventRecord(ev_mid[r], row_st[r]));
    for (int q = 0; q < n; ++q)
      if (alone[static_cast<size_t>(q)]) own(q);
    if (!grouped.empty()) {
      if (par)
        for (int r = 0; r < ns; ++r) TG_CUDA(cudaStreamWaitEvent(home, ev_mid[r], 0));
      tensordot_group<T>(grouped, home);
    }
    if (par)
      for (int r = 0; r < ns; ++r) {
        TG_CUDA(cudaEventRecord(ev_join[r], row_st[r]));
        TG_CUDA(cudaStreamWaitEvent(home, ev_join[r], 0));
      }
    std::vector<DT<T>> out;
    for (TdPlan<T>& pl : plans) {
      // tensors made on a row stream: released on `st`, after the join
      for (DT<T>* t : {&pl.A, &pl.B, &pl.C})
        if (t->mem) t->mem->st = home;
      out.push_back(pl.C);
    }
    return out;
  }

  void absorb(const std::vector<CtmAbs>& cj, const std::vector<EtAbs>& ej) {
    std::vector<TdSpec> ps;
    auto plan = [&](const DT<T>& a, const DT<T>& b, const V& x, const V& y, bool ca = false) {
      ps.push_back({a, b, x, y, ca});
    };
    auto run = [&](std::vector<TdSpec>& sp) {
      std::vector<DT<T>> out = td_stage(sp);
      sp.clear();
      return out;
    };
    const size_t nc = cj.size(), ne = ej.size();
    // stage 1: C1 eT1, eT6 C4 (next_ctm), eT8 PL (next_et)
    for (const CtmAbs& c : cj) {
      plan(*c.C1, *c.eT1, {1}, {0});
      plan(*c.eT6, *c.C4, {1}, {0});
    }
    for (const EtAbs& e : ej) plan(*e.eT8, *e.PL, {1}, {0});
    std::vector<DT<T>> r1 = run(ps);
    // stage 2: the new corners, and the bra layer of the new edges
    for (size_t q = 0; q < nc; ++q) {
      plan(*cj[q].PU, r1[2 * q], {0, 1, 2}, {0, 2, 3});
      plan(r1[2 * q + 1], *cj[q].PL, {3, 1, 2}, {0, 1, 2});
    }
    for (size_t q = 0; q < ne; ++q) plan(bra(*ej[q].T1), r1[2 * nc + q], {0, 1}, {2, 4}, true);
    std::vector<DT<T>> r2 = run(ps);
    r1.clear();
    for (size_t q = 0; q < nc; ++q) {
      normalize_into(r2[2 * q], *cj[q].C1o);
      normalize_into(r2[2 * q + 1], *cj[q].C4o);
    }
    if (ne == 0) return;
    // stage 3: the ket layer
    for (size_t q = 0; q < ne; ++q) plan(*ej[q].T1, r2[2 * nc + q], {0, 1, 4}, {4, 5, 2});
    std::vector<DT<T>> r3 = run(ps);
    r2.clear();
    // stage 4: PU closes the new edges
    for (size_t q = 0; q < ne; ++q) plan(r3[q], *ej[q].PU, {1, 3, 4}, {1, 2, 0});
    std::vector<DT<T>> r4 = run(ps);
    r3.clear();
    for (size_t q = 0; q < ne; ++q) normalize_into(tr(r4[q], {3, 2, 0, 1}), *ej[q].out);
  }

  // ------------------------------------------------------------- the moves
  //
  // Each move has the two passes of Left_move (ctm.cpp:562-616): all the
  // projectors of the line (rows on their own streams), then the new corners
  // and edges of the next line (absorb, all rows at once).  The reference
  // writes into copies (C1_bak, ...) and copies back; here the results go
  // straight into the environment storage.  The reference computes every new
  // edge tensor twice -- row iy's eT[k] and row iy-1's eT[j] are the same
  // Calc_Next_eT of the same inputs -- so each distinct (output, inputs) job
  // runs once; when two jobs write one output the later one wins, as in the
  // reference.
  struct EtJob {
    int out, src, site, pu, pl;
    bool same_inputs(const EtJob& o) const { return src == o.src && site == o.site && pu == o.pu && pl == o.pl; }
  };
  static std::vector<EtJob> final_jobs(const std::vector<EtJob>& jobs) {
    std::vector<EtJob> out;
    for (size_t a = 0; a < jobs.size(); ++a) {
      bool superseded = false;
      for (size_t b = a + 1; b < jobs.size(); ++b)
        if (jobs[b].out == jobs[a].out && !jobs[b].same_inputs(jobs[a])) superseded = true;
      bool repeated = false;
      for (const EtJob& o : out)
        if (o.out == jobs[a].out && o.same_inputs(jobs[a])) repeated = true;
      if (!superseded && !repeated) out.push_back(jobs[a]);
    }
    return out;
  }

  void left_move(int ix) {
    auto &C1 = C[0], &C2 = C[1], &C3 = C[2], &C4 = C[3];
    auto &eTt = E[0], &eTr = E[1], &eTb = E[2], &eTl = E[3];
    const int LY = lat.LY_noskew;
    const bool par = rows_parallel();
    if (density) prepare_rotations();  // Ts, before the rows fork
    std::vector<DT<T>> PUs(LY), PLs(LY);
    for_rows(LY, par, [&](int iy) {
      proj_key = (0 * 4096 + ix) * 4096 + iy;
      const int i = lat.index(ix, iy), j = lat.right(i), k = lat.bottom(j), l = lat.left(k);
      if (P.projector_corner)
        proj_left_block(C1[i], C4[l], eTt[i], eTb[l], eTl[l], eTl[i], mt(i), mt(l), PUs[iy], PLs[iy]);
      else
        proj_updown(C1[i], C2[j], C3[k], C4[l], eTt[i], eTt[j], eTr[j], eTr[k], eTb[k], eTb[l], eTl[l], eTl[i],
                    mt(i), mt(j), mt(k), mt(l), PUs[iy], PLs[iy]);
    });
    std::vector<EtJob> jobs;
    for (int iy = 0; iy < LY; ++iy) {
      const int i = lat.index(ix, iy), j = lat.right(i), k = lat.bottom(j), l = lat.left(k);
      const int up = (iy + 1) % LY, dn = (iy - 1 + LY) % LY;
      jobs.push_back({j, i, i, iy, up});
      jobs.push_back({k, l, l, dn, iy});
    }
    const std::vector<EtJob> fin = final_jobs(jobs);
    std::vector<CtmAbs> cj;
    std::vector<EtAbs> ej;
    for (int iy = 0; iy < LY; ++iy) {
      const int i = lat.index(ix, iy), j = lat.right(i), k = lat.bottom(j), l = lat.left(k);
      const int up = (iy + 1) % LY, dn = (iy - 1 + LY) % LY;
      cj.push_back({&C1[i], &C4[l], &eTt[i], &eTb[l], &PUs[up], &PLs[dn], &C1[j], &C4[k]});
    }
    for (const EtJob& b : fin) ej.push_back({&eTl[b.src], &mt(b.site), &PUs[b.pu], &PLs[b.pl], &eTl[b.out]});
    absorb(cj, ej);
    keep(PUs);
    keep(PLs);
  }

  void right_move(int ix) {
    auto &C1 = C[0], &C2 = C[1], &C3 = C[2], &C4 = C[3];
    auto &eTt = E[0], &eTr = E[1], &eTb = E[2], &eTl = E[3];
    const int LY = lat.LY_noskew;
    const bool par = rows_parallel();
    prepare_rotations();  // before the rows fork
    std::vector<DT<T>> PUs(LY), PLs(LY);
    for_rows(LY, par, [&](int iy) {
      proj_key = (1 * 4096 + ix) * 4096 + iy;
      const int k = lat.index(ix, iy), l = lat.left(k), i = lat.top(l), j = lat.right(i);
      if (P.projector_corner)
        proj_left_block(C3[k], C2[j], eTb[k], eTt[j], eTr[j], eTr[k], rot(k, 0), rot(j, 0), PUs[iy], PLs[iy]);
      else
        proj_updown(C3[k], C4[l], C1[i], C2[j], eTb[k], eTb[l], eTl[l], eTl[i], eTt[i], eTt[j], eTr[j], eTr[k],
                    rot(k, 0), rot(l, 0), rot(i, 0), rot(j, 0), PUs[iy], PLs[iy]);
    });
    std::vector<EtJob> jobs;
    for (int iy = 0; iy < LY; ++iy) {
      const int k = lat.index(ix, iy), l = lat.left(k), i = lat.top(l), j = lat.right(i);
      const int up = (iy + 1) % LY, dn = (iy - 1 + LY) % LY;
      jobs.push_back({l, k, k, iy, dn});
      jobs.push_back({i, j, j, up, iy});
    }
    const std::vector<EtJob> fin = final_jobs(jobs);
    std::vector<CtmAbs> cj;
    std::vector<EtAbs> ej;
    for (int iy = 0; iy < LY; ++iy) {
      const int k = lat.index(ix, iy), l = lat.left(k), i = lat.top(l), j = lat.right(i);
      const int up = (iy + 1) % LY, dn = (iy - 1 + LY) % LY;
      cj.push_back({&C3[k], &C2[j], &eTb[k], &eTt[j], &PUs[dn], &PLs[up], &C3[l], &C2[i]});
    }
    for (const EtJob& b : fin) ej.push_back({&eTr[b.src], &rot(b.site, 0), &PUs[b.pu], &PLs[b.pl], &eTr[b.out]});
    absorb(cj, ej);
    keep(PUs);
    keep(PLs);
  }

  void top_move(int iy) {
    auto &C1 = C[0], &C2 = C[1], &C3 = C[2], &C4 = C[3];
    auto &eTt = E[0], &eTr = E[1], &eTb = E[2], &eTl = E[3];
    const int LX = lat.LX_noskew;
    const bool par = rows_parallel();
    prepare_rotations();
    std::vector<DT<T>> PUs(LX), PLs(LX);
    for_rows(LX, par, [&](int ix) {
      proj_key = (2 * 4096 + iy) * 4096 + ix;
      const int j = lat.index(ix, iy), k = lat.bottom(j), l = lat.left(k), i = lat.top(l);
      if (P.projector_corner)
        proj_left_block(C2[j], C1[i], eTr[j], eTl[i], eTt[i], eTt[j], rot(j, 1), rot(i, 1), PUs[ix], PLs[ix]);
      else
        proj_updown(C2[j], C3[k], C4[l], C1[i], eTr[j], eTr[k], eTb[k], eTb[l], eTl[l], eTl[i], eTt[i], eTt[j],
                    rot(j, 1), rot(k, 1), rot(l, 1), rot(i, 1), PUs[ix], PLs[ix]);
    });
    std::vector<EtJob> jobs;
    for (int ix = 0; ix < LX; ++ix) {
      const int j = lat.index(ix, iy), k = lat.bottom(j), l = lat.left(k), i = lat.top(l);
      const int rt = (ix + 1) % LX, lf = (ix - 1 + LX) % LX;
      jobs.push_back({k, j, j, ix, rt});
      jobs.push_back({l, i, i, lf, ix});
    }
    const std::vector<EtJob> fin = final_jobs(jobs);
    std::vector<CtmAbs> cj;
    std::vector<EtAbs> ej;
    for (int ix = 0; ix < LX; ++ix) {
      const int j = lat.index(ix, iy), k = lat.bottom(j), l = lat.left(k), i = lat.top(l);
      const int rt = (ix + 1) % LX, lf = (ix - 1 + LX) % LX;
      cj.push_back({&C2[j], &C1[i], &eTr[j], &eTl[i], &PUs[rt], &PLs[lf], &C2[k], &C1[l]});
    }
    for (const EtJob& b : fin) ej.push_back({&eTt[b.src], &rot(b.site, 1), &PUs[b.pu], &PLs[b.pl], &eTt[b.out]});
    absorb(cj, ej);
    keep(PUs);
    keep(PLs);
  }

  void bottom_move(int iy) {
    auto &C1 = C[0], &C2 = C[1], &C3 = C[2], &C4 = C[3];
    auto &eTt = E[0], &eTr = E[1], &eTb = E[2], &eTl = E[3];
    const int LX = lat.LX_noskew;
    const bool par = rows_parallel();
    prepare_rotations();
    std::vector<DT<T>> PUs(LX), PLs(LX);
    for_rows(LX, par, [&](int ix) {
      proj_key = (3 * 4096 + iy) * 4096 + ix;
      const int l = lat.index(ix, iy), i = lat.top(l), j = lat.right(i), k = lat.bottom(j);
      if (P.projector_corner)
        proj_left_block(C4[l], C3[k], eTl[l], eTr[k], eTb[k], eTb[l], rot(l, 2), rot(k, 2), PUs[ix], PLs[ix]);
      else
        proj_updown(C4[l], C1[i], C2[j], C3[k], eTl[l], eTl[i], eTt[i], eTt[j], eTr[j], eTr[k], eTb[k], eTb[l],
                    rot(l, 2), rot(i, 2), rot(j, 2), rot(k, 2), PUs[ix], PLs[ix]);
    });
    std::vector<EtJob> jobs;
    for (int ix = 0; ix < LX; ++ix) {
      const int l = lat.index(ix, iy), i = lat.top(l), j = lat.right(i), k = lat.bottom(j);
      const int rt = (ix + 1) % LX, lf = (ix - 1 + LX) % LX;
      jobs.push_back({i, l, l, ix, lf});
      jobs.push_back({j, k, k, rt, ix});
    }
    const std::vector<EtJob> fin = final_jobs(jobs);
    std::vector<CtmAbs> cj;
    std::vector<EtAbs> ej;
    for (int ix = 0; ix < LX; ++ix) {
      const int l = lat.index(ix, iy), i = lat.top(l), j = lat.right(i), k = lat.bottom(j);
      const int rt = (ix + 1) % LX, lf = (ix - 1 + LX) % LX;
      cj.push_back({&C4[l], &C3[k], &eTl[l], &eTr[k], &PUs[lf], &PLs[rt], &C4[i], &C3[j]});
    }
    for (const EtJob& b : fin) ej.push_back({&eTb[b.src], &rot(b.site, 2), &PUs[b.pu], &PLs[b.pl], &eTb[b.out]});
    absorb(cj, ej);
    keep(PUs);
    keep(PLs);
  }

  // ------------------------------------------------------ initialisation
  // zero-pad / slice X to the static environment shape, into `out`'s storage
  void fit(const DT<T>& X, int64_t d1, int64_t d2, int64_t rest, DT<T>& out) {
    const int64_t chi = P.chi;
    // corners are rank 2; edges keep their two physical-bond legs even when those are 1
    Shape s = out.rank() == 2 ? Shape{chi, chi} : Shape{chi, chi, X.dim(4), X.dim(5)};
    if (s != out.sh) fail(TG_E_RUNTIME, "environment initialisation: shape mismatch");
    fit_chi<T>(X.p, d1, d2, rest, out.p, chi, st);
  }

  // Calc_CTM_Environment_density's initialisation (ctm_single.cpp:752-960):
  // every corner / edge is the neighbouring site's Ts summed over its outer
  // legs (a contraction with all-ones vectors).  The reference keeps these
  // at their natural size; here they are zero-padded to chi, which changes
  // no contraction and no kept singular value.
  void ctm_init_density() {
    prepare_rotations();  // Ts
    auto sum_leg = [&](const DT<T>& A, int leg) {
      const int64_t n = A.dim(leg);
      std::vector<double> h(static_cast<size_t>(n * NW), 0.0);
      for (int64_t k = 0; k < n; ++k) h[static_cast<size_t>(k * NW)] = 1.0;
      return td(A, from_host({n}, h.data()), {leg}, {0});
    };
    auto put = [&](const DT<T>& X, DT<T>& out) {  // X (d1, d2, rest...) into (chi, chi, rest...)
      int64_t rest = 1;
      for (int a = 2; a < X.rank(); ++a) rest *= X.dim(a);
      fit_chi<T>(X.p, X.dim(0), X.dim(1), rest, out.p, P.chi, st);
    };
    for (int i = 0; i < lat.N; ++i) {
      put(tr(sum_leg(sum_leg(Ts[lat.top(lat.left(i))], 0), 0), {1, 0, 2}), C[0][i]);       // (b, r)
      put(sum_leg(sum_leg(Ts[lat.top(lat.right(i))], 1), 1), C[1][i]);                     // (l, b)
      put(tr(sum_leg(sum_leg(Ts[lat.bottom(lat.right(i))], 2), 2), {1, 0, 2}), C[2][i]);   // (t, l)
      put(tr(sum_leg(sum_leg(Ts[lat.bottom(lat.left(i))], 0), 2), {1, 0, 2}), C[3][i]);    // (r, t)
      put(sum_leg(Ts[lat.top(i)], 1), E[0][i]);                                            // (l, r, b)
      put(tr(sum_leg(Ts[lat.right(i)], 2), {1, 2, 0, 3}), E[1][i]);                        // (t, b, l)
      put(tr(sum_leg(Ts[lat.bottom(i)], 3), {2, 0, 1, 3}), E[2][i]);                       // (r, l, t)
      put(tr(sum_leg(Ts[lat.left(i)], 0), {2, 0, 1, 3}), E[3][i]);                         // (b, t, r)
    }
    env_ready = true;
    spec_old = spectra();
    spec_old_ok = true;
    TG_CUDA(cudaStreamSynchronize(st));
  }

  void ctm_init() override {
    if (density) {
      ctm_init_density();
      return;
    }
    for (int i = 0; i < lat.N; ++i) {
      int num = lat.top(lat.left(i));
      const DT<T>* t = &Tn[num];
      DT<T> X = tr(td(*t, *t, {0, 1, 4}, {0, 1, 4}, false, true), {1, 3, 0, 2});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), 1, C[0][i]);
      num = lat.top(lat.right(i));
      t = &Tn[num];
      X = tr(td(*t, *t, {1, 2, 4}, {1, 2, 4}, false, true), {0, 2, 1, 3});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), 1, C[1][i]);
      num = lat.bottom(lat.right(i));
      t = &Tn[num];
      X = tr(td(*t, *t, {2, 3, 4}, {2, 3, 4}, false, true), {1, 3, 0, 2});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), 1, C[2][i]);
      num = lat.bottom(lat.left(i));
      t = &Tn[num];
      X = tr(td(*t, *t, {0, 3, 4}, {0, 3, 4}, false, true), {1, 3, 0, 2});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), 1, C[3][i]);
      num = lat.top(i);
      t = &Tn[num];
      X = tr(td(*t, *t, {1, 4}, {1, 4}, false, true), {0, 3, 1, 4, 2, 5});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), X.dim(4) * X.dim(5), E[0][i]);
      num = lat.right(i);
      t = &Tn[num];
      X = tr(td(*t, *t, {2, 4}, {2, 4}, false, true), {1, 4, 2, 5, 0, 3});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), X.dim(4) * X.dim(5), E[1][i]);
      num = lat.bottom(i);
      t = &Tn[num];
      X = tr(td(*t, *t, {3, 4}, {3, 4}, false, true), {2, 5, 0, 3, 1, 4});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), X.dim(4) * X.dim(5), E[2][i]);
      num = lat.left(i);
      t = &Tn[num];
      X = tr(td(*t, *t, {0, 4}, {0, 4}, false, true), {2, 5, 0, 3, 1, 4});
      fit(X, X.dim(0) * X.dim(1), X.dim(2) * X.dim(3), X.dim(4) * X.dim(5), E[3][i]);
    }
    env_ready = true;
    spec_old = spectra();
    spec_old_ok = true;
    TG_CUDA(cudaStreamSynchronize(st));
  }

  void require_env() const {
    if (!env_ready) fail(TG_E_STATE, "environment not initialised (call tg_ctm_init or tg_set_env first)");
  }

  void ctm_move(int dir, int line) override {
    require_env();
    PrecScope prec(this, abs_prec);
    const int L = (dir <= 1) ? lat.LX_noskew : lat.LY_noskew;
    if (line < 0 || line >= L) fail(TG_E_INPUT, "move line out of range");
    switch (dir) {
      case 0: left_move(line); break;
      case 1: right_move(line); break;
      case 2: top_move(line); break;
      case 3: bottom_move(line); break;
      default: fail(TG_E_INPUT, "move direction must be 0..3");
    }
    check_infos();
  }

  void sweep_impl() {
    PrecScope prec(this, abs_prec);
    noise_stream = 0;  // the same perturbation keys in every sweep, eager or replayed
    const int LX = lat.LX_noskew, LY = lat.LY_noskew;
    for (int ix = 0; ix < LX; ++ix) left_move(ix);
    for (int ix = 0; ix > -LX; --ix) right_move((ix + 1 + LX) % LX);
    for (int iy = 0; iy > -LY; --iy) top_move((iy + 1 + LY) % LY);
    for (int iy = 0; iy < LY; ++iy) bottom_move(iy);
  }

  // ------------------------------------------------ CUDA-graph sweep
  //
  // With rSVD corner projectors a sweep has no host synchronisation and all
  // shapes are static (the environment is kept at chi), so one sweep is
  // captured into a CUDA graph and replayed: ~4000 launches become one
  // graph launch.  The graph bakes in the addresses of the site tensors,
  // their rotations and the environment; it is re-captured when any of them
  // changes.  The first sweep after a change runs eagerly (it also fixes the
  // kernels' shared-memory attributes), the second is captured.
  cudaGraphExec_t g_exec = nullptr;
  std::vector<const void*> g_addr;
  uint64_t g_kernels = 0;
  bool g_warm = false, g_broken = false;

  std::vector<const void*> state_addresses() {
    std::vector<const void*> a;
    for (int i = 0; i < lat.N; ++i) {
      a.push_back(Tn[i].p);
      for (int w = 0; w < 3; ++w) a.push_back(rot(i, w).p);
      if (density) a.push_back(Ts[i].p);
      for (int k = 0; k < 4; ++k) {
        a.push_back(C[k][i].p);
        a.push_back(E[k][i].p);
      }
    }
    a.push_back(reinterpret_cast<const void*>(static_cast<intptr_t>(abs_prec)));
    return a;
  }

  bool graph_capable() const {
    if (!P.cuda_graph || g_broken || !P.use_rsvd || !P.projector_corner || profile_enabled()) return false;
    for (int i = 0; i < lat.N; ++i)
      for (int l = 0; l < 4; ++l)
        if (lat.vdim[i][l] == 1) return false;  // D = 1 legs can select the full-SVD branch
    return true;
  }

  void drop_graph() {
    if (g_exec) cudaGraphExecDestroy(g_exec);
    g_exec = nullptr;
    g_addr.clear();
    g_warm = false;
  }

  void capture_sweep() {
    drop_graph();
    const uint64_t before = launch_count();
    TG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    try {
      sweep_impl();
    } catch (...) {
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      g_broken = true;  // eager sweeps from now on
      uncount_launch(launch_count() - before);
      return;
    }
    TG_CUDA(cudaStreamEndCapture(st, &g));
    g_kernels = launch_count() - before;
    uncount_launch(g_kernels);  // recorded, not run
    const cudaError_t e = cudaGraphInstantiate(&g_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      cudaGetLastError();
      g_exec = nullptr;
      g_broken = true;
      return;
    }
    g_addr = state_addresses();
  }

  void run_sweep() {
    if (!graph_capable()) {
      sweep_impl();
      return;
    }
    const std::vector<const void*> addr = state_addresses();  // also refreshes the rotations
    if (!g_exec || addr != g_addr) {
      if (g_exec) drop_graph();
      if (!g_warm) {
        sweep_impl();
        g_warm = true;
        return;
      }
      capture_sweep();
      if (!g_exec) {
        sweep_impl();
        return;
      }
    }
    TG_CUDA(cudaGraphLaunch(g_exec, st));
    count_launch(g_kernels);
  }

  void ctm_sweep() override {
    require_env();
    run_sweep();
    check_infos();
    TG_CUDA(cudaStreamSynchronize(st));
  }

  // normalised corner spectra of every site, ordered (site, corner)
  DT<double> spectra() {
    const int cnt = 4 * lat.N;
    TG_CUDA(cudaStreamSynchronize(st));  // h_ptrs is reused
    for (int i = 0; i < lat.N; ++i)
      for (int k = 0; k < 4; ++k) h_ptrs[4 * i + k] = C[k][i].p;
    TG_CUDA(cudaMemcpyAsync(d_ptrs, h_ptrs, sizeof(T*) * cnt, cudaMemcpyHostToDevice, st));
    DT<double> out({cnt, static_cast<int64_t>(P.chi)}, st);
    batched_spectrum<T>(d_ptrs, cnt, P.chi, out.p, nullptr, st);
    return out;
  }

  void check_convergence(int* converged, double* sig_max) override {
    require_env();
    if (!spec_old_ok) fail(TG_E_STATE, "no previous corner spectra");
    DT<double> now = spectra();
    const int cnt = 4 * lat.N;
    DT<double> sig({cnt}, st);
    spectrum_distance(now.p, spec_old.p, cnt, P.chi, sig.p, st);
    TG_CUDA(cudaMemcpyAsync(h_sig, sig.p, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st));
    check_infos();
    // early break on the first corner above epsilon, in the reference's
    // order (site-major, C1..C4), ctm.cpp:828-967
    double smax = 0.0;
    bool conv = true;
    for (int b = 0; b < cnt; ++b) {
      const double s = h_sig[b];
      if (s > P.ctm_convergence_epsilon) {
        smax = s;
        conv = false;
        break;
      } else if (s > smax) {
        smax = s;
      }
    }
    spec_old = now;
    if (converged) *converged = conv ? 1 : 0;
    if (sig_max) *sig_max = smax;
  }

  void ctm_run(int initialize, int* iterations, int* converged, double* sig_max) override {
    if (initialize) ctm_init();
    require_env();
    if (!initialize || !spec_old_ok) {
      spec_old = spectra();
      spec_old_ok = true;
    }
    int count = 0, conv = 0;
    double smax = 0.0;
    while (!conv && count < P.max_ctm_iteration) {
      run_sweep();
      check_convergence(&conv, &smax);
      ++count;
    }
    if (iterations) *iterations = count;
    if (converged) *converged = conv;
    if (sig_max) *sig_max = smax;
  }

  void corner_spectrum(int which, int site, double* host) override {
    require_env();
    check_site(site);
    if (which < 0 || which > 3) fail(TG_E_INPUT, "corner index must be 0..3");
    DT<double> sp = spectra();
    TG_CUDA(cudaMemcpyAsync(host, sp.p + (4 * site + which) * P.chi, sizeof(double) * P.chi,
                            cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
  }

  // ---------------------------------------------------------- observables
  // Contract_one_site_iTPS_CTM (contract_itps_ctm/ctm.cpp:89-113)
  // (iTPO: Contract_one_site_density_CTM, contract_density_ctm/ctm.cpp:89-116,
  // as the single-layer network of the site tensor with op traced in)
  T one_site(int i, const DT<T>& op) {
    if (density) return one_site_t(i, traced(i, op), one1);
    return one_site_t(i, Tn[i], op);
  }
  T one_site_t(int i, const DT<T>& T1, const DT<T>& op) {
    const DT<T>&C1 = C[0][i], &C2 = C[1][i], &C3 = C[2][i], &C4 = C[3][i];
    const DT<T>&eT1 = E[0][i], &eT2 = E[1][i], &eT3 = E[2][i], &eT4 = E[3][i];
    DT<T> X = td(td(C2, td(C3, eT2, {0}, {1}), {1}, {1}), td(C1, eT1, {1}, {0}), {0}, {1});
    DT<T> Y = td(td(td(C4, eT4, {1}, {0}), eT3, {0}, {1}), bra(T1), {2, 5}, {0, 3}, false, true);
    DT<T> Z = td(X, Y, {0, 2, 3, 5}, {2, 5, 0, 4});
    DT<T> W = td(Z, T1, {0, 1, 2, 3}, {2, 1, 0, 3});
    return scalar(td(W, op, {0, 1}, {1, 0}));
  }

  void measure_onesite(int site, const double* op, double* out) override {
    require_env();
    check_site(site);
    const int64_t d = lat.pdim[site];
    DT<T> o = from_host({d, d}, op);
    T v = one_site(site, o);
    std::memcpy(out, &v, sizeof(T));
    if constexpr (!CPLX) out[1] = 0.0;
  }

  // Contract_two_sites_horizontal_op12_iTPS_CTM (contract_itps_ctm/ctm.cpp:213-264) up to the
  // operator: X with <op12> = sum op12[a,b,c,d] X[a,c,b,d]
  DT<T> bond_X_h(const DT<T>& C1, const DT<T>& C2, const DT<T>& C3, const DT<T>& C4, const DT<T>& eT1,
                 const DT<T>& eT2, const DT<T>& eT3, const DT<T>& eT4, const DT<T>& eT5, const DT<T>& eT6,
                 const DT<T>& T1, const DT<T>& T2) {
    DT<T> A = td(eT5, td(C1, td(C4, eT6, {1}, {0}), {0}, {1}), {1}, {1});
    A = td(bra(T1), A, {0, 3}, {5, 2}, true, false);
    A = td(T1, A, {0, 3}, {6, 4});
    A = td(eT1, A, {0, 2, 3}, {7, 0, 3});
    DT<T> B = td(eT4, td(C2, td(C3, eT3, {0}, {1}), {1}, {1}), {0}, {1});
    B = td(bra(T2), B, {2, 3}, {5, 2}, true, false);
    B = td(T2, B, {2, 3}, {6, 4});
    B = td(eT2, B, {1, 2, 3}, {7, 1, 4});
    return td(A, B, {0, 1, 3, 5}, {0, 1, 3, 5});
  }
  T two_sites_h(const DT<T>& C1, const DT<T>& C2, const DT<T>& C3, const DT<T>& C4, const DT<T>& eT1,
                const DT<T>& eT2, const DT<T>& eT3, const DT<T>& eT4, const DT<T>& eT5, const DT<T>& eT6,
                const DT<T>& T1, const DT<T>& T2, const DT<T>& op12) {
    const DT<T> X = bond_X_h(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, T1, T2);
    if (density) return density_op12(X, op12);
    return scalar(td(op12, X, {0, 1, 2, 3}, {0, 2, 1, 3}));
  }

  // Contract_two_sites_vertical_op12_iTPS_CTM (contract_itps_ctm/ctm.cpp:266-319) up to the
  // operator, as bond_X_h
  DT<T> bond_X_v(const DT<T>& C1, const DT<T>& C2, const DT<T>& C3, const DT<T>& C4, const DT<T>& eT1,
                 const DT<T>& eT2, const DT<T>& eT3, const DT<T>& eT4, const DT<T>& eT5, const DT<T>& eT6,
                 const DT<T>& T1, const DT<T>& T2) {
    DT<T> A = td(eT6, td(C1, td(C2, eT1, {0}, {1}), {1}, {1}), {1}, {0});
    A = td(bra(T1), A, {0, 1}, {2, 5}, true, false);
    A = td(T1, A, {0, 1}, {4, 6});
    A = td(eT2, A, {0, 2, 3}, {7, 0, 3});
    DT<T> B = td(eT5, td(C3, td(C4, eT4, {0}, {1}), {1}, {1}), {0}, {1});
    B = td(bra(T2), B, {0, 3}, {2, 5}, true, false);
    B = td(T2, B, {0, 3}, {4, 6});
    B = td(eT3, B, {1, 2, 3}, {7, 1, 4});
    return td(A, B, {0, 1, 3, 5}, {0, 1, 3, 5});
  }
  T two_sites_v(const DT<T>& C1, const DT<T>& C2, const DT<T>& C3, const DT<T>& C4, const DT<T>& eT1,
                const DT<T>& eT2, const DT<T>& eT3, const DT<T>& eT4, const DT<T>& eT5, const DT<T>& eT6,
                const DT<T>& T1, const DT<T>& T2, const DT<T>& op12) {
    const DT<T> X = bond_X_v(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, T1, T2);
    if (density) return density_op12(X, op12);
    return scalar(td(op12, X, {0, 1, 2, 3}, {0, 2, 1, 3}));
  }

  // An iTPO bond: with the single-layer bra the X of bond_X_h / bond_X_v
  // keeps each site's merged physical pair (p,q) open (its other leg has
  // dimension 1), so X read as R[(p1,q1), (p2,q2)] is the environment of the
  // two density tensors and <op12> = sum op12[p1,p2,q1,q2] R -- the
  // contraction of Contract_two_sites_{horizontal,vertical}_op12_density_CTM
  // (contract_density_ctm/ctm.cpp:196-274)
  T density_op12(const DT<T>& X, const DT<T>& op12) {
    const int64_t n1 = op12.dim(0) * op12.dim(2), n2 = op12.dim(1) * op12.dim(3);
    if (X.dim(0) * X.dim(1) != n1 || X.dim(2) * X.dim(3) != n2) fail(TG_E_INPUT, "op12 does not match the bond");
    return scalar(td(reshape(X, {n1, n2}), reshape(tr(op12, {0, 2, 1, 3}), {n1, n2}), {0, 1}, {0, 1}));
  }

  // twosite_obs.cpp:186-222: nearest-neighbour op12 with the source/target
  // orientation rule
  void measure_bond_op12(int source, int dx, int dy, const double* op, double* out) override {
    require_env();
    check_site(source);
    if (std::abs(dx) + std::abs(dy) != 1) fail(TG_E_INPUT, "op12 bond must be a nearest-neighbour bond");
    const int target = lat.other(source, dx, dy);
    const int64_t d1 = lat.pdim[source], d2 = lat.pdim[target];
    T v;
    auto swapped = [&](int64_t a, int64_t b) {
      // transpose(op, {1,0,3,2}) on the host
      std::vector<double> h(static_cast<size_t>(a * b * a * b * NW));
      for (int64_t i = 0; i < b; ++i)
        for (int64_t j = 0; j < a; ++j)
          for (int64_t k = 0; k < b; ++k)
            for (int64_t l = 0; l < a; ++l) {
              const int64_t src = ((j * b + i) * a + l) * b + k;
              const int64_t dst = ((i * a + j) * b + k) * a + l;
              for (int w = 0; w < NW; ++w) h[static_cast<size_t>(dst * NW + w)] = op[src * NW + w];
            }
      return from_host({b, a, b, a}, h.data());
    };
    if (dy == 0) {
      const int source_col = dx >= 0 ? 0 : 1;
      const int left = lat.other(source, -source_col, 0), right = lat.other(source, 1 - source_col, 0);
      DT<T> o = (left == source) ? from_host({d1, d2, d1, d2}, op) : swapped(d1, d2);
      v = two_sites_h(C[0][left], C[1][right], C[2][right], C[3][left], E[0][left], E[0][right], E[1][right],
                      E[2][right], E[2][left], E[3][left], Tn[left], Tn[right], o);
    } else {
      const int source_row = dy >= 0 ? 1 : 0;
      const int top = lat.other(source, 0, source_row), bottom = lat.other(source, 0, source_row - 1);
      DT<T> o = (top == source) ? from_host({d1, d2, d1, d2}, op) : swapped(d1, d2);
      v = two_sites_v(C[0][top], C[1][top], C[2][bottom], C[3][bottom], E[0][top], E[1][top], E[1][bottom],
                      E[2][bottom], E[3][bottom], E[3][top], Tn[top], Tn[bottom], o);
    }
    std::memcpy(out, &v, sizeof(T));
    if constexpr (!CPLX) out[1] = 0.0;
  }

  // The two-site reduced density matrix of a nearest-neighbour bond,
  // unnormalised, legs (source, target, source', target'): every op12 of
  // twosite_obs.cpp:186-222 measures as sum op12 * rdm, the norm as
  // sum_ab rdm[a,b,a,b] -- one contraction of the bond for any number of
  // operators.
  void measure_bond_rdm(int source, int dx, int dy, double* out) override {
    require_env();
    check_site(source);
    if (std::abs(dx) + std::abs(dy) != 1) fail(TG_E_INPUT, "bond must be a nearest-neighbour bond");
    DT<T> X;
    bool source_first;
    if (dy == 0) {
      const int source_col = dx >= 0 ? 0 : 1;
      const int left = lat.other(source, -source_col, 0), right = lat.other(source, 1 - source_col, 0);
      X = bond_X_h(C[0][left], C[1][right], C[2][right], C[3][left], E[0][left], E[0][right], E[1][right],
                   E[2][right], E[2][left], E[3][left], Tn[left], Tn[right]);
      source_first = left == source;
    } else {
      const int source_row = dy >= 0 ? 1 : 0;
      const int top = lat.other(source, 0, source_row), bottom = lat.other(source, 0, source_row - 1);
      X = bond_X_v(C[0][top], C[1][top], C[2][bottom], C[3][bottom], E[0][top], E[1][top], E[1][bottom],
                   E[2][bottom], E[3][bottom], E[3][top], Tn[top], Tn[bottom]);
      source_first = top == source;
    }
    // X[a,c,b,d] with (a,c) the first site's legs: rdm_first[a,b,c,d] = X[a,c,b,d]; with the
    // source second, rdm_source[b,a,d,c] = X[a,c,b,d]
    if (density) {
      // an iTPO: R[(p_s,q_s), (p_t,q_t)], <op12> = sum op12[p_s,p_t,q_s,q_t] R (density_op12)
      const DT<T> R = reshape(X, {X.dim(0) * X.dim(1), X.dim(2) * X.dim(3)});
      download(source_first ? R : tr(R, {1, 0}), out);
      return;
    }
    download(tr(X, source_first ? V{0, 2, 1, 3} : V{2, 0, 3, 1}), out);
  }

  // ------------------------------------------------ correlations (strip)
  // StartCorrelation_iTPS_CTM (contract_itps_ctm/correlation.cpp:30-57):
  // the strip state, legs (e1r, e3r, n1r, n2r)
  DT<T> corr_start(const DT<T>& C1, const DT<T>& C4, const DT<T>& eT1, const DT<T>& eT3, const DT<T>& eT4,
                   const DT<T>& Tn1, const DT<T>& op) {
    DT<T> X = td(eT3, td(C1, td(C4, eT4, {1}, {0}), {0}, {1}), {1}, {1});
    X = td(td(bra(Tn1), op, {4}, {1}, true, false), X, {0, 3}, {5, 2});
    X = td(Tn1, X, {0, 3, 4}, {6, 4, 2});
    return tr(td(eT1, X, {0, 2, 3}, {5, 0, 2}), {0, 3, 1, 2});
  }
  // Transfer_iTPS_CTM (correlation.cpp:59-77)
  DT<T> corr_transfer(const DT<T>& A, const DT<T>& eT1, const DT<T>& eT3, const DT<T>& Tn1) {
    DT<T> X = td(bra(Tn1), td(A, eT3, {1}, {1}), {0, 3}, {2, 5}, true, false);
    X = td(Tn1, X, {0, 3, 4}, {4, 6, 2});
    return tr(td(eT1, X, {0, 2, 3}, {4, 0, 2}), {0, 3, 1, 2});
  }
  // FinishCorrelation_iTPS_CTM (correlation.cpp:79-104)
  T corr_finish(const DT<T>& A, const DT<T>& C2, const DT<T>& C3, const DT<T>& eT1, const DT<T>& eT2,
                const DT<T>& eT3, const DT<T>& Tn1, const DT<T>& op) {
    DT<T> X = td(eT3, td(C2, td(C3, eT2, {0}, {1}), {1}, {1}), {0}, {1});
    X = td(bra(Tn1), X, {2, 3}, {5, 2}, true, false);
    X = td(td(A, eT1, {0}, {0}), X, {0, 2, 3, 5}, {3, 0, 5, 1});
    X = td(Tn1, X, {0, 1, 2, 3}, {0, 1, 4, 3});
    return scalar(td(op, X, {0, 1}, {0, 1}));
  }
  static std::complex<double> as_complex(const T& v) {
    if constexpr (CPLX) return {v.x, v.y};
    else return {v, 0.0};
  }
  DT<T> identity_op(int site) {
    const int64_t d = lat.pdim[site];
    std::vector<double> h(static_cast<size_t>(d * d * NW), 0.0);
    for (int64_t k = 0; k < d; ++k) h[static_cast<size_t>((k * d + k) * NW)] = 1.0;
    return from_host({d, d}, h.data());
  }

  // measure_correlation_ctm's strip for one left site and direction
  // (correlation_function.cpp:70-212): <O_left O_right> / <1> at distances
  // 1..r_max to the right (dir 0) or up (dir 1).  right_ops holds, site by
  // site over the unit cell, nright d x d operators of that site.
  void measure_correlation(int left, int dir, int r_max, const double* left_op, int nright, const double* right_ops,
                           double* out) override {
    require_env();
    check_site(left);
    if (dir != 0 && dir != 1) fail(TG_E_INPUT, "correlation direction must be 0 (right) or 1 (up)");
    if (r_max < 1 || nright < 1) fail(TG_E_INPUT, "r_max and the number of right operators must be positive");
    std::vector<int64_t> off(static_cast<size_t>(lat.N + 1), 0);
    for (int i = 0; i < lat.N; ++i)
      off[static_cast<size_t>(i + 1)] = off[static_cast<size_t>(i)] + static_cast<int64_t>(nright) * lat.pdim[i] * lat.pdim[i] * NW;
    static const V vrot = {3, 0, 1, 2, 4};
    if (density) prepare_rotations();  // Ts
    // the site tensor an operator enters with, rotated for the vertical
    // strip: Tn with op, or for an iTPO the traced tensor with [[1]]
    // (StartCorrelation / FinishCorrelation_density_CTM, correlation.cpp:33-98)
    auto with_op = [&](int site, const DT<T>& op, DT<T>& k, DT<T>& o) {
      k = density ? traced(site, op) : Tn[site];
      if (dir == 1) k = tr(k, vrot);
      o = density ? one1 : op;
    };
    // the tensor a transfer step absorbs (Transfer_density_CTM takes Ts)
    auto plain = [&](int site) { return dir == 0 ? mt(site) : tr(mt(site), vrot); };
    const int64_t dl = lat.pdim[left];
    const DT<T> lop = from_host({dl, dl}, left_op);
    const DT<T> lid = identity_op(left);
    DT<T> A, An, k, o;
    if (dir == 0) {
      with_op(left, lop, k, o);
      A = corr_start(C[0][left], C[3][left], E[0][left], E[2][left], E[3][left], k, o);
      with_op(left, lid, k, o);
      An = corr_start(C[0][left], C[3][left], E[0][left], E[2][left], E[3][left], k, o);
    } else {
      with_op(left, lop, k, o);
      A = corr_start(C[3][left], C[2][left], E[3][left], E[1][left], E[2][left], k, o);
      with_op(left, lid, k, o);
      An = corr_start(C[3][left], C[2][left], E[3][left], E[1][left], E[2][left], k, o);
    }
    int site = left;
    for (int r = 0; r < r_max; ++r) {
      site = dir == 0 ? lat.right(site) : lat.top(site);
      auto fin = [&](const DT<T>& S, const DT<T>& op) {
        DT<T> kk, oo;
        with_op(site, op, kk, oo);
        return dir == 0 ? corr_finish(S, C[1][site], C[2][site], E[0][site], E[1][site], E[2][site], kk, oo)
                        : corr_finish(S, C[0][site], C[1][site], E[3][site], E[0][site], E[1][site], kk, oo);
      };
      const std::complex<double> nrm = as_complex(fin(An, identity_op(site)));
      const int64_t d = lat.pdim[site];
      for (int q = 0; q < nright; ++q) {
        const DT<T> rop = from_host({d, d}, right_ops + off[static_cast<size_t>(site)] + q * d * d * NW);
        const std::complex<double> v = as_complex(fin(A, rop)) / nrm;
        out[2 * (r * nright + q)] = v.real();
        out[2 * (r * nright + q) + 1] = v.imag();
      }
      if (r + 1 < r_max) {
        const DT<T> tn = plain(site);
        if (dir == 0) {
          A = corr_transfer(A, E[0][site], E[2][site], tn);
          An = corr_transfer(An, E[0][site], E[2][site], tn);
        } else {
          A = corr_transfer(A, E[3][site], E[1][site], tn);
          An = corr_transfer(An, E[3][site], E[1][site], tn);
        }
      }
    }
  }

  // ------------------------------------------------- N x M window <op...>
  static V moved_to_end(int rank, int pos, int cnt) {  // legs pos..pos+cnt-1 to the end
    V p;
    for (int i = 0; i < rank; ++i)
      if (i < pos || i >= pos + cnt) p.push_back(i);
    for (int i = 0; i < cnt; ++i) p.push_back(pos + i);
    return p;
  }
  static V moved_from_end(int rank, int pos, int cnt) {  // inverse of moved_to_end
    V p;
    const int keep = rank - cnt;
    for (int i = 0; i < rank; ++i) {
      if (i < pos) p.push_back(i);
      else if (i < pos + cnt) p.push_back(keep + (i - pos));
      else p.push_back(i - cnt);
    }
    return p;
  }

  // Contract_RxC_iTPS_CTM (contract_itps_ctm/ctm.cpp:45-87, ctm_RxC.cpp) for
  // the window whose source site sits at (source_row, source_col), row 0 on
  // top; ops[r*ncol + c] is the operator of that site (empty = identity),
  // applied as sum_{p,q} Tn[..p] op[p,q] conj(Tn[..q]).  Contracted row by
  // row through a boundary tensor (a, k0, kb0, ..., r).
  T window(int source, int nrow, int ncol, int source_row, int source_col, const std::vector<DT<T>>& ops) {
    if (nrow < 1 || ncol < 1 || nrow > 4 || ncol > 4) fail(TG_E_INPUT, "window must be 1..4 x 1..4");
    std::vector<std::vector<int>> idx(nrow, std::vector<int>(ncol));
    for (int r = 0; r < nrow; ++r)
      for (int c = 0; c < ncol; ++c) idx[r][c] = lat.other(source, c - source_col, source_row - r);
    DT<T> B = C[0][idx[0][0]];
    for (int c = 0; c < ncol; ++c) {
      B = td(B, E[0][idx[0][c]], {B.rank() - 1}, {0});  // (..., b', k, kb)
      B = tr(B, moved_to_end(B.rank(), B.rank() - 3, 1));
    }
    B = td(B, C[1][idx[0][ncol - 1]], {B.rank() - 1}, {0});
    for (int r = 0; r < nrow; ++r) {
      B = td(E[3][idx[r][0]], B, {1}, {0});  // (a', y, yb, k0, kb0, ..., r)
      for (int c = 0; c < ncol; ++c) {
        // an iTPO site enters with its operator (or the identity) traced in
        const DT<T>& o = ops[static_cast<size_t>(r * ncol + c)];
        const DT<T> Tk = density ? traced(idx[r][c], o.empty() ? identity_op(idx[r][c]) : o) : Tn[idx[r][c]];
        const int pos = 1 + 2 * c;
        B = tr(B, moved_to_end(B.rank(), pos, 4));  // (..., y, yb, k, kb)
        int n = B.rank();
        B = td(B, Tk, {n - 4, n - 2}, {0, 1});  // (..., yb, kb, y', z, p)
        if (!o.empty() && !density) B = td(B, o, {B.rank() - 1}, {0});
        n = B.rank();
        B = td(B, bra(Tk), {n - 5, n - 4, n - 1}, {0, 1, 4}, false, true);  // (..., y', z, yb', zb)
        n = B.rank();
        V p;
        for (int i = 0; i < n - 4; ++i) p.push_back(i);
        p.insert(p.end(), {n - 3, n - 1, n - 4, n - 2});  // (..., z, zb, y', yb')
        B = tr(B, p);
        B = tr(B, moved_from_end(B.rank(), pos, 4));
      }
      const int n = B.rank();
      B = td(B, E[1][idx[r][ncol - 1]], {n - 1, n - 3, n - 2}, {0, 2, 3});  // (a', z..., r')
    }
    DT<T> X = td(C[3][idx[nrow - 1][0]], B, {1}, {0});
    for (int c = 0; c < ncol; ++c) X = td(E[2][idx[nrow - 1][c]], X, {1, 2, 3}, {0, 1, 2});
    return scalar(td(X, C[2][idx[nrow - 1][ncol - 1]], {0, X.rank() - 1}, {1, 0}));
  }

  void measure_window(int source, int nrow, int ncol, int source_row, int source_col, int nops,
                      const int* op_row, const int* op_col, const double* ops, double* out) override {
    require_env();
    check_site(source);
    if (nrow < 1 || ncol < 1 || nrow > 4 || ncol > 4) fail(TG_E_INPUT, "window must be 1..4 x 1..4");
    if (source_row < 0 || source_row >= nrow || source_col < 0 || source_col >= ncol)
      fail(TG_E_INPUT, "source position outside the window");
    std::vector<DT<T>> grid(static_cast<size_t>(nrow * ncol));
    int64_t off = 0;
    for (int i = 0; i < nops; ++i) {
      const int r = op_row[i], c = op_col[i];
      if (r < 0 || r >= nrow || c < 0 || c >= ncol) fail(TG_E_INPUT, "operator position outside the window");
      const int site = lat.other(source, c - source_col, source_row - r);
      const int64_t d = lat.pdim[site];
      grid[static_cast<size_t>(r * ncol + c)] = from_host({d, d}, ops + off * NW);
      off += d * d;
    }
    T v = window(source, nrow, ncol, source_row, source_col, grid);
    std::memcpy(out, &v, sizeof(T));
    if constexpr (!CPLX) out[1] = 0.0;
  }

  // ----------------------------------------- transfer matrix eigenvalues
  // TransferMatrix_ctm::matvec_horizontal / matvec_vertical
  // (transfer_matrix.cpp:187-308) on a batch of vectors v (chi, chi, nb).
  DT<T> tm_apply(int dir, int fixed, DT<T> v) {
    if (dir == 0) {
      for (int x = 0; x < lat.LX; ++x) {
        const int site = lat.index(x, fixed);
        v = td(E[0][site], td(E[2][lat.top(site)], v, {1}, {1}), {0, 2, 3}, {3, 1, 2});
      }
    } else {
      int x = fixed;
      const int x0 = fixed;
      do {
        for (int y = 0; y < lat.LY; ++y) {
          const int site = lat.index(x, y);
          v = td(E[3][site], td(E[1][lat.left(site)], v, {1}, {1}), {0, 2, 3}, {3, 1, 2});
        }
        x = (x + lat.skew + lat.LX) % lat.LX;
      } while (x != x0);
    }
    return v;
  }

  // Xgeev of a column-major complex n x n matrix given on the host; when
  // vr_last is given it receives the last component of each right eigenvector
  std::vector<cplx> geev_host_matrix(const std::vector<cplx>& a, int64_t n, std::vector<cplx>* vr_last) {
    DT<cplx> A({n, n}, st), W({n}, st), VR({vr_last ? n * n : 1}, st);
    TG_CUDA(cudaMemcpyAsync(A.p, a.data(), sizeof(cplx) * n * n, cudaMemcpyHostToDevice, st));
    cusolverDnParams_t prm;
    check_sol(cusolverDnCreateParams(&prm), "cusolverDnCreateParams");
    size_t dws = 0, hws = 0;
    const cusolverEigMode_t jr = vr_last ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
    check_sol(cusolverDnXgeev_bufferSize(hsol(), prm, CUSOLVER_EIG_MODE_NOVECTOR, jr, n, CUDA_C_64F, A.p, n, CUDA_C_64F,
                                         W.p, CUDA_C_64F, nullptr, 1, CUDA_C_64F, VR.p, vr_last ? n : 1,
                                         CUDA_C_64F, &dws, &hws),
              "Xgeev_bufferSize");
    DT<unsigned char> dw({static_cast<int64_t>(std::max<size_t>(dws, 1))}, st);
    std::vector<unsigned char> hw(std::max<size_t>(hws, 1));
    ProfScope ps(PK_SOLVER, st, 10.0 * n * n * n, 0.0);
    check_sol(cusolverDnXgeev(hsol(), prm, CUSOLVER_EIG_MODE_NOVECTOR, jr, n, CUDA_C_64F, A.p, n, CUDA_C_64F, W.p,
                              CUDA_C_64F, nullptr, 1, CUDA_C_64F, VR.p, vr_last ? n : 1, CUDA_C_64F, dw.p, dws,
                              hw.data(), hws, info_slot()),
              "Xgeev");
    cusolverDnDestroyParams(prm);
    std::vector<cplx> w(static_cast<size_t>(n));
    TG_CUDA(cudaMemcpyAsync(w.data(), W.p, sizeof(cplx) * n, cudaMemcpyDeviceToHost, st));
    if (vr_last) {
      std::vector<cplx> vr(static_cast<size_t>(n * n));
      TG_CUDA(cudaMemcpyAsync(vr.data(), VR.p, sizeof(cplx) * n * n, cudaMemcpyDeviceToHost, st));
      TG_CUDA(cudaStreamSynchronize(st));
      vr_last->assign(static_cast<size_t>(n), cplx{});
      for (int64_t i = 0; i < n; ++i) (*vr_last)[static_cast<size_t>(i)] = vr[static_cast<size_t>(n - 1 + i * n)];
    }
    check_infos();
    return w;
  }

  // eigen() of src/tensor.cpp:91-112: the nev eigenvalues of largest modulus
  static std::vector<size_t> largest(const std::vector<cplx>& w, size_t nev) {
    std::vector<size_t> order(w.size());
    std::iota(order.begin(), order.end(), 0);
    auto a2 = [&](size_t i) { return w[i].x * w[i].x + w[i].y * w[i].y; };
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return a2(a) > a2(b); });
    order.resize(std::min(nev, order.size()));
    return order;
  }

  // Extent of leg `leg` (0 or 1) of an environment tensor (chi, chi, D, D)
  // that carries nonzero entries.  The environment is kept at the static
  // size chi with exact zeros beyond each projector's cut; the reference
  // stores the cut-sized tensors, so this is its shape()[leg].
  int64_t used_extent(const DT<T>& e, int leg) {
    std::vector<T> h(static_cast<size_t>(e.size()));
    TG_CUDA(cudaMemcpyAsync(h.data(), e.p, sizeof(T) * h.size(), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    const int64_t n0 = e.dim(0), n1 = e.dim(1), inner = e.size() / (n0 * n1);
    int64_t used = 0;
    for (int64_t i = 0; i < n0; ++i)
      for (int64_t j = 0; j < n1; ++j)
        for (int64_t k = 0; k < inner; ++k)
          if (!is_zero(h[static_cast<size_t>((i * n1 + j) * inner + k)])) {
            used = std::max(used, (leg == 0 ? i : j) + 1);
            break;
          }
    return used;
  }
  static bool is_zero(double v) { return v == 0.0; }
  static bool is_zero(cplx v) { return v.x == 0.0 && v.y == 0.0; }

  // TransferMatrix::eigenvalues (transfer_matrix.cpp:84-142) with the
  // Arnoldi of arnoldi.cpp:45-181 (classical Gram-Schmidt applied twice;
  // the Krylov space and its Ritz values are those of the reference's
  // modified Gram-Schmidt).  The matrix dimension N (dim(), which picks the
  // N = 1 shortcut, the dense solver for N <= maxdim_dense and the Krylov
  // size) is the product of the used extents of the boundary legs; the
  // zero-padded remainder of the chi x chi space is an invariant null block.
  void tm_eigenvalues(int dir, int fixed, int num_eigvals, int maxdim_dense, int maxdim, int restartdim,
                      int maxiter, double rtol, double* out, int* nev_out) override {
    require_env();
    if (dir != 0 && dir != 1) fail(TG_E_INPUT, "direction must be 0 (+x) or 1 (+y)");
    if (fixed < 0 || fixed >= (dir == 0 ? lat.LY : lat.LX)) fail(TG_E_INPUT, "fixed coordinate out of range");
    const int64_t chi = P.chi, Npad = chi * chi;
    const int s0 = dir == 0 ? lat.index(0, fixed) : lat.index(fixed, 0);
    const int64_t ea = dir == 0 ? used_extent(E[0][s0], 0) : used_extent(E[3][s0], 0);
    const int64_t eb = dir == 0 ? used_extent(E[2][lat.top(s0)], 1) : used_extent(E[1][lat.left(s0)], 1);
    const int64_t N = ea * eb;
    if (N == 0) fail(TG_E_RUNTIME, "transfer matrix: boundary tensors are zero");
    const int64_t nev = std::min<int64_t>(num_eigvals, N);
    std::vector<cplx> ev;
    if (N == 1) {
      ev.push_back(make_double2(1.0, 0.0));
    } else if (N <= maxdim_dense) {
      // T applied to the unit vectors of the used block, rows of the block kept
      std::vector<T> basis(static_cast<size_t>(Npad * N));
      std::memset(basis.data(), 0, sizeof(T) * basis.size());
      for (int64_t i = 0; i < ea; ++i)
        for (int64_t j = 0; j < eb; ++j) set_real(basis[static_cast<size_t>((i * chi + j) * N + i * eb + j)], 1.0);
      DT<T> I({chi, chi, N}, st);
      TG_CUDA(cudaMemcpyAsync(I.p, basis.data(), sizeof(T) * basis.size(), cudaMemcpyHostToDevice, st));
      DT<T> Mt = tm_apply(dir, fixed, I);  // (chi, chi, N): column c = T e_c
      std::vector<T> full(static_cast<size_t>(Npad * N));
      TG_CUDA(cudaMemcpyAsync(full.data(), Mt.p, sizeof(T) * full.size(), cudaMemcpyDeviceToHost, st));
      TG_CUDA(cudaStreamSynchronize(st));
      std::vector<cplx> a(static_cast<size_t>(N * N));
      for (int64_t i = 0; i < ea; ++i)
        for (int64_t j = 0; j < eb; ++j)
          for (int64_t c = 0; c < N; ++c) {
            const T v = full[static_cast<size_t>((i * chi + j) * N + c)];
            cplx z;
            if constexpr (CPLX) z = v; else z = make_double2(v, 0.0);
            a[static_cast<size_t>((i * eb + j) + c * N)] = z;  // column-major
          }
      std::vector<cplx> w = geev_host_matrix(a, N, nullptr);
      for (size_t i : largest(w, static_cast<size_t>(nev))) ev.push_back(w[i]);
    } else {
      ev = arnoldi(dir, fixed, static_cast<size_t>(nev), maxdim, restartdim, maxiter, rtol, Npad, N);
    }
    for (size_t i = 0; i < ev.size(); ++i) {
      out[2 * i] = ev[i].x;
      out[2 * i + 1] = ev[i].y;
    }
    if (nev_out) *nev_out = static_cast<int>(ev.size());
  }

  std::vector<cplx> hess_eigs(const std::vector<T>& H, int ldh, int64_t k, std::vector<cplx>* last) {
    std::vector<cplx> a(static_cast<size_t>(k * k));
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) {
        const T v = H[static_cast<size_t>(i * ldh + j)];
        cplx z;
        if constexpr (CPLX) z = v; else z = make_double2(v, 0.0);
        a[static_cast<size_t>(i + j * k)] = z;
      }
    return geev_host_matrix(a, k, last);
  }

  // N: length of the (zero-padded) vectors; n_used: the matrix dimension
  // of the reference, which bounds the Krylov size
  std::vector<cplx> arnoldi(int dir, int fixed, size_t nev, int maxvec_in, int mindim, int maxiter, double rtol,
                            int64_t N, int64_t n_used) {
    int64_t maxvec = maxvec_in;
    if (n_used < maxvec) {
      maxvec = n_used;
      maxiter = 1;
    }
    if (mindim < static_cast<int>(nev)) mindim = static_cast<int>(nev);
    const int ldh = static_cast<int>(maxvec);
    std::vector<T> H(static_cast<size_t>((maxvec + 1) * maxvec));
    std::memset(H.data(), 0, sizeof(T) * H.size());
    DT<T> Q = zeros<T>({maxvec + 1, N}, st);  // row j = Krylov vector j
    // initial vector: C1[site] . C4[top(site)] (dir 0) or C4[site] . C3[left(site)]
    // (transfer_matrix.cpp:161-185)
    {
      DT<T> v0;
      if (dir == 0) {
        const int site = lat.index(0, fixed);
        v0 = td(C[0][site], C[3][lat.top(site)], {0}, {1});
      } else {
        const int site = lat.index(fixed, 0);
        v0 = td(C[3][site], C[2][lat.left(site)], {0}, {1});
      }
      TG_CUDA(cudaMemcpyAsync(Q.p, v0.p, sizeof(T) * N, cudaMemcpyDeviceToDevice, st));
    }
    auto row = [&](int64_t j) { return Q.p + j * N; };
    // h[0..k) = Q[:k] q_k (conj), q_k -= Q[:k]^T h  -- twice; then normalise
    auto orthonormalize = [&](int64_t k) {
      PrecScope fp64(this, 0);
      std::vector<T> hacc(static_cast<size_t>(std::max<int64_t>(k, 1)));
      std::memset(hacc.data(), 0, sizeof(T) * hacc.size());
      for (int pass = 0; pass < (k > 0 ? 2 : 0); ++pass) {
        DT<T> h({k, 1}, st);
        MV qh{Q.p, k, N, N, 1, true};  // conj(Q[:k]) as k x N
        mm(qh, MV{row(k), N, 1, 1, N, false}, h.p, 1, 1);
        DT<T> proj({N, 1}, st);
        mm(MV{Q.p, N, k, 1, N, false}, MV{h.p, k, 1, 1, k, false}, proj.p, 1, 1);  // Q[:k]^T h
        axpy_neg(row(k), proj.p, N);
        std::vector<T> hh(static_cast<size_t>(k));
        TG_CUDA(cudaMemcpyAsync(hh.data(), h.p, sizeof(T) * k, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
        for (int64_t j = 0; j < k; ++j) add_to(hacc[static_cast<size_t>(j)], hh[static_cast<size_t>(j)]);
      }
      for (int64_t j = 0; j < k; ++j) H[static_cast<size_t>(j * ldh + (k - 1))] = hacc[static_cast<size_t>(j)];
      const double nrm = norm2(row(k), N);
      if (!(nrm > 0.0)) fail(TG_E_RUNTIME, "Arnoldi: Krylov space exhausted (zero vector)");
      scale<T>(row(k), N, 1.0 / nrm, st);
      if (k > 0) set_real(H[static_cast<size_t>(k * ldh + (k - 1))], nrm);
    };
    auto apply = [&](int64_t k) {  // q_k = T q_{k-1}
      DT<T> v({chi_(), chi_(), 1}, st);
      TG_CUDA(cudaMemcpyAsync(v.p, row(k - 1), sizeof(T) * N, cudaMemcpyDeviceToDevice, st));
      DT<T> w = tm_apply(dir, fixed, v);
      TG_CUDA(cudaMemcpyAsync(row(k), w.p, sizeof(T) * N, cudaMemcpyDeviceToDevice, st));
    };
    auto residue = [&](int64_t k) {  // arnoldi.cpp:170-181
      std::vector<cplx> last;
      std::vector<cplx> w = hess_eigs(H, ldh, k, &last);
      std::vector<size_t> ord = largest(w, nev);
      const T hk = H[static_cast<size_t>(k * ldh + (k - 1))];
      double hkr, hki;
      if constexpr (CPLX) { hkr = hk.x; hki = hk.y; } else { hkr = hk; hki = 0.0; }
      std::vector<double> res;
      for (size_t i : ord) {
        const cplx e = last[i];
        const double pr = hkr * e.x - hki * e.y, pi = hkr * e.y + hki * e.x;
        res.push_back(std::hypot(pr, pi) / std::hypot(w[i].x, w[i].y));
      }
      return res;
    };
    orthonormalize(0);
    for (size_t k = 1; k <= nev; ++k) {
      apply(static_cast<int64_t>(k));
      orthonormalize(static_cast<int64_t>(k));
    }
    double res_nev = 1.0;
    for (int iter = 1; iter <= maxiter; ++iter) {
      for (int64_t k = static_cast<int64_t>(nev) + 1; k <= maxvec; ++k) {
        apply(k);
        orthonormalize(k);
        res_nev = residue(k)[nev - 1];
        if (res_nev <= rtol) break;
      }
      if (res_nev <= rtol || iter == maxiter) break;
      restart(Q, H, ldh, maxvec, mindim, N);
    }
    std::vector<cplx> w = hess_eigs(H, ldh, maxvec, nullptr);
    std::vector<cplx> out;
    for (size_t i : largest(w, nev)) out.push_back(w[i]);
    return out;
  }

  // implicitly shifted restart (arnoldi.cpp:117-167): for the k - minvec
  // largest Ritz values sigma, h <- q^H h q with (h - sigma I) = q r, and the
  // basis rotated by q; then tiny entries of h dropped
  void restart(DT<T>& Q, std::vector<T>& H, int ldh, int64_t k, int minvec, int64_t N) {
    std::vector<cplx> w = hess_eigs(H, ldh, k, nullptr);
    std::vector<size_t> ord = largest(w, static_cast<size_t>(k));
    std::vector<cplx> h(static_cast<size_t>(k * k));
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) {
        const T v = H[static_cast<size_t>(i * ldh + j)];
        if constexpr (CPLX) h[static_cast<size_t>(i * k + j)] = v; else h[static_cast<size_t>(i * k + j)] = make_double2(v, 0.0);
      }
    for (int64_t s = 0; s < k - minvec; ++s) {
      cplx sigma = w[ord[static_cast<size_t>(s)]];
      if constexpr (!CPLX) sigma.y = 0.0;  // real_if_real (arnoldi.cpp:113-114)
      std::vector<cplx> q = small_qr_q(h, k, sigma);
      h = cmatmul(cmatmul(q, h, k, true), q, k, false);  // q^H h q
      // Q (rows = vectors) <- q^T Q  i.e. new vector j = sum_i Q_i q[i][j]
      rotate_basis(Q, q, k, N);
    }
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) {
        cplx z = h[static_cast<size_t>(i * k + j)];
        if (z.x * z.x + z.y * z.y < 1e-28) z = make_double2(0.0, 0.0);
        T v;
        if constexpr (CPLX) v = z; else v = z.x;
        H[static_cast<size_t>(i * ldh + j)] = v;
      }
  }

  // Q factor of (h - sigma I) (k x k, row-major, complex) by Householder
  // QR on the host-visible small matrix, computed with cuSOLVER
  std::vector<cplx> small_qr_q(const std::vector<cplx>& h, int64_t k, cplx sigma) {
    std::vector<cplx> a(static_cast<size_t>(k * k));  // column-major
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) {
        cplx z = h[static_cast<size_t>(i * k + j)];
        if (i == j) {
          z.x -= sigma.x;
          z.y -= sigma.y;
        }
        a[static_cast<size_t>(i + j * k)] = z;
      }
    DT<cplx> A({k, k}, st), tau({k}, st);
    TG_CUDA(cudaMemcpyAsync(A.p, a.data(), sizeof(cplx) * k * k, cudaMemcpyHostToDevice, st));
    int lw1 = 0, lw2 = 0;
    auto* ap = reinterpret_cast<cuDoubleComplex*>(A.p);
    auto* tp = reinterpret_cast<cuDoubleComplex*>(tau.p);
    const int ik = static_cast<int>(k);
    check_sol(cusolverDnZgeqrf_bufferSize(hsol(), ik, ik, ap, ik, &lw1), "Zgeqrf_bufferSize");
    check_sol(cusolverDnZungqr_bufferSize(hsol(), ik, ik, ik, ap, ik, tp, &lw2), "Zungqr_bufferSize");
    const int lw = std::max(std::max(lw1, lw2), 1);
    DT<cplx> work({lw}, st);
    auto* wp = reinterpret_cast<cuDoubleComplex*>(work.p);
    check_sol(cusolverDnZgeqrf(hsol(), ik, ik, ap, ik, tp, wp, lw, info_slot()), "Zgeqrf");
    check_sol(cusolverDnZungqr(hsol(), ik, ik, ik, ap, ik, tp, wp, lw, info_slot()), "Zungqr");
    TG_CUDA(cudaMemcpyAsync(a.data(), A.p, sizeof(cplx) * k * k, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    check_infos();
    std::vector<cplx> q(static_cast<size_t>(k * k));  // row-major
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) q[static_cast<size_t>(i * k + j)] = a[static_cast<size_t>(i + j * k)];
    return q;
  }

  static std::vector<cplx> cmatmul(const std::vector<cplx>& a, const std::vector<cplx>& b, int64_t k, bool adj_a) {
    std::vector<cplx> c(static_cast<size_t>(k * k), make_double2(0.0, 0.0));
    for (int64_t i = 0; i < k; ++i)
      for (int64_t l = 0; l < k; ++l) {
        cplx x = adj_a ? a[static_cast<size_t>(l * k + i)] : a[static_cast<size_t>(i * k + l)];
        if (adj_a) x.y = -x.y;
        for (int64_t j = 0; j < k; ++j) {
          const cplx y = b[static_cast<size_t>(l * k + j)];
          c[static_cast<size_t>(i * k + j)].x += x.x * y.x - x.y * y.y;
          c[static_cast<size_t>(i * k + j)].y += x.x * y.y + x.y * y.x;
        }
      }
    return c;
  }

  void rotate_basis(DT<T>& Q, const std::vector<cplx>& q, int64_t k, int64_t N) {
    std::vector<T> qt(static_cast<size_t>(k * k));  // qt[j][i] = q[i][j]
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) {
        const cplx z = q[static_cast<size_t>(i * k + j)];
        T v;
        if constexpr (CPLX) v = z; else v = z.x;
        qt[static_cast<size_t>(j * k + i)] = v;
      }
    DT<T> qd = from_host({k, k}, reinterpret_cast<const double*>(qt.data()));
    DT<T> newQ({k, N}, st);
    PrecScope fp64(this, 0);
    mm(rm(qd.p, k, k), rm(Q.p, k, N), newQ.p, N, 1);
    TG_CUDA(cudaMemcpyAsync(Q.p, newQ.p, sizeof(T) * k * N, cudaMemcpyDeviceToDevice, st));
  }

  int64_t chi_() const { return P.chi; }
  static void add_to(double& a, double b) { a += b; }
  static void add_to(cplx& a, cplx b) {
    a.x += b.x;
    a.y += b.y;
  }
  static void set_real(double& a, double v) { a = v; }
  static void set_real(cplx& a, double v) { a = make_double2(v, 0.0); }
  void axpy_neg(T* y, const T* x, int64_t n) { axpy<T>(y, x, -1.0, n, st); }
  double norm2(const T* x, int64_t n) {
    DT<T> h({1, 1}, st);
    PrecScope fp64(this, 0);
    MV xc{x, 1, n, n, 1, true};
    mm(xc, MV{x, n, 1, 1, n, false}, h.p, 1, 1);
    T v = scalar(h);
    if constexpr (CPLX) return std::sqrt(v.x); else return std::sqrt(v);
  }

  // -------------------------------------------------------- simple update
  void su_onesite(int site, const double* op) override {
    check_site(site);
    if (density) {
      const std::vector<double> k = density_site_op(op, lat.pdim[site]);
      su_onesite_raw(site, k.data());
    } else {
      su_onesite_raw(site, op);
    }
  }
  // Tn = tensordot(Tn, op, Axes(4), Axes(0)) (simple_update.cpp:27-30) with
  // op of the stored last leg
  void su_onesite_raw(int site, const double* op) {
    const int64_t d = tdim(site);
    DT<T> o = from_host({d, d}, op);
    Tn[site] = td(Tn[site], o, {4}, {0});
    rot_ok[site] = false;
    TG_CUDA(cudaStreamSynchronize(st));
  }

  // iTPS::simple_update_density (simple_update.cpp:141-178) on the merged
  // physical pair (p,q) -> p*d+q.  A one-site operator makes
  // Tn'[..,a,c] = sum_{p,q} Tn[..,p,q] op[p,a] conj(op[c,q]); a bond
  // operator acts as mptensor::kron(op, conj(op)), whose legs are
  // (i*d + j) of op's i and conj(op)'s j.
  std::vector<double> density_site_op(const double* op, int64_t d) const {
    std::vector<double> out(static_cast<size_t>(d * d * d * d * NW), 0.0);
    for (int64_t p = 0; p < d; ++p)
      for (int64_t q = 0; q < d; ++q)
        for (int64_t a = 0; a < d; ++a)
          for (int64_t c = 0; c < d; ++c) {
            const double* x = op + (p * d + a) * NW;
            const double* y = op + (c * d + q) * NW;
            const size_t o = static_cast<size_t>(((p * d + q) * d * d + (a * d + c)) * NW);
            cmul_conj(x, y, out.data() + o);
          }
    return out;
  }
  std::vector<double> density_bond_op(const double* op, int64_t d1, int64_t d2) const {
    const int64_t n = d1 * d2 * d1 * d2;
    std::vector<double> out(static_cast<size_t>(n * n * NW), 0.0);
    const int64_t dim[4] = {d1, d2, d1, d2};
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < n; ++j) {
        int64_t ii = i, jj = j, idx = 0;
        int64_t a[4], b[4];
        for (int l = 3; l >= 0; --l) {
          a[l] = ii % dim[l];
          ii /= dim[l];
          b[l] = jj % dim[l];
          jj /= dim[l];
        }
        for (int l = 0; l < 4; ++l) idx = idx * dim[l] * dim[l] + a[l] * dim[l] + b[l];
        cmul_conj(op + i * NW, op + j * NW, out.data() + idx * NW);
      }
    return out;
  }
  // out = x * conj(y) for NW doubles per value
  static void cmul_conj(const double* x, const double* y, double* out) {
    if constexpr (CPLX) {
      out[0] = x[0] * y[0] + x[1] * y[1];
      out[1] = x[1] * y[0] - x[0] * y[1];
    } else {
      out[0] = x[0] * y[0];
    }
  }

  DT<double> dvec(const std::vector<double>& h) {
    DT<double> t({static_cast<int64_t>(h.size())}, st);
    TG_CUDA(cudaMemcpyAsync(t.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));  // h may be a temporary
    return t;
  }

  // multiply leg `ax` of tensor t by v (multiply_vector)
  void mulvec(DT<T>& t, int ax, const std::vector<double>& v) {
    int64_t outer = 1, inner = 1;
    for (int i = 0; i < ax; ++i) outer *= t.dim(i);
    for (int i = ax + 1; i < t.rank(); ++i) inner *= t.dim(i);
    DT<double> dv = dvec(v);
    scale_leg<T>(t.p, outer, t.dim(ax), inner, dv.p, st);
  }

  // the weights: device table <-> host vectors, whichever is newer
  void lam_to_device() {
    if (!lam_dev_stale) return;
    std::vector<double> h(static_cast<size_t>(4 * lat.N * lam_ld), 0.0);
    for (int i = 0; i < lat.N; ++i)
      for (int l = 0; l < 4; ++l)
        std::copy(lambda[i][l].begin(), lambda[i][l].end(), h.begin() + (i * 4 + l) * lam_ld);
    TG_CUDA(cudaMemcpyAsync(d_lam, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));
    lam_dev_stale = false;
  }
  void lam_to_host() {
    if (!lam_host_stale) return;
    std::vector<double> h(static_cast<size_t>(4 * lat.N * lam_ld));
    TG_CUDA(cudaMemcpyAsync(h.data(), d_lam, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    check_infos();
    for (int i = 0; i < lat.N; ++i)
      for (int l = 0; l < 4; ++l)
        std::copy(h.begin() + (i * 4 + l) * lam_ld, h.begin() + (i * 4 + l) * lam_ld + lambda[i][l].size(),
                  lambda[i][l].begin());
    lam_host_stale = false;
  }
  // the device copy of an evolution operator; the cache is emptied only
  // between launches (trim_op_cache), never while a batch holds its pointers
  const DT<T>& device_op(const double* op, int64_t n) {
    std::vector<double> key(op, op + n * NW);
    auto it = op_cache.find(key);
    if (it != op_cache.end()) return it->second;
    DT<T> d = from_host({n}, op);
    return op_cache.emplace(std::move(key), std::move(d)).first->second;
  }
  void trim_op_cache(size_t incoming) {
    if (op_cache.size() + incoming > 256) op_cache.clear();
  }
  // the arguments of the fused bond step, or false when its shapes need the
  // multi-launch path
  bool fused_args(int source, int connect1, const double* op, SuBondArgs& a) {
    const int target = lat.neighbor(source, connect1);
    for (int q = 0; q < 5; ++q) {
      a.dims1[q] = static_cast<int>(Tn[source].dim(q));
      a.dims2[q] = static_cast<int>(Tn[target].dim(q));
    }
    if (!su_bond_fused_supported<T>(a.dims1, a.dims2, connect1, lam_ld)) return false;
    const int64_t nop = static_cast<int64_t>(a.dims1[4]) * a.dims2[4] * a.dims1[4] * a.dims2[4];
    a.tn1 = Tn[source].p;
    a.tn2 = Tn[target].p;
    a.lam = d_lam;
    a.lam_ld = lam_ld;
    a.site1 = source;
    a.site2 = target;
    a.connect1 = connect1;
    a.op = device_op(op, nop).p;
    a.lambda_cut = P.inverse_lambda_cut;
    a.flag = d_su_flag;
    return true;
  }

  // A sequence of simple-update steps in its order (legs[i] < 0: one-site).
  // Consecutive bond steps on pairwise disjoint site pairs commute -- none
  // reads a tensor or a weight that another writes -- so each run of them
  // goes to the device as one launch of one block per bond.
  void su_bonds(int n, const int* sources, const int* legs, const double* const* ops) override {
    if (n < 0) fail(TG_E_INPUT, "negative count");
    std::vector<std::vector<double>> conv;  // an iTPO's operators on the merged physical legs
    std::vector<const double*> cops;
    if (density) {
      conv.resize(static_cast<size_t>(n));
      cops.resize(static_cast<size_t>(n));
      for (int i = 0; i < n; ++i) {
        check_site(sources[i]);
        if (!ops || !ops[i]) fail(TG_E_INPUT, "null operator");
        if (legs[i] > 3) fail(TG_E_INPUT, "source_leg must be -1..3");
        conv[i] = legs[i] < 0 ? density_site_op(ops[i], lat.pdim[sources[i]])
                              : density_bond_op(ops[i], lat.pdim[sources[i]],
                                                lat.pdim[lat.neighbor(sources[i], legs[i])]);
        cops[i] = conv[i].data();
      }
      ops = cops.data();
    }
    trim_op_cache(static_cast<size_t>(n));
    std::vector<SuBondArgs> group;
    std::vector<char> busy(static_cast<size_t>(lat.N), 0);
    auto flush = [&]() {
      if (group.empty()) return;
      lam_to_device();
      su_bonds_fused<T>(group.data(), static_cast<int>(group.size()), st);
      lam_host_stale = true;
      group.clear();
      std::fill(busy.begin(), busy.end(), 0);
    };
    for (int i = 0; i < n; ++i) {
      check_site(sources[i]);
      if (!ops || !ops[i]) fail(TG_E_INPUT, "null operator");
      if (legs[i] < 0) {
        flush();
        su_onesite_raw(sources[i], ops[i]);
        continue;
      }
      if (legs[i] > 3) fail(TG_E_INPUT, "source_leg must be -1..3");
      const int target = lat.neighbor(sources[i], legs[i]);
      SuBondArgs a{};
      if (!fused_args(sources[i], legs[i], ops[i], a)) {
        flush();
        su_bond_raw(sources[i], legs[i], ops[i]);
        continue;
      }
      if (busy[static_cast<size_t>(sources[i])] || busy[static_cast<size_t>(target)] ||
          static_cast<int>(group.size()) == kSuBatchMax)
        flush();
      group.push_back(a);
      busy[static_cast<size_t>(sources[i])] = busy[static_cast<size_t>(target)] = 1;
      rot_ok[sources[i]] = rot_ok[target] = false;
    }
    flush();
  }

  void su_bond(int source, int connect1, const double* op) override {
    check_site(source);
    if (connect1 < 0 || connect1 > 3) fail(TG_E_INPUT, "source_leg must be 0..3");
    if (density) {
      const std::vector<double> k =
          density_bond_op(op, lat.pdim[source], lat.pdim[lat.neighbor(source, connect1)]);
      su_bond_raw(source, connect1, k.data());
    } else {
      su_bond_raw(source, connect1, op);
    }
  }
  // core::Simple_update_bond (core/simple_update.cpp:50-198) with op on the
  // stored last legs
  void su_bond_raw(int source, int connect1, const double* op) {
    const int target = lat.neighbor(source, connect1);
    const int connect2 = (connect1 + 2) % 4;
    {
      // the whole step in one thread block (su_fused.cu), in place
      SuBondArgs a{};
      trim_op_cache(1);
      if (fused_args(source, connect1, op, a)) {
        lam_to_device();
        su_bond_fused<T>(a, st);
        lam_host_stale = true;
        rot_ok[source] = rot_ok[target] = false;
        return;
      }
    }
    lam_to_host();
    lam_dev_stale = true;
    static const int outer[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    static const int to_last[4][5] = {{1, 2, 3, 0, 4}, {0, 2, 3, 1, 4}, {0, 1, 3, 2, 4}, {0, 1, 2, 3, 4}};
    static const int back1[4][5] = {{4, 0, 1, 2, 3}, {0, 4, 1, 2, 3}, {0, 1, 4, 2, 3}, {0, 1, 2, 4, 3}};
    static const int back2[4][5] = {{3, 0, 1, 2, 4}, {0, 3, 1, 2, 4}, {0, 1, 3, 2, 4}, {0, 1, 2, 3, 4}};
    auto& lam1 = lambda[source];
    auto& lam2 = lambda[target];
    auto inv = [&](const std::vector<double>& l) {
      std::vector<double> r(l.size());
      for (size_t j = 0; j < l.size(); ++j) r[j] = l[j] > P.inverse_lambda_cut ? 1.0 / l[j] : 0.0;
      return r;
    };
    const int64_t dc = Tn[source].dim(connect1);
    DT<T> T1 = clone(Tn[source], st);
    for (int a = 0; a < 3; ++a) mulvec(T1, outer[connect1][a], lam1[outer[connect1][a]]);
    T1 = tr(T1, V(to_last[connect1], to_last[connect1] + 5));
    DT<T> T2 = clone(Tn[target], st);
    for (int a = 0; a < 3; ++a) mulvec(T2, outer[connect2][a], lam2[outer[connect2][a]]);
    T2 = tr(T2, V(to_last[connect2], to_last[connect2] + 5));
    DT<T> Q1, R1, Q2, R2;
    const int64_t m1 = T1.dim(0) * T1.dim(1) * T1.dim(2), n1 = T1.dim(3) * T1.dim(4);
    const int64_t m2 = T2.dim(0) * T2.dim(1) * T2.dim(2), n2 = T2.dim(3) * T2.dim(4);
    qr(T1, m1, n1, Q1, R1);
    qr(T2, m2, n2, Q2, R2);
    const int64_t k1 = std::min(m1, n1), k2 = std::min(m2, n2);
    Q1 = reshape(Q1, {T1.dim(0), T1.dim(1), T1.dim(2), k1});
    R1 = reshape(R1, {k1, T1.dim(3), T1.dim(4)});
    Q2 = reshape(Q2, {T2.dim(0), T2.dim(1), T2.dim(2), k2});
    R2 = reshape(R2, {k2, T2.dim(3), T2.dim(4)});
    const int64_t d1 = T1.dim(4), d2 = T2.dim(4);
    DT<T> op12 = from_host({d1, d2, d1, d2}, op);
    DT<T> Theta = td(td(R1, R2, {1}, {1}), op12, {1, 3}, {0, 1});  // (c1, c2, m1o, m2o)
    DT<T> Th = tr(Theta, {0, 2, 1, 3});
    DT<T> U, VT;
    DT<double> s;
    const int64_t rows = k1 * d1, cols = k2 * d2;
    svd(Th, rows, cols, U, s, VT);
    const int64_t kk = std::min(rows, cols);
    std::vector<double> hs(static_cast<size_t>(kk));
    TG_CUDA(cudaMemcpyAsync(hs.data(), s.p, sizeof(double) * kk, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    if (dc > kk) fail(TG_E_RUNTIME, "simple update: bond dimension exceeds the rank of Theta");
    std::vector<double> lc(hs.begin(), hs.begin() + dc);
    double nrm = 0.0;
    for (double x : lc) nrm += x * x;
    nrm = std::sqrt(nrm);
    for (double& x : lc) x = std::sqrt(x / nrm);
    DT<double> dlc = dvec(lc);
    DT<T> Uc({rows, dc}, st);
    scale_cols<T>(U.p, kk, rows, static_cast<int>(dc), dlc.p, false, Uc.p, st);
    DT<T> VTc({dc, cols}, st);
    scale_rows<T>(VT.p, cols, cols, static_cast<int>(dc), dlc.p, false, VTc.p, st);
    Uc = reshape(Uc, {k1, d1, dc});
    VTc = reshape(VTc, {dc, k2, d2});
    auto il1 = lam1, il2 = lam2;
    for (int a = 0; a < 3; ++a) mulvec(Q1, a, inv(lam1[outer[connect1][a]]));
    for (int a = 0; a < 3; ++a) mulvec(Q2, a, inv(lam2[outer[connect2][a]]));
    Tn[source] = tr(td(Q1, Uc, {3}, {0}), V(back1[connect1], back1[connect1] + 5));
    Tn[target] = tr(td(Q2, VTc, {3}, {1}), V(back2[connect2], back2[connect2] + 5));
    lambda[source][connect1] = lc;
    lambda[target][connect2] = lc;
    rot_ok[source] = rot_ok[target] = false;
    check_infos();
  }

  // iTPS::initialize_tensors (src/iTPS/tensors.cpp:38-137): Tn[0,0,0,0,p] =
  // initial_state[p] (random when all zero), every other entry noise*U(-1,1)
  // drawn in first-leg-fastest order from mt19937(seed) (real part) and
  // mt19937(seed*11+137) (imaginary part); lambdas reset to one.
  void init_tensors(int seed, const double* dirs, const int* dir_len, const double* noises) override {
    if (density) {
      // iTPS::initialize_tensors_density (tensors.cpp:140-208): the identity
      // operator, Tn[0,0,0,0,p,p] = 1, on every site; seed, directions and
      // noise are not used
      for (int i = 0; i < lat.N; ++i) {
        const auto& v = lat.vdim[i];
        const int64_t d = lat.pdim[i];
        std::vector<double> h(static_cast<size_t>(Tn[i].size() * NW), 0.0);
        for (int64_t p = 0; p < d; ++p) h[static_cast<size_t>((p * d + p) * NW)] = 1.0;
        upload(Tn[i], h.data());
        rot_ok[i] = false;
        for (int l = 0; l < 4; ++l) lambda[i][l].assign(v[l], 1.0);
      }
      lam_host_stale = false;
      lam_dev_stale = true;
      return;
    }
    std::mt19937 gen(static_cast<unsigned>(seed));
    std::mt19937 gen_im(static_cast<unsigned>(seed * 11 + 137));
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    int off = 0;
    for (int i = 0; i < lat.N; ++i) {
      const auto& v = lat.vdim[i];
      const int pd = lat.pdim[i];
      const size_t ndim = static_cast<size_t>(v[0]) * v[1] * v[2] * v[3] * pd;
      std::vector<double> re(ndim), im(ndim);
      for (size_t j = 0; j < ndim; ++j) {
        re[j] = dist(gen);
        im[j] = dist(gen_im);
      }
      std::vector<double> d(dirs + off, dirs + off + dir_len[i]);
      off += dir_len[i];
      std::vector<double> d_im(pd, 0.0);
      if (std::all_of(d.begin(), d.end(), [](double x) { return x == 0.0; })) {
        d.assign(pd, 0.0);
        for (int j = 0; j < pd; ++j) {
          d[j] = dist(gen);
          d_im[j] = dist(gen_im);
        }
      }
      std::vector<T> h(ndim);
      for (int a = 0; a < v[0]; ++a)
        for (int b = 0; b < v[1]; ++b)
          for (int c = 0; c < v[2]; ++c)
            for (int e = 0; e < v[3]; ++e)
              for (int p = 0; p < pd; ++p) {
                const size_t rm = ((((static_cast<size_t>(a) * v[1] + b) * v[2] + c) * v[3] + e) * pd + p);
                double xr, xi;
                if (a == 0 && b == 0 && c == 0 && e == 0) {
                  xr = p < static_cast<int>(d.size()) ? d[p] : 0.0;
                  xi = d_im[p];
                } else {
                  const size_t nr = a + static_cast<size_t>(b) * v[0] + static_cast<size_t>(c) * v[0] * v[1] +
                                    static_cast<size_t>(e) * v[0] * v[1] * v[2] +
                                    static_cast<size_t>(p) * v[0] * v[1] * v[2] * v[3];
                  xr = noises[i] * re[nr];
                  xi = noises[i] * im[nr];
                }
                if constexpr (CPLX) {
                  h[rm] = make_double2(xr, xi);
                } else {
                  h[rm] = xr;
                }
              }
      upload(Tn[i], reinterpret_cast<const double*>(h.data()));
      rot_ok[i] = false;
      for (int l = 0; l < 4; ++l) lambda[i][l].assign(v[l], 1.0);
    }
    lam_host_stale = false;  // the reset host weights are the current ones
    lam_dev_stale = true;
  }

  // ------------------------------------------------------- full update
  // Eigendecomposition of a Hermitian row-major n x n matrix H (cuSOLVER
  // syevd / heevd): ascending w on the host, Z (n x n, column j the
  // eigenvector of w_j).  Read column-major the buffer is H^T = conj(H), whose
  // eigenvectors are conj(z_j); the column-major eigenvectors read row-major
  // are therefore Z^T (real) or Z^H (complex).
  void eigh(const DT<T>& A, int64_t n, std::vector<double>& w, DT<T>& Z) {
    DT<T> a = clone(A, st);
    DT<double> wd({n}, st);
    const int in = static_cast<int>(n);
    int lwork = 0;
    ProfScope ps(PK_SOLVER, st, (CPLX ? 4.0 : 1.0) * 9.0 * static_cast<double>(n) * n * n, 0.0);
    if constexpr (CPLX) {
      auto* ap = reinterpret_cast<cuDoubleComplex*>(a.p);
      check_sol(cusolverDnZheevd_bufferSize(hsol(), CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, in, ap, in, wd.p,
                                            &lwork),
                "Zheevd_bufferSize");
      DT<T> work({static_cast<int64_t>(std::max(lwork, 1))}, st);
      check_sol(cusolverDnZheevd(hsol(), CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, in, ap, in, wd.p,
                                 reinterpret_cast<cuDoubleComplex*>(work.p), lwork, info_slot()),
                "Zheevd");
      Z = transpose<T>(reshape(a, {n, n}), {1, 0}, st, true);
    } else {
      check_sol(cusolverDnDsyevd_bufferSize(hsol(), CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, in, a.p, in,
                                            wd.p, &lwork),
                "Dsyevd_bufferSize");
      DT<T> work({static_cast<int64_t>(std::max(lwork, 1))}, st);
      check_sol(cusolverDnDsyevd(hsol(), CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, in, a.p, in, wd.p, work.p,
                                 lwork, info_slot()),
                "Dsyevd");
      Z = tr(reshape(a, {n, n}), {1, 0});
    }
    w.resize(static_cast<size_t>(n));
    TG_CUDA(cudaMemcpyAsync(w.data(), wd.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
  }

  // Backend of full_update.hpp on this engine's device tensors: products and
  // permutations through td / tr, QR and SVD through cuSOLVER (qr, svd),
  // leg scaling through scale_leg, slicing as a product with a 0/1 matrix.
  struct FuBackend {
    using Ten = DT<T>;
    using Scalar = std::conditional_t<CPLX, std::complex<double>, double>;
    EngineT* e;
    static const Shape& shape(const Ten& t) { return t.sh; }
    Ten conj(const Ten& a) {
      if constexpr (CPLX) {
        V id(static_cast<size_t>(a.rank()));
        std::iota(id.begin(), id.end(), 0);
        return transpose<T>(a, id, e->st, true);
      } else {
        return a;
      }
    }
    Ten td(const Ten& a, const Ten& b, const V& x, const V& y, int) { return e->td(a, b, x, y); }
    Ten tr(const Ten& a, const V& q) { return e->tr(a, q); }
    Ten reshape(const Ten& a, const Shape& s) { return tg::reshape(a, s); }
    void axpy(Ten& y, const Ten& x, double alpha) { tg::axpy<T>(y.p, x.p, alpha, y.size(), e->st); }
    void scale(Ten& x, double alpha) { tg::scale<T>(x.p, x.size(), alpha, e->st); }
    Scalar scalar(const Ten& t) {
      const T v = e->scalar(t);
      if constexpr (CPLX) return {v.x, v.y};
      else return v;
    }
    void qr_matrix(const Ten& M, Ten& Q, Ten& R) { e->qr(M, M.dim(0), M.dim(1), Q, R); }
    void svd_matrix(const Ten& M, Ten& U, std::vector<double>& s, Ten& VT) {
      Ten A = clone(M, e->st);
      DT<double> sd;
      e->svd(A, M.dim(0), M.dim(1), U, sd, VT);
      s.resize(static_cast<size_t>(sd.size()));
      TG_CUDA(cudaMemcpyAsync(s.data(), sd.p, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, e->st));
      TG_CUDA(cudaStreamSynchronize(e->st));
    }
    void eigh_matrix(const Ten& M, std::vector<double>& w, Ten& Z) { e->eigh(M, M.dim(0), w, Z); }
    Ten mulvec(const Ten& A, const std::vector<double>& v, int leg) {
      Ten o = clone(A, e->st);
      e->mulvec(o, leg, v);
      return o;
    }
    Ten slice(const Ten& A, int leg, int64_t n) {
      const int64_t dim = A.dim(leg);
      if (n == dim) return A;
      std::vector<double> h(static_cast<size_t>(n * dim * NW), 0.0);
      for (int64_t i = 0; i < n; ++i) h[static_cast<size_t>((i * dim + i) * NW)] = 1.0;
      const Ten S = e->from_host({n, dim}, h.data());
      const Ten B = e->td(A, S, {leg}, {1});  // A's other legs, then the n kept entries
      V perm;
      const int r = A.rank();
      for (int i = 0; i < r; ++i) perm.push_back(i < leg ? i : (i == leg ? r - 1 : i - 1));
      return e->tr(B, perm);
    }
  };

  // core::Full_update_bond for the bond (source, leg) with the environment
  // tensors that face it (src/iTPS/full_update.cpp:42-116); the site tensors
  // are replaced, the environment is left to the caller's moves
  void fu_bond(int source, int leg, const double* op, const tg_fu_params* fp, int* iterations,
               int* converged) override {
    if (density) fail(TG_E_INPUT, "the full update is not defined for an iTPO (finite_temperature.cpp runs the simple update only)");
    {
      require_env();
      check_site(source);
      if (leg < 0 || leg > 3) fail(TG_E_INPUT, "source_leg must be 0..3");
      const int t = lat.neighbor(source, leg);
      auto &C1 = C[0], &C2 = C[1], &C3 = C[2], &C4 = C[3];
      auto &eTt = E[0], &eTr = E[1], &eTb = E[2], &eTl = E[3];
      const int s = source;
      const DT<T>* a[10];
      if (leg == 0) {
        const DT<T>* x[10] = {&C4[s], &C2[t], &C1[t], &C3[s], &eTb[s], &eTb[t], &eTl[t], &eTt[t], &eTt[s], &eTr[s]};
        std::copy(x, x + 10, a);
      } else if (leg == 1) {
        const DT<T>* x[10] = {&C4[s], &C1[t], &C2[t], &C3[s], &eTl[s], &eTl[t], &eTt[t], &eTr[t], &eTr[s], &eTb[s]};
        std::copy(x, x + 10, a);
      } else if (leg == 2) {
        const DT<T>* x[10] = {&C1[s], &C2[t], &C3[t], &C4[s], &eTt[s], &eTt[t], &eTr[t], &eTb[t], &eTb[s], &eTl[s]};
        std::copy(x, x + 10, a);
      } else {
        const DT<T>* x[10] = {&C2[s], &C3[t], &C4[t], &C1[s], &eTr[s], &eTr[t], &eTb[t], &eTl[t], &eTl[s], &eTt[s]};
        std::copy(x, x + 10, a);
      }
      const int64_t d1 = lat.pdim[s], d2 = lat.pdim[t];
      const DT<T> op12 = from_host({d1, d2, d1, d2}, op);
      PrecScope prec(this, 0);
      FuBackend bk{this};
      fu::Params p;
      p.inverse_env_cut = fp->inverse_env_cut;
      p.inverse_precision = fp->inverse_precision;
      p.convergence_epsilon = fp->convergence_epsilon;
      p.max_iteration = fp->max_iteration;
      p.gauge_fix = fp->gauge_fix != 0;
      fu::FullUpdate<FuBackend> f{bk, p};
      DT<T> n1, n2;
      const fu::Stats st_ = f.bond(*a[0], *a[1], *a[2], *a[3], *a[4], *a[5], *a[6], *a[7], *a[8], *a[9], Tn[s], Tn[t],
                                   op12, leg, n1, n2);
      if (n1.sh != Tn[s].sh || n2.sh != Tn[t].sh)
        fail(TG_E_RUNTIME, "full update: the updated bond lost rank (site tensor shape changed)");
      Tn[s] = n1;
      Tn[t] = n2;
      rot_ok[s] = rot_ok[t] = false;
      check_infos();
      if (iterations) *iterations = st_.iterations;
      if (converged) *converged = st_.converged ? 1 : 0;
    }
  }

  // iTPS::fix_local_gauge (src/iTPS/simple_update.cpp:49-101) over the
  // engine's site tensors and simple-update weights; the bond step and the
  // sweep are local_gauge.hpp's, on the same backend as the full update.
  // Site parity (-1)^(x+y) as SquareLattice builds it (site 0 is +1).
  void su_fix_gauge(int maxiter, double eps, int* sweeps, double* score) override {
    if (maxiter < 0) fail(TG_E_INPUT, "gauge_maxiter must be non-negative");
    PrecScope prec(this, 0);
    lam_to_host();
    lam_dev_stale = true;
    FuBackend bk{this};
    gauge::LocalGauge<FuBackend> g{bk, P.inverse_lambda_cut};
    std::vector<DT<T>> tn(Tn.begin(), Tn.end());
    std::vector<gauge::Weights> lam(lambda.begin(), lambda.end());
    double sc = 0.0;
    const int n = g.run(
        tn, lam, lat.vdim, [&](int s, int leg) { return lat.neighbor(s, leg); },
        [&](int s) { return ((s % lat.LX) + (s / lat.LX)) % 2 == 0 ? 1 : -1; }, maxiter, eps, &sc);
    check_infos();
    for (int i = 0; i < lat.N; ++i) {
      if (tn[static_cast<size_t>(i)].sh != Tn[static_cast<size_t>(i)].sh)
        fail(TG_E_RUNTIME, "local gauge fixing changed a site tensor's shape");
      Tn[static_cast<size_t>(i)] = tn[static_cast<size_t>(i)];
      lambda[static_cast<size_t>(i)] = lam[static_cast<size_t>(i)];
      rot_ok[static_cast<size_t>(i)] = false;
    }
    if (sweeps) *sweeps = n;
    if (score) *score = sc;
  }

  // ------------------------------------------------- energy gradient
  // E = sum_t coeff_t <ops_t>/<1>_t after `iterations` sweeps from the
  // initial environment, and dE/dTn by the reverse pass of adjoint.hpp
  void energy_grad(int nterms, const tg_window_term* terms, int iterations, int checkpoint_every,
                   double svd_broadening, double* energy, double* grad) override {
    if (density) fail(TG_E_INPUT, "the energy gradient is defined for an iTPS only");
    if constexpr (CPLX) {
      fail(TG_E_INPUT, "energy gradient: real site tensors only");
    } else {
      if (P.use_rsvd) fail(TG_E_INPUT, "energy gradient: full-SVD projectors only (use_rsvd = 0)");
      if (nterms < 1) fail(TG_E_INPUT, "energy gradient: no energy terms");
      if (!(svd_broadening >= 0.0)) fail(TG_E_INPUT, "energy gradient: svd_broadening must be >= 0");
      std::vector<ad::WindowTerm> w(static_cast<size_t>(nterms));
      for (int q = 0; q < nterms; ++q) {
        const tg_window_term& t = terms[q];
        check_site(t.source);
        if (t.nrow < 1 || t.ncol < 1 || t.nrow > 4 || t.ncol > 4) fail(TG_E_INPUT, "window must be 1..4 x 1..4");
        if (t.source_row < 0 || t.source_row >= t.nrow || t.source_col < 0 || t.source_col >= t.ncol)
          fail(TG_E_INPUT, "source position outside the window");
        if (t.nops < 0 || (t.nops > 0 && (!t.op_row || !t.op_col || !t.ops)))
          fail(TG_E_INPUT, "energy term: operators missing");
        ad::WindowTerm& a = w[static_cast<size_t>(q)];
        a.source = t.source;
        a.nrow = t.nrow;
        a.ncol = t.ncol;
        a.source_row = t.source_row;
        a.source_col = t.source_col;
        a.coeff = t.coeff;
        int64_t off = 0;
        for (int i = 0; i < t.nops; ++i) {
          const int r = t.op_row[i], c = t.op_col[i];
          if (r < 0 || r >= t.nrow || c < 0 || c >= t.ncol) fail(TG_E_INPUT, "operator position outside the window");
          for (int j = 0; j < i; ++j)
            if (t.op_row[j] == r && t.op_col[j] == c) fail(TG_E_INPUT, "two operators on one window site");
          const int site = lat.other(t.source, c - t.source_col, t.source_row - r);
          const int64_t d = lat.pdim[site];
          a.op_row.push_back(r);
          a.op_col.push_back(c);
          a.ops.emplace_back(t.ops + off, t.ops + off + d * d);
          off += d * d;
        }
      }
      ad::Options o;
      o.chi = P.chi;
      o.cutoff = P.inverse_projector_cut;
      o.eps = svd_broadening;
      o.iterations = iterations;
      o.checkpoint_every = checkpoint_every;
      o.prec_absorb = abs_prec;
      o.projector_corner = P.projector_corner != 0;
      std::vector<DT<double>> g;
      const SvdFn fn = [this](DT<double>& A, int64_t m, int64_t n, DT<double>& U, DT<double>& s, DT<double>& VT) {
        svd_jacobi(A, m, n, U, s, VT);
      };
      const double E = energy_grad_device(st, lat, Tn, w, o, fn, grad ? &g : nullptr);
      check_infos();
      *energy = E;
      if (grad) {
        int64_t off = 0;
        for (int i = 0; i < lat.N; ++i) {
          if (g[static_cast<size_t>(i)].size() != Tn[i].size()) fail(TG_E_RUNTIME, "energy gradient: shape mismatch");
          download(g[static_cast<size_t>(i)], grad + off);
          off += Tn[i].size();
        }
      }
    }
  }

  // ------------------------------------------------------------- host I/O
  void set_site_tensor(int site, const double* host) override {
    check_site(site);
    upload(Tn[site], host);
    rot_ok[site] = false;
  }
  void get_site_tensor(int site, double* host) override {
    check_site(site);
    download(Tn[site], host);
  }
  void set_lambda(int site, int leg, const double* host) override {
    check_site(site);
    if (leg < 0 || leg > 3) fail(TG_E_INPUT, "leg must be 0..3");
    lam_to_host();
    auto& l = lambda[site][leg];
    std::copy(host, host + l.size(), l.begin());
    lam_dev_stale = true;
  }
  void get_lambda(int site, int leg, double* host) override {
    check_site(site);
    if (leg < 0 || leg > 3) fail(TG_E_INPUT, "leg must be 0..3");
    lam_to_host();
    const auto& l = lambda[site][leg];
    std::copy(l.begin(), l.end(), host);
  }
  DT<T>& env_ref(int which, int site) {
    check_site(site);
    if (which < 0 || which > 7) fail(TG_E_INPUT, "environment index must be 0..7");
    return which < 4 ? C[which][site] : E[which - 4][site];
  }
  void set_env(int which, int site, const double* host) override {
    upload(env_ref(which, site), host);  // into the existing storage (captured sweeps hold its address)
    env_ready = true;
    spec_old_ok = false;
  }
  void get_env(int which, int site, double* host) override { download(env_ref(which, site), host); }
  void svd_stats(int64_t* out) override {
    out[0] = exact_solves;
    out[1] = exact_iters;
    out[2] = exact_checks;
    out[3] = exact_dense;
  }

  void sync() override {
    check_infos();
    TG_CUDA(cudaStreamSynchronize(st));
  }
  void* stream() override { return static_cast<void*>(st); }
};

Engine* make_engine(const tg_lattice_desc* lat, const tg_params* p, int is_complex, int device) {
  if (!lat || !p) fail(TG_E_INPUT, "null lattice or params");
  if (is_complex) return new EngineT<cplx>(lat, p, device);
  return new EngineT<double>(lat, p, device);
}

}  // namespace tg
