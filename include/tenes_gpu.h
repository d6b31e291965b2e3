/*
 * tenes_gpu.h -- C ABI of libtenes_gpu.so, the B200 (sm_100a) implementation
 * of TeNeS's iTPS CTMRG environment path.
 *
 * Every entry point returns a tg_status and never throws or aborts across the
 * ABI (the reference lets C++ exceptions escape tenes_itps_main,
 * src/iTPS/main.cpp:33-39; here they are turned into status codes).  The
 * message of the last failure is available from tg_last_error().
 *
 * Tensor layouts on the host side of the ABI are row-major (last leg fastest)
 * in the reference's leg order:
 *   site tensor Tn  [left, up, right, bottom, phys]   (D0, D1, D2, D3, d)
 *   corners C1..C4  [chi, chi]  legs (previous, next) going clockwise
 *   edges  eT*      [chi, chi, D, D]  (previous, next, ket, bra)
 * (src/iTPS/iTPS.hpp:301-318, src/iTPS/core/ctm.cpp:44-53).  Complex tensors
 * are interleaved (re, im) pairs of doubles.  Environment legs are padded to
 * chi with zeros; the reference's shrinking of a leg below chi when fewer
 * than chi singular values pass the cutoff is represented by zero rows and
 * columns, which leaves every contraction unchanged.
 *
 * Threading: a context is used by one host thread at a time.  All work is
 * issued on the context's own CUDA stream; every call returns after its work
 * is complete unless its name ends in _async.
 */
#ifndef TENES_GPU_H_
#define TENES_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tg_status {
  TG_OK = 0,
  TG_E_INPUT = 1,    /* bad argument, shape or parameter (tenes::input_error) */
  TG_E_LOAD = 2,     /* bad tensor data (tenes::load_error) */
  TG_E_RUNTIME = 3,  /* numerical failure, e.g. SVD did not converge */
  TG_E_NOCONV = 4,   /* CTMRG hit iteration_max without converging (warning-level) */
  TG_E_CUDA = 5,     /* CUDA / cuSOLVER error */
  TG_E_STATE = 6     /* call made in the wrong order (e.g. move before init) */
} tg_status;

typedef struct tg_ctx tg_ctx;

/* Unit cell (SquareLattice, src/SquareLattice.hpp:54-163). */
typedef struct tg_lattice_desc {
  int LX;
  int LY;
  int skew;
  const int* physical_dims; /* [LX*LY] */
  const int* virtual_dims;  /* [LX*LY][4]: left, up, right, bottom */
} tg_lattice_desc;

/* CTMRG / simple-update parameters (PEPS_Parameters,
 * src/iTPS/PEPS_Parameters.cpp:30-77, keys of [parameter.ctm] in
 * src/iTPS/load_toml.cpp:383-398). */
typedef struct tg_params {
  int chi;                          /* ctm.dimension */
  double inverse_projector_cut;     /* ctm.projector_cutoff (1e-12) */
  double ctm_convergence_epsilon;   /* ctm.convergence_epsilon (1e-6) */
  int max_ctm_iteration;            /* ctm.iteration_max (100) */
  int projector_corner;             /* ctm.projector_corner (1) */
  int use_rsvd;                     /* ctm.use_rsvd (0) */
  double rsvd_oversampling_factor;  /* ctm.rsvd_oversampling_factor (2.0) */
  int rsvd_oversample_abs;          /* >= 0: k = cut + this, overrides the factor */
  int rsvd_power_iters;             /* power iterations of the rSVD range finder (2) */
  uint64_t rsvd_seed;               /* key of the counter-based rSVD test matrix */
  double inverse_lambda_cut;        /* simple_update.lambda_cutoff (1e-12) */
  int mixed;                        /* 1: CTMRG absorption contractions and rSVD panel products as
                                       3xTF32 tensor-core products (FP64 tile accumulation); the
                                       orthonormalisation, SVDs and observables stay FP64.  Real
                                       tensors only.  0 (default): everything FP64. */
  int cuda_graph;                   /* 1 (default): with rSVD corner projectors, replay each CTMRG
                                       sweep from a captured CUDA graph (same kernels, same results);
                                       0: launch every kernel from the host. */
  int svd_solver;                   /* solver of the full-SVD projectors (use_rsvd = 0,
                                       ctm.cpp:267-302, 441-475): 0 (default) the leading singular
                                       triplets the truncation keeps, by block subspace iteration
                                       with Rayleigh-Ritz checks run until every kept triplet's
                                       residual is <= 1e-13 s_0 (a dense SVD when that cannot be
                                       reached); 1: the dense SVD (cuSOLVER gesvd) of the whole
                                       matrix.  Both give the reference's truncated factors. */
  int density;                      /* 1: the context holds an iTPO, the density operator of the
                                       finite-temperature mode (iTPS::finite_temperature,
                                       finite_temperature.cpp:22-86).  Site tensors are
                                       (D0,D1,D2,D3,d,d) (physical_dims hold d); the simple update
                                       applies kron(op, conj(op)) (simple_update.cpp:141-178); the
                                       CTMRG is the single-layer one of ctm_single.cpp on
                                       sum_p Tn[...,p,p], with edge tensors (chi,chi,D,1); the
                                       measurements are the density contractions of
                                       contract_density_ctm/ (sum_{p,q} op[p,q] Tn[...,p,q]).  Needs
                                       chi >= every bond dimension; no full update or gradient.
                                       0 (default): an iTPS. */
} tg_params;

/* One `tenes input.toml` run, as the reference's process-level entry point
 *   extern "C" int tenes_itps_main(const char*, MPI_Comm, int)
 * (src/iTPS/main.hpp:26-28, main.cpp:33-39) without the communicator (one
 * GPU, device 0 unless CUDA_VISIBLE_DEVICES says otherwise): reads the expert
 * input file, runs the simple / full update or the time evolution, the CTMRG
 * environment and the measurements, and writes the reference's output files
 * into the input's outdir (parameters.dat, density.dat, onesite_obs.dat,
 * twosite_obs.dat, multisite_obs_*.dat, correlation*.dat, time.dat, or their
 * TE_ forms).  Where the reference throws, this returns a status:
 * TG_E_INPUT (bad or unsupported input, missing file), TG_E_LOAD (tensor
 * checkpoint), TG_E_RUNTIME, TG_E_CUDA; the message is in tg_last_error().
 * The run is the library's Python front end (tenes_b200.itps), embedded:
 * from a process without Python the first call loads libpython
 * (TENES_GPU_LIBPYTHON overrides which; TENES_GPU_PYTHON_SITE the packages
 * directory).  Calls are serialised. */
int tenes_gpu_main(const char* input_toml, int print_level);

/* Fill *p with the reference defaults. */
void tg_params_default(tg_params* p);

/* Human-readable message of the last failing call on this thread. */
const char* tg_last_error(void);

/* Library version string. */
const char* tg_version(void);

/* Create / destroy a context on CUDA device `device`.  is_complex selects
 * complex128 tensors (TeNeS complex_tensor) instead of float64 (real_tensor). */
tg_status tg_ctx_create(const tg_lattice_desc* lattice, const tg_params* params,
                        int is_complex, int device, tg_ctx** out);
tg_status tg_ctx_destroy(tg_ctx* ctx);

/* Site tensors and simple-update weights (iTPS::Tn, lambda_tensor,
 * src/iTPS/iTPS.hpp:301-306).  `host` holds D0*D1*D2*D3*d values (twice as
 * many doubles when complex). */
tg_status tg_set_site_tensor(tg_ctx* ctx, int site, const double* host);
tg_status tg_get_site_tensor(tg_ctx* ctx, int site, double* host);
tg_status tg_set_lambda(tg_ctx* ctx, int site, int leg, const double* host);
tg_status tg_get_lambda(tg_ctx* ctx, int site, int leg, double* host);

/* Environment tensors.  which: 0..3 = C1..C4, 4..7 = eTt, eTr, eTb, eTl. */
tg_status tg_set_env(tg_ctx* ctx, int which, int site, const double* host);
tg_status tg_get_env(tg_ctx* ctx, int which, int site, double* host);

/* Environment initialisation from the site tensors
 * (core::Calc_CTM_Environment initialize branch, ctm.cpp:984-1193). */
tg_status tg_ctm_init(tg_ctx* ctx);

/* One directional move absorbing column ix / row iy
 * (core::Left_move / Right_move / Top_move / Bottom_move, ctm.cpp:562-813).
 * dir: 0 = left, 1 = right, 2 = top, 3 = bottom. */
tg_status tg_ctm_move(tg_ctx* ctx, int dir, int line);

/* One CTMRG iteration: all left, right, top, bottom moves (ctm.cpp:1205-1228). */
tg_status tg_ctm_sweep(tg_ctx* ctx);

/* Check_Convergence_CTM (ctm.cpp:815-969) against the corners saved by the
 * previous call (or by tg_ctm_init); saves the current corners. */
tg_status tg_ctm_check_convergence(tg_ctx* ctx, int* converged, double* sig_max);

/* Counters of the exact truncated SVD behind the full-SVD projectors
 * (svd_solver = 0; the dense SVD of ctm.cpp:273-302 and 441-475 restated as
 * block subspace iteration): out[0] solves, out[1] subspace iterations,
 * out[2] Rayleigh-Ritz checks, out[3] solves handed to the dense SVD.
 * Cumulative over the context's life. */
tg_status tg_projector_svd_stats(tg_ctx* ctx, int64_t* out);

/* core::Calc_CTM_Environment (ctm.cpp:971-1253): optional init, then sweeps
 * until converged or max_ctm_iteration.  Returns TG_OK also when not
 * converged (the reference only warns); *converged tells which. */
tg_status tg_ctm_run(tg_ctx* ctx, int initialize, int* iterations, int* converged,
                     double* sig_max);

/* L2-normalised singular values of corner `which` (0..3) of `site`
 * (the spectrum Check_Convergence_CTM compares, ctm.cpp:830-847); chi values. */
tg_status tg_corner_spectrum(tg_ctx* ctx, int which, int site, double* host);

/* <op> through the environment.  Results are (re, im) pairs.
 * One site: Contract_one_site_iTPS_CTM (contract_itps_ctm/ctm.cpp:89-113),
 *   op is d x d, applied as sum_{p,q} Tn[..p] op[p,q] conj(Tn[..q]).
 * Nearest-neighbour op12 (d1,d2,d1,d2): Contract_two_sites_{horizontal,vertical}_op12
 *   (ctm.cpp:213-319); source/target as in twosite_obs.cpp:189-222.
 * For an iTPO (params.density) the same calls are the density contractions
 * (contract_density_ctm/ctm.cpp:89-274): sum_{p,q} op[p,q] Tn[...,p,q] for
 * one site, sum op12[p1,p2,q1,q2] over the two density tensors for a bond;
 * tg_measure_window, tg_measure_correlation and the transfer matrix likewise
 * (Contract_RxC_density_CTM, *Correlation_density_CTM, the rank-3 matvecs of
 * transfer_matrix.cpp:187-308). */
tg_status tg_measure_onesite(tg_ctx* ctx, int site, const double* op, double* out);
tg_status tg_measure_bond_op12(tg_ctx* ctx, int source, int dx, int dy, const double* op,
                               double* out);

/* Two-site reduced density matrix of the nearest-neighbour bond of
 * tg_measure_bond_op12, unnormalised, legs (source, target, source', target')
 * (d_s * d_t * d_s * d_t values, interleaved pairs when complex): the op12
 * value of that call is sum op12 * rdm and the norm sum_ab rdm[a,b,a,b], so
 * one contraction of the bond serves any number of operators.  The same
 * contraction sequence as Contract_two_sites_*_op12 (ctm.cpp:213-319).
 * For an iTPO the values are R[(p_s*d_s + q_s), (p_t*d_t + q_t)], the
 * environment of the two density tensors: <op12> = sum op12[p_s,p_t,q_s,q_t] R
 * and the norm sum_ab R[(a,a),(b,b)]. */
tg_status tg_measure_bond_rdm(tg_ctx* ctx, int source, int dx, int dy, double* out);

/* Long-range correlations along a strip (StartCorrelation / Transfer /
 * FinishCorrelation_iTPS_CTM, contract_itps_ctm/correlation.cpp, as
 * measure_correlation_ctm uses them, correlation_function.cpp:70-212):
 * <O_left O_right> / <1> with O_left on `left` and O_right on the site r steps
 * to the right (dir 0) or up (dir 1), for r = 1..r_max.  left_op is d x d for
 * `left`; right_ops lists, for every site of the unit cell in order, nright
 * operators of that site's d x d.  out receives (re, im) pairs, r-major:
 * out[2*((r-1)*nright + q)].  Linear in r_max. */
tg_status tg_measure_correlation(tg_ctx* ctx, int left, int dir, int r_max, const double* left_op, int nright,
                                 const double* right_ops, double* out);

/* <prod of one-site ops> on an nrow x ncol window (1..4 each), unnormalised:
 * Contract_RxC_iTPS_CTM (contract_itps_ctm/ctm.cpp:45-87).  The window holds
 * site lat.other(source, c - source_col, source_row - r) at (r, c), row 0 on
 * top (twosite_obs.cpp:123-149); nops operators sit at (op_row[i], op_col[i]),
 * each d x d for that site's d, concatenated in `ops`; identity elsewhere.
 * The norm is the call with nops = 0. */
tg_status tg_measure_window(tg_ctx* ctx, int source, int nrow, int ncol, int source_row, int source_col, int nops,
                            const int* op_row, const int* op_col, const double* ops, double* out);

/* Leading eigenvalues (largest modulus first, (re, im) pairs) of the row
 * (dir 0, row y = fixed) or column (dir 1, column x = fixed) transfer matrix
 * built from the edge tensors: TransferMatrix::eigenvalues
 * (transfer_matrix.cpp:84-142) -- a dense eigensolver when chi^2 <=
 * maxdim_dense, else Arnoldi (arnoldi.cpp) with the given dimensions,
 * restarts and tolerance; *nev receives min(num_eigvals, chi^2). */
tg_status tg_tm_eigenvalues(tg_ctx* ctx, int dir, int fixed, int num_eigvals, int maxdim_dense, int arnoldi_maxdim,
                            int arnoldi_restartdim, int arnoldi_maxiter, double arnoldi_rtol, double* out,
                            int* nev);

/* Simple update (src/iTPS/simple_update.cpp:25-46).
 * One-site: Tn[site] <- tensordot(Tn[site], op, 4, 0).
 * Bond: core::Simple_update_bond (core/simple_update.cpp:50-198) between
 * `source` and its neighbour on `source_leg`; op is (d1, d2, d1, d2). */
tg_status tg_su_onesite(tg_ctx* ctx, int site, const double* op);
tg_status tg_su_bond(tg_ctx* ctx, int source, int source_leg, const double* op);
/* A sequence of simple-update steps applied in its order, as n calls of
 * tg_su_onesite (source_legs[i] < 0) and tg_su_bond would apply them -- one
 * Trotter step of iTPS::simple_update over the evolution operators
 * (src/iTPS/simple_update.cpp:113-119).  Consecutive bond steps on pairwise
 * disjoint site pairs commute exactly, so each run of them is one launch with
 * one thread block a bond.  ops[i] points at operator i. */
tg_status tg_su_bonds(tg_ctx* ctx, int n, const int* sources, const int* source_legs, const double* const* ops);

/* Full update of one bond (PEPS_Parameters full-update knobs,
 * src/iTPS/PEPS_Parameters.cpp:57-62; keys of [parameter.full_update] in
 * src/iTPS/load_toml.cpp:374-379). */
typedef struct tg_fu_params {
  double inverse_env_cut;     /* full_update.env_cutoff (1e-12) */
  double inverse_precision;   /* full_update.inverse_precision (1e-12) */
  double convergence_epsilon; /* full_update.convergence_epsilon (1e-6) */
  int max_iteration;          /* full_update.iteration_max (100) */
  int gauge_fix;              /* full_update.gauge_fix (1) */
} tg_fu_params;

/* Fill *p with the reference defaults. */
void tg_fu_params_default(tg_fu_params* p);

/* core::Full_update_bond (src/iTPS/core/full_update.cpp:31-455) of the bond
 * between `source` and its neighbour on `source_leg`, in the current
 * environment (the tensors that face the bond, src/iTPS/full_update.cpp:42-116);
 * op is (d1, d2, d1, d2).  Replaces the two site tensors and leaves the
 * environment alone: the fast full update follows with tg_ctm_move on the
 * two lines of the bond (full_update.cpp:122-148).  *iterations and
 * *converged (optional) report the least-squares loop.  Real and complex
 * tensors. */
tg_status tg_fu_bond(tg_ctx* ctx, int source, int source_leg, const double* op, const tg_fu_params* params,
                     int* iterations, int* converged);

/* iTPS::fix_local_gauge (src/iTPS/simple_update.cpp:49-101, with
 * core::fix_local_gauge and boundary_tensor, src/iTPS/core/local_gauge.cpp:44-224):
 * sweeps over the bonds (sites of parity +1, then -1; source legs 2, then 1;
 * legs of dimension 1 skipped) that bring each bond to the gauge in which both
 * boundary tensors are the identity, until the largest |eigenvalue - 1| of the
 * boundary tensors is below eps, at most maxiter sweeps.  Updates the site
 * tensors and the simple-update weights (inverse weights cut at the context's
 * inverse_lambda_cut).  *sweeps and *score (optional) report the sweeps done
 * and the last score. */
tg_status tg_su_fix_gauge(tg_ctx* ctx, int maxiter, double eps, int* sweeps, double* score);

/* iTPS::initialize_tensors (src/iTPS/tensors.cpp:38-137): per site,
 * Tn[0,0,0,0,:] = initial state (random when all entries are zero) and every
 * other entry noise * U(-1,1) from std::mt19937(seed) (real part) and
 * std::mt19937(seed*11+137) (imaginary part), drawn first-leg-fastest.
 * initial_dirs concatenates the per-site initial states (dir_len[i] values
 * each); noises has one value per site.  Resets the lambdas to one. */
tg_status tg_init_tensors(tg_ctx* ctx, int seed, const double* initial_dirs, const int* dir_len,
                          const double* noises);

/* One product term of an energy: <prod ops> on an nrow x ncol window, the
 * geometry and operator layout of tg_measure_window, divided by the same
 * window without operators (the norm, shared by all terms of one window as
 * twosite_obs.cpp:160-181 shares it).  A two-site operator enters as the sum
 * of the products of its singular components (twosite_obs.cpp:223-243). */
typedef struct tg_window_term {
  int source;
  int nrow, ncol, source_row, source_col;
  int nops;
  const int* op_row;
  const int* op_col;
  const double* ops; /* nops real d x d operators, concatenated */
  double coeff;
} tg_window_term;

/* Energy and its gradient with respect to the site tensors.  No counterpart
 * in the reference (TeNeS optimises by simple / full update only).
 *   E = sum_t coeff_t <ops_t> / <1>_t
 * on the environment reached after `iterations` CTMRG sweeps from the
 * initial environment of the current site tensors (tg_ctm_init, then
 * tg_ctm_sweep; full-SVD projectors, corner or up/down
 * (projector_corner), use_rsvd = 0; real tensors).  grad (optional, NULL
 * for E only) receives
 * dE/dTn of every site, concatenated in site order in the layout of
 * tg_set_site_tensor.  The gradient is a hand-written reverse pass through
 * the sweeps and the truncated SVDs of the projectors, whose adjoint uses the
 * Lorentzian-broadened factors (s_j^2 - s_i^2) / ((s_j^2 - s_i^2)^2 +
 * svd_broadening (s_i^2 + s_j^2)^2), broadened relative to each pair's
 * scale.  The sweeps are recomputed in segments of
 * checkpoint_every sweeps, so device memory holds one segment's
 * intermediates.  With params.mixed the moves' contractions (forward and
 * adjoint) run as 3xTF32 products; SVDs and the energy stay FP64.  The
 * context's own environment is left unchanged. */
tg_status tg_energy_grad(tg_ctx* ctx, int nterms, const tg_window_term* terms, int iterations,
                         int checkpoint_every, double svd_broadening, double* energy, double* grad);

/* Synchronise the context's stream; report asynchronous CUDA errors. */
tg_status tg_sync(tg_ctx* ctx);

/* Count of kernels this library has launched in the calling process. */
uint64_t tg_kernel_launch_count(void);

/* The CUDA stream (cudaStream_t) all work of the context is issued on, so a
 * caller can order its own work or timing events against it. */
tg_status tg_ctx_stream(tg_ctx* ctx, void** stream);

/* Per-launch CUDA-event profiling of the library's kernel families
 * (0 = FP64 DMMA matrix product, 1 = leg permutation, 2 = max-abs
 * normalisation, 3 = Jacobi corner spectra, 4 = dense factorisations
 * (cuSOLVER, CholeskyQR, Jacobi SVD), 5 = other, 6 = 3xTF32 tcgen05 product
 * including its split / pack pre-pass).
 * Adds two events per launch; off by default.  query returns the number of
 * launches, their summed device time in ms and the algorithmic flops and
 * bytes they were issued for since the last reset. */
tg_status tg_profile_enable(int on);
tg_status tg_profile_reset(void);
tg_status tg_profile_query(int kind, uint64_t* launches, double* ms, double* flops, double* bytes);

/* n independent products C_i = op(A_i) op(B_i) through the library's grouped
 * persistent contraction kernel (the one a move's absorptions run as), with
 * host buffers: A holds every A_i (M_i x K_i) back to back, B every B_i
 * (K_i x N_i), C receives every C_i (M_i x N_i, row-major); mnk = (M_i, N_i,
 * K_i) triples.  flags[i] (or all 0 if flags is NULL): bit 0 A_i stored
 * column-major, bit 1 B_i stored column-major, bit 2 conj(A_i), bit 3
 * conj(B_i) (complex only).  is_complex: elements are (re, im) pairs of
 * doubles, the products run as 3M.  For tests of the kernels; not part of
 * the CTMRG path. */
tg_status tg_gemm_group_host(int n, const int64_t* mnk, const int* flags, int is_complex, const double* A,
                             const double* B, double* C);
/* The grouped kernel's tile autotuner so far (process-wide): the number of
 * group shapes it has timed, and for each of the first nwins tile variants
 * (0: 64-row tiles, 1: 32-row tiles) how many of them it chose. */
tg_status tg_gemm_group_stats(int64_t* tuned, int64_t* wins, int nwins);

/* Microbenchmark of the library's contraction kernel: average device time of
 * one M x N x K real product (prec 0: FP64 DMMA, 1: 3xTF32), B row-major
 * (layout 0) or column-major (layout 1).  Allocates its own buffers; not part
 * of the CTMRG path. */
tg_status tg_bench_gemm(int64_t M, int64_t N, int64_t K, int layout, int prec, int iters, double* avg_ms);

/* One real product C = A B through the library's contraction kernels, with
 * host buffers and element strides: A(m,k) = A[m*sAm + k*sAk], B(k,n) =
 * B[k*sBk + n*sBn], C(m,n) = C[m*sCm + n*sCn] (one of each operand's strides
 * must be 1).  prec 0: FP64 DMMA; 1: 3xTF32 on tcgen05.  The buffers hold
 * the extents the strides reach.  For tests of the kernels; not part of the
 * CTMRG path. */
tg_status tg_gemm_host(int64_t M, int64_t N, int64_t K, const double* A, int64_t sAm, int64_t sAk,
                       const double* B, int64_t sBk, int64_t sBn, double* C, int64_t sCm, int64_t sCn,
                       int prec);

/* Orthonormal basis of the span of a real column-major n x k host panel Y
 * (in place) by the engine's shifted CholeskyQR: `passes` passes, the first
 * two shifted, a perturbation of relative size 1e-14 after the first, all in
 * one launch of one thread-block cluster.  *pivot_flag = 1 if a Cholesky
 * pivot was not positive.  k <= 96.  For tests of the kernel; the CTMRG path
 * calls it inside the rSVD projectors (src/iTPS/core/ctm.cpp:243-244). */
tg_status tg_cholqr_host(int64_t n, int64_t k, double* Y, int passes, int* pivot_flag);

/* Allocation-free corner spectra.  No counterpart in the reference: it exists
 * for callers that must not allocate device memory where they need the
 * spectra -- code that runs under a fixed device-memory budget, hosts that
 * hand out every device byte through their own pool, or a convergence check
 * slotted between other GPU work where a cudaMalloc could stall the device.
 *
 * Computes the same L2-normalised, descending singular values as
 * tg_corner_spectrum for `count` n x n matrices that already live in device
 * memory: device_mats is a HOST array of `count` DEVICE pointers (row-major
 * float64, or interleaved complex128 when is_complex), device_out is a device
 * buffer of count*n doubles.  Work is queued on `stream` (a cudaStream_t, NULL
 * for the legacy default stream); the call returns once it is queued.  The
 * pointer table is copied through a pageable staging array inside the call,
 * so device_mats may be reused (or freed) as soon as the call returns,
 * whether it is pageable or page-locked.
 *
 * It allocates nothing: the device-side copy of the pointer table goes into a
 * fixed 8 KiB array inside the library (at most 1024 matrices; n <= 160 real,
 * n <= 112 complex; larger requests fail with TG_E_INPUT).  Every GPU that
 * loads the library keeps that array until the process exits.  The first call
 * on each device looks up the array's device address, so make that first call
 * before any stream capture.  All calls share the array and it keeps the last
 * call's contents, so calls whose GPU work overlaps race on it: order them
 * on one stream, or synchronise between them. */
tg_status tg_corner_spectra_noalloc(const void* const* device_mats, int count, int n, int is_complex,
                                    double* device_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TENES_GPU_H_ */
