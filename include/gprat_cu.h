/*
 * gprat_cu.h — C ABI of the B200 (sm_100a) GP-regression library
 * libgprat_cuda.so.  Plain pointers and sizes; no C++ or torch types.
 *
 * One opaque handle (gprat_cu_gp) owns a device-resident copy of the
 * training series and outputs plus the device workspace for one GP.  Every
 * reference-facing call below takes HOST buffers, runs the whole pipeline on
 * the GPU (one CUDA stream per handle) and returns after the results are back
 * in the caller's buffers.  Calls on one handle are serialised by the
 * caller; different handles may be used from different threads.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   gpu::predict / predict_with_uncertainty / predict_with_full_cov /
 *   compute_loss / optimize / optimize_step / cholesky
 *   (core/include/gpu/gp_functions.cuh:27-199, core/src/gpu/gp_functions.cu:17-467)
 *   and their CPU twins cpu::* (core/src/cpu/gp_functions.cpp:18-1269), which
 *   gprat::GP dispatches to (core/src/gprat_c.cpp:106-361).
 *
 * Conventions (identical to the reference):
 *   - training input is a 1-D series; feature row i is in[i .. i+n_reg-1]
 *     (core/src/cpu/gp_algorithms.cpp:22-26), so n_in >= n_tiles*n_tile_size
 *     + n_reg - 1;
 *   - hyper = {lengthscale, vertical_lengthscale, noise_variance}
 *     (core/include/gp_kernels.hpp:14-39);
 *   - test size m = m_tiles * m_tile_size (utils::compute_test_tiles,
 *     core/src/utils_c.cpp:34-52, is the caller's business).
 *
 * Status codes: every function returns GPRAT_CU_OK (0) or one of the codes
 * below; gprat_cu_last_error() returns a thread-local message for the last
 * failure on the calling thread.
 */
#ifndef GPRAT_CU_H
#define GPRAT_CU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPRAT_CU_OK 0
#define GPRAT_CU_ERR_INVALID_ARG 1
#define GPRAT_CU_ERR_OOM 2
#define GPRAT_CU_ERR_NOT_SPD 3 /* Cholesky met a non-positive pivot */
#define GPRAT_CU_ERR_CUDA 4
#define GPRAT_CU_ERR_TIMEOUT 5 /* a bounded device wait gave up */
#define GPRAT_CU_ERR_NO_DEVICE 6

/* Precision of the factorisation and of the variance solve. */
#define GPRAT_CU_PREC_FP64 0       /* all FP64 (DMMA tensor cores) */
#define GPRAT_CU_PREC_MIXED_TF32 1 /* FP32 storage, TF32 tcgen05 trailing updates, FP64 diagonal */
#define GPRAT_CU_PREC_MIXED_BF16 2 /* FP32 storage, BF16 tcgen05 trailing updates, FP64 diagonal */
/* FP64 storage; every product of the factorisation and of the variance solve
 * emulated on the int8 tensor cores (Ozaki scheme, s digit planes, see
 * gprat_cu_gp_set_int8_slices); FP64 diagonal blocks and alpha solves. */
#define GPRAT_CU_PREC_FP64_INT8 3

typedef struct gprat_cu_gp gprat_cu_gp;

/* Thread-local text of the last error on this thread ("" if none). */
const char *gprat_cu_last_error(void);

/* Number of CUDA devices (gprat::gpu_count, core/src/target.cpp:143-155). */
int gprat_cu_device_count(int *count);

/* Library build identification, e.g. "gprat_cu sm_100a". */
const char *gprat_cu_version(void);

/*
 * Creates a GP on `device`: copies the training series (n_in doubles) and
 * outputs (n_out >= n_tiles*n_tile_size doubles) to HBM.  Replaces the
 * per-call host->device copies of gpu::predict* (core/src/gpu/gp_functions.cu:114-116)
 * and the state kept by gprat::GP (core/include/gprat_c.hpp:56-87).
 */
int gprat_cu_gp_create(int device,
                       const double *train_in,
                       int64_t n_in,
                       const double *train_out,
                       int64_t n_out,
                       int n_tiles,
                       int n_tile_size,
                       int n_regressors,
                       gprat_cu_gp **out);

int gprat_cu_gp_destroy(gprat_cu_gp *gp);

/* Selects GPRAT_CU_PREC_* for subsequent calls (default FP64).  The
 * tensor-core modes (TF32, BF16, FP64_INT8) need n_tiles * n_tile_size to be
 * a multiple of 128. */
int gprat_cu_gp_set_precision(gprat_cu_gp *gp, int precision);

/*
 * Digit planes of the int8-emulated FP64 products (GPRAT_CU_PREC_FP64_INT8),
 * 3 <= slices <= 7, default 5.  Each operand keeps 6 + 7.99 (slices - 1) bits
 * relative to the largest entry of its 128-column block; a product costs
 * slices * (slices + 1) / 2 int8 tensor-core passes.  No counterpart in the
 * reference (whose GPU path is FP64 cuBLAS/cuSOLVER only).
 */
int gprat_cu_gp_set_int8_slices(gprat_cu_gp *gp, int slices);

/*
 * Digit groups kept in the bulk of the int8-emulated products
 * (GPRAT_CU_PREC_FP64_INT8): group g holds the digit pairs (p, q) with
 * p + q = g, and a product keeps groups 0 .. G-1 (G (G + 1) / 2 int8 passes).
 * factor_groups applies to the factorisation's trailing updates (the panel
 * chain, whose accuracy sets alpha's, keeps every group), variance_groups to
 * the variance solve's updates (its 128-column leaves keep every group); 0
 * keeps all `slices` groups (default).  With 5 planes and 4 groups at
 * n = 32768, d = 64, mean and variance stay within 1e-8 of FP64 in about
 * three quarters of the time; at n = 16384, d = 8 they do not (about 1e-7):
 * the loss of accuracy depends on the problem.  No counterpart in the
 * reference.
 */
int gprat_cu_gp_set_int8_groups(gprat_cu_gp *gp, int factor_groups, int variance_groups);

/*
 * Tiled Cholesky factor (gprat::GP::cholesky, core/src/gprat_c.cpp:336-361;
 * cpu::cholesky core/src/cpu/gp_functions.cpp:18-78).  Writes n_tiles^2
 * row-major tiles of n_tile_size^2 doubles, tile (i,j) at offset
 * (i*n_tiles+j)*n_tile_size^2.  Lower tiles hold L; diagonal tiles keep K's
 * strict upper triangle (as LAPACKE dpotrf2('L') does); upper tiles are zero
 * (the reference returns them empty).
 */
int gprat_cu_cholesky(gprat_cu_gp *gp, const double hyper[3], double *tiles_out);

/* Predictive mean (gprat::GP::predict, core/src/gprat_c.cpp:106-154). */
int gprat_cu_predict(gprat_cu_gp *gp,
                     const double hyper[3],
                     const double *test_in,
                     int64_t n_test_in,
                     int m_tiles,
                     int m_tile_size,
                     double *mean);

/* Mean and per-point posterior variance
 * (gprat::GP::predict_with_uncertainty, core/src/gprat_c.cpp:156-203). */
int gprat_cu_predict_with_uncertainty(gprat_cu_gp *gp,
                                      const double hyper[3],
                                      const double *test_in,
                                      int64_t n_test_in,
                                      int m_tiles,
                                      int m_tile_size,
                                      double *mean,
                                      double *var);

/* gprat::GP::predict_with_full_cov (core/src/gprat_c.cpp:206-253): the
 * reference forms K** - V^T V and returns its diagonal; same outputs. */
int gprat_cu_predict_with_full_cov(gprat_cu_gp *gp,
                                   const double hyper[3],
                                   const double *test_in,
                                   int64_t n_test_in,
                                   int m_tiles,
                                   int m_tile_size,
                                   double *mean,
                                   double *var);

/* Full m x m posterior covariance K** - K*^T K^-1 K* (row-major, both
 * triangles).  No counterpart in the reference, which discards all but the
 * diagonal (core/src/cpu/gp_functions.cpp:663-676). */
int gprat_cu_predict_full_covariance(gprat_cu_gp *gp,
                                     const double hyper[3],
                                     const double *test_in,
                                     int64_t n_test_in,
                                     int m,
                                     double *mean,
                                     double *cov);

/* Mean negative log marginal likelihood 0.5*(y^T a + sum log L_ii^2 + N log 2pi)/N
 * (gprat::GP::calculate_loss, core/src/gprat_c.cpp:306-334). */
int gprat_cu_compute_loss(gprat_cu_gp *gp, const double hyper[3], double *loss);

/* Loss and its gradient w.r.t. the softplus-unconstrained hyper-parameters,
 * scaled like the reference's update_hyperparameter_tiled
 * (core/src/cpu/tiled_algorithms.cpp:296-426):
 *   g = sigmoid(u) * 0.5/N * (tr(K^-1 dK/dtheta) - a^T dK/dtheta a). */
int gprat_cu_loss_grad(gprat_cu_gp *gp, const double hyper[3], double *loss, double grad[3]);

/*
 * One Adam step (gprat::GP::optimize_step, core/src/gprat_c.cpp:280-301;
 * cpu::optimize_step core/src/cpu/gp_functions.cpp:1032-1269).
 * params[9] = {lengthscale, vertical_lengthscale, noise_variance, m_T[3], w_T[3]}
 * is read and updated in place; adam[4] = {learning_rate, beta1, beta2, epsilon};
 * trainable[3] flags; returns the loss at the pre-step parameters.
 */
int gprat_cu_optimize_step(gprat_cu_gp *gp,
                           double params[9],
                           const double adam[4],
                           const int trainable[3],
                           int iter,
                           double *loss);

/* opt_iter Adam steps with iter = 0..opt_iter-1 (gprat::GP::optimize,
 * core/src/gprat_c.cpp:255-278); losses[opt_iter] receives each step's loss. */
int gprat_cu_optimize(gprat_cu_gp *gp,
                      double params[9],
                      const double adam[4],
                      const int trainable[3],
                      int opt_iter,
                      double *losses);

/*
 * Device-resident fit + predict: assembly, Cholesky, alpha, mean and
 * variance with the test series, mean and var already in HBM on the same
 * device (d_var may be NULL for mean only).  Enqueued on `stream`, a
 * cudaStream_t; NULL is the legacy default stream (the work then runs on the
 * handle's own stream, ordered after the default stream's earlier work and
 * before its later work, so events recorded on the default stream around the
 * call time it).  Returns without synchronising.  No counterpart in the
 * reference (whose calls always copy from and to the host).
 */
int gprat_cu_fit_predict_device(gprat_cu_gp *gp,
                                const double hyper[3],
                                const double *d_test_in,
                                int64_t n_test_in,
                                int m,
                                double *d_mean,
                                double *d_var,
                                void *stream);

/* Checks the device status word after a device-resident call (non-SPD
 * pivot, timeouts); synchronises the handle's stream. */
int gprat_cu_check_status(gprat_cu_gp *gp);

/* Number of preconditioned-CG iterations the last mixed-precision alpha
 * solve of this handle took (0 in FP64 mode); waits for the device (the
 * count is kept there).  No counterpart in the reference. */
int gprat_cu_gp_pcg_iterations(gprat_cu_gp *gp, int *iterations);

/*
 * Loss without any memory allocation.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc -- code running under an allocator
 * or memory pool it does not own, or a latency-critical loop that must not
 * enter the driver's allocator (which can synchronise the device) -- this
 * computes the same value as gprat_cu_compute_loss from caller-owned DEVICE
 * buffers: the training series (n_in doubles), the outputs (n_out doubles)
 * and the result (one double at d_loss), on `stream` (a cudaStream_t; NULL =
 * the default stream); it returns after synchronising that stream.
 * hyper[3] is a host array.  All scratch lives in one fixed device array of
 * the library (about 9.4 MB per GPU that loads the library, held until the
 * process exits), so n_tiles * n_tile_size is limited to 1024; larger
 * problems return GPRAT_CU_ERR_INVALID_ARG.  The array is shared by every
 * call and keeps the last call's contents: calls that overlap on the GPU
 * race.  Every call reads the status word back and synchronises its stream,
 * so the call cannot be captured into a CUDA graph.  The first call on a
 * device resolves the array's device address (cudaGetSymbolAddress, once per
 * device).  With CUDA's lazy module loading that first call may also load the
 * library's device code and reserve the array, so a caller that must never
 * allocate makes one warm-up call outside its critical region; the address
 * is kept for the life of the process (cudaDeviceReset of that device
 * afterwards is not supported).
 */
int gprat_cu_compute_loss_noalloc(int device,
                                  const double *d_train_in,
                                  int64_t n_in,
                                  const double *d_train_out,
                                  int64_t n_out,
                                  int n_tiles,
                                  int n_tile_size,
                                  int n_regressors,
                                  const double hyper[3],
                                  double *d_loss,
                                  void *stream);

/*
 * Instrumentation (no counterpart in the reference; the reference times
 * phases with APEX, core/include/apex_utils.hpp:24-54).  Process-wide
 * counters: every kernel launch of this library increments `launches`.
 * With timing enabled, each FP64 tensor-core GEMM launch is bracketed by
 * CUDA events on its own stream; gprat_cu_stats_read synchronises those
 * events and returns the launch count, their summed device time (ms) and
 * their algorithmic FLOPs (2*M*N*K, lower-triangular updates counted as
 * the lower triangle only).
 */
int gprat_cu_stats_reset(void);
int gprat_cu_stats_enable_timing(int enable);
int gprat_cu_stats_read(int64_t *launches, int64_t *gemm_launches, double *gemm_ms, double *gemm_flops);

/*
 * Per-phase step timers, the counterpart of the reference's APEX step timers
 * (GPRAT_START_STEP / GPRAT_END_STEP, core/include/apex_utils.hpp:19-54) with
 * the same labels ("predict_uncer_step cholesky", "cholesky_step assembly",
 * ..., core/src/cpu/gp_functions.cpp:29-678) plus "... alpha refinement" for
 * the mixed-precision alpha and "... loss".  When enabled, every phase of
 * every call is bracketed by CUDA events on the stream that runs it (device
 * time; the look-ahead's side stream is included in "cholesky").
 * gprat_cu_steps_csv writes "label,calls,total_ms,mean_ms" rows (NUL
 * terminated, truncated to cap) and the size it needs into *needed.
 */
int gprat_cu_steps_enable(int enable);
int gprat_cu_steps_reset(void);
int gprat_cu_steps_csv(char *buf, int64_t cap, int64_t *needed);

/*
 * Kernel-level test entry (no counterpart in the reference): runs the
 * tcgen05 tensor-core GEMM of the mixed-precision path on the current
 * device, C = beta*C + alpha * A B^T with host buffers A (M x K, lda),
 * B (N x K, ldb), C (M x N, ldc; read when beta = 1, written back).
 * kind 0 = TF32 operands, 1 = BF16 operands (rounded from the FP32 input).
 * lower != 0: M == N and only C[i][j], i >= j, is written.  rowsq (optional,
 * N <= 128, beta = 0): rowsq[i] += sum_j C_new[i][j]^2.  K must be a multiple
 * of 64.  tile_mode: 0 = the library's choice, 1 = 128 x 128 tiles,
 * 2 = 128 x 256 tiles, 3 = 256 x 256 tiles on a pair of CTAs.
 */
int gprat_cu_test_tc_gemm(int kind,
                          int M,
                          int N,
                          int K,
                          const float *A,
                          int64_t lda,
                          const float *B,
                          int64_t ldb,
                          float *C,
                          int64_t ldc,
                          float alpha,
                          float beta,
                          int lower,
                          double *rowsq,
                          int tile_mode);

/*
 * Kernel-level test entry (no counterpart in the reference): the
 * single-launch blocked triangular solves of the library on the current
 * device.  L: n x n row-major host matrix whose lower triangle (diagonal
 * included) is the factor.  The inverses of its 128 x 128 diagonal blocks
 * are formed on the host; kind 0 = FP64 factor and inverses (the FP64
 * alpha solve), 1 = both rounded to FP32 (the preconditioner of the
 * mixed-precision refinement).  x_fwd = L^-1 b and x_bwd = L^-T b, each
 * from b.  max_ctas > 0 bounds the grid.
 */
int gprat_cu_test_trsv(int kind, int n, const double *L, const double *b, double *x_fwd, double *x_bwd, int max_ctas);

/*
 * Test entry (no counterpart in the reference, which bounds no wait): the
 * number of polls after which a wait of the single-launch triangular solves
 * on an unsolved row block gives up, on the current device; the call then
 * returns GPRAT_CU_ERR_TIMEOUT.  polls < 0 restores the default (about
 * 0.5-1 s of polling).  The waits only re-read global memory, so a budget of
 * 0 ends them at once and nothing is left in flight.
 */
int gprat_cu_test_set_wait_budget(int64_t polls);

/*
 * Kernel-level test entry (no counterpart in the reference): splits the
 * host matrix src (rows x cols, row-major FP64, cols a multiple of 128) into
 * s int8 digit planes on the current device, as the int8-emulated FP64
 * products do:  src[r][c] ~= 2^(e - 6) * sum_{p<s} D_p[r][c] * 2^(-7 p),
 * one exponent e per row and 128-column block (block = 0) or per 128 x 128
 * block (block != 0).  digits: s * rows * cols bytes (plane-major);
 * exps: rows * (cols / 128) (or ceil(rows / 128) * (cols / 128)) ints.
 * 3 <= s <= 7.
 */
int gprat_cu_test_oz_split(int rows, int cols, const double *src, int s, int block, int8_t *digits, int32_t *exps);

/*
 * Kernel-level test entry (no counterpart in the reference): the FP64 GEMM
 * emulated on the int8 tensor cores (tcgen05.mma kind::i8, Ozaki scheme),
 * C = beta * C + alpha * A B^T with host buffers A (M x K), B (N x K),
 * C (M x N; read when beta = 1), all row-major FP64 with K a multiple of 128.
 * A is split with row exponents, B with block exponents, into s digit
 * planes; groups (0 = s) digit groups are kept.  lower != 0: M == N and only
 * C[i][j], i >= j, is written.  rowsq (optional, beta = 0):
 * rowsq[i] += sum_j C_new[i][j]^2.  max_ctas > 0 bounds the grid.
 */
int gprat_cu_test_oz_gemm(int M,
                          int N,
                          int K,
                          const double *A,
                          const double *B,
                          double *C,
                          double alpha,
                          double beta,
                          int lower,
                          int s,
                          int groups,
                          double *rowsq,
                          int max_ctas);

/*
 * Serving (no counterpart in the reference, whose every predict call
 * re-assembles and re-factorises K, core/src/cpu/gp_functions.cpp:110-189).
 * A server owns fitted models resident on one GPU (factor L and alpha stay
 * in HBM) and answers asynchronous requests:
 *   submit_predict: m test points of one model (sliding windows of d values
 *                   over test_in, as in gprat_cu_predict_with_uncertainty);
 *                   result = mean and variance.
 *   submit_fit:     a new model from training data and hyper-parameters;
 *                   result = its model id (ready for predict requests).
 * Pending predict requests of the same model are batched into one launch
 * sequence (continuous batching: a batch forms whenever the model's previous
 * batch has finished); batches of different models and fits run
 * concurrently on separate streams.  Admission: resident models plus the
 * working set of in-flight batches stay within memory_budget_bytes
 * (<= 0: 80 % of the free device memory at creation); a fit that can never
 * fit fails with GPRAT_CU_ERR_OOM.  Every predict result is bit-identical to
 * the same request run alone.  precision: GPRAT_CU_PREC_* for every model.
 * wait() blocks until the request is done, copies mean/var (m doubles each,
 * NULL to skip), the model id and the request's latency (submit to
 * completion, ms); each request id can be waited on once.  stats():
 * latency percentiles of completed predict requests, test points per second
 * since the first submit, completed requests and launched batches.
 */
typedef struct gprat_cu_server gprat_cu_server;

int gprat_cu_server_create(int device, int64_t memory_budget_bytes, int precision, gprat_cu_server **out);
int gprat_cu_server_destroy(gprat_cu_server *server);
int gprat_cu_server_add_model(gprat_cu_server *server,
                              const double *train_in,
                              int64_t n_in,
                              const double *train_out,
                              int64_t n_out,
                              int n_tiles,
                              int n_tile_size,
                              int n_regressors,
                              const double hyper[3],
                              int *model_id);
int gprat_cu_server_submit_predict(gprat_cu_server *server,
                                   int model_id,
                                   const double *test_in,
                                   int64_t n_test_in,
                                   int m,
                                   int64_t *request_id);
int gprat_cu_server_submit_fit(gprat_cu_server *server,
                               const double *train_in,
                               int64_t n_in,
                               const double *train_out,
                               int64_t n_out,
                               int n_tiles,
                               int n_tile_size,
                               int n_regressors,
                               const double hyper[3],
                               int64_t *request_id);
int gprat_cu_server_wait(gprat_cu_server *server,
                         int64_t request_id,
                         double *mean,
                         double *var,
                         int *model_id,
                         double *latency_ms);
int gprat_cu_server_stats(gprat_cu_server *server,
                          double *p50_ms,
                          double *p99_ms,
                          double *predictions_per_s,
                          int64_t *completed,
                          int64_t *batches);

/*
 * Replica serving over several GPUs (no counterpart in the reference): one
 * server per entry of devices (a device may repeat), every model replicated
 * on each.  Test points are independent given a model's factor and alpha, so
 * predict throughput scales with the replicas and no data crosses between
 * GPUs.  add_model and submit_fit yield one model id for all replicas:
 * by default (GPRAT_CU_REPLICATE_COPY) the model is fitted on the first
 * replica and its fitted state (factor, alpha, training data) copied to the
 * others over NVLink, the copy counted in the fit's latency; with
 * GPRAT_CU_REPLICATE_REFIT (set_replication) every replica fits it at once
 * (the pipeline is deterministic, so the copies are identical either way);
 * submit_predict goes to the replica with the fewest test points submitted
 * and not yet waited on.  A predict result is bit-identical to the same
 * request on a single server.  wait/stats as for a server: latencies are the
 * serving replica's (a fit's is its slowest replica's), predictions_per_s
 * and batches are summed over the replicas.  replica_completed: predict
 * requests waited on that replica served.  memory_budget_bytes and
 * precision apply to each replica.
 */
typedef struct gprat_cu_multiserver gprat_cu_multiserver;

int gprat_cu_multiserver_create(const int *devices,
                                int n_devices,
                                int64_t memory_budget_bytes,
                                int precision,
                                gprat_cu_multiserver **out);
int gprat_cu_multiserver_destroy(gprat_cu_multiserver *server);
int gprat_cu_multiserver_add_model(gprat_cu_multiserver *server,
                                   const double *train_in,
                                   int64_t n_in,
                                   const double *train_out,
                                   int64_t n_out,
                                   int n_tiles,
                                   int n_tile_size,
                                   int n_regressors,
                                   const double hyper[3],
                                   int *model_id);
int gprat_cu_multiserver_submit_predict(gprat_cu_multiserver *server,
                                        int model_id,
                                        const double *test_in,
                                        int64_t n_test_in,
                                        int m,
                                        int64_t *request_id);
int gprat_cu_multiserver_submit_fit(gprat_cu_multiserver *server,
                                    const double *train_in,
                                    int64_t n_in,
                                    const double *train_out,
                                    int64_t n_out,
                                    int n_tiles,
                                    int n_tile_size,
                                    int n_regressors,
                                    const double hyper[3],
                                    int64_t *request_id);
int gprat_cu_multiserver_wait(gprat_cu_multiserver *server,
                              int64_t request_id,
                              double *mean,
                              double *var,
                              int *model_id,
                              double *latency_ms);
int gprat_cu_multiserver_stats(gprat_cu_multiserver *server,
                               double *p50_ms,
                               double *p99_ms,
                               double *predictions_per_s,
                               int64_t *completed,
                               int64_t *batches);
int gprat_cu_multiserver_replica_completed(gprat_cu_multiserver *server, int replica, int64_t *completed);
/* Bytes of device memory the resident models of one replica hold (the
 * replica's admission count).  A replicated fit or add that fails on one
 * replica frees the models it made on the others, so they do not stay
 * resident without a global id. */
int gprat_cu_multiserver_resident_bytes(gprat_cu_multiserver *server, int replica, int64_t *bytes);
/* Test entry: the next copy of a fitted model to `replica` (>= 1) reports
 * GPRAT_CU_ERR_OOM instead of copying (a failure made on the host). */
int gprat_cu_test_multiserver_fail_copy(gprat_cu_multiserver *server, int replica);
#define GPRAT_CU_REPLICATE_COPY 0
#define GPRAT_CU_REPLICATE_REFIT 1
int gprat_cu_multiserver_set_replication(gprat_cu_multiserver *server, int mode);

#ifdef __cplusplus
}
#endif

#endif /* GPRAT_CU_H */
