/*
 * mcnla_b200: the C ABI of a B200-native integrated randomized SVD (iSVD).
 *
 * It covers one pipeline of MCNLA 0.7.2 (emfomy/mcnla): Gaussian-projection
 * sketching -> Gramian orthogonalization -> Kolmogorov-Nagumo or Wen-Yin
 * integration -> SVD forming.  Each entry point below replaces the `runImpl`
 * of one reference stage (cited per function; paths are relative to the
 * reference project root).  The reference's MPI decomposition over sketches
 * and row blocks collapses into on-device batching on one GPU, so the
 * "row-block" and "column-block" variants differ here only in the layout of A
 * and in the algorithm the stage runs, never in a collective.
 *
 * Conventions
 *   - All matrix pointers are DEVICE pointers to double (FP64) unless stated.
 *   - A is m x n, row-major (MCNLA_B200_ROW_MAJOR, leading dimension lda >= n)
 *     or column-major (MCNLA_B200_COL_MAJOR, lda >= m).
 *   - The sketch collection Q is "unfolded": one row-major m x (N*l) matrix
 *     whose column block i is sketch i (the reference's
 *     DenseMatrixCollectionColBlockRowMajor,
 *     include/mcnla/core/matrix/collection/dense/dense_matrix_collection_col_block.hpp:44-55).
 *   - Q-bar is row-major m x l; U is row-major m x k; V is row-major n x k;
 *     S holds the k leading singular values in descending order.
 *   - Every function returns MCNLA_B200_OK (0) or an error status; none aborts.
 *     The reference has no error returns (it asserts); see
 *     mcnla_b200_status_string() for the meanings.
 *   - Work is enqueued on the context's stream.  Functions that must read a
 *     device result to decide what to do next (the integrators' convergence
 *     tests) synchronize that stream; all others return without waiting.
 */
#ifndef MCNLA_B200_H_
#define MCNLA_B200_H_

#include <stdint.h>

#if defined(__GNUC__)
#define MCNLA_B200_API __attribute__((visibility("default")))
#else
#define MCNLA_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define MCNLA_B200_OK                  0
#define MCNLA_B200_ERR_SHAPE           1  /* sizes non-positive, inconsistent or over a limit */
#define MCNLA_B200_ERR_LAYOUT          2  /* a strided operand without a unit stride */
#define MCNLA_B200_ERR_WORKSPACE       3  /* internal: a split-K GEMM was given no workspace */
#define MCNLA_B200_ERR_CUDA            4  /* a CUDA runtime call failed (see mcnla_b200_last_error) */
#define MCNLA_B200_ERR_NOMEM           5  /* device allocation failed */
#define MCNLA_B200_ERR_ARG             6  /* null pointer or invalid enumerator */
#define MCNLA_B200_ERR_UNSUPPORTED     7  /* shape beyond a kernel's stated limit (e.g. l > 160) */
#define MCNLA_B200_ERR_SINGULAR        8  /* exact zero pivot in a small inverse */
#define MCNLA_B200_ERR_DEVICE_TIMEOUT  9  /* a bounded device-side wait ran out (results invalid) */
#define MCNLA_B200_ERR_IO             10  /* a file is missing, unreadable, or not in the expected format */

/* ---- enumerators -------------------------------------------------------- */
#define MCNLA_B200_ROW_MAJOR 0
#define MCNLA_B200_COL_MAJOR 1

/* Integrators (include/mcnla/isvd/integrator/) */
#define MCNLA_B200_KOLMOGOROV_NAGUMO                   0  /* kolmogorov_nagumo_integrator.hpp */
#define MCNLA_B200_ROW_BLOCK_KOLMOGOROV_NAGUMO         1  /* row_block_kolmogorov_nagumo_integrator.hpp */
#define MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO 2  /* row_block_gramian_kolmogorov_nagumo_integrator.hpp */
#define MCNLA_B200_ROW_BLOCK_WEN_YIN                   3  /* row_block_wen_yin_integrator.hpp */
#define MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN           4  /* row_block_gramian_wen_yin_integrator.hpp */

/* Formers (include/mcnla/isvd/former/) */
#define MCNLA_B200_SVD_FORMER                0  /* svd_former.hpp (with V) */
#define MCNLA_B200_GRAMIAN_FORMER            1  /* gramian_former.hpp (with V) */
#define MCNLA_B200_ROW_BLOCK_GRAMIAN_FORMER  2  /* row_block_gramian_former.hpp (with V) */
#define MCNLA_B200_COL_BLOCK_GRAMIAN_FORMER  3  /* col_block_gramian_former.hpp (with V) */

/* Largest sketch dimension l = k + p the small on-chip solvers accept. */
#define MCNLA_B200_MAX_DIM_SKETCH        160
#define MCNLA_B200_MAX_DIM_SKETCH_WENYIN 80

/* ---- parameters ----------------------------------------------------------
 * Mirror of mcnla::isvd::Parameters<_Val>::params_
 * (include/mcnla/isvd/core/parameters.hh:54-69): number of rows/columns of A,
 * desired rank k, oversampling p (reference default 12) and number of
 * sketches N (reference default 16).  dimSketch l = k + p.                     */
typedef struct mcnla_b200_params {
  int64_t nrow;
  int64_t ncol;
  int64_t rank;
  int64_t over_rank;
  int64_t num_sketch;
} mcnla_b200_params;

typedef struct mcnla_b200_ctx mcnla_b200_ctx;

/* ---- context -------------------------------------------------------------
 * Replaces mcnla::init()/gpuInit (include/mcnla/core/def.hpp:42-61,
 * include/mcnla/core_gpu/def.hpp:42-47): binds one device and one stream.
 * stream is a cudaStream_t; NULL means CUDA's default stream.  The context
 * never destroys the stream it is given.                                     */
MCNLA_B200_API int mcnla_b200_create(mcnla_b200_ctx** ctx, int device, void* stream);
MCNLA_B200_API int mcnla_b200_destroy(mcnla_b200_ctx* ctx);
MCNLA_B200_API int mcnla_b200_set_stream(mcnla_b200_ctx* ctx, void* stream);
MCNLA_B200_API const char* mcnla_b200_status_string(int status);
/* Text of the last CUDA error (thread-local). */
MCNLA_B200_API const char* mcnla_b200_last_error(void);
/* Number of kernels this context has launched (for launch accounting). */
MCNLA_B200_API int64_t mcnla_b200_kernels_launched(const mcnla_b200_ctx* ctx);
/* Chunks of KN iterations this context ran as a replayed CUDA graph. */
MCNLA_B200_API int64_t mcnla_b200_graph_replays(const mcnla_b200_ctx* ctx);

/* Kolmogorov-Nagumo step method.  The reference forms C = f(Z) and inv(C)
 * from an eigendecomposition of Z (row_block_kolmogorov_nagumo_integrator.hpp:159-180).
 * MCNLA_B200_KN_AUTO (default) evaluates the same matrix functions as power
 * series in Z on the FP64 MMA of ceil(l/8) CTAs when 4 ||Z||_F <= 1/2 (all
 * but the first iterations), else by coupled Newton-Schulz iterations
 * (l <= 80) or the eigendecomposition.  MCNLA_B200_KN_NEWTON_SCHULZ skips the
 * series; MCNLA_B200_KN_EIGEN always uses the eigendecomposition (parallel
 * Jacobi).                                                                   */
/* GEMM tile autotuner (on by default): the first call of an FP64 product of
 * at most 5 GFLOP inside an integrator's iteration loop (where the shape then
 * repeats every iteration) times every tile configuration and split-K count
 * that its workspace allows, on the call's own operands into a scratch
 * output, and keeps the fastest for the rest of the process (shared by all
 * contexts, so a shape always runs the same configuration).  Other products,
 * and all products when off, use a fixed shape heuristic.                    */
MCNLA_B200_API int mcnla_b200_set_autotune(mcnla_b200_ctx* ctx, int on);
/* CUDA-graph iteration loops (on by default): the Kolmogorov-Nagumo
 * integrators that launch their products per iteration (kolmogorov_nagumo_
 * integrator.hpp:109-183 and the row-block forms) run the first chunk of 8
 * iterations as ordinary launches, capture the next chunk once as a CUDA
 * graph and replay it for every later full chunk; results are bit-identical
 * either way.  Off: every iteration is launched.                             */
MCNLA_B200_API int mcnla_b200_set_graph_loop(mcnla_b200_ctx* ctx, int on);

/* SM share of the context's persistent cooperative kernels (the row-block
 * Gramian KN integrator): at most `ctas` CTAs, 0 = one per SM.  For callers
 * that run several contexts side by side on one GPU (the server sets it to
 * SMs / workers for each worker's context).                                 */
MCNLA_B200_API int mcnla_b200_set_cta_limit(mcnla_b200_ctx* ctx, int ctas);

#define MCNLA_B200_KN_AUTO  0
#define MCNLA_B200_KN_EIGEN 1
#define MCNLA_B200_KN_NEWTON_SCHULZ 2
MCNLA_B200_API int mcnla_b200_set_kn_method(mcnla_b200_ctx* ctx, int method);

/* Stage timers: seconds per part of the last stage call, the reference's
 * StageWrapper::times() (include/mcnla/isvd/core/stage_wrapper.hpp:128-135),
 * measured with CUDA events.  Synchronizes the stream.  Returns the number of
 * parts written (at most capacity) or a negative status.                     */
MCNLA_B200_API int mcnla_b200_last_times(mcnla_b200_ctx* ctx, double* times, int capacity);

/* Pre-allocates the workspaces a pipeline with these parameters, integrator
 * and former will use, like StageWrapper::initialize()
 * (include/mcnla/isvd/core/stage_wrapper.hpp:37-46).  Optional: stages grow
 * the workspace on first use otherwise.                                      */
MCNLA_B200_API int mcnla_b200_initialize(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former);

/* ---- sketcher ------------------------------------------------------------
 * Q := A * Omega on the unfolded collection, then `exponent` power
 * iterations (Omega := A' Q; Q := A Omega).  Replaces
 * GaussianProjectionSketcher::runImpl
 * (include/mcnla/isvd/sketcher/gaussian_projection_sketcher.hpp:65-103), its
 * row-block (row_block_gaussian_projection_sketcher.hpp:65-114) and
 * column-block (col_block_gaussian_projection_sketcher.hpp:63-102) variants.
 * omega: n x (N*l) row-major; it is overwritten when exponent > 0.           */
MCNLA_B200_API int mcnla_b200_sketch(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, const double* A, int a_layout,
                      int64_t lda, double* omega, int exponent, double* Q);

/* Fills out[0..count) with N(0,1) samples from a counter-based generator
 * (Philox-4x32-10 + Box-Muller) keyed by seed; the on-device stand-in for
 * random::gaussian (include/mcnla/core/random/routine/gaussian.hpp:39-56).
 * The same (seed, count) always gives the same values.                       */
MCNLA_B200_API int mcnla_b200_gaussian(mcnla_b200_ctx* ctx, uint64_t seed, int64_t count, double* out);

/* ---- orthogonalizer --------------------------------------------------------
 * In place on Q (m x N*l): W_i := Q_i' Q_i; eig(W_i) = V_i S_i V_i';
 * Q_i := Q_i V_i S_i^(-1/2), eigenvalues in descending order.  Replaces
 * GramianOrthogonalizer::runImpl
 * (include/mcnla/isvd/orthogonalizer/gramian_orthogonalizer.hpp:62-104) and
 * RowBlockGramianOrthogonalizer::runImpl
 * (row_block_gramian_orthogonalizer.hpp:62-105).                            */
MCNLA_B200_API int mcnla_b200_orthogonalize(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, double* Q);

/* ---- integrators -----------------------------------------------------------
 * Qbar := the integrated basis of the N orthonormal bases in Q.  kind is one
 * of the MCNLA_B200_*KOLMOGOROV_NAGUMO / *WEN_YIN enumerators; each runs the
 * algorithm of the reference stage named beside it.  *iteration receives the
 * number of iterations executed (the reference's iteration()).  Synchronizes
 * the stream.                                                                */
MCNLA_B200_API int mcnla_b200_integrate(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int kind, const double* Q,
                         int max_iteration, double tolerance, double* Qbar, int* iteration);

/* ---- formers ---------------------------------------------------------------
 * Rank-k SVD of A from Qbar: S (k), U (m x k), V (n x k).  kind is one of the
 * MCNLA_B200_*_FORMER enumerators.  Replaces SvdFormer<_,true>::runImpl
 * (include/mcnla/isvd/former/svd_former.hpp:70-116) and the Gramian formers
 * (gramian_former.hpp:72-132, row_block_gramian_former.hpp:78-146,
 * col_block_gramian_former.hpp:73-131).  U or V may be NULL to skip them.     */
MCNLA_B200_API int mcnla_b200_form(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int kind, const double* A, int a_layout,
                    int64_t lda, const double* Qbar, double* S, double* U, double* V);

/* ---- whole solve -----------------------------------------------------------
 * Sketch -> orthogonalize -> integrate -> form, as the reference drivers wire
 * the stages (src/isvd_dense_rb.cpp:46-286, src/isvd_dense_cb.cpp:46-303).
 * mcnla_b200_isvd takes device buffers; omega may be NULL to draw it on the
 * device from seed.  mcnla_b200_isvd_host takes HOST buffers (A, omega, S, U,
 * V) and does the host<->device copies itself, the path of the reference's
 * GPU drivers (src/isvd_dense_rb_gpu.cpp).                                    */
MCNLA_B200_API int mcnla_b200_isvd(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former,
                    const double* A, int a_layout, int64_t lda, const double* omega, uint64_t seed,
                    int max_iteration, double tolerance, double* S, double* U, double* V, int* iteration);
MCNLA_B200_API int mcnla_b200_isvd_host(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former,
                         const double* A_host, int a_layout, const double* omega_host, int max_iteration,
                         double tolerance, double* S_host, double* U_host, double* V_host, int* iteration);
/* Streamed ingest: the whole solve of a row-major A that the caller produces
 * row block by row block, e.g. from a file (the reference's row-block
 * loaders, include/mcnla/core/io/binary/dense_load.hpp:70-141 and
 * matrix_market/dense_load_block.hpp, read into a host matrix before its
 * stages start).  read_rows(user, row0, rows, buf) fills buf (rows x ncol,
 * row-major, pinned host memory the library owns) with rows [row0, row0 +
 * rows) of A and returns 0, or non-zero to abort the solve
 * (MCNLA_B200_ERR_ARG).  Rows come in order, in blocks of at least 128 rows
 * (about 1 GB at most, at least four blocks); while the device copies block
 * b and sketches it, the caller reads block b + 1.  A stays on the device
 * for the former.  The result is bit-identical to mcnla_b200_isvd_host's on
 * the same A and Omega.                                                      */
typedef int (*mcnla_b200_read_rows_fn)(void* user, int64_t row0, int64_t rows, double* buf);
MCNLA_B200_API int mcnla_b200_isvd_stream(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator,
                                          int former, mcnla_b200_read_rows_fn read_rows, void* user,
                                          const double* omega_host, int max_iteration, double tolerance,
                                          double* S_host, double* U_host, double* V_host, int* iteration);

/* ---- files (the reference's io module; host only, no device work) -----------
 * Dense MatrixMarket "array" text (include/mcnla/core/io/matrix_market/
 * dense_load.hpp:70-251, dense_load_block.hpp, dense_save.hpp): '%' lines,
 * then "m n" (a matrix) or "m n l" (a 3-D collection of l m x n matrices),
 * then the values column-major, matrix after matrix.  A collection is read
 * and written as its unfolded m x (n l) matrix (matrix k = columns
 * [k n, (k + 1) n)), the layout of mcnla_b200_sketch's Q.                      */
/* dims[0..2] := m, n, l (l = 1 for a matrix); *ndim := 2 or 3.               */
MCNLA_B200_API int mcnla_b200_mm_size(const char* path, int64_t* dims, int* ndim);
/* Rows [row0, row0 + rows) x columns [col0, col0 + cols) of the (unfolded)
 * matrix into out, row-major (layout 0) or column-major (1) with leading
 * dimension ldo: the whole matrix, a row block (loadMatrixMarketRowBlock,
 * dense_load_block.hpp:86-130) or a column block (loadMatrixMarketColBlock,
 * :31-74).                                                                   */
MCNLA_B200_API int mcnla_b200_mm_load(const char* path, int64_t row0, int64_t rows, int64_t col0, int64_t cols,
                                      double* out, int64_t ldo, int layout);
/* Writes the unfolded m x (n nmat) matrix a (row- or column-major, leading
 * dimension lda) as a matrix (nmat = 1) or a 3-D collection, values as the
 * reference writes them (scientific, 16 digits after the point: exact for
 * doubles); comment (optional, one line) follows the banner.                  */
MCNLA_B200_API int mcnla_b200_mm_save(const char* path, const double* a, int64_t m, int64_t n, int64_t nmat,
                                      int64_t lda, int layout, const char* comment);
/* MCNLA dense binary files (include/mcnla/core/io/binary/dense_load.hpp:70-141,
 * dense_save.hpp; format in doxygen/tutorial/io/binary.dox:17-30): a 128-byte
 * header, int64 ndim, int64 dims[ndim], the values contiguous along dims[0]
 * (a column-major matrix has dims {m, n}; the reference's row-major matrix
 * {n, m}).  Size and value type ("R8", "R4", ...; 9 bytes with the NUL).      */
MCNLA_B200_API int mcnla_b200_binary_size(const char* path, int64_t* dims, int* ndim, char* val_type);
/* Slices [first, first + count) along the last dimension (each the product of
 * the other dims), converted to double (R8 or R4 files): a row block of a
 * row-major matrix, a column block of a column-major one
 * (loadBinaryRowBlock / ColBlock, binary/dense_load_block.hpp).              */
MCNLA_B200_API int mcnla_b200_binary_load(const char* path, int64_t first, int64_t count, double* out);
/* Writes a (dims[0] fastest) as an R8 dense binary file.                     */
MCNLA_B200_API int mcnla_b200_binary_save(const char* path, const double* a, int ndim, const int64_t* dims,
                                          const char* comment);

/* ---- mixed precision (BF16 tensor cores, tcgen05) ---------------------------
 * The sketch A * Omega is where the plain FP64 path spends most of its time.
 * The mixed path keeps A as two or three BF16 parts, A = A_hi + A_lo (+
 * A_lo2): 16 or 24 bits of mantissa (three parts hold an FP32 A exactly),
 * draws Omega directly in BF16, and runs the sketch on the tcgen05 tensor
 * cores with FP32 accumulation; large Gramian-integrator products and, when
 * BF16 parts of A' are given, the former's product run there too, and every
 * small factorization stays FP64.  BF16 buffers are uint16_t bit patterns,
 * K-major (row pitch a multiple of 8 elements, 16-byte aligned base).        */

/* hi := bf16(A), lo := bf16(A - hi), lo2 := bf16(A - hi - lo) (lo, lo2 may be
 * NULL), row-major m x n with pitch ldo, from FP64 A (row- or column-major). */
MCNLA_B200_API int mcnla_b200_split_bf16(mcnla_b200_ctx* ctx, const double* A, int a_layout, int64_t lda, int64_t m,
                                         int64_t n, uint16_t* hi, uint16_t* lo, uint16_t* lo2, int64_t ldo);
/* Omega' (L x n, pitch ldo) in BF16 from the stream of mcnla_b200_gaussian
 * (element (i, j) of the n x L Omega is sample i*L + j) rounded to BF16;
 * omega (optional, n x L FP64) receives the same rounded values.            */
MCNLA_B200_API int mcnla_b200_gaussian_bf16(mcnla_b200_ctx* ctx, uint64_t seed, int64_t n, int64_t L,
                                            uint16_t* omega_t, int64_t ldo, double* omega);
/* D (M x N, FP64 when out_fp64 else FP32, pitch ldd) := (A_hi + A_lo + A_lo2) B'
 * with A_* M x K and B N x K BF16 K-major; a_lo, a_lo2 may be NULL (a_lo2
 * only with a_lo).  Synchronizes.                                            */
MCNLA_B200_API int mcnla_b200_gemm_bf16(mcnla_b200_ctx* ctx, int64_t M, int64_t N, int64_t K, const uint16_t* a_hi,
                                        const uint16_t* a_lo, const uint16_t* a_lo2, int64_t lda, const uint16_t* b,
                                        int64_t ldb, void* D, int64_t ldd, int out_fp64);
/* Mixed-precision sketch: Q (m x N l, FP64) := (A_hi + A_lo + A_lo2) * Omega
 * with Omega' given in BF16 (L x n, pitch ldo).  Synchronizes.               */
MCNLA_B200_API int mcnla_b200_sketch_bf16(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, const uint16_t* a_hi,
                                          const uint16_t* a_lo, const uint16_t* a_lo2, int64_t lda16,
                                          const uint16_t* omega_t, int64_t ldo, double* Q);
/* Precision-form former (svd_former.hpp:70-116, gramian_former.hpp:72-132):
 * the product Q' A (l x n) that the former takes from A runs on tcgen05 from
 * the BF16 parts of A' (n x m, pitch ldat: mcnla_b200_split_bf16 of A read
 * with the other layout, e.g. row-major A as a column-major n x m matrix) and
 * a three-part split of Qbar, the rest of the former in FP64.  Three parts of
 * A' keep the former's products to 2^-24; at_lo, at_lo2 may be NULL.
 * Synchronizes.                                                              */
MCNLA_B200_API int mcnla_b200_form_bf16(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int former,
                                        const uint16_t* at_hi, const uint16_t* at_lo, const uint16_t* at_lo2,
                                        int64_t ldat, const double* Qbar, double* S, double* U, double* V);
/* Whole solve with the mixed-precision sketch (Omega drawn in BF16 from seed),
 * FP64 orthogonalizer and integrator steps (the Gramian integrators form
 * Qs' Qs from BF16 parts of Qs and re-orthonormalize Qbar once in FP64), and
 * the former in the precision form when at_hi is given (BF16 parts of A' as
 * in mcnla_b200_form_bf16; A may then be NULL), else in FP64 from A.  a_lo,
 * a_lo2, at_lo, at_lo2 may be NULL (fewer parts).                           */
MCNLA_B200_API int mcnla_b200_isvd_mixed(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator,
                                         int former, const double* A, int a_layout, int64_t lda, const uint16_t* a_hi,
                                         const uint16_t* a_lo, const uint16_t* a_lo2, int64_t lda16,
                                         const uint16_t* at_hi, const uint16_t* at_lo, const uint16_t* at_lo2,
                                         int64_t ldat, uint64_t seed, int max_iteration, double tolerance, double* S,
                                         double* U, double* V, int* iteration);

/* ---- batched and served solves ----------------------------------------------
 * Many independent solves of uneven sizes share the GPU.  (The reference runs
 * one problem per MPI job; this has no counterpart there.)
 *   mcnla_b200_server_* keeps a pool of workers (each with its own stream and
 *   workspaces) for requests that arrive over time: a request is admitted when
 *   a worker is free and the estimated device bytes of the requests in flight
 *   stay within the budget; the workers' solves overlap on the device.
 *   mcnla_b200_isvd_batched runs a whole batch through such a pool.
 *   mcnla_b200_isvd_grouped runs a batch in phases instead, in waves that fit
 *   the budget: the problems that use the row-block Gramian Kolmogorov-Nagumo
 *   integrator with N l <= 1536 are sketched, orthogonalized and given their
 *   Gramians by the workers; one grouped persistent kernel then runs every
 *   problem's iterations (a cluster of CTAs per problem from a device work
 *   queue, per-problem iteration counts); the workers finish Qbar and the
 *   formers.  Other problems run whole solves on the workers.
 * A itself is the caller's and is not counted.  Every solve is deterministic:
 * a problem gives the same bits alone, in a batch of the pool and in a served
 * mix; in a grouped batch it gives the same bits in any batch and agrees with
 * the single solve to rounding with the same iteration count (the grouped
 * kernel sums its products in its own fixed order).
 * Precisions: FP64 runs the plain path (an FP32 A is converted to FP64 on the
 * device for the sketch and the former).  The mixed precisions run the
 * precision form: the sketch on tcgen05 from BF16 parts of A, Omega drawn in
 * BF16, the orthogonalizer and the integrator's small factorizations in FP64,
 * and the former's product Q' A on tcgen05 from three BF16 parts of A'.  The
 * parts are split from A (FP32 or FP64) per solve, or read from the caller's
 * resident copies when a_hi / at_hi are given (mcnla_b200_split_bf16).     */
#define MCNLA_B200_PRECISION_FP64  0   /* FP64 sketch (plain path) */
#define MCNLA_B200_PRECISION_MIXED 1   /* BF16 hi+lo tcgen05 sketch, precision former */
#define MCNLA_B200_PRECISION_MIXED3 2  /* BF16 hi+lo+lo2 (24 bits: exact for FP32 A) */

typedef struct mcnla_b200_problem {
  mcnla_b200_params params;
  const double* A;        /* device, FP64; or NULL when A32 is given */
  const float* A32;       /* device, FP32 (converted on the worker's stream) */
  int a_layout;
  int64_t lda;
  uint64_t seed;          /* Omega is drawn on the device from this seed */
  int integrator, former, max_iteration;
  double tolerance;
  int precision;          /* MCNLA_B200_PRECISION_* */
  double* S;              /* device outputs: k, m x k, n x k (U, V may be NULL) */
  double* U;
  double* V;
  int iteration;          /* out */
  int status;             /* out */
  double seconds;         /* out: device time of the solve */
  double latency;         /* out: host seconds from submit (or the batch's start) to completion */
  /* mixed precisions, optional: the caller's resident BF16 parts of A
   * (row-major m x n, pitch lda16; a_lo2 for MIXED3) and of A' (n x m, pitch
   * ldat16, three parts); NULL a_hi / at_hi: split from A per solve.          */
  const uint16_t* a_hi;
  const uint16_t* a_lo;
  const uint16_t* a_lo2;
  int64_t lda16;
  const uint16_t* at_hi;
  const uint16_t* at_lo;
  const uint16_t* at_lo2;
  int64_t ldat16;
} mcnla_b200_problem;

typedef struct mcnla_b200_server mcnla_b200_server;

/* Device bytes a problem needs while in flight (workspaces and sketches).   */
MCNLA_B200_API int64_t mcnla_b200_problem_bytes(const mcnla_b200_problem* problem);
/* `workers` host threads, each with its own context and stream.  Admission
 * keeps the workers' device memory within budget_bytes: an idle worker counts
 * the workspaces it holds between solves, a running one the larger of those
 * and its problem's bytes; when the next problem does not fit while work is
 * running, idle workers release the workspaces they hold.                   */
MCNLA_B200_API int mcnla_b200_server_create(mcnla_b200_server** server, int device, int workers,
                                            int64_t budget_bytes);
/* Queues a copy of *problem; returns at once with a ticket.                  */
MCNLA_B200_API int mcnla_b200_server_submit(mcnla_b200_server* server, const mcnla_b200_problem* problem,
                                            int64_t* ticket);
/* Blocks until the ticket's problem is done and copies it (with iteration,
 * status, seconds and latency filled) to *out.  Each ticket can be waited on
 * once.                                                                      */
MCNLA_B200_API int mcnla_b200_server_wait(mcnla_b200_server* server, int64_t ticket, mcnla_b200_problem* out);
/* Estimated bytes of the problems in flight right now, and the most ever in
 * flight at once.                                                            */
MCNLA_B200_API int mcnla_b200_server_stats(mcnla_b200_server* server, int64_t* in_flight_bytes, int64_t* peak_bytes,
                                           int64_t* completed);
/* Finishes the queued work, stops the workers and frees everything.        */
MCNLA_B200_API int mcnla_b200_server_destroy(mcnla_b200_server* server);
/* All problems through a temporary server; returns the first non-zero status
 * (each problem's own status is in problems[i].status).                      */
MCNLA_B200_API int mcnla_b200_isvd_batched(int device, mcnla_b200_problem* problems, int count, int workers,
                                           int64_t budget_bytes);
/* All problems as a grouped batch (see above); same statuses.                */
MCNLA_B200_API int mcnla_b200_isvd_grouped(int device, mcnla_b200_problem* problems, int count, int workers,
                                           int64_t budget_bytes);
/* Seconds of the phases of the last mcnla_b200_isvd_grouped call in this
 * process (host clock): [0] sketch / orthogonalizer / Gramian of the grouped
 * problems, [1] the grouped integrator kernels, [2] the iterations they handed
 * back, [3] Qbar and the formers, [4] the other problems' whole solves; and
 * (device clock, summed over the grouped problems) [5] Bs Bc, [6] [Dc | Dgc],
 * [7] the KN step, [8] the E~ and B updates.  Returns the number of entries
 * (9); writes at most capacity.                                              */
MCNLA_B200_API int mcnla_b200_grouped_times(double* seconds, int capacity);

/* ---- row-block decomposition over several GPUs -------------------------------
 * The reference's MPI decomposition of one solve (src/isvd_dense_rb.cpp:118-221
 * with the row-block stages): every rank holds a block of rows of A, sketches
 * them with the same Omega, and keeps its rows of Q, Qbar and U; the stages
 * sum their row-dependent partial products over the ranks where the
 * reference calls MPI:
 *   orthogonalizer  W_i = sum_r Y_ir' Y_ir  (row_block_gramian_orthogonalizer.hpp:86)
 *   integrators     row-block KN: Bc once and Bgc per iteration
 *                   (row_block_kolmogorov_nagumo_integrator.hpp:115, :143);
 *                   Gramian KN / WY: Bs once (row_block_gramian_kolmogorov_
 *                   nagumo_integrator.hpp:117, row_block_gramian_wen_yin_
 *                   integrator.hpp:126); row-block WY: Bc, Bgc and per
 *                   iteration Bgc and the three step-size inner products
 *                   (row_block_wen_yin_integrator.hpp:117, :129, :229, :269);
 *                   plain KN: B = Qs' Qc and Z = X' X per iteration (the
 *                   reference distributes that integrator over sketches
 *                   instead, kolmogorov_nagumo_integrator.hpp:109-136)
 *   formers         Z = A' Qbar (Gramian) or Q' A (SVD former): the reference
 *                   reduce-scatters Z over column blocks and all-reduces W
 *                   (row_block_gramian_former.hpp:111, :121); here every rank
 *                   receives all of Z and returns all of V
 * Once a context has a communicator, every stage and whole-solve entry point
 * above runs on the rank's rows: params->nrow is the number of LOCAL rows,
 * A, Q, Qbar and U are the rank's row blocks, and S, V (and the iteration
 * count) come out the same on every rank.  All ranks must call the same
 * entry points with the same parameters (apart from nrow) in the same order.
 * The iteration loops run without CUDA-graph replay on such a context.
 *
 * mcnla_b200_allreduce_fn: sum `count` doubles at the DEVICE pointer buf over
 * the ranks, in place, ordered on `stream` (a cudaStream_t) like a kernel
 * launched there; return 0 on success.  NULL fn detaches.                    */
typedef int (*mcnla_b200_allreduce_fn)(void* user, double* buf, int64_t count, void* stream);
MCNLA_B200_API int mcnla_b200_set_allreduce(mcnla_b200_ctx* ctx, mcnla_b200_allreduce_fn fn, void* user);
/* The library's own NCCL communicator (NCCL over NVLink / NVSwitch; libnccl.so.2
 * is loaded on first use).  mcnla_b200_nccl_unique_id writes the 128-byte id
 * that rank 0 creates and every rank then passes to mcnla_b200_set_nccl, with
 * the context's device current (one GPU per rank).                           */
#define MCNLA_B200_NCCL_ID_BYTES 128
MCNLA_B200_API int mcnla_b200_nccl_unique_id(unsigned char* id);
MCNLA_B200_API int mcnla_b200_set_nccl(mcnla_b200_ctx* ctx, const unsigned char* id, int nranks, int rank);
/* Number of all-reduces this context has issued. */
MCNLA_B200_API int64_t mcnla_b200_allreduces(const mcnla_b200_ctx* ctx);

/* ---- building blocks (exposed for tests) ----------------------------------
 * FP64 GEMM C := alpha*A*B + beta*C on strided device matrices (element (i,j)
 * of X at X[i*x_rs + j*x_cs]); the reference's la::mm
 * (include/mcnla/core/la/dense/routine/gemm.hpp:35-148).  force_splits > 0
 * forces that many K splits.                                                  */
MCNLA_B200_API int mcnla_b200_dgemm(mcnla_b200_ctx* ctx, int64_t M, int64_t N, int64_t K, double alpha, const double* A,
                     int64_t a_rs, int64_t a_cs, const double* B, int64_t b_rs, int64_t b_cs, double beta, double* C,
                     int64_t c_rs, int64_t c_cs, int force_splits);

/* Batched symmetric eigendecomposition of `batch` row-major n x n matrices
 * (consecutive in A): eigenvalues to W (n per matrix), eigenvectors as the
 * columns of row-major V (n x n per matrix).  order 0 = ascending (dsyev,
 * include/mcnla/core/la/dense/driver/syev.hpp:150-160), 1 = descending by
 * absolute value (dgesvd of a symmetric positive semi-definite matrix,
 * gesvd.hpp:159-193).                                                        */
MCNLA_B200_API int mcnla_b200_syev_batched(mcnla_b200_ctx* ctx, int n, int batch, const double* A, double* W, double* V,
                            int order);

/* In-place inverse of `batch` row-major n x n matrices (consecutive in A),
 * the reference's getrfi (include/mcnla/core/la/dense/driver/getrfi.hpp:117-124).
 * n <= 2 * MCNLA_B200_MAX_DIM_SKETCH_WENYIN.                                 */
MCNLA_B200_API int mcnla_b200_inverse_batched(mcnla_b200_ctx* ctx, int n, int batch, double* A);

/* FP64 GEMM that allocates nothing (no counterpart in the reference; an
 * addition of this library).  For callers that cannot call cudaMalloc: a
 * plugin whose host framework owns the device memory pool, or a
 * latency-critical loop that cannot take the implicit synchronization of an
 * allocation.  Same operation and strides as mcnla_b200_dgemm, but it needs no
 * context: it runs on `stream` (NULL: the default stream) on the current
 * device, and keeps the split-K partial sums in a 16 MiB device array that
 * the library defines (held on every GPU that loads the library until the
 * process exits).  Every call looks that array's address up
 * (cudaGetSymbolAddress), so the entry point stays valid across a
 * cudaDeviceReset; the first call on each device may load the library's
 * module for that lookup, so make it before any stream capture (calls on a
 * capturing stream reuse the device's last looked-up address).
 * Shapes whose partial sums need more than MCNLA_B200_NOALLOC_SCRATCH_BYTES
 * are rejected with MCNLA_B200_ERR_SHAPE (mcnla_b200_last_error names the
 * size).  All calls on a device share the array: calls that overlap on the
 * GPU (other streams, other host threads) race; serialize them.            */
#define MCNLA_B200_NOALLOC_SCRATCH_BYTES (16u << 20)
MCNLA_B200_API int mcnla_b200_dgemm_noalloc(void* stream, int64_t M, int64_t N, int64_t K, double alpha,
                                            const double* A, int64_t a_rs, int64_t a_cs, const double* B,
                                            int64_t b_rs, int64_t b_cs, double beta, double* C, int64_t c_rs,
                                            int64_t c_cs);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* MCNLA_B200_H_ */
