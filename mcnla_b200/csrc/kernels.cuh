// Launchers of the small and elementwise kernels the stages compose (the
// large products go through dgemm()).  Every launcher enqueues on
// ctx->stream and returns a status.
#pragma once
#include "common.cuh"

namespace mb {

// Eigendecomposition of `batch` symmetric n x n matrices A (row stride lda,
// batch stride a_bs): eigenvalues to W (batch stride n), eigenvectors as the
// columns of V (row-major n x n, batch stride n*n).  order 0: ascending;
// order 1: descending by |lambda| with W = |lambda| (gesvd of a PSD matrix).
int launch_syev(Context* c, int n, int batch, const double* A, int64_t lda, int64_t a_bs, double* W, double* V,
                int order);

// Scales the columns of V (row-major n x n, batch) by 1/sqrt(W): T = V diag(W^-1/2)
// (the orthogonalizer's Q_i := Y_i V_i S_i^-1/2 step).
int launch_scale_cols_rsqrt(Context* c, int n, int batch, const double* V, const double* W, double* T);

// Kolmogorov-Nagumo l x l step (one CTA).
//   plain (dd == nullptr): Z given (l x l) -> out = [C; inv(C)] (2l x l)
//   row-block: dd = [Dc | Dgc] (l x 2l), Z := Dgc - Dc Dc' ->
//       out  = [Fc; inv(C)], Fc = C - Dc inv(C)
//       outn = [Fc; inv(C)/N]          (optional)
//       ffn  = ff * Fc                 (optional, ff/ffn l x l)
// scal->norm := || s - 1 ||_2, s = sqrt(1/2 + sqrt(1/4 - eig(Z))).
// vwork: kn_series_work_doubles(l) doubles of global scratch.
// Method (mcnla_b200_set_kn_method): KN_AUTO runs the series kernel and, for
// the iterations it declines, the Newton-Schulz kernel (its matrices in shared
// memory for l <= 80, in vwork above), and the eigendecomposition only where
// Newton-Schulz fails; KN_NEWTON_SCHULZ starts at Newton-Schulz; KN_EIGEN
// always uses the eigendecomposition.
// When the context's iteration guard is set, the step is skipped for an
// iteration past convergence, and scal->stop_it is set to the guard
// iteration when ||s - 1||_2 < tol fails to hold as "norm >= tol" (a NaN norm
// converges, like the reference's !(nrm2 >= tol)).
int launch_kn_step(Context* c, int l, const double* z, const double* dd, double inv_n, double* out, double* outn,
                   const double* ff, double* ffn, double* vwork, double tol, bool allow_series = true);
// Global scratch (doubles) the KN step needs in vwork.
size_t kn_series_work_doubles(int l);
// The series form of the step on ceil(l/8) cooperative CTAs (kn_series.cu);
// same operands as launch_kn_step.  Sets scal->kn_fallback when ||Z|| is too
// large for the series; the launcher then runs the other form after it.
int launch_kn_series(Context* c, int l, const double* z, const double* dd, double inv_n, double* out, double* outn,
                     const double* ff, double* ffn, double* work, double tol);
// Persistent row-block Gramian KN integrator (gkn_persistent.cu): runs
// iterations [it0, maxit) of one problem on one cooperative grid (the single
// solve: lowest latency).  On return (after a stream sync) scal->stop_it is the
// converged iteration, or scal->resume_it the iteration whose KN step the
// series declined (to be run by the caller with allow_series = false), or
// neither (maxit reached).  EB, FF, DD, FC, FCN, work: the buffers of the
// launch-per-product loop.
bool gkn_persistent_fits(const Context* c, int l, int64_t L);
int launch_gkn_persistent(Context* c, int l, int64_t L, int N, double tol, int it0, int maxit, const double* Bs,
                          double* const EB[2], double* const FF[2], double* DD, double* FC, double* FCN,
                          double* work);
// Grouped row-block Gramian KN integrator (gkn_grouped.cu): the iterations of
// many problems (a batch: highest throughput), a cluster of CTAs per problem
// from a device work queue.  A job's fields above stop_it are inputs (the buffers of the
// launch-per-product loop, plus cbuf: l x l doubles and ddp:
// gkn_grouped_ddp_doubles of scratch); after the launch stop_it is the
// converged iteration (INT_MAX: not converged), resume_it the iteration whose
// KN step the series declined (-1: none; the caller runs it on the
// launch-per-product path), else maxit was reached.
struct GknJob {
  int l, L, it0, maxit, smax, pad0;
  double inv_n, tol;
  const double* bs;
  double *eb0, *eb1, *ff0, *ff1, *dd, *fc, *fcn, *work, *cbuf, *ddp;
  int stop_it, resume_it;
  double norm;
  int degree, pad1;
  long long ns;     // out: nanoseconds the cluster spent on the job (device global timer)
  long long phase_ns[4];   // out: of which in P1 (Bs Bc), P2 ([Dc | Dgc]), the KN step, P4 (E~+, B+)
};
// Largest N l the grouped kernel takes (beyond it the launch-per-product loop's
// shared-memory-pipelined GEMMs are faster).
constexpr int64_t kGknGroupedMaxL = 1536;
bool gkn_grouped_fits(const Context* c, int l, int64_t L);
// Dynamic shared memory of a job with this l (0: l unsupported) and its power slabs.
size_t gkn_grouped_smem(const Context* c, int l);
int gkn_grouped_smax(const Context* c, int l);
size_t gkn_grouped_ddp_doubles(int l, int64_t L);
// Runs jobs_dev[0 .. njobs) (device memory) on clusters of `cluster` CTAs with
// `smem` bytes each (at least gkn_grouped_smem of every job's l); next_dev: one
// device int of scratch.
int launch_gkn_grouped(Context* c, GknJob* jobs_dev, int njobs, int* next_dev, size_t smem, int cluster);

// Opts a kernel in to the device's whole dynamic shared memory (once per
// device and kernel); fails when `bytes` exceeds it.
int set_smem(const Context* c, const void* fn, size_t bytes);

// Wen-Yin line-search trial (one CTA): from dd = [Dc | Dgc] and tau builds the
// 2l x 2l C, inverts it and writes F = [Fc; Fgc] (2l x l) and optionally
// FN = [Fc; Fgc * inv_n].
int launch_wy_trial(Context* c, int l, const double* dd, double tau, double inv_n, double* F, double* FN);

// Deterministic sums (two-stage, fixed order) into c->scal fields.
//   sumsq: scal->phit = scale * sum(X .* X) over a rows x cols strided block.
int launch_sumsq(Context* c, const double* X, int64_t rows, int64_t cols, int64_t ld, double scale, double* partials,
                 double* out);
//   dot: out = sum(X .* Y).
int launch_dot(Context* c, const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t rows, int64_t cols,
               double* partials, double* out);
//   wy deltas: d1 = Qc - Qp, d2 = Xc - Xp: out[0] = <d1,d1>, out[1] = <d1,d2>, out[2] = <d2,d2>.
int launch_wy_delta_dots(Context* c, const double* qc, const double* qp, int64_t ldq, const double* xc,
                         const double* xp, int64_t ldx, int64_t rows, int64_t cols, double* partials, double* out);
//   wy mu: out = sum |diag(Dgc)| - ||Dc||_F^2, dd = [Dc | Dgc] (l x 2l).
int launch_wy_mu(Context* c, int l, const double* dd, double* out);
// Number of partial sums the reductions above need.
int reduce_partials(const Context* c);

// Y := alpha X + beta Y on rows x cols strided blocks (beta == 0 ignores Y).
int launch_axpby(Context* c, int64_t rows, int64_t cols, double alpha, const double* X, int64_t ldx, double beta,
                 double* Y, int64_t ldy);
// Identity / zero helpers.
int launch_set_identity(Context* c, int64_t n, double* X, int64_t ld);
int launch_fill(Context* c, int64_t rows, int64_t cols, double v, double* X, int64_t ld);
// Gramian integrators: Bs := lower(Bs) mirrored; Bc := Bs(:, 0:l) with the
// strict upper triangle of its top l x l block zeroed.
int launch_gramian_prepare(Context* c, int64_t L, int l, double* bs, double* bc, int64_t ldbc);
// Wen-Yin Gramian helpers: phi1 = Fc - I; phi2 = Dc - Fc D+ (l x l).
int launch_wy_gramian_phis(Context* c, int l, const double* F, const double* dc, int64_t lddc, const double* dp,
                           int64_t lddp, double* phi1, double* phi2);

// SVD of one n x n row-major matrix M by one-sided (Hestenes) Jacobi:
// M = W diag(sig) Z', sig descending; W, Z row-major n x n.  Columns of W
// belonging to a zero singular value are returned as zero.
int launch_svd_small(Context* c, int n, const double* M, double* W, double* sig, double* Z);
// P := diag(w^-1/2) Ue' for the eigenpairs (w descending, Ue columns) of a
// Gram matrix; rows whose w_i <= (n eps)^2 w_0 are set to zero.
int launch_rsqrt_rows_t(Context* c, int n, const double* Ue, const double* w, double* P);
// Y(:, j) := X(:, j) * f(s_j) for j < cols; mode 0: f = 1/s, mode 1: f = s, mode 2: f = 1/sqrt(s).
int launch_scale_cols(Context* c, int64_t rows, int64_t cols, const double* X, int64_t ldx, const double* s,
                      int mode, double* Y, int64_t ldy);
// out[j] := sqrt(w[j]) for j < n.
int launch_sqrt_vec(Context* c, int n, const double* w, double* out);
// The l x l dot products of the Gramian Wen-Yin step size into out[0..6]:
// <P1,P1> <P1,P2> <P2,P2> <P1,BU1> <P1,BU2> <P2,BU1> <P2,BU2>, with
// bcu = [Bc'U1 | Bc'U2] (l x 2l).
int launch_gwy_small_dots(Context* c, int l, const double* phi1, const double* phi2, const double* bcu, double* out);

// In-place inverse of `batch` row-major n x n matrices (consecutive), one CTA
// each; a zero pivot sets scal->status to MCNLA_B200_ERR_SINGULAR.
int launch_inverse(Context* c, int n, int batch, double* A);

// Philox-4x32-10 + Box-Muller normal samples.
int launch_gaussian(Context* c, uint64_t seed, int64_t count, double* out);

}  // namespace mb
