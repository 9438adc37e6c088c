// FP64 GEMM on the sm_100a double-precision MMA (mma.sync m8n8k4 f64), the
// arithmetic core of the plain FP64 iSVD path.  tcgen05 has no f64 kind, so
// the FP64 path runs on DMMA; operand tiles are staged global -> shared memory
// with cp.async in a multi-stage pipeline.
//
//   C(M x N) := alpha * A(M x K) * B(K x N) + beta * C
//
// A, B, C are strided views (element (i, j) at p[i*rs + j*cs]).  Each of A and
// B must have one unit stride; the kernel is specialised on which one.
// Batched calls add a per-batch element stride to every pointer.  Split-K
// (over the K = m reductions of tall-skinny products) writes raw partial tiles
// to a workspace and reduces them in a fixed order, so results are
// deterministic run to run.
#pragma once
#include "common.cuh"

namespace mb {

struct GemmBatch {
  int count = 1;
  int64_t a = 0, b = 0, c = 0;   // element strides between batch members
};

// Bytes of workspace dgemm() needs for this shape (0 when no split-K is used).
size_t dgemm_workspace_bytes(const Context* c, int64_t M, int64_t N, int64_t K, int batch);
// The split-K count the shape heuristic picks for this product (1: none).  Every
// element's sum depends only on K and this count, not on M, so row blocks of a
// product computed with the same count equal the rows of the whole product.
int dgemm_heuristic_splits(const Context* c, int64_t M, int64_t N, int64_t K, int batch);

// Launches C := alpha*A*B + beta*C on ctx->stream.  ws may be null when
// dgemm_workspace_bytes() is 0.  force_splits > 0 overrides the split choice
// (tests use it to cover the split-K path at small sizes).  lower_only: C is
// square and only its lower triangle is needed (SYRK-like: tiles strictly
// above the diagonal are skipped and the elements above it are unspecified).
int dgemm(Context* ctx, int64_t M, int64_t N, int64_t K, double alpha, CMat A, CMat B, double beta, DMat C,
          GemmBatch batch = GemmBatch(), double* ws = nullptr, int force_splits = 0, bool lower_only = false);

// C := A B where C holds the same rows as A (an in-place update of A's row
// panels, e.g. Q_i := Q_i T_i): run only when one CTA covers all N output
// columns of its rows with no split-K, so that it has read its rows of A
// before it writes them; otherwise MCNLA_B200_ERR_UNSUPPORTED (nothing runs).
// The element arithmetic is that of dgemm() with the same shape.
int dgemm_rows_in_place(Context* ctx, int64_t M, int64_t N, int64_t K, CMat A, CMat B, DMat C,
                        GemmBatch batch = GemmBatch());

}  // namespace mb
