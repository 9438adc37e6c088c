// BF16 tensor-core products and the conversions feeding them (the
// mixed-precision sketch).
#pragma once
#include "common.cuh"

namespace mb {

// D (M x N) = (A_hi + A_lo + A_lo2) * B', all BF16 K-major (row pitch in
// elements, multiple of 8), FP32 accumulation on tcgen05; D is FP64
// (out_fp64) or FP32 row-major with leading dimension ldd.  a_lo, a_lo2 may
// be null (fewer parts; a_lo2 only with a_lo).  Device-side wait timeouts
// are reported in c->scal->status.
// accumulate: D += the product (FP64 D read back); lower: M == N and only the
// tiles touching the lower triangle are computed (the others are left as they are).
int bf16_gemm(Context* c, int64_t M, int64_t N, int64_t K, const uint16_t* a_hi, const uint16_t* a_lo,
              const uint16_t* a_lo2, int64_t lda, const uint16_t* b, int64_t ldb, void* D, int64_t ldd, bool out_fp64,
              bool accumulate = false, bool lower = false);

// Split-K plan of a bf16_gemm_split call: split z accumulates k-tiles
// [z kt_per, min(KT, (z + 1) kt_per)) into its own D slice (D + z split_stride
// elements); the slices are added afterwards by launch_sum_splits in a fixed
// order.  chunked forces the chunked configuration (FP64 sums of FP32 chunks)
// whatever the number of parts.
struct Bf16Split {
  int splits = 1;
  int kt_per = 0;
  int64_t split_stride = 0;
  bool chunked = false;
  int chunk_kt = 0;   // k-tiles per FP32 chunk in the chunked configuration (0: the default, 3)
};
int bf16_gemm_split(Context* c, int64_t M, int64_t N, int64_t K, const uint16_t* a_hi, const uint16_t* a_lo,
                    const uint16_t* a_lo2, int64_t lda, const uint16_t* b, int64_t ldb, void* D, int64_t ldd,
                    bool out_fp64, bool accumulate, bool lower, const Bf16Split& sp);
Bf16Split plan_bf16_split(const Context* c, int64_t M, int64_t N, int64_t K, bool chunked, int max_splits);
// D := scale x the sum over z of P + z stride (M x N, pitch ldp), added in
// order z = 0, 1, ...; with groups > 1 each slice contributes its column
// blocks [g group_cols, g group_cols + N) for g = 0 .. groups-1 (in order).
// D is written N x M when transpose.  Honours the context's iteration guard.
int launch_sum_splits(Context* c, const double* P, int splits, int64_t stride, int64_t M, int64_t N, int64_t ldp,
                      double* D, int64_t ldd, bool transpose, double scale = 1.0, int groups = 1,
                      int64_t group_cols = 0);

// hi := bf16(A), lo := bf16(A - hi), lo2 := bf16(A - hi - lo) (lo, lo2 may be
// null), written row-major (K contiguous) with pitch ldo, from row-major
// (layout 0) or column-major (layout 1) FP64 A.
int launch_split_bf16(Context* c, const double* A, int layout, int64_t lda, int64_t m, int64_t n, uint16_t* hi,
                      uint16_t* lo, uint16_t* lo2, int64_t ldo);
// The same from FP32 A (the parts of its exact FP64 copy).
int launch_split_bf16_f32(Context* c, const float* A, int layout, int64_t lda, int64_t m, int64_t n, uint16_t* hi,
                          uint16_t* lo, uint16_t* lo2, int64_t ldo);

// Omega' in BF16 (L x n, pitch ldo) from the same Philox stream as the FP64
// generator (element (i, j) of the n x L Omega is sample i L + j), rounded to
// BF16; omega (n x L FP64, optional) receives the same rounded values.
int launch_gaussian_bf16(Context* c, uint64_t seed, int64_t n, int64_t L, uint16_t* omega_t, int64_t ldo,
                         double* omega);

}  // namespace mb
