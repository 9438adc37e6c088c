// CTA-level FP64 dense routines for the l x l (and 2l x 2l) steps of the iSVD
// stages: symmetric eigendecomposition (the reference calls LAPACK dsyev /
// dgesvd there, include/mcnla/core/la/dense/driver/syev.hpp:150-160,
// gesvd.hpp:159-193), matrix inversion (dgetrf + dgetri,
// include/mcnla/core/la/dense/driver/getrfi.hpp:117-124) and small products.
//
// One thread block owns one small problem.  The eigensolver is the cyclic
// two-sided Jacobi method with a round-robin (tournament) ordering, so the
// n/2 rotations of a round touch disjoint row/column pairs and run in
// parallel (Golub & Van Loan, Matrix Computations, 4th ed., sec. 8.5:
// Algorithm 8.5.2 for the 2 x 2 rotation, sec. 8.5.5 for the parallel
// ordering).  The inverse is Gauss-Jordan elimination with partial pivoting,
// done in place.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace mb {
namespace small {

// Round-robin pairing of P (even) players over P-1 rounds: pair 0 is
// (r, P-1); pair k >= 1 is ((r+k) mod (P-1), (r-k) mod (P-1)).  Every pair of
// distinct players meets exactly once per sweep.
__device__ __forceinline__ void rr_pair(int P, int r, int k, int& p, int& q) {
  if (k == 0) { p = r; q = P - 1; }
  else {                        // 0 <= r < P - 1 and 1 <= k < P / 2: one wrap at most
    p = r + k;
    if (p >= P - 1) p -= P - 1;
    q = r - k;
    if (q < 0) q += P - 1;
  }
  if (p > q) { int t = p; p = q; q = t; }
}

struct JacobiScratch {
  double2* cs;  // npairs: (cos, sin) of each pair's rotation
  int2* pq;     // npairs: the pair's indices (p < q)
  double* t;    // npairs (tangent, for the exact diagonal update)
  double* apq;  // npairs
  double* app;  // npairs
  double* aqq;  // npairs
  int* count;   // 1 (rotations applied this round)
  double* red;  // 32
};

// Frobenius norm^2 of the n x n matrix a (lda), all threads return it.
__device__ inline double cta_frob2(const double* a, int lda, int n, double* red) {
  double s = 0.0;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    double v = a[(e / n) * lda + (e % n)];
    s += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  double tot = 0.0;
  const int nw = (blockDim.x + 31) >> 5;
  for (int w = 0; w < nw; ++w) tot += red[w];
  __syncthreads();
  return tot;
}

// Eigendecomposition of the symmetric n x n matrix a (row stride lda, any
// memory space; shared memory is fastest).  On return diag(a) holds the
// eigenvalues (unsorted) and the ROWS of v (row stride ldv) the eigenvectors:
// v[k * ldv + i] is component i of eigenvector k (the transpose of the usual
// V, so that a rotation of two eigenvectors touches two contiguous rows, which
// matters when v lives in global memory).  When init_v is false, v must hold
// an orthogonal starting basis (rows) in which a is expressed (warm start);
// otherwise v is set to I.  Returns the number of sweeps.
//
// A round has two phases and two barriers: the angles (one thread per pair),
// then one update phase.  The rotations of a round act on disjoint index
// pairs, so a <- J' a J splits into 2 x 2 blocks (rows of pair K1, columns of
// pair K2) that depend only on their own four entries and the two pairs'
// rotations: each (K1, K2) block is one item (rows rotated first, then
// columns; the diagonal blocks are written exactly, J' B J = diag(app - t apq,
// aqq + t apq)).  The eigenvector rows of each pair are items of the same
// phase.  The rounds are latency-bound: launch it with many warps (1024
// threads) rather than give a thread several items' loads at once.
__device__ inline int cta_jacobi_eig(double* a, int lda, double* v, int ldv, int n, bool init_v,
                                     const JacobiScratch& js, int max_sweeps) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (init_v) {
    for (int e = tid; e < n * n; e += nt) v[(e / n) * ldv + (e % n)] = ((e / n) == (e % n)) ? 1.0 : 0.0;
  }
  __syncthreads();
  if (n <= 1) return 0;
  const int P = (n + 1) & ~1;
  const int npairs = P / 2;
  const double fro2 = cta_frob2(a, lda, n, js.red);
  // An off-diagonal entry is left alone when it is below eps * sqrt(|app aqq|)
  // (relative test) or below eps * ||A||_F (absolute floor: LAPACK's
  // eigensolvers are normwise accurate to that level, and below it rounding
  // in the rotations regenerates off-diagonal noise faster than a sweep
  // removes it).  Both tests compare squares.
  const double eps = 2.220446049250313e-16;
  const double eps2 = eps * eps;
  const double abs_floor = eps2 * fro2;
  // block items (K1, K2), K2 fastest, and eigenvector items (pair k, component i), i fastest:
  // thread tid takes e = tid, tid + nt, ..., walked with fixed increments
  const int b1_start = tid / npairs, b2_start = tid - b1_start * npairs;
  const int b1_step = nt / npairs, b2_step = nt - b1_step * npairs;
  const int k_start = tid / n, i_start = tid - k_start * n;
  const int k_step = nt / n, i_step = nt - k_step * n;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    int rotated = 0;
    for (int r = 0; r < P - 1; ++r) {
      // 1. angles, one thread per pair
      int mine = 0;
      for (int k = tid; k < npairs; k += nt) {
        int p, q;
        rr_pair(P, r, k, p, q);
        double c = 1.0, s = 0.0, t = 0.0, apq = 0.0, app = 0.0, aqq = 0.0;
        if (q < n) {
          apq = a[p * lda + q];
          app = a[p * lda + p];
          aqq = a[q * lda + q];
          const double apq2 = apq * apq;
          if (apq2 > eps2 * fabs(app * aqq) && apq2 > abs_floor) {
            // t = sgn(theta) / (|theta| + sqrt(1 + theta^2)), theta = d / g (d = aqq - app,
            // g = 2 apq), written as sgn(d) g / (|d| + sqrt(d^2 + g^2)): one division, one
            // square root and one reciprocal square root on the round's critical path.  t is
            // invariant under scaling d and g together, so entries far from 1 are scaled by
            // 2^-600 or 2^600 (exactly) before d^2 + g^2 could overflow or lose precision.
            double d = aqq - app, g = 2.0 * apq;
            const double mx = fmax(fabs(d), fabs(g));
            if (mx > 1e150) { d *= 0x1p-600; g *= 0x1p-600; }
            else if (mx < 1e-150) { d *= 0x1p600; g *= 0x1p600; }
            t = (d >= 0.0 ? g : -g) / (fabs(d) + sqrt(fma(d, d, g * g)));
            c = rsqrt(fma(t, t, 1.0));
            s = t * c;
            ++mine;
          } else {
            apq = 0.0;
          }
        }
        js.cs[k] = make_double2(c, s);
        js.pq[k] = make_int2(p, q);
        js.t[k] = t; js.apq[k] = apq; js.app[k] = app; js.aqq[k] = aqq;
      }
      // the barrier also counts the threads that set up a rotation
      const int cnt = __syncthreads_count(mine);
      if (cnt == 0) continue;
      rotated += cnt;
      // 2a. a <- J' a J by 2 x 2 blocks
      for (int k1 = b1_start, k2 = b2_start; k1 < npairs;) {
        const double2 cs1 = js.cs[k1], cs2 = js.cs[k2];
        const double s1 = cs1.y, s2 = cs2.y;
        if (s1 != 0.0 || s2 != 0.0) {
          const int2 pq1 = js.pq[k1], pq2 = js.pq[k2];
          const int p1 = pq1.x, q1 = pq1.y, p2 = pq2.x, q2 = pq2.y;
          if (k1 == k2) {
            const double ta = js.t[k1] * js.apq[k1];
            a[p1 * lda + p1] = js.app[k1] - ta;
            a[q1 * lda + q1] = js.aqq[k1] + ta;
            a[p1 * lda + q1] = 0.0;
            a[q1 * lda + p1] = 0.0;
          } else {
            // q1 / q2 is the padding index n of an odd n only in a pair that does not rotate
            const bool h1 = q1 < n, h2 = q2 < n;
            double xpp = a[p1 * lda + p2];
            double xpq = h2 ? a[p1 * lda + q2] : 0.0;
            double xqp = h1 ? a[q1 * lda + p2] : 0.0;
            double xqq = (h1 && h2) ? a[q1 * lda + q2] : 0.0;
            if (s1 != 0.0) {
              const double c1 = cs1.x;
              const double rpp = c1 * xpp - s1 * xqp, rqp = s1 * xpp + c1 * xqp;
              const double rpq = c1 * xpq - s1 * xqq, rqq = s1 * xpq + c1 * xqq;
              xpp = rpp; xqp = rqp; xpq = rpq; xqq = rqq;
            }
            if (s2 != 0.0) {
              const double c2 = cs2.x;
              const double ypp = c2 * xpp - s2 * xpq, ypq = s2 * xpp + c2 * xpq;
              const double yqp = c2 * xqp - s2 * xqq, yqq = s2 * xqp + c2 * xqq;
              xpp = ypp; xpq = ypq; xqp = yqp; xqq = yqq;
            }
            a[p1 * lda + p2] = xpp;
            if (h2) a[p1 * lda + q2] = xpq;
            if (h1) a[q1 * lda + p2] = xqp;
            if (h1 && h2) a[q1 * lda + q2] = xqq;
          }
        }
        k1 += b1_step;
        k2 += b2_step;
        if (k2 >= npairs) { k2 -= npairs; ++k1; }
      }
      // 2b. rows p, q of v
      for (int k = k_start, i = i_start; k < npairs;) {
        const double2 cs = js.cs[k];
        if (cs.y != 0.0) {
          const int2 pq = js.pq[k];
          const double vx = v[pq.x * ldv + i], vy = v[pq.y * ldv + i];
          v[pq.x * ldv + i] = cs.x * vx - cs.y * vy;
          v[pq.y * ldv + i] = cs.y * vx + cs.x * vy;
        }
        k += k_step;
        i += i_step;
        if (i >= n) { i -= n; ++k; }
      }
      __syncthreads();
    }
    if (rotated == 0) break;
  }
  return sweep;
}

// Scratch of cta_gj_inverse (shared memory).
constexpr int kGjMaxGroups = 32;
constexpr int kGjBatch = 2;
struct GjScratch {
  int* piv;        // n: the pivot position of each step
  double* col;     // 2 n: the pivot column, double-buffered across steps
  double* prow;    // n: the scaled pivot row
  double* cand_v;  // kGjMaxGroups: pivot candidates, one per row group
  int* cand_i;     // kGjMaxGroups
};

// In-place inverse of the n x n matrix a (row stride lda, n <= blockDim.x) by
// Gauss-Jordan elimination with partial pivoting: the same operations, pivots
// and rounding as the row-interchange form (pivot = first position of the
// largest |a(i, k)|, i >= k, as idamax; rows swapped, the pivot row scaled,
// every other row eliminated; the interchanges undone as column swaps at the
// end).  Each thread owns one column and every R-th row of it (R row groups,
// R = min(blockDim.x / n, kGjMaxGroups)), so a step takes two block barriers
// and no index division: (1) every thread picks the pivot from the candidates
// of the row groups, and one thread per column moves the old row k to the
// pivot's position and scales the pivot row into prow; (2) the elimination,
// in which the owners of column k+1 keep the new column and leave the next
// candidates.  Returns 0, or k+1 when the k-th pivot is exactly zero (the
// matrix is singular; a is then left partially reduced, as LAPACK's getri
// would refuse).  All threads return the same value.
__device__ inline int cta_gj_inverse(double* a, int lda, int n, const GjScratch& s) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int R = min(nt / n, kGjMaxGroups);
  const bool own = tid < R * n;
  const int j = own ? tid % n : 0, r0 = own ? tid / n : 0;
  if (own && j == 0) {
    double best = -1.0;
    int bi = 0;
    for (int i = r0; i < n; i += R) {
      const double v = a[i * lda];
      s.col[i] = v;
      if (fabs(v) > best) { best = fabs(v); bi = i; }
    }
    s.cand_v[r0] = best;
    s.cand_i[r0] = bi;
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const double* colk = s.col + (k & 1) * n;
    double* coln = s.col + ((k + 1) & 1) * n;
    double best = s.cand_v[0];
    int p = s.cand_i[0];
    for (int g = 1; g < R; ++g) {
      const double v = s.cand_v[g];
      const int i = s.cand_i[g];
      if (v > best || (v == best && i < p)) { best = v; p = i; }
    }
    const double pivot = colk[p];
    if (pivot == 0.0) return k + 1;
    const double inv = 1.0 / pivot;
    if (own && r0 == 0) {
      const double x = a[p * lda + j];
      s.prow[j] = (j == k) ? inv : x * inv;
      a[p * lda + j] = a[k * lda + j];
    }
    if (tid == 0) s.piv[k] = p;
    __syncthreads();
    if (own) {
      const double pj = s.prow[j];
      const double fk = colk[k];
      double nb = -1.0;
      int ni = k + 1;
      // rows in batches of kGjBatch: all loads of a batch before its stores, so they overlap
      for (int i0 = r0; i0 < n; i0 += kGjBatch * R) {
        double x[kGjBatch], f[kGjBatch];
#pragma unroll
        for (int u = 0; u < kGjBatch; ++u) {
          const int i = i0 + u * R;
          x[u] = 0.0;
          f[u] = 0.0;
          if (i < n) {
            x[u] = a[i * lda + j];
            f[u] = (i == p) ? fk : colk[i];
          }
        }
#pragma unroll
        for (int u = 0; u < kGjBatch; ++u) {
          const int i = i0 + u * R;
          if (i < n) {
            const double v = (i == k) ? pj : ((j == k) ? -f[u] * inv : x[u] - f[u] * pj);
            a[i * lda + j] = v;
            if (j == k + 1) {
              coln[i] = v;
              if (i > k && fabs(v) > nb) { nb = fabs(v); ni = i; }
            }
          }
        }
      }
      if (j == k + 1) {
        s.cand_v[r0] = nb;
        s.cand_i[r0] = ni;
      }
    }
    __syncthreads();
  }
  // undo the row interchanges as column interchanges, last first; one thread per row
  for (int i = tid; i < n; i += nt) {
    for (int k = n - 1; k >= 0; --k) {
      const int pr = s.piv[k];
      if (pr != k) {
        const double t = a[i * lda + k];
        a[i * lda + k] = a[i * lda + pr];
        a[i * lda + pr] = t;
      }
    }
  }
  __syncthreads();
  return 0;
}

// C := alpha * op(A) * op(B) + beta * C for small matrices (any memory space),
// all threads of the block cooperating; op(X) = X or X' (tA / tB).  C must not
// alias A or B.  Ends with a block barrier.
__device__ inline void cta_mm(int M, int N, int K, double alpha, const double* A, int lda, bool tA, const double* B,
                              int ldb, bool tB, double beta, double* C, int ldc) {
  for (int e = threadIdx.x; e < M * N; e += blockDim.x) {
    const int i = e / N, j = e % N;
    double s = 0.0;
    for (int k = 0; k < K; ++k) {
      const double x = tA ? A[k * lda + i] : A[i * lda + k];
      const double y = tB ? B[j * ldb + k] : B[k * ldb + j];
      s = fma(x, y, s);
    }
    C[i * ldc + j] = (beta == 0.0) ? alpha * s : alpha * s + beta * C[i * ldc + j];
  }
  __syncthreads();
}

// Block-wide sum of one value per thread; every thread gets the total.
__device__ inline double cta_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double tot = 0.0;
  const int nw = (blockDim.x + 31) >> 5;
  for (int w = 0; w < nw; ++w) tot += red[w];
  __syncthreads();
  return tot;
}

}  // namespace small
}  // namespace mb
