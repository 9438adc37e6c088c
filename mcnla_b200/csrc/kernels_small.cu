// Small and elementwise kernels of the iSVD stages (see kernels.cuh).
#include "kernels.cuh"
#include "small.cuh"
#include "philox.cuh"
#include <algorithm>
#include <mutex>
#include <map>
#include <utility>

namespace mb {
namespace {

constexpr int kSmallThreads = 512;
constexpr int kSyevThreads = 1024;   // the Jacobi rounds are latency-bound: more warps hide more of it
constexpr int kMaxSweeps = 40;
constexpr int kKnNsMaxDim = 80;   // the matrix-function KN step keeps four padded l x l matrices on chip
constexpr int kGjThreads = 1024;   // the Gauss-Jordan steps are latency-bound: fewer rows per thread per step
static_assert(2 * MCNLA_B200_MAX_DIM_SKETCH_WENYIN <= kGjThreads, "cta_gj_inverse needs n <= blockDim.x");

// Shared-memory carve-up shared by the one-CTA solvers.
struct SmemCarve {
  char* base;
  size_t off = 0;
  __device__ explicit SmemCarve(char* b) : base(b) {}
  template <class T>
  __device__ T* take(size_t n) {
    off = (off + 15) & ~size_t(15);
    T* p = reinterpret_cast<T*>(base + off);
    off += n * sizeof(T);
    return p;
  }
};

__host__ __device__ inline size_t jacobi_scratch_bytes(int n) {
  const int np = (n + 2) / 2;   // cs, pq, t, apq, app, aqq, count, red (16-byte aligned each)
  return (np * 16 + 16) + (np * 8 + 16) + 4 * (np * 8 + 16) + 16 + 32 * 8 + 16 + (n + 4) * 4 + 64;
}

__device__ small::JacobiScratch carve_jacobi(SmemCarve& sc, int n) {
  const int np = (n + 2) / 2;
  small::JacobiScratch js;
  js.cs = sc.take<double2>(np);
  js.pq = sc.take<int2>(np);
  js.t = sc.take<double>(np);
  js.apq = sc.take<double>(np);
  js.app = sc.take<double>(np);
  js.aqq = sc.take<double>(np);
  js.count = sc.take<int>(1);
  js.red = sc.take<double>(32);
  return js;
}

__host__ __device__ inline size_t gj_scratch_bytes(int n) {   // piv, col, prow, cand_v, cand_i
  return (size_t(n) * 4 + 16) + (size_t(n) * 16 + 16) + (size_t(n) * 8 + 16) + (small::kGjMaxGroups * 8 + 16) +
         (small::kGjMaxGroups * 4 + 16);
}

__device__ small::GjScratch carve_gj(SmemCarve& sc, int n) {
  small::GjScratch g;
  g.piv = sc.take<int>(n);
  g.col = sc.take<double>(2 * size_t(n));
  g.prow = sc.take<double>(n);
  g.cand_v = sc.take<double>(small::kGjMaxGroups);
  g.cand_i = sc.take<int>(small::kGjMaxGroups);
  return g;
}

// rank[j] = position of eigenvalue j in the requested order (ties by index).
__device__ void eig_ranks(const double* a, int lda, int n, int order, int* rank) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double dj = order ? fabs(a[j * lda + j]) : a[j * lda + j];
    int r = 0;
    for (int i = 0; i < n; ++i) {
      const double di = order ? fabs(a[i * lda + i]) : a[i * lda + i];
      const bool before = order ? (di > dj || (di == dj && i < j)) : (di < dj || (di == dj && i < j));
      r += before ? 1 : 0;
    }
    rank[j] = r;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// batched symmetric eigendecomposition
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kSyevThreads) k_syev(int n, const double* A, int64_t lda, int64_t a_bs,
                                                        double* W, double* V, int order, int v_smem,
                                                        double* vwork_all) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemCarve sc(smem_raw);
  const int ld = n + 1;
  double* a = sc.take<double>(size_t(n) * ld);
  double* v;
  int ldv;
  if (v_smem) { v = sc.take<double>(size_t(n) * ld); ldv = ld; }
  else { v = vwork_all + size_t(blockIdx.x) * n * n; ldv = n; }
  small::JacobiScratch js = carve_jacobi(sc, n);
  int* rank = sc.take<int>(n);
  const double* Ab = A + blockIdx.x * a_bs;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) a[(e / n) * ld + (e % n)] = Ab[(e / n) * lda + (e % n)];
  __syncthreads();
  small::cta_jacobi_eig(a, ld, v, ldv, n, true, js, kMaxSweeps);
  eig_ranks(a, ld, n, order, rank);
  double* Wb = W + size_t(blockIdx.x) * n;
  double* Vb = V + size_t(blockIdx.x) * n * n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double d = a[j * ld + j];
    Wb[rank[j]] = order ? fabs(d) : d;
  }
  if (v_smem) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      Vb[i * n + rank[j]] = v[j * ldv + i];
    }
  } else {
    __syncthreads();
    // eigenvectors (rows of the global work copy) to ranked columns
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      Vb[i * n + rank[j]] = v[j * ldv + i];
    }
  }
}

__global__ void k_scale_cols_rsqrt(int n, int batch, const double* V, const double* W, double* T) {
  const int64_t total = int64_t(batch) * n * n;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / (int64_t(n) * n);
    const int j = int(e % n);
    T[e] = V[e] / sqrt(W[b * n + j]);
  }
}

// ---------------------------------------------------------------------------
// Kolmogorov-Nagumo step
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kSyevThreads) k_kn_step(int l, const double* z_in, const double* dd,
                                                           double inv_n, double* out, double* outn,
                                                           const double* ff, double* ffn, double* vwork,
                                                           int v_smem, DevScalars* scal, double tol,
                                                           const int* guard_stop, int guard_it, const int* only_if) {
  extern __shared__ __align__(16) char smem_raw[];
  if (guard_stop && *guard_stop < guard_it) return;
  if (only_if && *only_if == 0) return;
  SmemCarve sc(smem_raw);
  const int ld = l + 1;
  double* a = sc.take<double>(size_t(l) * ld);
  double* v;
  int ldv;
  if (v_smem) { v = sc.take<double>(size_t(l) * ld); ldv = ld; }
  else { v = vwork; ldv = l; }
  small::JacobiScratch js = carve_jacobi(sc, l);
  double* sv = sc.take<double>(l);    // sqrt(s)
  const int tid = threadIdx.x, nt = blockDim.x;
  // Z
  if (dd == nullptr) {
    for (int e = tid; e < l * l; e += nt) a[(e / l) * ld + (e % l)] = z_in[e];
  } else {
    // Z := Dgc - Dc * Dc'   (Dc = dd(:, 0:l), Dgc = dd(:, l:2l), row stride 2l)
    // row_block_kolmogorov_nagumo_integrator.hpp:150-156
    const int ldd = 2 * l;
    for (int e = tid; e < l * l; e += nt) {
      const int i = e / l, j = e % l;
      double s = 0.0;
      for (int k = 0; k < l; ++k) s = fma(dd[i * ldd + k], dd[j * ldd + k], s);
      a[i * ld + j] = dd[i * ldd + l + j] - s;
    }
  }
  __syncthreads();
  const int sweeps = small::cta_jacobi_eig(a, ld, v, ldv, l, true, js, kMaxSweeps);
  // s := sqrt(1/2 + sqrt(1/4 - lambda)); ss := sqrt(s)
  double part = 0.0;
  for (int i = tid; i < l; i += nt) {
    const double s = sqrt(0.5 + sqrt(0.25 - a[i * ld + i]));
    sv[i] = sqrt(s);
    part += (s - 1.0) * (s - 1.0);
  }
  const double norm2 = small::cta_sum(part, js.red);
  // C = V diag(s) V', inv(C) = V diag(1/s) V'  -> out rows [0, l) hold C or Fc,
  // rows [l, 2l) hold inv(C).
  double* cmat = out;                 // l x l, row-major (ld l)
  double* cinv = out + size_t(l) * l;
  for (int e = tid; e < l * l; e += nt) {
    const int i = e / l, j = e % l;
    double c = 0.0, ci = 0.0;
    for (int k = 0; k < l; ++k) {
      const double x = v[k * ldv + i] * sv[k], y = v[k * ldv + j] * sv[k];
      const double xi = v[k * ldv + i] / sv[k], yi = v[k * ldv + j] / sv[k];
      c = fma(x, y, c);
      ci = fma(xi, yi, ci);
    }
    cmat[i * l + j] = c;
    cinv[i * l + j] = ci;
  }
  __syncthreads();
  if (dd != nullptr) {
    // Fc := C - Dc * inv(C)   (row_block_kolmogorov_nagumo_integrator.hpp:186)
    // computed into the Jacobi matrix space, then written over C
    const int ldd = 2 * l;
    for (int e = tid; e < l * l; e += nt) {
      const int i = e / l, j = e % l;
      double s = 0.0;
      for (int k = 0; k < l; ++k) s = fma(dd[i * ldd + k], cinv[k * l + j], s);
      a[i * ld + j] = cmat[i * l + j] - s;
    }
    __syncthreads();
    for (int e = tid; e < l * l; e += nt) cmat[e] = a[(e / l) * ld + (e % l)];
    __syncthreads();
    if (outn) {
      for (int e = tid; e < l * l; e += nt) {
        outn[e] = cmat[e];
        outn[size_t(l) * l + e] = cinv[e] * inv_n;
      }
    }
    if (ff && ffn) {
      // F~+ := F~c * Fc  (row_block_gramian_kolmogorov_nagumo_integrator.hpp:197)
      for (int e = tid; e < l * l; e += nt) {
        const int i = e / l, j = e % l;
        double s = 0.0;
        for (int k = 0; k < l; ++k) s = fma(ff[i * l + k], a[k * ld + j], s);
        ffn[i * l + j] = s;
      }
    }
  }
  if (tid == 0) {
    const double norm = sqrt(norm2);
    scal->norm = norm;
    scal->sweeps = sweeps;
    if (guard_stop && !(norm >= tol)) scal->stop_it = guard_it;
  }
}

// ---------------------------------------------------------------------------
// Kolmogorov-Nagumo step by matrix functions
//
// The step needs C = f(Z) and inv(C) for f(x) = sqrt(1/2 + sqrt(1/4 - x)),
// which the reference forms from an eigendecomposition of Z
// (row_block_kolmogorov_nagumo_integrator.hpp:159-180).  Here they come from
// two coupled Newton-Schulz iterations (Higham, Functions of Matrices, 2008,
// eq. 6.35; inversion-free, built from matrix products only):
//   S = (I - 4Z)^(1/2)            -> sqrt(1/4 - Z) = S/2
//   C = ((I + S)/2)^(1/2), inv(C) = ((I + S)/2)^(-1/2)
// The products run on the FP64 MMA inside one CTA, on matrices in shared
// memory (l <= 80) or in global memory (L2-resident, l <= 160).  Jacobi on the
// clustered spectrum Z has near convergence (dozens of near-zero
// eigenvalues) needs 15-20 sweeps; the iteration above needs a handful of
// products.  When an iteration fails (non-finite values or no convergence,
// e.g. an eigenvalue of Z above 1/4 where the reference produces NaN), the
// kernel falls back to the eigendecomposition path of k_kn_step.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void small_dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// C := A * op(B) for lp x lp matrices in shared memory (lp a multiple of 16,
// row stride ld, zero padding outside the active block).  Each warp owns
// 16 x 16 output blocks (four independent 8 x 8 MMA accumulators).  C must not
// alias A or B.  Ends with a block barrier.
template <bool TB>
__device__ void cta_mm16(double* C, const double* A, const double* B, int lp, int ld) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int nb = lp >> 4;
  for (int blk = warp; blk < nb * nb; blk += nw) {
    const int bi = (blk / nb) * 16, bj = (blk % nb) * 16;
    double c[2][2][2] = {{{0.0, 0.0}, {0.0, 0.0}}, {{0.0, 0.0}, {0.0, 0.0}}};
    for (int k = 0; k < lp; k += 4) {
      const double a0 = A[(bi + g) * ld + k + t4];
      const double a1 = A[(bi + 8 + g) * ld + k + t4];
      const double b0 = TB ? B[(bj + g) * ld + k + t4] : B[(k + t4) * ld + bj + g];
      const double b1 = TB ? B[(bj + 8 + g) * ld + k + t4] : B[(k + t4) * ld + bj + 8 + g];
      small_dmma(c[0][0][0], c[0][0][1], a0, b0);
      small_dmma(c[0][1][0], c[0][1][1], a0, b1);
      small_dmma(c[1][0][0], c[1][0][1], a1, b0);
      small_dmma(c[1][1][0], c[1][1][1], a1, b1);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        double* cp = C + (bi + i * 8 + g) * ld + bj + j * 8 + 2 * t4;
        cp[0] = c[i][j][0];
        cp[1] = c[i][j][1];
      }
  }
  __syncthreads();
}

// Coupled Newton-Schulz for M^(1/2) and M^(-1/2): on entry *Y holds M; on
// success *Y = M^(1/2), *Zm = M^(-1/2).  Buffers are rotated through the four
// pointers.  Returns the iterations used, or -1 (non-finite or no convergence).
__device__ int cta_ns_sqrt(double*& Y, double*& Zm, double*& T, double*& W, int l, int lp, int ld, double* red,
                           int maxit) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < lp * lp; e += nt) {
    const int i = e / lp, j = e % lp;
    Zm[i * ld + j] = (i == j && i < l) ? 1.0 : 0.0;
  }
  __syncthreads();
  bool polish = false;
  for (int it = 0; it < maxit; ++it) {
    cta_mm16<false>(W, Zm, Y, lp, ld);                      // P = Zm Y
    double part = 0.0;
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      const double pij = W[i * ld + j];
      const double d = ((i == j && i < l) ? 1.0 : 0.0) - pij;
      part += d * d;
      T[i * ld + j] = (i < l && j < l) ? 0.5 * (((i == j) ? 3.0 : 0.0) - pij) : 0.0;   // T = (3I - P)/2
    }
    const double r2 = small::cta_sum(part, red);
    if (!(r2 < 1e300)) return -1;                           // non-finite
    if (polish) return it;
    if (r2 < 1e-18) polish = true;                          // one more step reaches rounding level
    cta_mm16<false>(W, Y, T, lp, ld);                       // Y+ = Y T
    double* oldY = Y;
    Y = W;
    cta_mm16<false>(oldY, T, Zm, lp, ld);                   // Z+ = T Zm
    W = Zm;
    Zm = oldY;
  }
  return -1;
}

// GMEM: the four matrices live in vwork (global memory, L2-resident) instead of
// shared memory (80 < l <= 160); a failed iteration then sets
// scal->kn_ns_failed, and the launcher's eigendecomposition kernel after it
// takes the step (it returns at once otherwise).
template <bool GMEM>
__global__ void __launch_bounds__(GMEM ? kSyevThreads : kSmallThreads)
    k_kn_step_ns(int l, const double* z_in, const double* dd, double inv_n, double* out, double* outn,
                 const double* ff, double* ffn, double* vwork, DevScalars* scal, double tol, const int* guard_stop,
                 int guard_it, const int* only_if) {
  extern __shared__ __align__(16) char smem_raw[];
  if (GMEM && threadIdx.x == 0) scal->kn_ns_failed = 0;
  if (guard_stop && *guard_stop < guard_it) return;
  if (only_if && *only_if == 0) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lp = (l + 15) & ~15, ld = lp + 4;
  const size_t mat = size_t(lp) * ld;
  double* buf = GMEM ? vwork : reinterpret_cast<double*>(smem_raw);
  double* B0 = buf;
  double* B1 = buf + mat;
  double* B2 = buf + 2 * mat;
  double* B3 = buf + 3 * mat;
  double* red = GMEM ? reinterpret_cast<double*>(smem_raw) : buf + 4 * mat;   // 64 doubles
  double* sv = red + 64;                // 96 doubles (eigen fallback)
  const int ldd = 2 * l;
  // ---- Z (upper triangle mirrored, as a symmetric eigensolver reads it) into B0
  if (dd == nullptr) {
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      B0[i * ld + j] = (i < l && j < l) ? z_in[min(i, j) * l + max(i, j)] : 0.0;
    }
    __syncthreads();
  } else {
    // Z := Dgc - Dc Dc'   (row_block_kolmogorov_nagumo_integrator.hpp:150-156)
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      B1[i * ld + j] = (i < l && j < l) ? dd[i * ldd + j] : 0.0;
    }
    __syncthreads();
    cta_mm16<true>(B2, B1, B1, lp, ld);
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      const int a = min(i, j), b = max(i, j);
      B0[i * ld + j] = (i < l && j < l) ? dd[a * ldd + l + b] - B2[a * ld + b] : 0.0;
    }
    __syncthreads();
  }
  // ---- M1 = I - 4Z; S = M1^(1/2)
  for (int e = tid; e < lp * lp; e += nt) {
    const int i = e / lp, j = e % lp;
    const double z = B0[i * ld + j];
    B0[i * ld + j] = (i < l && j < l) ? ((i == j) ? 1.0 : 0.0) - 4.0 * z : 0.0;
  }
  __syncthreads();
  double *Y = B0, *Zm = B1, *T = B2, *W = B3;
  int it1 = cta_ns_sqrt(Y, Zm, T, W, l, lp, ld, red, 60);
  int it2 = -1;
  if (it1 >= 0) {
    // M2 = (I + S)/2 into Zm's buffer, then C = M2^(1/2), inv(C) = M2^(-1/2)
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      Zm[i * ld + j] = (i < l && j < l) ? 0.5 * (((i == j) ? 1.0 : 0.0) + Y[i * ld + j]) : 0.0;
    }
    __syncthreads();
    double* tmp = Y;
    Y = Zm;
    Zm = tmp;
    it2 = cta_ns_sqrt(Y, Zm, T, W, l, lp, ld, red, 60);
  }
  if ((it1 < 0 || it2 < 0) && GMEM) {
    // the eigendecomposition kernel launched after this one takes the step
    if (tid == 0) {
      scal->sweeps = -1;
      scal->kn_ns_failed = 1;
    }
    return;
  }
  if (it1 < 0 || it2 < 0) {
    // eigendecomposition fallback (the reference's path, NaN semantics included)
    if (tid == 0) scal->sweeps = -1;
    // recompute Z into B0 (as above) and run the Jacobi step on it
    if (dd == nullptr) {
      for (int e = tid; e < l * l; e += nt) B0[(e / l) * (l + 1) + (e % l)] = z_in[e];
    } else {
      for (int e = tid; e < l * l; e += nt) {
        const int i = e / l, j = e % l;
        double s = 0.0;
        for (int k = 0; k < l; ++k) s = fma(dd[i * ldd + k], dd[j * ldd + k], s);
        B0[i * (l + 1) + j] = dd[i * ldd + l + j] - s;
      }
    }
    __syncthreads();
    // the Jacobi matrices sit in B0 | B1 (l (l+1) <= lp (lp+4)), its scratch after sv
    SmemCarve sc(reinterpret_cast<char*>(sv + 96));
    small::JacobiScratch js = carve_jacobi(sc, l);
    double* v = B1;
    small::cta_jacobi_eig(B0, l + 1, v, l + 1, l, true, js, kMaxSweeps);
    for (int i = tid; i < l; i += nt) sv[i] = sqrt(sqrt(0.5 + sqrt(0.25 - B0[i * (l + 1) + i])));
    __syncthreads();
    // C and inv(C) into B2 / B3 in the padded layout
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      double cc = 0.0, ci = 0.0;
      if (i < l && j < l) {
        for (int k = 0; k < l; ++k) {
          const double x = v[k * (l + 1) + i], y = v[k * (l + 1) + j];
          cc = fma(x * sv[k], y * sv[k], cc);
          ci = fma(x / sv[k], y / sv[k], ci);
        }
      }
      B2[i * ld + j] = cc;
      B3[i * ld + j] = ci;
    }
    __syncthreads();
    Y = B2;
    Zm = B3;
    T = B0;
    W = B1;
  }
  // ---- C in *Y, inv(C) in *Zm;  ||e - 1||_2 = ||C - I||_F
  double part = 0.0;
  for (int e = tid; e < l * l; e += nt) {
    const int i = e / l, j = e % l;
    const double d = Y[i * ld + j] - ((i == j) ? 1.0 : 0.0);
    part += d * d;
    out[size_t(l) * l + e] = Zm[i * ld + j];                  // rows [l, 2l): inv(C)
  }
  const double norm2 = small::cta_sum(part, red);
  if (dd == nullptr) {
    for (int e = tid; e < l * l; e += nt) out[e] = Y[(e / l) * ld + (e % l)];   // rows [0, l): C
  } else {
    // Fc := C - Dc inv(C)   (row_block_kolmogorov_nagumo_integrator.hpp:186)
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      T[i * ld + j] = (i < l && j < l) ? dd[i * ldd + j] : 0.0;
    }
    __syncthreads();
    cta_mm16<false>(W, T, Zm, lp, ld);
    for (int e = tid; e < lp * lp; e += nt) {
      const int i = e / lp, j = e % lp;
      const double fc = (i < l && j < l) ? Y[i * ld + j] - W[i * ld + j] : 0.0;
      W[i * ld + j] = fc;
      if (i < l && j < l) {
        out[i * l + j] = fc;
        if (outn) {
          outn[i * l + j] = fc;
          outn[size_t(l) * l + i * l + j] = Zm[i * ld + j] * inv_n;
        }
      }
    }
    __syncthreads();
    if (ff && ffn) {
      // F~+ := F~c Fc  (row_block_gramian_kolmogorov_nagumo_integrator.hpp:197)
      for (int e = tid; e < lp * lp; e += nt) {
        const int i = e / lp, j = e % lp;
        T[i * ld + j] = (i < l && j < l) ? ff[i * l + j] : 0.0;
      }
      __syncthreads();
      cta_mm16<false>(Y, T, W, lp, ld);
      for (int e = tid; e < l * l; e += nt) ffn[e] = Y[(e / l) * ld + (e % l)];
    }
  }
  if (tid == 0) {
    const double norm = sqrt(norm2);
    scal->norm = norm;
    if (it1 >= 0 && it2 >= 0) scal->sweeps = it1 * 100 + it2;
    if (guard_stop && !(norm >= tol)) scal->stop_it = guard_it;
  }
}

// ---------------------------------------------------------------------------
// Wen-Yin trial
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kGjThreads) k_wy_trial(int l, const double* dd, double tau, double inv_n,
                                                            double* F, double* FN, DevScalars* scal) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemCarve sc(smem_raw);
  const int n = 2 * l, ld = n + 1, ldd = 2 * l;
  double* cm = sc.take<double>(size_t(n) * ld);
  const small::GjScratch gs = carve_gj(sc, n);
  const int tid = threadIdx.x, nt = blockDim.x;
  const double it = 1.0 / tau;
  // C := [ Dc/2 - I/tau , I/2 ; -Dgc/2 , -Dc/2 - I/tau ]
  // (row_block_wen_yin_integrator.hpp:176-183)
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e % n;
    const int bi = i / l, bj = j / l, ii = i % l, jj = j % l;
    double x;
    if (bi == 0 && bj == 0) x = 0.5 * dd[ii * ldd + jj] - (ii == jj ? it : 0.0);
    else if (bi == 0) x = (ii == jj) ? 0.5 : 0.0;
    else if (bj == 0) x = -0.5 * dd[ii * ldd + l + jj];
    else x = -0.5 * dd[ii * ldd + jj] - (ii == jj ? it : 0.0);
    cm[i * ld + j] = x;
  }
  __syncthreads();
  const int sing = small::cta_gj_inverse(cm, ld, n, gs);
  if (sing) {
    if (tid == 0) scal->status = MCNLA_B200_ERR_SINGULAR;
    return;
  }
  // T := inv(C)(:, l:2l) * Dc - inv(C)(:, 0:l); Fgc = T(0:l, :), Fc = T(l:2l, :) + I
  // F = [Fc; Fgc]   (row_block_wen_yin_integrator.hpp:189-193)
  for (int e = tid; e < n * l; e += nt) {
    const int i = e / l, j = e % l;
    double s = 0.0;
    for (int k = 0; k < l; ++k) s = fma(cm[i * ld + l + k], dd[k * ldd + j], s);
    s -= cm[i * ld + j];
    if (i >= l) {   // Fc row
      const int r = i - l;
      const double fc = s + (r == j ? 1.0 : 0.0);
      F[r * l + j] = fc;
      if (FN) FN[r * l + j] = fc;
    } else {        // Fgc row
      F[size_t(l) * l + i * l + j] = s;
      if (FN) FN[size_t(l) * l + i * l + j] = s * inv_n;
    }
  }
}

// ---------------------------------------------------------------------------
// one-sided Jacobi SVD of a small square matrix
// ---------------------------------------------------------------------------
// One-sided (Hestenes) Jacobi SVD of one n x n matrix: columns p, q of a are
// rotated until all pairs are orthogonal; a = W diag(sig), and the rotations
// accumulated in z give M = W diag(sig) Z'.  Per round: the angles of the
// n/2 disjoint pairs (a warp per pair: column dot products by shuffles), then
// the rotations of a's columns and of z spread over the CTA as (pair, row)
// items.  z is kept transposed (z[k * ldz + i] = Z(i, k)) so that a rotation
// touches two contiguous rows when it lives in global memory.
__global__ void __launch_bounds__(kSmallThreads) k_svd_small(int n, const double* M, double* W, double* sig,
                                                             double* Z, double* zwork, int z_smem) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemCarve sc(smem_raw);
  const int ld = n + 1;
  double* a = sc.take<double>(size_t(n) * ld);
  double* z;
  int ldz;
  if (z_smem) { z = sc.take<double>(size_t(n) * ld); ldz = ld; }
  else { z = zwork; ldz = n; }
  int* count = sc.take<int>(4);
  int* rank = sc.take<int>(n);
  double* nrm = sc.take<double>(n);
  const int P = (n + 1) & ~1, npairs = P / 2;
  double* rc = sc.take<double>(npairs);
  double* rs = sc.take<double>(npairs);
  int* rp = sc.take<int>(npairs);
  int* rq = sc.take<int>(npairs);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e % n;
    a[i * ld + j] = M[e];
    z[i * ldz + j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int items = npairs * n;
  for (int sweep = 0; sweep < 40 && n > 1; ++sweep) {
    int rotated = 0;
    for (int r = 0; r < P - 1; ++r) {
      // angles: a warp per pair
      int mine = 0;
      for (int k = warp; k < npairs; k += nwarps) {
        int p, q;
        small::rr_pair(P, r, k, p, q);
        double c = 1.0, sn = 0.0;
        if (q < n) {
          double al = 0.0, be = 0.0, ga = 0.0;
          for (int i = lane; i < n; i += 32) {
            const double x = a[i * ld + p], y = a[i * ld + q];
            al = fma(x, x, al);
            be = fma(y, y, be);
            ga = fma(x, y, ga);
          }
          for (int o = 16; o > 0; o >>= 1) {
            al += __shfl_xor_sync(0xffffffffu, al, o);
            be += __shfl_xor_sync(0xffffffffu, be, o);
            ga += __shfl_xor_sync(0xffffffffu, ga, o);
          }
          if (fabs(ga) > 1e-15 * sqrt(al * be) && ga * ga > 1e-300) {
            const double zeta = (be - al) / (2.0 * ga);
            const double az = fabs(zeta);
            const double t = (az > 1e150) ? 0.5 / zeta : ((zeta >= 0.0 ? 1.0 : -1.0) / (az + sqrt(1.0 + zeta * zeta)));
            c = 1.0 / sqrt(1.0 + t * t);
            sn = c * t;
            if (lane == 0) ++mine;
          }
        }
        if (lane == 0) { rc[k] = c; rs[k] = sn; rp[k] = p; rq[k] = q; }
      }
      // the barrier also counts the rotations set up this round
      const int cnt = __syncthreads_count(mine);
      if (cnt == 0) continue;
      rotated += cnt;
      // rotations: (pair, row) items over the CTA
      for (int e = tid; e < items; e += nt) {
        const int k = e / n, i = e - k * n;
        const double sn = rs[k];
        if (sn == 0.0) continue;
        const double c = rc[k];
        const int p = rp[k], q = rq[k];
        const double x = a[i * ld + p], y = a[i * ld + q];
        a[i * ld + p] = c * x - sn * y;
        a[i * ld + q] = sn * x + c * y;
        const double zx = z[p * ldz + i], zy = z[q * ldz + i];
        z[p * ldz + i] = c * zx - sn * zy;
        z[q * ldz + i] = sn * zx + c * zy;
      }
      __syncthreads();
    }
    if (rotated == 0) break;
  }
  for (int j = warp; j < n; j += nwarps) {
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s = fma(a[i * ld + j], a[i * ld + j], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) nrm[j] = sqrt(s);
  }
  __syncthreads();
  for (int j = tid; j < n; j += nt) {
    int r = 0;
    for (int i = 0; i < n; ++i) r += (nrm[i] > nrm[j] || (nrm[i] == nrm[j] && i < j)) ? 1 : 0;
    rank[j] = r;
    sig[r] = nrm[j];
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e % n;
    const double sj = nrm[j];
    W[i * n + rank[j]] = sj > 0.0 ? a[i * ld + j] / sj : 0.0;
    Z[i * n + rank[j]] = z[j * ldz + i];
  }
}

__global__ void k_rsqrt_rows_t(int n, const double* Ue, const double* w, double* P) {
  const double floor = (n * 2.220446049250313e-16) * (n * 2.220446049250313e-16) * fabs(w[0]);
  for (int e = threadIdx.x + blockIdx.x * blockDim.x; e < n * n; e += blockDim.x * gridDim.x) {
    const int i = e / n, j = e % n;
    const double wi = w[i];
    P[e] = (wi > floor && wi > 0.0) ? Ue[j * n + i] / sqrt(wi) : 0.0;
  }
}

__global__ void k_scale_cols(int64_t rows, int64_t cols, const double* X, int64_t ldx, const double* s, int mode,
                             double* Y, int64_t ldy) {
  const int64_t total = rows * cols;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols, c = e % cols;
    const double f = mode == 0 ? 1.0 / s[c] : (mode == 1 ? s[c] : 1.0 / sqrt(s[c]));
    Y[r * ldy + c] = X[r * ldx + c] * f;
  }
}

__global__ void k_sqrt_vec(int n, const double* w, double* out) {
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < n; i += blockDim.x * gridDim.x) out[i] = sqrt(w[i]);
}

__global__ void __launch_bounds__(kGjThreads) k_inverse(int n, double* A, DevScalars* scal) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemCarve sc(smem_raw);
  const int ld = n + 1;
  double* a = sc.take<double>(size_t(n) * ld);
  const small::GjScratch gs = carve_gj(sc, n);
  double* Ab = A + size_t(blockIdx.x) * n * n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) a[(e / n) * ld + (e % n)] = Ab[e];
  __syncthreads();
  const int sing = small::cta_gj_inverse(a, ld, n, gs);
  if (sing) {
    if (threadIdx.x == 0) scal->status = MCNLA_B200_ERR_SINGULAR;
    return;
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) Ab[e] = a[(e / n) * ld + (e % n)];
}

// ---------------------------------------------------------------------------
// deterministic reductions
// ---------------------------------------------------------------------------
constexpr int kRedThreads = 256;

__device__ inline double block_sum(double v) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  }
  __syncthreads();
  return t;
}

__global__ void k_dot_partial(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t rows,
                              int64_t cols, double* partials) {
  const int64_t total = rows * cols;
  double s = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols, c = e % cols;
    s = fma(X[r * ldx + c], Y[r * ldy + c], s);
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void k_wy_delta_partial(const double* qc, const double* qp, int64_t ldq, const double* xc,
                                   const double* xp, int64_t ldx, int64_t rows, int64_t cols, double* partials) {
  const int64_t total = rows * cols;
  double s11 = 0.0, s12 = 0.0, s22 = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols, c = e % cols;
    const double d1 = qc[r * ldq + c] - qp[r * ldq + c];
    const double d2 = xc[r * ldx + c] - xp[r * ldx + c];
    s11 = fma(d1, d1, s11);
    s12 = fma(d1, d2, s12);
    s22 = fma(d2, d2, s22);
  }
  s11 = block_sum(s11);
  s12 = block_sum(s12);
  s22 = block_sum(s22);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x + 0] = s11;
    partials[3 * blockIdx.x + 1] = s12;
    partials[3 * blockIdx.x + 2] = s22;
  }
}

// Sums `count` groups of `width` partials in a fixed order: out[w] = scale * sum_b p[b*width + w].
__global__ void k_final_sum(const double* partials, int count, int width, double scale, double* out) {
  for (int w = 0; w < width; ++w) {
    double s = 0.0;
    for (int b = threadIdx.x; b < count; b += blockDim.x) s += partials[b * width + w];
    s = block_sum(s);
    if (threadIdx.x == 0) out[w] = scale * s;
  }
}

__global__ void k_gwy_small_dots(int l, const double* p1, const double* p2, const double* bcu, double* out) {
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  const int ldb = 2 * l;
  for (int e = threadIdx.x; e < l * l; e += blockDim.x) {
    const int i = e / l, j = e % l;
    const double a = p1[e], b = p2[e], u1 = bcu[i * ldb + j], u2 = bcu[i * ldb + l + j];
    s[0] = fma(a, a, s[0]);
    s[1] = fma(a, b, s[1]);
    s[2] = fma(b, b, s[2]);
    s[3] = fma(a, u1, s[3]);
    s[4] = fma(a, u2, s[4]);
    s[5] = fma(b, u1, s[5]);
    s[6] = fma(b, u2, s[6]);
  }
  for (int k = 0; k < 7; ++k) {
    const double t = block_sum(s[k]);
    if (threadIdx.x == 0) out[k] = t;
  }
}

__global__ void k_wy_mu(int l, const double* dd, double* out) {
  // mu := asum(diag(Dgc)) - ||Dc||_F^2   (row_block_wen_yin_integrator.hpp:143)
  const int ldd = 2 * l;
  double s = 0.0;
  for (int e = threadIdx.x; e < l * l; e += blockDim.x) {
    const int i = e / l, j = e % l;
    const double d = dd[i * ldd + j];
    s -= d * d;
    if (i == j) s += fabs(dd[i * ldd + l + j]);
  }
  s = block_sum(s);
  if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// elementwise
// ---------------------------------------------------------------------------
__global__ void k_axpby(int64_t rows, int64_t cols, double alpha, const double* X, int64_t ldx, double beta,
                        double* Y, int64_t ldy) {
  const int64_t total = rows * cols;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols, c = e % cols;
    const double x = alpha * X[r * ldx + c];
    Y[r * ldy + c] = (beta == 0.0) ? x : x + beta * Y[r * ldy + c];
  }
}

__global__ void k_fill(int64_t rows, int64_t cols, double v, double* X, int64_t ld, int identity) {
  const int64_t total = rows * cols;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols, c = e % cols;
    X[r * ld + c] = identity ? (r == c ? 1.0 : 0.0) : v;
  }
}

__global__ void k_gramian_prepare(int64_t L, int l, double* bs, double* bc, int64_t ldbc) {
  // Bs(i, j) := Bs(j, i) for i < j (keep the lower triangle, as the reference's
  // syrk into Bs.syml() does); Bc := Bs(:, 0:l) with the strict upper triangle
  // of its top l x l block zero (row_block_gramian_kolmogorov_nagumo_integrator.hpp:112-125).
  const int64_t total = L * L;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / L, j = e % L;
    if (i < j) bs[i * L + j] = bs[j * L + i];
    if (j < l) bc[i * ldbc + j] = (i < j) ? 0.0 : bs[(i >= j ? i * L + j : j * L + i)];
  }
}

__global__ void k_wy_gramian_phis(int l, const double* F, const double* dc, int64_t lddc, const double* dp,
                                  int64_t lddp, double* phi1, double* phi2) {
  // Phi1 := Fc - I; Phi2 := Dc - Fc * D+  (row_block_gramian_wen_yin_integrator.hpp:261-266)
  for (int e = threadIdx.x + blockIdx.x * blockDim.x; e < l * l; e += blockDim.x * gridDim.x) {
    const int i = e / l, j = e % l;
    const double* fc = F;  // rows [0, l) of F
    double s = 0.0;
    for (int k = 0; k < l; ++k) s = fma(fc[i * l + k], dp[k * lddp + j], s);
    phi2[e] = dc[i * lddc + j] - s;
    phi1[e] = fc[e] - (i == j ? 1.0 : 0.0);
  }
}

__global__ void k_gaussian(uint64_t seed, int64_t count, double* out) {
  const int64_t pairs = (count + 1) / 2;
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < pairs; j += int64_t(gridDim.x) * blockDim.x) {
    double z0, z1;
    gaussian_pair(seed, uint64_t(j), z0, z1);
    out[2 * j] = z0;
    if (2 * j + 1 < count) out[2 * j + 1] = z1;
  }
}

int grid_for(const Context* c, int64_t total, int threads) {
  return int(std::max<int64_t>(1, std::min<int64_t>(cdiv(total, threads), int64_t(c->num_sms) * 16)));
}

size_t small_smem_syev(int n, bool v_smem) {
  const size_t mat = size_t(n) * (n + 1) * sizeof(double) + 16;
  return mat * (v_smem ? 2 : 1) + jacobi_scratch_bytes(n) + (n + 4) * sizeof(int) + 64;
}



}  // namespace

// Opts a kernel in to all the dynamic shared memory the device allows it (the
// per-block opt-in limit less its static shared memory), once per (device,
// kernel).  The limit is a property of the function shared by every host
// thread, so it is never lowered to one launch's size (a concurrent launch of
// the same kernel with a larger size on another thread would then fail).
int set_smem(const Context* c, const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limits;
  std::lock_guard<std::mutex> lock(mu);
  auto it = limits.find({c->device, fn});
  if (it == limits.end()) {
    // static shared memory of the kernel counts against the same per-block limit
    cudaFuncAttributes fa;
    MB_CHECK_CUDA(cudaFuncGetAttributes(&fa, fn));
    const size_t limit = c->smem_optin > fa.sharedSizeBytes ? c->smem_optin - fa.sharedSizeBytes : 0;
    MB_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(limit)));
    it = limits.emplace(std::make_pair(c->device, fn), limit).first;
  }
  return bytes <= it->second ? MCNLA_B200_OK : MCNLA_B200_ERR_UNSUPPORTED;
}

int reduce_partials(const Context* c) { return c->num_sms * 2; }

int launch_syev(Context* c, int n, int batch, const double* A, int64_t lda, int64_t a_bs, double* W, double* V,
                int order) {
  if (n < 1 || n > MCNLA_B200_MAX_DIM_SKETCH || batch < 1) return MCNLA_B200_ERR_UNSUPPORTED;
  bool v_smem = small_smem_syev(n, true) <= c->smem_optin;
  double* vwork = nullptr;
  if (!v_smem) {
    // global eigenvector work copies (one n x n per matrix); from the arena
    vwork = ctx_take<double>(c, size_t(batch) * n * n);
    if (!vwork) return MCNLA_B200_ERR_WORKSPACE;
  }
  const size_t smem = small_smem_syev(n, v_smem);
  if (smem > c->smem_optin) return MCNLA_B200_ERR_UNSUPPORTED;
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_syev), smem));
  k_syev<<<batch, kSyevThreads, smem, c->stream>>>(n, A, lda, a_bs, W, V, order, v_smem ? 1 : 0, vwork);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_scale_cols_rsqrt(Context* c, int n, int batch, const double* V, const double* W, double* T) {
  const int64_t total = int64_t(batch) * n * n;
  k_scale_cols_rsqrt<<<grid_for(c, total, 256), 256, 0, c->stream>>>(n, batch, V, W, T);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_kn_step(Context* c, int l, const double* z, const double* dd, double inv_n, double* out, double* outn,
                   const double* ff, double* ffn, double* vwork, double tol, bool allow_series) {
  if (l < 1 || l > MCNLA_B200_MAX_DIM_SKETCH) return MCNLA_B200_ERR_UNSUPPORTED;
  // the series kernel first; the kernels below then run only when it declined
  const int* only_if = nullptr;
  if (c->kn_mode == MCNLA_B200_KN_AUTO && allow_series) {
    MB_CHECK(launch_kn_series(c, l, z, dd, inv_n, out, outn, ff, ffn, vwork, tol));
    only_if = &c->scal->kn_fallback;
  }
  if (l <= kKnNsMaxDim && c->kn_mode != MCNLA_B200_KN_EIGEN) {
    const int lp = (l + 15) & ~15;
    const size_t smem = 4 * size_t(lp) * (lp + 4) * sizeof(double) + (64 + 96) * sizeof(double) +
                        jacobi_scratch_bytes(l) + 64;
    if (smem <= c->smem_optin) {
      MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_kn_step_ns<false>), smem));
      k_kn_step_ns<false><<<1, kSmallThreads, smem, c->stream>>>(l, z, dd, inv_n, out, outn, ff, ffn, vwork, c->scal,
                                                                 tol, c->guard_stop, c->guard_it, only_if);
      c->kernels_launched++;
      MB_CHECK_CUDA(cudaGetLastError());
      return MCNLA_B200_OK;
    }
  }
  if (l > kKnNsMaxDim && c->kn_mode != MCNLA_B200_KN_EIGEN) {
    // Newton-Schulz with its matrices in vwork (kn_series_work_doubles(l) covers them); the
    // eigendecomposition kernel below runs only if it fails
    const size_t smem = (64 + 96) * sizeof(double) + 64;
    k_kn_step_ns<true><<<1, kSyevThreads, smem, c->stream>>>(l, z, dd, inv_n, out, outn, ff, ffn, vwork, c->scal, tol,
                                                             c->guard_stop, c->guard_it, only_if);
    c->kernels_launched++;
    MB_CHECK_CUDA(cudaGetLastError());
    only_if = &c->scal->kn_ns_failed;
  }
  const bool v_smem = small_smem_syev(l, true) + l * 8 + 64 <= c->smem_optin;
  const size_t smem = small_smem_syev(l, v_smem) + l * 8 + 64;
  if (smem > c->smem_optin) return MCNLA_B200_ERR_UNSUPPORTED;
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_kn_step), smem));
  k_kn_step<<<1, kSyevThreads, smem, c->stream>>>(l, z, dd, inv_n, out, outn, ff, ffn, vwork, v_smem ? 1 : 0,
                                                    c->scal, tol, c->guard_stop, c->guard_it, only_if);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_wy_trial(Context* c, int l, const double* dd, double tau, double inv_n, double* F, double* FN) {
  if (l < 1 || l > MCNLA_B200_MAX_DIM_SKETCH_WENYIN) return MCNLA_B200_ERR_UNSUPPORTED;
  const int n = 2 * l;
  const size_t smem = size_t(n) * (n + 1) * 8 + 16 + gj_scratch_bytes(n) + 64;
  if (smem > c->smem_optin) return MCNLA_B200_ERR_UNSUPPORTED;
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_wy_trial), smem));
  k_wy_trial<<<1, kGjThreads, smem, c->stream>>>(l, dd, tau, inv_n, F, FN, c->scal);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_sumsq(Context* c, const double* X, int64_t rows, int64_t cols, int64_t ld, double scale, double* partials,
                 double* out) {
  const int nb = reduce_partials(c);
  k_dot_partial<<<nb, kRedThreads, 0, c->stream>>>(X, ld, X, ld, rows, cols, partials);
  k_final_sum<<<1, kRedThreads, 0, c->stream>>>(partials, nb, 1, scale, out);
  c->kernels_launched += 2;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_dot(Context* c, const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t rows, int64_t cols,
               double* partials, double* out) {
  const int nb = reduce_partials(c);
  k_dot_partial<<<nb, kRedThreads, 0, c->stream>>>(X, ldx, Y, ldy, rows, cols, partials);
  k_final_sum<<<1, kRedThreads, 0, c->stream>>>(partials, nb, 1, 1.0, out);
  c->kernels_launched += 2;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_wy_delta_dots(Context* c, const double* qc, const double* qp, int64_t ldq, const double* xc,
                         const double* xp, int64_t ldx, int64_t rows, int64_t cols, double* partials, double* out) {
  const int nb = reduce_partials(c);
  k_wy_delta_partial<<<nb, kRedThreads, 0, c->stream>>>(qc, qp, ldq, xc, xp, ldx, rows, cols, partials);
  k_final_sum<<<1, kRedThreads, 0, c->stream>>>(partials, nb, 3, 1.0, out);
  c->kernels_launched += 2;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_wy_mu(Context* c, int l, const double* dd, double* out) {
  k_wy_mu<<<1, kRedThreads, 0, c->stream>>>(l, dd, out);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_axpby(Context* c, int64_t rows, int64_t cols, double alpha, const double* X, int64_t ldx, double beta,
                 double* Y, int64_t ldy) {
  if (rows <= 0 || cols <= 0) return MCNLA_B200_OK;
  k_axpby<<<grid_for(c, rows * cols, 256), 256, 0, c->stream>>>(rows, cols, alpha, X, ldx, beta, Y, ldy);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_set_identity(Context* c, int64_t n, double* X, int64_t ld) {
  k_fill<<<grid_for(c, n * n, 256), 256, 0, c->stream>>>(n, n, 0.0, X, ld, 1);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_fill(Context* c, int64_t rows, int64_t cols, double v, double* X, int64_t ld) {
  if (rows <= 0 || cols <= 0) return MCNLA_B200_OK;
  k_fill<<<grid_for(c, rows * cols, 256), 256, 0, c->stream>>>(rows, cols, v, X, ld, 0);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_gramian_prepare(Context* c, int64_t L, int l, double* bs, double* bc, int64_t ldbc) {
  k_gramian_prepare<<<grid_for(c, L * L, 256), 256, 0, c->stream>>>(L, l, bs, bc, ldbc);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_wy_gramian_phis(Context* c, int l, const double* F, const double* dc, int64_t lddc, const double* dp,
                           int64_t lddp, double* phi1, double* phi2) {
  k_wy_gramian_phis<<<grid_for(c, int64_t(l) * l, 256), 256, 0, c->stream>>>(l, F, dc, lddc, dp, lddp, phi1, phi2);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_svd_small(Context* c, int n, const double* M, double* W, double* sig, double* Z) {
  if (n < 1 || n > MCNLA_B200_MAX_DIM_SKETCH) return MCNLA_B200_ERR_UNSUPPORTED;
  const size_t mat = size_t(n) * (n + 1) * 8 + 16;
  const int npairs = (n + 2) / 2;
  const size_t extra = 64 + n * 4 + 16 + n * 8 + 16 + 2 * (npairs * 8 + 16) + 2 * (npairs * 4 + 16) + 64;
  const bool z_smem = 2 * mat + extra <= c->smem_optin;
  const size_t smem = (z_smem ? 2 : 1) * mat + extra;
  if (smem > c->smem_optin) return MCNLA_B200_ERR_UNSUPPORTED;
  double* zwork = z_smem ? nullptr : ctx_take<double>(c, size_t(n) * n);
  if (!z_smem && !zwork) return MCNLA_B200_ERR_WORKSPACE;
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_svd_small), smem));
  k_svd_small<<<1, kSmallThreads, smem, c->stream>>>(n, M, W, sig, Z, zwork, z_smem ? 1 : 0);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_rsqrt_rows_t(Context* c, int n, const double* Ue, const double* w, double* P) {
  k_rsqrt_rows_t<<<grid_for(c, int64_t(n) * n, 256), 256, 0, c->stream>>>(n, Ue, w, P);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_scale_cols(Context* c, int64_t rows, int64_t cols, const double* X, int64_t ldx, const double* s,
                      int mode, double* Y, int64_t ldy) {
  if (rows <= 0 || cols <= 0) return MCNLA_B200_OK;
  k_scale_cols<<<grid_for(c, rows * cols, 256), 256, 0, c->stream>>>(rows, cols, X, ldx, s, mode, Y, ldy);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_sqrt_vec(Context* c, int n, const double* w, double* out) {
  k_sqrt_vec<<<1, 256, 0, c->stream>>>(n, w, out);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_gwy_small_dots(Context* c, int l, const double* phi1, const double* phi2, const double* bcu, double* out) {
  k_gwy_small_dots<<<1, kRedThreads, 0, c->stream>>>(l, phi1, phi2, bcu, out);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_inverse(Context* c, int n, int batch, double* A) {
  if (n < 1 || n > 2 * MCNLA_B200_MAX_DIM_SKETCH_WENYIN || batch < 1) return MCNLA_B200_ERR_UNSUPPORTED;
  const size_t smem = size_t(n) * (n + 1) * 8 + 16 + gj_scratch_bytes(n) + 64;
  if (smem > c->smem_optin) return MCNLA_B200_ERR_UNSUPPORTED;
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_inverse), smem));
  k_inverse<<<batch, kGjThreads, smem, c->stream>>>(n, A, c->scal);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_gaussian(Context* c, uint64_t seed, int64_t count, double* out) {
  if (count <= 0) return MCNLA_B200_OK;
  k_gaussian<<<grid_for(c, (count + 1) / 2, 256), 256, 0, c->stream>>>(seed, count, out);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

}  // namespace mb
