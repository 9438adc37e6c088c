// Kolmogorov-Nagumo step by power series, on several CTAs.
//
// The step needs C = f(Z) and inv(C) for f(x) = sqrt(1/2 + sqrt(1/4 - x)),
// which the reference forms from an eigendecomposition of the symmetric Z
// (row_block_kolmogorov_nagumo_integrator.hpp:159-180,
// kolmogorov_nagumo_integrator.hpp:146-164).  With c(x) the generating
// function of the Catalan numbers, c(x) = (1 - sqrt(1 - 4x)) / (2x), one has
// (1 + sqrt(1 - 4x)) / 2 = 1 / c(x), so
//     f(x) = c(x)^(-1/2),   1 / f(x) = c(x)^(1/2),
// and the powers of c have the closed-form series (Lagrange inversion)
//     c(x)^r = sum_n  r / (2n + r) * binom(2n + r, n) * x^n,   |x| < 1/4.
// Both series have |a_{n+1}| / |a_n| < 4, so for z = ||Z||_F (>= ||Z||_2)
// the tail after degree d is below |a_{d+1}| z^(d+1) / (1 - 4z).  The kernel
// picks the smallest d with a tail under 1e-17 and evaluates both
// polynomials by Paterson-Stockmeyer (Z^2 .. Z^s, then Horner in Z^s) on the
// FP64 MMA.  Near convergence Z is tiny (4 ||Z|| ~ 1e-4 .. 1e-2: degree 3 to
// 10); when 4 ||Z||_F > 1/2 (the first iterations) the kernel sets
// scal->kn_fallback and the matrix-function / eigendecomposition kernel that
// follows it in the stream does the step instead.
//
// Work split: CTA b owns rows [8b, 8b + 8) of every l x l matrix.  A product
// X Y with Y = Z or Z^s (read-only, in global memory) only needs the CTA's
// own rows of X, so the powers and the Horner steps run without exchange;
// grid barriers (cooperative launch, bounded waits) separate the phases that
// read whole matrices written by other CTAs: Z, Z^s, inv(C) and Fc.
#include "kernels.cuh"

namespace mb {
namespace {

constexpr int kSerThreads = 256;
constexpr int kSerCoefs = 128;          // series coefficients kept on chip
constexpr int kSerMaxDegree = 94;       // degree search limit (s, q <= 10)
constexpr int kSerMaxS = 10;            // power slabs Z^1 .. Z^s on chip
constexpr double kSerMaxRho = 0.5;      // 4 ||Z||_F above this: fallback kernel
constexpr double kSerTail = 1e-17;
constexpr long long kBarrierCycles = 4000000000LL;   // about 2 s at the boost clock

struct SeriesArgs {
  int l;
  const double* z_in;     // plain: Z (l x l), upper triangle read
  const double* dd;       // row block: [Dc | Dgc] (l x 2l)
  double inv_n;
  double* out;            // [C; inv(C)] or [Fc; inv(C)]  (2l x l)
  double* outn;           // [Fc; inv(C)/N] (optional)
  const double* ff;       // F~c (optional, l x l)
  double* ffn;            // F~c Fc
  double* zg;             // scratch: Z (l x l)
  double* zsg;            // scratch: Z^s (l x l)
  double* partials;       // scratch: 2 * gridDim.x
  DevScalars* scal;
  double tol;
  const int* guard_stop;
  int guard_it;
};

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Barrier over the whole (co-resident) grid.  Returns false when the wait
// gave up; the kernel then records MCNLA_B200_ERR_DEVICE_TIMEOUT and returns.
__device__ bool grid_sync(DevScalars* scal, volatile int* flag) {
  __syncthreads();
  if (gridDim.x == 1) return true;
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &scal->bar_gen;
    const unsigned g = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&scal->bar_count, 1u) == gridDim.x - 1) {
      atomicExch(&scal->bar_count, 0u);
      __threadfence();
      atomicAdd(&scal->bar_gen, 1u);
    } else {
      const long long t0 = clock64();
      while (*gen == g) {
        if (clock64() - t0 > kBarrierCycles) {
          ok = 0;
          atomicExch(&scal->status, MCNLA_B200_ERR_DEVICE_TIMEOUT);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    *flag = ok;
  }
  __syncthreads();
  return *flag != 0;
}

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w];
  return s;                       // valid in thread 0
}

// C1 = A1 Y (and C2 = A2 Y): A 8 x l slabs in shared memory (row stride ld,
// zero beyond column l), Y l x l in global memory (row stride ldy), C slabs
// in shared memory.  One warp per 8-column tile; the Y fragments are shared
// by the two products.  Ends with a block barrier.
__device__ void slab_mm(const double* A1, const double* A2, int ld, const double* Y, int ldy, int l, double* C1,
                        double* C2) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int ntiles = (l + 7) >> 3;
  const int kend = (l + 3) & ~3;
  for (int t = warp; t < ntiles; t += kSerThreads / 32) {
    const int n = t * 8 + g;
    double c10 = 0.0, c11 = 0.0, c20 = 0.0, c21 = 0.0;
    double e10 = 0.0, e11 = 0.0, e20 = 0.0, e21 = 0.0;    // second chain (k0 = 4 mod 8)
    int k0 = 0;
    for (; k0 + 8 <= kend; k0 += 8) {
      const int ka = k0 + t4, kb = k0 + 4 + t4;
      const double ya = (ka < l && n < l) ? __ldcg(Y + size_t(ka) * ldy + n) : 0.0;
      const double yb = (kb < l && n < l) ? __ldcg(Y + size_t(kb) * ldy + n) : 0.0;
      dmma(c10, c11, A1[g * ld + ka], ya);
      dmma(e10, e11, A1[g * ld + kb], yb);
      if (A2) {
        dmma(c20, c21, A2[g * ld + ka], ya);
        dmma(e20, e21, A2[g * ld + kb], yb);
      }
    }
    if (k0 < kend) {
      const int ka = k0 + t4;
      const double ya = (ka < l && n < l) ? __ldcg(Y + size_t(ka) * ldy + n) : 0.0;
      dmma(c10, c11, A1[g * ld + ka], ya);
      if (A2) dmma(c20, c21, A2[g * ld + ka], ya);
    }
    double* o1 = C1 + g * ld + t * 8 + 2 * t4;
    o1[0] = c10 + e10;
    o1[1] = c11 + e11;
    if (A2) {
      double* o2 = C2 + g * ld + t * 8 + 2 * t4;
      o2[0] = c20 + e20;
      o2[1] = c21 + e21;
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kSerThreads) k_kn_series(SeriesArgs a) {
  extern __shared__ __align__(16) double sm[];
  if (a.guard_stop && *a.guard_stop < a.guard_it) return;
  __shared__ int s_flag, s_d, s_s;
  const int l = a.l, tid = threadIdx.x, nt = blockDim.x;
  const int lp8 = (l + 7) & ~7, ld = lp8 + 4;
  const int r0 = blockIdx.x * 8, G = gridDim.x;
  const int slab = 8 * ld;
  double* P = sm;                                   // P + (j-1) slab: rows of Z^j, j = 1 .. s
  double* accF = P + kSerMaxS * slab;
  double* accG = accF + slab;
  double* tF = accG + slab;
  double* tG = tF + slab;
  double* coefF = tG + slab;                        // c^(-1/2): C
  double* coefG = coefF + kSerCoefs;                // c^(1/2):  inv(C)
  double* red = coefG + kSerCoefs;
  for (int e = tid; e < (kSerMaxS + 4) * slab; e += nt) sm[e] = 0.0;
  __syncthreads();

  // ---- Z rows [r0, r0 + 8): the upper triangle mirrored (the symmetric
  // eigensolver of the reference reads one triangle)
  const int ldd = 2 * l;
  double part = 0.0;
  for (int e = tid; e < 8 * l; e += nt) {
    const int rr = e / l, j = e % l, i = r0 + rr;
    if (i >= l) continue;
    const int p = min(i, j), q = max(i, j);
    double v;
    if (a.dd == nullptr) {
      v = a.z_in[size_t(p) * l + q];
    } else {
      // Z := Dgc - Dc Dc'   (row_block_kolmogorov_nagumo_integrator.hpp:150-156)
      const double* dp = a.dd + size_t(p) * ldd;
      const double* dq = a.dd + size_t(q) * ldd;
      double s = 0.0;
      for (int k = 0; k < l; ++k) s = fma(dp[k], dq[k], s);
      v = dp[l + q] - s;
    }
    P[rr * ld + j] = v;
    a.zg[size_t(i) * l + j] = v;
    part += v * v;
  }
  part = block_sum(part, red);
  if (tid == 0) a.partials[blockIdx.x] = part;
  if (!grid_sync(a.scal, &s_flag)) return;

  // ---- degree from ||Z||_F (same arithmetic in every CTA)
  if (tid == 0) {
    double s2 = 0.0;
    for (int b = 0; b < G; ++b) s2 += __ldcg(a.partials + b);
    const double z = sqrt(s2);
    int d = -1;
    if (4.0 * z <= kSerMaxRho) {                    // false for NaN
      double bF = 1.0, bG = 1.0;                    // binom(2n + r, n), r = -1/2, +1/2
      for (int n = 0; n < kSerCoefs; ++n) {
        coefF[n] = -0.5 / (2.0 * n - 0.5) * bF;
        coefG[n] = 0.5 / (2.0 * n + 0.5) * bG;
        bF *= (2.0 * n + 1.5) * (2.0 * n + 0.5) / ((n + 1.0) * (n + 0.5));
        bG *= (2.0 * n + 2.5) * (2.0 * n + 1.5) / ((n + 1.0) * (n + 1.5));
      }
      const double scale = 1.0 / (1.0 - 4.0 * z);
      double zn = 1.0;
      for (int n = 1; n <= kSerMaxDegree + 1; ++n) {
        zn *= z;
        if (fmax(fabs(coefF[n]), fabs(coefG[n])) * zn * scale <= kSerTail) { d = n - 1; break; }
      }
      if (d == 0) d = 1;
    }
    int s = 1;
    while (d >= 0 && s * s < d + 1) ++s;
    s_d = d;
    s_s = s;
    if (blockIdx.x == 0) a.scal->kn_fallback = d < 0 ? 1 : 0;
  }
  __syncthreads();
  const int d = s_d;
  if (d < 0) return;                                // uniform over the grid
  const int s = s_s;
  const int nq = (d + s) / s;                       // blocks of s coefficients: degree nq*s - 1 >= d

  // ---- rows of Z^2 .. Z^s
  for (int j = 2; j <= s; ++j) slab_mm(P + (j - 2) * slab, nullptr, ld, a.zg, l, l, P + (j - 1) * slab, nullptr);
  if (nq > 1) {
    for (int e = tid; e < 8 * l; e += nt) {
      const int rr = e / l, j = e % l, i = r0 + rr;
      if (i < l) a.zsg[size_t(i) * l + j] = P[(s - 1) * slab + rr * ld + j];
    }
    if (!grid_sync(a.scal, &s_flag)) return;
  }

  // ---- Horner in Z^s:  acc = B_{nq-1};  acc = acc Z^s + B_q,  B_q = sum_j a_{qs+j} Z^j
  auto add_block = [&](int q, double* dF, double* dG, bool accumulate) {
    for (int e = tid; e < 8 * lp8; e += nt) {
      const int rr = e / lp8, j = e % lp8, i = r0 + rr;
      double vF = 0.0, vG = 0.0;
      if (i < l && j < l) {
        if (i == j) {
          vF = coefF[q * s];
          vG = coefG[q * s];
        }
        for (int p = 1; p < s; ++p) {
          const double x = P[(p - 1) * slab + rr * ld + j];
          vF = fma(coefF[q * s + p], x, vF);
          vG = fma(coefG[q * s + p], x, vG);
        }
      }
      const int o = rr * ld + j;
      if (accumulate) {
        dF[o] += vF;
        dG[o] += vG;
      } else {
        dF[o] = vF;
        dG[o] = vG;
      }
    }
    __syncthreads();
  };
  add_block(nq - 1, accF, accG, false);
  for (int q = nq - 2; q >= 0; --q) {
    slab_mm(accF, accG, ld, a.zsg, l, l, tF, tG);
    add_block(q, tF, tG, true);
    double* x = accF; accF = tF; tF = x;
    x = accG; accG = tG; tG = x;
  }

  // ---- C in accF, inv(C) in accG;  ||e - 1||_2 = ||C - I||_F
  double* cinv = a.out + size_t(l) * l;
  part = 0.0;
  for (int e = tid; e < 8 * l; e += nt) {
    const int rr = e / l, j = e % l, i = r0 + rr;
    if (i >= l) continue;
    const int o = rr * ld + j;
    const double c = accF[o];
    const double dlt = c - (i == j ? 1.0 : 0.0);
    part += dlt * dlt;
    cinv[size_t(i) * l + j] = accG[o];
    if (a.dd == nullptr) a.out[size_t(i) * l + j] = c;
  }
  part = block_sum(part, red);
  if (tid == 0) a.partials[G + blockIdx.x] = part;
  if (!grid_sync(a.scal, &s_flag)) return;

  if (a.dd != nullptr) {
    // Fc := C - Dc inv(C)   (row_block_kolmogorov_nagumo_integrator.hpp:186)
    for (int e = tid; e < 8 * lp8; e += nt) {
      const int rr = e / lp8, j = e % lp8, i = r0 + rr;
      tF[rr * ld + j] = (i < l && j < l) ? a.dd[size_t(i) * ldd + j] : 0.0;
    }
    __syncthreads();
    slab_mm(tF, nullptr, ld, cinv, l, l, tG, nullptr);
    for (int e = tid; e < 8 * l; e += nt) {
      const int rr = e / l, j = e % l, i = r0 + rr;
      if (i >= l) continue;
      const int o = rr * ld + j;
      const double fc = accF[o] - tG[o];
      a.out[size_t(i) * l + j] = fc;
      if (a.outn) {
        a.outn[size_t(i) * l + j] = fc;
        a.outn[size_t(l) * l + size_t(i) * l + j] = accG[o] * a.inv_n;
      }
    }
    if (a.ff && a.ffn) {
      // F~+ := F~c Fc   (row_block_gramian_kolmogorov_nagumo_integrator.hpp:197)
      if (!grid_sync(a.scal, &s_flag)) return;
      for (int e = tid; e < 8 * lp8; e += nt) {
        const int rr = e / lp8, j = e % lp8, i = r0 + rr;
        tF[rr * ld + j] = (i < l && j < l) ? a.ff[size_t(i) * l + j] : 0.0;
      }
      __syncthreads();
      slab_mm(tF, nullptr, ld, a.out, l, l, tG, nullptr);
      for (int e = tid; e < 8 * l; e += nt) {
        const int rr = e / l, j = e % l, i = r0 + rr;
        if (i < l) a.ffn[size_t(i) * l + j] = tG[rr * ld + j];
      }
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    double s2 = 0.0;
    for (int b = 0; b < G; ++b) s2 += __ldcg(a.partials + G + b);
    const double norm = sqrt(s2);
    a.scal->norm = norm;
    a.scal->sweeps = 1000 + d;
    if (a.guard_stop && !(norm >= a.tol)) a.scal->stop_it = a.guard_it;
  }
}

}  // namespace

size_t kn_series_work_doubles(int l) { return 2 * size_t(l) * l + 2 * size_t((l + 7) / 8) + 8; }

int launch_kn_series(Context* c, int l, const double* z, const double* dd, double inv_n, double* out, double* outn,
                     const double* ff, double* ffn, double* work, double tol) {
  if (l < 1 || l > MCNLA_B200_MAX_DIM_SKETCH) return MCNLA_B200_ERR_UNSUPPORTED;
  const int G = (l + 7) / 8;
  const int ld = ((l + 7) & ~7) + 4;
  const size_t smem = (size_t(kSerMaxS + 4) * 8 * ld + 2 * kSerCoefs + 32) * sizeof(double);
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_kn_series), smem));
  SeriesArgs a;
  a.l = l;
  a.z_in = z;
  a.dd = dd;
  a.inv_n = inv_n;
  a.out = out;
  a.outn = outn;
  a.ff = ff;
  a.ffn = ffn;
  a.zg = work;
  a.zsg = work + size_t(l) * l;
  a.partials = work + 2 * size_t(l) * l;
  a.scal = c->scal;
  a.tol = tol;
  a.guard_stop = c->guard_stop;
  a.guard_it = c->guard_it;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(G));
  cfg.blockDim = dim3(kSerThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MB_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_kn_series, a));
  c->kernels_launched++;
  return MCNLA_B200_OK;
}

}  // namespace mb
