// Kolmogorov-Nagumo step by power series: device building blocks shared by
// the stand-alone step kernel (kn_series.cu) and the persistent row-block
// Gramian integrator (gkn_persistent.cu).
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
// the tail after degree d is below |a_{d+1}| z^(d+1) / (1 - 4z).  The step
// picks the smallest d with a tail under 1e-17 and evaluates both
// polynomials by Paterson-Stockmeyer (Z^2 .. Z^s, then Horner in Z^s) on the
// FP64 MMA.  Near convergence Z is tiny (4 ||Z|| ~ 1e-4 .. 1e-2: degree 3 to
// 10); when 4 ||Z||_F > 1/2 (the first iterations) the step declines and the
// caller runs the matrix-function / eigendecomposition form instead.
//
// Work split: CTA b < ceil(l/8) owns rows [8b, 8b + 8) of every l x l
// matrix.  A product X Y with Y = Z or Z^s (read-only, in global memory)
// only needs the CTA's own rows of X, so the powers and the Horner steps run
// without exchange; grid barriers (cooperative launch, bounded waits)
// separate the phases that read whole matrices written by other CTAs: Z,
// Z^s, inv(C) and Fc.  Every CTA of the grid takes part in the barriers.
#pragma once
#include "kernels.cuh"

namespace mb {
namespace {

constexpr int kSerCoefs = 320;          // series coefficients kept in constant memory
constexpr int kSerMaxDegree = 300;      // degree search limit
constexpr int kSerMaxS = 18;            // most power slabs Z^1 .. Z^s on chip (fewer when they do not fit)
constexpr int kSerDirectMax = 12;       // degree up to which plain powers replace Paterson-Stockmeyer
constexpr int kSerZsMax = 112;          // l up to which Z is staged in shared memory for its products
constexpr double kSerMaxRho = 0.9;      // 4 ||Z|| above this: the step declines
constexpr double kSerTail = 1e-17;
constexpr long long kBarrierCycles = 4000000000LL;   // about 2 s at the boost clock

// Series coefficients a_n(r) = r / (2n + r) * binom(2n + r, n) of c(x)^r
// for r = -1/2 (C) and r = +1/2 (inv(C)), from the ratio
// binom(2n + r + 2, n + 1) / binom(2n + r, n) = (2n + r + 2)(2n + r + 1) / ((n + 1)(n + r + 1)),
// evaluated at compile time (IEEE double arithmetic, the same on host and device).
struct SeriesCoefs {
  double f[kSerCoefs];
  double g[kSerCoefs];
};

constexpr SeriesCoefs make_series_coefs() {
  SeriesCoefs t{};
  double bF = 1.0, bG = 1.0;
  for (int n = 0; n < kSerCoefs; ++n) {
    t.f[n] = -0.5 / (2.0 * n - 0.5) * bF;
    t.g[n] = 0.5 / (2.0 * n + 0.5) * bG;
    bF *= (2.0 * n + 1.5) * (2.0 * n + 0.5) / ((n + 1.0) * (n + 0.5));
    bG *= (2.0 * n + 2.5) * (2.0 * n + 1.5) / ((n + 1.0) * (n + 1.5));
  }
  return t;
}

__constant__ SeriesCoefs c_series = make_series_coefs();

// Operands of one step (all l x l blocks row-major with row stride l).
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
  double* partials;       // scratch: 3 * ceil(l/8)
  DevScalars* scal;
  int smax;               // power slabs on chip (kn_series_smax)
};

// Shared memory of the step: smax + 4 slabs of 8 rows, reduction space and,
// for l <= kSerZsMax, a copy of Z (l rows, the slab row stride).
__host__ __device__ constexpr size_t kn_series_smem_doubles(int l, int smax) {
  return size_t(smax + 4) * 8 * (((l + 7) & ~7) + 4) + 32 +
         (l <= kSerZsMax ? size_t(l) * (((l + 7) & ~7) + 4) : 0);
}

// Most power slabs (<= kSerMaxS) whose step fits `optin` bytes of shared
// memory next to `extra` doubles of the calling kernel (0 when even 4 do not).
inline int kn_series_smax(int l, size_t optin, size_t extra) {
  for (int smax = kSerMaxS; smax >= 4; --smax)
    if ((kn_series_smem_doubles(l, smax) + extra) * sizeof(double) + 1024 <= optin) return smax;
  return 0;
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Barrier over the whole (co-resident) grid.  scal->bar_count only grows: at
// a launch it is a multiple of the grid size (zeroed with the scalars at the
// start of a stage; every CTA passes the same number of barriers), so an
// arriving CTA whose atomic returns `old` waits until the count reaches the
// next multiple of gridDim.x.  One release (fence + relaxed add) per CTA and
// acquire polls: no reset on the critical path.  Returns false when the wait
// gave up (MCNLA_B200_ERR_DEVICE_TIMEOUT is recorded); the kernel returns.
__device__ bool grid_sync(DevScalars* scal, volatile int* flag) {
  __syncthreads();
  if (gridDim.x == 1) return true;
  if (threadIdx.x == 0) {
    unsigned* cnt = &scal->bar_count;
    unsigned old;
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    asm volatile("atom.add.relaxed.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(cnt) : "memory");
    const unsigned target = (old / gridDim.x + 1) * gridDim.x;
    int ok = 1;
    const long long t0 = clock64();
    while (true) {
      unsigned cur;
      asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(cnt) : "memory");
      if (int(cur - target) >= 0) break;
      if (clock64() - t0 > kBarrierCycles) {
        ok = 0;
        atomicExch(&scal->status, MCNLA_B200_ERR_DEVICE_TIMEOUT);
        break;
      }
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
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

// Fragment loop of one 8 x 8 output tile: c += sum_{k in [kb, ke)} A(g, k) B(k, g')
// with the m8n8k4 FP64 MMA, where lane (g, t4) supplies fa(k) = A(row g, k)
// and fb(k) = B(k, column g) for k = k0 + t4 (both return 0 outside the
// operands; k < ke is checked here).  The loads of kU consecutive k-steps are
// issued before their MMAs so that kU L2 round trips overlap; two
// accumulation chains.  c0, c1: the lane's two accumulator elements.
constexpr int kU = 8;

template <class FA, class FB>
__device__ __forceinline__ void tile_acc(FA fa, FB fb, int kb, int ke, double& c0, double& c1) {
  const int t4 = threadIdx.x & 3;
  double e0 = 0.0, e1 = 0.0;
  for (int k = kb; k < ke; k += 4 * kU) {
    double a[kU], b[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int kk = k + 4 * u + t4;
      const bool kv = kk < ke;
      a[u] = kv ? fa(kk) : 0.0;
      b[u] = kv ? fb(kk) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kU; u += 2) {
      dmma(c0, c1, a[u], b[u]);
      dmma(e0, e1, a[u + 1], b[u + 1]);
    }
  }
  c0 += e0;
  c1 += e1;
}

// Two tiles with the same B fragments: c += A1 B, d += A2 B.
template <class FA1, class FA2, class FB>
__device__ __forceinline__ void tile_acc2(FA1 fa1, FA2 fa2, FB fb, int kb, int ke, double& c0, double& c1, double& d0,
                                          double& d1) {
  const int t4 = threadIdx.x & 3;
  for (int k = kb; k < ke; k += 4 * kU) {
    double a1[kU], a2[kU], b[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int kk = k + 4 * u + t4;
      const bool kv = kk < ke;
      a1[u] = kv ? fa1(kk) : 0.0;
      a2[u] = kv ? fa2(kk) : 0.0;
      b[u] = kv ? fb(kk) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      dmma(c0, c1, a1[u], b[u]);
      dmma(d0, d1, a2[u], b[u]);
    }
  }
}

// C1 = A1 Y (and C2 = A2 Y): A 8 x l slabs in shared memory (row stride ld,
// zero beyond column l), Y l x l in global memory (row stride ldy; or in
// shared memory for SMEM_Y), C slabs in shared memory.  One warp per 8-column
// tile; the two products share the Y fragments.  Ends with a block barrier.
template <bool TRANS_Y = false, bool SMEM_Y = false>
__device__ void slab_mm(const double* A1, const double* A2, int ld, const double* Y, int ldy, int l, double* C1,
                        double* C2) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int ntiles = (l + 7) >> 3;
  for (int t = warp; t < ntiles; t += nw) {
    const int n = t * 8 + g;
    const bool nv = n < l;
    // Y(k, n), or Y(n, k) for TRANS_Y
    auto fy = [&](int k) {
      const double* y = TRANS_Y ? Y + size_t(n) * ldy + k : Y + size_t(k) * ldy + n;
      return nv ? (SMEM_Y ? *y : __ldcg(y)) : 0.0;
    };
    double c0 = 0.0, c1 = 0.0;
    double* o1 = C1 + g * ld + t * 8 + 2 * t4;
    if (A2) {
      double d0 = 0.0, d1 = 0.0;
      tile_acc2([&](int k) { return A1[g * ld + k]; }, [&](int k) { return A2[g * ld + k]; }, fy, 0, l, c0, c1, d0,
                d1);
      double* o2 = C2 + g * ld + t * 8 + 2 * t4;
      o2[0] = d0;
      o2[1] = d1;
    } else {
      tile_acc([&](int k) { return A1[g * ld + k]; }, fy, 0, l, c0, c1);
    }
    o1[0] = c0;
    o1[1] = c1;
  }
  __syncthreads();
}

// Step operands with the scratch carved out of `work` (kn_series_work_doubles(l)).
inline SeriesArgs series_args(Context* c, int l, const double* z, const double* dd, double inv_n, double* out,
                       double* outn, const double* ff, double* ffn, double* work, int smax) {
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
  a.smax = smax;
  return a;
}

enum : int { kStepTimeout = -1, kStepDeclined = 0, kStepDone = 1 };

// One KN step (see the file comment).  Every CTA of the grid calls it; CTAs
// [0, ceil(l/8)) do the work.  Returns kStepDone (C / Fc / inv(C) / F~+ in
// global memory, *norm = ||C - I||_F and *degree in every thread),
// kStepDeclined (4 min(||Z||_F, ||Z||_inf) > 0.9 or not finite; nothing
// written but Z) or
// kStepTimeout.  end_barrier: end with a grid barrier after [Fc; inv(C)] are
// written (when other CTAs read them next); F~+ is written after it.
__device__ int kn_series_step(const SeriesArgs& a, double* sm, volatile int* flag, bool end_barrier, double* norm,
                              int* degree) {
  __shared__ int s_d, s_s;
  __shared__ double s_norm;
  const int l = a.l, tid = threadIdx.x, nt = blockDim.x;
  const int gkn = (l + 7) >> 3;
  const bool mine = int(blockIdx.x) < gkn;
  const int lp8 = (l + 7) & ~7, ld = lp8 + 4;
  const int r0 = blockIdx.x * 8;
  const int slab = 8 * ld;
  double* P = sm;                                   // P + (j-1) slab: rows of Z^j, j = 1 .. s
  const int smax = a.smax;
  double* accF = P + smax * slab;
  double* accG = accF + slab;
  double* tF = accG + slab;
  double* tG = tF + slab;
  double* red = tG + slab;
  const double* coefF = c_series.f;                 // c^(-1/2): C
  const double* coefG = c_series.g;                 // c^(1/2):  inv(C)
  const int ldd = 2 * l;
  if (mine) {
    for (int e = tid; e < (smax + 4) * slab; e += nt) sm[e] = 0.0;
    __syncthreads();
    // ---- Z rows [r0, r0 + 8)
    if (a.dd != nullptr) {
      // Z := Dgc - Dc Dc'   (row_block_kolmogorov_nagumo_integrator.hpp:150-156): Dc rows into tF,
      // Dc Dc' rows into tG on the MMA
      for (int e = tid; e < 8 * lp8; e += nt) {
        const int rr = e / lp8, j = e % lp8, i = r0 + rr;
        tF[rr * ld + j] = (i < l && j < l) ? __ldcg(a.dd + size_t(i) * ldd + j) : 0.0;
      }
      __syncthreads();
      slab_mm<true>(tF, nullptr, ld, a.dd, ldd, l, tG, nullptr);
    }
    double part = 0.0;
    for (int e = tid; e < 8 * l; e += nt) {
      const int rr = e / l, j = e % l, i = r0 + rr;
      if (i >= l) continue;
      double v;
      if (a.dd == nullptr) {
        // the upper triangle mirrored (the reference's symmetric eigensolver reads one triangle)
        v = __ldcg(a.z_in + size_t(min(i, j)) * l + max(i, j));
      } else {
        v = __ldcg(a.dd + size_t(i) * ldd + l + j) - tG[rr * ld + j];
      }
      P[rr * ld + j] = v;
      a.zg[size_t(i) * l + j] = v;
      part += v * v;
    }
    part = block_sum(part, red);
    if (tid == 0) a.partials[blockIdx.x] = part;
    // absolute row sums of the CTA's rows (a warp per row, fixed order) for
    // the infinity-norm bound; red[16 ..] is clear of block_sum's slots
    const int warp = tid >> 5, lane = tid & 31;
    if (warp < 8) {
      double rs = 0.0;
      for (int j = lane; j < l; j += 32) rs += fabs(P[warp * ld + j]);
      for (int o = 16; o > 0; o >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, o);
      if (lane == 0) red[16 + warp] = rs;
    }
    __syncthreads();
    if (tid == 0) {
      double mx = 0.0;
      for (int w = 0; w < 8; ++w) mx = fmax(mx, red[16 + w]);
      a.partials[2 * gkn + blockIdx.x] = mx;
    }
  }
  if (!grid_sync(a.scal, flag)) return kStepTimeout;

  // ---- degree from z = min(||Z||_F, ||Z||_inf) >= ||Z||_2 (the same arithmetic in every CTA)
  if (tid == 0) {
    double s2 = 0.0, zi = 0.0;
    for (int b = 0; b < gkn; ++b) {
      s2 += __ldcg(a.partials + b);
      zi = fmax(zi, __ldcg(a.partials + 2 * gkn + b));
    }
    const double z = fmin(sqrt(s2), zi);
    int d = -1;
    if (4.0 * z <= kSerMaxRho) {                    // false for NaN
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
    if (s > smax) s = smax;
    s_d = d;
    s_s = s;
  }
  __syncthreads();
  const int d = s_d;
  if (d < 0) return kStepDeclined;                  // uniform over the grid
  const int s = s_s;
  const int nq = (d + s) / s;                       // blocks of s coefficients: degree nq*s - 1 >= d
  double* cinv = a.out + size_t(l) * l;
  const bool rb = a.dd != nullptr;
  // Z for the products below: a shared-memory copy when it fits
  const bool zs_smem = l <= kSerZsMax;
  double* zs = red + 32;
  if (mine && zs_smem) {
    for (int e = tid; e < l * l; e += nt) zs[(e / l) * ld + (e % l)] = __ldcg(a.zg + e);
    __syncthreads();
  }
  auto mm_z = [&](const double* A1, const double* A2, double* C1, double* C2) {
    if (zs_smem) slab_mm<false, true>(A1, A2, ld, zs, ld, l, C1, C2);
    else slab_mm(A1, A2, ld, a.zg, l, l, C1, C2);
  };

  if (d <= kSerDirectMax) {
    // ---- plain powers: C = sum f_j Z^j, inv(C) = sum g_j Z^j and, for the
    // row-block step, Dc inv(C) = sum g_j (Dc Z^j), all accumulated from the
    // CTA's rows of Z^j and Dc Z^j (products with the full Z only), so Fc
    // = C - Dc inv(C) needs no exchange of C or inv(C).
    if (mine) {
      double* Pa = P;                               // rows of Z (from above)
      double* Pb = P + 1 * slab;
      double* Wa = P + 2 * slab;                    // rows of Dc Z^j
      double* Wb = P + 3 * slab;
      double* DW = P + 4 * slab;                    // rows of sum g_j Dc Z^j
      for (int e = tid; e < 8 * lp8; e += nt) {
        const int rr = e / lp8, j = e % lp8, i = r0 + rr;
        const int o = rr * ld + j;
        const double id = (i == j && i < l) ? 1.0 : 0.0;
        accF[o] = coefF[0] * id + coefF[1] * Pa[o];
        accG[o] = coefG[0] * id + coefG[1] * Pa[o];
        if (rb) DW[o] = coefG[0] * tF[o];           // tF: rows of Dc
      }
      __syncthreads();
      if (rb) {
        mm_z(tF, nullptr, Wa, nullptr);
        for (int e = tid; e < 8 * lp8; e += nt) {
          const int o = (e / lp8) * ld + e % lp8;
          DW[o] += coefG[1] * Wa[o];
        }
        __syncthreads();
      }
      double *pc = Pa, *pn = Pb, *wc = Wa, *wn = Wb;
      for (int j = 2; j <= d; ++j) {
        mm_z(pc, rb ? wc : nullptr, pn, rb ? wn : nullptr);
        for (int e = tid; e < 8 * lp8; e += nt) {
          const int o = (e / lp8) * ld + e % lp8;
          accF[o] += coefF[j] * pn[o];
          accG[o] += coefG[j] * pn[o];
          if (rb) DW[o] += coefG[j] * wn[o];
        }
        __syncthreads();
        double* x = pc; pc = pn; pn = x;
        x = wc; wc = wn; wn = x;
      }
      double part = 0.0;
      for (int e = tid; e < 8 * l; e += nt) {
        const int rr = e / l, j = e % l, i = r0 + rr;
        if (i >= l) continue;
        const int o = rr * ld + j;
        const double c = accF[o], ci = accG[o];
        const double dlt = c - (i == j ? 1.0 : 0.0);
        part += dlt * dlt;
        cinv[size_t(i) * l + j] = ci;
        if (!rb) {
          a.out[size_t(i) * l + j] = c;
        } else {
          // Fc := C - Dc inv(C)   (row_block_kolmogorov_nagumo_integrator.hpp:186)
          const double fc = c - DW[o];
          a.out[size_t(i) * l + j] = fc;
          if (a.outn) {
            a.outn[size_t(i) * l + j] = fc;
            a.outn[size_t(l) * l + size_t(i) * l + j] = ci * a.inv_n;
          }
        }
      }
      part = block_sum(part, red);
      if (tid == 0) a.partials[gkn + blockIdx.x] = part;
    }
    if (!grid_sync(a.scal, flag)) return kStepTimeout;
    if (tid == 0) {
      double s2 = 0.0;
      for (int b = 0; b < gkn; ++b) s2 += __ldcg(a.partials + gkn + b);
      s_norm = sqrt(s2);
    }
    if (rb && a.ff && a.ffn && mine) {
      // F~+ := F~c Fc   (row_block_gramian_kolmogorov_nagumo_integrator.hpp:197)
      for (int e = tid; e < 8 * lp8; e += nt) {
        const int rr = e / lp8, j = e % lp8, i = r0 + rr;
        tF[rr * ld + j] = (i < l && j < l) ? __ldcg(a.ff + size_t(i) * l + j) : 0.0;
      }
      __syncthreads();
      slab_mm(tF, nullptr, ld, a.out, l, l, tG, nullptr);
      for (int e = tid; e < 8 * l; e += nt) {
        const int rr = e / l, j = e % l, i = r0 + rr;
        if (i < l) a.ffn[size_t(i) * l + j] = tG[rr * ld + j];
      }
    }
    __syncthreads();
    *norm = s_norm;
    *degree = d;
    return kStepDone;
  }

  // ---- rows of Z^2 .. Z^s (Z^s only when a Horner step needs it)
  if (mine) {
    const int top = nq > 1 ? s : s - 1;
    for (int j = 2; j <= top; ++j) mm_z(P + (j - 2) * slab, nullptr, P + (j - 1) * slab, nullptr);
    if (nq > 1) {
      for (int e = tid; e < 8 * l; e += nt) {
        const int rr = e / l, j = e % l, i = r0 + rr;
        if (i < l) a.zsg[size_t(i) * l + j] = P[(s - 1) * slab + rr * ld + j];
      }
    }
  }
  if (nq > 1 && !grid_sync(a.scal, flag)) return kStepTimeout;

  if (mine) {
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
    double part = 0.0;
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
    if (tid == 0) a.partials[gkn + blockIdx.x] = part;
  }
  if (!grid_sync(a.scal, flag)) return kStepTimeout;
  if (tid == 0) {
    double s2 = 0.0;
    for (int b = 0; b < gkn; ++b) s2 += __ldcg(a.partials + gkn + b);
    s_norm = sqrt(s2);
  }

  if (rb) {
    if (mine) {
      // Fc := C - Dc inv(C)   (row_block_kolmogorov_nagumo_integrator.hpp:186)
      for (int e = tid; e < 8 * lp8; e += nt) {
        const int rr = e / lp8, j = e % lp8, i = r0 + rr;
        tF[rr * ld + j] = (i < l && j < l) ? __ldcg(a.dd + size_t(i) * ldd + j) : 0.0;
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
    }
    const bool ffu = a.ff && a.ffn;
    if ((end_barrier || ffu) && !grid_sync(a.scal, flag)) return kStepTimeout;
    if (ffu && mine) {
      // F~+ := F~c Fc   (row_block_gramian_kolmogorov_nagumo_integrator.hpp:197)
      for (int e = tid; e < 8 * lp8; e += nt) {
        const int rr = e / lp8, j = e % lp8, i = r0 + rr;
        tF[rr * ld + j] = (i < l && j < l) ? __ldcg(a.ff + size_t(i) * l + j) : 0.0;
      }
      __syncthreads();
      slab_mm(tF, nullptr, ld, a.out, l, l, tG, nullptr);
      for (int e = tid; e < 8 * l; e += nt) {
        const int rr = e / l, j = e % l, i = r0 + rr;
        if (i < l) a.ffn[size_t(i) * l + j] = tG[rr * ld + j];
      }
    }
  } else if (end_barrier && !grid_sync(a.scal, flag)) {
    return kStepTimeout;
  }
  __syncthreads();
  *norm = s_norm;
  *degree = d;
  return kStepDone;
}

}  // namespace
}  // namespace mb
