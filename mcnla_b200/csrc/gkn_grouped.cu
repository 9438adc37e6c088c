// Grouped row-block Gramian Kolmogorov-Nagumo integrator: the iterations of
// many independent problems of uneven sizes in one persistent launch over a
// device work queue (row_block_gramian_kolmogorov_nagumo_integrator.hpp:137-214
// for each problem): the batch's throughput path.  A single solve instead
// spreads one problem over the whole GPU (gkn_persistent.cu) for latency.
//
// The launch is a grid of thread-block clusters.  Each cluster takes the next
// problem from the queue (one atomic add on a device counter; the host orders
// the problems by cost, largest first), runs that problem's iterations with
// hardware cluster barriers between the phases, until it converges, reaches
// maxit or meets an iteration whose KN step the power series declines, and
// then takes the next problem.  Per iteration:
//   P1  Bgc := 1/N Bs Bc                                              (:152)
//   P2  [Dc | Dgc] := 1/N Bc' [Bc | Bgc]                              (:155-158)
//   P3  the KN step by power series: Z, C, inv(C), Fc, F~+ := F~c Fc  (:164-214)
//   P4  E~+ := [E~c Bc] [Fc; inv(C)/N],  B+ := [Bc Bgc] [Fc; inv(C)]  (:194-204)
// The products are cut into units (a block of at most 64 output rows by 128
// columns over a range of K) that one CTA computes alone: operands staged
// through shared memory 32 K-steps at a time, 16 x 16 warp tiles on the FP64
// MMA, every element summed over K in ascending order.  P2's long K (= N l) is
// cut into fixed slices of 256 whose partial sums are added in order
// afterwards.  The KN step walks its 8-row blocks, block b on the cluster's
// CTA b mod (cluster size).  No element's arithmetic depends on the cluster
// size or on which CTA computes it, so a problem gives the same bits in any
// batch (and agrees with the single solve's differently ordered sums to
// rounding).  A declined iteration (usually the first) is recorded in
// the problem's resume field; the host runs it on the launch-per-product path
// with the matrix-function / eigendecomposition step and queues the problem
// again from the next iteration.  The only waits are cluster barriers among
// CTAs the hardware schedules together.
#include "kn_series.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

namespace cg = cooperative_groups;

namespace mb {
namespace {

constexpr int kGThreads = 256;
constexpr int kUnitK = 32;              // K steps per shared-memory stage
constexpr int kUnitMaxRows = 64;
constexpr int kUnitMaxCols = 128;
constexpr int kLdA = kUnitK + 4;        // A stage: row r at r * kLdA (conflict-free fragment reads)
constexpr int kLdB = kUnitMaxCols + 8;  // B stage: k-row at k * kLdB
constexpr int kStageDoubles = kUnitMaxRows * (kLdA + 1) + kUnitK * kLdB;
constexpr int kDdSlice = 256;           // K slice of the [Dc | Dgc] product

__host__ __device__ constexpr size_t unit_smem_doubles() { return 2 * size_t(kStageDoubles); }

__device__ __forceinline__ void cluster_sync(const cg::cluster_group& cl) { cl.sync(); }

// out(r, c) := sum_{k in [k0, k1)} A(r0 + r, k) B(k, c0 + c) for r < R, c < Cn
// (R <= 64, Cn <= 128), written through fo(r0 + r, c0 + c, value).  A(i, k) at
// A[i * ars + k * acs], B(k, j) at B[k * brs + j * bcs] (global memory, read
// through L2: other CTAs of the cluster may have written them).  sm:
// unit_smem_doubles().  Begins and ends with a block barrier.  Every element is
// one chain of MMA steps over k in ascending order, whatever R, Cn and the CTA.
template <class FO>
__device__ void gemm_unit(const double* A, int64_t ars, int64_t acs, const double* B, int64_t brs, int64_t bcs,
                          int r0, int R, int c0, int Cn, int k0, int k1, double* sm, FO fo) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  // 2 x 4 warps of 32 x 32 (4 x 4 MMA tiles of 8 x 8) over the unit's at most 64 x 128 outputs.
  // The stages hold the 32-aligned extents Rp x 32 and 32 x Cp, zeros past R / Cn.
  const int Rp = (R + 31) & ~31, Cp = (Cn + 31) & ~31;
  const int wr = (warp >> 2) * 32, wc = (warp & 3) * 32;
  const bool active = wr < Rp && wc < Cp;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nA = Rp * kUnitK, nB = kUnitK * Cp;
  const bool a_k_contig = acs == 1;
  // A staged k-contiguous: row r at r * ldA.  With A's rows contiguous in memory instead, threads
  // walk r fastest (coalesced reads) and an odd stride keeps their stores off each other's banks.
  const int ldA = a_k_contig ? kLdA : kLdA + 1;
  constexpr int kAPer = kUnitMaxRows * kUnitK / kGThreads;    // 8
  constexpr int kBPer = kUnitK * kUnitMaxCols / kGThreads;    // 16
  double reg[kAPer + kBPer];
  // chunk [kc, kc + 32) of A and B into registers (zeros outside the operands)
  auto fetch = [&](int kc) {
#pragma unroll
    for (int q = 0; q < kAPer; ++q) {
      const int e = tid + q * kGThreads;
      if (e < nA) {
        int r, k;
        if (a_k_contig) { r = e / kUnitK; k = e % kUnitK; } else { k = e / Rp; r = e % Rp; }
        const int kk = kc + k;
        reg[q] = (kk < k1 && r < R) ? __ldcg(A + int64_t(r0 + r) * ars + int64_t(kk) * acs) : 0.0;
      }
    }
#pragma unroll
    for (int q = 0; q < kBPer; ++q) {
      const int e = tid + q * kGThreads;
      if (e < nB) {
        const int k = e / Cp, cc = e % Cp, kk = kc + k;
        reg[kAPer + q] = (kk < k1 && cc < Cn) ? __ldcg(B + int64_t(kk) * brs + int64_t(c0 + cc) * bcs) : 0.0;
      }
    }
  };
  auto stash = [&](double* st) {
    double* As = st;
    double* Bs = st + kUnitMaxRows * (kLdA + 1);
#pragma unroll
    for (int q = 0; q < kAPer; ++q) {
      const int e = tid + q * kGThreads;
      if (e < nA) {
        int r, k;
        if (a_k_contig) { r = e / kUnitK; k = e % kUnitK; } else { k = e / Rp; r = e % Rp; }
        As[r * ldA + k] = reg[q];
      }
    }
#pragma unroll
    for (int q = 0; q < kBPer; ++q) {
      const int e = tid + q * kGThreads;
      if (e < nB) Bs[(e / Cp) * kLdB + e % Cp] = reg[kAPer + q];
    }
  };
  __syncthreads();
  const int nchunks = (k1 - k0 + kUnitK - 1) / kUnitK;
  if (nchunks > 0) {
    fetch(k0);
    stash(sm);
  }
  __syncthreads();
  for (int ch = 0; ch < nchunks; ++ch) {
    const double* st = sm + (ch & 1) * kStageDoubles;
    if (ch + 1 < nchunks) fetch(k0 + (ch + 1) * kUnitK);
    const double* As = st;
    const double* Bs = st + kUnitMaxRows * (kLdA + 1);
    if (active) {
#pragma unroll
      for (int ks = 0; ks < kUnitK; ks += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[(wr + 8 * i + g) * ldA + ks + t4];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[(ks + t4) * kLdB + wc + 8 * j + g];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
    }
    if (ch + 1 < nchunks) {
      // the other stage was last read in chunk ch - 1, which every warp finished
      // before the barrier at the end of that chunk
      stash(sm + ((ch + 1) & 1) * kStageDoubles);
    }
    __syncthreads();
  }
  if (active) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wr + 8 * i + g, cc = wc + 8 * j + 2 * t4 + h;
          if (r < R && cc < Cn) fo(r0 + r, c0 + cc, acc[i][j][h]);
        }
  }
  __syncthreads();
}

// The KN step of kn_series_step with its 8-row blocks spread over the
// cluster: block b on CTA b mod ncta, one block after another.  Between the
// step's phases only global memory carries state (Z, Z^s, the partial sums,
// inv(C), Fc and C in cbuf), so each block's shared-memory slabs are rebuilt
// from it, starting from zeroed slabs like a CTA of the cooperative step.
__device__ int kn_series_step_cluster(const SeriesArgs& a, double* sm, double* cbuf, const cg::cluster_group& cl,
                                      int rank, int ncta, double* norm, int* degree) {
  __shared__ int s_d, s_s;
  __shared__ double s_norm;
  const int l = a.l, tid = threadIdx.x, nt = blockDim.x;
  const int gkn = (l + 7) >> 3;
  const int lp8 = (l + 7) & ~7, ld = lp8 + 4;
  const int slab = 8 * ld;
  double* P = sm;
  const int smax = a.smax;
  double* accF0 = P + smax * slab;
  double* accG0 = accF0 + slab;
  double* tF0 = accG0 + slab;
  double* tG0 = tF0 + slab;
  double* red = tG0 + slab;
  const double* coefF = c_series.f;
  const double* coefG = c_series.g;
  const int ldd = 2 * l;
  const bool rb = a.dd != nullptr;
  auto zero_slabs = [&]() {
    for (int e = tid; e < (smax + 4) * slab; e += nt) sm[e] = 0.0;
    __syncthreads();
  };
  auto load_dc = [&](int r0, double* tF) {
    for (int e = tid; e < 8 * lp8; e += nt) {
      const int rr = e / lp8, j = e % lp8, i = r0 + rr;
      tF[rr * ld + j] = (i < l && j < l) ? __ldcg(a.dd + size_t(i) * ldd + j) : 0.0;
    }
    __syncthreads();
  };
  auto load_z = [&](int r0, double* dst) {
    for (int e = tid; e < 8 * l; e += nt) {
      const int rr = e / l, j = e % l, i = r0 + rr;
      if (i < l) dst[rr * ld + j] = __ldcg(a.zg + size_t(i) * l + j);
    }
    __syncthreads();
  };

  // ---- phase 1: Z rows, ||Z||_F^2 and row-sum partials per block
  for (int b = rank; b < gkn; b += ncta) {
    const int r0 = 8 * b;
    zero_slabs();
    double* tF = tF0;
    double* tG = tG0;
    if (rb) {
      load_dc(r0, tF);
      slab_mm<true>(tF, nullptr, ld, a.dd, ldd, l, tG, nullptr);
    }
    double part = 0.0;
    for (int e = tid; e < 8 * l; e += nt) {
      const int rr = e / l, j = e % l, i = r0 + rr;
      if (i >= l) continue;
      double v;
      if (!rb) v = __ldcg(a.z_in + size_t(min(i, j)) * l + max(i, j));
      else v = __ldcg(a.dd + size_t(i) * ldd + l + j) - tG[rr * ld + j];
      P[rr * ld + j] = v;
      a.zg[size_t(i) * l + j] = v;
      part += v * v;
    }
    part = block_sum(part, red);
    if (tid == 0) a.partials[b] = part;
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
      a.partials[2 * gkn + b] = mx;
    }
    __syncthreads();
  }
  cluster_sync(cl);

  // ---- degree (the arithmetic of kn_series_step, the same in every CTA)
  if (tid == 0) {
    double s2 = 0.0, zi = 0.0;
    for (int b = 0; b < gkn; ++b) {
      s2 += __ldcg(a.partials + b);
      zi = fmax(zi, __ldcg(a.partials + 2 * gkn + b));
    }
    const double z = fmin(sqrt(s2), zi);
    int d = -1;
    if (4.0 * z <= kSerMaxRho) {
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
  if (d < 0) return kStepDeclined;                  // the same decision in every CTA
  const int s = s_s;
  const int nq = (d + s) / s;
  double* cinv = a.out + size_t(l) * l;
  const bool zs_smem = l <= kSerZsMax;
  double* zs = red + 32;
  if (zs_smem) {
    for (int e = tid; e < l * l; e += nt) zs[(e / l) * ld + (e % l)] = __ldcg(a.zg + e);
    __syncthreads();
  }
  auto mm_z = [&](const double* A1, const double* A2, double* C1, double* C2) {
    if (zs_smem) slab_mm<false, true>(A1, A2, ld, zs, ld, l, C1, C2);
    else slab_mm(A1, A2, ld, a.zg, l, l, C1, C2);
  };
  auto reduce_norm = [&]() {
    if (tid == 0) {
      double s2 = 0.0;
      for (int b = 0; b < gkn; ++b) s2 += __ldcg(a.partials + gkn + b);
      s_norm = sqrt(s2);
    }
    __syncthreads();
  };
  // F~+ := F~c Fc for rows [r0, r0 + 8)   (row_block_gramian_kolmogorov_nagumo_integrator.hpp:197)
  auto ff_rows = [&](int r0) {
    double* tF = tF0;
    double* tG = tG0;
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
    __syncthreads();
  };

  if (d <= kSerDirectMax) {
    // ---- plain powers, block by block (no exchange inside the branch)
    for (int b = rank; b < gkn; b += ncta) {
      const int r0 = 8 * b;
      zero_slabs();
      double* accF = accF0;
      double* accG = accG0;
      double* tF = tF0;
      double* Pa = P;
      double* Pb = P + 1 * slab;
      double* Wa = P + 2 * slab;
      double* Wb = P + 3 * slab;
      double* DW = P + 4 * slab;
      load_z(r0, Pa);
      if (rb) load_dc(r0, tF);
      for (int e = tid; e < 8 * lp8; e += nt) {
        const int rr = e / lp8, j = e % lp8, i = r0 + rr;
        const int o = rr * ld + j;
        const double id = (i == j && i < l) ? 1.0 : 0.0;
        accF[o] = coefF[0] * id + coefF[1] * Pa[o];
        accG[o] = coefG[0] * id + coefG[1] * Pa[o];
        if (rb) DW[o] = coefG[0] * tF[o];
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
          const double fc = c - DW[o];
          a.out[size_t(i) * l + j] = fc;
          if (a.outn) {
            a.outn[size_t(i) * l + j] = fc;
            a.outn[size_t(l) * l + size_t(i) * l + j] = ci * a.inv_n;
          }
        }
      }
      part = block_sum(part, red);
      if (tid == 0) a.partials[gkn + b] = part;
      __syncthreads();
    }
    cluster_sync(cl);
    reduce_norm();
    if (rb && a.ff && a.ffn)
      for (int b = rank; b < gkn; b += ncta) ff_rows(8 * b);
    cluster_sync(cl);
    *norm = s_norm;
    *degree = d;
    return kStepDone;
  }

  // ---- Paterson-Stockmeyer: rows of Z^2 .. Z^top per block (Z^s rows to zsg)
  auto powers = [&](int r0, int top) {
    zero_slabs();
    load_z(r0, P);
    for (int j = 2; j <= top; ++j) mm_z(P + (j - 2) * slab, nullptr, P + (j - 1) * slab, nullptr);
  };
  if (nq > 1) {
    for (int b = rank; b < gkn; b += ncta) {
      const int r0 = 8 * b;
      powers(r0, s);
      for (int e = tid; e < 8 * l; e += nt) {
        const int rr = e / l, j = e % l, i = r0 + rr;
        if (i < l) a.zsg[size_t(i) * l + j] = P[(s - 1) * slab + rr * ld + j];
      }
      __syncthreads();
    }
    cluster_sync(cl);
  }
  // ---- Horner in Z^s per block; C rows to cbuf (the Fc pass below reads them back)
  for (int b = rank; b < gkn; b += ncta) {
    const int r0 = 8 * b;
    powers(r0, s - 1);
    double* accF = accF0;
    double* accG = accG0;
    double* tF = tF0;
    double* tG = tG0;
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
    double part = 0.0;
    for (int e = tid; e < 8 * l; e += nt) {
      const int rr = e / l, j = e % l, i = r0 + rr;
      if (i >= l) continue;
      const int o = rr * ld + j;
      const double c = accF[o];
      const double dlt = c - (i == j ? 1.0 : 0.0);
      part += dlt * dlt;
      cinv[size_t(i) * l + j] = accG[o];
      if (!rb) a.out[size_t(i) * l + j] = c;
      else cbuf[size_t(i) * l + j] = c;
    }
    part = block_sum(part, red);
    if (tid == 0) a.partials[gkn + b] = part;
    __syncthreads();
  }
  cluster_sync(cl);
  reduce_norm();
  if (rb) {
    // Fc := C - Dc inv(C)   (row_block_kolmogorov_nagumo_integrator.hpp:186)
    for (int b = rank; b < gkn; b += ncta) {
      const int r0 = 8 * b;
      double* tF = tF0;
      double* tG = tG0;
      load_dc(r0, tF);
      slab_mm(tF, nullptr, ld, cinv, l, l, tG, nullptr);
      for (int e = tid; e < 8 * l; e += nt) {
        const int rr = e / l, j = e % l, i = r0 + rr;
        if (i >= l) continue;
        const int o = rr * ld + j;
        const double fc = __ldcg(cbuf + size_t(i) * l + j) - tG[o];
        a.out[size_t(i) * l + j] = fc;
        if (a.outn) {
          a.outn[size_t(i) * l + j] = fc;
          a.outn[size_t(l) * l + size_t(i) * l + j] = __ldcg(cinv + size_t(i) * l + j) * a.inv_n;
        }
      }
      __syncthreads();
    }
    if (a.ff && a.ffn) {
      cluster_sync(cl);
      for (int b = rank; b < gkn; b += ncta) ff_rows(8 * b);
    }
  }
  cluster_sync(cl);
  *norm = s_norm;
  *degree = d;
  return kStepDone;
}

__global__ void __launch_bounds__(kGThreads, 1) k_gkn_grouped(GknJob* jobs, int njobs, int* next) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_job;
  const cg::cluster_group cl = cg::this_cluster();
  const int rank = int(cl.block_rank()), ncta = int(cl.num_blocks());
  const int tid = threadIdx.x;
  while (true) {
    if (rank == 0 && tid == 0) s_job = atomicAdd(next, 1);
    cluster_sync(cl);
    const int j = *cl.map_shared_rank(&s_job, 0);
    cluster_sync(cl);            // every CTA has read the job before rank 0 may fetch the next
    if (j >= njobs) return;      // the same j in every CTA of the cluster
    GknJob& a = jobs[j];
    long long t_start = 0;
    if (tid == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
    const int l = a.l, L = a.L, l3 = 3 * l, l2 = 2 * l;
    const double inv_n = a.inv_n;
    int stop = INT_MAX, resume = -1, degree = 0;
    double norm = 0.0;
    long long ph[4] = {0, 0, 0, 0};
    auto stamp = [&](int i, long long& t) {   // rank 0 accumulates the phases' wall time
      if (rank == 0 && tid == 0) {
        long long now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        if (i >= 0) ph[i] += now - t;
        t = now;
      }
    };
    long long tph = 0;
    stamp(-1, tph);
    for (int it = a.it0; it < a.maxit; ++it) {
      const int cur = it & 1;
      double* E = cur ? a.eb1 : a.eb0;                   // [E~c | Bc | Bgc]
      double* En = cur ? a.eb0 : a.eb1;
      // P1: Bgc := 1/N Bs Bc   (row panels x column panels of at most 128)
      {
        const int R = kUnitMaxRows, rp = (L + R - 1) / R, cp = (l + kUnitMaxCols - 1) / kUnitMaxCols;
        const int cw = (l + cp - 1) / cp;
        for (int u = rank; u < rp * cp; u += ncta) {
          const int r0 = (u / cp) * R, c0 = (u % cp) * cw;
          gemm_unit(a.bs, L, 1, E + l, l3, 1, r0, min(R, L - r0), c0, min(cw, l - c0), 0, L, sm,
                    [&](int i, int jj, double v) { E[int64_t(i) * l3 + 2 * l + jj] = inv_n * v; });
        }
      }
      cluster_sync(cl);
      stamp(0, tph);
      // P2: [Dc | Dgc] := 1/N Bc' [Bc | Bgc]: partial sums over K slices of 256 into
      // the slices buffer, then the slices added in order
      {
        const int ns = (L + kDdSlice - 1) / kDdSlice;
        const int rp = (l + kUnitMaxRows - 1) / kUnitMaxRows, cp = (l2 + kUnitMaxCols - 1) / kUnitMaxCols;
        const int rw = (l + rp - 1) / rp, cw = (l2 + cp - 1) / cp;
        double* part = a.ddp;
        for (int u = rank; u < ns * rp * cp; u += ncta) {
          const int sl = u / (rp * cp), rc = u % (rp * cp);
          const int r0 = (rc / cp) * rw, c0 = (rc % cp) * cw;
          double* dst = part + size_t(sl) * l * l2;
          gemm_unit(E + l, 1, l3, E + l, l3, 1, r0, min(rw, l - r0), c0, min(cw, l2 - c0), sl * kDdSlice,
                    min(L, (sl + 1) * kDdSlice), sm, [&](int i, int jj, double v) { dst[int64_t(i) * l2 + jj] = v; });
        }
        cluster_sync(cl);
        for (int e = rank * kGThreads + tid; e < l * l2; e += ncta * kGThreads) {
          double v = 0.0;
          for (int sl = 0; sl < ns; ++sl) v += __ldcg(part + size_t(sl) * l * l2 + e);
          a.dd[e] = inv_n * v;
        }
      }
      cluster_sync(cl);
      stamp(1, tph);
      // P3: KN step (C, inv(C), Fc, F~+) by power series
      SeriesArgs s;
      s.l = l;
      s.z_in = nullptr;
      s.dd = a.dd;
      s.inv_n = inv_n;
      s.out = a.fc;
      s.outn = a.fcn;
      s.ff = cur ? a.ff1 : a.ff0;
      s.ffn = cur ? a.ff0 : a.ff1;
      s.zg = a.work;
      s.zsg = a.work + size_t(l) * l;
      s.partials = a.work + 2 * size_t(l) * l;
      s.scal = nullptr;
      s.smax = a.smax;
      const int step = kn_series_step_cluster(s, sm, a.cbuf, cl, rank, ncta, &norm, &degree);
      stamp(2, tph);
      if (step == kStepDeclined) {
        resume = it;
        break;
      }
      // P4: E~+ := [E~c Bc] [Fc; inv(C)/N];  B+ := [Bc Bgc] [Fc; inv(C)]
      {
        const int R = kUnitMaxRows, rp = (L + R - 1) / R, cp = (l + kUnitMaxCols - 1) / kUnitMaxCols;
        const int cw = (l + cp - 1) / cp;
        for (int u = rank; u < 2 * rp * cp; u += ncta) {
          const int which = u / (rp * cp), rc = u % (rp * cp);
          const int r0 = (rc / cp) * R, c0 = (rc % cp) * cw;
          const double* A = E + which * l;
          const double* B = which ? a.fc : a.fcn;
          double* dst = En + which * l;
          gemm_unit(A, l3, 1, B, l, 1, r0, min(R, L - r0), c0, min(cw, l - c0), 0, l2, sm,
                    [&](int i, int jj, double v) { dst[int64_t(i) * l3 + jj] = v; });
        }
      }
      cluster_sync(cl);
      stamp(3, tph);
      if (!(norm >= a.tol)) {                            // the same norm in every CTA
        stop = it;
        break;
      }
    }
    if (rank == 0 && tid == 0) {
      long long t_end;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_end));
      a.stop_it = stop;
      a.resume_it = resume;
      a.norm = norm;
      a.degree = degree;
      a.ns = t_end - t_start;
      for (int i = 0; i < 4; ++i) a.phase_ns[i] = ph[i];
    }
    cluster_sync(cl);
  }
}

}  // namespace

size_t gkn_grouped_smem(const Context* c, int l) {
  const int smax = gkn_grouped_smax(c, l);
  if (smax == 0) return 0;
  return std::max<size_t>(kn_series_smem_doubles(l, smax), unit_smem_doubles()) * sizeof(double);
}

int gkn_grouped_smax(const Context* c, int l) { return kn_series_smax(l, c->smem_optin, 0); }

size_t gkn_grouped_ddp_doubles(int l, int64_t L) { return size_t((L + kDdSlice - 1) / kDdSlice) * l * 2 * l; }

bool gkn_grouped_fits(const Context* c, int l, int64_t L) {
  return l >= 1 && l <= MCNLA_B200_MAX_DIM_SKETCH && L <= kGknGroupedMaxL && gkn_grouped_smax(c, l) > 0;
}

int launch_gkn_grouped(Context* c, GknJob* jobs_dev, int njobs, int* next_dev, size_t smem, int cluster) {
  if (njobs <= 0) return MCNLA_B200_OK;
  if (cluster < 1 || cluster > 16) return MCNLA_B200_ERR_ARG;
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_gkn_grouped), smem));
  if (cluster > 8) MB_CHECK_CUDA(cudaFuncSetAttribute(k_gkn_grouped, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(kGThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = unsigned(cluster);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // clusters the device can hold at once (at least one), at most one per problem
  cfg.gridDim = dim3(unsigned(cluster));
  int active = 0;
  if (cudaOccupancyMaxActiveClusters(&active, k_gkn_grouped, &cfg) != cudaSuccess || active < 1) {
    (void)cudaGetLastError();
    active = std::max(1, c->num_sms / cluster);
  }
  const int clusters = std::max(1, std::min(njobs, active));
  cfg.gridDim = dim3(unsigned(clusters * cluster));
  MB_CHECK_CUDA(cudaMemsetAsync(next_dev, 0, sizeof(int), c->stream));
  MB_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_gkn_grouped, jobs_dev, njobs, next_dev));
  c->kernels_launched++;
  return MCNLA_B200_OK;
}

}  // namespace mb
