// FP64 DMMA GEMM (see dgemm.cuh).
//
// Tiling: a CTA computes a BM x BN tile of C; its warps own WM x WN sub-tiles
// made of 8x8 DMMA fragments.  K advances in steps of BK = 16 (32 for the
// large 128x128 configuration: half the barriers per flop) through a
// STAGES-deep cp.async ring.  Shared-memory rows are padded (K-contiguous
// rows by 4 doubles, M/N-contiguous rows by 8) so every fragment load of a
// warp touches each bank pair at most twice: the minimum two wavefronts for
// 32 lanes x 8 bytes.
#include "dgemm.cuh"
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

namespace mb {
namespace {

constexpr int BK = 16;
constexpr int PAD_K = 4;
constexpr int PAD_MN = 8;

struct KArgs {
  int64_t M, N, K;
  double alpha, beta;
  const double* A; int64_t a_rs, a_cs, a_bs;
  const double* B; int64_t b_rs, b_cs, b_bs;
  double* C; int64_t c_rs, c_cs, c_bs;
  double* ws;
  int splits;
  int64_t kps;
  const int* guard_stop;   // skip the launch when *guard_stop < guard_it
  int guard_it;
  int lower;               // 1: only tiles touching the lower triangle (row >= column) are computed
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int BM_, int BN_, int WM_, int WN_, bool AK_, bool BKM_, int VEC_, int STAGES_, int BK_ = BK>
struct Cfg {
  static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_, VEC = VEC_, STAGES = STAGES_;
  static constexpr int BKT = BK_;   // k-tile depth
  static constexpr bool AK = AK_, BKM = BKM_;
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
  static constexpr int THREADS = WARPS_M * WARPS_N * 32;
  static constexpr int MT = WM / 8, NT = WN / 8;
  static constexpr int LDA = AK ? (BKT + PAD_K) : (BM + PAD_MN);
  static constexpr int LDB = BKM ? (BKT + PAD_K) : (BN + PAD_MN);
  static constexpr int A_ELEMS = AK ? BM * LDA : BKT * LDA;
  static constexpr int B_ELEMS = BKM ? BN * LDB : BKT * LDB;
  static constexpr int STAGE_ELEMS = A_ELEMS + B_ELEMS;
  static constexpr size_t SMEM = size_t(STAGES) * STAGE_ELEMS * sizeof(double);
};

// Per-thread copy plan of one operand tile.  The chunks a thread copies are
// the same for every k-tile, so their global addresses and row validity are
// computed once; each k-tile only adds k0 * (k stride) and re-checks the K end.
//   KROWS: the tile's rows run along M (or N) and K is contiguous;
//   otherwise the rows run along K and M (or N) is contiguous.
template <int ROWS_MN, bool KCONTIG, int V, int THREADS, int LD, int TK>
struct TileLoader {
  static constexpr int CPR = KCONTIG ? TK / V : ROWS_MN / V;        // chunks per smem row
  static constexpr int TOTAL = KCONTIG ? ROWS_MN * CPR : TK * CPR;
  static constexpr int PER = (TOTAL + THREADS - 1) / THREADS;
  const double* src[PER];
  int mn_valid[PER];   // KCONTIG: row in range; else valid elements along M/N (0..V)
  int kk[PER];         // k offset of the chunk inside the tile
  int dst[PER];        // element offset in the smem tile
  int64_t kstride;     // element stride of k in global memory

  __device__ __forceinline__ void init(const double* base, int64_t mn0, int64_t mn_extent, int64_t ld_mn,
                                       int64_t ld_k, int tid) {
    kstride = ld_k;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int c = tid + i * THREADS;
      if (c >= TOTAL) {   // no chunk for this slot
        src[i] = base; mn_valid[i] = 0; kk[i] = 0; dst[i] = -1;
        continue;
      }
      if (KCONTIG) {
        const int r = c / CPR, kc = (c % CPR) * V;
        const int64_t gmn = mn0 + r;
        mn_valid[i] = (gmn < mn_extent) ? 1 : 0;
        src[i] = base + (mn_valid[i] ? gmn * ld_mn : 0) + kc;
        kk[i] = kc;
        dst[i] = r * LD + kc;
      } else {
        const int kr = c / CPR, mc = (c % CPR) * V;
        const int64_t gmn = mn0 + mc;
        const int64_t v = mn_extent - gmn;
        mn_valid[i] = v <= 0 ? 0 : (v >= V ? V : int(v));
        src[i] = base + (mn_valid[i] ? gmn : 0) + kr * ld_k;
        kk[i] = kr;
        dst[i] = kr * LD + mc;
      }
    }
  }

  __device__ __forceinline__ void load(double* s, int64_t k0, int64_t kend) const {
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      if (PER * THREADS > TOTAL && dst[i] < 0) continue;
      int valid;
      if (KCONTIG) {
        const int64_t v = kend - (k0 + kk[i]);
        valid = mn_valid[i] ? (v <= 0 ? 0 : (v >= V ? V : int(v))) : 0;
      } else {
        valid = (k0 + kk[i] < kend) ? mn_valid[i] : 0;
      }
      const double* g = valid ? src[i] + (KCONTIG ? k0 : k0 * kstride) : src[i];
      if (V == 2) cp_async16(s + dst[i], g, valid * 8); else cp_async8(s + dst[i], g, valid * 8);
    }
  }
};

template <class C>
__global__ void __launch_bounds__(C::THREADS) dgemm_kernel(KArgs g) {
  extern __shared__ __align__(16) double smem[];
  if (g.guard_stop && *g.guard_stop < g.guard_it) return;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp / C::WARPS_N, wn = warp % C::WARPS_N;
  const int gq = lane >> 2, t4 = lane & 3;

  const int64_t n0 = int64_t(blockIdx.x) * C::BN;
  const int64_t m0 = int64_t(blockIdx.y) * C::BM;
  if (g.lower && n0 >= m0 + C::BM) return;        // every element of the tile has column > row
  const int bz = blockIdx.z / g.splits;
  const int split = blockIdx.z % g.splits;
  const double* A = g.A + bz * g.a_bs;
  const double* B = g.B + bz * g.b_bs;
  const int64_t kbeg = split * g.kps;
  const int64_t kend = min(g.K, kbeg + g.kps);
  constexpr int TK = C::BKT;
  const int KT = kend > kbeg ? int((kend - kbeg + TK - 1) / TK) : 0;

  double acc[C::MT][C::NT][2];
#pragma unroll
  for (int i = 0; i < C::MT; ++i)
#pragma unroll
    for (int j = 0; j < C::NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // A tile: BM rows along M (K contiguous) or BK rows along K (M contiguous);
  // B tile: BN rows along N (K contiguous) or BK rows along K (N contiguous).
  TileLoader<C::BM, C::AK, C::VEC, C::THREADS, C::LDA, TK> la;
  TileLoader<C::BN, C::BKM, C::VEC, C::THREADS, C::LDB, TK> lb;
  la.init(A, m0, g.M, C::AK ? g.a_rs : 1, C::AK ? 1 : g.a_cs, tid);
  lb.init(B, n0, g.N, C::BKM ? g.b_cs : 1, C::BKM ? 1 : g.b_rs, tid);

#pragma unroll
  for (int s = 0; s < C::STAGES - 1; ++s) {
    if (s < KT) {
      double* st = smem + s * C::STAGE_ELEMS;
      la.load(st, kbeg + int64_t(s) * TK, kend);
      lb.load(st + C::A_ELEMS, kbeg + int64_t(s) * TK, kend);
    }
    cp_commit();
  }

  for (int kt = 0; kt < KT; ++kt) {
    cp_wait<C::STAGES - 2>();
    __syncthreads();
    {
      const int nt = kt + C::STAGES - 1;
      if (nt < KT) {
        double* st = smem + (nt % C::STAGES) * C::STAGE_ELEMS;
        la.load(st, kbeg + int64_t(nt) * TK, kend);
        lb.load(st + C::A_ELEMS, kbeg + int64_t(nt) * TK, kend);
      }
      cp_commit();
    }
    const double* sA = smem + (kt % C::STAGES) * C::STAGE_ELEMS;
    const double* sB = sA + C::A_ELEMS;
#pragma unroll
    for (int kk = 0; kk < TK / 4; ++kk) {
      const int k = kk * 4 + t4;
      double af[C::MT], bf[C::NT];
#pragma unroll
      for (int i = 0; i < C::MT; ++i) {
        const int m = wm * C::WM + i * 8 + gq;
        af[i] = C::AK ? sA[m * C::LDA + k] : sA[k * C::LDA + m];
      }
#pragma unroll
      for (int j = 0; j < C::NT; ++j) {
        const int n = wn * C::WN + j * 8 + gq;
        bf[j] = C::BKM ? sB[n * C::LDB + k] : sB[k * C::LDB + n];
      }
#pragma unroll
      for (int i = 0; i < C::MT; ++i)
#pragma unroll
        for (int j = 0; j < C::NT; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_wait<0>();

  // Epilogue: direct strided stores (C) or raw partials (split-K workspace).
  double* Cb = g.C + bz * g.c_bs;
  double* W = g.ws ? g.ws + (int64_t(bz) * g.splits + split) * g.M * g.N : nullptr;
#pragma unroll
  for (int i = 0; i < C::MT; ++i) {
    const int64_t row = m0 + wm * C::WM + i * 8 + gq;
    if (row >= g.M) continue;
#pragma unroll
    for (int j = 0; j < C::NT; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t col = n0 + wn * C::WN + j * 8 + 2 * t4 + h;
        if (col >= g.N) continue;
        if (g.splits == 1) {
          double* cp = Cb + row * g.c_rs + col * g.c_cs;
          double v = g.alpha * acc[i][j][h];
          if (g.beta != 0.0) v += g.beta * *cp;
          *cp = v;
        } else {
          W[row * g.N + col] = acc[i][j][h];
        }
      }
    }
  }
}

__global__ void splitk_reduce_kernel(const double* ws, int splits, int batch, int64_t M, int64_t N, double alpha,
                                     double beta, double* C, int64_t c_rs, int64_t c_cs, int64_t c_bs,
                                     const int* guard_stop, int guard_it, int lower) {
  if (guard_stop && *guard_stop < guard_it) return;
  const int64_t MN = M * N;
  const int64_t total = MN * batch;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = idx / MN, e = idx % MN;
    const int64_t r = e / N, c = e % N;
    if (lower && c > r) continue;
    const double* w = ws + b * splits * MN + e;
    double s = 0.0;
    for (int k = 0; k < splits; ++k) s += w[k * MN];
    double* cp = C + b * c_bs + r * c_rs + c * c_cs;
    double v = alpha * s;
    if (beta != 0.0) v += beta * *cp;
    *cp = v;
  }
}

template <class C>
int launch(Context* ctx, const KArgs& g, int batch) {
  // the shared-memory opt-in is a per-device property of the function: one bit per device
  static std::atomic<uint64_t> attr_set{0};
  auto kern = dgemm_kernel<C>;
  const uint64_t bit = uint64_t(1) << (ctx->device & 63);
  if (!(attr_set.load(std::memory_order_acquire) & bit)) {
    MB_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(C::SMEM)));
    attr_set.fetch_or(bit, std::memory_order_acq_rel);
  }
  dim3 grid(unsigned(cdiv(g.N, C::BN)), unsigned(cdiv(g.M, C::BM)), unsigned(batch * g.splits));
  kern<<<grid, C::THREADS, C::SMEM, ctx->stream>>>(g);
  ctx->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

// Tile shape families, picked by the output shape.
enum Shape { S128x128 = 0, S128x64 = 1, S64x64 = 2, S128x32 = 3, S64x32 = 4, S128x128w16 = 5, S128x128k32 = 6,
             S64x128 = 7 };

template <bool AK, bool BKM, int VEC>
int dispatch_shape(Context* ctx, const KArgs& g, int batch, Shape s) {
  switch (s) {
    case S128x128: return launch<Cfg<128, 128, 64, 32, AK, BKM, VEC, 4>>(ctx, g, batch);
    case S128x128w16: return launch<Cfg<128, 128, 32, 32, AK, BKM, VEC, 4>>(ctx, g, batch);
    case S128x128k32: return launch<Cfg<128, 128, 32, 32, AK, BKM, VEC, 3, 32>>(ctx, g, batch);
    case S64x128: return launch<Cfg<64, 128, 32, 64, AK, BKM, VEC, 4>>(ctx, g, batch);
    case S128x64: return launch<Cfg<128, 64, 32, 32, AK, BKM, VEC, 4>>(ctx, g, batch);
    case S64x64: return launch<Cfg<64, 64, 32, 32, AK, BKM, VEC, 4>>(ctx, g, batch);
    case S128x32: return launch<Cfg<128, 32, 32, 16, AK, BKM, VEC, 4>>(ctx, g, batch);
    default: return launch<Cfg<64, 32, 32, 16, AK, BKM, VEC, 4>>(ctx, g, batch);
  }
}

struct Plan {
  Shape shape;
  int bm, bn;
  int splits;
  int64_t kps;
};

Plan make_plan(const Context* ctx, int64_t M, int64_t N, int64_t K, int batch, int force_splits) {
  Plan p;
  if (N <= 32) { p.shape = M <= 64 ? S64x32 : S128x32; p.bn = 32; }
  else if (N <= 64) { p.shape = M <= 64 ? S64x64 : S128x64; p.bn = 64; }
  else { p.shape = M <= 64 ? S64x64 : S128x128w16; p.bn = M <= 64 ? 64 : 128; }
  p.bm = (p.shape == S64x64 || p.shape == S64x32) ? 64 : 128;
  const int64_t tiles = cdiv(M, p.bm) * cdiv(N, p.bn) * batch;
  int splits = 1;
  const int64_t target = 2 * int64_t(ctx->num_sms);
  if (force_splits > 0) {
    splits = force_splits;
  } else if (tiles < target && K >= 8 * BK) {
    int64_t want = cdiv(target, tiles);
    int64_t maxs = K / (8 * BK);           // at least 128 of K per split
    splits = int(std::max<int64_t>(1, std::min<int64_t>({want, maxs, 128})));
  }
  int64_t kps = cdiv(cdiv(K, splits), BK) * BK;
  if (kps == 0) kps = BK;
  splits = int(std::max<int64_t>(1, cdiv(K, kps)));
  p.splits = splits;
  p.kps = kps;
  // long K per CTA: 32-deep k-tiles (half the barriers per flop)
  if (p.shape == S128x128w16 && kps >= 512) p.shape = S128x128k32;
  return p;
}

// The large-output plan for N-contiguous B (the sketch A Omega with A row- or
// column-major, the Gramian Qs' Qs): 64 x 128 tiles of four 32 x 64 warps, two CTAs per
// SM, so one CTA's barrier bubbles are filled by the other's MMAs (sketch 33.4 vs 30.9
// TFLOP/s on 16384 x 4096 x 20000; Gramian 4096 x 4096 x 100000 lower triangle 60.3 ->
// 58.0 ms).
Plan prefer_two_cta(Plan p, bool AK, bool BKM, int64_t M, int64_t N, bool lower_only) {
  (void)AK;
  (void)lower_only;
  if (!BKM && (p.shape == S128x128k32 || p.shape == S128x128w16) && M > 64 && N > 64) {
    p.shape = S64x128;
    p.bm = 64;
    p.bn = 128;
  }
  return p;
}

}  // namespace

int dgemm_heuristic_splits(const Context* c, int64_t M, int64_t N, int64_t K, int batch) {
  return (M <= 0 || N <= 0) ? 1 : make_plan(c, M, N, K, batch, 0).splits;
}

size_t dgemm_workspace_bytes(const Context* c, int64_t M, int64_t N, int64_t K, int batch) {
  if (M <= 0 || N <= 0) return 0;
  Plan p = make_plan(c, M, N, K, batch, 0);
  return p.splits > 1 ? size_t(p.splits) * batch * M * N * sizeof(double) : 0;
}

namespace {

Plan plan_for(Shape shape, int64_t M, int64_t N, int64_t K, int batch, int splits) {
  (void)batch;
  Plan p;
  p.shape = shape;
  p.bm = (shape == S64x64 || shape == S64x32 || shape == S64x128) ? 64 : 128;
  p.bn = (shape == S128x32 || shape == S64x32) ? 32 : ((shape == S128x64 || shape == S64x64) ? 64 : 128);
  (void)M; (void)N;
  int64_t kps = cdiv(cdiv(K, splits), BK) * BK;
  if (kps == 0) kps = BK;
  p.splits = int(std::max<int64_t>(1, cdiv(K, kps)));
  p.kps = kps;
  return p;
}

// Launches g with plan p (the kernel, then the split-K reduction into g.C).
int run_plan(Context* ctx, KArgs g, int batch, const Plan& p, bool AK, bool BKM, bool vec2) {
  g.splits = p.splits;
  g.kps = p.kps;
  int st;
  if (AK && BKM) st = vec2 ? dispatch_shape<true, true, 2>(ctx, g, batch, p.shape)
                           : dispatch_shape<true, true, 1>(ctx, g, batch, p.shape);
  else if (AK) st = vec2 ? dispatch_shape<true, false, 2>(ctx, g, batch, p.shape)
                         : dispatch_shape<true, false, 1>(ctx, g, batch, p.shape);
  else if (BKM) st = vec2 ? dispatch_shape<false, true, 2>(ctx, g, batch, p.shape)
                          : dispatch_shape<false, true, 1>(ctx, g, batch, p.shape);
  else st = vec2 ? dispatch_shape<false, false, 2>(ctx, g, batch, p.shape)
                 : dispatch_shape<false, false, 1>(ctx, g, batch, p.shape);
  if (st != MCNLA_B200_OK) return st;
  if (p.splits > 1) {
    const int64_t total = g.M * g.N * batch;
    const int threads = 256;
    const int blocks = int(std::min<int64_t>(cdiv(total, threads), int64_t(ctx->num_sms) * 8));
    splitk_reduce_kernel<<<blocks, threads, 0, ctx->stream>>>(g.ws, p.splits, batch, g.M, g.N, g.alpha, g.beta, g.C,
                                                             g.c_rs, g.c_cs, g.c_bs, g.guard_stop, g.guard_it,
                                                             g.lower);
    ctx->kernels_launched++;
    MB_CHECK_CUDA(cudaGetLastError());
  }
  return MCNLA_B200_OK;
}

// ---- autotuner: the first call of an iteration-loop shape (up to kTuneMaxFlops; the
// context's tune_hot) times every
// tile configuration with the split counts its workspace allows and keeps the
// fastest for the rest of the process.  Candidates run on the call's own
// operands into a scratch output with the iteration guard off, so the tuning
// neither depends on nor disturbs the state of an iteration loop.  One global
// mutex: a key is tuned once, and every later call (in any context) uses the
// same decision, so results do not depend on which context tuned it.
struct TuneKey {
  int device;
  int64_t M, N, K;
  int batch, layout, lower, max_splits;   // max_splits: what the call's workspace holds
  bool operator<(const TuneKey& o) const {
    return std::tie(device, M, N, K, batch, layout, lower, max_splits) <
           std::tie(o.device, o.M, o.N, o.K, o.batch, o.layout, o.lower, o.max_splits);
  }
};

constexpr double kTuneMaxFlops = 5e9;

std::mutex g_tune_mu;
std::map<TuneKey, Plan>& tune_cache() {
  static std::map<TuneKey, Plan> m;
  return m;
}

int tune(Context* ctx, const KArgs& g0, int batch, const Plan& heuristic, int max_splits, bool AK, bool BKM,
         bool vec2, Plan* best) {
  *best = heuristic;
  const size_t out_bytes = size_t(batch) * g0.M * g0.N * sizeof(double);
  double* scratch = nullptr;
  MB_CHECK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&scratch), out_bytes, ctx->stream));
  KArgs g = g0;
  g.C = scratch;
  g.c_rs = g0.N;
  g.c_cs = 1;
  g.c_bs = g0.M * g0.N;
  g.beta = 0.0;
  g.guard_stop = nullptr;
  g.guard_it = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int st = MCNLA_B200_OK;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) st = MCNLA_B200_ERR_CUDA;
  float best_ms = 1e30f;
  const Shape shapes[] = {S64x128, S128x128k32, S128x128w16, S128x128, S128x64, S64x64, S128x32, S64x32};
  const int split_opts[] = {1, 2, 4, 8, 16, 32};
  for (Shape sh : shapes) {
    for (int so : split_opts) {
      if (st != MCNLA_B200_OK) break;
      if (so > 1 && g0.K < int64_t(so) * 4 * BK) continue;
      const Plan p = plan_for(sh, g0.M, g0.N, g0.K, batch, so);
      if (p.splits > max_splits) continue;
      float ms = 0.f;
      for (int rep = 0; rep < 2 && st == MCNLA_B200_OK; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        st = run_plan(ctx, g, batch, p, AK, BKM, vec2);
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = MCNLA_B200_ERR_CUDA;
        cudaEventElapsedTime(&ms, e0, e1);
      }
      if (st == MCNLA_B200_OK && ms < best_ms) {
        best_ms = ms;
        *best = p;
      }
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFreeAsync(scratch, ctx->stream);
  return st;
}

}  // namespace

int dgemm(Context* ctx, int64_t M, int64_t N, int64_t K, double alpha, CMat A, CMat B, double beta, DMat Cm,
          GemmBatch batch, double* ws, int force_splits, bool lower_only) {
  if (M < 0 || N < 0 || K < 0 || batch.count < 1) return MCNLA_B200_ERR_SHAPE;
  if (M == 0 || N == 0) return MCNLA_B200_OK;
  bool AK, BKM;
  if (A.cs == 1) AK = true; else if (A.rs == 1) AK = false; else return MCNLA_B200_ERR_LAYOUT;
  if (B.cs == 1) BKM = false; else if (B.rs == 1) BKM = true; else return MCNLA_B200_ERR_LAYOUT;
  const int64_t lda = AK ? A.rs : A.cs;
  const int64_t ldb = BKM ? B.cs : B.rs;
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  const bool vec2 = al16(A.p) && al16(B.p) && (lda % 2 == 0 || (AK ? M == 1 : K == 1)) &&
                    (ldb % 2 == 0 || (BKM ? N == 1 : K == 1)) && batch.a % 2 == 0 && batch.b % 2 == 0;
  Plan p = prefer_two_cta(make_plan(ctx, M, N, K, batch.count, force_splits), AK, BKM, M, N, lower_only);
  KArgs g;
  g.M = M; g.N = N; g.K = K; g.alpha = alpha; g.beta = beta;
  g.A = A.p; g.a_rs = A.rs; g.a_cs = A.cs; g.a_bs = batch.a;
  g.B = B.p; g.b_rs = B.rs; g.b_cs = B.cs; g.b_bs = batch.b;
  g.C = Cm.p; g.c_rs = Cm.rs; g.c_cs = Cm.cs; g.c_bs = batch.c;
  g.splits = p.splits; g.kps = p.kps;
  g.ws = nullptr;
  g.guard_stop = ctx->guard_stop;
  g.guard_it = ctx->guard_it;
  g.lower = lower_only ? 1 : 0;
  // split-K workspace available to this call (the planned need, or the stage's buffer)
  const bool have_ws = ws && ws == ctx->gws;
  const size_t ws_bytes = have_ws ? ctx->gws_bytes : 0;
  g.ws = have_ws ? ws : nullptr;
  if (ctx->autotune && ctx->tune_hot && force_splits == 0 && 2.0 * M * N * K * batch.count <= kTuneMaxFlops) {
    const size_t out_bytes = size_t(batch.count) * M * N * sizeof(double);
    const int max_splits = int(std::min<size_t>(32, std::max<size_t>(1, ws_bytes / out_bytes)));
    const TuneKey key{ctx->device, M, N, K, batch.count, (AK ? 1 : 0) | (BKM ? 2 : 0) | (vec2 ? 4 : 0),
                      lower_only ? 1 : 0, max_splits};
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = tune_cache().find(key);
    if (it != tune_cache().end()) {
      p = it->second;
    } else {
      Plan best;
      MB_CHECK(tune(ctx, g, batch.count, p, max_splits, AK, BKM, vec2, &best));
      tune_cache()[key] = best;
      p = best;
    }
  }
  if (p.splits > 1) {
    const size_t need = size_t(p.splits) * batch.count * M * N * sizeof(double);
    if (!have_ws || need > ws_bytes) return MCNLA_B200_ERR_WORKSPACE;
  }
  return run_plan(ctx, g, batch.count, p, AK, BKM, vec2);
}

int dgemm_rows_in_place(Context* ctx, int64_t M, int64_t N, int64_t K, CMat A, CMat B, DMat Cm, GemmBatch batch) {
  if (M < 0 || N < 0 || K < 0 || batch.count < 1) return MCNLA_B200_ERR_SHAPE;
  if (M == 0 || N == 0) return MCNLA_B200_OK;
  bool AK, BKM;
  if (A.cs == 1) AK = true; else if (A.rs == 1) AK = false; else return MCNLA_B200_ERR_LAYOUT;
  if (B.cs == 1) BKM = false; else if (B.rs == 1) BKM = true; else return MCNLA_B200_ERR_LAYOUT;
  const int64_t lda = AK ? A.rs : A.cs;
  const int64_t ldb = BKM ? B.cs : B.rs;
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  const bool vec2 = al16(A.p) && al16(B.p) && (lda % 2 == 0 || (AK ? M == 1 : K == 1)) &&
                    (ldb % 2 == 0 || (BKM ? N == 1 : K == 1)) && batch.a % 2 == 0 && batch.b % 2 == 0;
  const Plan p = prefer_two_cta(make_plan(ctx, M, N, K, batch.count, 1), AK, BKM, M, N, false);
  // one CTA per row panel: it reads all of its rows' K before its epilogue writes them
  if (p.bn < N || p.splits != 1) return MCNLA_B200_ERR_UNSUPPORTED;
  KArgs g;
  g.M = M; g.N = N; g.K = K; g.alpha = 1.0; g.beta = 0.0;
  g.A = A.p; g.a_rs = A.rs; g.a_cs = A.cs; g.a_bs = batch.a;
  g.B = B.p; g.b_rs = B.rs; g.b_cs = B.cs; g.b_bs = batch.b;
  g.C = Cm.p; g.c_rs = Cm.rs; g.c_cs = Cm.cs; g.c_bs = batch.c;
  g.splits = 1; g.kps = p.kps;
  g.ws = nullptr;
  g.guard_stop = ctx->guard_stop;
  g.guard_it = ctx->guard_it;
  g.lower = 0;
  return run_plan(ctx, g, batch.count, p, AK, BKM, vec2);
}

}  // namespace mb
