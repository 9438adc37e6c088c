// Persistent row-block Gramian Kolmogorov-Nagumo integrator
// (row_block_gramian_kolmogorov_nagumo_integrator.hpp:137-214): one
// cooperative kernel runs the iterations back to back with every operand in
// L2 / HBM and no host round trip, instead of five to seven launches per
// iteration.
//
// State (the same buffers and parity as the launch-per-product loop):
// EB[i & 1] = [E~c | Bc | Bgc] (L x 3l), FF[i & 1] = F~c (l x l); Bs (L x L).
// Iteration i (the products over 16 x 16 tiles spread over the grid, each
// element the same fold of K chunks whatever the grid size; grid_tiles):
//   P1  Bgc := 1/N Bs Bc                                              (:152)
//   --- grid barrier
//   P2  [Dc | Dgc] := 1/N Bc' [Bc | Bgc]                              (:155-158)
//   --- grid barrier
//   P3  the KN step by power series on CTAs [0, ceil(l/8)) (kn_series.cuh):
//       Z, C, inv(C), Fc, F~+ := F~c Fc, ||C - I||_F                  (:164-214)
//   P4  E~+ := [E~c Bc] [Fc; inv(C)/N],  B+ := [Bc Bgc] [Fc; inv(C)]  (:194-204)
//   --- grid barrier; stop when !(||C - I||_F >= tol) (after P4, like the
//       reference's loop condition) or at maxit.
// When the series declines an iteration (4 ||Z||_F > 1/2, usually the first
// one or two), the kernel records it in scal->resume_it and returns; the host
// runs that iteration on the launch-per-product path with the
// matrix-function / eigendecomposition step and starts the kernel again at
// the next one.
#include "kn_series.cuh"

namespace mb {
namespace {

constexpr int kGknThreads = 256;
constexpr int kGknWarps = kGknThreads / 32;
static_assert(kGknThreads == 256, "grid_tiles reduces a 16 x 16 tile with one thread per element");
constexpr int64_t kGknMaxL = 1536;

struct GknArgs {
  int l, L;
  double inv_n, tol;
  int it0, maxit;
  const double* bs;         // L x L
  double* eb0;              // L x 3l: [E~ | Bc | Bgc], even iterations
  double* eb1;              //   odd iterations
  double* ff0;              // l x l
  double* ff1;
  double* dd;               // l x 2l
  double* fc;               // [Fc; inv(C)]     (2l x l)
  double* fcn;              // [Fc; inv(C)/N]
  double* work;             // series scratch (kn_series_work_doubles(l))
  DevScalars* scal;
  int smax;                 // power slabs of the series step
};

// Sum over k in [kb, ke) of one 16 x 16 tile with the m8n8k4 FP64 MMA: 2 x 2
// register blocking (four DMMAs per pair of A and B fragment loads), the loads
// of kU consecutive k-steps issued before their MMAs, two chains (even and odd
// k-steps) added at the end; s[ib][jb][h] := the lane's elements.
template <class FA, class FB>
__device__ __forceinline__ void tile_chunk(FA fa, FB fb, int i0, int j0, bool iv0, bool iv1, bool jv0, bool jv1, int kb,
                                           int ke, double (&s)[2][2][2]) {
  const int t4 = threadIdx.x & 3;
  const int i1 = i0 + 8, j1 = j0 + 8;
  double c[2][2][2], e[2][2][2];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    (&c[0][0][0])[q] = 0.0;
    (&e[0][0][0])[q] = 0.0;
  }
  for (int k = kb; k < ke; k += 4 * kU) {
    double a0[kU], a1[kU], b0[kU], b1[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int kk = k + 4 * u + t4;
      const bool kv = kk < ke;
      a0[u] = kv && iv0 ? fa(i0, kk) : 0.0;
      a1[u] = kv && iv1 ? fa(i1, kk) : 0.0;
      b0[u] = kv && jv0 ? fb(kk, j0) : 0.0;
      b1[u] = kv && jv1 ? fb(kk, j1) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kU; u += 2) {
      dmma(c[0][0][0], c[0][0][1], a0[u], b0[u]);
      dmma(c[0][1][0], c[0][1][1], a0[u], b1[u]);
      dmma(c[1][0][0], c[1][0][1], a1[u], b0[u]);
      dmma(c[1][1][0], c[1][1][1], a1[u], b1[u]);
      dmma(e[0][0][0], e[0][0][1], a0[u + 1], b0[u + 1]);
      dmma(e[0][1][0], e[0][1][1], a0[u + 1], b1[u + 1]);
      dmma(e[1][0][0], e[1][0][1], a1[u + 1], b0[u + 1]);
      dmma(e[1][1][0], e[1][1][1], a1[u + 1], b1[u + 1]);
    }
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) (&s[0][0][0])[q] = (&c[0][0][0])[q] + (&e[0][0][0])[q];
}

// out(i, j) := sum_k A(i, k) B(k, j) for an M x N product over 16 x 16 tiles
// distributed round-robin over the grid.  Every element is the same fold:
// K is cut into kGknWarps chunks (a function of K alone), each chunk summed by
// tile_chunk, and the chunk sums added in chunk order starting from zero.
// Two ways to compute it, chosen per launch (the bits do not change):
//  * fewer tiles than the grid has warps: a CTA takes one tile at a time,
//    warp w sums chunk w, and the chunk sums are folded in warp order through
//    shared memory (red: kGknWarps x 256 doubles, two block barriers);
//  * otherwise a warp takes whole tiles and folds their chunks itself (no
//    shared memory, no barrier) — on a small share of the SMs (a server
//    worker's) the reduction and its barriers dominated.
// fa(i, k), fb(k, j) load operands; fo(i, j, v) stores.
template <class FA, class FB, class FO>
__device__ void grid_tiles(FA fa, FB fb, FO fo, int M, int N, int K, double* red) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int mt = (M + 15) >> 4, ntl = (N + 15) >> 4, ntiles = mt * ntl;
  const int chunk = ((K + kGknWarps - 1) / kGknWarps + 3) & ~3;
  if (ntiles >= int(gridDim.x) * kGknWarps) {
    for (int t = int(blockIdx.x) * kGknWarps + warp; t < ntiles; t += int(gridDim.x) * kGknWarps) {
      const int ti = (t / ntl) * 16, tj = (t % ntl) * 16;
      const int i0 = ti + g, j0 = tj + g;
      double acc[2][2][2];
#pragma unroll
      for (int q = 0; q < 8; ++q) (&acc[0][0][0])[q] = 0.0;
      for (int w = 0; w < kGknWarps; ++w) {
        const int kb = min(K, w * chunk), ke = min(K, kb + chunk);
        double cs[2][2][2];
        tile_chunk(fa, fb, i0, j0, i0 < M, i0 + 8 < M, j0 < N, j0 + 8 < N, kb, ke, cs);
#pragma unroll
        for (int q = 0; q < 8; ++q) (&acc[0][0][0])[q] += (&cs[0][0][0])[q];
      }
#pragma unroll
      for (int ib = 0; ib < 2; ++ib)
#pragma unroll
        for (int jb = 0; jb < 2; ++jb)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int i = ti + 8 * ib + g, j = tj + 8 * jb + 2 * t4 + h;
            if (i < M && j < N) fo(i, j, acc[ib][jb][h]);
          }
    }
    return;
  }
  const int kb = min(K, warp * chunk), ke = min(K, kb + chunk);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int ti = (t / ntl) * 16, tj = (t % ntl) * 16;
    const int i0 = ti + g, j0 = tj + g;
    double cs[2][2][2];
    tile_chunk(fa, fb, i0, j0, i0 < M, i0 + 8 < M, j0 < N, j0 + 8 < N, kb, ke, cs);
#pragma unroll
    for (int ib = 0; ib < 2; ++ib)
#pragma unroll
      for (int jb = 0; jb < 2; ++jb)
#pragma unroll
        for (int h = 0; h < 2; ++h) red[warp * 256 + (8 * ib + g) * 16 + 8 * jb + 2 * t4 + h] = cs[ib][jb][h];
    __syncthreads();
    {
      const int r = threadIdx.x >> 4, cc = threadIdx.x & 15;   // kGknThreads = 256 outputs
      double v = 0.0;
      for (int w = 0; w < kGknWarps; ++w) v += red[w * 256 + threadIdx.x];
      if (ti + r < M && tj + cc < N) fo(ti + r, tj + cc, v);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kGknThreads, 1) k_gkn_persistent(GknArgs a) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_flag;
  const int l = a.l, L = a.L, l3 = 3 * l;
  // the products' reduction space (kGknWarps x 256 doubles) aliases the series step's
  // shared memory: the step zeroes and reloads it on every call and ends on a grid barrier
  double* red = sm;
  for (int it = a.it0; it < a.maxit; ++it) {
    const int cur = it & 1;
    double* E = cur ? a.eb1 : a.eb0;                   // [E~c | Bc | Bgc]
    double* En = cur ? a.eb0 : a.eb1;
    // P1: Bgc := 1/N Bs Bc
    const double* bs = a.bs;
    const double inv_n = a.inv_n;
    grid_tiles([&](int i, int k) { return __ldg(bs + int64_t(i) * L + k); },
               [&](int k, int j) { return __ldcg(E + int64_t(k) * l3 + l + j); },
               [&](int i, int j, double v) { E[int64_t(i) * l3 + 2 * l + j] = inv_n * v; }, L, l, L, red);
    if (!grid_sync(a.scal, &s_flag)) return;
    // P2: [Dc | Dgc] := 1/N Bc' [Bc | Bgc]
    double* dd = a.dd;
    grid_tiles([&](int i, int k) { return __ldcg(E + int64_t(k) * l3 + l + i); },
               [&](int k, int j) { return __ldcg(E + int64_t(k) * l3 + l + j); },
               [&](int i, int j, double v) { dd[int64_t(i) * 2 * l + j] = inv_n * v; }, l, 2 * l, L, red);
    if (!grid_sync(a.scal, &s_flag)) return;
    // P3: KN step (C, inv(C), Fc, F~+) by power series
    SeriesArgs s;
    s.l = l;
    s.z_in = nullptr;
    s.dd = a.dd;
    s.inv_n = a.inv_n;
    s.out = a.fc;
    s.outn = a.fcn;
    s.ff = cur ? a.ff1 : a.ff0;
    s.ffn = cur ? a.ff0 : a.ff1;
    s.zg = a.work;
    s.zsg = a.work + size_t(l) * l;
    s.partials = a.work + 2 * size_t(l) * l;
    s.scal = a.scal;
    s.smax = a.smax;
    double norm = 0.0;
    int degree = 0;
    const int r = kn_series_step(s, sm, &s_flag, true, &norm, &degree);
    if (r == kStepTimeout) return;
    if (r == kStepDeclined) {
      if (blockIdx.x == 0 && threadIdx.x == 0) a.scal->resume_it = it;
      return;
    }
    // P4: E~+ := [E~c Bc] [Fc; inv(C)/N];  B+ := [Bc Bgc] [Fc; inv(C)]
    const double* fcn = a.fcn;
    const double* fc = a.fc;
    grid_tiles([&](int i, int k) { return __ldcg(E + int64_t(i) * l3 + k); },
               [&](int k, int j) { return __ldcg(fcn + int64_t(k) * l + j); },
               [&](int i, int j, double v) { En[int64_t(i) * l3 + j] = v; }, L, l, 2 * l, red);
    grid_tiles([&](int i, int k) { return __ldcg(E + int64_t(i) * l3 + l + k); },
               [&](int k, int j) { return __ldcg(fc + int64_t(k) * l + j); },
               [&](int i, int j, double v) { En[int64_t(i) * l3 + l + j] = v; }, L, l, 2 * l, red);
    const bool converged = !(norm >= a.tol);
    if (converged) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.scal->norm = norm;
        a.scal->sweeps = 1000 + degree;
        a.scal->stop_it = it;
      }
      return;
    }
    if (!grid_sync(a.scal, &s_flag)) return;
  }
}

}  // namespace

// Grid: enough CTAs for two 8 x 8 tiles of Bs Bc each, at most one per SM
// or the context's share of the SMs, and at least the ceil(l/8) CTAs of the
// KN step.
int gkn_persistent_grid(const Context* c, int l, int64_t L) {
  const int64_t tiles = ((L + 7) / 8) * ((l + 7) / 8);
  int64_t cap = c->num_sms;
  if (c->coop_cta_limit > 0) cap = std::min<int64_t>(cap, c->coop_cta_limit);
  return int(std::max<int64_t>(std::min<int64_t>(cap, (tiles + 1) / 2), (l + 7) / 8));
}

bool gkn_persistent_fits(const Context* c, int l, int64_t L) {
  // Bs Bc here reads its operands straight from L2; past L ~ 1536 the
  // smem-pipelined GEMM of the launch-per-product loop is faster
  if (l < 1 || l > MCNLA_B200_MAX_DIM_SKETCH || L > kGknMaxL) return false;
  return kn_series_smax(l, c->smem_optin, kGknWarps * 64) > 0 && (l + 7) / 8 <= c->num_sms;
}

int launch_gkn_persistent(Context* c, int l, int64_t L, int N, double tol, int it0, int maxit, const double* Bs,
                          double* const EB[2], double* const FF[2], double* DD, double* FC, double* FCN,
                          double* work) {
  if (!gkn_persistent_fits(c, l, L)) return MCNLA_B200_ERR_UNSUPPORTED;
  const int smax = kn_series_smax(l, c->smem_optin, kGknWarps * 64);
  const size_t smem =
      std::max<size_t>(kn_series_smem_doubles(l, smax) + kGknWarps * 64, kGknWarps * 256) * sizeof(double);
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_gkn_persistent), smem));
  GknArgs a;
  a.l = l;
  a.L = int(L);
  a.inv_n = 1.0 / N;
  a.tol = tol;
  a.it0 = it0;
  a.maxit = maxit;
  const int G = gkn_persistent_grid(c, l, L);
  a.bs = Bs;
  a.eb0 = EB[0];
  a.eb1 = EB[1];
  a.ff0 = FF[0];
  a.ff1 = FF[1];
  a.dd = DD;
  a.fc = FC;
  a.fcn = FCN;
  a.work = work;
  a.scal = c->scal;
  a.smax = smax;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(G));
  cfg.blockDim = dim3(kGknThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MB_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_gkn_persistent, a));
  c->kernels_launched++;
  return MCNLA_B200_OK;
}

}  // namespace mb
