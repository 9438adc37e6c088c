// The iSVD stages on one B200: sketch, Gramian orthogonalizer, the five
// integrators and the two former families, plus the whole-solve pipeline and
// the C ABI entry points (declared in include/mcnla_b200.h).
//
// Each stage follows its reference runImpl step for step (citations inline);
// the products run on the FP64 DMMA GEMM, the l x l work on the one-CTA
// solvers, and the reference's MPI collectives disappear because every
// sketch and every row lives on the one device.  Operands the reference keeps
// in separate matrices are packed side by side where that turns two GEMMs
// into one (e.g. [Qc | Gc] * [Fc; inv(C)] for Q+ := Qc Fc + Gc inv(C)).
#include "common.cuh"
#include "dgemm.cuh"
#include "kernels.cuh"
#include "bf16.cuh"
#include "solve.cuh"
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <mutex>
#include <thread>
#include <vector>

namespace mb {
namespace {

// Wen-Yin line-search constants (include/mcnla/isvd/integrator/row_block_wen_yin_integrator.hh:76-94).
constexpr double kTau0 = 1.0, kTauMax = 1e14, kTauMin = 1e-14, kBeta = 0.5, kSigma = 1e-4, kEta = 0.85;
constexpr int kTauMaxIter = 20;

struct Dims {
  int64_t m, n;
  int k, p, l, N;
  int64_t L;
};

int get_dims(const mcnla_b200_params* p, Dims& d) {
  if (!p) return MCNLA_B200_ERR_ARG;
  if (p->nrow <= 0 || p->ncol <= 0 || p->rank <= 0 || p->over_rank < 0 || p->num_sketch <= 0)
    return MCNLA_B200_ERR_SHAPE;
  const int64_t l = p->rank + p->over_rank;
  if (l > MCNLA_B200_MAX_DIM_SKETCH) return MCNLA_B200_ERR_UNSUPPORTED;
  if (p->num_sketch > (int64_t(1) << 24)) return MCNLA_B200_ERR_SHAPE;
  d.m = p->nrow; d.n = p->ncol;
  d.k = int(p->rank); d.p = int(p->over_rank); d.l = int(l); d.N = int(p->num_sketch);
  d.L = l * p->num_sketch;
  return MCNLA_B200_OK;
}

// Workspace planner: accumulates the sizes of the buffers a stage will carve.
struct Plan {
  size_t bytes = 0;
  void add(size_t count, size_t elem = sizeof(double)) { bytes += arena_bytes_for(count, elem); }
};

size_t gemm_ws(const Context* c, std::initializer_list<std::array<int64_t, 4>> shapes) {
  size_t w = 0;
  for (auto& s : shapes) w = std::max(w, dgemm_workspace_bytes(c, s[0], s[1], s[2], int(s[3])));
  return w;
}

// Every stage carves its buffers after one ctx_reserve(); a carve past the
// reservation is a planning bug and is reported instead of corrupting memory.
int check_arena(const Context* c) {
  return c->arena_top <= c->arena_bytes ? MCNLA_B200_OK : MCNLA_B200_ERR_WORKSPACE;
}

// Carves the split-K workspace of a stage and registers it with the context.
double* take_ws(Context* c, size_t bytes) {
  double* p = ctx_take<double>(c, bytes / 8 + 1);
  c->gws = p;
  c->gws_bytes = p ? bytes + 8 : 0;
  return p;
}

int copy2d(Context* c, double* dst, int64_t ldd, const double* src, int64_t lds, int64_t rows, int64_t cols) {
  if (rows <= 0 || cols <= 0) return MCNLA_B200_OK;
  MB_CHECK_CUDA(cudaMemcpy2DAsync(dst, ldd * sizeof(double), src, lds * sizeof(double), cols * sizeof(double), rows,
                                  cudaMemcpyDeviceToDevice, c->stream));
  return MCNLA_B200_OK;
}

// ---------------------------------------------------------------------------
// Sketcher
// ---------------------------------------------------------------------------
int run_sketch(Context* c, const Dims& d, const double* A, int layout, int64_t lda, double* omega, int exponent,
               double* Q, bool timed_generation) {
  if (layout != MCNLA_B200_ROW_MAJOR && layout != MCNLA_B200_COL_MAJOR) return MCNLA_B200_ERR_ARG;
  if (layout == MCNLA_B200_ROW_MAJOR ? lda < d.n : lda < d.m) return MCNLA_B200_ERR_SHAPE;
  if (exponent < 0) return MCNLA_B200_ERR_ARG;
  const CMat Am = layout == MCNLA_B200_ROW_MAJOR ? crow(A, lda) : ccol(A, lda);
  Plan pl;
  pl.add(gemm_ws(c, {{d.m, d.L, d.n, 1}, {d.n, d.L, d.m, 1}}) / 8 + 1);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  double* ws = take_ws(c, gemm_ws(c, {{d.m, d.L, d.n, 1}, {d.n, d.L, d.m, 1}}));
  MB_CHECK(check_arena(c));
  if (!timed_generation) { MB_CHECK(ctx_tic(c)); MB_CHECK(ctx_toc(c)); }   // "random generating" part
  // Q := A * Omega   (gaussian_projection_sketcher.hpp:96)
  MB_CHECK(dgemm(c, d.m, d.L, d.n, 1.0, Am, crow(omega, d.L), 0.0, drow(Q, d.L), GemmBatch(), ws));
  // power iterations (gaussian_projection_sketcher.hpp:97-100)
  for (int i = 0; i < exponent; ++i) {
    MB_CHECK(dgemm(c, d.n, d.L, d.m, 1.0, ctr(Am), crow(Q, d.L), 0.0, drow(omega, d.L), GemmBatch(), ws));
    MB_CHECK(dgemm(c, d.m, d.L, d.n, 1.0, Am, crow(omega, d.L), 0.0, drow(Q, d.L), GemmBatch(), ws));
  }
  MB_CHECK(ctx_toc(c));
  return MCNLA_B200_OK;
}

// ---------------------------------------------------------------------------
// Gramian orthogonalizer (gramian_orthogonalizer.hpp:62-104)
// ---------------------------------------------------------------------------
int run_orthogonalize(Context* c, const Dims& d, double* Q) {
  const int l = d.l, N = d.N;
  const int64_t m = d.m, L = d.L;
  const size_t ll = size_t(l) * l;
  const size_t wsb = gemm_ws(c, {{l, l, m, N}, {m, l, l, N}});
  Plan pl;
  pl.add(ll * N); pl.add(size_t(l) * N); pl.add(ll * N); pl.add(ll * N); pl.add(size_t(m) * L);
  pl.add(wsb / 8 + 1); pl.add(ll * N);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  double* W = ctx_take<double>(c, ll * N);
  double* S = ctx_take<double>(c, size_t(l) * N);
  double* V = ctx_take<double>(c, ll * N);
  double* T = ctx_take<double>(c, ll * N);
  double* tmp = ctx_take<double>(c, size_t(m) * L);
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  MB_CHECK(ctx_tic(c));
  // W_i := Q_i' Q_i   (:84-86)
  MB_CHECK(dgemm(c, l, l, m, 1.0, cm(Q, 1, L), cm(Q, L, 1), 0.0, drow(W, l), GemmBatch{N, l, l, int64_t(ll)}, ws));
  MB_CHECK(ctx_allreduce(c, W, int64_t(ll) * N));   // row blocks over ranks (row_block_gramian_orthogonalizer.hpp:86)
  // eig(W_i) = V_i S_i V_i', descending (gesvd<'N','O'> of an SPD matrix, :89-91)
  MB_CHECK(launch_syev(c, l, N, W, l, int64_t(ll), S, V, 1));
  // T_i := V_i diag(S_i)^(-1/2)   (:94-99)
  MB_CHECK(launch_scale_cols_rsqrt(c, l, N, V, S, T));
  // Q_i := Q_i T_i in place: each CTA reads its rows of Q_i before it writes them (the reference
  // copies Q to a temporary first, :97-101; that copy remains for the shapes where one CTA cannot
  // own whole row panels)
  const int st = dgemm_rows_in_place(c, m, l, l, crow(Q, L), crow(T, l), drow(Q, L), GemmBatch{N, l, int64_t(ll), l});
  if (st == MCNLA_B200_ERR_UNSUPPORTED) {
    MB_CHECK_CUDA(cudaMemcpyAsync(tmp, Q, size_t(m) * L * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    MB_CHECK(dgemm(c, m, l, l, 1.0, crow(tmp, L), crow(T, l), 0.0, drow(Q, L), GemmBatch{N, l, int64_t(ll), l}, ws));
  } else {
    MB_CHECK(st);
  }
  MB_CHECK(ctx_toc(c));
  return MCNLA_B200_OK;
}

// ---------------------------------------------------------------------------
// Integrators
// ---------------------------------------------------------------------------
// Kolmogorov-Nagumo iteration driver.  The reference's loop
//   for (it = 0; it < maxit && !converged; ++it) { body; converged = !(norm >= tol); }
// runs here without a host round trip per iteration: iterations are launched
// in chunks, the KN step records on the device the first iteration whose
// norm converged (scal->stop_it), and every kernel launched for a later
// iteration returns at once.  The host reads stop_it once per chunk.
// Returns the number of executed bodies (the reference's iteration()).
// Marks the products launched while it lives as iteration-loop products (the
// GEMM autotuner tunes those shapes on their first call).
struct HotLoop {
  Context* c;
  explicit HotLoop(Context* ctx) : c(ctx) { c->tune_hot = true; }
  ~HotLoop() { c->tune_hot = false; }
};

//
// CUDA graph: the bodies of one chunk depend on the iteration only through
// its parity (double buffers) and the guard index, so after the first chunk
// (launched directly: it also tunes every product shape) the next full chunk
// is captured once with guard indices relative to the chunk start, and every
// later full chunk replays that graph.  Relative indices work because the KN
// step records the converged iteration as the guard index it was given: the
// host adds the chunk start.  A capture that fails (an operation the graph
// cannot hold) is abandoned and the loop continues with direct launches.
struct LoopGraph {
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr;
  ~LoopGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (cap) cudaStreamDestroy(cap);
  }
};

template <class Body>
int capture_chunk(Context* c, int it0, int chunk, Body& body, LoopGraph& g, int64_t* kernels) {
  if (cudaStreamCreateWithFlags(&g.cap, cudaStreamNonBlocking) != cudaSuccess) return MCNLA_B200_ERR_CUDA;
  struct Swap { Context* c; cudaStream_t s; ~Swap() { c->stream = s; } } swap{c, c->stream};
  const int64_t k0 = c->kernels_launched;
  if (cudaStreamBeginCapture(g.cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return MCNLA_B200_ERR_CUDA;
  c->stream = g.cap;
  int st = MCNLA_B200_OK;
  for (int r = 0; r < chunk && st == MCNLA_B200_OK; ++r) {
    c->guard_it = r;
    st = body(it0 + r);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(g.cap, &graph);
  c->stream = swap.s;
  *kernels = c->kernels_launched - k0;
  c->kernels_launched = k0;            // nothing ran yet: replays count themselves
  if (st == MCNLA_B200_OK && (ec != cudaSuccess || !graph)) st = MCNLA_B200_ERR_CUDA;
  if (st == MCNLA_B200_OK && cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) {
    g.exec = nullptr;
    st = MCNLA_B200_ERR_CUDA;
  }
  if (graph) cudaGraphDestroy(graph);
  if (st != MCNLA_B200_OK) cudaGetLastError();   // capture errors are not sticky: clear and go on eagerly
  return st;
}

template <class Body>
int kn_loop(Context* c, int maxit, Body body, int* iters) {
  MB_CHECK_CUDA(cudaMemsetAsync(&c->scal->stop_it, 0x7f, sizeof(int), c->stream));   // "not yet"
  struct Reset { Context* c; ~Reset() { c->guard_stop = nullptr; c->guard_it = 0; } } reset{c};
  HotLoop hot(c);
  c->guard_stop = &c->scal->stop_it;
  const int chunk = 8;   // even: every chunk starts on the same buffer parity
  int launched = 0, done = -1;
  LoopGraph graph;
  bool use_graph = c->graph_loop && !ctx_distributed(c);   // a caller's all-reduce may not be capturable
  int64_t graph_kernels = 0;
  while (launched < maxit) {
    const int end = std::min(maxit, launched + chunk);
    // graph replays for full chunks after the first, when at least two remain
    if (use_graph && launched > 0 && end - launched == chunk && !graph.exec && maxit - launched >= 2 * chunk) {
      if (capture_chunk(c, launched, chunk, body, graph, &graph_kernels) != MCNLA_B200_OK) use_graph = false;
    }
    if (use_graph && graph.exec && end - launched == chunk) {
      MB_CHECK_CUDA(cudaGraphLaunch(graph.exec, c->stream));
      c->kernels_launched += graph_kernels;
      c->graph_replays++;
    } else {
      for (int it = launched; it < end; ++it) {
        c->guard_it = it;
        MB_CHECK(body(it));
      }
    }
    const bool relative = use_graph && graph.exec && end - launched == chunk;
    const int start = launched;
    launched = end;
    MB_CHECK(ctx_sync_scalars(c));
    if (c->scal_host->status) return c->scal_host->status;
    const int stop = c->scal_host->stop_it;
    if (relative) {
      if (stop < chunk) { done = start + stop + 1; break; }
    } else if (stop < launched) {
      done = stop + 1;
      break;
    }
  }
  *iters = done < 0 ? launched : done;
  return MCNLA_B200_OK;
}

// KolmogorovNagumoIntegrator (kolmogorov_nagumo_integrator.hpp:76-185)
int run_kn(Context* c, const Dims& d, const double* Qs, int maxit, double tol, double* Qbar, int* iters) {
  const int l = d.l;
  const int64_t m = d.m, L = d.L;
  const double inv_n = 1.0 / d.N;
  const size_t wsb = gemm_ws(c, {{L, l, m, 1}, {l, l, L, 1}, {m, l, L, 1}, {m, l, l, 1}, {l, l, m, 1}, {m, l, 2 * l, 1}});
  Plan pl;
  pl.add(size_t(m) * 2 * l); pl.add(size_t(m) * 2 * l); pl.add(size_t(L) * l); pl.add(size_t(l) * l);
  pl.add(size_t(l) * l); pl.add(size_t(2) * l * l); pl.add(kn_series_work_doubles(l)); pl.add(wsb / 8 + 1);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  double* QX[2] = {ctx_take<double>(c, size_t(m) * 2 * l), ctx_take<double>(c, size_t(m) * 2 * l)};
  double* B = ctx_take<double>(c, size_t(L) * l);
  double* D = ctx_take<double>(c, size_t(l) * l);
  double* Z = ctx_take<double>(c, size_t(l) * l);
  double* CC = ctx_take<double>(c, size_t(2) * l * l);
  double* vwork = ctx_take<double>(c, kn_series_work_doubles(l));
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  const int64_t lq = 2 * l;
  MB_CHECK(ctx_tic(c));
  // Qc := Q0   (:105)
  MB_CHECK(copy2d(c, QX[0], lq, Qs, L, m, l));
  MB_CHECK(ctx_toc(c));
  int it = 0;
  MB_CHECK(kn_loop(c, maxit, [&](int i) -> int {
    const int cur = i & 1;
    double* Qc = QX[cur];
    double* X = QX[cur] + l;
    // B := Qs' Qc   (:117)
    MB_CHECK(dgemm(c, L, l, m, 1.0, cm(Qs, 1, L), crow(Qc, lq), 0.0, drow(B, l), GemmBatch(), ws));
    MB_CHECK(ctx_allreduce(c, B, L * l));   // row blocks over ranks
    // D := B' B   (:123)
    MB_CHECK(dgemm(c, l, l, L, 1.0, cm(B, 1, l), crow(B, l), 0.0, drow(D, l), GemmBatch(), ws));
    // X := Qs B / N;  X -= Qc D / N   (:126-129)
    MB_CHECK(dgemm(c, m, l, L, inv_n, crow(Qs, L), crow(B, l), 0.0, drow(X, lq), GemmBatch(), ws));
    MB_CHECK(dgemm(c, m, l, l, -inv_n, crow(Qc, lq), crow(D, l), 1.0, drow(X, lq), GemmBatch(), ws));
    // Z := X' X   (:143)
    MB_CHECK(dgemm(c, l, l, m, 1.0, cm(X, 1, lq), crow(X, lq), 0.0, drow(Z, l), GemmBatch(), ws));
    MB_CHECK(ctx_allreduce(c, Z, int64_t(l) * l));
    // eig(Z); C, inv(C); convergence test   (:146-164, :174-181)
    MB_CHECK(launch_kn_step(c, l, Z, nullptr, inv_n, CC, nullptr, nullptr, nullptr, vwork, tol));
    // Qc := Qc C + X inv(C) = [Qc X] [C; inv(C)]   (:170-171)
    MB_CHECK(dgemm(c, m, l, 2 * l, 1.0, crow(QX[cur], lq), crow(CC, l), 0.0, drow(QX[1 - cur], lq), GemmBatch(), ws));
    return MCNLA_B200_OK;
  }, &it));
  const int cur = it & 1;
  MB_CHECK(copy2d(c, Qbar, l, QX[cur], lq, m, l));
  MB_CHECK(ctx_toc(c));
  *iters = it;
  return MCNLA_B200_OK;
}

// RowBlockKolmogorovNagumoIntegrator (row_block_kolmogorov_nagumo_integrator.hpp:79-208)
int run_rb_kn(Context* c, const Dims& d, const double* Qs, int maxit, double tol, double* Qbar, int* iters) {
  const int l = d.l;
  const int64_t m = d.m, L = d.L;
  const double inv_n = 1.0 / d.N;
  const size_t wsb = gemm_ws(c, {{L, l, m, 1}, {m, l, L, 1}, {l, 2 * l, L, 1}, {m, l, 2 * l, 1}, {L, l, 2 * l, 1}});
  Plan pl;
  for (int i = 0; i < 2; ++i) { pl.add(size_t(m) * 2 * l); pl.add(size_t(L) * 2 * l); }
  pl.add(size_t(2) * l * l); pl.add(size_t(2) * l * l); pl.add(kn_series_work_doubles(l)); pl.add(wsb / 8 + 1);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  double* QG[2] = {ctx_take<double>(c, size_t(m) * 2 * l), ctx_take<double>(c, size_t(m) * 2 * l)};
  double* BB[2] = {ctx_take<double>(c, size_t(L) * 2 * l), ctx_take<double>(c, size_t(L) * 2 * l)};
  double* DD = ctx_take<double>(c, size_t(2) * l * l);
  double* FC = ctx_take<double>(c, size_t(2) * l * l);
  double* vwork = ctx_take<double>(c, kn_series_work_doubles(l));
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  const int64_t l2 = 2 * l;
  MB_CHECK(ctx_tic(c));
  // Qc := Q0; Bc := Qs' Qc   (:110-113)
  MB_CHECK(copy2d(c, QG[0], l2, Qs, L, m, l));
  MB_CHECK(dgemm(c, L, l, m, 1.0, cm(Qs, 1, L), crow(QG[0], l2), 0.0, drow(BB[0], l2), GemmBatch(), ws));
  MB_CHECK(ctx_allreduce2d(c, BB[0], l2, L, l));   // (:115)
  MB_CHECK(ctx_toc(c));
  int it = 0;
  MB_CHECK(kn_loop(c, maxit, [&](int i) -> int {
    const int cur = i & 1;
    // Gc := 1/N Qs Bc   (:138)
    MB_CHECK(dgemm(c, m, l, L, inv_n, crow(Qs, L), crow(BB[cur], l2), 0.0, drow(QG[cur] + l, l2), GemmBatch(), ws));
    // Bgc := Qs' Gc   (:141)
    MB_CHECK(dgemm(c, L, l, m, 1.0, cm(Qs, 1, L), crow(QG[cur] + l, l2), 0.0, drow(BB[cur] + l, l2), GemmBatch(), ws));
    MB_CHECK(ctx_allreduce2d(c, BB[cur] + l, l2, L, l));   // (:143)
    // [Dc | Dgc] := 1/N Bc' [Bc | Bgc]   (:147-150)
    MB_CHECK(dgemm(c, l, l2, L, inv_n, cm(BB[cur], 1, l2), crow(BB[cur], l2), 0.0, drow(DD, l2), GemmBatch(), ws));
    // Z := Dgc - Dc^2; eig; C, inv(C); Fc := C - Dc inv(C); convergence test   (:156-201)
    MB_CHECK(launch_kn_step(c, l, nullptr, DD, inv_n, FC, nullptr, nullptr, nullptr, vwork, tol));
    // Q+ := [Qc Gc] [Fc; inv(C)];  B+ := [Bc Bgc] [Fc; inv(C)]   (:189-194)
    MB_CHECK(dgemm(c, m, l, l2, 1.0, crow(QG[cur], l2), crow(FC, l), 0.0, drow(QG[1 - cur], l2), GemmBatch(), ws));
    MB_CHECK(dgemm(c, L, l, l2, 1.0, crow(BB[cur], l2), crow(FC, l), 0.0, drow(BB[1 - cur], l2), GemmBatch(), ws));
    return MCNLA_B200_OK;
  }, &it));
  const int cur = it & 1;
  MB_CHECK(copy2d(c, Qbar, l, QG[cur], l2, m, l));   // (:205)
  MB_CHECK(ctx_toc(c));
  *iters = it;
  return MCNLA_B200_OK;
}

// Precision form of Bs = Qs' Qs on the tensor cores: X = Qs' split into
// three BF16 parts (24 bits), Bs = sum X_p X_q' over the six part products
// with p + q <= 2 (the dropped ones are below 2^-24 relative): the 3-part
// product runs in the chunked configuration (FP32 chunks summed in FP64), the
// two smaller ones accumulate into Bs.  Lower-triangle tiles only.
// BF16 elements of the three parts of Qs' that gramian_bs_bf16 writes (x).
size_t gramian_bs16_count(const Dims& d) { return 3 * size_t(d.L) * size_t((d.m + 7) & ~int64_t(7)); }

int gramian_bs_bf16(Context* c, const Dims& d, const double* Qs, double* Bs, uint16_t* x) {
  const int64_t L = d.L, m = d.m, ldo = (m + 7) & ~int64_t(7);
  const size_t part = size_t(L) * ldo;
  uint16_t *hi = x, *lo = x + part, *lo2 = x + 2 * part;
  // X (L x m) is Qs (m x L row-major) read column-major
  MB_CHECK(launch_split_bf16(c, Qs, MCNLA_B200_COL_MAJOR, L, L, m, hi, lo, lo2, ldo));
  MB_CHECK(bf16_gemm(c, L, L, m, hi, lo, lo2, ldo, hi, ldo, Bs, L, true, false, true));   // (hi + lo + lo2) hi'
  MB_CHECK(bf16_gemm(c, L, L, m, hi, lo, nullptr, ldo, lo, ldo, Bs, L, true, true, true));  // + (hi + lo) lo'
  MB_CHECK(bf16_gemm(c, L, L, m, hi, nullptr, nullptr, ldo, lo2, ldo, Bs, L, true, true, true));   // + hi lo2'
  return MCNLA_B200_OK;
}

// Bs := Qs' Qs with the reference's triangle convention (see launch_gramian_prepare):
// the lower triangle only (the reference's syrk), mirrored afterwards.
// x: gramian_bs16_count(d) BF16 elements of workspace when c->mixed_gramian
int gramian_bs(Context* c, const Dims& d, const double* Qs, double* Bs, double* Bc, int64_t ldbc, double* ws,
               uint16_t* x) {
  if (c->mixed_gramian) MB_CHECK(gramian_bs_bf16(c, d, Qs, Bs, x));
  else MB_CHECK(dgemm(c, d.L, d.L, d.m, 1.0, cm(Qs, 1, d.L), crow(Qs, d.L), 0.0, drow(Bs, d.L), GemmBatch(), ws, 0,
                      true));
  // row blocks over ranks (row_block_gramian_kolmogorov_nagumo_integrator.hpp:117,
  // row_block_gramian_wen_yin_integrator.hpp:126): the lower triangles are summed
  MB_CHECK(ctx_allreduce(c, Bs, d.L * d.L));
  MB_CHECK(launch_gramian_prepare(c, d.L, d.l, Bs, Bc, ldbc));
  return MCNLA_B200_OK;
}

// Buffers of the row-block Gramian Kolmogorov-Nagumo integrator for one problem
// (carved by gkn_carve below).
struct GknBufs {
  uint16_t* bs16 = nullptr;   // precision form: BF16 parts of Qs', of Bs and of Bc', split-K slices
  uint16_t* bsp = nullptr;
  uint16_t* bcp = nullptr;
  double* slices = nullptr;
  double* Bs = nullptr;       // L x L
  double* EB[2] = {nullptr, nullptr};   // [E~ | Bc | Bgc] (L x 3l), current / next
  double* DD = nullptr;       // [Dc | Dgc] (l x 2l)
  double* FC = nullptr;       // [Fc; inv(C)] (2l x l)
  double* FCN = nullptr;      // [Fc; inv(C)/N]
  double* FF[2] = {nullptr, nullptr};   // F~ (l x l)
  double* Ebar = nullptr;     // L x l
  double* vwork = nullptr;    // KN step scratch
  double* cbuf = nullptr;     // l x l scratch of the grouped kernel's step
  double* ddp = nullptr;      // the grouped kernel's K-slice partials of [Dc | Dgc]
  double* job = nullptr;      // device GknJob and work-queue counter (the grouped kernel's single-job use)
  Bf16Split spb;
  bool bf16_bgc = false;
};

// Qbar := Q0 F~ + Qs E~ = Qs (E~ + [F~; 0])
int gramian_form_qbar(Context* c, const Dims& d, const double* Qs, const double* E, int64_t lde, const double* F,
                      double* Ebar, double* Qbar, double* ws) {
  const int l = d.l;
  MB_CHECK(copy2d(c, Ebar, l, E, lde, d.L, l));
  MB_CHECK(launch_axpby(c, l, l, 1.0, F, l, 1.0, Ebar, l));
  MB_CHECK(dgemm(c, d.m, l, d.L, 1.0, crow(Qs, d.L), crow(Ebar, l), 0.0, drow(Qbar, l), GemmBatch(), ws));
  return MCNLA_B200_OK;
}

// RowBlockGramianKolmogorovNagumoIntegrator
// (row_block_gramian_kolmogorov_nagumo_integrator.hpp:79-229), in pieces that
// the single solve below and the grouped batch (batch.cu) share: the
// buffers, the preparation (Bs, Bc, F~, E~), one launch-per-product
// iteration and the final Qbar.  Both run the same operations on the same
// shapes, so a problem gives the same bits either way.
size_t gkn_ws_bytes(const Context* c, const Dims& d) {
  const int64_t L = d.L, l = d.l, m = d.m;
  return gemm_ws(c, {{L, L, m, 1}, {L, l, L, 1}, {l, 2 * l, L, 1}, {L, l, 2 * l, 2}, {m, l, L, 1}});
}

// Visits the buffers in carve order: fn(count, element bytes).
template <class Fn>
void gkn_layout(const Context* c, const Dims& d, Fn fn, Bf16Split* spb_out = nullptr) {
  const int64_t L = d.L, l = d.l;
  const int64_t l3 = 3 * l, l2 = 2 * l;
  const size_t n16 = c->mixed_gramian ? gramian_bs16_count(d) : 0;
  const bool bf16_bgc = c->mixed_gramian;
  const int64_t ldL = (L + 7) & ~int64_t(7);
  Bf16Split spb;
  if (bf16_bgc) {
    spb = plan_bf16_split(c, L, 3 * l, L, true, 16);
    spb.split_stride = L * 3 * l;
  }
  if (spb_out) *spb_out = spb;
  const size_t nbs = bf16_bgc ? 3 * size_t(L) * ldL : 0, nbc = bf16_bgc ? 3 * size_t(l) * ldL : 0;
  const size_t nsl = bf16_bgc ? size_t(spb.splits) * L * 3 * l : 0;
  fn(n16, 2); fn(nbs, 2); fn(nbc, 2); fn(nsl, 8);
  fn(size_t(L) * L, 8); fn(size_t(L) * l3, 8); fn(size_t(L) * l3, 8); fn(size_t(l2) * l, 8);
  fn(size_t(l2) * l, 8); fn(size_t(l2) * l, 8); fn(size_t(l) * l, 8); fn(size_t(l) * l, 8);
  fn(size_t(L) * l, 8); fn(kn_series_work_doubles(int(l)), 8); fn(size_t(l) * l, 8);
  fn(gkn_grouped_ddp_doubles(int(l), L), 8); fn((sizeof(GknJob) + 64) / 8, 8);
}

size_t gkn_state_bytes(const Context* c, const Dims& d) {
  size_t b = 0;
  gkn_layout(c, d, [&](size_t count, size_t elem) { b += arena_bytes_for(count, elem); });
  return b;
}

// Carves the buffers with take(count, elem) (returns char*, null past the end).
template <class Take>
void gkn_carve(const Context* c, const Dims& d, Take take, GknBufs& b) {
  char* p[17];
  int i = 0;
  gkn_layout(c, d, [&](size_t count, size_t elem) { p[i++] = take(count, elem); }, &b.spb);
  b.bf16_bgc = c->mixed_gramian;
  b.bs16 = reinterpret_cast<uint16_t*>(p[0]);
  b.bsp = reinterpret_cast<uint16_t*>(p[1]);
  b.bcp = reinterpret_cast<uint16_t*>(p[2]);
  b.slices = reinterpret_cast<double*>(p[3]);
  b.Bs = reinterpret_cast<double*>(p[4]);
  b.EB[0] = reinterpret_cast<double*>(p[5]);
  b.EB[1] = reinterpret_cast<double*>(p[6]);
  b.DD = reinterpret_cast<double*>(p[7]);
  b.FC = reinterpret_cast<double*>(p[8]);
  b.FCN = reinterpret_cast<double*>(p[9]);
  b.FF[0] = reinterpret_cast<double*>(p[10]);
  b.FF[1] = reinterpret_cast<double*>(p[11]);
  b.Ebar = reinterpret_cast<double*>(p[12]);
  b.vwork = reinterpret_cast<double*>(p[13]);
  b.cbuf = reinterpret_cast<double*>(p[14]);
  b.ddp = reinterpret_cast<double*>(p[15]);
  b.job = reinterpret_cast<double*>(p[16]);
}

// Cluster size of the grouped kernel for a problem: about three 64-row units
// of the Bs Bc product per CTA (fuller units keep the FP64 MMA busier than more
// CTAs would; the results do not depend on it).
int gkn_cluster_for(int l, int64_t L) {
  const int64_t units = ((L + 63) / 64) * ((l + 127) / 128);
  return units <= 3 ? 1 : (units <= 7 ? 2 : (units <= 15 ? 4 : 8));
}

GknJob gkn_job(const Context* c, const Dims& d, const GknBufs& b, int it0, int maxit, double tol) {
  GknJob j = {};
  j.l = d.l;
  j.L = int(d.L);
  j.it0 = it0;
  j.maxit = maxit;
  j.smax = gkn_grouped_smax(c, d.l);
  j.inv_n = 1.0 / d.N;
  j.tol = tol;
  j.bs = b.Bs;
  j.eb0 = b.EB[0];
  j.eb1 = b.EB[1];
  j.ff0 = b.FF[0];
  j.ff1 = b.FF[1];
  j.dd = b.DD;
  j.fc = b.FC;
  j.fcn = b.FCN;
  j.work = b.vwork;
  j.cbuf = b.cbuf;
  j.ddp = b.ddp;
  j.stop_it = INT_MAX;
  j.resume_it = -1;
  return j;
}

// Bs := Qs' Qs; Bc := Bs(:, 0:l); F~ := I; E~ := 0   (:112-133)
int gkn_prepare(Context* c, const Dims& d, const double* Qs, const GknBufs& b, double* ws) {
  const int l = d.l;
  const int64_t L = d.L, l3 = 3 * l;
  MB_CHECK(gramian_bs(c, d, Qs, b.Bs, b.EB[0] + l, l3, ws, b.bs16));
  MB_CHECK(launch_fill(c, L, l, 0.0, b.EB[0], l3));
  MB_CHECK(launch_set_identity(c, l, b.FF[0], l));
  const int64_t ldL = (L + 7) & ~int64_t(7);
  const size_t bpart = size_t(L) * ldL;
  if (b.bf16_bgc)
    MB_CHECK(launch_split_bf16(c, b.Bs, MCNLA_B200_ROW_MAJOR, L, L, L, b.bsp, b.bsp + bpart, b.bsp + 2 * bpart, ldL));
  return MCNLA_B200_OK;
}

// Iteration i on the launch-per-product path (:152-204).
int gkn_iteration(Context* c, const Dims& d, const GknBufs& b, int i, bool allow_series, double tol, double* ws) {
  const int l = d.l;
  const int64_t L = d.L, l3 = 3 * l, l2 = 2 * l;
  const double inv_n = 1.0 / d.N;
  const int cur = i & 1;
  double* Ec = b.EB[cur];
  double* Bc = b.EB[cur] + l;
  double* Bgc = b.EB[cur] + l2;
  // Bgc := 1/N Bs Bc   (:152)
  if (b.bf16_bgc) {
    // (Bs_hi + Bs_lo + Bs_lo2) [Bc_hi | Bc_lo | Bc_lo2] on tcgen05 (Bc' split from the column-major view
    // of Bc), the three column groups and the K slices added in order, times 1/N
    const int64_t ldL = (L + 7) & ~int64_t(7);
    const size_t bpart = size_t(L) * ldL, cpart = size_t(l) * ldL;
    MB_CHECK(launch_split_bf16(c, Bc, MCNLA_B200_COL_MAJOR, l3, l, L, b.bcp, b.bcp + cpart, b.bcp + 2 * cpart, ldL));
    MB_CHECK(bf16_gemm_split(c, L, 3 * l, L, b.bsp, b.bsp + bpart, b.bsp + 2 * bpart, ldL, b.bcp, ldL, b.slices,
                             3 * l, true, false, false, b.spb));
    MB_CHECK(launch_sum_splits(c, b.slices, b.spb.splits, b.spb.split_stride, L, l, 3 * l, Bgc, l3, false, inv_n, 3,
                               l));
  } else {
    MB_CHECK(dgemm(c, L, l, L, inv_n, crow(b.Bs, L), crow(Bc, l3), 0.0, drow(Bgc, l3), GemmBatch(), ws));
  }
  // [Dc | Dgc] := 1/N Bc' [Bc | Bgc]   (:155-158)
  MB_CHECK(dgemm(c, l, l2, L, inv_n, cm(Bc, 1, l3), crow(Bc, l3), 0.0, drow(b.DD, l2), GemmBatch(), ws));
  // Z, eig, C, inv(C), Fc; F~+ := F~c Fc; convergence test   (:164-214)
  MB_CHECK(launch_kn_step(c, l, nullptr, b.DD, inv_n, b.FC, b.FCN, b.FF[cur], b.FF[1 - cur], b.vwork, tol,
                          allow_series));
  // E~+ := E~c Fc + 1/N Bc inv(C) = [E~c Bc] [Fc; inv(C)/N]   (:194, :200)
  // B+ := [Bc Bgc] [Fc; inv(C)]   (:203-204)
  // one batched launch: member 0 reads columns [0, 2l) of the state and [Fc; inv(C)/N], member 1
  // columns [l, 3l) and [Fc; inv(C)], writing E~+ and B+ side by side
  MB_CHECK(dgemm(c, L, l, l2, 1.0, crow(Ec, l3), crow(b.FCN, l), 0.0, drow(b.EB[1 - cur], l3),
                 GemmBatch{2, l, int64_t(b.FC - b.FCN), l}, ws));
  return MCNLA_B200_OK;
}

// Qbar := Q0 F~ + Qs E~ after `it` iterations   (:225-226)
int gkn_finish(Context* c, const Dims& d, const double* Qs, const GknBufs& b, int it, double* Qbar, double* ws) {
  const int cur = it & 1;
  return gramian_form_qbar(c, d, Qs, b.EB[cur], 3 * d.l, b.FF[cur], b.Ebar, Qbar, ws);
}

int run_rb_gramian_kn(Context* c, const Dims& d, const double* Qs, int maxit, double tol, double* Qbar, int* iters) {
  const int l = d.l;
  const int64_t L = d.L;
  const size_t wsb = gkn_ws_bytes(c, d);
  Plan pl;
  gkn_layout(c, d, [&](size_t count, size_t elem) { pl.add(count, elem); });
  pl.add(wsb / 8 + 1);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  GknBufs b;
  gkn_carve(c, d, [&](size_t count, size_t elem) -> char* {
    return elem == 2 ? reinterpret_cast<char*>(ctx_take<uint16_t>(c, count))
                     : reinterpret_cast<char*>(ctx_take<double>(c, count));
  }, b);
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  MB_CHECK(ctx_tic(c));
  MB_CHECK(gkn_prepare(c, d, Qs, b, ws));
  MB_CHECK(ctx_toc(c));
  auto body = [&](int i, bool allow_series) -> int { return gkn_iteration(c, d, b, i, allow_series, tol, ws); };
  int it = 0;
  if (c->kn_mode == MCNLA_B200_KN_AUTO && gkn_persistent_fits(c, l, L)) {
    // whole iterations on one cooperative grid; an iteration whose KN step the
    // series declines runs here on the launch-per-product path
    MB_CHECK_CUDA(cudaMemsetAsync(&c->scal->stop_it, 0x7f, sizeof(int), c->stream));   // "not yet"
    int it0 = 0, done = -1;
    while (it0 < maxit && done < 0) {
      MB_CHECK_CUDA(cudaMemsetAsync(&c->scal->resume_it, 0xff, sizeof(int), c->stream));   // -1
      MB_CHECK(launch_gkn_persistent(c, l, L, d.N, tol, it0, maxit, b.Bs, b.EB, b.FF, b.DD, b.FC, b.FCN, b.vwork));
      MB_CHECK(ctx_sync_scalars(c));
      if (c->scal_host->status) return c->scal_host->status;
      if (c->scal_host->stop_it < maxit) { done = c->scal_host->stop_it + 1; break; }
      const int r = c->scal_host->resume_it;
      if (r < 0) break;                                       // maxit reached
      struct Reset { Context* c; ~Reset() { c->guard_stop = nullptr; c->guard_it = 0; } } reset{c};
      c->guard_stop = &c->scal->stop_it;
      c->guard_it = r;
      MB_CHECK(body(r, false));
      MB_CHECK(ctx_sync_scalars(c));
      if (c->scal_host->status) return c->scal_host->status;
      if (c->scal_host->stop_it == r) done = r + 1;
      it0 = r + 1;
    }
    it = done < 0 ? maxit : done;
  } else {
    MB_CHECK(kn_loop(c, maxit, [&](int i) -> int { return body(i, true); }, &it));
  }
  MB_CHECK(ctx_toc(c));
  MB_CHECK(gkn_finish(c, d, Qs, b, it, Qbar, ws));
  MB_CHECK(ctx_toc(c));
  *iters = it;
  return MCNLA_B200_OK;
}

// Wen-Yin line search shared by both Wen-Yin integrators
// (row_block_wen_yin_integrator.hpp:171-214).  bbc = [Bc | Bgc] (row stride
// ldb); B+ is written to bp (row stride ldp).  Returns phit through *phit.
int wy_line_search(Context* c, const Dims& d, const double* dd, const double* bbc, int64_t ldb, double* bp,
                   int64_t ldp, double taug, double phi, double mu, double* F, double* FN, double* partials,
                   double* ws, double* phit) {
  const int l = d.l;
  const double inv_n = 1.0 / d.N;
  double tau = taug;
  double pt = phi;
  for (int trial = 0; trial < kTauMaxIter; ++trial, tau *= kBeta) {
    MB_CHECK(launch_wy_trial(c, l, dd, tau, inv_n, F, FN));
    MB_CHECK(dgemm(c, d.L, l, 2 * l, 1.0, crow(bbc, ldb), crow(F, l), 0.0, drow(bp, ldp), GemmBatch(), ws));
    MB_CHECK(launch_sumsq(c, bp, d.L, l, ldp, 0.5 * inv_n, partials, &c->scal->phit));
    MB_CHECK(ctx_sync_scalars(c));
    if (c->scal_host->status) return c->scal_host->status;
    pt = c->scal_host->phit;
    if (pt >= phi + tau * kSigma * mu) break;
  }
  *phit = pt;
  return MCNLA_B200_OK;
}

// RowBlockWenYinIntegrator (row_block_wen_yin_integrator.hpp:79-281)
int run_rb_wy(Context* c, const Dims& d, const double* Qs, int maxit, double tol, double* Qbar, int* iters) {
  const int l = d.l;
  const int64_t m = d.m, L = d.L, l2 = 2 * l;
  const double inv_n = 1.0 / d.N;
  if (l > MCNLA_B200_MAX_DIM_SKETCH_WENYIN) return MCNLA_B200_ERR_UNSUPPORTED;
  const size_t wsb = gemm_ws(c, {{L, l, m, 1}, {m, l, L, 1}, {l, l2, L, 1}, {m, l, l, 1}, {L, l, l2, 1}, {m, l, l2, 1}});
  const int np = reduce_partials(c) * 3;
  Plan pl;
  for (int i = 0; i < 2; ++i) { pl.add(size_t(m) * l2); pl.add(size_t(m) * l); pl.add(size_t(L) * l2); }
  pl.add(size_t(l) * l2); pl.add(size_t(l2) * l); pl.add(size_t(np)); pl.add(wsb / 8 + 1);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  double* QG[2] = {ctx_take<double>(c, size_t(m) * l2), ctx_take<double>(c, size_t(m) * l2)};
  double* X[2] = {ctx_take<double>(c, size_t(m) * l), ctx_take<double>(c, size_t(m) * l)};
  double* BB[2] = {ctx_take<double>(c, size_t(L) * l2), ctx_take<double>(c, size_t(L) * l2)};
  double* DD = ctx_take<double>(c, size_t(l) * l2);
  double* F = ctx_take<double>(c, size_t(l2) * l);
  double* partials = ctx_take<double>(c, size_t(np));
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
  MB_CHECK(ctx_tic(c));
  // Initializing (:112-143)
  MB_CHECK(copy2d(c, QG[0], l2, Qs, L, m, l));                                                        // Qc := Q0
  MB_CHECK(dgemm(c, L, l, m, 1.0, cm(Qs, 1, L), crow(QG[0], l2), 0.0, drow(BB[0], l2), GemmBatch(), ws));  // Bc
  MB_CHECK(ctx_allreduce2d(c, BB[0], l2, L, l));   // (:117)
  MB_CHECK(dgemm(c, m, l, L, inv_n, crow(Qs, L), crow(BB[0], l2), 0.0, drow(QG[0] + l, l2), GemmBatch(), ws));  // Gc
  MB_CHECK(dgemm(c, L, l, m, 1.0, cm(Qs, 1, L), crow(QG[0] + l, l2), 0.0, drow(BB[0] + l, l2), GemmBatch(), ws));  // Bgc
  MB_CHECK(ctx_allreduce2d(c, BB[0] + l, l2, L, l));   // (:129)
  MB_CHECK(dgemm(c, l, l2, L, inv_n, cm(BB[0], 1, l2), crow(BB[0], l2), 0.0, drow(DD, l2), GemmBatch(), ws));  // Dc|Dgc
  // Xc := Gc - Qc Dc
  MB_CHECK(copy2d(c, X[0], l, QG[0] + l, l2, m, l));
  MB_CHECK(dgemm(c, m, l, l, -1.0, crow(QG[0], l2), crow(DD, l2), 1.0, drow(X[0], l), GemmBatch(), ws));
  // phi := 1/2N ||Bc||_F^2; mu := tr(Dgc) - ||Dc||_F^2
  MB_CHECK(launch_sumsq(c, BB[0], L, l, l2, 0.5 * inv_n, partials, &c->scal->dot[0]));
  MB_CHECK(launch_wy_mu(c, l, DD, &c->scal->mu));
  MB_CHECK(ctx_sync_scalars(c));
  double taug = kTau0, zeta = 1.0, phi = c->scal_host->dot[0], mu = c->scal_host->mu;
  MB_CHECK(ctx_toc(c));
  int cur = 0, it = 0, fin = 0;
  bool is_odd = false;
  HotLoop hot(c);
  for (; it < maxit;) {
    const int nx = 1 - cur;
    is_odd = !is_odd;
    double phit = phi;
    // B+ := Bc Fc + Bgc Fgc with the accepted step   (:171-214)
    MB_CHECK(wy_line_search(c, d, DD, BB[cur], l2, BB[nx], l2, taug, phi, mu, F, nullptr, partials, ws, &phit));
    phi = (kEta * zeta * phi + phit) / (kEta * zeta + 1);   // (:217)
    zeta = kEta * zeta + 1;                                  // (:218)
    // Q+ := [Qc Gc] [Fc; Fgc]   (:221-222)
    MB_CHECK(dgemm(c, m, l, l2, 1.0, crow(QG[cur], l2), crow(F, l), 0.0, drow(QG[nx], l2), GemmBatch(), ws));
    // G+ := 1/N Qs B+; Bg+ := Qs' G+; [D+ | Dg+] := 1/N B+' [B+ | Bg+]   (:224-236)
    MB_CHECK(dgemm(c, m, l, L, inv_n, crow(Qs, L), crow(BB[nx], l2), 0.0, drow(QG[nx] + l, l2), GemmBatch(), ws));
    MB_CHECK(dgemm(c, L, l, m, 1.0, cm(Qs, 1, L), crow(QG[nx] + l, l2), 0.0, drow(BB[nx] + l, l2), GemmBatch(), ws));
    MB_CHECK(ctx_allreduce2d(c, BB[nx] + l, l2, L, l));   // (:229)
    MB_CHECK(dgemm(c, l, l2, L, inv_n, cm(BB[nx], 1, l2), crow(BB[nx], l2), 0.0, drow(DD, l2), GemmBatch(), ws));
    // mu := tr(Dg+) - ||D+||_F^2   (:240)
    MB_CHECK(launch_wy_mu(c, l, DD, &c->scal->mu));
    MB_CHECK(ctx_sync_scalars(c));
    mu = c->scal_host->mu;
    if (mu < tol * tol) {   // (:249-250)
      ++it;
      fin = nx;
      break;
    }
    // X+ := G+ - Q+ D+   (:253-254)
    MB_CHECK(copy2d(c, X[nx], l, QG[nx] + l, l2, m, l));
    MB_CHECK(dgemm(c, m, l, l, -1.0, crow(QG[nx], l2), crow(DD, l2), 1.0, drow(X[nx], l), GemmBatch(), ws));
    // Delta1 := Qc - Q+, Delta2 := Xc - X+ and their inner products   (:261-274)
    MB_CHECK(launch_wy_delta_dots(c, QG[cur], QG[nx], l2, X[cur], X[nx], l, m, l, partials, &c->scal->dot[0]));
    MB_CHECK(ctx_allreduce(c, &c->scal->dot[0], 3));   // (:269)
    MB_CHECK(ctx_sync_scalars(c));
    const double d11 = c->scal_host->dot[0], d12 = c->scal_host->dot[1], d22 = c->scal_host->dot[2];
    const double t1 = is_odd ? d11 : d12, t2 = is_odd ? d12 : d22;
    taug = std::fabs(t1 / t2);   // (:278-280)
    if (taug < kTauMin) taug = kTauMin;
    if (taug > kTauMax) taug = kTauMax;
    cur = nx;
    fin = cur;
    ++it;
  }
  MB_CHECK(copy2d(c, Qbar, l, QG[fin], l2, m, l));
  MB_CHECK(ctx_toc(c));
  *iters = it;
  return MCNLA_B200_OK;
}

// RowBlockGramianWenYinIntegrator (row_block_gramian_wen_yin_integrator.hpp:86-331)
int run_rb_gramian_wy(Context* c, const Dims& d, const double* Qs, int maxit, double tol, double* Qbar, int* iters) {
  const int l = d.l;
  const int64_t m = d.m, L = d.L, l2 = 2 * l, l3 = 3 * l;
  const double inv_n = 1.0 / d.N;
  if (l > MCNLA_B200_MAX_DIM_SKETCH_WENYIN) return MCNLA_B200_ERR_UNSUPPORTED;
  const size_t wsb = gemm_ws(c, {{L, L, m, 1}, {L, l, L, 1}, {l, l2, L, 1}, {L, l, l2, 1}, {L, l, l, 1}, {l, l, l, 1},
                                 {m, l, L, 1}});
  const int np = reduce_partials(c) * 3;
  Plan pl;
  pl.add(size_t(L) * L);
  for (int i = 0; i < 2; ++i) { pl.add(size_t(L) * l3); pl.add(size_t(l) * l2); pl.add(size_t(l) * l); }
  pl.add(size_t(l2) * l); pl.add(size_t(l2) * l); pl.add(size_t(L) * l2); pl.add(size_t(L) * l);
  pl.add(size_t(l) * l); pl.add(size_t(l) * l); pl.add(size_t(l) * l2); pl.add(size_t(L) * l);
  pl.add(size_t(np)); pl.add(wsb / 8 + 1);
  const size_t n16 = c->mixed_gramian ? gramian_bs16_count(d) : 0;
  pl.add(n16, sizeof(uint16_t));
  MB_CHECK(ctx_reserve(c, pl.bytes));
  uint16_t* bs16 = ctx_take<uint16_t>(c, n16);
  double* Bs = ctx_take<double>(c, size_t(L) * L);
  double* EB[2] = {ctx_take<double>(c, size_t(L) * l3), ctx_take<double>(c, size_t(L) * l3)};
  double* DD[2] = {ctx_take<double>(c, size_t(l) * l2), ctx_take<double>(c, size_t(l) * l2)};
  double* FF[2] = {ctx_take<double>(c, size_t(l) * l), ctx_take<double>(c, size_t(l) * l)};
  double* F = ctx_take<double>(c, size_t(l2) * l);
  double* FN = ctx_take<double>(c, size_t(l2) * l);
  double* U = ctx_take<double>(c, size_t(L) * l2);     // [U1 | U2]
  double* BsU = ctx_take<double>(c, size_t(L) * l);
  double* PHI1 = ctx_take<double>(c, size_t(l) * l);
  double* PHI2 = ctx_take<double>(c, size_t(l) * l);
  double* BCU = ctx_take<double>(c, size_t(l) * l2);   // [Bc'U1 | Bc'U2]
  double* Ebar = ctx_take<double>(c, size_t(L) * l);
  double* partials = ctx_take<double>(c, size_t(np));
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
  MB_CHECK(ctx_tic(c));
  // Initializing (:121-155)
  MB_CHECK(gramian_bs(c, d, Qs, Bs, EB[0] + l, l3, ws, bs16));
  MB_CHECK(dgemm(c, L, l, L, inv_n, crow(Bs, L), crow(EB[0] + l, l3), 0.0, drow(EB[0] + l2, l3), GemmBatch(), ws));
  MB_CHECK(dgemm(c, l, l2, L, inv_n, cm(EB[0] + l, 1, l3), crow(EB[0] + l, l3), 0.0, drow(DD[0], l2), GemmBatch(), ws));
  MB_CHECK(launch_set_identity(c, l, FF[0], l));
  MB_CHECK(launch_fill(c, L, l, 0.0, EB[0], l3));
  MB_CHECK(launch_sumsq(c, EB[0] + l, L, l, l3, 0.5 * inv_n, partials, &c->scal->dot[0]));
  MB_CHECK(launch_wy_mu(c, l, DD[0], &c->scal->mu));
  MB_CHECK(ctx_sync_scalars(c));
  double taug = kTau0, zeta = 1.0, phi = c->scal_host->dot[0], mu = c->scal_host->mu;
  MB_CHECK(ctx_toc(c));
  int cur = 0, it = 0;
  bool is_odd = false;
  HotLoop hot(c);
  for (; it < maxit;) {
    const int nx = 1 - cur;
    double* Ec = EB[cur];
    double* Bc = EB[cur] + l;
    double* Bp = EB[nx] + l;
    is_odd = !is_odd;
    double phit = phi;
    MB_CHECK(wy_line_search(c, d, DD[cur], Bc, l3, Bp, l3, taug, phi, mu, F, FN, partials, ws, &phit));
    phi = (kEta * zeta * phi + phit) / (kEta * zeta + 1);   // (:225)
    zeta = kEta * zeta + 1;
    // U1 := 1/N Bc Fgc   (:229)
    MB_CHECK(dgemm(c, L, l, l, inv_n, crow(Bc, l3), crow(F + size_t(l) * l, l), 0.0, drow(U, l2), GemmBatch(), ws));
    // F~+ := F~c Fc   (:232)
    MB_CHECK(dgemm(c, l, l, l, 1.0, crow(FF[cur], l), crow(F, l), 0.0, drow(FF[nx], l), GemmBatch(), ws));
    // E~+ := E~c Fc + U1 = [E~c Bc] [Fc; Fgc/N]   (:235-236)
    MB_CHECK(dgemm(c, L, l, l2, 1.0, crow(Ec, l3), crow(FN, l), 0.0, drow(EB[nx], l3), GemmBatch(), ws));
    // Bg+ := 1/N Bs B+; [D+ | Dg+] := 1/N B+' [B+ | Bg+]   (:239-245)
    MB_CHECK(dgemm(c, L, l, L, inv_n, crow(Bs, L), crow(Bp, l3), 0.0, drow(EB[nx] + l2, l3), GemmBatch(), ws));
    MB_CHECK(dgemm(c, l, l2, L, inv_n, cm(Bp, 1, l3), crow(Bp, l3), 0.0, drow(DD[nx], l2), GemmBatch(), ws));
    MB_CHECK(launch_wy_mu(c, l, DD[nx], &c->scal->mu));   // (:248)
    MB_CHECK(ctx_sync_scalars(c));
    mu = c->scal_host->mu;
    cur = nx;
    if (mu < tol * tol) {   // (:252)
      ++it;
      break;
    }
    // Phi2 := Dc - Fc D+; Phi1 := Fc - I   (:261-266)
    MB_CHECK(launch_wy_gramian_phis(c, l, F, DD[1 - cur], l2, DD[cur], l2, PHI1, PHI2));
    // U2 := 1/N (B+ - Bc) - U1 D+   (:269-271)
    MB_CHECK(launch_axpby(c, L, l, inv_n, Bp, l3, 0.0, U + l, l2));
    MB_CHECK(launch_axpby(c, L, l, -inv_n, Bc, l3, 1.0, U + l, l2));
    MB_CHECK(dgemm(c, L, l, l, -1.0, crow(U, l2), crow(DD[cur], l2), 1.0, drow(U + l, l2), GemmBatch(), ws));
    // [Bc'U1 | Bc'U2]   (:274-277)
    MB_CHECK(dgemm(c, l, l2, L, 1.0, cm(Bc, 1, l3), crow(U, l2), 0.0, drow(BCU, l2), GemmBatch(), ws));
    // Bs U1 (odd) or Bs U2 (even)   (:286, :298)
    const double* Usel = is_odd ? U : U + l;
    MB_CHECK(dgemm(c, L, l, L, 1.0, crow(Bs, L), crow(Usel, l2), 0.0, drow(BsU, l), GemmBatch(), ws));
    MB_CHECK(launch_gwy_small_dots(c, l, PHI1, PHI2, BCU, &c->scal->dot[0]));
    MB_CHECK(launch_dot(c, U, l2, BsU, l, L, l, partials, &c->scal->dot[8]));
    MB_CHECK(launch_dot(c, U + l, l2, BsU, l, L, l, partials, &c->scal->dot[9]));
    MB_CHECK(ctx_sync_scalars(c));
    const double* s = c->scal_host->dot;
    // s: 0 <P1,P1> 1 <P1,P2> 2 <P2,P2> 3 <P1,BU1> 4 <P1,BU2> 5 <P2,BU1> 6 <P2,BU2> 8 <U1,BsU> 9 <U2,BsU>
    double t1, t2;
    if (is_odd) {   // (:284-293)
      t1 = s[0] + 2 * s[3] + s[8];
      t2 = s[1] + s[4] + s[5] + s[9];
    } else {        // (:294-306)
      t1 = s[1] + s[4] + s[5] + s[8];
      t2 = s[2] + 2 * s[6] + s[9];
    }
    taug = std::fabs(t1 / t2);   // (:309-311)
    if (taug < kTauMin) taug = kTauMin;
    if (taug > kTauMax) taug = kTauMax;
    ++it;
  }
  MB_CHECK(ctx_toc(c));
  // Qbar := Q0 F~ + Qs E~   (:327-328)
  MB_CHECK(gramian_form_qbar(c, d, Qs, EB[cur], l3, FF[cur], Ebar, Qbar, ws));
  MB_CHECK(ctx_toc(c));
  *iters = it;
  return MCNLA_B200_OK;
}

int run_integrate(Context* c, const Dims& d, int kind, const double* Qs, int maxit, double tol, double* Qbar,
                  int* iters) {
  if (!Qs || !Qbar || !iters) return MCNLA_B200_ERR_ARG;
  if (maxit < 0 || !(tol >= 0.0)) return MCNLA_B200_ERR_ARG;
  // device status, convergence scalars and grid-barrier counters start clean
  MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
  switch (kind) {
    case MCNLA_B200_KOLMOGOROV_NAGUMO: return run_kn(c, d, Qs, maxit, tol, Qbar, iters);
    case MCNLA_B200_ROW_BLOCK_KOLMOGOROV_NAGUMO: return run_rb_kn(c, d, Qs, maxit, tol, Qbar, iters);
    case MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO: return run_rb_gramian_kn(c, d, Qs, maxit, tol, Qbar, iters);
    case MCNLA_B200_ROW_BLOCK_WEN_YIN: return run_rb_wy(c, d, Qs, maxit, tol, Qbar, iters);
    case MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN: return run_rb_gramian_wy(c, d, Qs, maxit, tol, Qbar, iters);
    default: return MCNLA_B200_ERR_ARG;
  }
}

// ---------------------------------------------------------------------------
// Formers
// ---------------------------------------------------------------------------
// SvdFormer<_, true> (svd_former.hpp:70-116).  gesvd(Vt) is replaced by an
// accuracy-preserving equivalent: two Gram re-orthonormalizations of the rows
// of Vt give Y2 (orthonormal rows spanning the same space), M := Vt Y2' is
// formed by a GEMM, and M's SVD is taken by one-sided Jacobi:
// Vt = M Y2 = W S (Y2' Z)'.
// BF16 parts of A' (n x m, K-major: row j of A' is column j of A) for the
// precision-form former; lo and lo2 may be null.
struct AtParts {
  const uint16_t* hi = nullptr;
  const uint16_t* lo = nullptr;
  const uint16_t* lo2 = nullptr;
  int64_t ld = 0;
};

// Precision-form former product Q' A (l x n) on tcgen05 from the BF16 parts
// of A' and a three-part BF16 split of Qbar:
//   (Q_hi + Q_lo + Q_lo2) A'_hi' + (Q_hi + Q_lo) A'_lo' + Q_hi A'_lo2'
// (every product down to 2^-24 of the leading one), the first in the chunked
// configuration (FP64 sums of FP32 chunks; the K loop runs over all m rows),
// split over K so that the CTAs fill the SMs, the slices added in a fixed
// order into out: Q' A (l x n, pitch ldo) or, with transpose, A' Q (n x l).
constexpr int kFormMaxSplits = 16;

// Workspace of form_product_bf16: BF16 elements (the three parts of Q') and
// doubles (the split slices).
size_t form16_count(const Dims& d) { return 3 * size_t(d.l) * size_t((d.m + 7) & ~int64_t(7)); }
size_t form_split_doubles(const Context* c, const Dims& d) {
  return size_t(plan_bf16_split(c, d.l, d.n, d.m, true, kFormMaxSplits).splits) * d.l * d.n;
}

int form_product_bf16(Context* c, const Dims& d, const AtParts& at, const double* Qbar, double* out, int64_t ldo,
                      bool transpose, uint16_t* q16, double* parts) {
  const int64_t l = d.l, m = d.m, n = d.n, ldq = (m + 7) & ~int64_t(7);
  if (!at.hi || (at.lo2 && !at.lo) || at.ld < m) return MCNLA_B200_ERR_ARG;
  Bf16Split sp = plan_bf16_split(c, l, n, m, true, kFormMaxSplits);
  sp.split_stride = l * n;
  sp.chunk_kt = 1;   // sigma takes this product's error to first order: 12 accumulator updates per chunk
  const size_t qpart = size_t(l) * ldq;
  uint16_t *qh = q16, *ql = q16 + qpart, *ql2 = q16 + 2 * qpart;
  // Q' parts: Qbar (m x l, row-major) read as the column-major l x m matrix Q'
  MB_CHECK(launch_split_bf16(c, Qbar, MCNLA_B200_COL_MAJOR, l, l, m, qh, ql, ql2, ldq));
  MB_CHECK(bf16_gemm_split(c, l, n, m, qh, ql, ql2, ldq, at.hi, at.ld, parts, n, true, false, false, sp));
  if (at.lo) MB_CHECK(bf16_gemm_split(c, l, n, m, qh, ql, nullptr, ldq, at.lo, at.ld, parts, n, true, true, false, sp));
  if (at.lo2)
    MB_CHECK(bf16_gemm_split(c, l, n, m, qh, nullptr, nullptr, ldq, at.lo2, at.ld, parts, n, true, true, false, sp));
  MB_CHECK(launch_sum_splits(c, parts, sp.splits, sp.split_stride, l, n, n, out, ldo, transpose));
  return MCNLA_B200_OK;
}

int run_form_svd(Context* c, const Dims& d, const CMat& Am, const double* Qbar, double* S, double* U, double* V,
                 const AtParts* at) {
  const int l = d.l, k = d.k;
  const int64_t m = d.m, n = d.n;
  const size_t ll = size_t(l) * l;
  const size_t wsb = gemm_ws(c, {{l, n, m, 1}, {l, l, n, 1}, {l, n, l, 1}, {m, k, l, 1}, {n, k, l, 1}});
  Plan pl;
  pl.add(size_t(l) * n); pl.add(size_t(l) * n); pl.add(size_t(l) * n);
  for (int i = 0; i < 6; ++i) pl.add(ll);
  pl.add(size_t(2) * l); pl.add(wsb / 8 + 1);
  for (int i = 0; i < 4; ++i) pl.add(ll);   // on-chip solver spill copies (l > 112)
  const size_t n16 = at ? form16_count(d) : 0, nsp = at ? form_split_doubles(c, d) : 0;
  pl.add(n16, sizeof(uint16_t)); pl.add(nsp);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  uint16_t* q16 = ctx_take<uint16_t>(c, n16);
  double* slices = ctx_take<double>(c, nsp);
  double* Vt = ctx_take<double>(c, size_t(l) * n);
  double* Y1 = ctx_take<double>(c, size_t(l) * n);
  double* Y2 = ctx_take<double>(c, size_t(l) * n);
  double* G = ctx_take<double>(c, ll);
  double* Ue = ctx_take<double>(c, ll);
  double* P = ctx_take<double>(c, ll);
  double* M = ctx_take<double>(c, ll);
  double* Wm = ctx_take<double>(c, ll);
  double* Zm = ctx_take<double>(c, ll);
  double* w = ctx_take<double>(c, size_t(2) * l);
  double* sig = w + l;
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  MB_CHECK(ctx_tic(c));
  // Vt := Q' A   (:99)
  if (at) MB_CHECK(form_product_bf16(c, d, *at, Qbar, Vt, n, false, q16, slices));
  else MB_CHECK(dgemm(c, l, n, m, 1.0, cm(Qbar, 1, l), Am, 0.0, drow(Vt, n), GemmBatch(), ws));
  MB_CHECK(ctx_allreduce(c, Vt, int64_t(l) * n));   // row blocks over ranks
  MB_CHECK(ctx_toc(c));
  // svd(Vt)   (:106)
  const double* Yin = Vt;
  double* Yout[2] = {Y1, Y2};
  for (int pass = 0; pass < 2; ++pass) {
    MB_CHECK(dgemm(c, l, l, n, 1.0, crow(Yin, n), cm(Yin, 1, n), 0.0, drow(G, l), GemmBatch(), ws));
    MB_CHECK(launch_syev(c, l, 1, G, l, 0, w, Ue, 1));
    MB_CHECK(launch_rsqrt_rows_t(c, l, Ue, w, P));
    MB_CHECK(dgemm(c, l, n, l, 1.0, crow(P, l), crow(Yin, n), 0.0, drow(Yout[pass], n), GemmBatch(), ws));
    Yin = Yout[pass];
  }
  MB_CHECK(dgemm(c, l, l, n, 1.0, crow(Vt, n), cm(Y2, 1, n), 0.0, drow(M, l), GemmBatch(), ws));
  MB_CHECK(launch_svd_small(c, l, M, Wm, sig, Zm));
  MB_CHECK(ctx_toc(c));
  // U := Q W(:, 0:k); V := (Y2' Z)(:, 0:k)   (:113, :142)
  if (U) MB_CHECK(dgemm(c, m, k, l, 1.0, crow(Qbar, l), crow(Wm, l), 0.0, drow(U, k), GemmBatch(), ws));
  if (V) MB_CHECK(dgemm(c, n, k, l, 1.0, cm(Y2, 1, n), crow(Zm, l), 0.0, drow(V, k), GemmBatch(), ws));
  if (S) MB_CHECK_CUDA(cudaMemcpyAsync(S, sig, size_t(k) * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  MB_CHECK(ctx_toc(c));
  return MCNLA_B200_OK;
}

// GramianFormer / RowBlockGramianFormer / ColBlockGramianFormer (with V)
// (gramian_former.hpp:72-132; row_block_gramian_former.hpp:78-146;
//  col_block_gramian_former.hpp:73-131): on one device the three agree.
int run_form_gramian(Context* c, const Dims& d, const CMat& Am, const double* Qbar, double* S, double* U,
                     double* V, const AtParts* at) {
  const int l = d.l, k = d.k;
  const int64_t m = d.m, n = d.n;
  const size_t ll = size_t(l) * l;
  const size_t wsb = gemm_ws(c, {{n, l, m, 1}, {l, l, n, 1}, {m, k, l, 1}, {n, k, l, 1}});
  Plan pl;
  pl.add(size_t(n) * l); pl.add(ll); pl.add(ll); pl.add(ll); pl.add(size_t(2) * l);
  pl.add(wsb / 8 + 1);
  for (int i = 0; i < 2; ++i) pl.add(ll);   // on-chip solver spill copy (l > 112)
  const size_t n16 = at ? form16_count(d) : 0, nsp = at ? form_split_doubles(c, d) : 0;
  pl.add(n16, sizeof(uint16_t)); pl.add(nsp);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  uint16_t* q16 = ctx_take<uint16_t>(c, n16);
  double* slices = ctx_take<double>(c, nsp);
  double* Z = ctx_take<double>(c, size_t(n) * l);
  double* W = ctx_take<double>(c, ll);
  double* Ue = ctx_take<double>(c, ll);
  double* Wk = ctx_take<double>(c, ll);
  double* w = ctx_take<double>(c, size_t(2) * l);
  double* s = w + l;
  double* ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  MB_CHECK(ctx_tic(c));
  // Z := A' Q   (gramian_former.hpp:101)
  if (at) MB_CHECK(form_product_bf16(c, d, *at, Qbar, Z, l, true, q16, slices));
  else MB_CHECK(dgemm(c, n, l, m, 1.0, ctr(Am), crow(Qbar, l), 0.0, drow(Z, l), GemmBatch(), ws));
  MB_CHECK(ctx_allreduce(c, Z, n * l));   // row blocks over ranks (row_block_gramian_former.hpp:111)
  MB_CHECK(ctx_toc(c));
  // W := Z' Z; eig(W) = W S W' (descending); S := sqrt(S)   (:108-115)
  MB_CHECK(dgemm(c, l, l, n, 1.0, cm(Z, 1, l), crow(Z, l), 0.0, drow(W, l), GemmBatch(), ws));
  MB_CHECK(launch_syev(c, l, 1, W, l, 0, w, Ue, 1));
  MB_CHECK(launch_sqrt_vec(c, l, w, s));
  MB_CHECK(ctx_toc(c));
  // U := Q W(:, 0:k); V := Z W(:, 0:k) diag(1/S)   (:123-128)
  if (U) MB_CHECK(dgemm(c, m, k, l, 1.0, crow(Qbar, l), crow(Ue, l), 0.0, drow(U, k), GemmBatch(), ws));
  if (V) {
    MB_CHECK(launch_scale_cols(c, l, k, Ue, l, s, 0, Wk, k));
    MB_CHECK(dgemm(c, n, k, l, 1.0, crow(Z, l), crow(Wk, k), 0.0, drow(V, k), GemmBatch(), ws));
  }
  if (S) MB_CHECK_CUDA(cudaMemcpyAsync(S, s, size_t(k) * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  MB_CHECK(ctx_toc(c));
  return MCNLA_B200_OK;
}

int run_form(Context* c, const Dims& d, int kind, const double* A, int layout, int64_t lda, const double* Qbar,
             double* S, double* U, double* V, const AtParts* at = nullptr) {
  // the precision form (at) reads the BF16 parts of A' instead of A
  if (!Qbar || (!A && !at)) return MCNLA_B200_ERR_ARG;
  if (layout != MCNLA_B200_ROW_MAJOR && layout != MCNLA_B200_COL_MAJOR) return MCNLA_B200_ERR_ARG;
  if (A && (layout == MCNLA_B200_ROW_MAJOR ? lda < d.n : lda < d.m)) return MCNLA_B200_ERR_SHAPE;
  if (d.k > d.l) return MCNLA_B200_ERR_SHAPE;
  const CMat Am = layout == MCNLA_B200_ROW_MAJOR ? crow(A, lda) : ccol(A, lda);
  switch (kind) {
    case MCNLA_B200_SVD_FORMER: return run_form_svd(c, d, Am, Qbar, S, U, V, at);
    case MCNLA_B200_GRAMIAN_FORMER:
    case MCNLA_B200_ROW_BLOCK_GRAMIAN_FORMER:
    case MCNLA_B200_COL_BLOCK_GRAMIAN_FORMER: return run_form_gramian(c, d, Am, Qbar, S, U, V, at);
    default: return MCNLA_B200_ERR_ARG;
  }
}

int run_isvd(Context* c, const Dims& d, int integrator, int former, const double* A, int layout, int64_t lda,
             const double* omega_in, uint64_t seed, int maxit, double tol, double* S, double* U, double* V,
             int* iters, char* pbase) {
  // pipeline buffers live in the pipeline arena (after whatever the caller put there)
  auto take = [&](size_t count) {
    double* p = reinterpret_cast<double*>(pbase);
    pbase += arena_bytes_for(count, sizeof(double));
    return p;
  };
  double* Q = take(size_t(d.m) * d.L);
  double* Qbar = take(size_t(d.m) * d.l);
  double* omega = take(size_t(d.n) * d.L);
  if (!omega_in) {
    MB_CHECK(launch_gaussian(c, seed, int64_t(d.n) * d.L, omega));
  } else {
    omega = const_cast<double*>(omega_in);   // read only: the sketch runs without power iterations
  }
  MB_CHECK(run_sketch(c, d, A, layout, lda, omega, 0, Q, false));
  MB_CHECK(run_orthogonalize(c, d, Q));
  MB_CHECK(run_integrate(c, d, integrator, Q, maxit, tol, Qbar, iters));
  MB_CHECK(run_form(c, d, former, A, layout, lda, Qbar, S, U, V));
  return MCNLA_B200_OK;
}

// Host-buffer solve with A streamed in: the row-major host A is copied to the
// device in row blocks on the context's copy stream, and the sketch GEMM of
// each block (Q rows := A rows * Omega, gaussian_projection_sketcher.hpp:96)
// starts as soon as its block has landed, so the copy of A hides behind the
// sketch.  Each block's GEMM uses the split-K count of the whole product, so
// every element of Q equals the whole-product GEMM's.
// Row blocks of a sketch streamed from host memory: at least 128 rows, about
// 1 GB at most, at least four blocks, and a first block of about 128 MB so the
// first GEMM starts early; each block's GEMM uses the split-K count of the
// whole product, so every row of the result is the device-resident sketch's
// bit for bit whatever the block boundaries.
struct RowBlocks {
  int64_t rows_per;   // rows of every block after the first (the largest block)
  int64_t first;      // rows of the first block
  int nblocks;
  int splits;
  int64_t start(int b) const { return b == 0 ? 0 : first + int64_t(b - 1) * rows_per; }
  int64_t rows(int b, int64_t m) const { return std::min<int64_t>(b == 0 ? first : rows_per, m - start(b)); }
};

RowBlocks stream_blocks(Context* c, const Dims& d) {
  const size_t row_bytes = size_t(d.n) * sizeof(double);
  RowBlocks rb;
  rb.rows_per = std::max<int64_t>(128, std::min<int64_t>(int64_t((size_t(1) << 30) / row_bytes), cdiv(d.m, 4)));
  rb.first = std::min<int64_t>(rb.rows_per, std::max<int64_t>(128, int64_t((size_t(128) << 20) / row_bytes)));
  rb.nblocks = 1 + int(cdiv(std::max<int64_t>(0, d.m - rb.first), rb.rows_per));
  rb.splits = dgemm_heuristic_splits(c, d.m, d.L, d.n, 1);
  return rb;
}

// The common part of the streamed sketches: the GEMM workspace, the copy
// stream, one event per block (plus one ordering the copies after the work
// already queued on the compute stream) and Omega copied ahead of the blocks.
struct StreamSetup {
  std::vector<cudaEvent_t> ev;
  double* ws = nullptr;
  ~StreamSetup() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
};

int stream_setup(Context* c, const Dims& d, const RowBlocks& rb, const double* omega_host, double* omega,
                 StreamSetup& st) {
  const size_t wsb = rb.splits > 1 ? size_t(rb.splits) * rb.rows_per * d.L * sizeof(double) : 0;
  Plan pl;
  pl.add(wsb / 8 + 1);
  MB_CHECK(ctx_reserve(c, pl.bytes));
  st.ws = take_ws(c, wsb);
  MB_CHECK(check_arena(c));
  if (!c->copy_stream) MB_CHECK_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  st.ev.assign(size_t(rb.nblocks) + 1, nullptr);
  for (auto& e : st.ev) MB_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  // the copies start after the work already queued on the compute stream (which may still use the buffers)
  MB_CHECK_CUDA(cudaEventRecord(st.ev[rb.nblocks], c->stream));
  MB_CHECK_CUDA(cudaStreamWaitEvent(c->copy_stream, st.ev[rb.nblocks], 0));
  MB_CHECK_CUDA(cudaMemcpyAsync(omega, omega_host, size_t(d.n) * d.L * sizeof(double), cudaMemcpyHostToDevice,
                                c->copy_stream));
  MB_CHECK(ctx_tic(c));
  MB_CHECK(ctx_toc(c));   // "random generating" part: Omega is given
  return MCNLA_B200_OK;
}

int sketch_block(Context* c, const Dims& d, const RowBlocks& rb, const StreamSetup& st, int b, const double* A,
                 const double* omega, double* Q) {
  const int64_t r0 = rb.start(b), rows = rb.rows(b, d.m);
  MB_CHECK_CUDA(cudaStreamWaitEvent(c->stream, st.ev[b], 0));
  return dgemm(c, rows, d.L, d.n, 1.0, crow(A + r0 * d.n, d.n), crow(omega, d.L), 0.0, drow(Q + r0 * d.L, d.L),
               GemmBatch(), st.ws, rb.splits);
}

int run_sketch_streamed(Context* c, const Dims& d, const double* A_host, double* A, const double* omega_host,
                        double* omega, double* Q) {
  const RowBlocks rb = stream_blocks(c, d);
  StreamSetup st;
  MB_CHECK(stream_setup(c, d, rb, omega_host, omega, st));
  for (int b = 0; b < rb.nblocks; ++b) {
    const int64_t r0 = rb.start(b), rows = rb.rows(b, d.m);
    MB_CHECK_CUDA(cudaMemcpyAsync(A + r0 * d.n, A_host + r0 * d.n, size_t(rows) * d.n * sizeof(double),
                                  cudaMemcpyHostToDevice, c->copy_stream));
    MB_CHECK_CUDA(cudaEventRecord(st.ev[b], c->copy_stream));
  }
  for (int b = 0; b < rb.nblocks; ++b) MB_CHECK(sketch_block(c, d, rb, st, b, A, omega, Q));
  MB_CHECK(ctx_toc(c));
  return MCNLA_B200_OK;
}

// Streamed ingest: the caller's reader fills pinned staging buffers (two,
// alternating) block by block; block b's copy and GEMM run on the device while
// the reader fills block b + 1.
int run_sketch_ingest(Context* c, const Dims& d, mcnla_b200_read_rows_fn read_rows, void* user, double* A,
                      const double* omega_host, double* omega, double* Q) {
  const RowBlocks rb = stream_blocks(c, d);
  const size_t stage = size_t(rb.rows_per) * d.n * sizeof(double);
  if (c->stage_host_bytes < stage) {
    MB_CHECK_CUDA(cudaStreamSynchronize(c->copy_stream ? c->copy_stream : c->stream));
    for (auto& h : c->stage_host) {
      if (h) cudaFreeHost(h);
      h = nullptr;
    }
    c->stage_host_bytes = 0;
    for (auto& h : c->stage_host) MB_CHECK_CUDA(cudaHostAlloc(&h, stage, cudaHostAllocDefault));
    c->stage_host_bytes = stage;
  }
  StreamSetup st;
  MB_CHECK(stream_setup(c, d, rb, omega_host, omega, st));
  for (int b = 0; b < rb.nblocks; ++b) {
    const int64_t r0 = rb.start(b), rows = rb.rows(b, d.m);
    double* buf = static_cast<double*>(c->stage_host[b & 1]);
    if (b >= 2) MB_CHECK_CUDA(cudaEventSynchronize(st.ev[b - 2]));   // the buffer's last copy has landed
    if (read_rows(user, r0, rows, buf) != 0) {
      cudaStreamSynchronize(c->copy_stream);
      set_last_message("the row reader returned an error for rows " + std::to_string(r0) + " .. " +
                       std::to_string(r0 + rows));
      return MCNLA_B200_ERR_ARG;
    }
    MB_CHECK_CUDA(cudaMemcpyAsync(A + r0 * d.n, buf, size_t(rows) * d.n * sizeof(double), cudaMemcpyHostToDevice,
                                  c->copy_stream));
    MB_CHECK_CUDA(cudaEventRecord(st.ev[b], c->copy_stream));
    MB_CHECK(sketch_block(c, d, rb, st, b, A, omega, Q));
  }
  MB_CHECK(ctx_toc(c));
  // the staging buffers are free again once the last copies have landed
  MB_CHECK_CUDA(cudaStreamSynchronize(c->copy_stream));
  return MCNLA_B200_OK;
}

// Mixed solve: Omega drawn in BF16, sketch on tcgen05, FP64 afterwards.
int run_isvd_mixed(Context* c, const Dims& d, int integrator, int former, const double* A, int layout, int64_t lda,
                   const uint16_t* a_hi, const uint16_t* a_lo, const uint16_t* a_lo2, int64_t lda16,
                   const AtParts* at, uint64_t seed, int maxit, double tol, double* S, double* U, double* V,
                   int* iters, char* pbase) {
  auto take = [&](size_t bytes) {
    char* p = pbase;
    pbase += (bytes + 511) & ~size_t(511);
    return p;
  };
  const int64_t ldo = (d.n + 7) & ~int64_t(7);
  double* Q = reinterpret_cast<double*>(take(size_t(d.m) * d.L * 8));
  double* Qbar = reinterpret_cast<double*>(take(size_t(d.m) * d.l * 8));
  uint16_t* omega_t = reinterpret_cast<uint16_t*>(take(size_t(d.L) * ldo * 2));
  MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
  MB_CHECK(ctx_tic(c));
  MB_CHECK(launch_gaussian_bf16(c, seed, d.n, d.L, omega_t, ldo, nullptr));
  MB_CHECK(ctx_toc(c));
  MB_CHECK(bf16_gemm(c, d.m, d.L, d.n, a_hi, a_lo, a_lo2, lda16, omega_t, ldo, Q, d.L, true));
  MB_CHECK(ctx_toc(c));
  MB_CHECK(run_orthogonalize(c, d, Q));
  // The Gramian integrators' Bs (and the loop's Bs Bc) from BF16 parts (the
  // precision form) only where the FP64 product is long: below ~1e11 flops it
  // takes a few milliseconds at most, less than the split and the FP64
  // re-orthonormalization the BF16 form needs afterwards.
  const bool gramian = integrator == MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO ||
                       integrator == MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN;
  double m_all = 0.0;   // the rows of all ranks: every rank takes the same path
  MB_CHECK(ctx_sum_host(c, double(d.m), &m_all));
  const bool bf16_gramian = gramian && double(d.L) * double(d.L) * m_all >= kMixedGramianMinFlops;
  {
    struct Mixed { Context* c; Mixed(Context* x, bool on) : c(x) { c->mixed_gramian = on; }
                   ~Mixed() { c->mixed_gramian = false; } } mixed(c, bf16_gramian);
    MB_CHECK(run_integrate(c, d, integrator, Q, maxit, tol, Qbar, iters));
  }
  if (bf16_gramian) {
    // Bs carried the BF16 rounding of Qs into the iterates: one FP64 Gramian
    // pass (Qbar := Qbar V S^(-1/2), an orthonormal basis of the same span)
    // brings ||Qbar' Qbar - I|| back to FP64 rounding
    Dims one = d;
    one.N = 1;
    one.L = d.l;
    MB_CHECK(run_orthogonalize(c, one, Qbar));
  }
  MB_CHECK(run_form(c, d, former, A, layout, lda, Qbar, S, U, V, at));
  MB_CHECK(ctx_sync_scalars(c));
  if (c->scal_host->status) return c->scal_host->status;
  return MCNLA_B200_OK;
}

size_t pipeline_bytes_mixed(const Dims& d) {
  const int64_t ldo = (d.n + 7) & ~int64_t(7);
  auto r = [](size_t b) { return (b + 511) & ~size_t(511); };
  return r(size_t(d.m) * d.L * 8) + r(size_t(d.m) * d.l * 8) + r(size_t(d.L) * ldo * 2);
}

size_t pipeline_bytes(const Dims& d) {
  return arena_bytes_for(size_t(d.m) * d.L, 8) + arena_bytes_for(size_t(d.m) * d.l, 8) +
         arena_bytes_for(size_t(d.n) * d.L, 8);
}

// Workspace bytes each stage will ask for (for mcnla_b200_initialize).
size_t stage_bytes_upper(Context* c, const Dims& d) {
  const int64_t m = d.m, n = d.n, L = d.L, l = d.l;
  size_t b = 0;
  b = std::max(b, size_t(m) * L * 8 + 5 * size_t(l) * l * d.N * 8 + gemm_ws(c, {{l, l, m, d.N}, {m, l, l, d.N}}));
  b = std::max(b, size_t(L) * L * 8 + 8 * size_t(L) * 3 * l * 8 + 4 * size_t(m) * 2 * l * 8 +
                      gemm_ws(c, {{L, L, m, 1}, {L, l, m, 1}, {m, l, L, 1}, {l, 2 * l, L, 1}}));
  b = std::max(b, 3 * size_t(l) * n * 8 + size_t(n) * l * 8 + gemm_ws(c, {{l, n, m, 1}, {n, l, m, 1}, {l, l, n, 1}}));
  return b + (64 << 20);
}

}  // namespace

// ---------------------------------------------------------------------------
// Batched and served problems (mcnla_b200_problem): the whole solve of one
// problem on a worker, and the grouped batch
// ---------------------------------------------------------------------------
namespace {

__global__ void k_f32_to_f64(const float* src, int64_t rows, int64_t cols, int64_t lds, double* dst, int64_t ldd) {
  const int64_t total = rows * cols;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols, cc = e % cols;
    dst[r * ldd + cc] = double(src[r * lds + cc]);
  }
}

// Grows a stream-ordered device buffer to at least `need` bytes.
int grow(Context* c, void** p, size_t* have, size_t need) {
  if (need <= *have) return MCNLA_B200_OK;
  if (*p) MB_CHECK_CUDA(cudaFreeAsync(*p, c->stream));
  *p = nullptr;
  *have = 0;
  const cudaError_t e = cudaMallocAsync(p, need, c->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_last_cuda_error(e, "problem scratch cudaMalloc", __FILE__, __LINE__);
    *p = nullptr;
    return MCNLA_B200_ERR_NOMEM;
  }
  *have = need;
  return MCNLA_B200_OK;
}

bool problem_mixed(const mcnla_b200_problem& p) {
  return p.precision == MCNLA_B200_PRECISION_MIXED || p.precision == MCNLA_B200_PRECISION_MIXED3;
}

int problem_check(const mcnla_b200_problem& p, Dims& d) {
  MB_CHECK(get_dims(&p.params, d));
  if (p.precision < MCNLA_B200_PRECISION_FP64 || p.precision > MCNLA_B200_PRECISION_MIXED3) return MCNLA_B200_ERR_ARG;
  if (!p.A && !p.A32 && !(problem_mixed(p) && p.a_hi && p.at_hi)) return MCNLA_B200_ERR_ARG;
  if (p.a_layout != MCNLA_B200_ROW_MAJOR && p.a_layout != MCNLA_B200_COL_MAJOR) return MCNLA_B200_ERR_ARG;
  return MCNLA_B200_OK;
}

}  // namespace

void solve_scratch_free(Context* c, SolveScratch& s) {
  if (s.a64) cudaFreeAsync(s.a64, c->stream);
  if (s.split) cudaFreeAsync(s.split, c->stream);
  if (s.tsplit) cudaFreeAsync(s.tsplit, c->stream);
  s = SolveScratch();
}

// A in FP64: the caller's, or an FP32 A converted into scratch.
int problem_a64(Context* c, const mcnla_b200_problem& p, SolveScratch& s, const double** A, int64_t* lda) {
  if (p.A) {
    *A = p.A;
    *lda = p.lda;
    return MCNLA_B200_OK;
  }
  if (!p.A32) return MCNLA_B200_ERR_ARG;
  const int64_t m = p.params.nrow, n = p.params.ncol;
  MB_CHECK(grow(c, reinterpret_cast<void**>(&s.a64), &s.a64_bytes, size_t(m) * n * sizeof(double)));
  const bool row = p.a_layout == MCNLA_B200_ROW_MAJOR;
  const int64_t rows = row ? m : n, cols = row ? n : m;
  const int blocks = int(std::min<int64_t>(cdiv(rows * cols, 256), int64_t(c->num_sms) * 16));
  k_f32_to_f64<<<blocks, 256, 0, c->stream>>>(p.A32, rows, cols, p.lda, s.a64, cols);
  MB_CHECK_CUDA(cudaGetLastError());
  c->kernels_launched++;
  *A = s.a64;
  *lda = cols;
  return MCNLA_B200_OK;
}

// BF16 parts of A (row-major m x n) for the mixed sketch: the caller's, or split into scratch.
int problem_parts(Context* c, const mcnla_b200_problem& p, SolveScratch& s, const uint16_t** part, int64_t* ld) {
  const int nparts = p.precision == MCNLA_B200_PRECISION_MIXED3 ? 3 : 2;
  if (p.a_hi) {
    part[0] = p.a_hi;
    part[1] = p.a_lo;
    part[2] = nparts == 3 ? p.a_lo2 : nullptr;
    *ld = p.lda16;
    if (!p.a_lo || (nparts == 3 && !p.a_lo2)) return MCNLA_B200_ERR_ARG;
    return MCNLA_B200_OK;
  }
  const int64_t m = p.params.nrow, n = p.params.ncol, ldo = (n + 7) & ~int64_t(7);
  MB_CHECK(grow(c, reinterpret_cast<void**>(&s.split), &s.split_bytes, nparts * size_t(m) * ldo * sizeof(uint16_t)));
  part[0] = s.split;
  part[1] = s.split + size_t(m) * ldo;
  part[2] = nparts == 3 ? s.split + 2 * size_t(m) * ldo : nullptr;
  uint16_t* w[3] = {s.split, s.split + size_t(m) * ldo, nparts == 3 ? s.split + 2 * size_t(m) * ldo : nullptr};
  if (p.A32) MB_CHECK(launch_split_bf16_f32(c, p.A32, p.a_layout, p.lda, m, n, w[0], w[1], w[2], ldo));
  else MB_CHECK(launch_split_bf16(c, p.A, p.a_layout, p.lda, m, n, w[0], w[1], w[2], ldo));
  *ld = ldo;
  return MCNLA_B200_OK;
}

// Three BF16 parts of A' (n x m) for the precision former: A read with the other layout.
int problem_tparts(Context* c, const mcnla_b200_problem& p, SolveScratch& s, AtParts* at) {
  if (p.at_hi) {
    if (!p.at_lo || !p.at_lo2) return MCNLA_B200_ERR_ARG;
    at->hi = p.at_hi;
    at->lo = p.at_lo;
    at->lo2 = p.at_lo2;
    at->ld = p.ldat16;
    return MCNLA_B200_OK;
  }
  const int64_t m = p.params.nrow, n = p.params.ncol, ldo = (m + 7) & ~int64_t(7);
  MB_CHECK(grow(c, reinterpret_cast<void**>(&s.tsplit), &s.tsplit_bytes, 3 * size_t(n) * ldo * sizeof(uint16_t)));
  uint16_t* w[3] = {s.tsplit, s.tsplit + size_t(n) * ldo, s.tsplit + 2 * size_t(n) * ldo};
  const int tl = p.a_layout == MCNLA_B200_ROW_MAJOR ? MCNLA_B200_COL_MAJOR : MCNLA_B200_ROW_MAJOR;
  if (p.A32) MB_CHECK(launch_split_bf16_f32(c, p.A32, tl, p.lda, n, m, w[0], w[1], w[2], ldo));
  else MB_CHECK(launch_split_bf16(c, p.A, tl, p.lda, n, m, w[0], w[1], w[2], ldo));
  at->hi = w[0];
  at->lo = w[1];
  at->lo2 = w[2];
  at->ld = ldo;
  return MCNLA_B200_OK;
}

size_t problem_scratch_bytes(const mcnla_b200_problem& p) {
  const int64_t m = p.params.nrow, n = p.params.ncol;
  if (!problem_mixed(p)) return p.A ? 0 : size_t(m) * n * 8;
  const int nparts = p.precision == MCNLA_B200_PRECISION_MIXED3 ? 3 : 2;
  size_t b = 0;
  if (!p.a_hi) b += nparts * size_t(m) * ((n + 7) & ~int64_t(7)) * 2;
  if (!p.at_hi) b += 3 * size_t(n) * ((m + 7) & ~int64_t(7)) * 2;
  return b;
}

// One whole solve on a worker: the plain path, or the precision form with
// the sketch and the former on tcgen05 (mcnla_b200_isvd / _isvd_mixed).
int solve_problem(Context* c, mcnla_b200_problem& p, SolveScratch& s) {
  Dims d;
  MB_CHECK(problem_check(p, d));
  if (!problem_mixed(p)) {
    const double* A = nullptr;
    int64_t lda = 0;
    MB_CHECK(problem_a64(c, p, s, &A, &lda));
    return mcnla_b200_isvd(static_cast<mcnla_b200_ctx*>(c), &p.params, p.integrator, p.former, A, p.a_layout, lda, nullptr, p.seed,
                           p.max_iteration, p.tolerance, p.S, p.U, p.V, &p.iteration);
  }
  const uint16_t* part[3];
  int64_t ld16 = 0;
  MB_CHECK(problem_parts(c, p, s, part, &ld16));
  AtParts at;
  MB_CHECK(problem_tparts(c, p, s, &at));
  return mcnla_b200_isvd_mixed(static_cast<mcnla_b200_ctx*>(c), &p.params, p.integrator, p.former, nullptr, MCNLA_B200_ROW_MAJOR, 0, part[0],
                               part[1], part[2], ld16, at.hi, at.lo, at.lo2, at.ld, p.seed, p.max_iteration,
                               p.tolerance, p.S, p.U, p.V, &p.iteration);
}

namespace {

// A problem of the grouped batch and its device state (carved from the wave arena).
struct GItem {
  mcnla_b200_problem* p = nullptr;
  Dims d;
  double* Q = nullptr;
  double* Qbar = nullptr;
  double* omega = nullptr;        // FP64 path
  uint16_t* omega_t = nullptr;    // mixed path (L x ldo BF16)
  GknBufs b;
  int it0 = 0, iters = 0, status = MCNLA_B200_OK;
  bool done = false;
  double seconds = 0.0;
};

size_t gitem_bytes(const Context* c, const Dims& d, bool mixed) {
  const int64_t ldo = (d.n + 7) & ~int64_t(7);
  return arena_bytes_for(size_t(d.m) * d.L, 8) + arena_bytes_for(size_t(d.m) * d.l, 8) +
         (mixed ? arena_bytes_for(size_t(d.L) * ldo, 2) : arena_bytes_for(size_t(d.n) * d.L, 8)) +
         gkn_state_bytes(c, d);
}

// A problem runs in the grouped batch when it uses the row-block Gramian KN
// integrator on the path whose iterations a single solve runs in one
// persistent kernel too (the default step method, N l <= 1536) with the FP64
// Gramian.  The grouped kernel sums each product in its own fixed order, so a
// batch result matches the single solve to rounding (same iteration count).
bool grouped_eligible(const Context* c, const mcnla_b200_problem& p) {
  Dims d;
  if (problem_check(p, d) != MCNLA_B200_OK) return false;
  if (p.integrator != MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO) return false;
  if (p.former < MCNLA_B200_SVD_FORMER || p.former > MCNLA_B200_COL_BLOCK_GRAMIAN_FORMER || d.k > d.l) return false;
  if (p.max_iteration < 0 || !(p.tolerance >= 0.0)) return false;
  if (c->kn_mode != MCNLA_B200_KN_AUTO || !gkn_grouped_fits(c, d.l, d.L) || !gkn_persistent_fits(c, d.l, d.L))
    return false;
  if (gkn_grouped_smem(c, d.l) == 0) return false;
  if (problem_mixed(p) && double(d.L) * double(d.L) * double(d.m) >= kMixedGramianMinFlops) return false;
  return true;
}

template <class F>
int parallel_for(int device, int workers, int n, F f) {
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  for (int w = 0; w < workers; ++w) {
    th.emplace_back([&, w] {
      cudaSetDevice(device);
      for (int i = next++; i < n; i = next++) f(w, i);
    });
  }
  for (auto& t : th) t.join();
  return MCNLA_B200_OK;
}

// Phase A of a grouped problem: Omega, the sketch, the orthogonalizer and the
// Gramian (the operations of mcnla_b200_isvd / _isvd_mixed up to the
// integrator's iterations).
int gitem_phase_a(Context* c, GItem& it, SolveScratch& s) {
  mcnla_b200_problem& p = *it.p;
  const Dims& d = it.d;
  if (!problem_mixed(p)) {
    const double* A = nullptr;
    int64_t lda = 0;
    MB_CHECK(problem_a64(c, p, s, &A, &lda));
    MB_CHECK(launch_gaussian(c, p.seed, int64_t(d.n) * d.L, it.omega));
    MB_CHECK(run_sketch(c, d, A, p.a_layout, lda, it.omega, 0, it.Q, false));
  } else {
    const uint16_t* part[3];
    int64_t ld16 = 0;
    MB_CHECK(problem_parts(c, p, s, part, &ld16));
    const int64_t ldo = (d.n + 7) & ~int64_t(7);
    MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
    MB_CHECK(launch_gaussian_bf16(c, p.seed, d.n, d.L, it.omega_t, ldo, nullptr));
    MB_CHECK(bf16_gemm(c, d.m, d.L, d.n, part[0], part[1], part[2], ld16, it.omega_t, ldo, it.Q, d.L, true));
  }
  MB_CHECK(run_orthogonalize(c, d, it.Q));
  MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
  const size_t wsb = gkn_ws_bytes(c, d);
  MB_CHECK(ctx_reserve(c, wsb + 512));
  double* ws = take_ws(c, wsb);
  MB_CHECK(gkn_prepare(c, d, it.Q, it.b, ws));
  MB_CHECK(ctx_sync_scalars(c));
  return c->scal_host->status;
}

// A declined iteration r on the launch-per-product path (the single solve's
// host step).  Sets it.done / it.iters, or it.it0 = r + 1.
int gitem_fallback(Context* c, GItem& it, int r) {
  const Dims& d = it.d;
  const size_t wsb = gkn_ws_bytes(c, d);
  MB_CHECK(ctx_reserve(c, wsb + 512));
  double* ws = take_ws(c, wsb);
  MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
  MB_CHECK_CUDA(cudaMemsetAsync(&c->scal->stop_it, 0x7f, sizeof(int), c->stream));
  {
    struct Reset { Context* c; ~Reset() { c->guard_stop = nullptr; c->guard_it = 0; } } reset{c};
    c->guard_stop = &c->scal->stop_it;
    c->guard_it = r;
    MB_CHECK(gkn_iteration(c, d, it.b, r, false, it.p->tolerance, ws));
  }
  MB_CHECK(ctx_sync_scalars(c));
  if (c->scal_host->status) return c->scal_host->status;
  if (c->scal_host->stop_it == r) {
    it.done = true;
    it.iters = r + 1;
  } else {
    it.it0 = r + 1;
    if (it.it0 >= it.p->max_iteration) {
      it.done = true;
      it.iters = it.p->max_iteration;
    }
  }
  return MCNLA_B200_OK;
}

// Phase C: Qbar and the former.
int gitem_phase_c(Context* c, GItem& it, SolveScratch& s) {
  mcnla_b200_problem& p = *it.p;
  const Dims& d = it.d;
  const size_t wsb = gkn_ws_bytes(c, d);
  MB_CHECK(ctx_reserve(c, wsb + 512));
  double* ws = take_ws(c, wsb);
  MB_CHECK_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
  MB_CHECK(gkn_finish(c, d, it.Q, it.b, it.iters, it.Qbar, ws));
  if (!problem_mixed(p)) {
    const double* A = nullptr;
    int64_t lda = 0;
    MB_CHECK(problem_a64(c, p, s, &A, &lda));
    MB_CHECK(run_form(c, d, p.former, A, p.a_layout, lda, it.Qbar, p.S, p.U, p.V));
  } else {
    AtParts at;
    MB_CHECK(problem_tparts(c, p, s, &at));
    MB_CHECK(run_form(c, d, p.former, nullptr, MCNLA_B200_ROW_MAJOR, 0, it.Qbar, p.S, p.U, p.V, &at));
  }
  MB_CHECK(ctx_sync_scalars(c));
  return c->scal_host->status;
}

using Clock = std::chrono::steady_clock;

// The grouped integrator over the wave's problems: per round one launch per
// cluster size (on the first workers' streams, side by side), then the
// declined iterations on the workers.
int grouped_rounds(int device, std::vector<Context*>& ctx, std::vector<GItem*>& items, double* t_kernel,
                   double* t_fallback, double* t_parts) {
  Context* c0 = ctx[0];
  const int n = int(items.size());
  if (n == 0) return MCNLA_B200_OK;
  constexpr int kClasses = 4;                        // clusters of 1, 2, 4, 8 CTAs
  auto cls = [](const GItem& it) {
    const int c = gkn_cluster_for(it.d.l, it.d.L);
    return c >= 8 ? 3 : (c >= 4 ? 2 : (c >= 2 ? 1 : 0));
  };
  size_t smem[kClasses] = {0, 0, 0, 0};
  for (auto* it : items) smem[cls(*it)] = std::max(smem[cls(*it)], gkn_grouped_smem(c0, it->d.l));
  GknJob* jobs_dev = nullptr;
  MB_CHECK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&jobs_dev), sizeof(GknJob) * n + 256, c0->stream));
  int* next_dev = reinterpret_cast<int*>(reinterpret_cast<char*>(jobs_dev) + sizeof(GknJob) * n);
  MB_CHECK_CUDA(cudaStreamSynchronize(c0->stream));
  struct Free { Context* c; void* p; ~Free() { cudaFreeAsync(p, c->stream); cudaStreamSynchronize(c->stream); } }
      release{c0, jobs_dev};
  std::vector<GknJob> jobs;
  std::vector<GItem*> pending;
  for (auto* it : items)
    if (!it->done && it->status == MCNLA_B200_OK) pending.push_back(it);
  while (!pending.empty()) {
    // jobs ordered by class (largest first), each class a contiguous range
    std::stable_sort(pending.begin(), pending.end(), [&](const GItem* a, const GItem* b) { return cls(*a) > cls(*b); });
    const int np = int(pending.size());
    jobs.assign(size_t(np), GknJob());
    int first[kClasses + 1] = {0, 0, 0, 0, 0};
    for (int i = 0; i < np; ++i) {
      GItem& it = *pending[size_t(i)];
      jobs[size_t(i)] = gkn_job(c0, it.d, it.b, it.it0, it.p->max_iteration, it.p->tolerance);
    }
    for (int k = kClasses - 1, i = 0; k >= 0; --k) {
      first[k + 1] = i;
      while (i < np && cls(*pending[size_t(i)]) == k) ++i;
      first[k] = i;
    }
    const auto tk = Clock::now();
    MB_CHECK_CUDA(cudaMemcpyAsync(jobs_dev, jobs.data(), sizeof(GknJob) * np, cudaMemcpyHostToDevice, c0->stream));
    MB_CHECK_CUDA(cudaStreamSynchronize(c0->stream));
    int lane = 0;
    for (int k = kClasses - 1; k >= 0; --k) {
      const int b0 = first[k + 1], cnt = first[k] - first[k + 1];
      if (cnt == 0) continue;
      Context* c = ctx[size_t(lane % int(ctx.size()))];
      MB_CHECK(launch_gkn_grouped(c, jobs_dev + b0, cnt, next_dev + k, smem[k], 1 << k));
      ++lane;
    }
    for (int w = 0; w < std::min(lane, int(ctx.size())); ++w) MB_CHECK_CUDA(cudaStreamSynchronize(ctx[size_t(w)]->stream));
    MB_CHECK_CUDA(cudaMemcpyAsync(jobs.data(), jobs_dev, sizeof(GknJob) * np, cudaMemcpyDeviceToHost, c0->stream));
    MB_CHECK_CUDA(cudaStreamSynchronize(c0->stream));
    *t_kernel += std::chrono::duration<double>(Clock::now() - tk).count();
    const auto tf0 = Clock::now();
    std::vector<std::pair<GItem*, int>> fallback;
    for (int i = 0; i < np; ++i) {
      GItem& it = *pending[size_t(i)];
      const GknJob& j = jobs[size_t(i)];
      it.seconds += double(j.ns) * 1e-9;
      for (int q = 0; q < 4; ++q) t_parts[q] += double(j.phase_ns[q]) * 1e-9;
      if (j.stop_it != INT_MAX) {
        it.done = true;
        it.iters = j.stop_it + 1;
      } else if (j.resume_it >= 0) {
        fallback.emplace_back(&it, j.resume_it);
      } else {
        it.done = true;
        it.iters = it.p->max_iteration;
      }
    }
    parallel_for(device, int(ctx.size()), int(fallback.size()), [&](int w, int i) {
      GItem& it = *fallback[size_t(i)].first;
      const auto tf = Clock::now();
      const int st = gitem_fallback(ctx[size_t(w)], it, fallback[size_t(i)].second);
      it.seconds += std::chrono::duration<double>(Clock::now() - tf).count();
      if (st != MCNLA_B200_OK) {
        it.status = st;
        it.done = true;
      }
    });
    *t_fallback += std::chrono::duration<double>(Clock::now() - tf0).count();
    pending.clear();
    for (auto* it : items)
      if (!it->done && it->status == MCNLA_B200_OK) pending.push_back(it);
  }
  return MCNLA_B200_OK;
}

}  // namespace

// Host seconds of the phases of the last grouped batch (mcnla_b200_batched_times).
std::mutex g_batch_times_mu;
double g_batch_times[kBatchPhases] = {};

// The grouped batch (mcnla_b200_isvd_batched): problems the grouped kernel
// takes (grouped_eligible) run in waves through phases A / grouped rounds / C
// on `workers` contexts; the others run whole solves through a worker pool.
int batched_solve(int device, mcnla_b200_problem* problems, int count, int workers, int64_t budget) {
  if (count < 0 || (count > 0 && !problems) || workers < 1 || workers > 256 || budget <= 0) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(device));
  const auto t0 = Clock::now();
  double phase[kBatchPhases] = {};
  auto since = [](Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); };
  std::vector<Context*> ctx;
  std::vector<cudaStream_t> streams;
  std::vector<SolveScratch> scratch(static_cast<size_t>(workers));
  struct Cleanup {
    std::vector<Context*>& ctx;
    std::vector<cudaStream_t>& streams;
    std::vector<SolveScratch>& scratch;
    ~Cleanup() {
      for (size_t i = 0; i < ctx.size(); ++i) {
        solve_scratch_free(ctx[i], scratch[i]);
        mcnla_b200_destroy(static_cast<mcnla_b200_ctx*>(ctx[i]));
      }
      for (auto s : streams) cudaStreamDestroy(s);
    }
  } cleanup{ctx, streams, scratch};
  for (int w = 0; w < workers; ++w) {
    cudaStream_t st = nullptr;
    MB_CHECK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    streams.push_back(st);
    mcnla_b200_ctx* c = nullptr;
    MB_CHECK(mcnla_b200_create(&c, device, st));
    ctx.push_back(c);
  }
  for (int i = 0; i < count; ++i) {
    problems[i].status = -1;
    problems[i].iteration = 0;
    problems[i].seconds = 0;
    problems[i].latency = 0;
  }
  // ---- partition; grouped problems largest first (the work queue's order)
  std::vector<GItem> items;
  std::vector<int> others;
  for (int i = 0; i < count; ++i) {
    if (grouped_eligible(ctx[0], problems[i])) {
      GItem it;
      it.p = &problems[i];
      problem_check(problems[i], it.d);
      items.push_back(it);
    } else {
      others.push_back(i);
    }
  }
  auto cost = [](const GItem& it) { return double(it.d.L) * double(it.d.L) * double(it.d.l); };
  std::stable_sort(items.begin(), items.end(), [&](const GItem& a, const GItem& b) { return cost(a) > cost(b); });
  // ---- waves within the budget (besides the workers' own workspaces and scratch)
  size_t worker_bytes = 0;
  for (auto& it : items) {
    worker_bytes = std::max(worker_bytes, problem_scratch_bytes(*it.p) + size_t(it.d.m) * it.d.L * 8 +
                                              gkn_ws_bytes(ctx[0], it.d) + (size_t(64) << 20));
  }
  const int64_t wave_cap = std::max<int64_t>(1, budget - int64_t(worker_bytes) * workers);
  size_t pos = 0;
  while (pos < items.size()) {
    size_t end = pos, bytes = 0;
    while (end < items.size()) {
      const size_t b = gitem_bytes(ctx[0], items[end].d, problem_mixed(*items[end].p));
      if (end > pos && int64_t(bytes + b) > wave_cap) break;
      bytes += b;
      ++end;
    }
    void* arena = nullptr;
    MB_CHECK_CUDA(cudaMallocAsync(&arena, bytes + 4096, ctx[0]->stream));
    MB_CHECK_CUDA(cudaStreamSynchronize(ctx[0]->stream));
    struct Arena { Context* c; void* p; ~Arena() { cudaFreeAsync(p, c->stream); cudaStreamSynchronize(c->stream); } }
        wave_arena{ctx[0], arena};
    char* base = static_cast<char*>(arena);
    size_t top = 0;
    auto take = [&](size_t count_, size_t elem) -> char* {
      const size_t off = (top + 255) & ~size_t(255);
      top = off + count_ * elem + 256;
      return base + off;
    };
    std::vector<GItem*> wave;
    for (size_t i = pos; i < end; ++i) {
      GItem& it = items[i];
      const int64_t ldo = (it.d.n + 7) & ~int64_t(7);
      it.Q = reinterpret_cast<double*>(take(size_t(it.d.m) * it.d.L, 8));
      it.Qbar = reinterpret_cast<double*>(take(size_t(it.d.m) * it.d.l, 8));
      if (problem_mixed(*it.p)) it.omega_t = reinterpret_cast<uint16_t*>(take(size_t(it.d.L) * ldo, 2));
      else it.omega = reinterpret_cast<double*>(take(size_t(it.d.n) * it.d.L, 8));
      gkn_carve(ctx[0], it.d, take, it.b);
      wave.push_back(&it);
    }
    auto tp = Clock::now();
    parallel_for(device, workers, int(wave.size()), [&](int w, int i) {
      GItem& it = *wave[size_t(i)];
      const auto ta = Clock::now();
      it.status = gitem_phase_a(ctx[size_t(w)], it, scratch[size_t(w)]);
      it.seconds += std::chrono::duration<double>(Clock::now() - ta).count();
    });
    phase[0] += since(tp);
    MB_CHECK(grouped_rounds(device, ctx, wave, &phase[1], &phase[2], &phase[5]));
    tp = Clock::now();
    parallel_for(device, workers, int(wave.size()), [&](int w, int i) {
      GItem& it = *wave[size_t(i)];
      const auto tc = Clock::now();
      if (it.status == MCNLA_B200_OK) it.status = gitem_phase_c(ctx[size_t(w)], it, scratch[size_t(w)]);
      it.seconds += std::chrono::duration<double>(Clock::now() - tc).count();
      mcnla_b200_problem& p = *it.p;
      p.status = it.status;
      p.iteration = it.iters;
      p.seconds = it.seconds;
      p.latency = std::chrono::duration<double>(Clock::now() - t0).count();
    });
    phase[3] += since(tp);
    pos = end;
  }
  // ---- the rest: whole solves on the workers
  const auto to = Clock::now();
  parallel_for(device, workers, int(others.size()), [&](int w, int i) {
    mcnla_b200_problem& p = problems[others[size_t(i)]];
    Context* c = ctx[size_t(w)];
    const auto ts = Clock::now();
    int st = solve_problem(c, p, scratch[size_t(w)]);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess && st == MCNLA_B200_OK) st = MCNLA_B200_ERR_CUDA;
    p.status = st;
    p.seconds = std::chrono::duration<double>(Clock::now() - ts).count();
    p.latency = std::chrono::duration<double>(Clock::now() - t0).count();
  });
  phase[4] = since(to);
  {
    std::lock_guard<std::mutex> lock(g_batch_times_mu);
    for (int i = 0; i < kBatchPhases; ++i) g_batch_times[i] = phase[i];
  }
  int first = MCNLA_B200_OK;
  for (int i = 0; i < count; ++i)
    if (problems[i].status != MCNLA_B200_OK && first == MCNLA_B200_OK) first = problems[i].status;
  return first;
}

int batched_times(double* seconds, int capacity) {
  std::lock_guard<std::mutex> lock(g_batch_times_mu);
  const int n = std::min(capacity, kBatchPhases);
  for (int i = 0; i < n; ++i) seconds[i] = g_batch_times[i];
  return kBatchPhases;
}

}  // namespace mb

using mb::Context;
using mb::Dims;

extern "C" {

int mcnla_b200_initialize(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former) {
  if (!ctx) return MCNLA_B200_ERR_ARG;
  (void)integrator; (void)former;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK(mb::ctx_reserve(ctx, mb::stage_bytes_upper(ctx, d)));
  return MCNLA_B200_OK;
}

int mcnla_b200_sketch(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, const double* A, int a_layout,
                      int64_t lda, double* omega, int exponent, double* Q) {
  if (!ctx || !A || !omega || !Q) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  return mb::run_sketch(ctx, d, A, a_layout, lda, omega, exponent, Q, false);
}

int mcnla_b200_gaussian(mcnla_b200_ctx* ctx, uint64_t seed, int64_t count, double* out) {
  if (!ctx || (!out && count > 0) || count < 0) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  return mb::launch_gaussian(ctx, seed, count, out);
}

int mcnla_b200_orthogonalize(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, double* Q) {
  if (!ctx || !Q) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  return mb::run_orthogonalize(ctx, d, Q);
}

int mcnla_b200_integrate(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int kind, const double* Q,
                         int max_iteration, double tolerance, double* Qbar, int* iteration) {
  if (!ctx) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  return mb::run_integrate(ctx, d, kind, Q, max_iteration, tolerance, Qbar, iteration);
}

int mcnla_b200_form(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int kind, const double* A, int a_layout,
                    int64_t lda, const double* Qbar, double* S, double* U, double* V) {
  if (!ctx) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  return mb::run_form(ctx, d, kind, A, a_layout, lda, Qbar, S, U, V);
}

int mcnla_b200_isvd(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former,
                    const double* A, int a_layout, int64_t lda, const double* omega, uint64_t seed,
                    int max_iteration, double tolerance, double* S, double* U, double* V, int* iteration) {
  if (!ctx || !A || !iteration) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK(mb::ctx_reserve_pipeline(ctx, mb::pipeline_bytes(d)));
  return mb::run_isvd(ctx, d, integrator, former, A, a_layout, lda, omega, seed, max_iteration, tolerance, S, U, V,
                      iteration, static_cast<char*>(ctx->parena));
}

int mcnla_b200_isvd_host(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former,
                         const double* A_host, int a_layout, const double* omega_host, int max_iteration,
                         double tolerance, double* S_host, double* U_host, double* V_host, int* iteration) {
  if (!ctx || !A_host || !omega_host || !iteration) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  const size_t a_elems = size_t(d.m) * d.n;
  const size_t io = mb::arena_bytes_for(a_elems, 8) + mb::arena_bytes_for(size_t(d.k), 8) +
                    mb::arena_bytes_for(size_t(d.m) * d.k, 8) + mb::arena_bytes_for(size_t(d.n) * d.k, 8);
  MB_CHECK(mb::ctx_reserve_pipeline(ctx, io + mb::pipeline_bytes(d)));
  char* base = static_cast<char*>(ctx->parena);
  double* A = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(a_elems, 8);
  double* S = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(size_t(d.k), 8);
  double* U = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(size_t(d.m) * d.k, 8);
  double* V = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(size_t(d.n) * d.k, 8);
  // omega goes straight into its pipeline slot
  char* pbase = base;
  double* Q = reinterpret_cast<double*>(pbase);
  double* Qbar = reinterpret_cast<double*>(pbase + mb::arena_bytes_for(size_t(d.m) * d.L, 8));
  double* omega_dev = reinterpret_cast<double*>(pbase + mb::arena_bytes_for(size_t(d.m) * d.L, 8) +
                                                mb::arena_bytes_for(size_t(d.m) * d.l, 8));
  const int64_t lda = a_layout == MCNLA_B200_ROW_MAJOR ? d.n : d.m;
  if (a_layout == MCNLA_B200_ROW_MAJOR && a_elems * sizeof(double) >= (size_t(64) << 20)) {
    // large row-major A: copied in row blocks behind the sketch
    MB_CHECK(mb::run_sketch_streamed(ctx, d, A_host, A, omega_host, omega_dev, Q));
    MB_CHECK(mb::run_orthogonalize(ctx, d, Q));
    MB_CHECK(mb::run_integrate(ctx, d, integrator, Q, max_iteration, tolerance, Qbar, iteration));
    MB_CHECK(mb::run_form(ctx, d, former, A, a_layout, lda, Qbar, S, U, V));
  } else {
    MB_CHECK_CUDA(cudaMemcpyAsync(A, A_host, a_elems * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    MB_CHECK_CUDA(cudaMemcpyAsync(omega_dev, omega_host, size_t(d.n) * d.L * sizeof(double),
                                  cudaMemcpyHostToDevice, ctx->stream));
    MB_CHECK(mb::run_isvd(ctx, d, integrator, former, A, a_layout, lda, omega_dev, 0, max_iteration, tolerance, S,
                          U, V, iteration, pbase));
  }
  MB_CHECK_CUDA(cudaMemcpyAsync(S_host, S, size_t(d.k) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (U_host)
    MB_CHECK_CUDA(cudaMemcpyAsync(U_host, U, size_t(d.m) * d.k * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (V_host)
    MB_CHECK_CUDA(cudaMemcpyAsync(V_host, V, size_t(d.n) * d.k * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return MCNLA_B200_OK;
}

int mcnla_b200_isvd_stream(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former,
                           mcnla_b200_read_rows_fn read_rows, void* user, const double* omega_host, int max_iteration,
                           double tolerance, double* S_host, double* U_host, double* V_host, int* iteration) {
  if (!ctx || !read_rows || !omega_host || !iteration || !S_host) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  const size_t a_elems = size_t(d.m) * d.n;
  const size_t io = mb::arena_bytes_for(a_elems, 8) + mb::arena_bytes_for(size_t(d.k), 8) +
                    mb::arena_bytes_for(size_t(d.m) * d.k, 8) + mb::arena_bytes_for(size_t(d.n) * d.k, 8);
  MB_CHECK(mb::ctx_reserve_pipeline(ctx, io + mb::pipeline_bytes(d)));
  char* base = static_cast<char*>(ctx->parena);
  double* A = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(a_elems, 8);
  double* S = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(size_t(d.k), 8);
  double* U = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(size_t(d.m) * d.k, 8);
  double* V = reinterpret_cast<double*>(base);
  base += mb::arena_bytes_for(size_t(d.n) * d.k, 8);
  double* Q = reinterpret_cast<double*>(base);
  double* Qbar = reinterpret_cast<double*>(base + mb::arena_bytes_for(size_t(d.m) * d.L, 8));
  double* omega_dev = reinterpret_cast<double*>(base + mb::arena_bytes_for(size_t(d.m) * d.L, 8) +
                                                mb::arena_bytes_for(size_t(d.m) * d.l, 8));
  MB_CHECK_CUDA(cudaMemsetAsync(ctx->scal, 0, sizeof(mb::DevScalars), ctx->stream));
  MB_CHECK(mb::run_sketch_ingest(ctx, d, read_rows, user, A, omega_host, omega_dev, Q));
  MB_CHECK(mb::run_orthogonalize(ctx, d, Q));
  MB_CHECK(mb::run_integrate(ctx, d, integrator, Q, max_iteration, tolerance, Qbar, iteration));
  MB_CHECK(mb::run_form(ctx, d, former, A, MCNLA_B200_ROW_MAJOR, d.n, Qbar, S, U, V));
  MB_CHECK_CUDA(cudaMemcpyAsync(S_host, S, size_t(d.k) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (U_host)
    MB_CHECK_CUDA(cudaMemcpyAsync(U_host, U, size_t(d.m) * d.k * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (V_host)
    MB_CHECK_CUDA(cudaMemcpyAsync(V_host, V, size_t(d.n) * d.k * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return MCNLA_B200_OK;
}

int mcnla_b200_dgemm(mcnla_b200_ctx* ctx, int64_t M, int64_t N, int64_t K, double alpha, const double* A,
                     int64_t a_rs, int64_t a_cs, const double* B, int64_t b_rs, int64_t b_cs, double beta, double* C,
                     int64_t c_rs, int64_t c_cs, int force_splits) {
  if (!ctx || (M > 0 && N > 0 && (!C || (K > 0 && (!A || !B))))) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  // workspace for the split-K path (forced splits need their own size)
  size_t wsb = mb::dgemm_workspace_bytes(ctx, M, N, K, 1);
  if (force_splits > 0) wsb = std::max(wsb, size_t(force_splits) * M * N * sizeof(double));
  MB_CHECK(mb::ctx_reserve(ctx, wsb + 512));
  double* ws = nullptr;
  if (wsb) {
    ws = mb::ctx_take<double>(ctx, wsb / 8 + 1);
    ctx->gws = ws;
    ctx->gws_bytes = ws ? wsb + 8 : 0;
  }
  // a caller of the building block repeats its shapes: tune them like loop products
  mb::HotLoop hot(ctx);
  return mb::dgemm(ctx, M, N, K, alpha, mb::cm(A, a_rs, a_cs), mb::cm(B, b_rs, b_cs), beta, mb::dm(C, c_rs, c_cs),
                   mb::GemmBatch(), ws, force_splits);
}

int mcnla_b200_inverse_batched(mcnla_b200_ctx* ctx, int n, int batch, double* A) {
  if (!ctx || !A || n < 1 || batch < 1) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK_CUDA(cudaMemsetAsync(ctx->scal, 0, sizeof(mb::DevScalars), ctx->stream));
  MB_CHECK(mb::launch_inverse(ctx, n, batch, A));
  MB_CHECK(mb::ctx_sync_scalars(ctx));
  return ctx->scal_host->status ? ctx->scal_host->status : MCNLA_B200_OK;
}

int mcnla_b200_split_bf16(mcnla_b200_ctx* ctx, const double* A, int a_layout, int64_t lda, int64_t m, int64_t n,
                          uint16_t* hi, uint16_t* lo, uint16_t* lo2, int64_t ldo) {
  if (!ctx || !A || !hi || m < 0 || n < 0 || (lo2 && !lo)) return MCNLA_B200_ERR_ARG;
  if (a_layout != MCNLA_B200_ROW_MAJOR && a_layout != MCNLA_B200_COL_MAJOR) return MCNLA_B200_ERR_ARG;
  if (ldo < n || (a_layout == MCNLA_B200_ROW_MAJOR ? lda < n : lda < m)) return MCNLA_B200_ERR_SHAPE;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  return mb::launch_split_bf16(ctx, A, a_layout, lda, m, n, hi, lo, lo2, ldo);
}

int mcnla_b200_gaussian_bf16(mcnla_b200_ctx* ctx, uint64_t seed, int64_t n, int64_t L, uint16_t* omega_t,
                             int64_t ldo, double* omega) {
  if (!ctx || !omega_t || n < 0 || L < 0 || ldo < n) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  return mb::launch_gaussian_bf16(ctx, seed, n, L, omega_t, ldo, omega);
}

int mcnla_b200_gemm_bf16(mcnla_b200_ctx* ctx, int64_t M, int64_t N, int64_t K, const uint16_t* a_hi,
                         const uint16_t* a_lo, const uint16_t* a_lo2, int64_t lda, const uint16_t* b, int64_t ldb,
                         void* D, int64_t ldd, int out_fp64) {
  if (!ctx || !a_hi || !b || !D || ldd < N) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK_CUDA(cudaMemsetAsync(ctx->scal, 0, sizeof(mb::DevScalars), ctx->stream));
  MB_CHECK(mb::bf16_gemm(ctx, M, N, K, a_hi, a_lo, a_lo2, lda, b, ldb, D, ldd, out_fp64 != 0));
  MB_CHECK(mb::ctx_sync_scalars(ctx));
  return ctx->scal_host->status ? ctx->scal_host->status : MCNLA_B200_OK;
}

int mcnla_b200_sketch_bf16(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, const uint16_t* a_hi,
                           const uint16_t* a_lo, const uint16_t* a_lo2, int64_t lda16, const uint16_t* omega_t,
                           int64_t ldo, double* Q) {
  if (!ctx || !a_hi || !omega_t || !Q) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK_CUDA(cudaMemsetAsync(ctx->scal, 0, sizeof(mb::DevScalars), ctx->stream));
  MB_CHECK(mb::ctx_tic(ctx));
  MB_CHECK(mb::ctx_toc(ctx));
  MB_CHECK(mb::bf16_gemm(ctx, d.m, d.L, d.n, a_hi, a_lo, a_lo2, lda16, omega_t, ldo, Q, d.L, true));
  MB_CHECK(mb::ctx_toc(ctx));
  MB_CHECK(mb::ctx_sync_scalars(ctx));
  return ctx->scal_host->status ? ctx->scal_host->status : MCNLA_B200_OK;
}

int mcnla_b200_form_bf16(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int former, const uint16_t* at_hi,
                         const uint16_t* at_lo, const uint16_t* at_lo2, int64_t ldat, const double* Qbar, double* S,
                         double* U, double* V) {
  if (!ctx || !at_hi || !Qbar) return MCNLA_B200_ERR_ARG;
  if (at_lo2 && !at_lo) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK_CUDA(cudaMemsetAsync(ctx->scal, 0, sizeof(mb::DevScalars), ctx->stream));
  mb::AtParts at;
  at.hi = at_hi;
  at.lo = at_lo;
  at.lo2 = at_lo2;
  at.ld = ldat;
  MB_CHECK(mb::ctx_tic(ctx));
  MB_CHECK(mb::run_form(ctx, d, former, nullptr, MCNLA_B200_ROW_MAJOR, 0, Qbar, S, U, V, &at));
  MB_CHECK(mb::ctx_sync_scalars(ctx));
  return ctx->scal_host->status ? ctx->scal_host->status : MCNLA_B200_OK;
}

int mcnla_b200_isvd_mixed(mcnla_b200_ctx* ctx, const mcnla_b200_params* params, int integrator, int former,
                          const double* A, int a_layout, int64_t lda, const uint16_t* a_hi, const uint16_t* a_lo,
                          const uint16_t* a_lo2, int64_t lda16, const uint16_t* at_hi, const uint16_t* at_lo,
                          const uint16_t* at_lo2, int64_t ldat, uint64_t seed, int max_iteration, double tolerance,
                          double* S, double* U, double* V, int* iteration) {
  if (!ctx || (!A && !at_hi) || !a_hi || !iteration) return MCNLA_B200_ERR_ARG;
  if ((a_lo2 && !a_lo) || (at_lo2 && !at_lo)) return MCNLA_B200_ERR_ARG;
  Dims d;
  MB_CHECK(mb::get_dims(params, d));
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK(mb::ctx_reserve_pipeline(ctx, mb::pipeline_bytes_mixed(d)));
  mb::AtParts at;
  at.hi = at_hi;
  at.lo = at_lo;
  at.lo2 = at_lo2;
  at.ld = ldat;
  return mb::run_isvd_mixed(ctx, d, integrator, former, A, a_layout, lda, a_hi, a_lo, a_lo2, lda16,
                            at_hi ? &at : nullptr, seed, max_iteration, tolerance, S, U, V, iteration,
                            static_cast<char*>(ctx->parena));
}

int mcnla_b200_syev_batched(mcnla_b200_ctx* ctx, int n, int batch, const double* A, double* W, double* V,
                            int order) {
  if (!ctx || !A || !W || !V || n < 1 || batch < 1 || (order != 0 && order != 1)) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK(mb::ctx_reserve(ctx, mb::arena_bytes_for(size_t(batch) * n * n, 8)));
  return mb::launch_syev(ctx, n, batch, A, n, int64_t(n) * n, W, V, order);
}

}  // extern "C"
