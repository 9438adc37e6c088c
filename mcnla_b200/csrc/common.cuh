// Shared definitions of the B200 iSVD library: status codes, error checks,
// strided matrix references and the per-device context that owns workspaces.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <vector>
#include <string>

#include "../../include/mcnla_b200.h"

namespace mb {

// Status is returned by every host entry point; kernels report device-side
// failures (non-convergence is not a failure; a bounded wait that ran out is)
// through the context's device status word.
#define MB_CHECK_CUDA(expr)                                            \
  do {                                                                 \
    cudaError_t _e = (expr);                                           \
    if (_e != cudaSuccess) { ::mb::set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
                             return MCNLA_B200_ERR_CUDA; }             \
  } while (0)

#define MB_CHECK(expr)                                                 \
  do { int _s = (expr); if (_s != MCNLA_B200_OK) return _s; } while (0)

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void set_last_message(const std::string& msg);
const char* last_error_text();

// Element (i, j) of a strided matrix lives at p[i * rs + j * cs].
struct CMat { const double* p; int64_t rs, cs; };
struct DMat { double* p; int64_t rs, cs; };

inline CMat cm(const double* p, int64_t rs, int64_t cs) { return CMat{p, rs, cs}; }
inline DMat dm(double* p, int64_t rs, int64_t cs) { return DMat{p, rs, cs}; }
inline CMat cmc(DMat m) { return CMat{m.p, m.rs, m.cs}; }
// Row-major and column-major helpers (leading dimension ld).
inline CMat crow(const double* p, int64_t ld) { return CMat{p, ld, 1}; }
inline CMat ccol(const double* p, int64_t ld) { return CMat{p, 1, ld}; }
inline DMat drow(double* p, int64_t ld) { return DMat{p, ld, 1}; }
inline CMat ctr(CMat a) { return CMat{a.p, a.cs, a.rs}; }

// Device-resident scalars of one stage run (read back by the host between steps).
struct DevScalars {
  double norm;        // convergence norm (KN: ||e - 1||_2)
  double phit;        // WY: 1/2N ||B+||_F^2 of the last trial
  double mu;          // WY: tr(Dg) - ||D||_F^2
  double t1, t2;      // WY: step-size inner products
  double dot[16];     // scratch reductions
  int status;         // device-side error code (0 = ok)
  int sweeps;         // Jacobi sweeps used by the last small solve
  int stop_it;        // iteration at which an integrator converged (INT_MAX: not yet)
  int kn_fallback;    // 1: the series KN step declined this iteration (||Z|| too large)
  unsigned bar_count; // grid barrier of cooperative kernels: arrivals (only grows within a stage)
  unsigned bar_spare;
  int resume_it;      // persistent integrator: iteration it handed back to the host (-1: none)
  int kn_ns_failed;   // 1: the Newton-Schulz KN step with its matrices in global memory failed
};

// Per-device context: one stream, a growable workspace arena, timing events.
struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;   // host-to-device copies overlapped with compute (created on first use)
  void* stage_host[2] = {nullptr, nullptr};   // pinned staging of the streamed ingest (grown on demand)
  size_t stage_host_bytes = 0;
  bool own_stream = false;
  int num_sms = 148;
  size_t smem_optin = 0;
  // workspace arena (grown on demand by reserve(); never shrunk until destroy)
  void* arena = nullptr;
  size_t arena_bytes = 0;
  size_t arena_top = 0;
  // pipeline arena: buffers that live across the stages of one whole solve
  void* parena = nullptr;
  size_t parena_bytes = 0;
  // split-K workspace of the current stage (set by the stage; dgemm checks
  // every split-K launch against its size)
  double* gws = nullptr;
  size_t gws_bytes = 0;
  // iteration guard: while guard_stop is set, every kernel launched for
  // iteration guard_it returns at once when *guard_stop < guard_it (the
  // integrator converged earlier on the device).
  const int* guard_stop = nullptr;
  int guard_it = 0;
  // KN step method (MCNLA_B200_KN_*)
  int kn_mode = 0;
  // most CTAs a cooperative (persistent) grid of this context may take; 0:
  // all SMs.  Concurrent solves (the server's workers) each take a share so
  // that their persistent kernels can be resident together.
  int coop_cta_limit = 0;
  // time the tile configurations of a GEMM shape on its first call (dgemm.cu);
  // only the products of integrator iteration loops (tune_hot), whose shapes
  // repeat for every iteration, are tuned
  bool autotune = true;
  bool tune_hot = false;
  // KN iteration loops replay one captured CUDA graph per chunk of iterations
  bool graph_loop = true;
  // precision form: the Gramian integrators form Bs = Qs' Qs from BF16 parts of Qs
  bool mixed_gramian = false;
  // row-block decomposition over several GPUs: the stages sum their row-dependent
  // partial products over the ranks at the reference's MPI reduction points, through a
  // caller-supplied all-reduce or the library's own NCCL communicator (comm.cu)
  mcnla_b200_allreduce_fn allreduce_fn = nullptr;
  void* allreduce_user = nullptr;
  void* nccl_comm = nullptr;
  int comm_size = 1;
  int comm_rank = 0;
  int64_t allreduces = 0;
  double* comm_tmp = nullptr;     // contiguous staging of strided blocks for the all-reduce
  size_t comm_tmp_bytes = 0;
  DevScalars* scal = nullptr;       // device scalars
  DevScalars* scal_host = nullptr;  // pinned mirror
  // stage part timers (CUDA events), filled by the last stage call
  std::vector<cudaEvent_t> events;
  int nevents_used = 0;
  std::vector<double> last_times;   // seconds per part of the last stage call
  bool timing = true;
  // bookkeeping
  int64_t kernels_launched = 0;
  int64_t graph_replays = 0;   // chunks of KN iterations run as a replayed CUDA graph
};

// Arena allocation: every call of a stage first computes the bytes it needs,
// reserves them (one cudaMalloc at most, when the arena must grow), then
// carves aligned sub-buffers in order.
int ctx_reserve(Context* c, size_t bytes);
int ctx_reserve_pipeline(Context* c, size_t bytes);
// Device bytes the context's arenas hold between calls, and releasing them
// (stream-ordered; the next call grows them again).
int64_t ctx_held_bytes(const Context* c);
void ctx_trim(Context* c);
// Returns nullptr when the carve would pass the reservation (callers check).
template <class T>
T* ctx_take(Context* c, size_t count) {
  size_t off = (c->arena_top + 255) & ~size_t(255);
  c->arena_top = off + count * sizeof(T);
  if (c->arena_top > c->arena_bytes) return nullptr;
  return reinterpret_cast<T*>(static_cast<char*>(c->arena) + off);
}
inline size_t arena_bytes_for(size_t count, size_t elem) { return ((count * elem + 255) & ~size_t(255)) + 256; }

// Timing of stage parts (the reference's tic/toc moments,
// include/mcnla/isvd/core/stage_wrapper.hpp:170-192, on CUDA events).
int ctx_tic(Context* c);
int ctx_toc(Context* c);
int ctx_collect_times(Context* c);

int ctx_sync_scalars(Context* c);   // copies DevScalars to the pinned mirror and waits

// Sums `count` doubles at the device pointer buf over the ranks of the context's
// row-block decomposition, in place, ordered on the context's stream (comm.cu).  A
// no-op without one.  Every rank must make the same calls in the same order.
int ctx_allreduce(Context* c, double* buf, int64_t count);
inline bool ctx_distributed(const Context* c) { return c->allreduce_fn != nullptr || c->nccl_comm != nullptr; }
// The same for a rows x cols block with row stride ld (staged through a
// contiguous buffer of the context when ld != cols).
int ctx_allreduce2d(Context* c, double* p, int64_t ld, int64_t rows, int64_t cols);
// Sum over the ranks of a host value (1 without a communicator: the value itself).
int ctx_sum_host(Context* c, double v, double* out);
// Frees the communicator and the staging buffer (mcnla_b200_destroy).
void ctx_release_comm(Context* c);

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// FP64 flops of the lower-triangle Bs = Qs' Qs ((N l)^2 m) from which a mixed
// solve forms Bs (and its Gramian loop's Bs Bc) from BF16 parts instead.
constexpr double kMixedGramianMinFlops = 1e11;

}  // namespace mb

// The opaque handle of the C ABI is the context itself.
struct mcnla_b200_ctx : public mb::Context {};
