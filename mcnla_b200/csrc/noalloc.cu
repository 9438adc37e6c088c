// FP64 GEMM that allocates nothing.
//
// Some callers cannot call cudaMalloc: plugins hosted by a framework whose
// memory pool owns the device memory (a second allocator would exceed the
// pool's budget or fragment it), and latency-critical host loops that cannot
// take the implicit device synchronization a cudaMalloc/cudaFree may cause.
// mcnla_b200_dgemm needs a context whose workspace arena is allocated with
// cudaMalloc; this entry point takes only a stream, and keeps the split-K
// partial sums of the long-K products in a fixed array of device memory
// defined in this file.  That array (16 MiB) exists on every GPU that loads
// the library, from the first use until the process exits.
#include "common.cuh"
#include "dgemm.cuh"

#include <mutex>

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;   // MCNLA_B200_NOALLOC_SCRATCH_BYTES

// The partial sums of the split-K reduction.  Every call on a device shares
// it; a call writes every partial it later reads, so nothing needs clearing
// between calls, but two calls that overlap on the GPU (different streams, or
// different host threads) race on it.
static __device__ __align__(256) double g_splitk_scratch[kScratchBytes / sizeof(double)];

// In host code g_splitk_scratch names a host-side shadow, not device memory:
// the device address is looked up with the device current.  It is looked up
// again on every call, because a cudaDeviceReset recreates the device's
// primary context and the library's module with it, which may move the
// array; the last address seen on each device is kept only for calls made
// while their stream is being captured into a CUDA graph (a lookup that has
// to load the module is not allowed then).
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

int scratch_address(int device, cudaStream_t stream, double** out) {
  if (device < 0 || device >= kMaxDevices) return MCNLA_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
    (void)cudaGetLastError();
    cap = cudaStreamCaptureStatusNone;
  }
  if (cap != cudaStreamCaptureStatusNone && g_scratch_addr[device]) {
    *out = g_scratch_addr[device];
    return MCNLA_B200_OK;
  }
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_splitk_scratch);
  if (e != cudaSuccess) {
    mb::set_last_cuda_error(e, "cudaGetSymbolAddress(g_splitk_scratch)", __FILE__, __LINE__);
    return MCNLA_B200_ERR_CUDA;
  }
  g_scratch_addr[device] = static_cast<double*>(p);
  *out = g_scratch_addr[device];
  return MCNLA_B200_OK;
}

}  // namespace

extern "C" int mcnla_b200_dgemm_noalloc(void* stream, int64_t M, int64_t N, int64_t K, double alpha,
                                        const double* A, int64_t a_rs, int64_t a_cs, const double* B,
                                        int64_t b_rs, int64_t b_cs, double beta, double* C, int64_t c_rs,
                                        int64_t c_cs) {
  if (M < 0 || N < 0 || K < 0) return MCNLA_B200_ERR_SHAPE;
  if (M > 0 && N > 0 && (!C || (K > 0 && (!A || !B)))) return MCNLA_B200_ERR_ARG;
  int device = 0;
  MB_CHECK_CUDA(cudaGetDevice(&device));
  double* scratch = nullptr;
  MB_CHECK(scratch_address(device, static_cast<cudaStream_t>(stream), &scratch));
  int sms = 0;
  MB_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  // A context on the stack: stream, SM count and the static scratch as the
  // split-K workspace; no arena, no scalars, no events.
  mb::Context c;
  c.device = device;
  c.stream = static_cast<cudaStream_t>(stream);
  c.num_sms = sms;
  c.gws = scratch;
  c.gws_bytes = kScratchBytes;
  c.timing = false;
  c.autotune = false;   // the tuner allocates a scratch output
  const size_t need = mb::dgemm_workspace_bytes(&c, M, N, K, 1);
  if (need > kScratchBytes) {
    mb::set_last_message("mcnla_b200_dgemm_noalloc: the split-K partial sums of this shape need " +
                         std::to_string(need) + " bytes; the static scratch holds " +
                         std::to_string(kScratchBytes));
    return MCNLA_B200_ERR_SHAPE;
  }
  return mb::dgemm(&c, M, N, K, alpha, mb::cm(A, a_rs, a_cs), mb::cm(B, b_rs, b_cs), beta, mb::dm(C, c_rs, c_cs),
                   mb::GemmBatch(), need ? scratch : nullptr, 0);
}
