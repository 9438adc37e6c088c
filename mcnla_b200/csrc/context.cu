#include <algorithm>
// Context lifecycle, workspace arena, stage timers and status strings.
#include "common.cuh"
#include <cstdio>
#include <cstring>
#include <new>

namespace mb {

namespace {
thread_local char g_last_error[512] = "";
}

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
}

void set_last_message(const std::string& msg) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg.c_str());
}

const char* last_error_text() { return g_last_error; }

// The arenas grow stream-ordered (cudaFreeAsync / cudaMallocAsync on the
// context's stream): no device-wide synchronisation, so a growing context does
// not stall the work of other contexts (the server's workers).
int ctx_reserve(Context* c, size_t bytes) {
  c->arena_top = 0;
  if (bytes <= c->arena_bytes) return MCNLA_B200_OK;
  if (c->arena) {
    MB_CHECK_CUDA(cudaFreeAsync(c->arena, c->stream));
    c->arena = nullptr;
    c->arena_bytes = 0;
  }
  const size_t want = bytes + std::min(bytes >> 1, size_t(256) << 20);   // grow with headroom
  cudaError_t e = cudaMallocAsync(&c->arena, want, c->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_last_cuda_error(e, "workspace cudaMalloc", __FILE__, __LINE__);
    c->arena = nullptr;
    return MCNLA_B200_ERR_NOMEM;
  }
  c->arena_bytes = want;
  return MCNLA_B200_OK;
}

int ctx_reserve_pipeline(Context* c, size_t bytes) {
  if (bytes <= c->parena_bytes) return MCNLA_B200_OK;
  if (c->parena) {
    MB_CHECK_CUDA(cudaFreeAsync(c->parena, c->stream));
    c->parena = nullptr;
    c->parena_bytes = 0;
  }
  const size_t want = bytes + std::min(bytes >> 1, size_t(256) << 20);
  cudaError_t e = cudaMallocAsync(&c->parena, want, c->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_last_cuda_error(e, "pipeline cudaMalloc", __FILE__, __LINE__);
    c->parena = nullptr;
    return MCNLA_B200_ERR_NOMEM;
  }
  c->parena_bytes = want;
  return MCNLA_B200_OK;
}

int64_t ctx_held_bytes(const Context* c) {
  return int64_t(c->arena_bytes) + int64_t(c->parena_bytes) + int64_t(c->comm_tmp_bytes);
}

void ctx_trim(Context* c) {
  if (c->arena) cudaFreeAsync(c->arena, c->stream);
  if (c->parena) cudaFreeAsync(c->parena, c->stream);
  c->arena = c->parena = nullptr;
  c->arena_bytes = c->parena_bytes = 0;
  c->arena_top = 0;
}

int ctx_tic(Context* c) {
  c->nevents_used = 0;
  return ctx_toc(c);
}

int ctx_toc(Context* c) {
  if (!c->timing) return MCNLA_B200_OK;
  if (c->nevents_used >= int(c->events.size())) {
    cudaEvent_t ev;
    MB_CHECK_CUDA(cudaEventCreate(&ev));
    c->events.push_back(ev);
  }
  MB_CHECK_CUDA(cudaEventRecord(c->events[c->nevents_used], c->stream));
  c->nevents_used++;
  return MCNLA_B200_OK;
}

int ctx_collect_times(Context* c) {
  c->last_times.clear();
  if (!c->timing || c->nevents_used < 2) return MCNLA_B200_OK;
  MB_CHECK_CUDA(cudaEventSynchronize(c->events[c->nevents_used - 1]));
  for (int i = 1; i < c->nevents_used; ++i) {
    float ms = 0.f;
    MB_CHECK_CUDA(cudaEventElapsedTime(&ms, c->events[i - 1], c->events[i]));
    c->last_times.push_back(ms * 1e-3);
  }
  return MCNLA_B200_OK;
}

int ctx_sync_scalars(Context* c) {
  MB_CHECK_CUDA(cudaMemcpyAsync(c->scal_host, c->scal, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(c->stream));
  return MCNLA_B200_OK;
}

}  // namespace mb

using mb::Context;

extern "C" {

const char* mcnla_b200_last_error(void) { return mb::last_error_text(); }

const char* mcnla_b200_status_string(int status) {
  switch (status) {
    case MCNLA_B200_OK: return "ok";
    case MCNLA_B200_ERR_SHAPE: return "invalid or inconsistent sizes";
    case MCNLA_B200_ERR_LAYOUT: return "operand has no unit stride";
    case MCNLA_B200_ERR_WORKSPACE: return "missing workspace";
    case MCNLA_B200_ERR_CUDA: return "CUDA runtime error";
    case MCNLA_B200_ERR_NOMEM: return "device out of memory";
    case MCNLA_B200_ERR_ARG: return "invalid argument";
    case MCNLA_B200_ERR_UNSUPPORTED: return "shape beyond a kernel limit";
    case MCNLA_B200_ERR_SINGULAR: return "singular matrix in a small inverse";
    case MCNLA_B200_ERR_DEVICE_TIMEOUT: return "a bounded device-side wait ran out";
    case MCNLA_B200_ERR_IO: return "a file is missing, unreadable, or not in the expected format";
    default: return "unknown status";
  }
}

int mcnla_b200_create(mcnla_b200_ctx** out, int device, void* stream) {
  if (!out) return MCNLA_B200_ERR_ARG;
  *out = nullptr;
  mcnla_b200_ctx* c = new (std::nothrow) mcnla_b200_ctx();
  if (!c) return MCNLA_B200_ERR_NOMEM;
  c->device = device;
  auto fail = [&](int st) { delete c; return st; };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { mb::set_last_cuda_error(e, "cudaSetDevice", __FILE__, __LINE__); return fail(MCNLA_B200_ERR_CUDA); }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) { mb::set_last_cuda_error(e, "cudaGetDeviceProperties", __FILE__, __LINE__); return fail(MCNLA_B200_ERR_CUDA); }
  c->num_sms = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  // NULL is CUDA's (legacy) default stream, as in every CUDA API
  c->stream = static_cast<cudaStream_t>(stream);
  c->own_stream = false;
  e = cudaMalloc(&c->scal, sizeof(mb::DevScalars));
  if (e != cudaSuccess) { mb::set_last_cuda_error(e, "cudaMalloc scalars", __FILE__, __LINE__); return fail(MCNLA_B200_ERR_NOMEM); }
  e = cudaMallocHost(&c->scal_host, sizeof(mb::DevScalars));
  if (e != cudaSuccess) { mb::set_last_cuda_error(e, "cudaMallocHost", __FILE__, __LINE__); return fail(MCNLA_B200_ERR_NOMEM); }
  std::memset(c->scal_host, 0, sizeof(mb::DevScalars));
  e = cudaMemsetAsync(c->scal, 0, sizeof(mb::DevScalars), c->stream);
  if (e != cudaSuccess) { mb::set_last_cuda_error(e, "cudaMemset", __FILE__, __LINE__); return fail(MCNLA_B200_ERR_CUDA); }
  *out = c;
  return MCNLA_B200_OK;
}

int mcnla_b200_destroy(mcnla_b200_ctx* c) {
  if (!c) return MCNLA_B200_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);   // copies land in the arenas freed below
  mb::ctx_release_comm(c);
  cudaStreamSynchronize(c->stream);
  for (auto ev : c->events) cudaEventDestroy(ev);
  if (c->arena) cudaFree(c->arena);
  if (c->parena) cudaFree(c->parena);
  if (c->scal) cudaFree(c->scal);
  if (c->scal_host) cudaFreeHost(c->scal_host);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  for (void* h : c->stage_host)
    if (h) cudaFreeHost(h);
  delete c;
  return MCNLA_B200_OK;
}

int mcnla_b200_set_stream(mcnla_b200_ctx* c, void* stream) {
  if (!c) return MCNLA_B200_ERR_ARG;
  // the arenas are freed stream-ordered on the context's stream: work still
  // queued on the old stream must finish before another stream may free them
  if (c->stream != static_cast<cudaStream_t>(stream)) MB_CHECK_CUDA(cudaStreamSynchronize(c->stream));
  if (c->own_stream && c->stream) {
    MB_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    MB_CHECK_CUDA(cudaStreamDestroy(c->stream));
  }
  c->stream = static_cast<cudaStream_t>(stream);
  c->own_stream = false;
  return MCNLA_B200_OK;
}

int64_t mcnla_b200_kernels_launched(const mcnla_b200_ctx* c) { return c ? c->kernels_launched : 0; }
int64_t mcnla_b200_graph_replays(const mcnla_b200_ctx* c) { return c ? c->graph_replays : 0; }

int mcnla_b200_set_autotune(mcnla_b200_ctx* c, int on) {
  if (!c) return MCNLA_B200_ERR_ARG;
  c->autotune = on != 0;
  return MCNLA_B200_OK;
}

int mcnla_b200_set_cta_limit(mcnla_b200_ctx* c, int ctas) {
  if (!c || ctas < 0) return MCNLA_B200_ERR_ARG;
  c->coop_cta_limit = ctas;
  return MCNLA_B200_OK;
}

int mcnla_b200_set_graph_loop(mcnla_b200_ctx* c, int on) {
  if (!c) return MCNLA_B200_ERR_ARG;
  c->graph_loop = on != 0;
  return MCNLA_B200_OK;
}

int mcnla_b200_set_kn_method(mcnla_b200_ctx* c, int method) {
  if (!c || method < MCNLA_B200_KN_AUTO || method > MCNLA_B200_KN_NEWTON_SCHULZ) return MCNLA_B200_ERR_ARG;
  c->kn_mode = method;
  return MCNLA_B200_OK;
}

int mcnla_b200_last_times(mcnla_b200_ctx* c, double* times, int capacity) {
  if (!c || (!times && capacity > 0)) return -MCNLA_B200_ERR_ARG;
  int st = mb::ctx_collect_times(c);
  if (st != MCNLA_B200_OK) return -st;
  const int n = std::min<int>(capacity, int(c->last_times.size()));
  for (int i = 0; i < n; ++i) times[i] = c->last_times[i];
  return int(c->last_times.size()) < capacity ? int(c->last_times.size()) : n;
}

}  // extern "C"
