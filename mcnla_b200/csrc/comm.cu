// Collectives of the row-block decomposition over several GPUs.
//
// The reference decomposes one solve over MPI ranks by rows of A and sums the
// row-dependent partial products with MPI_Allreduce / reduce-scatter at a few
// points of each stage.  Here each rank is one process with one GPU, and the
// sums go through either the library's own NCCL communicator (NCCL over
// NVLink / NVSwitch, ordered on the context's stream) or an all-reduce the
// caller supplies.  libnccl.so.2 is opened on first use rather than linked, so
// the library loads next to whichever NCCL a host framework (e.g. torch)
// already brought into the process, and needs none when no communicator is
// used.
#include "common.cuh"

#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <mutex>
#include <string>

namespace mb {
namespace {

struct NcclApi {
  bool loaded = false;
  std::string error;
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                             cudaStream_t) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
};

std::mutex g_nccl_mutex;
NcclApi g_nccl;

const NcclApi* nccl_api() {
  std::lock_guard<std::mutex> lock(g_nccl_mutex);
  if (g_nccl.loaded) return &g_nccl;
  if (!g_nccl.error.empty()) return nullptr;
  // an NCCL already in the process (RTLD_NOLOAD) is preferred over loading one
  void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL | RTLD_NOLOAD);
  if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    g_nccl.error = std::string("libnccl.so.2 could not be loaded: ") + dlerror();
    return nullptr;
  }
  g_nccl.get_unique_id = reinterpret_cast<decltype(g_nccl.get_unique_id)>(dlsym(h, "ncclGetUniqueId"));
  g_nccl.comm_init_rank = reinterpret_cast<decltype(g_nccl.comm_init_rank)>(dlsym(h, "ncclCommInitRank"));
  g_nccl.all_reduce = reinterpret_cast<decltype(g_nccl.all_reduce)>(dlsym(h, "ncclAllReduce"));
  g_nccl.comm_destroy = reinterpret_cast<decltype(g_nccl.comm_destroy)>(dlsym(h, "ncclCommDestroy"));
  g_nccl.error_string = reinterpret_cast<decltype(g_nccl.error_string)>(dlsym(h, "ncclGetErrorString"));
  if (!g_nccl.get_unique_id || !g_nccl.comm_init_rank || !g_nccl.all_reduce || !g_nccl.comm_destroy ||
      !g_nccl.error_string) {
    g_nccl.error = "libnccl.so.2 lacks an expected symbol";
    return nullptr;
  }
  g_nccl.loaded = true;
  return &g_nccl;
}

int nccl_status(const NcclApi* api, ncclResult_t r, const char* what) {
  if (r == ncclSuccess) return MCNLA_B200_OK;
  set_last_message(std::string(what) + ": " + api->error_string(r));
  return MCNLA_B200_ERR_CUDA;
}

}  // namespace

int ctx_allreduce(Context* c, double* buf, int64_t count) {
  if (count <= 0) return MCNLA_B200_OK;
  if (c->nccl_comm) {
    const NcclApi* api = nccl_api();
    if (!api) return MCNLA_B200_ERR_CUDA;
    MB_CHECK(nccl_status(api, api->all_reduce(buf, buf, size_t(count), ncclFloat64, ncclSum,
                                              static_cast<ncclComm_t>(c->nccl_comm), c->stream),
                         "ncclAllReduce"));
    c->allreduces++;
    return MCNLA_B200_OK;
  }
  if (c->allreduce_fn) {
    const int r = c->allreduce_fn(c->allreduce_user, buf, count, c->stream);
    if (r != 0) {
      set_last_message("the row-block all-reduce callback returned " + std::to_string(r));
      return MCNLA_B200_ERR_CUDA;
    }
    c->allreduces++;
  }
  return MCNLA_B200_OK;
}

int ctx_allreduce2d(Context* c, double* p, int64_t ld, int64_t rows, int64_t cols) {
  if (!ctx_distributed(c) || rows <= 0 || cols <= 0) return MCNLA_B200_OK;
  if (ld == cols) return ctx_allreduce(c, p, rows * cols);
  const size_t bytes = size_t(rows) * cols * sizeof(double);
  if (bytes > c->comm_tmp_bytes) {
    if (c->comm_tmp) MB_CHECK_CUDA(cudaFreeAsync(c->comm_tmp, c->stream));
    c->comm_tmp = nullptr;
    c->comm_tmp_bytes = 0;
    MB_CHECK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&c->comm_tmp), bytes, c->stream));
    c->comm_tmp_bytes = bytes;
  }
  MB_CHECK_CUDA(cudaMemcpy2DAsync(c->comm_tmp, cols * sizeof(double), p, ld * sizeof(double), cols * sizeof(double),
                                  rows, cudaMemcpyDeviceToDevice, c->stream));
  MB_CHECK(ctx_allreduce(c, c->comm_tmp, rows * cols));
  MB_CHECK_CUDA(cudaMemcpy2DAsync(p, ld * sizeof(double), c->comm_tmp, cols * sizeof(double), cols * sizeof(double),
                                  rows, cudaMemcpyDeviceToDevice, c->stream));
  return MCNLA_B200_OK;
}

int ctx_sum_host(Context* c, double v, double* out) {
  *out = v;
  if (!ctx_distributed(c)) return MCNLA_B200_OK;
  double* d = &c->scal->dot[15];
  MB_CHECK_CUDA(cudaMemcpyAsync(d, &v, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  MB_CHECK(ctx_allreduce(c, d, 1));
  MB_CHECK(ctx_sync_scalars(c));
  *out = c->scal_host->dot[15];
  return MCNLA_B200_OK;
}

void ctx_release_comm(Context* c) {
  if (c->comm_tmp) {
    cudaFreeAsync(c->comm_tmp, c->stream);
    c->comm_tmp = nullptr;
    c->comm_tmp_bytes = 0;
  }
  if (c->nccl_comm) {
    if (const NcclApi* api = nccl_api()) api->comm_destroy(static_cast<ncclComm_t>(c->nccl_comm));
    c->nccl_comm = nullptr;
  }
  c->allreduce_fn = nullptr;
  c->allreduce_user = nullptr;
  c->comm_size = 1;
  c->comm_rank = 0;
}

}  // namespace mb

extern "C" {

int mcnla_b200_set_allreduce(mcnla_b200_ctx* ctx, mcnla_b200_allreduce_fn fn, void* user) {
  if (!ctx) return MCNLA_B200_ERR_ARG;
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  mb::ctx_release_comm(ctx);
  ctx->allreduce_fn = fn;
  ctx->allreduce_user = fn ? user : nullptr;
  return MCNLA_B200_OK;
}

int mcnla_b200_nccl_unique_id(unsigned char* id) {
  if (!id) return MCNLA_B200_ERR_ARG;
  const mb::NcclApi* api = mb::nccl_api();
  if (!api) {
    mb::set_last_message(mb::g_nccl.error);
    return MCNLA_B200_ERR_CUDA;
  }
  ncclUniqueId u;
  MB_CHECK(mb::nccl_status(api, api->get_unique_id(&u), "ncclGetUniqueId"));
  static_assert(sizeof(u) == MCNLA_B200_NCCL_ID_BYTES, "NCCL unique id size");
  std::memcpy(id, &u, sizeof(u));
  return MCNLA_B200_OK;
}

int mcnla_b200_set_nccl(mcnla_b200_ctx* ctx, const unsigned char* id, int nranks, int rank) {
  if (!ctx || !id || nranks < 1 || rank < 0 || rank >= nranks) return MCNLA_B200_ERR_ARG;
  const mb::NcclApi* api = mb::nccl_api();
  if (!api) {
    mb::set_last_message(mb::g_nccl.error);
    return MCNLA_B200_ERR_CUDA;
  }
  MB_CHECK_CUDA(cudaSetDevice(ctx->device));
  MB_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  mb::ctx_release_comm(ctx);
  ncclUniqueId u;
  std::memcpy(&u, id, sizeof(u));
  ncclComm_t comm = nullptr;
  MB_CHECK(mb::nccl_status(api, api->comm_init_rank(&comm, nranks, u, rank), "ncclCommInitRank"));
  ctx->nccl_comm = comm;
  ctx->comm_size = nranks;
  ctx->comm_rank = rank;
  return MCNLA_B200_OK;
}

int64_t mcnla_b200_allreduces(const mcnla_b200_ctx* ctx) { return ctx ? ctx->allreduces : 0; }

}  // extern "C"
