// Conversions feeding the BF16 tensor-core sketch: the hi/lo split of FP64 A
// and Omega' drawn directly in BF16.
#include "bf16.cuh"
#include "philox.cuh"

#include <cuda_bf16.h>
#include <algorithm>

namespace mb {
namespace {

__device__ __forceinline__ uint16_t bf16_bits(__nv_bfloat16 h) { return *reinterpret_cast<uint16_t*>(&h); }

// hi = bf16(x), lo = bf16(x - hi), lo2 = bf16(x - hi - lo) (round to nearest
// even; the differences are exact in FP64)
__device__ __forceinline__ void split(double x, uint16_t& hi, uint16_t& lo, uint16_t& lo2) {
  const __nv_bfloat16 h = __double2bfloat16(x);
  hi = bf16_bits(h);
  const double r = x - double(__bfloat162float(h));
  const __nv_bfloat16 l = __double2bfloat16(r);
  lo = bf16_bits(l);
  lo2 = bf16_bits(__double2bfloat16(r - double(__bfloat162float(l))));
}

// T: double, or float (an FP32 A splits to the same parts as its exact FP64 copy)
template <class T>
__global__ void k_split_rowmajor(const T* A, int64_t lda, int64_t m, int64_t n, uint16_t* hi, uint16_t* lo,
                                 uint16_t* lo2, int64_t ldo) {
  const int64_t total = m * n;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / n, j = e % n;
    uint16_t h, l, l2;
    split(double(A[i * lda + j]), h, l, l2);
    hi[i * ldo + j] = h;
    if (lo) lo[i * ldo + j] = l;
    if (lo2) lo2[i * ldo + j] = l2;
  }
}

// column-major A (element (i, j) at A[i + j lda]) to row-major hi/lo through
// 32 x 32 shared-memory tiles (coalesced on both sides)
template <class T>
__global__ void k_split_colmajor(const T* A, int64_t lda, int64_t m, int64_t n, uint16_t* hi, uint16_t* lo,
                                 uint16_t* lo2, int64_t ldo) {
  __shared__ double tile[32][33];
  const int64_t i0 = int64_t(blockIdx.x) * 32, j0 = int64_t(blockIdx.y) * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int64_t i = i0 + tx, j = j0 + r;
    tile[r][tx] = (i < m && j < n) ? double(A[i + j * lda]) : 0.0;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int64_t i = i0 + r, j = j0 + tx;
    if (i < m && j < n) {
      uint16_t h, l, l2;
      split(tile[tx][r], h, l, l2);
      hi[i * ldo + j] = h;
      if (lo) lo[i * ldo + j] = l;
      if (lo2) lo2[i * ldo + j] = l2;
    }
  }
}

// Omega (n x L): sample (i, j) = element i L + j of the FP64 stream; written
// transposed as Omega' (L x n, pitch ldo) in BF16 and, optionally, as the
// FP64 n x L Omega holding the same BF16-rounded values.
__global__ void k_gaussian_bf16(uint64_t seed, int64_t n, int64_t L, uint16_t* omega_t, int64_t ldo, double* omega) {
  __shared__ uint16_t tile[32][34];
  const int64_t i0 = int64_t(blockIdx.x) * 32, j0 = int64_t(blockIdx.y) * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int64_t i = i0 + r, j = j0 + tx;
    uint16_t v = 0;
    if (i < n && j < L) {
      const uint64_t e = uint64_t(i) * uint64_t(L) + uint64_t(j);
      double z0, z1;
      gaussian_pair(seed, e >> 1, z0, z1);
      const __nv_bfloat16 h = __double2bfloat16((e & 1) ? z1 : z0);
      v = bf16_bits(h);
      if (omega) omega[i * L + j] = double(__bfloat162float(h));
    }
    tile[r][tx] = v;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int64_t j = j0 + r, i = i0 + tx;
    if (i < n && j < L) omega_t[j * ldo + i] = tile[tx][r];
  }
}

}  // namespace

template <class T>
int split_bf16_any(Context* c, const T* A, int layout, int64_t lda, int64_t m, int64_t n, uint16_t* hi,
                   uint16_t* lo, uint16_t* lo2, int64_t ldo) {
  if (m <= 0 || n <= 0) return MCNLA_B200_OK;
  if (layout == MCNLA_B200_ROW_MAJOR) {
    const int64_t total = m * n;
    const int blocks = int(std::min<int64_t>(cdiv(total, 256), int64_t(c->num_sms) * 32));
    k_split_rowmajor<T><<<blocks, 256, 0, c->stream>>>(A, lda, m, n, hi, lo, lo2, ldo);
  } else {
    dim3 grid(unsigned(cdiv(m, 32)), unsigned(cdiv(n, 32)));
    if (grid.y > 65535) return MCNLA_B200_ERR_SHAPE;
    k_split_colmajor<T><<<grid, dim3(32, 8), 0, c->stream>>>(A, lda, m, n, hi, lo, lo2, ldo);
  }
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

int launch_split_bf16(Context* c, const double* A, int layout, int64_t lda, int64_t m, int64_t n, uint16_t* hi,
                      uint16_t* lo, uint16_t* lo2, int64_t ldo) {
  return split_bf16_any(c, A, layout, lda, m, n, hi, lo, lo2, ldo);
}

int launch_split_bf16_f32(Context* c, const float* A, int layout, int64_t lda, int64_t m, int64_t n, uint16_t* hi,
                          uint16_t* lo, uint16_t* lo2, int64_t ldo) {
  return split_bf16_any(c, A, layout, lda, m, n, hi, lo, lo2, ldo);
}

int launch_gaussian_bf16(Context* c, uint64_t seed, int64_t n, int64_t L, uint16_t* omega_t, int64_t ldo,
                         double* omega) {
  if (n <= 0 || L <= 0) return MCNLA_B200_OK;
  dim3 grid(unsigned(cdiv(n, 32)), unsigned(cdiv(L, 32)));
  if (grid.y > 65535) return MCNLA_B200_ERR_SHAPE;
  k_gaussian_bf16<<<grid, dim3(32, 8), 0, c->stream>>>(seed, n, L, omega_t, ldo, omega);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

}  // namespace mb
