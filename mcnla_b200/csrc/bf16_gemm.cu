// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05) for the
// mixed-precision sketch:
//
//   D (M x N, FP64 or FP32, row-major) = sum_p A_p (M x K, BF16, K-major) * B (N x K, BF16, K-major)'
//
// with p over one to three parts of A (A = A_hi + A_lo + A_lo2, all BF16: 8,
// 16 or 24 bits of mantissa in total).  A stage of the shared-memory ring holds
// the k-tile of every part of A and one k-tile of B, so B is streamed once
// whatever the number of parts, and the MMAs of all parts accumulate from it.
//
// Warp 0 (one lane) streams 128 x 64 BF16 tiles of A and BN x 64 tiles of B
// into a 3-stage shared-memory ring (64 KB stages) with TMA (128-byte
// swizzle); warp 1 (one lane) issues tcgen05.mma (M = 128, N = BN, K = 16,
// four per part per stage) and releases each stage with tcgen05.commit.  Two
// tile configurations:
//   wide     (one or two parts): a 128 x 256 tile per CTA, one FP32 TMEM
//            accumulator over the whole K loop, read back by warps 4-7 (one
//            TMEM lane quarter each) and stored;
//   chunked  (three parts): the tensor cores accumulate in FP32 and the
//            error of a long sum is no longer small next to the 24-bit
//            representation of A, so the K loop is cut into chunks of 3
//            k-tiles (36 MMAs of K = 16 over the three parts: 576 products
//            per element; a caller may ask for shorter chunks).  A 128 x
//            128 tile per CTA; chunks alternate between two 128-column TMEM
//            accumulators, and warps 2-9 (two per TMEM lane quarter, 64
//            columns each) add every finished chunk into FP64 registers while
//            the next chunk is accumulated; D is stored once at the end.
// Every mbarrier wait is bounded: when one runs out the kernel records the
// fact in a device status word, lets the work already in flight drain (also
// with bounded waits) and frees its TMEM before returning.
#include "common.cuh"
#include "bf16.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <mutex>

namespace mb {
namespace {

constexpr int BM = 128, BK = 64;
constexpr int A_TILE_BYTES = BM * BK * 2;                 // 16 KB
constexpr int CHUNK_KT = 3;                               // k-tiles per FP32 accumulation chunk (chunked)
constexpr int MAX_PARTS = 3;
constexpr long long kWaitCycles = 4000000000LL;           // ~2 s at 2 GHz: a bounded wait

template <bool CHUNKED>
struct TileCfg {
  static constexpr int BN = CHUNKED ? 128 : 256;
  static constexpr int STAGES = 3;
  static constexpr int A_PARTS = CHUNKED ? 3 : 2;                   // A tiles per stage
  static constexpr int B_TILE_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = A_PARTS * A_TILE_BYTES + B_TILE_BYTES;   // 64 KB
  static constexpr uint32_t TMEM_COLS = CHUNKED ? 2 * BN : BN;      // two accumulators / one
  static constexpr int THREADS = CHUNKED ? 320 : 256;              // epilogue warps 2-9 / 4-7
  static constexpr size_t SMEM_BYTES = size_t(STAGES) * STAGE_BYTES + 1024;   // + alignment slack
  // instruction descriptor, kind::f16: D f32, A bf16, B bf16, both K-major, M = 128, N = BN
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) |
                                    (uint32_t(BM >> 4) << 24);
};

struct Args {
  int M, N;
  int KT;          // k-tiles
  int kt_per;      // k-tiles per split (split z covers [z kt_per, min(KT, (z + 1) kt_per)))
  int64_t split_stride;   // elements between the D slices of consecutive splits
  int chunk_kt;    // k-tiles per FP32 accumulation chunk (chunked configuration)
  int parts;       // 1 (A_hi), 2 (A_hi + A_lo) or 3 (A_hi + A_lo + A_lo2)
  void* D;
  int64_t ldd;
  int* status;     // device status word: set to MCNLA_B200_ERR_DEVICE_TIMEOUT on a run-out wait
  int accumulate;  // 1: D += result (D read back), 0: D = result
  int lower;       // 1: tiles strictly above the diagonal (every column > every row) are skipped
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Waits for the phase of `bar` with the given parity to complete; false when
// the wait ran out (about two seconds).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the
// 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFFu) >> 4);        // start address, bits [0, 14)
  d |= uint64_t(1) << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= uint64_t(1024 >> 4) << 32;                 // stride byte offset: 8 rows x 128 B
  d |= uint64_t(1) << 46;                         // descriptor version (sm_100)
  d |= uint64_t(2) << 61;                         // layout: 128-byte swizzle
  return d;
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  // the values are read only after the wait (register dependencies on a volatile asm)
#pragma unroll
  for (int j = 0; j < 32; ++j) asm volatile("" : "+r"(r[j]));
}

// The same load without the wait: the caller issues tcgen05.wait::ld before
// reading r.
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}

// Epilogue staging: a warp's 32 x 32 block of the output in shared memory, row
// r at stg[r * 33 ..] (the odd pitch keeps a lane's row writes and the
// row-wise reads on distinct banks), stored row by row: lane c writes column
// col0 + c of rows row0 .. row0 + 31, so each store instruction covers 32
// consecutive elements of one row.
constexpr int kStageBlock = 32 * 33;   // doubles per epilogue warp
static_assert(8 * kStageBlock * 8 <= 3 * (3 * 128 * 64 * 2 + 128 * 64 * 2), "epilogue staging fits in the ring");

template <class OutT>
__device__ __forceinline__ void store_block(const double* stg, OutT* D, const Args& g, int row0, int col0, int lane) {
  const int col = col0 + lane;
  if (col >= g.N) return;
  for (int i = 0; i < 32; ++i) {
    const int row = row0 + i;
    if (row >= g.M) break;
    OutT* d = D + int64_t(row) * g.ldd + col;
    const double v = stg[i * 33 + lane];
    *d = OutT(g.accumulate ? double(*d) + v : v);
  }
}

template <class OutT, bool CHUNKED>
__global__ void __launch_bounds__(TileCfg<CHUNKED>::THREADS, 1)
    bf16_gemm_kernel(const __grid_constant__ CUtensorMap tm_a_hi, const __grid_constant__ CUtensorMap tm_a_lo,
                     const __grid_constant__ CUtensorMap tm_a_lo2, const __grid_constant__ CUtensorMap tm_b, Args g) {
  using T = TileCfg<CHUNKED>;
  constexpr int BN = T::BN, STAGES = T::STAGES, STAGE_BYTES = T::STAGE_BYTES;
  extern __shared__ uint8_t smem_dyn[];
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t acc_full[2];     // a chunk is in accumulator b
  __shared__ __align__(8) uint64_t acc_empty[2];    // accumulator b has been read
  __shared__ __align__(8) uint64_t mma_done;
  __shared__ uint32_t tmem_base_s;

  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
  if (g.lower && n0 >= m0 + BM) return;          // the whole CTA, before any allocation
  const int kt0 = int(blockIdx.z) * g.kt_per;     // this split's first k-tile
  const int total_kt = min(g.KT - kt0, g.kt_per);
  OutT* const dsplit = static_cast<OutT*>(g.D) + int64_t(blockIdx.z) * g.split_stride;
  const int chunk_kt = CHUNKED ? g.chunk_kt : total_kt;
  const int chunks = (total_kt + chunk_kt - 1) / chunk_kt;
  constexpr int EPI_WARPS = CHUNKED ? 8 : 4;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(T::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], EPI_WARPS);
    }
    mbar_init(&mma_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_base_s;

  if (warp == 0 && lane == 0) {
    // ---- producer: TMA into the ring
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_a_hi)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_b)) : "memory");
    int issued = 0;
    bool ok = true;
    for (int kt = 0; kt < total_kt; ++kt) {
      const int s = kt % STAGES;
      if (kt >= STAGES && !mbar_wait(&empty_bar[s], ((kt / STAGES) & 1) ^ 1)) { ok = false; break; }
      uint8_t* sa = smem + s * STAGE_BYTES;
      uint8_t* sb = sa + T::A_PARTS * A_TILE_BYTES;
      mbar_expect_tx(&full_bar[s], uint32_t(g.parts * A_TILE_BYTES + T::B_TILE_BYTES));
      const int kx = (kt0 + kt) * BK;
      tma_load_2d(sa, &tm_a_hi, &full_bar[s], kx, m0);
      if (g.parts > 1) tma_load_2d(sa + A_TILE_BYTES, &tm_a_lo, &full_bar[s], kx, m0);
      if (g.parts > 2) tma_load_2d(sa + 2 * A_TILE_BYTES, &tm_a_lo2, &full_bar[s], kx, m0);
      tma_load_2d(sb, &tm_b, &full_bar[s], kx, n0);
      ++issued;
    }
    if (!ok) {
      atomicExch(g.status, MCNLA_B200_ERR_DEVICE_TIMEOUT);
      // let the copies in flight land before the CTA's shared memory goes away
      for (int kt = issued > STAGES ? issued - STAGES : 0; kt < issued; ++kt)
        mbar_wait(&full_bar[kt % STAGES], (kt / STAGES) & 1);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    for (int kt = 0; kt < total_kt; ++kt) {
      const int s = kt % STAGES;
      const int c = kt / chunk_kt, b = c & 1;
      const bool first = kt % chunk_kt == 0;
      if (first && c >= 2) {
        // accumulator b must have been read (chunk c - 2)
        if (!mbar_wait(&acc_empty[b], ((c >> 1) - 1) & 1)) { atomicExch(g.status, MCNLA_B200_ERR_DEVICE_TIMEOUT); break; }
        fence_after();
      }
      if (!mbar_wait(&full_bar[s], (kt / STAGES) & 1)) { atomicExch(g.status, MCNLA_B200_ERR_DEVICE_TIMEOUT); break; }
      fence_after();
      const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
      const uint32_t sb = sa + T::A_PARTS * A_TILE_BYTES;
      // smallest part first: the FP32 accumulator rounds each update to its
      // own magnitude, so the small parts' updates cost least while it is small
      bool fresh = first;
      for (int part = g.parts - 1; part >= 0; --part) {
#pragma unroll
        for (int k = 0; k < BK / 16; ++k) {   // 16 BF16 = 32 bytes along K per MMA
          umma_bf16(tmem + uint32_t(b * BN), sw128_desc(sa + part * A_TILE_BYTES + k * 32), sw128_desc(sb + k * 32),
                    T::IDESC, fresh ? 0u : 1u);
          fresh = false;
        }
      }
      umma_commit(&empty_bar[s]);        // the stage is free once these MMAs have read it
      if (kt % chunk_kt == chunk_kt - 1 || kt == total_kt - 1) umma_commit(&acc_full[b]);
    }
    umma_commit(&mma_done);              // every MMA issued above has completed
    mbar_wait(&mma_done, 0);
  } else if (CHUNKED && warp >= 2) {
    // ---- epilogue (chunked): per chunk TMEM -> FP64 registers; D stored at the end
    const int q = warp & 3;              // TMEM lane quarter this warp may access
    const int h = (warp - 2) >> 2;       // column half
    const int row = m0 + q * 32 + lane;
    double acc[BN / 2];
#pragma unroll
    for (int j = 0; j < BN / 2; ++j) acc[j] = 0.0;
    bool ok = true;
    for (int c = 0; c < chunks && ok; ++c) {
      const int b = c & 1;
      // warp-uniform outcome: the TMEM loads below are .sync.aligned
      ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[b], (c >> 1) & 1));
      fence_after();
      if (!ok) break;
      uint32_t r0[32], r1[32];
      const uint32_t ta = tmem + (uint32_t(q * 32) << 16) + uint32_t(b * BN + h * (BN / 2));
      tmem_ld32_nowait(ta, r0);
      tmem_ld32_nowait(ta + 32, r1);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) asm volatile("" : "+r"(r0[j]), "+r"(r1[j]));
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        acc[j] += double(__uint_as_float(r0[j]));
        acc[32 + j] += double(__uint_as_float(r1[j]));
      }
      fence_before();
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[b])) : "memory");
    }
    if (!ok) {
      if (lane == 0) atomicExch(g.status, MCNLA_B200_ERR_DEVICE_TIMEOUT);
    } else {
      // every MMA has completed, so the ring is idle: each warp stages its 32 x 32 blocks there
      // and stores them a row at a time (32 consecutive columns per store instruction)
      double* stg = reinterpret_cast<double*>(smem) + (warp - 2) * kStageBlock;
      const int col = n0 + h * (BN / 2);
#pragma unroll
      for (int hh = 0; hh < BN / 64; ++hh) {
#pragma unroll
        for (int j = 0; j < 32; ++j) stg[lane * 33 + j] = acc[hh * 32 + j];
        __syncwarp();
        store_block<OutT>(stg, dsplit, g, m0 + q * 32, col + hh * 32, lane);
        __syncwarp();
      }
    }
  } else if (!CHUNKED && warp >= 4) {
    // ---- epilogue (wide): TMEM -> registers -> global
    const int q = warp & 3;
    // warp-uniform outcome: the TMEM loads below are .sync.aligned
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[0], 0));
    fence_after();
    if (!ok) {
      if (lane == 0) atomicExch(g.status, MCNLA_B200_ERR_DEVICE_TIMEOUT);
    } else {
      // every MMA has completed, so the ring is idle: each warp stages its 32 x 32 blocks there
      // and stores them a row at a time (32 consecutive columns per store instruction)
      double* stg = reinterpret_cast<double*>(smem) + (warp - 4) * kStageBlock;
#pragma unroll 1
      for (int c = 0; c < BN / 32; ++c) {
        uint32_t r[32];
        tmem_ld32(tmem + (uint32_t(q * 32) << 16) + uint32_t(c * 32), r);
#pragma unroll
        for (int j = 0; j < 32; ++j) stg[lane * 33 + j] = double(__uint_as_float(r[j]));
        __syncwarp();
        store_block<OutT>(stg, dsplit, g, m0 + q * 32, n0 + c * 32, lane);
        __syncwarp();
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::TMEM_COLS));
  }
}

// ---- host: tensor maps through the driver entry point (no libcuda link)
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mutex;

int encode_fn(PFN_cuTensorMapEncodeTiled_v12000* out) {
  std::lock_guard<std::mutex> lock(g_encode_mutex);
  if (!g_encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    MB_CHECK_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn) {
      set_last_message("cuTensorMapEncodeTiled is not available from the driver");
      return MCNLA_B200_ERR_CUDA;
    }
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  *out = g_encode;
  return MCNLA_B200_OK;
}

// 2-D BF16 K-major tensor: rows x cols (cols = K, contiguous), row pitch ld elements.
int make_map(CUtensorMap* map, const void* base, int64_t rows, int64_t cols, int64_t ld, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc;
  MB_CHECK(encode_fn(&enc));
  cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(ld) * 2};
  cuuint32_t box[2] = {cuuint32_t(BK), cuuint32_t(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_message("cuTensorMapEncodeTiled failed with CUresult " + std::to_string(int(r)));
    return MCNLA_B200_ERR_CUDA;
  }
  return MCNLA_B200_OK;
}

}  // namespace

int bf16_gemm(Context* c, int64_t M, int64_t N, int64_t K, const uint16_t* a_hi, const uint16_t* a_lo,
              const uint16_t* a_lo2, int64_t lda, const uint16_t* b, int64_t ldb, void* D, int64_t ldd, bool out_fp64,
              bool accumulate, bool lower) {
  Bf16Split one;
  return bf16_gemm_split(c, M, N, K, a_hi, a_lo, a_lo2, lda, b, ldb, D, ldd, out_fp64, accumulate, lower, one);
}

int bf16_gemm_split(Context* c, int64_t M, int64_t N, int64_t K, const uint16_t* a_hi, const uint16_t* a_lo,
                    const uint16_t* a_lo2, int64_t lda, const uint16_t* b, int64_t ldb, void* D, int64_t ldd,
                    bool out_fp64, bool accumulate, bool lower, const Bf16Split& sp) {
  if (M <= 0 || N <= 0 || K <= 0) return MCNLA_B200_ERR_SHAPE;
  if (M > (int64_t(1) << 31) - 1 || N > (int64_t(1) << 31) - 1) return MCNLA_B200_ERR_SHAPE;
  // TMA: 16-byte aligned bases and row pitches
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  if (a_lo2 && !a_lo) return MCNLA_B200_ERR_ARG;
  if (!al16(a_hi) || (a_lo && !al16(a_lo)) || (a_lo2 && !al16(a_lo2)) || !al16(b) || (lda * 2) % 16 ||
      (ldb * 2) % 16)
    return MCNLA_B200_ERR_LAYOUT;
  if (lda < K || ldb < K) return MCNLA_B200_ERR_SHAPE;
  // three parts: the chunked configuration (FP64 sums of FP32 chunks)
  const bool chunked = a_lo2 != nullptr || sp.chunked;
  const int bn = chunked ? TileCfg<true>::BN : TileCfg<false>::BN;
  CUtensorMap ta_hi, ta_lo, ta_lo2, tb;
  MB_CHECK(make_map(&ta_hi, a_hi, M, K, lda, BM));
  MB_CHECK(make_map(&ta_lo, a_lo ? a_lo : a_hi, M, K, lda, BM));
  MB_CHECK(make_map(&ta_lo2, a_lo2 ? a_lo2 : a_hi, M, K, lda, BM));
  MB_CHECK(make_map(&tb, b, N, K, ldb, bn));
  Args g;
  g.M = int(M);
  g.N = int(N);
  g.KT = int(cdiv(K, BK));
  if (sp.splits < 1 || sp.kt_per < 0) return MCNLA_B200_ERR_ARG;
  g.kt_per = sp.splits == 1 ? g.KT : sp.kt_per;
  if (sp.splits > 1 && (g.kt_per < 1 || int64_t(g.kt_per) * (sp.splits - 1) >= g.KT ||
                        int64_t(g.kt_per) * sp.splits < g.KT || sp.split_stride < M * ldd || lower))
    return MCNLA_B200_ERR_ARG;   // every split gets at least one k-tile; slices do not overlap
  g.split_stride = sp.split_stride;
  g.chunk_kt = sp.chunk_kt > 0 ? sp.chunk_kt : CHUNK_KT;
  g.parts = a_lo2 ? 3 : (a_lo ? 2 : 1);
  static_assert(TileCfg<true>::A_PARTS >= MAX_PARTS, "the chunked stage holds every part");
  g.D = D;
  g.ldd = ldd;
  g.status = &c->scal->status;
  g.accumulate = accumulate ? 1 : 0;
  g.lower = lower ? 1 : 0;
  dim3 grid(unsigned(cdiv(N, bn)), unsigned(cdiv(M, BM)), unsigned(sp.splits));
  if (grid.y > 65535 || grid.z > 65535) return MCNLA_B200_ERR_SHAPE;
  auto go = [&](auto kern, int threads, size_t smem) -> int {
    MB_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    kern<<<grid, threads, smem, c->stream>>>(ta_hi, ta_lo, ta_lo2, tb, g);
    return MCNLA_B200_OK;
  };
  using W = TileCfg<false>;
  using Ch = TileCfg<true>;
  if (out_fp64) {
    MB_CHECK(chunked ? go(bf16_gemm_kernel<double, true>, Ch::THREADS, Ch::SMEM_BYTES)
                     : go(bf16_gemm_kernel<double, false>, W::THREADS, W::SMEM_BYTES));
  } else {
    MB_CHECK(chunked ? go(bf16_gemm_kernel<float, true>, Ch::THREADS, Ch::SMEM_BYTES)
                     : go(bf16_gemm_kernel<float, false>, W::THREADS, W::SMEM_BYTES));
  }
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

namespace {

// D := scale sum_z sum_g P_z(:, g group_cols + (0:N)) (z, then g, in order:
// deterministic), P_z = P + z stride, row-major with pitch ldp; D is N x M
// (transpose) or M x N.  Returns at once when guard_stop says the iteration
// loop stopped before iteration guard_it.
__global__ void k_sum_splits(const double* __restrict__ P, int splits, int64_t stride, int M, int N, int64_t ldp,
                             int groups, int64_t group_cols, double scale, double* __restrict__ D, int64_t ldd,
                             int transpose, const int* guard_stop, int guard_it) {
  if (guard_stop && *guard_stop < guard_it) return;
  const int64_t total = int64_t(M) * N;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / N, j = e % N;
    double v = 0.0;
    for (int z = 0; z < splits; ++z)
      for (int g = 0; g < groups; ++g) v += P[z * stride + i * ldp + g * group_cols + j];
    v *= scale;
    if (transpose) D[j * ldd + i] = v; else D[i * ldd + j] = v;
  }
}

}  // namespace

int launch_sum_splits(Context* c, const double* P, int splits, int64_t stride, int64_t M, int64_t N, int64_t ldp,
                      double* D, int64_t ldd, bool transpose, double scale, int groups, int64_t group_cols) {
  if (M <= 0 || N <= 0 || splits < 1 || groups < 1) return MCNLA_B200_ERR_SHAPE;
  const int64_t total = M * N;
  const int blocks = int(std::min<int64_t>(cdiv(total, 256), int64_t(c->num_sms) * 8));
  k_sum_splits<<<blocks, 256, 0, c->stream>>>(P, splits, stride, int(M), int(N), ldp, groups, group_cols, scale, D,
                                              ldd, transpose ? 1 : 0, c->guard_stop, c->guard_it);
  c->kernels_launched++;
  MB_CHECK_CUDA(cudaGetLastError());
  return MCNLA_B200_OK;
}

// Split count for an M x N x K product with tile width bn: the smallest
// count (<= max_splits, each split at least 16 k-tiles) whose CTAs fill the
// SMs' waves to at least 90 %, else the best found.
Bf16Split plan_bf16_split(const Context* c, int64_t M, int64_t N, int64_t K, bool chunked, int max_splits) {
  const int bn = chunked ? TileCfg<true>::BN : TileCfg<false>::BN;
  const int64_t tiles = cdiv(M, BM) * cdiv(N, bn), kt = cdiv(K, BK), sms = std::max(1, c->num_sms);
  Bf16Split best;
  best.chunked = chunked;
  double best_eff = 0.0;
  for (int s = 1; s <= max_splits; ++s) {
    const int64_t per = cdiv(kt, s);
    if (s > 1 && (per < 16 || per * (s - 1) >= kt)) break;
    const int64_t ctas = tiles * s;
    const double eff = double(ctas) / double(cdiv(ctas, sms) * sms);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best.splits = s;
      best.kt_per = int(per);
    }
    if (eff >= 0.9) break;
  }
  return best;
}

}  // namespace mb
