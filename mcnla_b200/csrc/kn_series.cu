// Stand-alone Kolmogorov-Nagumo step by power series (kn_series.cuh) on
// ceil(l/8) cooperative CTAs.  Launched in front of the matrix-function /
// eigendecomposition step kernel, which runs only when this one declined
// (scal->kn_fallback).
#include <algorithm>
#include "kn_series.cuh"

namespace mb {
namespace {

constexpr int kSerThreads = 256;

struct StepArgs {
  SeriesArgs s;
  double tol;
  const int* guard_stop;
  int guard_it;
};

__global__ void __launch_bounds__(kSerThreads) k_kn_series(StepArgs a) {
  extern __shared__ __align__(16) double sm[];
  if (a.guard_stop && *a.guard_stop < a.guard_it) return;
  __shared__ int s_flag;
  double norm = 0.0;
  int degree = 0;
  const int r = kn_series_step(a.s, sm, &s_flag, false, &norm, &degree);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (r == kStepDeclined) {
      a.s.scal->kn_fallback = 1;
    } else if (r == kStepDone) {
      a.s.scal->kn_fallback = 0;
      a.s.scal->norm = norm;
      a.s.scal->sweeps = 1000 + degree;
      if (a.guard_stop && !(norm >= a.tol)) a.s.scal->stop_it = a.guard_it;
    }
  }
}

}  // namespace

size_t kn_series_work_doubles(int l) {
  // the series' scratch, or the four padded l x l matrices of the Newton-Schulz step where they do
  // not fit in shared memory (l > 80)
  const size_t lp = (size_t(l) + 15) & ~size_t(15);
  return std::max(2 * size_t(l) * l + 3 * size_t((l + 7) / 8) + 8, l > 80 ? 4 * lp * (lp + 4) : 0);
}

int launch_kn_series(Context* c, int l, const double* z, const double* dd, double inv_n, double* out, double* outn,
                     const double* ff, double* ffn, double* work, double tol) {
  if (l < 1 || l > MCNLA_B200_MAX_DIM_SKETCH) return MCNLA_B200_ERR_UNSUPPORTED;
  const int G = (l + 7) / 8;
  const int smax = kn_series_smax(l, c->smem_optin, 0);
  if (smax == 0) return MCNLA_B200_ERR_UNSUPPORTED;
  const size_t smem = kn_series_smem_doubles(l, smax) * sizeof(double);
  MB_CHECK(set_smem(c, reinterpret_cast<const void*>(k_kn_series), smem));
  StepArgs a;
  a.s = series_args(c, l, z, dd, inv_n, out, outn, ff, ffn, work, smax);
  a.tol = tol;
  a.guard_stop = c->guard_stop;
  a.guard_it = c->guard_it;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(G));
  cfg.blockDim = dim3(kSerThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MB_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_kn_series, a));
  c->kernels_launched++;
  return MCNLA_B200_OK;
}

}  // namespace mb
