// The binding a maintainer of MCNLA (emfomy/mcnla 0.7.2) adds to run its iSVD
// stages on a B200: new tags that specialise the reference's own stage
// templates (mcnla::isvd::Sketcher / Orthogonalizer / Integrator / Former,
// include/mcnla/isvd/{sketcher,orthogonalizer,integrator,former}/*.hpp) and
// call the C ABI of mcnla_b200.h from runImpl.  A driver picks them with its
// STYPE / OTYPE / ITYPE / FTYPE macros (src/isvd_dense_rb.cpp:12-34), e.g.
//   #define ITYPE RowBlockGramianKolmogorovNagumoIntegratorB200
// Include it after <mcnla/isvd.hpp>; link libmcnla_b200.so and libcudart.
//
// Each stage keeps its device buffers (sized from the Parameters at
// initialize()) for its lifetime and uses one library context per device
// (created on first use, on the device current at initialize()), so a run
// allocates nothing.  The stages take and return the reference's host
// matrices: runImpl copies its operands to the device and its results back,
// the way the reference's own GPU stages do (include/mcnla/isvd_gpu/**).
// The reference reports failures by assert; a non-zero status of the library
// is reported on stderr with the library's message and aborts.
//
// Differences from the CPU stages: the Gaussian sketcher draws Omega on the
// device from its seed (Philox-4x32-10 + Box-Muller) instead of the
// reference's host streams, so its sketches are the same distribution but not
// the same numbers; every other stage computes the reference's algorithm on
// the same inputs (singular values and vectors to 1e-10, identical iteration
// counts in the library's parity tests).
#ifndef MCNLA_B200_MCNLA_TAGS_HPP_
#define MCNLA_B200_MCNLA_TAGS_HPP_

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>

#include "../mcnla_b200.h"

namespace mcnla {
namespace isvd {
namespace b200 {

inline void check(int status, const char* what) {
  if (status != MCNLA_B200_OK) {
    std::fprintf(stderr, "mcnla_b200: %s failed: %s (%s)\n", what, mcnla_b200_status_string(status),
                 mcnla_b200_last_error());
    std::abort();
  }
}

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "mcnla_b200: %s failed: %s\n", what, cudaGetErrorString(e));
    std::abort();
  }
}

// The library context of the current device (one per device and process,
// on CUDA's default stream).
inline mcnla_b200_ctx* context() {
  static std::mutex mu;
  static std::map<int, mcnla_b200_ctx*> contexts;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(mu);
  mcnla_b200_ctx*& c = contexts[dev];
  if (!c) check(mcnla_b200_create(&c, dev, nullptr), "mcnla_b200_create");
  return c;
}

// Row blocks over the reference's MPI ranks (Parameters::mpi_size > 1, one GPU
// per rank): the context gets the library's NCCL communicator, its id made by
// the Parameters' root rank and broadcast over the Parameters' communicator,
// so each stage sums its row-dependent partial products over NVLink where the
// reference's row-block stages call MPI_Allreduce
// (row_block_gramian_orthogonalizer.hpp:86, the row-block integrators and
// formers).  Every rank then has to run the same stages in the same order, as
// the reference's drivers do.  force attaches on one rank too.
inline void attach_ranks(const Parameters<double>& p, mcnla_b200_ctx* c, bool force = false) {
  static std::mutex mu;
  static std::map<mcnla_b200_ctx*, MPI_Comm> attached;
  if (p.mpi_size <= 1 && !force) return;
  std::lock_guard<std::mutex> lock(mu);
  auto it = attached.find(c);
  if (it != attached.end()) {
    if (it->second != p.mpi_comm) {
      std::fprintf(stderr, "mcnla_b200: a device's context serves one MPI communicator\n");
      std::abort();
    }
    return;
  }
  unsigned char id[MCNLA_B200_NCCL_ID_BYTES] = {};
  if (p.mpi_rank == p.mpi_root) check(mcnla_b200_nccl_unique_id(id), "mcnla_b200_nccl_unique_id");
  if (MPI_Bcast(id, MCNLA_B200_NCCL_ID_BYTES, MPI_BYTE, p.mpi_root, p.mpi_comm) != MPI_SUCCESS) {
    std::fprintf(stderr, "mcnla_b200: MPI_Bcast of the NCCL id failed\n");
    std::abort();
  }
  check(mcnla_b200_set_nccl(c, id, int(p.mpi_size), int(p.mpi_rank)), "mcnla_b200_set_nccl");
  attached.emplace(c, p.mpi_comm);
}

// The context a stage runs on, with the ranks attached.
inline mcnla_b200_ctx* context(const Parameters<double>& p) {
  mcnla_b200_ctx* c = context();
  attach_ranks(p, c);
  return c;
}

// A device buffer owned by a stage.
struct DeviceBuffer {
  double* p = nullptr;
  size_t count = 0;
  void reserve(size_t n) {
    if (n <= count) return;
    if (p) cudaFree(p);
    p = nullptr;
    check_cuda(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(double)), "cudaMalloc");
    count = n;
  }
  ~DeviceBuffer() {
    if (p) cudaFree(p);
  }
};

inline mcnla_b200_params params_of(const Parameters<double>& p) {
  return mcnla_b200_params{p.nrowRank(), p.ncol(), p.rank(), p.overRank(), p.numSketch()};
}

// Host <-> device for the reference's row-major and column-major dense matrices.
inline void to_device(const DenseMatrixRowMajor<double>& a, double* d) {
  check_cuda(cudaMemcpy2D(d, a.ncol() * sizeof(double), a.valPtr(), a.pitch() * sizeof(double),
                          a.ncol() * sizeof(double), a.nrow(), cudaMemcpyHostToDevice), "cudaMemcpy2D");
}
inline void to_device(const DenseMatrixColMajor<double>& a, double* d) {
  check_cuda(cudaMemcpy2D(d, a.nrow() * sizeof(double), a.valPtr(), a.pitch() * sizeof(double),
                          a.nrow() * sizeof(double), a.ncol(), cudaMemcpyHostToDevice), "cudaMemcpy2D");
}
inline void to_host(const double* d, DenseMatrixRowMajor<double>& a) {
  check_cuda(cudaMemcpy2D(a.valPtr(), a.pitch() * sizeof(double), d, a.ncol() * sizeof(double),
                          a.ncol() * sizeof(double), a.nrow(), cudaMemcpyDeviceToHost), "cudaMemcpy2D");
}
inline int layout_of(const DenseMatrixRowMajor<double>&) { return MCNLA_B200_ROW_MAJOR; }
inline int layout_of(const DenseMatrixColMajor<double>&) { return MCNLA_B200_COL_MAJOR; }
inline int64_t ld_of(const DenseMatrixRowMajor<double>& a) { return a.ncol(); }
inline int64_t ld_of(const DenseMatrixColMajor<double>& a) { return a.nrow(); }

}  // namespace b200

// ---- Gaussian projection sketcher (gaussian_projection_sketcher.hpp:65-103)
struct GaussianProjectionSketcherB200Tag {};
template <typename _Val>
using GaussianProjectionSketcherB200 = Sketcher<GaussianProjectionSketcherB200Tag, _Val>;
template <typename _Val>
using RowBlockGaussianProjectionSketcherB200 = Sketcher<GaussianProjectionSketcherB200Tag, _Val>;
template <typename _Val>
using ColBlockGaussianProjectionSketcherB200 = Sketcher<GaussianProjectionSketcherB200Tag, _Val>;

template <>
class Sketcher<GaussianProjectionSketcherB200Tag, double>
    : public StageWrapper<GaussianProjectionSketcherB200<double>> {
  friend StageWrapper<GaussianProjectionSketcherB200<double>>;
  using BaseType = StageWrapper<GaussianProjectionSketcherB200<double>>;

 protected:
  static constexpr const char* name_ = "Gaussian Projection Sketcher (B200)";
  static constexpr const char* names_ = "random generating / projection";
  index_t seed_;
  b200::DeviceBuffer a_, omega_, q_;
  using BaseType::parameters_;
  using BaseType::moments_;
  using BaseType::comm_times_;

 public:
  explicit Sketcher(const Parameters<double>& parameters, const index_t seed = 0) noexcept
      : BaseType(parameters), seed_(seed) {}
  index_t seed() const noexcept { return seed_; }
  Sketcher& setSeed(const index_t seed) noexcept {
    seed_ = seed;
    return *this;
  }

 protected:
  void initializeImpl() noexcept {
    const size_t m = parameters_.nrowRank(), n = parameters_.ncol(), L = parameters_.dimSketchTotal();
    a_.reserve(m * n);
    omega_.reserve(n * L);
    q_.reserve(m * L);
  }
  template <class _Matrix>
  void runImpl(const _Matrix& matrix_a, DenseMatrixCollectionColBlockRowMajor<double>& collection_q) noexcept {
    mcnla_b200_ctx* ctx = b200::context(parameters_);
    const mcnla_b200_params p = b200::params_of(parameters_);
    const int64_t n = parameters_.ncol(), L = parameters_.dimSketchTotal();
    double comm_time;
    this->tic(comm_time);
    b200::check(mcnla_b200_gaussian(ctx, uint64_t(seed_), n * L, omega_.p), "mcnla_b200_gaussian");
    this->toc(comm_time);
    b200::to_device(matrix_a, a_.p);
    b200::check(mcnla_b200_sketch(ctx, &p, a_.p, b200::layout_of(matrix_a), b200::ld_of(matrix_a), omega_.p, 0, q_.p),
                "mcnla_b200_sketch");
    auto qu = collection_q.unfold();
    b200::to_host(q_.p, qu);
    this->toc(comm_time);
  }
};

// ---- Gramian orthogonalizer (gramian_orthogonalizer.hpp:62-104, row-block form :62-105)
struct GramianOrthogonalizerB200Tag {};
template <typename _Val>
using GramianOrthogonalizerB200 = Orthogonalizer<GramianOrthogonalizerB200Tag, _Val>;
template <typename _Val>
using RowBlockGramianOrthogonalizerB200 = Orthogonalizer<GramianOrthogonalizerB200Tag, _Val>;

template <>
class Orthogonalizer<GramianOrthogonalizerB200Tag, double>
    : public StageWrapper<GramianOrthogonalizerB200<double>> {
  friend StageWrapper<GramianOrthogonalizerB200<double>>;
  using BaseType = StageWrapper<GramianOrthogonalizerB200<double>>;

 protected:
  static constexpr const char* name_ = "Gramian Orthogonalizer (B200)";
  static constexpr const char* names_ = "orthogonalization";
  b200::DeviceBuffer q_;
  using BaseType::parameters_;
  using BaseType::moments_;
  using BaseType::comm_times_;

 public:
  explicit Orthogonalizer(const Parameters<double>& parameters) noexcept : BaseType(parameters) {}

 protected:
  void initializeImpl() noexcept { q_.reserve(size_t(parameters_.nrowRank()) * parameters_.dimSketchTotal()); }
  void runImpl(DenseMatrixCollectionColBlockRowMajor<double>& collection_q) noexcept {
    const mcnla_b200_params p = b200::params_of(parameters_);
    double comm_time;
    this->tic(comm_time);
    auto qu = collection_q.unfold();
    b200::to_device(qu, q_.p);
    b200::check(mcnla_b200_orthogonalize(b200::context(parameters_), &p, q_.p), "mcnla_b200_orthogonalize");
    b200::to_host(q_.p, qu);
    this->toc(comm_time);
  }
};

// ---- integrators (include/mcnla/isvd/integrator/): _kind is one of the
// MCNLA_B200_*KOLMOGOROV_NAGUMO / *WEN_YIN enumerators
template <int _kind>
struct IntegratorB200Tag {};
template <typename _Val>
using KolmogorovNagumoIntegratorB200 = Integrator<IntegratorB200Tag<MCNLA_B200_KOLMOGOROV_NAGUMO>, _Val>;
template <typename _Val>
using RowBlockKolmogorovNagumoIntegratorB200 =
    Integrator<IntegratorB200Tag<MCNLA_B200_ROW_BLOCK_KOLMOGOROV_NAGUMO>, _Val>;
template <typename _Val>
using RowBlockGramianKolmogorovNagumoIntegratorB200 =
    Integrator<IntegratorB200Tag<MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO>, _Val>;
template <typename _Val>
using RowBlockWenYinIntegratorB200 = Integrator<IntegratorB200Tag<MCNLA_B200_ROW_BLOCK_WEN_YIN>, _Val>;
template <typename _Val>
using RowBlockGramianWenYinIntegratorB200 = Integrator<IntegratorB200Tag<MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN>, _Val>;

template <int _kind>
class Integrator<IntegratorB200Tag<_kind>, double> : public StageWrapper<Integrator<IntegratorB200Tag<_kind>, double>> {
  friend StageWrapper<Integrator<IntegratorB200Tag<_kind>, double>>;
  using BaseType = StageWrapper<Integrator<IntegratorB200Tag<_kind>, double>>;

 protected:
  static constexpr const char* name_ = "Integrator (B200)";
  static constexpr const char* names_ = "copying in / iterating / copying out";
  index_t max_iteration_;
  double tolerance_;
  index_t iteration_ = -1;
  b200::DeviceBuffer q_, qbar_;
  using BaseType::parameters_;
  using BaseType::moments_;
  using BaseType::comm_times_;

 public:
  explicit Integrator(const Parameters<double>& parameters, const index_t max_iteration = 256,
                      const double tolerance = (_kind == MCNLA_B200_ROW_BLOCK_WEN_YIN ||
                                                _kind == MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN) ? 1e-3 : 1e-4) noexcept
      : BaseType(parameters), max_iteration_(max_iteration), tolerance_(tolerance) {}
  index_t maxIteration() const noexcept { return max_iteration_; }
  double tolerance() const noexcept { return tolerance_; }
  index_t iteration() const noexcept { return iteration_; }
  Integrator& setMaxIteration(const index_t max_iteration) noexcept {
    max_iteration_ = max_iteration;
    return *this;
  }
  Integrator& setTolerance(const double tolerance) noexcept {
    tolerance_ = tolerance;
    return *this;
  }

 protected:
  void initializeImpl() noexcept {
    const size_t m = parameters_.nrowRank();
    q_.reserve(m * parameters_.dimSketchTotal());
    qbar_.reserve(m * parameters_.dimSketch());
  }
  void runImpl(const DenseMatrixCollectionColBlockRowMajor<double>& collection_q,
               DenseMatrixRowMajor<double>& matrix_qbar) noexcept {
    const mcnla_b200_params p = b200::params_of(parameters_);
    double comm_time;
    this->tic(comm_time);
    b200::to_device(collection_q.unfold(), q_.p);
    this->toc(comm_time);
    int it = 0;
    b200::check(mcnla_b200_integrate(b200::context(parameters_), &p, _kind, q_.p, int(max_iteration_), tolerance_, qbar_.p, &it),
                "mcnla_b200_integrate");
    iteration_ = it;
    this->toc(comm_time);
    b200::to_host(qbar_.p, matrix_qbar);
    this->toc(comm_time);
  }
};

// ---- formers with V (svd_former.hpp:70-116, gramian_former.hpp:72-132,
// row_block_gramian_former.hpp:78-146, col_block_gramian_former.hpp:73-131):
// _kind is one of the MCNLA_B200_*_FORMER enumerators
template <int _kind>
struct FormerB200Tag {};
template <typename _Val>
using SvdFormerB200 = Former<FormerB200Tag<MCNLA_B200_SVD_FORMER>, _Val>;
template <typename _Val>
using GramianFormerB200 = Former<FormerB200Tag<MCNLA_B200_GRAMIAN_FORMER>, _Val>;
template <typename _Val>
using RowBlockGramianFormerB200 = Former<FormerB200Tag<MCNLA_B200_ROW_BLOCK_GRAMIAN_FORMER>, _Val>;
template <typename _Val>
using ColBlockGramianFormerB200 = Former<FormerB200Tag<MCNLA_B200_COL_BLOCK_GRAMIAN_FORMER>, _Val>;

template <int _kind>
class Former<FormerB200Tag<_kind>, double> : public StageWrapper<Former<FormerB200Tag<_kind>, double>> {
  friend StageWrapper<Former<FormerB200Tag<_kind>, double>>;
  using BaseType = StageWrapper<Former<FormerB200Tag<_kind>, double>>;

 protected:
  static constexpr const char* name_ = "Former (B200)";
  static constexpr const char* names_ = "forming";
  b200::DeviceBuffer a_, qbar_, s_, u_, v_;
  DenseVector<double> vector_s_;
  DenseMatrixRowMajor<double> matrix_u_, matrix_v_;
  using BaseType::parameters_;
  using BaseType::moments_;
  using BaseType::comm_times_;

 public:
  explicit Former(const Parameters<double>& parameters) noexcept : BaseType(parameters) {}
  const DenseVector<double>& vectorS() const noexcept { return vector_s_; }
  const DenseMatrixRowMajor<double>& matrixU() const noexcept { return matrix_u_; }
  const DenseMatrixRowMajor<double>& matrixV() const noexcept { return matrix_v_; }
  const DenseMatrixRowMajor<double>& matrixUj() const noexcept { return matrix_u_; }
  const DenseMatrixRowMajor<double>& matrixVj() const noexcept { return matrix_v_; }

 protected:
  void initializeImpl() noexcept {
    const size_t m = parameters_.nrowRank(), n = parameters_.ncol(), k = parameters_.rank();
    a_.reserve(m * n);
    qbar_.reserve(m * parameters_.dimSketch());
    s_.reserve(k);
    u_.reserve(m * k);
    v_.reserve(n * k);
    vector_s_.reconstruct(k);
    matrix_u_.reconstruct(m, k);
    matrix_v_.reconstruct(n, k);
  }
  template <class _Matrix>
  void runImpl(const _Matrix& matrix_a, const DenseMatrixRowMajor<double>& matrix_qbar) noexcept {
    const mcnla_b200_params p = b200::params_of(parameters_);
    double comm_time;
    this->tic(comm_time);
    b200::to_device(matrix_a, a_.p);
    b200::to_device(matrix_qbar, qbar_.p);
    b200::check(mcnla_b200_form(b200::context(parameters_), &p, _kind, a_.p, b200::layout_of(matrix_a), b200::ld_of(matrix_a),
                                qbar_.p, s_.p, u_.p, v_.p), "mcnla_b200_form");
    b200::check_cuda(cudaMemcpy(vector_s_.valPtr(), s_.p, vector_s_.len() * sizeof(double), cudaMemcpyDeviceToHost),
                     "cudaMemcpy");
    b200::to_host(u_.p, matrix_u_);
    b200::to_host(v_.p, matrix_v_);
    this->toc(comm_time);
  }
};

}  // namespace isvd
}  // namespace mcnla

#endif  // MCNLA_B200_MCNLA_TAGS_HPP_
