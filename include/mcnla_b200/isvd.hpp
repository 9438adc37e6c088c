// C++ stage API of the B200 iSVD: the reference's mcnla::isvd classes
// (Parameters, the Sketcher / Orthogonalizer / Integrator / Former stages with
// initialize(), operator(), time(), times(), iteration(), vectorS(), matrixU(),
// matrixV()), over the C ABI of mcnla_b200.h.  Header-only C++14; link
// libmcnla_b200.so and the CUDA runtime.
//
// Differences from the reference, all forced by the one-GPU design:
//  * matrices are device buffers (DeviceMatrix: pointer, sizes, leading
//    dimension, layout), not host DenseMatrix objects; the reference's
//    row-major / column-major distinction is the `layout` field;
//  * the stages throw mcnla_b200::Error on a non-zero status where the
//    reference asserts;
//  * MPI arguments are absent (one rank; sketches and row blocks are batched
//    on the device).
// Reference: include/mcnla/isvd/core/parameters.hh:31-119,
// include/mcnla/isvd/core/stage_wrapper.hh:35-101, and the stage headers cited
// per class below.
#ifndef MCNLA_B200_ISVD_HPP_
#define MCNLA_B200_ISVD_HPP_

#include <mcnla_b200.h>
#include <cuda_runtime.h>

#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace mcnla_b200 {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what)
      : std::runtime_error(what + ": " + mcnla_b200_status_string(status) +
                           (status == MCNLA_B200_ERR_CUDA ? std::string(" (") + mcnla_b200_last_error() + ")" : "")),
        status_(status) {}
  int status() const noexcept { return status_; }

 private:
  int status_;
};

inline void check(int status, const char* what) {
  if (status != MCNLA_B200_OK) throw Error(status, what);
}

// A device matrix view (no ownership): element (i, j) at p[i*ld + j]
// (row-major) or p[i + j*ld] (column-major).
struct DeviceMatrix {
  double* p = nullptr;
  int64_t nrow = 0, ncol = 0, ld = 0;
  int layout = MCNLA_B200_ROW_MAJOR;
};

// An owning device buffer (row-major unless stated).
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  DeviceBuffer(int64_t nrow, int64_t ncol, int layout = MCNLA_B200_ROW_MAJOR) { reconstruct(nrow, ncol, layout); }
  void reconstruct(int64_t nrow, int64_t ncol, int layout = MCNLA_B200_ROW_MAJOR) {
    double* p = nullptr;
    if (nrow * ncol > 0 && cudaMalloc(&p, sizeof(double) * nrow * ncol) != cudaSuccess)
      throw Error(MCNLA_B200_ERR_NOMEM, "DeviceBuffer");
    mem_.reset(p, [](double* q) { cudaFree(q); });
    view_.p = p;
    view_.nrow = nrow;
    view_.ncol = ncol;
    view_.ld = layout == MCNLA_B200_ROW_MAJOR ? ncol : nrow;
    view_.layout = layout;
  }
  const DeviceMatrix& view() const noexcept { return view_; }
  operator const DeviceMatrix&() const noexcept { return view_; }
  double* data() const noexcept { return view_.p; }
  int64_t nrow() const noexcept { return view_.nrow; }
  int64_t ncol() const noexcept { return view_.ncol; }
  std::vector<double> host() const {
    std::vector<double> h(size_t(view_.nrow * view_.ncol));
    check(cudaMemcpy(h.data(), view_.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess
              ? MCNLA_B200_OK : MCNLA_B200_ERR_CUDA, "DeviceBuffer::host");
    return h;
  }
  void upload(const std::vector<double>& h) {
    check(cudaMemcpy(view_.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess
              ? MCNLA_B200_OK : MCNLA_B200_ERR_CUDA, "DeviceBuffer::upload");
  }

 private:
  std::shared_ptr<double> mem_;
  DeviceMatrix view_;
};

// One context per device and stream (mcnla_b200_create).
class Context {
 public:
  explicit Context(int device = 0, cudaStream_t stream = nullptr) {
    mcnla_b200_ctx* c = nullptr;
    check(mcnla_b200_create(&c, device, stream), "mcnla_b200_create");
    ctx_.reset(c, [](mcnla_b200_ctx* q) { mcnla_b200_destroy(q); });
  }
  mcnla_b200_ctx* get() const noexcept { return ctx_.get(); }

 private:
  std::shared_ptr<mcnla_b200_ctx> ctx_;
};

// mcnla::isvd::Parameters (parameters.hh:31-119)
class Parameters {
 public:
  explicit Parameters(Context ctx = Context()) : ctx_(std::move(ctx)) {}
  Parameters& setSize(int64_t nrow, int64_t ncol) { p_.nrow = nrow; p_.ncol = ncol; sync_ = false; return *this; }
  Parameters& setSize(const DeviceMatrix& a) { return setSize(a.nrow, a.ncol); }
  Parameters& setRank(int64_t rank) { p_.rank = rank; sync_ = false; return *this; }
  Parameters& setOverRank(int64_t over_rank) { p_.over_rank = over_rank; sync_ = false; return *this; }
  Parameters& setNumSketch(int64_t num_sketch) { p_.num_sketch = num_sketch; sync_ = false; return *this; }
  Parameters& setNumSketchEach(int64_t num_sketch_each) { return setNumSketch(num_sketch_each); }
  Parameters& sync() {
    if (p_.nrow <= 0 || p_.ncol <= 0 || p_.rank <= 0 || p_.over_rank < 0 || p_.num_sketch <= 0)
      throw Error(MCNLA_B200_ERR_SHAPE, "Parameters::sync");
    if (dimSketch() > MCNLA_B200_MAX_DIM_SKETCH) throw Error(MCNLA_B200_ERR_UNSUPPORTED, "Parameters::sync");
    sync_ = true;
    return *this;
  }
  bool isSynchronized() const noexcept { return sync_; }
  int64_t nrow() const noexcept { return p_.nrow; }
  int64_t ncol() const noexcept { return p_.ncol; }
  int64_t nrowRank() const noexcept { return p_.nrow; }
  int64_t ncolRank() const noexcept { return p_.ncol; }
  int64_t rank() const noexcept { return p_.rank; }
  int64_t overRank() const noexcept { return p_.over_rank; }
  int64_t dimSketch() const noexcept { return p_.rank + p_.over_rank; }
  int64_t numSketch() const noexcept { return p_.num_sketch; }
  int64_t numSketchEach() const noexcept { return p_.num_sketch; }
  int64_t dimSketchTotal() const noexcept { return dimSketch() * p_.num_sketch; }
  int64_t dimSketchEach() const noexcept { return dimSketchTotal(); }
  DeviceBuffer createCollectionQ() const { return DeviceBuffer(p_.nrow, dimSketchTotal()); }
  DeviceBuffer createCollectionQj() const { return createCollectionQ(); }
  DeviceBuffer createMatrixQbar() const { return DeviceBuffer(p_.nrow, dimSketch()); }
  DeviceBuffer createMatrixQbarj() const { return createMatrixQbar(); }
  const mcnla_b200_params& c() const noexcept { return p_; }
  mcnla_b200_ctx* ctx() const noexcept { return ctx_.get(); }

 private:
  Context ctx_;
  mcnla_b200_params p_{0, 0, 0, 12, 16};   // defaults: parameters.hh:63-66
  bool sync_ = false;
};

// mcnla::isvd::StageWrapper (stage_wrapper.hh:35-101)
template <class Derived>
class StageWrapper {
 public:
  explicit StageWrapper(const Parameters& p) : parameters_(p) {}
  void initialize() {
    if (!parameters_.isSynchronized()) throw Error(MCNLA_B200_ERR_ARG, "initialize: parameters not synchronized");
    check(mcnla_b200_initialize(parameters_.ctx(), &parameters_.c(), -1, -1), "initialize");
    initialized_ = true;
    computed_ = false;
  }
  template <class... Args>
  void operator()(Args&&... args) {
    if (!initialized_) throw Error(MCNLA_B200_ERR_ARG, "stage not initialized");
    static_cast<Derived*>(this)->runImpl(std::forward<Args>(args)...);
    double t[16];
    const int n = mcnla_b200_last_times(parameters_.ctx(), t, 16);
    times_.assign(t, t + (n > 0 ? n : 0));
    computed_ = true;
  }
  bool isInitialized() const noexcept { return initialized_; }
  bool isComputed() const noexcept { return computed_; }
  double time() const noexcept { return std::accumulate(times_.begin(), times_.end(), 0.0); }
  std::vector<double> times() const { return times_; }
  double commTime() const noexcept { return 0.0; }

 protected:
  const Parameters& parameters_;
  bool initialized_ = false, computed_ = false;
  std::vector<double> times_;
};

// ---- sketchers (include/mcnla/isvd/sketcher/gaussian_projection_sketcher.hpp:65-103 and
//      the row-block / column-block variants)
class GaussianProjectionSketcher : public StageWrapper<GaussianProjectionSketcher> {
 public:
  static constexpr const char* name_ = "Gaussian Projection Sketcher";
  static constexpr const char* names_ = "random generating / projection";
  GaussianProjectionSketcher(const Parameters& p, uint64_t seed = 0, int exponent = 0)
      : StageWrapper(p), seed_(seed), exponent_(exponent) {}
  GaussianProjectionSketcher& setSeed(uint64_t s) { seed_ = s; computed_ = false; return *this; }
  GaussianProjectionSketcher& setExponent(int e) { exponent_ = e; computed_ = false; return *this; }
  // Uses the given n x (N l) row-major Omega (device) instead of drawing one.
  GaussianProjectionSketcher& setOmega(double* omega) { omega_given_ = omega; return *this; }
  uint64_t seed() const noexcept { return seed_; }
  int exponent() const noexcept { return exponent_; }
  void runImpl(const DeviceMatrix& a, DeviceBuffer& q) {
    const auto& c = parameters_.c();
    double* om = omega_given_;
    if (!om || exponent_ > 0) {
      omega_.reconstruct(c.ncol, parameters_.dimSketchTotal());
      if (om) {
        check(cudaMemcpy(omega_.data(), om, sizeof(double) * c.ncol * parameters_.dimSketchTotal(),
                         cudaMemcpyDeviceToDevice) == cudaSuccess ? MCNLA_B200_OK : MCNLA_B200_ERR_CUDA, "sketch");
      } else {
        check(mcnla_b200_gaussian(parameters_.ctx(), seed_, c.ncol * parameters_.dimSketchTotal(), omega_.data()),
              "gaussian");
      }
      om = omega_.data();
    }
    check(mcnla_b200_sketch(parameters_.ctx(), &c, a.p, a.layout, a.ld, om, exponent_, q.data()), "sketch");
  }

 private:
  uint64_t seed_;
  int exponent_;
  double* omega_given_ = nullptr;
  DeviceBuffer omega_;
};
using RowBlockGaussianProjectionSketcher = GaussianProjectionSketcher;
using ColBlockGaussianProjectionSketcher = GaussianProjectionSketcher;

// ---- orthogonalizers (include/mcnla/isvd/orthogonalizer/gramian_orthogonalizer.hpp:62-104)
class GramianOrthogonalizer : public StageWrapper<GramianOrthogonalizer> {
 public:
  static constexpr const char* name_ = "Gramian Orthogonalizer";
  static constexpr const char* names_ = "orthogonalization";
  using StageWrapper::StageWrapper;
  void runImpl(DeviceBuffer& q) { check(mcnla_b200_orthogonalize(parameters_.ctx(), &parameters_.c(), q.data()), "orthogonalize"); }
};
using RowBlockGramianOrthogonalizer = GramianOrthogonalizer;

// ---- integrators (include/mcnla/isvd/integrator/)
template <int Kind>
class IntegratorStage : public StageWrapper<IntegratorStage<Kind>> {
  using Base = StageWrapper<IntegratorStage<Kind>>;

 public:
  IntegratorStage(const Parameters& p, int max_iteration = 256,
                  double tolerance = (Kind >= MCNLA_B200_ROW_BLOCK_WEN_YIN ? 1e-3 : 1e-4))
      : Base(p), max_iteration_(max_iteration), tolerance_(tolerance) {}
  int maxIteration() const noexcept { return max_iteration_; }
  double tolerance() const noexcept { return tolerance_; }
  int iteration() const noexcept { return iteration_; }
  IntegratorStage& setMaxIteration(int m) { max_iteration_ = m; this->computed_ = false; return *this; }
  IntegratorStage& setTolerance(double t) { tolerance_ = t; this->computed_ = false; return *this; }
  void runImpl(const DeviceBuffer& q, DeviceBuffer& qbar) {
    check(mcnla_b200_integrate(this->parameters_.ctx(), &this->parameters_.c(), Kind, q.data(), max_iteration_,
                               tolerance_, qbar.data(), &iteration_), "integrate");
  }

 private:
  int max_iteration_;
  double tolerance_;
  int iteration_ = 0;
};
using KolmogorovNagumoIntegrator = IntegratorStage<MCNLA_B200_KOLMOGOROV_NAGUMO>;
using RowBlockKolmogorovNagumoIntegrator = IntegratorStage<MCNLA_B200_ROW_BLOCK_KOLMOGOROV_NAGUMO>;
using RowBlockGramianKolmogorovNagumoIntegrator = IntegratorStage<MCNLA_B200_ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO>;
using RowBlockWenYinIntegrator = IntegratorStage<MCNLA_B200_ROW_BLOCK_WEN_YIN>;
using RowBlockGramianWenYinIntegrator = IntegratorStage<MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN>;

// ---- formers (include/mcnla/isvd/former/), all with V
template <int Kind>
class FormerStage : public StageWrapper<FormerStage<Kind>> {
  using Base = StageWrapper<FormerStage<Kind>>;

 public:
  using Base::Base;
  void runImpl(const DeviceMatrix& a, const DeviceBuffer& qbar) {
    const auto& c = this->parameters_.c();
    s_.reconstruct(c.rank, 1);
    u_.reconstruct(c.nrow, c.rank);
    v_.reconstruct(c.ncol, c.rank);
    check(mcnla_b200_form(this->parameters_.ctx(), &c, Kind, a.p, a.layout, a.ld, qbar.data(), s_.data(), u_.data(),
                          v_.data()), "form");
  }
  const DeviceBuffer& vectorS() const noexcept { return s_; }
  const DeviceBuffer& matrixU() const noexcept { return u_; }
  const DeviceBuffer& matrixV() const noexcept { return v_; }
  const DeviceBuffer& matrixUj() const noexcept { return u_; }
  const DeviceBuffer& matrixVj() const noexcept { return v_; }

 private:
  DeviceBuffer s_, u_, v_;
};
using SvdFormer = FormerStage<MCNLA_B200_SVD_FORMER>;
using GramianFormer = FormerStage<MCNLA_B200_GRAMIAN_FORMER>;
using RowBlockGramianFormer = FormerStage<MCNLA_B200_ROW_BLOCK_GRAMIAN_FORMER>;
using ColBlockGramianFormer = FormerStage<MCNLA_B200_COL_BLOCK_GRAMIAN_FORMER>;

// Dense files with the reference's names (include/mcnla/core/io/): host
// matrices as std::vector<double> in the requested layout; a 3-D MatrixMarket
// collection is its unfolded m x (n l) matrix.
namespace io {

struct HostMatrix {
  std::vector<double> val;
  int64_t nrow = 0, ncol = 0;
  int layout = MCNLA_B200_ROW_MAJOR;   // leading dimension ncol (row-major) or nrow (column-major)
};

// (m, n, l) of a dense MatrixMarket file (matrix_market/dense_load_block.hpp:13-29)
inline std::vector<int64_t> loadMatrixMarketSize(const char* file) {
  std::vector<int64_t> dims(3);
  int nd = 0;
  check(mcnla_b200_mm_size(file, dims.data(), &nd), "loadMatrixMarketSize");
  return dims;
}

// rows [row0, row0 + rows) x columns [col0, col0 + cols); rows < 0 / cols < 0: to the end
inline HostMatrix loadMatrixMarketBlock(const char* file, int64_t row0, int64_t rows, int64_t col0, int64_t cols,
                                        int layout = MCNLA_B200_ROW_MAJOR) {
  const std::vector<int64_t> d = loadMatrixMarketSize(file);
  HostMatrix a;
  a.nrow = rows < 0 ? d[0] - row0 : rows;
  a.ncol = cols < 0 ? d[1] * d[2] - col0 : cols;
  a.layout = layout;
  a.val.resize(size_t(a.nrow * a.ncol));
  const int64_t ld = layout == MCNLA_B200_ROW_MAJOR ? a.ncol : a.nrow;
  check(mcnla_b200_mm_load(file, row0, a.nrow, col0, a.ncol, a.val.data(), ld > 0 ? ld : 1, layout),
        "loadMatrixMarket");
  return a;
}

// matrix_market/dense_load.hpp:70-251
inline HostMatrix loadMatrixMarket(const char* file, int layout = MCNLA_B200_ROW_MAJOR) {
  return loadMatrixMarketBlock(file, 0, -1, 0, -1, layout);
}
// matrix_market/dense_load_block.hpp:86-130 (row-major rows) and :31-74 (column-major columns)
inline HostMatrix loadMatrixMarketRowBlock(const char* file, int64_t row0, int64_t rows) {
  return loadMatrixMarketBlock(file, row0, rows, 0, -1, MCNLA_B200_ROW_MAJOR);
}
inline HostMatrix loadMatrixMarketColBlock(const char* file, int64_t col0, int64_t cols) {
  return loadMatrixMarketBlock(file, 0, -1, col0, cols, MCNLA_B200_COL_MAJOR);
}

// matrix_market/dense_save.hpp (nmat > 1: a 3-D collection)
inline void saveMatrixMarket(const HostMatrix& a, const char* file, int64_t nmat = 1, const char* comment = nullptr) {
  const int64_t ld = a.layout == MCNLA_B200_ROW_MAJOR ? a.ncol : a.nrow;
  check(mcnla_b200_mm_save(file, a.val.data(), a.nrow, a.ncol / nmat, nmat, ld > 0 ? ld : 1, a.layout, comment),
        "saveMatrixMarket");
}

// binary/dense_load.hpp:52-86 for a matrix: dims {ncol, nrow} hold a row-major
// matrix, {nrow, ncol} a column-major one (layout says which the file is)
inline HostMatrix loadBinary(const char* file, int layout = MCNLA_B200_ROW_MAJOR) {
  int64_t dims[3];
  int nd = 0;
  char vt[9];
  check(mcnla_b200_binary_size(file, dims, &nd, vt), "loadBinary");
  if (nd != 2) throw Error(MCNLA_B200_ERR_SHAPE, "loadBinary: not a matrix");
  HostMatrix a;
  a.layout = layout;
  a.nrow = layout == MCNLA_B200_ROW_MAJOR ? dims[1] : dims[0];
  a.ncol = layout == MCNLA_B200_ROW_MAJOR ? dims[0] : dims[1];
  a.val.resize(size_t(dims[0] * dims[1]));
  check(mcnla_b200_binary_load(file, 0, dims[1], a.val.data()), "loadBinary");
  return a;
}

// binary/dense_save.hpp:60-100
inline void saveBinary(const HostMatrix& a, const char* file, const char* comment = nullptr) {
  const int64_t dims[2] = {a.layout == MCNLA_B200_ROW_MAJOR ? a.ncol : a.nrow,
                           a.layout == MCNLA_B200_ROW_MAJOR ? a.nrow : a.ncol};
  check(mcnla_b200_binary_save(file, a.val.data(), 2, dims, comment), "saveBinary");
}

}  // namespace io

}  // namespace mcnla_b200

#endif  // MCNLA_B200_ISVD_HPP_
