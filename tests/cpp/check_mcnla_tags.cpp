// The reference's own stage templates run with the B200 tags of
// include/mcnla_b200/mcnla_tags.hpp, next to the reference's CPU stages on the
// same inputs (the reference's data/*.mtx fixtures, passed as raw little-endian
// float64 files by tests/test_reference_binding.py from
// tests/golden/mcnla_data.npz).  Checks, as the reference's own tests do
// (check/isvd/integrator/*.cpp, check/isvd/orthogonalizer/*.cpp,
// check/isvd/former/*.cpp): the row-block Gramian and plain KN integrators
// stop after 81 iterations with Qbar within 1e-8 of qb_kn; the Gramian
// orthogonalizer's and the formers' results agree with the CPU stages; and with
// the MPI row-block attachment (a one-rank NCCL communicator) the row-block
// integrators still agree while their sums go through the communicator.
// Built by oracle/Makefile (it includes the reference headers); test
// infrastructure, not part of the product.
#include <limits>
#include <mcnla/isvd.hpp>
#include <mcnla_b200/mcnla_tags.hpp>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

namespace {

int failures = 0;
#define EXPECT(cond, ...)                                  \
  do {                                                     \
    if (!(cond)) {                                         \
      std::printf("FAILED %s:%d: ", __FILE__, __LINE__);   \
      std::printf(__VA_ARGS__);                            \
      std::printf("\n");                                   \
      ++failures;                                          \
    }                                                      \
  } while (0)

std::vector<double> load(const std::string& path, size_t count) {
  std::vector<double> v(count);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), std::streamsize(count * sizeof(double)));
  if (!f) { std::printf("cannot read %s\n", path.c_str()); std::exit(2); }
  return v;
}

template <class Mat>
void fill(Mat& a, const std::vector<double>& v, int rows, int cols) {   // v row-major
  for (int i = 0; i < rows; ++i)
    for (int j = 0; j < cols; ++j) a(i, j) = v[size_t(i) * cols + j];
}

template <class M1, class M2>
double max_diff(const M1& a, const M2& b, int rows, int cols, bool up_to_sign = false) {
  double mx = 0;
  for (int j = 0; j < cols; ++j) {
    double sg = 1;
    if (up_to_sign) {
      double dot = 0;
      for (int i = 0; i < rows; ++i) dot += a(i, j) * b(i, j);
      sg = dot < 0 ? -1 : 1;
    }
    for (int i = 0; i < rows; ++i) mx = std::max(mx, std::fabs(sg * a(i, j) - b(i, j)));
  }
  return mx;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) { std::printf("usage: %s <fixture dir>\n", argv[0]); return 2; }
  const std::string dir = argv[1];
  // fixture sizes: qi 12 sketches of 101 x 11 (unfolded 101 x 132), a 101 x 1001, q 101 x 11
  const int m = 101, l = 11, N = 12, n = 1001;
  const auto qs = load(dir + "/qs.bin", size_t(m) * N * l);
  const auto ys = load(dir + "/ys.bin", size_t(m) * N * l);
  const auto qb = load(dir + "/qb_kn.bin", size_t(m) * l);
  const auto av = load(dir + "/a.bin", size_t(m) * n);
  const auto qv = load(dir + "/q.bin", size_t(m) * l);

  using namespace mcnla;
  isvd::Parameters<double> prm(0, MPI_COMM_WORLD);
  prm.setSize(m, l).setRank(l).setOverRank(0).setNumSketch(N);
  prm.sync();
  matrix::DenseMatrixRowMajor<double> qb_ref(m, l);
  fill(qb_ref, qb, m, l);

  // ---- integrators: the row-block Gramian KN (ITYPE of the row-block driver) and the plain KN
  {
    auto q = prm.createCollectionQj();
    fill(q.unfold(), qs, m, N * l);
    auto qbar_b = prm.createMatrixQbarj();
    auto qbar_c = prm.createMatrixQbarj();
    isvd::RowBlockGramianKolmogorovNagumoIntegratorB200<double> gpu(prm, 256, 1e-4);
    isvd::RowBlockGramianKolmogorovNagumoIntegrator<double> cpu(prm, 256, 1e-4);
    gpu.initialize();
    cpu.initialize();
    gpu(q, qbar_b);
    cpu(q, qbar_c);
    std::printf("rb_gramian_kn B200 iterations %d, reference %d, |Qbar - qb_kn| %.3e, |Qbar - reference| %.3e\n",
                int(gpu.iteration()), int(cpu.iteration()), max_diff(qbar_b, qb_ref, m, l),
                max_diff(qbar_b, qbar_c, m, l));
    EXPECT(gpu.iteration() == 81, "iterations %d", int(gpu.iteration()));
    EXPECT(gpu.iteration() == cpu.iteration(), "iterations %d vs %d", int(gpu.iteration()), int(cpu.iteration()));
    EXPECT(max_diff(qbar_b, qb_ref, m, l) < 1e-8, "Qbar vs the fixture");
    EXPECT(max_diff(qbar_b, qbar_c, m, l) < 1e-10, "Qbar vs the CPU stage");
    std::printf("stage parts: %s; times:", gpu.names());
    for (double t : gpu.times()) std::printf(" %.4f", t);
    std::printf("\n");
  }
  {
    auto q = prm.createCollectionQ();
    fill(q.unfold(), qs, m, N * l);
    auto qbar_b = prm.createMatrixQbar();
    isvd::KolmogorovNagumoIntegratorB200<double> gpu(prm, 256, 1e-4);
    gpu.initialize();
    gpu(q, qbar_b);
    std::printf("kn B200 iterations %d, |Qbar - qb_kn| %.3e, time %.4f s\n", int(gpu.iteration()),
                max_diff(qbar_b, qb_ref, m, l), gpu.time());
    EXPECT(gpu.iteration() == 81, "iterations %d", int(gpu.iteration()));
    EXPECT(max_diff(qbar_b, qb_ref, m, l) < 1e-8, "Qbar vs the fixture");
  }
  // ---- Gramian orthogonalizer on the fixture's sketches
  {
    auto qg = prm.createCollectionQj();
    auto qc = prm.createCollectionQj();
    fill(qg.unfold(), ys, m, N * l);
    fill(qc.unfold(), ys, m, N * l);
    isvd::RowBlockGramianOrthogonalizerB200<double> gpu(prm);
    isvd::RowBlockGramianOrthogonalizer<double> cpu(prm);
    gpu.initialize();
    cpu.initialize();
    gpu(qg);
    cpu(qc);
    const double d = max_diff(qg.unfold(), qc.unfold(), m, N * l, true);
    std::printf("orthogonalizer B200 vs reference %.3e\n", d);
    EXPECT(d < 1e-10, "orthogonalizer %.3e", d);
  }
  // ---- formers on a (101 x 1001) with the fixture's q
  {
    isvd::Parameters<double> pf(0, MPI_COMM_WORLD);
    pf.setSize(m, n).setRank(5).setOverRank(l - 5).setNumSketch(1);
    pf.sync();
    matrix::DenseMatrixRowMajor<double> a(m, n);
    fill(a, av, m, n);
    auto qbar = pf.createMatrixQbar();
    fill(qbar, qv, m, l);
    isvd::SvdFormerB200<double> gs(pf);
    isvd::SvdFormer<double, true> cs(pf);
    isvd::RowBlockGramianFormerB200<double> gg(pf);
    isvd::RowBlockGramianFormer<double, true> cg(pf);
    gs.initialize(); cs.initialize(); gg.initialize(); cg.initialize();
    gs(a, qbar); cs(a, qbar); gg(a, qbar); cg(a, qbar);
    double ds = 0, dg = 0;
    for (int i = 0; i < 5; ++i) {
      ds = std::max(ds, std::fabs(gs.vectorS()(i) - cs.vectorS()(i)) / cs.vectorS()(0));
      dg = std::max(dg, std::fabs(gg.vectorS()(i) - cg.vectorS()(i)) / cg.vectorS()(0));
    }
    const double du = max_diff(gs.matrixU(), cs.matrixU(), m, 5, true);
    const double dv = max_diff(gg.matrixVj(), cg.matrixVj(), n, 5, true);
    std::printf("svd former sigma %.3e U %.3e; row-block Gramian former sigma %.3e V %.3e\n", ds, du, dg, dv);
    EXPECT(ds < 1e-10 && du < 1e-10, "svd former");
    EXPECT(dg < 1e-10 && dv < 1e-10, "Gramian former");
  }
  // ---- sketcher (Omega from the device generator: shape and finiteness)
  {
    isvd::Parameters<double> ps(0, MPI_COMM_WORLD);
    ps.setSize(m, n).setRank(5).setOverRank(3).setNumSketch(4);
    ps.sync();
    matrix::DenseMatrixRowMajor<double> a(m, n);
    fill(a, av, m, n);
    auto q = ps.createCollectionQj();
    isvd::RowBlockGaussianProjectionSketcherB200<double> sk(ps, 7);
    sk.initialize();
    sk(a, q);
    double nrm = 0;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < 32; ++j) nrm += q.unfold()(i, j) * q.unfold()(i, j);
    std::printf("sketch ||Q||_F^2 %.3e\n", nrm);
    EXPECT(std::isfinite(nrm) && nrm > 0, "sketch");
  }
  // ---- the MPI row-block attachment (last: the device's context keeps it), at one rank:
  // the stages' sums now go through the library's NCCL communicator.  The row-block KN
  // integrator sums its row-dependent products every iteration
  // (row_block_kolmogorov_nagumo_integrator.hpp:115, :143), the Gramian one its Gramian once
  // (row_block_gramian_kolmogorov_nagumo_integrator.hpp:117); both must still match the CPU
  // stages, and the context counts the all-reduces.
  {
    mcnla_b200_ctx* ctx = isvd::b200::context();
    isvd::b200::attach_ranks(prm, ctx, /*force=*/true);
    auto q = prm.createCollectionQj();
    fill(q.unfold(), qs, m, N * l);
    auto qbar_b = prm.createMatrixQbarj();
    auto qbar_c = prm.createMatrixQbarj();
    int64_t before = mcnla_b200_allreduces(ctx);
    isvd::RowBlockKolmogorovNagumoIntegratorB200<double> gpu(prm, 256, 1e-4);
    isvd::RowBlockKolmogorovNagumoIntegrator<double> cpu(prm, 256, 1e-4);
    gpu.initialize();
    cpu.initialize();
    gpu(q, qbar_b);
    cpu(q, qbar_c);
    int64_t sums = mcnla_b200_allreduces(ctx) - before;
    std::printf("rb_kn over a one-rank NCCL communicator: iterations %d (reference %d), all-reduces %lld, "
                "|Qbar - reference| %.3e\n", int(gpu.iteration()), int(cpu.iteration()),
                static_cast<long long>(sums), max_diff(qbar_b, qbar_c, m, l));
    EXPECT(gpu.iteration() == cpu.iteration(), "iterations %d vs %d", int(gpu.iteration()), int(cpu.iteration()));
    EXPECT(max_diff(qbar_b, qbar_c, m, l) < 1e-10, "Qbar vs the CPU stage");
    EXPECT(sums >= gpu.iteration(), "all-reduces %lld", static_cast<long long>(sums));

    before = mcnla_b200_allreduces(ctx);
    isvd::RowBlockGramianKolmogorovNagumoIntegratorB200<double> gg(prm, 256, 1e-4);
    gg.initialize();
    gg(q, qbar_b);
    sums = mcnla_b200_allreduces(ctx) - before;
    std::printf("rb_gramian_kn over it: iterations %d, all-reduces %lld, |Qbar - qb_kn| %.3e\n", int(gg.iteration()),
                static_cast<long long>(sums), max_diff(qbar_b, qb_ref, m, l));
    EXPECT(gg.iteration() == 81, "iterations %d", int(gg.iteration()));
    EXPECT(max_diff(qbar_b, qb_ref, m, l) < 1e-8, "Qbar vs the fixture");
    EXPECT(sums >= 1, "all-reduces %lld", static_cast<long long>(sums));
  }
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
  return failures ? 1 : 0;
}
