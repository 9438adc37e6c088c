// The reference's stage checks (check/isvd/**.cpp), written against the C++
// stage API of include/mcnla_b200/isvd.hpp on the B200.  The fixtures arrive
// as raw little-endian float64 files (written by tests/test_gpu_cpp_api.py
// from tests/golden/mcnla_data.npz): qs (m x N l, unfolded), ys, qb_kn, qb_wy,
// a (m x n), q (m x l), u (m x l).
#include <mcnla_b200/isvd.hpp>

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

// max |Q1 Q1' - Q2 Q2'| for row-major m x k matrices
double projector_gap(const std::vector<double>& q1, const std::vector<double>& q2, int m, int k1, int ld1, int k2,
                     int ld2) {
  double mx = 0;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j <= i; ++j) {
      double a = 0, b = 0;
      for (int c = 0; c < k1; ++c) a += q1[i * ld1 + c] * q1[j * ld1 + c];
      for (int c = 0; c < k2; ++c) b += q2[i * ld2 + c] * q2[j * ld2 + c];
      mx = std::fmax(mx, std::fabs(a - b));
    }
  return mx;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  const int m = 101, l = 11, N = 12, n = 1001;
  using namespace mcnla_b200;
  Context ctx(0);

  // ---- KolmogorovNagumoIntegratorTest (check/isvd/integrator/kolmogorov_nagumo_integrator.cpp)
  {
    auto qs = load(dir + "/qs.bin", size_t(m) * l * N);
    auto qb_true = load(dir + "/qb_kn.bin", size_t(m) * l);
    Parameters parameters(ctx);
    parameters.setSize(m, l).setRank(l).setOverRank(0).setNumSketchEach(N).sync();
    KolmogorovNagumoIntegrator integrator(parameters, 256, 1e-4);
    integrator.initialize();
    auto qi = parameters.createCollectionQ();
    auto qbar = parameters.createMatrixQbar();
    qi.upload(qs);
    integrator(qi, qbar);
    EXPECT(integrator.iteration() == 81, "KN iteration %d", integrator.iteration());
    auto h = qbar.host();
    double mx = 0;
    for (size_t i = 0; i < h.size(); ++i) mx = std::fmax(mx, std::fabs(h[i] - qb_true[i]));
    EXPECT(mx < 1e-8, "KN qbar error %g", mx);
    EXPECT(integrator.times().size() == 2, "KN parts %zu", integrator.times().size());
  }
  // ---- RowBlockWenYinIntegratorTest (check/isvd/integrator/row_block_wen_yin_integrator.cpp)
  {
    auto qs = load(dir + "/qs.bin", size_t(m) * l * N);
    auto qb_true = load(dir + "/qb_wy.bin", size_t(m) * l);
    Parameters parameters(ctx);
    parameters.setSize(m, l).setRank(l).setOverRank(0).setNumSketch(N).sync();
    RowBlockGramianWenYinIntegrator integrator(parameters, 256, 1e-3);
    integrator.initialize();
    auto qi = parameters.createCollectionQj();
    auto qbar = parameters.createMatrixQbarj();
    qi.upload(qs);
    integrator(qi, qbar);
    EXPECT(integrator.iteration() == 21, "WY iteration %d", integrator.iteration());
    auto h = qbar.host();
    double mx = 0;
    for (size_t i = 0; i < h.size(); ++i) mx = std::fmax(mx, std::fabs(h[i] - qb_true[i]));
    EXPECT(mx < 1e-8, "WY qbar error %g", mx);
  }
  // ---- GramianOrthogonalizerTest (check/isvd/orthogonalizer/gramian_orthogonalizer.cpp)
  {
    auto ys = load(dir + "/ys.bin", size_t(m) * l * N);
    auto qs = load(dir + "/qs.bin", size_t(m) * l * N);
    Parameters parameters(ctx);
    parameters.setSize(m, l).setRank(l).setOverRank(0).setNumSketch(N).sync();
    GramianOrthogonalizer orthogonalizer(parameters);
    orthogonalizer.initialize();
    auto qi = parameters.createCollectionQ();
    qi.upload(ys);
    orthogonalizer(qi);
    auto h = qi.host();
    double mx = 0;
    for (int i = 0; i < N; ++i) {
      std::vector<double> a(h.begin(), h.end()), b(qs.begin(), qs.end());
      // compare sketch i (columns [i l, (i+1) l) of the unfolded collections)
      std::vector<double> ai(size_t(m) * l), bi(size_t(m) * l);
      for (int r = 0; r < m; ++r)
        for (int c = 0; c < l; ++c) {
          ai[r * l + c] = a[size_t(r) * l * N + i * l + c];
          bi[r * l + c] = b[size_t(r) * l * N + i * l + c];
        }
      mx = std::fmax(mx, projector_gap(ai, bi, m, l, l, l, l));
    }
    EXPECT(mx < 1e-8, "orthogonalizer projector gap %g", mx);
  }
  // ---- SvdFormerTest (check/isvd/former/svd_former.cpp): k = ncol(q) / 2
  {
    auto a = load(dir + "/a.bin", size_t(m) * n);
    auto q = load(dir + "/q.bin", size_t(m) * l);
    auto u_true = load(dir + "/u.bin", size_t(m) * l);
    const int k = l / 2, p = l - k;
    Parameters parameters(ctx);
    parameters.setSize(m, n).setRank(k).setOverRank(p).setNumSketchEach(1).sync();
    SvdFormer former(parameters);
    former.initialize();
    DeviceBuffer ad(m, n), qd(m, l);
    ad.upload(a);
    qd.upload(q);
    former(ad.view(), qd);
    auto u = former.matrixU().host();
    const double gap = projector_gap(u, u_true, m, k, k, k, l);
    EXPECT(gap < 1e-8, "SVD former U U' gap %g", gap);
    EXPECT(former.times().size() == 3, "former parts %zu", former.times().size());
  }
  // ---- error path: a status becomes an exception
  {
    Parameters parameters(ctx);
    parameters.setSize(10, 10).setRank(150).setOverRank(50).setNumSketch(1);
    bool thrown = false;
    try { parameters.sync(); } catch (const Error& e) { thrown = e.status() == MCNLA_B200_ERR_UNSUPPORTED; }
    EXPECT(thrown, "l > 160 must be rejected");
  }
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
  return failures ? 1 : 0;
}
